// newton_core.cuh — Newton solve of the friction law for the slip rate, and the
// small MLP that proposes its initial guess (no counterpart in the
// reference, whose ODE integrates V itself).
//
// Friction law with radiation damping, per element (sigma_eff = -(sigma+P)):
//   g(w) = tau - eta*V(w) - sigma_eff*a*w = 0,   V(w) = (2 V0/C) sinh(w),
//   C = exp((f0 + b psi)/a),  eta = mu/(2 cs).
// g is strictly decreasing in w for sigma_eff > 0, so Newton on w converges
// from any start once its steps are limited; the residual test is in FP64.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#define MLP_IN 7
#define MLP_H 64
#define MLP_NPAR (MLP_IN * MLP_H + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1)
// offsets in the flat weight array
#define MLP_W1 0
#define MLP_B1 (MLP_IN * MLP_H)
#define MLP_W2 (MLP_B1 + MLP_H)
#define MLP_B2 (MLP_W2 + MLP_H * MLP_H)
#define MLP_W3 (MLP_B2 + MLP_H)
#define MLP_B3 (MLP_W3 + MLP_H)

__host__ __device__ inline float silu_f(float z) { return z / (1.0f + expf(-z)); }
__host__ __device__ inline float dsilu_f(float z)
{
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// MLP inputs from the physical state: the analytic start wa (normalised
// shear stress bounded by radiation damping), log-state, effective normal
// stress, pore pressure, a, b, and the gap between the friction-only root
// w0 and the radiation-only root wr (how far radiation damping reaches).
__device__ __forceinline__ void mlp_features(double wa, double w0, double wr, double psi, double s, double P,
                                             double a, double b, float x[MLP_IN])
{
    x[0] = (float)(wa * 0.01);
    x[1] = (float)(psi / 30.0);
    x[2] = (float)(log(s) / 20.0 - 0.85);
    x[3] = (float)(P / (s + fabs(P)));
    x[4] = (float)(100.0 * a - 1.0);
    x[5] = (float)(100.0 * b - 1.0);
    x[6] = (float)(fmin(fmax(fabs(wr) - fabs(w0), -30.0), 30.0) / 10.0);
}

// Radiation-only root: eta V(wr) = tau, i.e. wr = asinh(tau / (eta A)) with
// ln A = lnA, evaluated without overflow (asinh(z) = ln 2z for large z).
__device__ __forceinline__ double w_radiation(double tau, double eta, double lnA)
{
    const double at = fabs(tau);
    if (at == 0.0) return 0.0;
    const double lz = log(at / eta) - lnA;
    const double wr = (lz > 20.0) ? lz + 0.6931471805599453 : asinh(exp(lz));
    return copysign(wr, tau);
}

// Inference only: the learned guess is judged by the FP64 residual, so the
// fast exponential and division (a few ulp) are enough.
__device__ __forceinline__ float silu_fast(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// ---------------------------------------------------------------------------
// Inference of the network by one warp on tensor cores. The 32 lanes' input
// rows form a 32 x 7 matrix (padded to 32 x 16); both layers are FP16 MMAs
// (m16n8k16) with FP32 accumulation: layer 1 is X[32x16] W1[16x64], layer 2
// H1[32x64] W2[64x64]. The m16n8 accumulator tiles of layer 1 are, after
// SiLU and packing to FP16, exactly the m16k16 A fragments of layer 2, so
// the hidden layer never leaves registers; the output layer is a dot
// product folded over the layer-2 tiles and summed over the 4 lanes that
// share a row. The learned guess is only a starting point that the FP64
// residual judges, so FP16 operands suffice.
struct __align__(16) MlpTC {
    __half w1t[MLP_H][8];            // W1 transposed, inputs padded to 8
    __half w2t[MLP_H][MLP_H + 8];    // W2 transposed; +8 spreads the rows over the banks
    float b1[MLP_H], b2[MLP_H], w3[MLP_H], b3;
};
static_assert(sizeof(MlpTC) % 16 == 0, "the image is copied in 16-byte units");
static const size_t kMlpImgBytes = sizeof(MlpTC);

// The image of the flat FP32 weights (whole block; S in shared or global memory).
__device__ __forceinline__ void mlp_tc_stage(MlpTC &S, const float *W)
{
    for (int p = threadIdx.x; p < MLP_H * 8; p += blockDim.x) {
        const int n = p % MLP_H, k = p / MLP_H;
        S.w1t[n][k] = __float2half_rn(k < MLP_IN ? W[MLP_W1 + k * MLP_H + n] : 0.0f);
    }
    for (int p = threadIdx.x; p < MLP_H * MLP_H; p += blockDim.x) {
        const int n = p % MLP_H, k = p / MLP_H;
        S.w2t[n][k] = __float2half_rn(W[MLP_W2 + p]);
    }
    for (int p = threadIdx.x; p < MLP_H; p += blockDim.x) {
        S.b1[p] = W[MLP_B1 + p];
        S.b2[p] = W[MLP_B2 + p];
        S.w3[p] = W[MLP_W3 + p];
    }
    if (threadIdx.x == 0) S.b3 = W[MLP_B3];
}

__device__ __forceinline__ void mma_16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_h2(float lo, float hi)
{
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// All 32 lanes call it (converged); returns the output for this lane's row.
__device__ __forceinline__ float mlp_warp_tc_body(const MlpTC &S, const float x[MLP_IN])
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // this lane's inputs as 4 packed pairs (input 7 is the zero pad)
    uint32_t xp[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float lo = x[2 * j], hi = (2 * j + 1 < MLP_IN) ? x[2 * j + 1] : 0.0f;
        xp[j] = pack_h2(lo, hi);
    }
    // layer-1 A fragments: rows 16 mt + g (+ 8), columns 2t, 2t+1
    uint32_t a1[2][2];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
            const int row = 16 * mt + g + 8 * hf;
            uint32_t v = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t s = __shfl_sync(full, xp[j], row);
                if (j == t) v = s;
            }
            a1[mt][hf] = v;
        }
    }
    // layer 1 -> SiLU -> layer-2 A fragments a2[mt][kt][4]
    uint32_t a2[2][4][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int col = 8 * nt + 2 * t;
        const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&S.w1t[8 * nt + g][2 * t]);
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            float c[4] = {S.b1[col], S.b1[col + 1], S.b1[col], S.b1[col + 1]};
            const uint32_t a[4] = {a1[mt][0], a1[mt][1], 0u, 0u};
            mma_16816(c, a, b0, 0u);
            const int kt = nt >> 1, q = (nt & 1) * 2;
            a2[mt][kt][q] = pack_h2(silu_fast(c[0]), silu_fast(c[1]));
            a2[mt][kt][q + 1] = pack_h2(silu_fast(c[2]), silu_fast(c[3]));
        }
    }
    // layer 2 tile by tile, folded into the output dot product
    float o[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int col = 8 * nt + 2 * t;
        float c[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            c[mt][0] = S.b2[col]; c[mt][1] = S.b2[col + 1];
            c[mt][2] = S.b2[col]; c[mt][3] = S.b2[col + 1];
        }
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&S.w2t[8 * nt + g][16 * kt + 2 * t]);
            const uint32_t b1 = *reinterpret_cast<const uint32_t *>(&S.w2t[8 * nt + g][16 * kt + 8 + 2 * t]);
            mma_16816(c[0], a2[0][kt], b0, b1);
            mma_16816(c[1], a2[1][kt], b0, b1);
        }
        const float w0 = S.w3[col], w1 = S.w3[col + 1];
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            o[mt][0] = fmaf(silu_fast(c[mt][0]), w0, fmaf(silu_fast(c[mt][1]), w1, o[mt][0]));
            o[mt][1] = fmaf(silu_fast(c[mt][2]), w0, fmaf(silu_fast(c[mt][3]), w1, o[mt][1]));
        }
    }
    // sum over the 4 lanes of a row, then row r goes to lane r
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
            o[mt][hf] += __shfl_xor_sync(full, o[mt][hf], 1);
            o[mt][hf] += __shfl_xor_sync(full, o[mt][hf], 2);
        }
    }
    const int src = 4 * (lane & 7), mt = lane >> 4, hf = (lane >> 3) & 1;
    float r = 0.0f;
#pragma unroll
    for (int m = 0; m < 2; m++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const float v = __shfl_sync(full, o[m][h], src);
            if (m == mt && h == hf) r = v;
        }
    }
    return r + S.b3;
}

__device__ __forceinline__ float mlp_warp_tc(const MlpTC &S, const float x[MLP_IN])
{
    return mlp_warp_tc_body(S, x);
}

// The same inference as a called function, for the stage kernel: its
// registers are then allocated apart from the element path's (which every
// element takes, while the inference runs in a few warps).
__device__ __noinline__ float mlp_warp_tc_call(const MlpTC *S, float x0, float x1, float x2, float x3, float x4,
                                               float x5, float x6)
{
    const float x[MLP_IN] = {x0, x1, x2, x3, x4, x5, x6};
    return mlp_warp_tc_body(*S, x);
}

// eta*V(w) and eta*dV/dw without overflow: V = (2V0/C) sinh(w) with
// ln(2V0/C) = lnA.
__device__ __forceinline__ void eta_v(double w, double lnA, double eta, double &ev, double &edv)
{
    const double aw = fabs(w);
    const double e = exp(lnA + aw - 0.6931471805599453);   // A e^|w| / 2
    const double q = exp(-2.0 * aw);
    ev = eta * copysign(e * (1.0 - q), w);
    edv = eta * e * (1.0 + q);
}

// Newton on w from `w`; returns the root, sets iterations and convergence.
__device__ __forceinline__ double newton_w(double tau, double s, double a, double lnA, double eta, double w,
                                           double tol, int maxit, int &iters, int &ok)
{
    iters = 0;
    ok = 0;
    for (int it = 0; it <= maxit; it++) {
        double ev, edv;
        eta_v(w, lnA, eta, ev, edv);
        const double g = tau - ev - s * a * w;
        if (fabs(g) <= tol * (fabs(tau) + s * a * fabs(w) + 1e-300)) { ok = 1; break; }
        if (it == maxit) break;
        double dw = g / (edv + s * a);   // -g/g', g' = -(edv + s a) < 0
        dw = fmax(fmin(dw, 10.0), -10.0);
        w += dw;
        iters++;
    }
    return w;
}

// V(w) = (2 V0/C) sinh(w)
__device__ __forceinline__ double v_of_w(double w, double lnA)
{
    const double aw = fabs(w);
    return copysign(exp(lnA + aw - 0.6931471805599453) * (1.0 - exp(-2.0 * aw)), w);
}

