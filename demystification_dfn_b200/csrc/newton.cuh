// newton.cuh — training kernels of the MLP initial guess (FP32, hand-written
// forward and backward passes); the solve itself is in newton_core.cuh.
#pragma once
#include "newton_core.cuh"

// ---------------------------------------------------------------------------
// Training kernels (FP32). One CTA of 256 threads takes MLP_SB samples and
// writes its partial gradient of the summed squared error (scaled by
// 1/n_total) and its partial loss; a second kernel adds the partials in a
// fixed order and applies Adam.
#define MLP_SB 32

struct MlpSmem {
    float W[MLP_NPAR];
    float X[MLP_SB][MLP_IN];
    float Z1[MLP_SB][MLP_H], H1[MLP_SB][MLP_H];
    float Z2[MLP_SB][MLP_H], H2[MLP_SB][MLP_H];
    float D1[MLP_SB][MLP_H], D2[MLP_SB][MLP_H];
    float dout[MLP_SB];
    float lsum[MLP_SB];
};

__global__ void __launch_bounds__(256) mlp_grad_kernel(const float *__restrict__ X, const float *__restrict__ T,
                                                       int64_t n, int64_t n_total, const float *__restrict__ W,
                                                       float *__restrict__ gpart, float *__restrict__ lpart)
{
    extern __shared__ __align__(16) unsigned char mlp_smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(mlp_smem_raw);
    const int tid = threadIdx.x;
    const int64_t s0 = (int64_t)blockIdx.x * MLP_SB;
    for (int p = tid; p < MLP_NPAR; p += blockDim.x) S.W[p] = W[p];
    for (int q = tid; q < MLP_SB * MLP_IN; q += blockDim.x) {
        const int s = q / MLP_IN, i = q % MLP_IN;
        S.X[s][i] = (s0 + s < n) ? X[(s0 + s) * MLP_IN + i] : 0.0f;
    }
    __syncthreads();
    // layer 1
    for (int q = tid; q < MLP_SB * MLP_H; q += blockDim.x) {
        const int s = q / MLP_H, j = q % MLP_H;
        float z = S.W[MLP_B1 + j];
        for (int i = 0; i < MLP_IN; i++) z = fmaf(S.X[s][i], S.W[MLP_W1 + i * MLP_H + j], z);
        S.Z1[s][j] = z;
        S.H1[s][j] = silu_f(z);
    }
    __syncthreads();
    // layer 2
    for (int q = tid; q < MLP_SB * MLP_H; q += blockDim.x) {
        const int s = q / MLP_H, j = q % MLP_H;
        float z = S.W[MLP_B2 + j];
        for (int i = 0; i < MLP_H; i++) z = fmaf(S.H1[s][i], S.W[MLP_W2 + i * MLP_H + j], z);
        S.Z2[s][j] = z;
        S.H2[s][j] = silu_f(z);
    }
    __syncthreads();
    // output, loss and its derivative (mean over n_total samples)
    if (tid < MLP_SB) {
        const int s = tid;
        float o = S.W[MLP_B3];
        for (int j = 0; j < MLP_H; j++) o = fmaf(S.H2[s][j], S.W[MLP_W3 + j], o);
        const bool valid = s0 + s < n;
        const float d = valid ? o - T[s0 + s] : 0.0f;
        S.lsum[s] = d * d;
        S.dout[s] = 2.0f * d / (float)n_total;
    }
    __syncthreads();
    for (int q = tid; q < MLP_SB * MLP_H; q += blockDim.x) {
        const int s = q / MLP_H, j = q % MLP_H;
        S.D2[s][j] = S.dout[s] * S.W[MLP_W3 + j] * dsilu_f(S.Z2[s][j]);
    }
    __syncthreads();
    for (int q = tid; q < MLP_SB * MLP_H; q += blockDim.x) {
        const int s = q / MLP_H, i = q % MLP_H;
        float g = 0.0f;
        for (int j = 0; j < MLP_H; j++) g = fmaf(S.D2[s][j], S.W[MLP_W2 + i * MLP_H + j], g);
        S.D1[s][i] = g * dsilu_f(S.Z1[s][i]);
    }
    __syncthreads();
    float *gp = gpart + (int64_t)blockIdx.x * MLP_NPAR;
    for (int p = tid; p < MLP_NPAR; p += blockDim.x) {
        float g = 0.0f;
        if (p < MLP_B1) {                        // W1[i][j]
            const int i = p / MLP_H, j = p % MLP_H;
            for (int s = 0; s < MLP_SB; s++) g = fmaf(S.X[s][i], S.D1[s][j], g);
        } else if (p < MLP_W2) {                 // b1[j]
            const int j = p - MLP_B1;
            for (int s = 0; s < MLP_SB; s++) g += S.D1[s][j];
        } else if (p < MLP_B2) {                 // W2[i][j]
            const int q = p - MLP_W2, i = q / MLP_H, j = q % MLP_H;
            for (int s = 0; s < MLP_SB; s++) g = fmaf(S.H1[s][i], S.D2[s][j], g);
        } else if (p < MLP_W3) {                 // b2[j]
            const int j = p - MLP_B2;
            for (int s = 0; s < MLP_SB; s++) g += S.D2[s][j];
        } else if (p < MLP_B3) {                 // W3[j]
            const int j = p - MLP_W3;
            for (int s = 0; s < MLP_SB; s++) g = fmaf(S.H2[s][j], S.dout[s], g);
        } else {                                 // b3
            for (int s = 0; s < MLP_SB; s++) g += S.dout[s];
        }
        gp[p] = g;
    }
    if (tid == 0) {
        float l = 0.0f;
        for (int s = 0; s < MLP_SB; s++) l += S.lsum[s];
        lpart[blockIdx.x] = l;
    }
}

// Sum of the block partials (fixed order); with lr > 0 also one Adam step.
// The FP16 tensor-core image of the FP32 weights (one block).
__global__ void mlp_image_kernel(const float *__restrict__ W, MlpTC *img) { mlp_tc_stage(*img, W); }

// Inference of n rows by the friction kernel's tensor-core path; every lane
// of every warp takes part (rows past n are zero inputs, not stored).
__global__ void __launch_bounds__(256) mlp_infer_kernel(const float *__restrict__ X, int64_t n,
                                                        const float *__restrict__ W, float *__restrict__ Y)
{
    extern __shared__ __align__(16) unsigned char infer_smem[];
    MlpTC &S = *reinterpret_cast<MlpTC *>(infer_smem);
    mlp_tc_stage(S, W);
    __syncthreads();
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    float x[MLP_IN];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) x[i] = (r < n) ? X[r * MLP_IN + i] : 0.0f;
    const float y = mlp_warp_tc(S, x);
    if (r < n) Y[r] = y;
}

__global__ void mlp_reduce_adam_kernel(const float *__restrict__ gpart, int nblk, float *W, float *m, float *v,
                                       float *gout, int step, float lr)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_NPAR) return;
    float g = 0.0f;
    for (int b = 0; b < nblk; b++) g += gpart[(int64_t)b * MLP_NPAR + p];
    if (gout) gout[p] = g;
    if (lr > 0.0f) {
        const float b1 = 0.9f, b2 = 0.999f, epsa = 1e-8f;
        const float mm = b1 * m[p] + (1.0f - b1) * g;
        const float vv = b2 * v[p] + (1.0f - b2) * g * g;
        m[p] = mm;
        v[p] = vv;
        const float mh = mm / (1.0f - powf(b1, (float)step)), vh = vv / (1.0f - powf(b2, (float)step));
        W[p] -= lr * mh / (sqrtf(vh) + epsa);
    }
}

__global__ void sum_kernel(const float *x, int n, float *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float s = 0.0f;
    for (int i = 0; i < n; i++) s += x[i];
    *out = s;
}
