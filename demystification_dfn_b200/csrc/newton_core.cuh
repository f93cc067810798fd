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
#include <stdint.h>

#define MLP_IN 6
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

// MLP inputs from the physical state.
__device__ __forceinline__ void mlp_features(double tau, double psi, double s, double P, double a, double b,
                                             double w0, float x[MLP_IN])
{
    x[0] = (float)(w0 * 0.01);
    x[1] = (float)(psi / 30.0);
    x[2] = (float)(log(s) / 20.0 - 0.85);
    x[3] = (float)(P / s);
    x[4] = (float)(100.0 * a - 1.0);
    x[5] = (float)(100.0 * b - 1.0);
}

// Forward pass, FP32; W may live in shared memory.
__device__ __forceinline__ float mlp_forward(const float *W, const float x[MLP_IN])
{
    float h1[MLP_H];
#pragma unroll
    for (int j = 0; j < MLP_H; j++) {
        float z = W[MLP_B1 + j];
#pragma unroll
        for (int i = 0; i < MLP_IN; i++) z = fmaf(x[i], W[MLP_W1 + i * MLP_H + j], z);
        h1[j] = silu_f(z);
    }
    float out = W[MLP_B3];
    for (int j = 0; j < MLP_H; j++) {
        float z = W[MLP_B2 + j];
#pragma unroll
        for (int i = 0; i < MLP_H; i++) z = fmaf(h1[i], W[MLP_W2 + i * MLP_H + j], z);
        out = fmaf(silu_f(z), W[MLP_W3 + j], out);
    }
    return out;
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

