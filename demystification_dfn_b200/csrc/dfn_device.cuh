// dfn_device.cuh — device code of the B200 earthquake-cycle hot path.
//
// Kernels (all FP64 arithmetic unless the stored kernel matrix is FP32/BF16):
//   geometry_kernel       element midpoints, ds, tangent, normal, loading
//                         projection, permeability_x
//                         (src/initialisation.f90:145-205,252-269)
//   assemble_kernel       dense kernel entries K_T/K_N (unscaled), formulas of
//                         src/hmatrix/eval_kernel_hmatrix.f90:7-199 (same pair
//                         terms as src/kernel_calculation/directModeII.f90:41-78)
//   gemv_kernel           K.V streamed from HBM, per-column-chunk partial sums
//                         (one launch covers every network of a batch)
//   pressure_cg_kernel    the reference's Jacobi-scaled CG for compute_P
//                         (src/fluid_diffusion.f90:24-152), one CTA per system
//   pressure_tridiag_kernel  exact per-segment Thomas solve of the same system
//   friction_kernel       closed-form dV/dt, dpsi/dt, dsigma/dt
//                         (src/friction/RateStateAgingModeII.f90:46-89) fused
//                         with the Cash-Karp stage combination, the 5th-order
//                         solution, the embedded error and its max-norm
//   step kernels          rkqs step control and solve() bookkeeping in FP64
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cooperative_groups.h>
#include <stdint.h>

#include "newton_core.cuh"

#define DFN_PI 3.141592653589793238

// ---------------------------------------------------------------------------
// Device-resident step controller (one per network).
struct StepCtl {
    double time;      // committed simulated time
    double t_try;     // trial step of the solve loop
    double x;         // rkqs x (offset of the step start; 0 in solve())
    double h;         // step of the current attempt
    double hnext, hdid;
    double eps;       // tol_solver
    unsigned long long errmax_bits;  // max |yerr/yscal| as ordered bits
    long long it_count, attempts, rejected, rhs_evals, cg_iters, halvings;
    int accepted;
    int status;       // dfn_status
    int probe_ier;
    int phase;        // PH_NEW / PH_RETRY / PH_DONE
    long long steps_done, target_steps;  // accepted steps in this solve call, and the goal
    double t_end;     // stop when time >= t_end (t_end > 0)
    int step_attempts, max_attempts;
    int pfail_mask;   // bit s: pressure system s of this attempt hit the CG cap
    int commit_bad;   // committed state of this step: bit 0 sigmaN > 0, bit 1 non-finite
    long long stage_noconv;  // stage pressure solves that hit the CG cap
    long long newton_solves, newton_iters, newton_fail;  // Newton formulation counters
    long long mlp_warps;     // warps that evaluated the learned guess
};

// Cash-Karp tableau, src/ode_solver/ode_bs.f90:200-210.
#define CK_A2 0.2
#define CK_A3 0.3
#define CK_A4 0.6
#define CK_A5 1.0
#define CK_A6 0.875
#define CK_B21 0.2
#define CK_B31 (3.0 / 40.0)
#define CK_B32 (9.0 / 40.0)
#define CK_B41 0.3
#define CK_B42 (-0.9)
#define CK_B43 1.2
#define CK_B51 (-11.0 / 54.0)
#define CK_B52 2.5
#define CK_B53 (-70.0 / 27.0)
#define CK_B54 (35.0 / 27.0)
#define CK_B61 (1631.0 / 55296.0)
#define CK_B62 (175.0 / 512.0)
#define CK_B63 (575.0 / 13824.0)
#define CK_B64 (44275.0 / 110592.0)
#define CK_B65 (253.0 / 4096.0)
#define CK_C1 (37.0 / 378.0)
#define CK_C3 (250.0 / 621.0)
#define CK_C4 (125.0 / 594.0)
#define CK_C6 (512.0 / 1771.0)
#define CK_DC1 (CK_C1 - 2825.0 / 27648.0)
#define CK_DC3 (CK_C3 - 18575.0 / 48384.0)
#define CK_DC4 (CK_C4 - 13525.0 / 55296.0)
#define CK_DC5 (-277.0 / 14336.0)
#define CK_DC6 (CK_C6 - 0.25)

// Non-contracted FP64 helpers: the stage combinations are written with
// explicit round-to-nearest mul/add so that they match the reference's
// expression order exactly (no FMA formation).
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }

// Stage abscissae: offset of stage s (1-based, s=2..6) from the step start.
__device__ __forceinline__ double ck_a(int s)
{
    switch (s) {
    case 2: return CK_A2;
    case 3: return CK_A3;
    case 4: return CK_A4;
    case 5: return CK_A5;
    default: return CK_A6;
    }
}

// ytemp of stage s (2..6) for one component, src/ode_solver/ode_bs.f90:213-221.
__device__ __forceinline__ double ck_combine(int s, double h, double y, const double *k, int64_t stride, int64_t i)
{
    const double k1 = k[i];
    switch (s) {
    case 2: return add_(y, mul_(mul_(CK_B21, h), k1));
    case 3: {
        const double k2 = k[stride + i];
        return add_(y, mul_(h, add_(mul_(CK_B31, k1), mul_(CK_B32, k2))));
    }
    case 4: {
        const double k2 = k[stride + i], k3 = k[2 * stride + i];
        return add_(y, mul_(h, add_(add_(mul_(CK_B41, k1), mul_(CK_B42, k2)), mul_(CK_B43, k3))));
    }
    case 5: {
        const double k2 = k[stride + i], k3 = k[2 * stride + i], k4 = k[3 * stride + i];
        return add_(y, mul_(h, add_(add_(add_(mul_(CK_B51, k1), mul_(CK_B52, k2)), mul_(CK_B53, k3)),
                                    mul_(CK_B54, k4))));
    }
    default: {
        const double k2 = k[stride + i], k3 = k[2 * stride + i], k4 = k[3 * stride + i], k5 = k[4 * stride + i];
        return add_(y, mul_(h, add_(add_(add_(add_(mul_(CK_B61, k1), mul_(CK_B62, k2)), mul_(CK_B63, k3)),
                                         mul_(CK_B64, k4)),
                                    mul_(CK_B65, k5))));
    }
    }
}

// ---------------------------------------------------------------------------
// Geometry: src/initialisation.f90:145-153 (element, ds, tangent, normal),
// :159-205 (loading projection), :252-269 (harmonic face permeability).
__global__ void geometry_kernel(int64_t N, int mode, const double *__restrict__ node, double *elem, double *ds,
                                double *tan, double *nrm, double *nload, double *sload, double *sig, const double *perm,
                                double *permx, double S11d, double S12d, double S22d, double S31d, double S32d)
{
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < N) {
        double x0 = node[2 * k], y0 = node[2 * k + 1], x1 = node[2 * k + 2], y1 = node[2 * k + 3];
        double dx = __dadd_rn(x1, -x0), dy = __dadd_rn(y1, -y0);
        elem[2 * k] = __dmul_rn(__dadd_rn(x1, x0), 0.5);
        elem[2 * k + 1] = __dmul_rn(__dadd_rn(y1, y0), 0.5);
        double d = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
        ds[k] = d;
        double t1 = __ddiv_rn(dx, d), t2 = __ddiv_rn(dy, d);
        tan[2 * k] = t1; tan[2 * k + 1] = t2;
        double n1 = -t2, n2 = t1;
        nrm[2 * k] = n1; nrm[2 * k + 1] = n2;
        if (mode == 3) {
            sload[k] = add_(add_(sload[k], -mul_(t2, S31d)), mul_(t1, S32d));
            sig[k] = add_(add_(sig[k], mul_(n1, add_(mul_(n1, S11d), mul_(n2, S12d)))),
                          mul_(n2, add_(mul_(n1, S12d), mul_(n2, S22d))));
        } else {
            nload[k] = add_(add_(nload[k], mul_(n1, add_(mul_(n1, S11d), mul_(n2, S12d)))),
                            mul_(n2, add_(mul_(n1, S12d), mul_(n2, S22d))));
            sload[k] = add_(add_(sload[k], mul_(t1, add_(mul_(n1, S11d), mul_(n2, S12d)))),
                            mul_(t2, add_(mul_(n1, S12d), mul_(n2, S22d))));
        }
    }
    if (k <= N) {
        double px = 0.0;
        if (k >= 1 && k < N) px = __ddiv_rn(mul_(mul_(2.0, perm[k - 1]), perm[k]), add_(perm[k - 1], perm[k]));
        permx[k] = px;
    }
}

// ---------------------------------------------------------------------------
// Kernel-matrix storage formats. Row k (receiver) is contiguous over source
// columns l; in mode II the shear and normal entries of one column are
// adjacent, so one pass streams both matrices and reads V once.
//   FP64   : mode II {T,N} double2 per column; mode III double per column
//   FP32   : mode II {T,N} float2;            mode III float
//   BF16X2 : entry = hi + lo, both bf16;      mode II {Th,Tl,Nh,Nl}; mode III {h,l}
template <int MODE, int STORE> struct KFmt;
template <> struct KFmt<2, 0> { static constexpr int BPC = 16; };
template <> struct KFmt<2, 1> { static constexpr int BPC = 8; };
template <> struct KFmt<2, 2> { static constexpr int BPC = 8; };
template <> struct KFmt<3, 0> { static constexpr int BPC = 8; };
template <> struct KFmt<3, 1> { static constexpr int BPC = 4; };
template <> struct KFmt<3, 2> { static constexpr int BPC = 4; };

// Entry formulas: src/hmatrix/eval_kernel_hmatrix.f90:36-47 (mode III),
// :91-115 (mode II shear), :160-195 (mode II normal).
__host__ __device__ inline double entry_mode3(double e1, double e2, double t1, double t2, double xl, double yl,
                                              double xr, double yr)
{
    double ax = xl - e1, ay = yl - e2, bx = xr - e1, by = yr - e2;
    double r1 = sqrt(ax * ax + ay * ay);
    double r2 = sqrt(bx * bx + by * by);
    double I1 = t1 / (r1 * r1) * (e1 - xl) + t2 / (r1 * r1) * (e2 - yl);
    double I2 = t1 / (r2 * r2) * (e1 - xr) + t2 / (r2 * r2) * (e2 - yr);
    return -I1 + I2;
}

__host__ __device__ inline void entry_mode2(double e1, double e2, double n1, double n2, double xl, double yl,
                                            double xr, double yr, double nl1, double nl2, double &T, double &Nn)
{
    double dxl = e1 - xl, dyl = e2 - yl, dxr = e1 - xr, dyr = e2 - yr;
    double rl = sqrt(dxl * dxl + dyl * dyl);
    double rr = sqrt(dxr * dxr + dyr * dyr);
    double g1l = dxl / rl, g2l = dyl / rl, g1r = dxr / rr, g2r = dyr / rr;
    double c4 = 4.0 * n1 * n2, c2 = n2 * n2 - n1 * n1, s2 = 2.0 * n1 * n2;
    double ql = (c4 * g1l * g2l + c2 * (g2l * g2l - g1l * g1l));
    double qr = (c4 * g1r * g2r + c2 * (g2r * g2r - g1r * g1r));
    double I1tl = ql * g1l / rl, I2tl = ql * g2l / rl, I1tr = qr * g1r / rr, I2tr = qr * g2r / rr;
    double wl = (s2 * (g2l * g2l - g1l * g1l) - c2 * 2.0 * g1l * g2l);
    double wr = (s2 * (g2r * g2r - g1r * g1r) - c2 * 2.0 * g1r * g2r);
    double I1nl = g1l / rl - g2l / rl * wl, I2nl = g2l / rl + g1l / rl * wl;
    double I1nr = g1r / rr - g2r / rr * wr, I2nr = g2r / rr + g1r / rr * wr;
    T = nl2 * I1tl - nl2 * I1tr - nl1 * I2tl + nl1 * I2tr;
    Nn = nl1 * I1nl - nl1 * I1nr + nl2 * I2nl - nl2 * I2nr;
}

__device__ __forceinline__ void split_bf16(double v, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __double2bfloat16(v);
    lo = __double2bfloat16(v - (double)__bfloat162float(hi));
}

// One thread per (row k, column l); Np padded columns (zeros beyond N).
template <int MODE, int STORE>
__global__ void assemble_kernel(int64_t N, int64_t Np, const double *__restrict__ node,
                                const double *__restrict__ elem, const double *__restrict__ tan,
                                const double *__restrict__ nrm, void *Kout)
{
    int64_t k = blockIdx.x;
    int64_t l = blockIdx.y * (int64_t)blockDim.x + threadIdx.x;
    if (l >= Np || k >= N) return;
    double T = 0.0, Nn = 0.0;
    if (l < N) {
        double e1 = elem[2 * k], e2 = elem[2 * k + 1];
        double xl = node[2 * l], yl = node[2 * l + 1], xr = node[2 * l + 2], yr = node[2 * l + 3];
        if (MODE == 3) T = entry_mode3(e1, e2, tan[2 * k], tan[2 * k + 1], xl, yl, xr, yr);
        else entry_mode2(e1, e2, nrm[2 * k], nrm[2 * k + 1], xl, yl, xr, yr, nrm[2 * l], nrm[2 * l + 1], T, Nn);
    }
    int64_t idx = k * Np + l;
    if (STORE == 0) {
        if (MODE == 2) reinterpret_cast<double2 *>(Kout)[idx] = make_double2(T, Nn);
        else reinterpret_cast<double *>(Kout)[idx] = T;
    } else if (STORE == 1) {
        if (MODE == 2) reinterpret_cast<float2 *>(Kout)[idx] = make_float2((float)T, (float)Nn);
        else reinterpret_cast<float *>(Kout)[idx] = (float)T;
    } else {
        __nv_bfloat16 th, tl, nh, nl;
        split_bf16(T, th, tl);
        if (MODE == 2) {
            split_bf16(Nn, nh, nl);
            __nv_bfloat16 *o = reinterpret_cast<__nv_bfloat16 *>(Kout) + 4 * idx;
            o[0] = th; o[1] = tl; o[2] = nh; o[3] = nl;
        } else {
            __nv_bfloat16 *o = reinterpret_cast<__nv_bfloat16 *>(Kout) + 2 * idx;
            o[0] = th; o[1] = tl;
        }
    }
}

// ---------------------------------------------------------------------------
// K.V streaming kernel.
//
// Work unit: a column chunk of CW columns (4 KiB of one row) for a block of
// rows. Every lane keeps the V values of its columns in registers and reuses
// them for all rows of the block; each warp owns rows r0+w, r0+w+8, ... and
// issues 8 coalesced 128-bit loads per lane per row (two rows in flight).
// The per-(chunk,row) warp sum goes to part[c*N + row]; the friction kernel
// adds the chunks in a fixed order, so the result is deterministic.
constexpr int GEMV_WARPS = 8;
constexpr int GEMV_LPL = 8;                       // 16-byte loads per lane per row-chunk
constexpr int GEMV_CHUNK_BYTES = 32 * GEMV_LPL * 16;  // 4096
constexpr int GEMV_ROWS = 64;                     // rows per CTA

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int MODE, int STORE>
__device__ __forceinline__ void fma_vec(const uint4 &q, const double *v, double &aT, double &aN)
{
    if (STORE == 0) {
        const double *d = reinterpret_cast<const double *>(&q);
        if (MODE == 2) { aT = fma(d[0], v[0], aT); aN = fma(d[1], v[0], aN); }
        else { aT = fma(d[0], v[0], aT); aT = fma(d[1], v[1], aT); }
    } else if (STORE == 1) {
        const float *f = reinterpret_cast<const float *>(&q);
        if (MODE == 2) {
            aT = fma((double)f[0], v[0], aT); aN = fma((double)f[1], v[0], aN);
            aT = fma((double)f[2], v[1], aT); aN = fma((double)f[3], v[1], aN);
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) aT = fma((double)f[j], v[j], aT);
        }
    } else {
        const __nv_bfloat162 *b = reinterpret_cast<const __nv_bfloat162 *>(&q);
        if (MODE == 2) {
#pragma unroll
            for (int j = 0; j < 2; j++) {
                float2 t = __bfloat1622float2(b[2 * j]);
                float2 n = __bfloat1622float2(b[2 * j + 1]);
                aT = fma((double)(t.x + t.y), v[j], aT);
                aN = fma((double)(n.x + n.y), v[j], aN);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float2 t = __bfloat1622float2(b[j]);
                aT = fma((double)(t.x + t.y), v[j], aT);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Batch of independent networks ("instances"). A single network is a batch
// of one. Per-instance data are concatenated; Inst gives the offsets.
enum { PH_NEW = 0, PH_RETRY = 1, PH_DONE = 2 };
enum { M_NEW = 1, M_RETRY = 2, M_ACTIVE = 3, M_ALL = 7 };

struct Inst {
    int64_t N;        // elements of the instance (fake ones included)
    int64_t Np;       // padded columns of its kernel matrix
    int64_t eoff;     // first element in the concatenated element arrays
    int64_t nchunk;   // 4 KiB column chunks per row
    int64_t kvec;     // offset of its kernel matrix in 16-byte vectors
    int64_t poff;     // offset of its K.V partial sums (nchunk*N per component)
    int64_t soff, nsrc;  // its injection sources
    double prefT, mu_2cs;
    double porosity, dyn_visc, comp, tol;
    double t0;        // time at which the slip is zero (Newton formulation)
};

__device__ __forceinline__ bool takes_part(const StepCtl *ctl, int i, int mask)
{
    return (mask >> ctl[i].phase) & 1;
}

// Pressure solves: kind 3 (the commit solve of the permeability coupling,
// dt = the step just accepted) only for networks whose attempt was accepted.
__device__ __forceinline__ bool press_takes_part(const StepCtl *ctl, int i, int mask, int kind)
{
    return takes_part(ctl, i, mask) && !(kind == 3 && (!ctl[i].accepted || ctl[i].status != 0));
}

// K.V streaming kernel (direct 128-bit loads).
//
// Work unit (tile): one 4 KiB column chunk of one instance for a block of
// GEMV_ROWS rows. Every lane keeps the V values of its columns in registers
// and reuses them for all rows of the block; each warp owns rows r0+w,
// r0+w+8, ... and issues 8 coalesced 128-bit loads per lane per row (two rows
// in flight). The per-(chunk,row) warp sum goes to part[c*N + row]; the
// consumer adds the chunks in a fixed order, so the result is deterministic.
// V of instance i is Vbase[vmul*eoff_i + l].
template <int MODE, int STORE>
__global__ void __launch_bounds__(GEMV_WARPS * 32)
    gemv_kernel(const int4 *__restrict__ tiles, const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                int mask, const uint4 *__restrict__ Kbase, const double *__restrict__ Vbase, int vmul,
                double *__restrict__ partT, double *__restrict__ partN)
{
    constexpr int BPC = KFmt<MODE, STORE>::BPC;
    constexpr int CPV = 16 / BPC;                 // columns per 16-byte vector
    constexpr int CW = GEMV_CHUNK_BYTES / BPC;    // columns per chunk
    const int4 t = tiles[blockIdx.x];
    if (!takes_part(ctl, t.x, mask)) return;
    const Inst I = inst[t.x];
    const int64_t N = I.N;
    const uint4 *K = Kbase + I.kvec;
    const double *Vin = Vbase + (int64_t)vmul * I.eoff;
    double *pT = partT + I.poff, *pN = partN + I.poff;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t c = t.y;
    const int64_t r0 = (int64_t)t.z * GEMV_ROWS;
    const int64_t row_vecs = I.Np * BPC / 16;

    double v[GEMV_LPL * CPV];
#pragma unroll
    for (int i = 0; i < GEMV_LPL; i++)
#pragma unroll
        for (int j = 0; j < CPV; j++) {
            int64_t col = c * CW + (int64_t)(i * 32 + lane) * CPV + j;
            v[i * CPV + j] = (col < N) ? Vin[col] : 0.0;
        }

    const int64_t vec0 = c * (CW * BPC / 16) + lane;
    for (int64_t r = r0 + warp; r < r0 + GEMV_ROWS && r < N; r += 2 * GEMV_WARPS) {
        const int64_t rb = r + GEMV_WARPS;
        const bool two = (rb < r0 + GEMV_ROWS) && (rb < N);
        const uint4 *pa = K + r * row_vecs + vec0;
        const uint4 *pb = K + (two ? rb : r) * row_vecs + vec0;
        uint4 qa[GEMV_LPL], qb[GEMV_LPL];
#pragma unroll
        for (int i = 0; i < GEMV_LPL; i++) qa[i] = __ldcs(pa + i * 32);
#pragma unroll
        for (int i = 0; i < GEMV_LPL; i++) qb[i] = two ? __ldcs(pb + i * 32) : make_uint4(0, 0, 0, 0);
        double aT = 0.0, aN = 0.0, bT = 0.0, bN = 0.0;
#pragma unroll
        for (int i = 0; i < GEMV_LPL; i++) fma_vec<MODE, STORE>(qa[i], v + i * CPV, aT, aN);
#pragma unroll
        for (int i = 0; i < GEMV_LPL; i++) fma_vec<MODE, STORE>(qb[i], v + i * CPV, bT, bN);
        aT = warp_sum(aT); bT = warp_sum(bT);
        if (MODE == 2) { aN = warp_sum(aN); bN = warp_sum(bN); }
        if (lane == 0) {
            pT[c * N + r] = aT;
            if (MODE == 2) pN[c * N + r] = aN;
            if (two) {
                pT[c * N + rb] = bT;
                if (MODE == 2) pN[c * N + rb] = bN;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// TMA bulk-copy variant: one producer warp streams 4 KiB row-chunks with
// cp.async.bulk into a ring of shared-memory stages completed on mbarriers;
// eight consumer warps read the stages with 128-bit shared loads. Rows of the
// CTA's block are assigned to consumer warps round-robin, one stage per row.
constexpr int TMA_STAGES = 16;
constexpr int TMA_CONSUMERS = 8;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait: returns false if the phase did not complete within `limit`
// polls (0: give up at once).
constexpr int MBAR_POLLS = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int limit = MBAR_POLLS)
{
    uint32_t ok = 0;
    for (int it = 0; it < limit; it++) {
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(smem_u32(bar)), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// TMA bulk-copy variant of the same tiling: one producer warp streams the
// 4 KiB row-chunks of the tile with cp.async.bulk into a 16-stage ring of
// shared memory completed on mbarriers; eight consumer warps read the stages
// with 128-bit shared loads. Rows of the tile go to consumer warps
// round-robin, one stage per row (stage s is always read by warp s % 8).
template <int MODE, int STORE>
__global__ void __launch_bounds__((TMA_CONSUMERS + 1) * 32)
    gemv_tma_kernel(const int4 *__restrict__ tiles, const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                    int mask, const uint4 *__restrict__ Kbase, const double *__restrict__ Vbase, int vmul,
                    double *__restrict__ partT, double *__restrict__ partN, int wait_polls, int *err_flag)
{
    constexpr int BPC = KFmt<MODE, STORE>::BPC;
    constexpr int CPV = 16 / BPC;
    constexpr int CW = GEMV_CHUNK_BYTES / BPC;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint4 *stage = reinterpret_cast<uint4 *>(smem_raw);                       // TMA_STAGES x 4 KiB
    uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw + TMA_STAGES * GEMV_CHUNK_BYTES);
    uint64_t *empty = full + TMA_STAGES;
    __shared__ int issued_s, bad_s;

    const int4 t = tiles[blockIdx.x];
    if (!takes_part(ctl, t.x, mask)) return;   // CTA-uniform: before any barrier
    const Inst I = inst[t.x];
    const int64_t N = I.N;
    const unsigned char *K = reinterpret_cast<const unsigned char *>(Kbase + I.kvec);
    const double *Vin = Vbase + (int64_t)vmul * I.eoff;
    double *pT = partT + I.poff, *pN = partN + I.poff;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t c = t.y;
    const int64_t r0 = (int64_t)t.z * GEMV_ROWS;
    const int64_t rend = (r0 + GEMV_ROWS < N) ? r0 + GEMV_ROWS : N;
    const int nrows = (int)(rend - r0);
    const int64_t row_bytes = I.Np * BPC;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TMA_STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        issued_s = 0;
        bad_s = 0;
    }
    __syncthreads();
    if (warp == TMA_CONSUMERS) {
        // producer: one elected lane issues the bulk copies
        if (lane == 0) {
            int i = 0;
            for (; i < nrows; i++) {
                int s = i % TMA_STAGES;
                if (i >= TMA_STAGES && !mbar_wait(&empty[s], ((i / TMA_STAGES) - 1) & 1, wait_polls)) {
                    bad_s = 1;
                    break;
                }
                mbar_expect_tx(&full[s], GEMV_CHUNK_BYTES);
                tma_bulk_g2s(stage + s * (GEMV_CHUNK_BYTES / 16), K + (r0 + i) * row_bytes + c * GEMV_CHUNK_BYTES,
                             GEMV_CHUNK_BYTES, &full[s]);
            }
            issued_s = i;
        }
    } else {
        double v[GEMV_LPL * CPV];
#pragma unroll
        for (int i = 0; i < GEMV_LPL; i++)
#pragma unroll
            for (int j = 0; j < CPV; j++) {
                int64_t col = c * CW + (int64_t)(i * 32 + lane) * CPV + j;
                v[i * CPV + j] = (col < N) ? Vin[col] : 0.0;
            }
        for (int i = warp; i < nrows; i += TMA_CONSUMERS) {
            int s = i % TMA_STAGES;
            if (!mbar_wait(&full[s], (i / TMA_STAGES) & 1, wait_polls)) { bad_s = 1; break; }
            const uint4 *sp = stage + s * (GEMV_CHUNK_BYTES / 16) + lane;
            uint4 q[GEMV_LPL];
#pragma unroll
            for (int j = 0; j < GEMV_LPL; j++) q[j] = sp[j * 32];
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
            double aT = 0.0, aN = 0.0;
#pragma unroll
            for (int j = 0; j < GEMV_LPL; j++) fma_vec<MODE, STORE>(q[j], v + j * CPV, aT, aN);
            aT = warp_sum(aT);
            if (MODE == 2) aN = warp_sum(aN);
            if (lane == 0) {
                pT[c * N + r0 + i] = aT;
                if (MODE == 2) pN[c * N + r0 + i] = aN;
            }
        }
    }
    __syncthreads();
    if (bad_s && threadIdx.x == 0) {
        // error path: wait (bounded, with the full limit whatever wait_polls
        // is) for the copies still in flight before the CTA's shared memory
        // is released, then report
        int issued = issued_s;
        for (int i = (issued > TMA_STAGES ? issued - TMA_STAGES : 0); i < issued; i++)
            mbar_wait(&full[i % TMA_STAGES], (i / TMA_STAGES) & 1);
        atomicExch(err_flag, 1);
    }
}

// ---------------------------------------------------------------------------
// Pore pressure (src/fluid_diffusion.f90). The parameters of the implicit
// step are shared by both solvers.
struct PressParams {
    int64_t N;
    const double *P;       // committed pressure
    const double *permx;   // [N+1] face permeability (0-based: face j between elements j-1 and j)
    const double *ds;
    double porosity, dyn_visc, comp;  // comp = fluid_comp + rock_comp
    double tol;
    int64_t nsrc;
    const int64_t *src_fault;   // 1-based fault id
    const int64_t *src_elem;    // 0-based global element index
    const double *src_Q, *src_tb, *src_te;
    const double *ctl_time;     // &ctl->time
    // fault crossings (null when the network has none): contributions of
    // row k are xcon[xptr[k] .. xptr[k+1]); xrows lists the nxrows rows
    // that have any
    const int64_t *xptr;
    const struct XCon *xcon;
    const int64_t *xrows;
    int64_t nxrows;
    // tridiagonal solver: per element the dt-free factors (u, v, w) of its
    // row, A1 = -dt u, A2 = 1 + dt v, A3 = -dt w (tridiagonal handles only)
    const double *tcoef;
};

// One fault-crossing contribution to a row of the pressure system: partner
// elements a and b (instance-local; the row itself where the partner is
// absent) and the harmonic means kl, kr of the permeabilities (0 where
// absent). Built on the host as find_fault_crossing
// (src/initialisation.f90:279-344) finds the crossings.
struct XCon {
    int64_t a, b;
    double kl, kr;
};

// kx*dt/(porosity*dyn_viscosity*(fluid_comp+rock_comp)*ds**2)
__device__ __forceinline__ double pcoef(const PressParams &p, double kx, double dt, double dsv)
{
    return __ddiv_rn(mul_(kx, dt), mul_(mul_(mul_(p.porosity, p.dyn_visc), p.comp), mul_(dsv, dsv)));
}

// Row coefficients of the unscaled matrix (compute_MatrixVector,
// src/fluid_diffusion.f90:175-204); A2 equals compute_diag's diagonal.
__device__ __forceinline__ void prow(const PressParams &p, int64_t k, double dt, double &A1, double &A2, double &A3)
{
    const int64_t N = p.N;
    if (k == 0) {
        A1 = 0.0;
        A2 = add_(1.0, pcoef(p, p.permx[1], dt, p.ds[0]));
        A3 = -pcoef(p, p.permx[1], dt, p.ds[0]);
    } else if (k == N - 1) {
        A1 = -pcoef(p, p.permx[N - 1], dt, p.ds[N - 1]);
        A2 = add_(1.0, pcoef(p, p.permx[N - 1], dt, p.ds[N - 1]));
        A3 = 0.0;
    } else {
        A1 = -pcoef(p, p.permx[k], dt, p.ds[k - 1]);
        A2 = add_(1.0, pcoef(p, add_(p.permx[k], p.permx[k + 1]), dt, p.ds[k]));
        A3 = -pcoef(p, p.permx[k + 1], dt, p.ds[k + 1]);
    }
}

// Row coefficients for the tridiagonal solver (tridiagonal handles, which
// always carry p.tcoef): from the precomputed dt-free factors, one
// multiplication each instead of a division; equal to prow up to rounding.
__device__ __forceinline__ void prow_tri(const PressParams &p, int64_t k, double dt, double &A1, double &A2,
                                         double &A3)
{
    const double *t = p.tcoef + 3 * k;
    A1 = -(dt * t[0]);
    A2 = 1.0 + dt * t[1];
    A3 = -(dt * t[2]);
}

// Fault-crossing coupling of row k (src/fluid_diffusion.f90:213-295,
// 338-405, with the element length of the row itself in every coefficient
// and every term divided by the diagonal): the diagonal gains
// kl dt/(c ds_k^2) + kr dt/(c ds_k^2) per contribution, the product gains
// (-cl v_a + (cl + cr) v_k - cr v_b) / diag_k, both in contribution order
// after the row's own stencil.
__device__ __forceinline__ double pdiag_x(const PressParams &p, int64_t k, double dt, double A2)
{
    for (int64_t c = p.xptr[k]; c < p.xptr[k + 1]; c++) {
        const XCon x = p.xcon[c];
        A2 = add_(add_(A2, pcoef(p, x.kl, dt, p.ds[k])), pcoef(p, x.kr, dt, p.ds[k]));
    }
    return A2;
}
__device__ __forceinline__ double pterms_x(const PressParams &p, int64_t k, double dt, double dg, const double *v,
                                           double m)
{
    for (int64_t c = p.xptr[k]; c < p.xptr[k + 1]; c++) {
        const XCon x = p.xcon[c];
        const double cl = pcoef(p, x.kl, dt, p.ds[k]), cr = pcoef(p, x.kr, dt, p.ds[k]);
        const double t = add_(add_(mul_(-cl, v[x.a]), mul_(add_(cl, cr), v[k])), mul_(-cr, v[x.b]));
        m = add_(m, __ddiv_rn(t, dg));
    }
    return m;
}

// Source contribution (before division by diag) at element k for step dt:
// src/fluid_diffusion.f90:52-64 with the reference's vector subscripts
// (every source of a fault is added once per active source of that fault).
__device__ __forceinline__ double psource(const PressParams &p, int64_t k, double dt)
{
    double add = 0.0;
    const double t = add_(*p.ctl_time, dt);
    for (int64_t s = 0; s < p.nsrc; s++) {
        if (!(t >= p.src_tb[s] && t < p.src_te[s])) continue;
        for (int64_t j = 0; j < p.nsrc; j++) {
            if (p.src_fault[j] != p.src_fault[s] || p.src_elem[j] != k) continue;
            add = add_(add, __ddiv_rn(__ddiv_rn(mul_(dt, p.src_Q[j]), mul_(p.porosity, p.comp)), p.ds[k]));
        }
    }
    return add;
}

// Block-wide reductions for the one-CTA CG (blockDim = 1024).
__device__ __forceinline__ double block_sum(double v, double *red)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = (lane < (blockDim.x >> 5)) ? red[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) red[32] = t;
    }
    __syncthreads();
    return red[32];
}
__device__ __forceinline__ double block_max(double v, double *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = (lane < (blockDim.x >> 5)) ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (lane == 0) red[32] = t;
    }
    __syncthreads();
    return red[32];
}

// Sum of a and max of b over the CTA in one pass (red: 66 doubles).
__device__ __forceinline__ void block_sum_max(double a, double b, double *red, double &sa, double &mb)
{
    a = warp_sum(a);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) { red[w] = a; red[33 + w] = b; }
    __syncthreads();
    if (w == 0) {
        double t = (lane < (blockDim.x >> 5)) ? red[lane] : 0.0;
        double u = (lane < (blockDim.x >> 5)) ? red[33 + lane] : 0.0;
        t = warp_sum(t);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) u = fmax(u, __shfl_xor_sync(0xffffffffu, u, o));
        if (lane == 0) { red[32] = t; red[65] = u; }
    }
    __syncthreads();
    sa = red[32];
    mb = red[65];
}

// Segments of at most TRI_SHORT_MAX elements are solved by one warp each
// (pressure_tridiag_kernel, up to TRI_WMAXM rows per lane), longer ones by a
// CTA of TRI_NT threads (pressure_tridiag_long_kernel), rows in registers up
// to TRI_MAXM rows per thread.
#define TRI_SHORT_MAX 64
#define TRI_WMAXM 2
#define TRI_NT 256
#define TRI_MAXM 16

// System s of a pressure launch gets its dt from the controller:
//   kind 0: dt = ctl->t_try (probe / first RHS), halving on non-convergence
//   kind 1: dt = ctl->x + A_{s+1} * ctl->h   (stage s+1, s = 1..5)
//   kind 2: dt = explicit value
struct PressSys {
    int kind;
    double dt_explicit;
};

// dt of a pressure system: 0 the probe (t_try), 1 a stage (x + c h),
// 2 explicit, 3 the commit solve of the step just accepted (its hdid).
__device__ __forceinline__ double sys_dt(const StepCtl *ctl, int kind, int sys, double dt_explicit)
{
    if (kind == 0) return ctl->t_try;
    if (kind == 1) return add_(ctl->x, mul_(ck_a(sys + 1), ctl->h));
    if (kind == 3) return ctl->hdid;
    return dt_explicit;
}

// One Jacobi-scaled CG solve (reference algorithm) by the whole CTA.
// Work vectors live in global memory (w: 4*N doubles). Returns ier.
// Row k of compute_MatrixVector (src/fluid_diffusion.f90:175-204): the
// Jacobi-scaled stencil (A1 v(k-1) + A2 v(k) + A3 v(k+1)) / diag(k), in the
// reference's operand order without FMA (diag(k) equals A2 of row k).
__device__ __forceinline__ double pmatvec_row(const PressParams &p, int64_t k, double dt, const double *v)
{
    double A1, A2, A3;
    prow(p, k, dt, A1, A2, A3);
    double m;
    if (k == 0) m = add_(mul_(A2, v[0]), mul_(A3, v[1]));
    else if (k == p.N - 1) m = add_(mul_(A1, v[k - 1]), mul_(A2, v[k]));
    else m = add_(add_(mul_(A1, v[k - 1]), mul_(A2, v[k])), mul_(A3, v[k + 1]));
    return __ddiv_rn(m, A2);
}

// Row k of a row with fault-crossing contributions, from scratch: its own
// stencil over the diagonal that includes the crossings, then the crossing
// terms (the reference's order).
__device__ __forceinline__ double pmatvec_row_x(const PressParams &p, int64_t k, double dt, const double *v)
{
    double A1, A2, A3;
    prow(p, k, dt, A1, A2, A3);
    const double dg = pdiag_x(p, k, dt, A2);
    double m;
    if (k == 0) m = add_(mul_(A2, v[0]), mul_(A3, v[1]));
    else if (k == p.N - 1) m = add_(mul_(A1, v[k - 1]), mul_(A2, v[k]));
    else m = add_(add_(mul_(A1, v[k - 1]), mul_(A2, v[k])), mul_(A3, v[k + 1]));
    return pterms_x(p, k, dt, dg, v, __ddiv_rn(m, dg));
}

// The same row with the coefficients of prow taken from a cache (identical
// operands and order, so identical results).
__device__ __forceinline__ double pmatvec_row_c(int64_t k, int64_t N, double A1, double A2, double A3, const double *v)
{
    double m;
    if (k == 0) m = add_(mul_(A2, v[0]), mul_(A3, v[1]));
    else if (k == N - 1) m = add_(mul_(A1, v[k - 1]), mul_(A2, v[k]));
    else m = add_(add_(mul_(A1, v[k - 1]), mul_(A2, v[k])), mul_(A3, v[k + 1]));
    return __ddiv_rn(m, A2);
}

// The Jacobi-scaled row with the off-diagonal coefficients divided by the
// diagonal once per solve (s1 = A1/A2, s3 = A3/A2): equal to pmatvec_row up
// to rounding, without a division per element and iteration.
__device__ __forceinline__ double pmatvec_row_s(int64_t k, int64_t N, double s1, double s3, const double *v)
{
    if (k == 0) return fma(s3, v[1], v[0]);
    if (k == N - 1) return fma(s1, v[k - 1], v[k]);
    return fma(s1, v[k - 1], fma(s3, v[k + 1], v[k]));
}

// b1(k) = P(k)/diag(k) plus the injection terms, each added separately as
// in src/fluid_diffusion.f90:45-64.
__device__ __forceinline__ double pb1(const PressParams &p, int64_t k, double dt, double diag)
{
    double b1 = __ddiv_rn(p.P[k], diag);
    const double t = add_(*p.ctl_time, dt);
    for (int64_t s = 0; s < p.nsrc; s++) {
        if (!(t >= p.src_tb[s] && t < p.src_te[s])) continue;
        for (int64_t j = 0; j < p.nsrc; j++) {
            if (p.src_fault[j] != p.src_fault[s] || p.src_elem[j] != k) continue;
            const double c = __ddiv_rn(__ddiv_rn(mul_(dt, p.src_Q[j]), mul_(p.porosity, p.comp)), p.ds[k]);
            b1 = add_(b1, __ddiv_rn(c, diag));
        }
    }
    return b1;
}

// sum(a*b) over the vectors in index order by one thread (the reference's
// sequential summation); every thread gets the result.
__device__ __forceinline__ double seq_dot(const double *a, const double *b, int64_t N, double *red)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int64_t k = 0; k < N; k++) s = add_(s, mul_(a[k], b[k]));
        red[32] = s;
    }
    __syncthreads();
    const double v = red[32];
    __syncthreads();
    return v;
}

// One Jacobi-scaled CG solve (src/fluid_diffusion.f90:79-131) by the whole
// CTA. Work vectors live in global memory. Element-wise arithmetic follows
// the reference's operand order without FMA. exact = 1 also sums the dot
// products sequentially, which reproduces the reference's rounding and so
// its iteration counts bit for bit (needed where a solve sits at the
// 200-iteration cap or at the tolerance, since that decides t_try halving);
// exact = 0 sums them with a tree reduction. Returns ier.
// With cf (3N doubles, or null): the row coefficients, which do not change
// during a solve, are computed once into cf, and the residual's sum of
// squares and max-norm share one reduction (red: 66 doubles); the iterates
// are the same as without.
// XC: the network has fault crossings (rows with crossing terms are
// recomputed after the plain stencil pass; instantiated only for such
// handles).
template <bool XC>
__device__ int cg_solve(const PressParams &p, double dt, double *x, double *r, double *pv, double *Mp, double *red,
                        long long *iters, int exact, double *cf = nullptr)
{
    const int64_t N = p.N;
    const int tid = threadIdx.x, nt = blockDim.x;
    double *c1 = cf, *c2 = cf ? cf + N : nullptr, *c3 = cf ? cf + 2 * N : nullptr;
    // x = P, r = b1 - M x, p = r
    double lmax = 0.0, lrr = 0.0;
    for (int64_t k = tid; k < N; k += nt) {
        double A1, A2, A3;
        prow(p, k, dt, A1, A2, A3);
        if (cf) {
            if (exact) { c1[k] = A1; c2[k] = A2; c3[k] = A3; }
            else { c1[k] = A1 / A2; c3[k] = A3 / A2; }
        }
        const double rk = add_(pb1(p, k, dt, A2), -(cf ? pmatvec_row_c(k, N, A1, A2, A3, p.P)
                                                        : pmatvec_row(p, k, dt, p.P)));
        x[k] = p.P[k];
        r[k] = rk;
        pv[k] = rk;
        lmax = fmax(lmax, fabs(rk));
        lrr += rk * rk;
    }
    if constexpr (XC) {
        // rows with fault crossings, from scratch, by the thread that owns
        // them; then the reductions over the corrected residual
        for (int64_t q = 0; q < p.nxrows; q++) {
            const int64_t k = p.xrows[q];
            if (k % nt != tid) continue;
            double A1, A2, A3;
            prow(p, k, dt, A1, A2, A3);
            const double rk = add_(pb1(p, k, dt, pdiag_x(p, k, dt, A2)), -pmatvec_row_x(p, k, dt, p.P));
            r[k] = rk;
            pv[k] = rk;
        }
        lmax = 0.0;
        lrr = 0.0;
        for (int64_t k = tid; k < N; k += nt) {
            lmax = fmax(lmax, fabs(r[k]));
            lrr += r[k] * r[k];
        }
    }
    double errmax = block_max(lmax, red) / p.tol;
    long long it = 0;
    // rr carried between iterations: sum(rk**2) of iteration i+1 equals
    // sum(rk1**2) of iteration i (rk = rk1, same summation), so it is
    // computed once.
    double rr = exact ? seq_dot(r, r, N, red) : block_sum(lrr, red);
    while (errmax >= 1.0) {
        it++;
        double lpap = 0.0;
        for (int64_t k = tid; k < N; k += nt) {
            const double m = !cf ? pmatvec_row(p, k, dt, pv)
                                 : (exact ? pmatvec_row_c(k, N, c1[k], c2[k], c3[k], pv)
                                          : pmatvec_row_s(k, N, c1[k], c3[k], pv));
            Mp[k] = m;
            lpap += pv[k] * m;
        }
        if constexpr (XC) {
            // rows with fault crossings, from scratch, by their owner thread
            for (int64_t q = 0; q < p.nxrows; q++) {
                const int64_t k = p.xrows[q];
                if (k % nt != tid) continue;
                const double m = pmatvec_row_x(p, k, dt, pv);
                lpap += pv[k] * (m - Mp[k]);
                Mp[k] = m;
            }
        }
        const double pap = exact ? seq_dot(pv, Mp, N, red) : block_sum(lpap, red);
        const double alpha = rr / pap;
        double lr1 = 0.0, lm = 0.0;
        for (int64_t k = tid; k < N; k += nt) {
            x[k] = add_(x[k], mul_(alpha, pv[k]));
            const double r1 = add_(r[k], -mul_(alpha, Mp[k]));
            r[k] = r1;
            lr1 += r1 * r1;
            lm = fmax(lm, fabs(r1));
        }
        double r1r1, mx;
        if (exact) {
            r1r1 = seq_dot(r, r, N, red);
            mx = block_max(lm, red);
        } else if (cf) {
            block_sum_max(lr1, lm, red, r1r1, mx);
        } else {
            r1r1 = block_sum(lr1, red);
            mx = block_max(lm, red);
        }
        const double beta = r1r1 / rr;
        for (int64_t k = tid; k < N; k += nt) pv[k] = add_(r[k], mul_(beta, pv[k]));
        // the next stencil reads the neighbours' pv: all updates first
        __syncthreads();
        rr = r1r1;
        if (it > 200) { *iters += it; return 1; }
        errmax = mx / p.tol;
    }
    *iters += it;
    return 0;
}

// One system of the reference CG for one instance (whole CTA), shared by
// the batched solver and the allocation-free entry point.
template <bool XC = false>
__device__ void cg_system(const PressParams &p, StepCtl *ctl, int kind, int sys, double dt_explicit, double *Pt,
                          double *Pd, double *x, double *r, double *pv, double *Mp, double *red, long long *iters,
                          int exact, double *cf = nullptr)
{
    const int64_t N = p.N;
    double dt = sys_dt(ctl, kind, sys, dt_explicit);
    int ier = cg_solve<XC>(p, dt, x, r, pv, Mp, red, iters, exact, cf);
    if (kind == 0) {
        // probe: src/solver.f90:81-92, halve t_try until the solve converges
        int guard = 0;
        while (ier == 1 && guard < 1100) {
            dt = dt / 2.0;
            guard++;
            ier = cg_solve<XC>(p, dt, x, r, pv, Mp, red, iters, exact, cf);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            ctl->t_try = dt;
            ctl->halvings += guard;
        }
    }
    __syncthreads();
    // A stage solve (kind 1) that hits the cap: the reference goes on with an
    // uninitialised P_temp and a stale P_dot (RateStateAgingModeII.f90:37-68
    // after compute_P returned early); here the stage uses the last CG
    // iterate instead, the attempt goes on, and the failure is counted. If it
    // is the stage-5 system, the commit keeps P unchanged, as the reference's
    // commit compute_P(t_did) (the same solve) returns early too.
    const int write = (ier == 0) || (kind == 1);
    if (write) {
        double lmx = 0.0;
        for (int64_t k = threadIdx.x; k < N; k += blockDim.x) {
            Pd[k] = (dt < 1e-9) ? 0.0 : (x[k] - p.P[k]) / dt;
            Pt[k] = x[k];
            lmx = fmax(lmx, fabs(x[k]));
        }
        double mx = block_max(lmx, red);
        if (!(mx <= 1.7976931348623157e308)) {
            if (threadIdx.x == 0) atomicCAS(&ctl->status, 0, 4);
        }
    }
    if (threadIdx.x == 0) {
        atomicAdd((unsigned long long *)&ctl->cg_iters, (unsigned long long)*iters);
        if (ier) {
            if (kind == 1) {
                atomicOr(&ctl->pfail_mask, 1 << sys);
                atomicAdd((unsigned long long *)&ctl->stage_noconv, 1ull);
            } else if (kind == 3) {
                // the commit solve: P stays as it was (the reference's
                // compute_P(t_did) returns early; its ier is not checked)
                atomicOr(&ctl->pfail_mask, 1 << 6);
            } else {
                if (kind == 0) ctl->probe_ier = 1;
                atomicCAS(&ctl->status, 0, 1);
            }
        }
    }
}

// Single system with explicit pointers (allocation-free entry point).
__global__ void __launch_bounds__(1024) pressure_cg_kernel(PressParams p, StepCtl *ctl, int kind, int sys0,
                                                           double dt_explicit, double *Ptemp, double *Pdot,
                                                           double *work)
{
    __shared__ double red[33];
    __shared__ long long iters;
    const int sys = sys0 + blockIdx.x;
    const int64_t N = p.N;
    double *x = work + (int64_t)sys * 4 * N, *r = x + N, *pv = r + N, *Mp = pv + N;
    if (threadIdx.x == 0) iters = 0;
    __syncthreads();
    cg_system(p, ctl, kind, sys, dt_explicit, Ptemp + (int64_t)sys * N, Pdot + (int64_t)sys * N, x, r, pv, Mp, red,
              &iters, 0);
}

// Global (all-instance) pressure arrays; instance i's slice starts at eoff_i
// (face permeabilities at eoff_i + i, they have N_i + 1 entries).
struct PressGlobal {
    const double *P, *permx, *ds;
    const int64_t *src_fault, *src_elem;   // src_elem: 0-based within the instance
    const double *src_Q, *src_tb, *src_te;
    const int64_t *xptr;                   // [Ntot + 1] crossing rows (null: no crossings)
    const XCon *xcon;
    const int64_t *xrows, *xrows_ptr;      // rows with crossings of instance i: xrows[xrows_ptr[i] ..)
    const double *tcoef;                   // [3 Ntot] tridiagonal row factors (null: computed by prow)
};

__device__ __forceinline__ PressParams press_params(const PressGlobal &g, const Inst &I, int i, const StepCtl *ctl)
{
    PressParams p;
    p.N = I.N; p.P = g.P + I.eoff; p.permx = g.permx + I.eoff + i; p.ds = g.ds + I.eoff;
    p.porosity = I.porosity; p.dyn_visc = I.dyn_visc; p.comp = I.comp; p.tol = I.tol;
    p.nsrc = I.nsrc; p.src_fault = g.src_fault + I.soff; p.src_elem = g.src_elem + I.soff;
    p.src_Q = g.src_Q + I.soff; p.src_tb = g.src_tb + I.soff; p.src_te = g.src_te + I.soff;
    p.ctl_time = &ctl[i].time;
    p.xptr = g.xptr ? g.xptr + I.eoff : nullptr;
    p.xcon = g.xcon;
    p.xrows = g.xptr ? g.xrows + g.xrows_ptr[i] : nullptr;
    p.nxrows = g.xptr ? g.xrows_ptr[i + 1] - g.xrows_ptr[i] : 0;
    p.tcoef = g.tcoef ? g.tcoef + 3 * I.eoff : nullptr;
    return p;
}

// Batched CG: CTA (system s, instance i). Work of instance i: 24*eoff, then
// 4*N_i per system; outputs Ptemp/Pdot at 6*eoff + sys*N_i.
template <bool XC>
__global__ void __launch_bounds__(1024) pressure_cg_batch_kernel(PressGlobal g, const Inst *inst, StepCtl *ctl,
                                                                 int mask, int kind, int sys0, double dt_explicit,
                                                                 double *Ptemp, double *Pdot, double *work, int exact,
                                                                 double *coef)
{
    __shared__ double red[66];
    __shared__ long long iters;
    const int i = blockIdx.y;
    if (!press_takes_part(ctl, i, mask, kind)) return;
    const Inst I = inst[i];
    const PressParams p = press_params(g, I, i, ctl);
    const int sys = sys0 + blockIdx.x;
    const int64_t N = I.N;
    double *x = work + 24 * I.eoff + (int64_t)sys * 4 * N, *r = x + N, *pv = r + N, *Mp = pv + N;
    if (threadIdx.x == 0) iters = 0;
    __syncthreads();
    cg_system<XC>(p, ctl + i, kind, sys, dt_explicit, Ptemp + 6 * I.eoff + (int64_t)sys * N,
                  Pdot + 6 * I.eoff + (int64_t)sys * N, x, r, pv, Mp, red, &iters, exact,
                  coef + 18 * I.eoff + (int64_t)sys * 3 * N);
}

// ---------------------------------------------------------------------------
// Cluster form of the Jacobi-scaled CG (exact = 0) for a few large systems.
// The CL CTAs of a thread-block cluster split the elements of one system
// into contiguous ranges of n elements (the last range may be shorter) and
// keep every vector of the solve in shared memory; a range's neighbour
// entries of the search direction and the CTAs' partial sums are read from
// the other CTAs' shared memory (distributed shared memory). Per iteration:
// two cluster barriers (one per reduction), no global-memory traffic. Each
// CTA sums the CL partial sums with the same butterfly, so every CTA holds
// the same scalars and takes the same branches. Iterates equal cg_solve's
// (exact = 0 with cached coefficients) up to the order of the dot-product
// sums.
//
// Race-freedom: a CTA's reduction slots and its r and direction entries are
// read by other CTAs only between the two barriers that follow their write;
// the direction is double-buffered by iteration parity, and the entry a
// neighbour needs at a range boundary for the next iteration is computed
// locally from the neighbour's r and current direction (both final after
// the second barrier, rewritten only after the next iteration's first).
//
// Layouts: "roomy" keeps x and M p in shared memory too; "lean" (ranges too
// long for that) keeps x in the system's global work area and recomputes
// M p in the second pass from the same operands (the same value), which
// lets a cluster of 16 CTAs hold systems of up to about 92 000 elements.
#define PCL_THREADS 1024
#define PCL_NTARGET 2048           // elements per CTA the cluster size aims at
#define PCL_SMEM_CAP (226 * 1024)  // dynamic shared memory per CTA (the rest: static)

// Dynamic shared memory of a cluster CTA with ranges of n elements: eight
// slot doubles, s1, s3, r (and x, M p unless lean) of n each, two direction
// buffers of n + 2.
__host__ __device__ constexpr size_t pcl_smem_bytes(int n, bool lean)
{
    return ((size_t)(lean ? 5 : 7) * n + 12) * sizeof(double);
}

namespace cgrp = cooperative_groups;

// Sum over the cluster: CTA tree sum, the CTA's partial into slot, cluster
// barrier, then each warp sums the CL partials (bitwise the same result in
// every lane, warp and CTA).
__device__ __forceinline__ double cluster_sum(double v, double *red, double *slot)
{
    cgrp::cluster_group cl = cgrp::this_cluster();
    v = block_sum(v, red);
    if (threadIdx.x == 0) *slot = v;
    cl.sync();
    const int lane = threadIdx.x & 31;
    double t = (lane < (int)cl.num_blocks()) ? *cl.map_shared_rank(slot, lane) : 0.0;
    return warp_sum(t);
}
// Sum of a and max of b over the cluster (slot: 2 doubles).
__device__ __forceinline__ void cluster_sum_max(double a, double b, double *red, double *slot, double &sa, double &mb)
{
    cgrp::cluster_group cl = cgrp::this_cluster();
    block_sum_max(a, b, red, sa, mb);
    if (threadIdx.x == 0) { slot[0] = sa; slot[1] = mb; }
    cl.sync();
    const int lane = threadIdx.x & 31;
    const bool on = lane < (int)cl.num_blocks();
    double t = on ? cl.map_shared_rank(slot, lane)[0] : 0.0;
    double u = on ? cl.map_shared_rank(slot, lane)[1] : 0.0;
    sa = warp_sum(t);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) u = fmax(u, __shfl_xor_sync(0xffffffffu, u, o));
    mb = u;
}

// Vectors of one cluster CTA (range of n elements): shared memory, except
// x in the lean layout (xg: this range's slice of the global work area).
struct PclVec {
    double *s1, *s3, *x, *r, *Mp, *pv;   // pv: two buffers of n + 2 (halo at 0 and n + 1); Mp null when lean
    double *slot;                        // reduction slots: [0..1] sum/max, [2] sum
};

__device__ __forceinline__ PclVec pcl_vec(double *sm, int n, bool lean, double *xg)
{
    PclVec v;
    v.slot = sm;
    v.s1 = sm + 8; v.s3 = v.s1 + n; v.r = v.s3 + n; v.pv = v.r + n;
    if (lean) {
        v.x = xg;
        v.Mp = nullptr;
    } else {
        v.x = v.pv + 2 * (n + 2);
        v.Mp = v.x + n;
    }
    return v;
}

// Row j of the Jacobi-scaled stencil on direction buffer pc (halo at 0).
__device__ __forceinline__ double pcl_row(const PclVec &v, const double *pc, int j, int64_t k, int64_t N)
{
    if (k == 0) return fma(v.s3[j], pc[j + 2], pc[j + 1]);
    if (k == N - 1) return fma(v.s1[j], pc[j], pc[j + 1]);
    return fma(v.s1[j], pc[j], fma(v.s3[j], pc[j + 2], pc[j + 1]));
}

// One CG solve by the cluster; this CTA owns elements [k0, k0 + nk) of a
// range of capacity n (ranges before the last are full). Returns ier, the
// same in every CTA.
__device__ int cg_solve_cluster(const PressParams &p, double dt, int64_t k0, int nk, int n, const PclVec &v,
                                double *red, long long *iters)
{
    cgrp::cluster_group cl = cgrp::this_cluster();
    const int rank = (int)cl.block_rank(), ncl = (int)cl.num_blocks();
    const int64_t N = p.N;
    const int tid = threadIdx.x, nt = blockDim.x;
    double *pc = v.pv;
    double lmax = 0.0, lrr = 0.0;
    for (int j = tid; j < nk; j += nt) {
        const int64_t k = k0 + j;
        double A1, A2, A3;
        prow(p, k, dt, A1, A2, A3);
        v.s1[j] = A1 / A2;
        v.s3[j] = A3 / A2;
        const double rk = add_(pb1(p, k, dt, A2), -pmatvec_row_c(k, N, A1, A2, A3, p.P));
        v.x[j] = p.P[k];
        v.r[j] = rk;
        pc[j + 1] = rk;
        lmax = fmax(lmax, fabs(rk));
        lrr += rk * rk;
    }
    double rr, mx0;
    cluster_sum_max(lrr, lmax, red, v.slot, rr, mx0);
    // halo of the first direction (= r) from the neighbours
    if (tid == 0 && rank > 0) pc[0] = cl.map_shared_rank(pc, rank - 1)[n];
    if (tid == 32 && rank < ncl - 1) pc[nk + 1] = cl.map_shared_rank(pc, rank + 1)[1];
    __syncthreads();
    double errmax = mx0 / p.tol;
    long long it = 0;
    int cur = 0;
    int ier = 0;
    while (errmax >= 1.0) {
        it++;
        pc = v.pv + cur * (n + 2);
        double lpap = 0.0;
        for (int j = tid; j < nk; j += nt) {
            const double m = pcl_row(v, pc, j, k0 + j, N);
            if (v.Mp) v.Mp[j] = m;
            lpap += pc[j + 1] * m;
        }
        const double pap = cluster_sum(lpap, red, v.slot + 2);
        const double alpha = rr / pap;
        double lr1 = 0.0, lm = 0.0;
        for (int j = tid; j < nk; j += nt) {
            v.x[j] = add_(v.x[j], mul_(alpha, pc[j + 1]));
            const double m = v.Mp ? v.Mp[j] : pcl_row(v, pc, j, k0 + j, N);
            const double r1 = add_(v.r[j], -mul_(alpha, m));
            v.r[j] = r1;
            lr1 += r1 * r1;
            lm = fmax(lm, fabs(r1));
        }
        double r1r1, mx;
        cluster_sum_max(lr1, lm, red, v.slot, r1r1, mx);
        const double beta = r1r1 / rr;
        double *pn = v.pv + (cur ^ 1) * (n + 2);
        for (int j = tid; j < nk; j += nt) pn[j + 1] = add_(v.r[j], mul_(beta, pc[j + 1]));
        if (tid == 0 && rank > 0)
            pn[0] = add_(cl.map_shared_rank(v.r, rank - 1)[n - 1], mul_(beta, cl.map_shared_rank(pc, rank - 1)[n]));
        if (tid == 32 && rank < ncl - 1)
            pn[nk + 1] = add_(cl.map_shared_rank(v.r, rank + 1)[0], mul_(beta, cl.map_shared_rank(pc, rank + 1)[1]));
        __syncthreads();
        cur ^= 1;
        rr = r1r1;
        if (it > 200) { ier = 1; break; }
        errmax = mx / p.tol;
    }
    // the next solve (or the output) may reuse the slots and buffers only
    // after every CTA has read this one's last partial sums
    cl.sync();
    *iters += it;
    return ier;
}

// Batched cluster CG: cluster (system s, instance i) of CL CTAs along x.
// Same systems, outputs and controller updates as pressure_cg_batch_kernel
// with exact = 0. Instance i is split into ranges of ceil(N_i / CL)
// elements (dynamic shared memory sized for the largest instance); lean:
// x of system s in work + 24 eoff_i + 4 N_i s (the one-CTA solver's x).
// With clusters of one CTA (launched with PCL_SMEM_CAP bytes) the layout is
// chosen per system (roomy, lean, or, when even the lean layout does not
// fit, the one-CTA solver on global memory: cg_system with the work vectors
// and cached coefficients of pressure_cg_batch_kernel).
__global__ void __launch_bounds__(PCL_THREADS, 1)
    pressure_cg_cluster_kernel(PressGlobal g, const Inst *inst, StepCtl *ctl, int mask, int kind, int sys0,
                               double dt_explicit, double *Ptemp, double *Pdot, double *work, int lean,
                               double *coef)
{
    extern __shared__ __align__(16) double pcl_sm[];
    __shared__ double red[66];
    __shared__ long long iters;
    cgrp::cluster_group cl = cgrp::this_cluster();
    const int ncl = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int i = blockIdx.y;
    if (!press_takes_part(ctl, i, mask, kind)) return;   // uniform over the cluster
    const Inst I = inst[i];
    const PressParams p = press_params(g, I, i, ctl);
    const int sys = sys0 + (int)(blockIdx.x / ncl);
    const int64_t N = I.N;
    const int n = (int)((N + ncl - 1) / ncl);
    StepCtl *c = ctl + i;
    if (threadIdx.x == 0) iters = 0;
    __syncthreads();
    if (ncl == 1) {
        if (pcl_smem_bytes(n, true) > (size_t)PCL_SMEM_CAP) {
            double *x = work + 24 * I.eoff + (int64_t)sys * 4 * N, *r = x + N, *pv = r + N, *Mp = pv + N;
            cg_system(p, c, kind, sys, dt_explicit, Ptemp + 6 * I.eoff + (int64_t)sys * N,
                      Pdot + 6 * I.eoff + (int64_t)sys * N, x, r, pv, Mp, red, &iters, 0,
                      coef + 18 * I.eoff + (int64_t)sys * 3 * N);
            return;
        }
        lean = pcl_smem_bytes(n, false) > (size_t)PCL_SMEM_CAP ? 1 : 0;
    }
    const int64_t k0 = (int64_t)rank * n;
    const int nk = (int)max((int64_t)0, min((int64_t)n, N - k0));
    const PclVec v = pcl_vec(pcl_sm, n, lean != 0, work + 24 * I.eoff + (int64_t)sys * 4 * N + k0);
    double dt = sys_dt(c, kind, sys, dt_explicit);
    int ier = cg_solve_cluster(p, dt, k0, nk, n, v, red, &iters);
    int guard = 0;
    if (kind == 0) {
        // probe: src/solver.f90:81-92, halve t_try until the solve converges
        while (ier == 1 && guard < 1100) {
            dt = dt / 2.0;
            guard++;
            ier = cg_solve_cluster(p, dt, k0, nk, n, v, red, &iters);
        }
    }
    // as cg_system: a stage solve that hits the cap still writes its last iterate
    const int write = (ier == 0) || (kind == 1);
    double mxx = 0.0;
    if (write) {
        double *Pt = Ptemp + 6 * I.eoff + (int64_t)sys * N, *Pd = Pdot + 6 * I.eoff + (int64_t)sys * N;
        double lmx = 0.0;
        for (int j = threadIdx.x; j < nk; j += blockDim.x) {
            const int64_t k = k0 + j;
            const double xk = v.x[j];
            Pd[k] = (dt < 1e-9) ? 0.0 : (xk - p.P[k]) / dt;
            Pt[k] = xk;
            lmx = fmax(lmx, fabs(xk));
        }
        double unused;
        cluster_sum_max(0.0, lmx, red, v.slot, unused, mxx);
    }
    if (rank == 0 && threadIdx.x == 0) {
        if (kind == 0) {
            c->t_try = dt;
            c->halvings += guard;
        }
        if (write && !(mxx <= 1.7976931348623157e308)) atomicCAS(&c->status, 0, 4);
        atomicAdd((unsigned long long *)&c->cg_iters, (unsigned long long)iters);
        if (ier) {
            if (kind == 1) {
                atomicOr(&c->pfail_mask, 1 << sys);
                atomicAdd((unsigned long long *)&c->stage_noconv, 1ull);
            } else if (kind == 3) {
                atomicOr(&c->pfail_mask, 1 << 6);   // the commit solve: P stays (as cg_system)
            } else {
                if (kind == 0) c->probe_ier = 1;
                atomicCAS(&c->status, 0, 1);
            }
        }
    }
    cl.sync();   // no CTA leaves while another may still read its shared memory
}

// Exact solve of the unscaled tridiagonal system A x = P + source, one
// thread per decoupled segment (a maximal run of elements joined by nonzero
// face permeability; the fake elements between faults are segments of one).
// seg_start holds global element indices; segments never cross instances.
// ---------------------------------------------------------------------------
// The Thomas recurrences of one segment evaluated by a group of NTG threads
// (a warp for short segments, a CTA for long ones).
//
// Thread t owns rows [t*m, t*m + m) of the segment (m = ceil(L / NTG)).
// The three sequential recurrences of the Thomas algorithm are each a scan
// over an associative operator, so the group computes the value entering
// every thread's rows with a scan of the per-thread compositions (warp
// shuffles, plus shared memory across the warps of a CTA) and each thread
// then reruns the exact recurrence over its own rows:
//   c_k = A3_k / (A2_k - A1_k c_{k-1})       a Moebius map of c_{k-1}: the
//        2x2 matrix [[0, A3], [-A1, A2]] acting on (p, q), c = p/q; products
//        are rescaled by a power of two near their largest entry (exact; the
//        ratio is unchanged);
//   d_k = (r_k - A1_k d_{k-1}) / den_k        affine in d_{k-1};
//   x_k = d_k - c_k x_{k+1}                   affine in x_{k+1}, scanned from
//        the end of the segment.
// The system is an M-matrix (diagonally dominant, A1, A3 <= 0), so |c| < 1
// and every composed map is contracting; the result equals the sequential
// solve to rounding. Rows live in registers for m <= TRI_MAXM, otherwise in
// the global work area of the system.
struct Mob { double a, b, c, d; };   // [[a, b], [c, d]]
struct Aff { double a, b; };         // x -> a x + b

__device__ __forceinline__ Mob mob_id() { return {1.0, 0.0, 0.0, 1.0}; }
__device__ __forceinline__ Aff aff_id() { return {1.0, 0.0}; }
// 2^-e for s in [2^e, 2^(e+1)) (normal s), else 1: an exact rescaling.
__device__ __forceinline__ double pow2_inv(double s)
{
    const long long bits = __double_as_longlong(s);
    const int ex = (int)((bits >> 52) & 0x7FF);
    if (ex == 0 || ex >= 2046) return 1.0;
    return __longlong_as_double((long long)(2046 - ex) << 52);
}
// outer o applied after inner i
__device__ __forceinline__ Mob compose(const Mob &o, const Mob &i)
{
    Mob r{o.a * i.a + o.b * i.c, o.a * i.b + o.b * i.d, o.c * i.a + o.d * i.c, o.c * i.b + o.d * i.d};
    const double q = pow2_inv(fmax(fmax(fabs(r.a), fabs(r.b)), fmax(fabs(r.c), fabs(r.d))));
    r.a *= q; r.b *= q; r.c *= q; r.d *= q;
    return r;
}
__device__ __forceinline__ Aff compose(const Aff &o, const Aff &i) { return {o.a * i.a, o.a * i.b + o.b}; }
__device__ __forceinline__ Mob shfl_up(const Mob &v, int d)
{
    return {__shfl_up_sync(0xffffffffu, v.a, d), __shfl_up_sync(0xffffffffu, v.b, d),
            __shfl_up_sync(0xffffffffu, v.c, d), __shfl_up_sync(0xffffffffu, v.d, d)};
}
__device__ __forceinline__ Aff shfl_up(const Aff &v, int d)
{
    return {__shfl_up_sync(0xffffffffu, v.a, d), __shfl_up_sync(0xffffffffu, v.b, d)};
}
__device__ __forceinline__ Aff shfl_down(const Aff &v, int d)
{
    return {__shfl_down_sync(0xffffffffu, v.a, d), __shfl_down_sync(0xffffffffu, v.b, d)};
}

// Exclusive forward scan over the group (thread 0 first): returns the
// composition of the maps of threads 0..t-1 (identity for t = 0).
template <int NTG, typename T>
__device__ __forceinline__ T grp_scan_excl(T v, T ident, T *sm)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = NTG / 32;
    for (int d = 1; d < 32; d <<= 1) {
        T o = shfl_up(v, d);
        if (lane >= d) v = compose(v, o);
    }
    if constexpr (NTG == 32) {
        T prev = shfl_up(v, 1);
        return (lane == 0) ? ident : prev;
    }
    __syncthreads();
    if (lane == 31) sm[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        T acc = ident;
        for (int q = 0; q < nw; q++) {
            T tot = sm[q];
            sm[q] = acc;               // prefix of the warps before q
            acc = compose(tot, acc);
        }
    }
    __syncthreads();
    T prev = shfl_up(v, 1);
    const T wp = sm[w];
    return (lane == 0) ? wp : compose(prev, wp);
}

// Exclusive backward scan for affine maps: the composition of the maps of
// threads t+1..NTG-1, the last thread's applied first (identity for the last).
template <int NTG>
__device__ __forceinline__ Aff grp_scan_excl_back(Aff v, Aff *sm)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = NTG / 32;
    for (int d = 1; d < 32; d <<= 1) {
        Aff o = shfl_down(v, d);
        if (lane + d < 32) v = compose(v, o);
    }
    if constexpr (NTG == 32) {
        Aff next = shfl_down(v, 1);
        return (lane == 31) ? aff_id() : next;
    }
    __syncthreads();
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        Aff acc = aff_id();
        for (int q = nw - 1; q >= 0; q--) {
            Aff tot = sm[q];
            sm[q] = acc;               // composition of the warps after q
            acc = compose(tot, acc);
        }
    }
    __syncthreads();
    Aff next = shfl_down(v, 1);
    const Aff ws = sm[w];
    return (lane == 31) ? ws : compose(next, ws);
}

// f(j) for the rows j < nr of this thread, in order (REV: reverse order);
// with MAXM > 0 the loop is unrolled so that register arrays stay registers.
template <int MAXM, bool REV, typename F>
__device__ __forceinline__ void tri_rows(int nr, F f)
{
    if constexpr (MAXM > 0) {
#pragma unroll
        for (int q = 0; q < MAXM; q++) {
            const int j = REV ? MAXM - 1 - q : q;
            if (j < nr) f(j);
        }
    } else {
        for (int q = 0; q < nr; q++) f(REV ? nr - 1 - q : q);
    }
}

template <int NTG, int MAXM>
__device__ __forceinline__ void tri_segment(const PressParams &p, double dt, int64_t k0, int64_t k1, double *Pt,
                                            double *Pd, double *gw, int64_t N, Mob *smm, Aff *sma, int &bad)
{
    const int64_t L = k1 - k0;
    const int tid = (NTG == 32) ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
    const int64_t m = (L + NTG - 1) / NTG;
    const int64_t r0 = (int64_t)tid * m;
    const int nr = (int)max((int64_t)0, min(m, L - r0));
    constexpr int R = (MAXM > 0) ? MAXM : 1;
    double reg[4][R];
    // row q of element j of this thread: A1, 1/den (A2 on input), c (A3 on
    // input), d (right-hand side on input)
    auto at = [&](int q, int j) -> double & {
        if constexpr (MAXM > 0) return reg[q][j];
        else return gw[(int64_t)q * N + k0 + r0 + j];
    };
    tri_rows<MAXM, false>(nr, [&](int j) {
        const int64_t k = k0 + r0 + j;
        double A1, A2, A3;
        prow_tri(p, k, dt, A1, A2, A3);
        if (k == k0) A1 = 0.0;
        if (k == k1 - 1) A3 = 0.0;
        at(0, j) = A1; at(1, j) = A2; at(2, j) = A3;
        at(3, j) = add_(p.P[k], psource(p, k, dt));
    });
    // c recurrence
    Mob T = mob_id();
    tri_rows<MAXM, false>(nr, [&](int j) { T = compose(Mob{0.0, at(2, j), -at(0, j), at(1, j)}, T); });
    const Mob E = grp_scan_excl<NTG>(T, mob_id(), smm);
    double c = (tid == 0) ? 0.0 : E.b / E.d;
    tri_rows<MAXM, false>(nr, [&](int j) {
        const double rden = 1.0 / (at(1, j) - at(0, j) * c);
        c = at(2, j) * rden;
        at(1, j) = rden; at(2, j) = c;
    });
    // d recurrence
    Aff F = aff_id();
    tri_rows<MAXM, false>(nr, [&](int j) { F = compose(Aff{-at(0, j) * at(1, j), at(3, j) * at(1, j)}, F); });
    double d = grp_scan_excl<NTG>(F, aff_id(), sma).b;
    tri_rows<MAXM, false>(nr, [&](int j) {
        d = (at(3, j) - at(0, j) * d) * at(1, j);
        at(3, j) = d;
    });
    // back substitution
    Aff G = aff_id();
    tri_rows<MAXM, true>(nr, [&](int j) { G = compose(Aff{-at(2, j), at(3, j)}, G); });
    double x = grp_scan_excl_back<NTG>(G, sma).b;
    const double rdt = (dt < 1e-9) ? 0.0 : 1.0 / dt;
    tri_rows<MAXM, true>(nr, [&](int j) {
        const int64_t k = k0 + r0 + j;
        x = at(3, j) - at(2, j) * x;
        Pt[k] = x;
        Pd[k] = (x - p.P[k]) * rdt;
        if (!isfinite(x)) bad = 1;
    });
}

// Short segments, one thread each (the sequential Thomas algorithm): for
// launches with many more segments than a wave of warps, where the scans'
// instructions would outweigh the latency they hide. grid (ceil(segments /
// 128), systems), blockDim 128.
__global__ void __launch_bounds__(128) pressure_tridiag_thread_kernel(PressGlobal g, const Inst *inst, StepCtl *ctl,
                                                                      int mask, int kind, int sys0,
                                                                      double dt_explicit, const int64_t *seg_start,
                                                                      const int *seg_inst, const int *seg_list,
                                                                      int64_t nlist, double *Ptemp, double *Pdot,
                                                                      double *work)
{
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= nlist) return;
    const int sg = seg_list[q];
    const int i = seg_inst[sg];
    if (!press_takes_part(ctl, i, mask, kind)) return;
    const Inst I = inst[i];
    const PressParams p = press_params(g, I, i, ctl);
    const int sys = sys0 + blockIdx.y;
    const int64_t N = I.N;
    const double dt = sys_dt(ctl + i, kind, sys, dt_explicit);
    const int64_t k0 = seg_start[sg] - I.eoff, k1 = seg_start[sg + 1] - I.eoff;
    double *cp = work + 24 * I.eoff + (int64_t)sys * 4 * N;   // modified super-diagonal
    double *dp = cp + N;                                       // modified right-hand side
    double *Pt = Ptemp + 6 * I.eoff + (int64_t)sys * N, *Pd = Pdot + 6 * I.eoff + (int64_t)sys * N;
    double cprev = 0.0, dprev = 0.0;
#pragma unroll 4
    for (int64_t k = k0; k < k1; k++) {
        double A1, A2, A3;
        prow_tri(p, k, dt, A1, A2, A3);
        if (k == k0) A1 = 0.0;
        if (k == k1 - 1) A3 = 0.0;
        const double rhs = add_(p.P[k], psource(p, k, dt));
        const double rden = 1.0 / (A2 - A1 * cprev);
        const double c = A3 * rden;
        const double d = (rhs - A1 * dprev) * rden;
        cp[k] = c; dp[k] = d;
        cprev = c; dprev = d;
    }
    const double rdt = (dt < 1e-9) ? 0.0 : 1.0 / dt;
    double xn = 0.0;
    bool bad = false;
#pragma unroll 4
    for (int64_t k = k1 - 1; k >= k0; k--) {
        const double xk = dp[k] - cp[k] * xn;
        xn = xk;
        Pt[k] = xk;
        Pd[k] = (xk - p.P[k]) * rdt;
        if (!isfinite(xk)) bad = true;
    }
    if (bad) atomicCAS(&ctl[i].status, 0, 4);
}

// dt-free row factors of the tridiagonal solver (prow's coefficients divided
// by dt): u = kx_k / (c ds_{k-1}^2), v = (kx_k + kx_{k+1}) / (c ds_k^2),
// w = kx_{k+1} / (c ds_{k+1}^2), c = porosity dyn_viscosity (fluid_comp +
// rock_comp), with prow's first and last rows.
__global__ void tri_coef_kernel(PressGlobal g, const Inst *inst, const int *inst_of, int64_t Ntot, double *tcoef)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= Ntot) return;
    const int i = inst_of[e];
    const Inst I = inst[i];
    const int64_t N = I.N, k = e - I.eoff;
    const double *px = g.permx + I.eoff + i, *ds = g.ds + I.eoff;
    const double c = I.porosity * I.dyn_visc * I.comp;
    double u, v, w;
    if (k == 0) {
        u = 0.0;
        v = px[1] / (c * (ds[0] * ds[0]));
        w = v;
    } else if (k == N - 1) {
        u = px[N - 1] / (c * (ds[N - 1] * ds[N - 1]));
        v = u;
        w = 0.0;
    } else {
        u = px[k] / (c * (ds[k - 1] * ds[k - 1]));
        v = (px[k] + px[k + 1]) / (c * (ds[k] * ds[k]));
        w = px[k + 1] / (c * (ds[k + 1] * ds[k + 1]));
    }
    tcoef[3 * e] = u;
    tcoef[3 * e + 1] = v;
    tcoef[3 * e + 2] = w;
}

// Short segments in tiles: one 128-thread CTA per tile of consecutive
// short segments (at most TRI_TILE elements and 128 segments: tiles[b] =
// (first entry in seg_list, count)), grid (tiles, systems). P, ds and the
// face permeabilities of the tile are staged into shared memory with
// coalesced loads (P and the precomputed row factors), each thread solves
// one segment with the recurrence of pressure_tridiag_thread_kernel (the
// same operations: identical results) from shared memory, and the results
// leave with coalesced stores.
#define TRI_TILE 512   // 24 KB of shared memory: one tile CTA fits beside a persistent GEMM CTA

__global__ void __launch_bounds__(128) pressure_tridiag_tile_kernel(PressGlobal g, const Inst *inst, StepCtl *ctl,
                                                                    int mask, int kind, int sys0,
                                                                    double dt_explicit, const int64_t *seg_start,
                                                                    const int *seg_inst, const int *seg_list,
                                                                    const int2 *tiles, double *Ptemp, double *Pdot)
{
    __shared__ double sP[TRI_TILE], st[3 * TRI_TILE], sc[TRI_TILE], sd[TRI_TILE];
    const int2 t = tiles[blockIdx.x];
    const int sg0 = seg_list[t.x];
    const int i = seg_inst[sg0];
    if (!press_takes_part(ctl, i, mask, kind)) return;   // one instance per tile
    const Inst I = inst[i];
    const PressParams p = press_params(g, I, i, ctl);
    const int sys = sys0 + blockIdx.y;
    const int64_t N = I.N;
    const double dt = sys_dt(ctl + i, kind, sys, dt_explicit);
    const int64_t e0 = seg_start[sg0] - I.eoff, e1 = seg_start[seg_list[t.x + t.y - 1] + 1] - I.eoff;
    const int n = (int)(e1 - e0);
    for (int j = threadIdx.x; j < n; j += blockDim.x) sP[j] = p.P[e0 + j];
    for (int j = threadIdx.x; j < 3 * n; j += blockDim.x) st[j] = p.tcoef[3 * e0 + j];
    __syncthreads();
    PressParams q = p;   // the same parameters, P and the row factors in shared memory
    q.P = sP - e0;
    q.tcoef = st - 3 * e0;
    bool bad = false;
    if ((int)threadIdx.x < t.y) {
        const int sg = seg_list[t.x + threadIdx.x];
        const int64_t k0 = seg_start[sg] - I.eoff, k1 = seg_start[sg + 1] - I.eoff;
        double cprev = 0.0, dprev = 0.0;
        for (int64_t k = k0; k < k1; k++) {
            double A1, A2, A3;
            prow_tri(q, k, dt, A1, A2, A3);
            if (k == k0) A1 = 0.0;
            if (k == k1 - 1) A3 = 0.0;
            const double rhs = add_(q.P[k], psource(q, k, dt));
            const double rden = 1.0 / (A2 - A1 * cprev);
            const double c = A3 * rden;
            const double d = (rhs - A1 * dprev) * rden;
            sc[k - e0] = c;
            sd[k - e0] = d;
            cprev = c;
            dprev = d;
        }
            const double rdt = (dt < 1e-9) ? 0.0 : 1.0 / dt;
        double xn = 0.0;
        for (int64_t k = k1 - 1; k >= k0; k--) {
            const double xk = sd[k - e0] - sc[k - e0] * xn;
            xn = xk;
            sc[k - e0] = xk;                       // P_temp
            sd[k - e0] = (xk - q.P[k]) * rdt;      // P_dot
            if (!isfinite(xk)) bad = true;
        }
    }
    __syncthreads();
    double *Pt = Ptemp + 6 * I.eoff + (int64_t)sys * N, *Pd = Pdot + 6 * I.eoff + (int64_t)sys * N;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        Pt[e0 + j] = sc[j];
        Pd[e0 + j] = sd[j];
    }
    if (bad) atomicCAS(&ctl[i].status, 0, 4);
}

// Short segments, one warp each: grid (ceil(segments / 8), systems),
// blockDim 256; seg_list holds the launch's short segments.
__global__ void __launch_bounds__(256) pressure_tridiag_kernel(PressGlobal g, const Inst *inst, StepCtl *ctl,
                                                               int mask, int kind, int sys0, double dt_explicit,
                                                               const int64_t *seg_start, const int *seg_inst,
                                                               const int *seg_list, int64_t nlist, double *Ptemp,
                                                               double *Pdot, double *work)
{
    const int64_t q = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= nlist) return;                      // whole warp
    const int sg = seg_list[q];
    const int i = seg_inst[sg];
    if (!press_takes_part(ctl, i, mask, kind)) return;       // whole warp
    const Inst I = inst[i];
    const PressParams p = press_params(g, I, i, ctl);
    const int sys = sys0 + blockIdx.y;
    const int64_t N = I.N;
    const double dt = sys_dt(ctl + i, kind, sys, dt_explicit);
    const int64_t k0 = seg_start[sg] - I.eoff, k1 = seg_start[sg + 1] - I.eoff;
    double *Pt = Ptemp + 6 * I.eoff + (int64_t)sys * N, *Pd = Pdot + 6 * I.eoff + (int64_t)sys * N;
    int bad = 0;
    tri_segment<32, TRI_WMAXM>(p, dt, k0, k1, Pt, Pd, nullptr, N, nullptr, nullptr, bad);
    if (bad) atomicCAS(&ctl[i].status, 0, 4);
}

// grid (long segments of the launch, systems); blockDim = TRI_NT.
__global__ void __launch_bounds__(TRI_NT, 1) pressure_tridiag_long_kernel(PressGlobal g, const Inst *inst,
                                                                          StepCtl *ctl, int mask, int kind, int sys0,
                                                                          double dt_explicit,
                                                                          const int64_t *seg_start,
                                                                          const int *seg_inst, const int *long_seg,
                                                                          double *Ptemp, double *Pdot, double *work)
{
    __shared__ Mob smm[TRI_NT / 32];
    __shared__ Aff sma[TRI_NT / 32];
    __shared__ int sbad;
    const int sg = long_seg[blockIdx.x];
    const int i = seg_inst[sg];
    if (!press_takes_part(ctl, i, mask, kind)) return;       // uniform over the CTA
    const Inst I = inst[i];
    const PressParams p = press_params(g, I, i, ctl);
    const int sys = sys0 + blockIdx.y;
    const int64_t N = I.N;
    const double dt = sys_dt(ctl + i, kind, sys, dt_explicit);
    const int64_t k0 = seg_start[sg] - I.eoff, k1 = seg_start[sg + 1] - I.eoff;
    double *Pt = Ptemp + 6 * I.eoff + (int64_t)sys * N, *Pd = Pdot + 6 * I.eoff + (int64_t)sys * N;
    double *gw = work + 24 * I.eoff + (int64_t)sys * 4 * N;
    if (threadIdx.x == 0) sbad = 0;
    int bad = 0;
    if (k1 - k0 <= (int64_t)TRI_NT * TRI_MAXM)
        tri_segment<TRI_NT, TRI_MAXM>(p, dt, k0, k1, Pt, Pd, gw, N, smm, sma, bad);
    else
        tri_segment<TRI_NT, 0>(p, dt, k0, k1, Pt, Pd, gw, N, smm, sma, bad);
    if (bad) atomicOr(&sbad, 1);
    __syncthreads();
    if (threadIdx.x == 0 && sbad) atomicCAS(&ctl[i].status, 0, 4);
}

// ---------------------------------------------------------------------------
// Friction right-hand side fused with the Cash-Karp stage arithmetic.
struct FricParams {
    int64_t Ntot;                 // elements of all instances
    int mode;
    const Inst *inst;
    const int *inst_of;           // instance of each global element
    const double *a, *b, *Dc, *f0, *V0, *nload, *sload;
    const unsigned char *fake;
    const double *partT, *partN;  // per instance [nchunk][N] at poff
    double *SigT, *SigN;          // stress rates of this evaluation
    const double *Ptemp, *Pdot;   // per instance [6][N] at 6*eoff
    const double *Pc;             // committed pressure [Ntot]
    const double *y;              // state at the step start, [3N] at 3*eoff
    double *ytmp;                 // ytemp of this stage (in) / next stage (out)
    double *kbuf;                 // per instance [6][3N] at 18*eoff
    double *yscal, *yout;         // [3N] at 3*eoff
    StepCtl *ctl;
    // Newton formulation
    int form;                     // 0 = V formulation, 1 = Newton
    int guess;                    // DFN_GUESS_*
    int maxit;
    double tol;
    double off_explicit;          // stage-0 offset of the evaluation from the step start
    const double *tau0;           // [Ntot] shear traction at slip 0
    double *wlast;                // [Ntot] last solution, warm start
    double *vnow;                 // [Ntot] V of this evaluation
    const MlpTC *mlp;             // tensor-core image of the learned guess (global)
    double mlp_gate;              // relative residual of the analytic start above which it is evaluated
    // V formulation: slip as a passive component (dslip/dt = V)
    const double *slip;           // [Ntot] committed
    double *slip_out, *slip_acc;  // [Ntot] the attempt's 5th-order slip, partial stage sum
    float *rec_x, *rec_t;         // recorded solves
    unsigned long long *rec_n;
    long long rec_cap;
};

// Newton formulation of one element: stresses from slip, V from the
// friction law (newton_core.cuh), derivatives of slip and log-state. The
// normal-stress slot of the state holds sigmaN at slip 0 (derivative 0).
// First half: stresses of the stage, the bounded analytic start and its
// residual, the network inputs where the start misses the tolerance.
struct NPre {
    double tau, s, lnA, wa, ga;
    int kind;          // 0 fake element, 1 no frictional strength, 2 solve
    bool wa_ok;        // the analytic start meets the tolerance
    bool need;         // the analytic start misses the tolerance (the learned guess may help)
    bool big;          // ... by more than the gate: calls for the network in this warp
    float x[MLP_IN];
};

__device__ __forceinline__ void newton_pre(const FricParams &f, int64_t e, int mode, double eta, double tt,
                                           double psi, double sig0, double T, double Nn, double Pt, NPre &q)
{
    const double a = f.a[e], b = f.b[e], V0 = f.V0[e];
    q.tau = f.tau0[e] + T + f.sload[e] * tt;
    const double sig = ((mode == 2) ? sig0 + Nn : sig0) + f.nload[e] * tt;
    q.s = -(sig + Pt);
    q.wa_ok = true;
    q.need = false;
    q.big = false;
    q.kind = f.fake[e] ? 0 : (q.s > 0.0 ? 2 : 1);
    if (q.kind != 2) return;
    const double s = q.s, tau = q.tau;
    q.lnA = log(2.0 * V0) - (f.f0[e] + b * psi) / a;
    // g(w) = tau - eta V(w) - s a w is decreasing, concave for w > 0 (convex
    // for w < 0); the friction-only root w0 and the radiation-only root wr
    // both lie beyond the root on the same side, so the one nearer zero is a
    // start from which Newton approaches the root monotonically.
    const double w0 = tau / (s * a);
    const double wr = w_radiation(tau, eta, q.lnA);
    q.wa = (f.guess != 3 && fabs(wr) < fabs(w0)) ? wr : w0;
    q.ga = 0.0;
    // residual of the analytic start; where it meets the tolerance (slow
    // slip, radiation damping negligible) Newton takes no step and the
    // network is neither evaluated nor trained on the solve
    if (f.guess == 1 || f.rec_cap > 0) {
        double eva, da;
        eta_v(q.wa, q.lnA, eta, eva, da);
        q.ga = fabs(tau - eva - s * a * q.wa);
        q.wa_ok = q.ga <= f.tol * (fabs(tau) + s * a * fabs(q.wa) + 1e-300);
        if (!q.wa_ok) mlp_features(q.wa, w0, wr, psi, s, Pt, a, b, q.x);
        // the network is worth its cost only in warps where Newton from the
        // analytic start would take several iterations (a relative residual
        // above the gate); the warp then offers the guess to every element
        // whose start misses the tolerance, since its slowest lane sets the
        // warp's iteration count
        q.need = (f.guess == 1) && !q.wa_ok;
        q.big = q.need && q.ga > f.mlp_gate * (fabs(tau) + s * a * fabs(q.wa) + 1e-300);
    }
}

// Second half: the solve from the chosen start, the slip rate and the
// derivatives [dslip, dpsi, dsigma0]; ym is the network's output.
__device__ __forceinline__ void newton_post(const FricParams &f, int64_t e, double eta, double psi, const NPre &q,
                                            float ym, bool have_ym, double &dV, double &dpsi, double &dsig, int &iters, int &ok)
{
    iters = 0;
    ok = 1;
    dsig = 0.0;
    if (q.kind == 0) {
        dV = 0.0; dpsi = 0.0;
        return;
    }
    const double a = f.a[e], V0 = f.V0[e], Dc = f.Dc[e];
    double V;
    if (q.kind == 1) {
        // effective normal stress not compressive: no frictional strength,
        // the traction is balanced by radiation damping alone
        V = q.tau / eta;
    } else {
        double w = q.wa;
        if (q.need && have_ym) {
            // the learned guess is judged by the FP64 residual: Newton
            // starts from whichever of the two guesses fits better
            const double wm = q.wa + 10.0 * (double)ym;
            double ev1, d1;
            eta_v(wm, q.lnA, eta, ev1, d1);
            if (fabs(q.tau - ev1 - q.s * a * wm) < q.ga) w = wm;
        }
        if (f.guess == 2 && f.wlast[e] != 0.0) w = f.wlast[e];
        w = newton_w(q.tau, q.s, a, q.lnA, eta, w, f.tol, f.maxit, iters, ok);
        f.wlast[e] = w;
        V = v_of_w(w, q.lnA);
        // recorded: converged solves the analytic start does not settle,
        // the only ones that evaluate the network when it is deployed
        if (ok && !q.wa_ok && f.rec_cap > 0) {
            const unsigned long long r = atomicAdd(f.rec_n, 1ull);
            if ((long long)r < f.rec_cap) {
#pragma unroll
                for (int i = 0; i < MLP_IN; i++) f.rec_x[r * MLP_IN + i] = q.x[i];
                f.rec_t[r] = (float)((w - q.wa) / 10.0);
            }
        }
    }
    f.vnow[e] = V;
    dV = V;                                        // d slip / dt
    dpsi = V0 / Dc * exp(-psi) - fabs(V) / Dc;     // aging law, as the reference
}

__device__ __forceinline__ void rsf_rhs(const FricParams &f, int mode, int64_t e, double mu_2cs, double V, double psi,
                                        double sig, double T, double Nn, double Pt, double Pd, double &dV,
                                        double &dpsi, double &dsig)
{
    // src/friction/RateStateAgingModeII.f90:46-76 (mode III: dsig = loading only)
    dsig = (mode == 2) ? (Nn + f.nload[e]) : f.nload[e];
    const double a = f.a[e], b = f.b[e], V0 = f.V0[e], Dc = f.Dc[e];
    double B = V / (2.0 * V0);
    double C = exp((f.f0[e] + b * psi) / a);
    double D = 1.0 / (C * C) + B * B;
    D = 1.0 / sqrt(D);
    double heal = V0 / Dc * exp(-psi) - fabs(V) / Dc;
    double num = f.sload[e] + T + (dsig + Pd) * a * asinh(B * C) + B * D * (sig + Pt) * b * heal;
    double den = mu_2cs - D * (sig + Pt) * a / (2.0 * V0);
    dV = num / den;
    dpsi = heal;
    if (f.fake[e]) { dV = 0.0; dpsi = 0.0; dsig = 0.0; }
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *addr, double v)
{
    // non-negative doubles order like their bit patterns
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// stage: 0 = standalone evaluation (ytmp in, kbuf slot 0 out)
//        1 = k1 at the step start (y in), also yscal
//        2..5 = k_s, then ytemp of stage s+1 in place
//        6 = k6, then yout, yerr and the max-norm contribution
// sys: pressure system of this evaluation; mask: phases that take part.
// LEARNED: Newton formulation with the learned guess (a separate
// instantiation keeps the tensor-core inference's registers out of the
// other variants).
// Without the learned guess the kernel is held to 64 registers (8 blocks of
// 128 threads per SM, 136 bytes of spills to L1): it waits on memory, and
// the extra warps raise the tensor-core round by 5-6 % over 5 blocks at 84
// registers.
template <bool LEARNED>
__global__ void __launch_bounds__(128, LEARNED ? 5 : 8) friction_kernel(FricParams f, int stage, int sys, int mask)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int myi = -1;
    int nit = 0, nsolve = 0, nfail = 0;
    double emax = 0.0;
    if (e < f.Ntot) {
        const int i = f.inst_of[e];
        if (takes_part(f.ctl, i, mask)) myi = i;
    }
    // phase 1: stresses, stage state and pressure; for the Newton
    // formulation the analytic start and the network inputs
    double T = 0.0, Nn = 0.0, V = 0.0, psi = 0.0, sig = 0.0, Pt = 0.0, Pd = 0.0;
    NPre q;
    q.kind = 0;
    q.need = false;
    q.big = false;
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) q.x[i] = 0.0f;
    if (myi >= 0) {
        const Inst &I = f.inst[myi];
        const int64_t N = I.N, k = e - I.eoff;
        const StepCtl *ctl = f.ctl + myi;
        const double *pT = f.partT + I.poff + k;
        for (int64_t c = 0; c < I.nchunk; c++) T += pT[c * N];
        T = I.prefT * T;
        if (f.mode == 2) {
            const double *pN = f.partN + I.poff + k;
            for (int64_t c = 0; c < I.nchunk; c++) Nn += pN[c * N];
            Nn = I.prefT * Nn;
        }
        f.SigT[e] = T;
        f.SigN[e] = Nn;
        const double *yin = (stage == 1) ? f.y + 3 * I.eoff : f.ytmp + 3 * I.eoff;
        V = yin[k]; psi = yin[N + k]; sig = yin[2 * N + k];
        Pt = f.Ptemp[6 * I.eoff + (int64_t)sys * N + k];
        Pd = f.Pdot[6 * I.eoff + (int64_t)sys * N + k];
        if (f.form == 1 && stage >= 1) {
            // Newton formulation: the stress balance uses P itself, so the
            // stage pressure must be smooth in the stage time. It is linear
            // between the committed P (c = 0) and the implicit-Euler P over
            // the whole step (system 4, c = 1), which is what is committed.
            // (stage 1 takes P itself: the full-step system of this attempt
            // is not solved yet)
            const double p0 = f.Pc[I.eoff + k];
            Pt = (stage == 1) ? p0 : add_(p0, mul_(ck_a(stage), f.Ptemp[6 * I.eoff + 4 * N + k] - p0));
        }
        if (f.form == 1) {
            const double off = (stage == 0) ? f.off_explicit
                                            : (stage == 1 ? 0.0 : add_(ctl->x, mul_(ck_a(stage), ctl->h)));
            const double tt = (ctl->time - I.t0) + off;
            newton_pre(f, e, f.mode, I.mu_2cs, tt, psi, sig, T, Nn, Pt, q);
        }
    }
    // the learned guess: evaluated only by warps that hold an element whose
    // analytic start misses the tolerance by more than the gate; the
    // network's FP16 image is read from global memory (11 KB, L1-resident
    // after the first warp), so warps need no block barrier
    float ym = 0.0f;
    bool have_ym = false;
    if constexpr (LEARNED) {
        if (__any_sync(0xffffffffu, q.big)) {
            ym = mlp_warp_tc_call(f.mlp, q.x[0], q.x[1], q.x[2], q.x[3], q.x[4], q.x[5], q.x[6]);
            have_ym = true;
            if ((threadIdx.x & 31) == 0 && myi >= 0) atomicAdd((unsigned long long *)&f.ctl[myi].mlp_warps, 1ull);
        }
    }
    // phase 2: derivatives and the Cash-Karp stage arithmetic
    if (myi >= 0) {
        const Inst &I = f.inst[myi];
        const int64_t N = I.N, k = e - I.eoff, S = 3 * N;
        StepCtl *ctl = f.ctl + myi;
        const double *yi = f.y + 3 * I.eoff;
        double *yt = f.ytmp + 3 * I.eoff;
        double dV, dpsi, dsig;
        if (f.form == 1) {
            int ok = 1;
            newton_post(f, e, I.mu_2cs, psi, q, ym, have_ym, dV, dpsi, dsig, nit, ok);
            nsolve = f.fake[e] ? 0 : 1;
            nfail = ok ? 0 : 1;
        } else {
            rsf_rhs(f, f.mode, e, I.mu_2cs, V, psi, sig, T, Nn, Pt, Pd, dV, dpsi, dsig);
        }
        double *kb = f.kbuf + 18 * I.eoff;
        const int slot = (stage == 0) ? 0 : stage - 1;
        double *ks = kb + (int64_t)slot * S;
        ks[k] = dV; ks[N + k] = dpsi; ks[2 * N + k] = dsig;
        if (stage == 1) {
            const double tt = ctl->t_try, tol = ctl->eps;
            double *ysc = f.yscal + 3 * I.eoff;
            // yscal = abs(Y)+abs(Y_dot*t_try)+tol_solver (src/solver.f90:102)
            ysc[k] = add_(add_(fabs(yi[k]), fabs(mul_(dV, tt))), tol);
            ysc[N + k] = add_(add_(fabs(yi[N + k]), fabs(mul_(dpsi, tt))), tol);
            ysc[2 * N + k] = add_(add_(fabs(yi[2 * N + k]), fabs(mul_(dsig, tt))), tol);
        } else if (stage >= 2 && stage <= 5) {
            const double h = ctl->h;
#pragma unroll
            for (int j = 0; j < 3; j++) yt[j * N + k] = ck_combine(stage + 1, h, yi[j * N + k], kb, S, j * N + k);
        }
        if (f.form == 0 && stage >= 3) {
            // slip of the V formulation: k_s(slip) = V of the stage input,
            // 5th-order combination in the reference's operand order
            // (src/ode_solver/ode_bs.f90:223), outside the error norm
            if (stage == 3) f.slip_acc[e] = add_(mul_(CK_C1, yi[k]), mul_(CK_C3, V));
            else if (stage == 4) f.slip_acc[e] = add_(f.slip_acc[e], mul_(CK_C4, V));
            else if (stage == 6)
                f.slip_out[e] = add_(f.slip[e], mul_(ctl->h, add_(f.slip_acc[e], mul_(CK_C6, V))));
        }
        if (stage == 6) {
            const double h = ctl->h;
            const double *ysc = f.yscal + 3 * I.eoff;
            double *yo = f.yout + 3 * I.eoff;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int64_t q = j * N + k;
                const double k1 = kb[q], k3 = kb[2 * S + q], k4 = kb[3 * S + q], k5 = kb[4 * S + q],
                             k6 = kb[5 * S + q];
                // src/ode_solver/ode_bs.f90:223-224
                yo[q] = add_(yi[q], mul_(h, add_(add_(add_(mul_(CK_C1, k1), mul_(CK_C3, k3)), mul_(CK_C4, k4)),
                                                 mul_(CK_C6, k6))));
                double yerr = mul_(h, add_(add_(add_(add_(mul_(CK_DC1, k1), mul_(CK_DC3, k3)), mul_(CK_DC4, k4)),
                                                mul_(CK_DC5, k5)),
                                           mul_(CK_DC6, k6)));
                double er = fabs(__ddiv_rn(yerr, ysc[q]));
                if (!(er == er) || isinf(er)) er = 1.0e300;   // non-finite error rejects the attempt
                emax = fmax(emax, er);
            }
        }
        if (k == 0 && stage >= 1) atomicAdd((unsigned long long *)&ctl->rhs_evals, 1ull);
    }
    if (stage == 6) {
        // warp-level max when the warp lies in one instance, else per lane
        const unsigned full = 0xffffffffu;
        const int i0 = __shfl_sync(full, myi, 0);
        if (__all_sync(full, myi == i0)) {
            double w = emax;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_xor_sync(full, w, o));
            if ((threadIdx.x & 31) == 0 && i0 >= 0) atomic_max_pos(&f.ctl[i0].errmax_bits, w);
        } else if (myi >= 0) {
            atomic_max_pos(&f.ctl[myi].errmax_bits, emax);
        }
    }
    if (f.form == 1) {
        // Newton counters: warp sums when the warp lies in one instance
        const unsigned full = 0xffffffffu;
        const int i0 = __shfl_sync(full, myi, 0);
        if (__all_sync(full, myi == i0)) {
            int a = nit, b = nsolve, c = nfail;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a += __shfl_xor_sync(full, a, o);
                b += __shfl_xor_sync(full, b, o);
                c += __shfl_xor_sync(full, c, o);
            }
            if ((threadIdx.x & 31) == 0 && i0 >= 0) {
                atomicAdd((unsigned long long *)&f.ctl[i0].newton_iters, (unsigned long long)a);
                atomicAdd((unsigned long long *)&f.ctl[i0].newton_solves, (unsigned long long)b);
                if (c) atomicAdd((unsigned long long *)&f.ctl[i0].newton_fail, (unsigned long long)c);
            }
        } else if (myi >= 0) {
            atomicAdd((unsigned long long *)&f.ctl[myi].newton_iters, (unsigned long long)nit);
            atomicAdd((unsigned long long *)&f.ctl[myi].newton_solves, (unsigned long long)nsolve);
            if (nfail) atomicAdd((unsigned long long *)&f.ctl[myi].newton_fail, (unsigned long long)nfail);
        }
    }
}

// tau0 of the Newton formulation: the shear traction for which the initial
// V satisfies the friction law at slip 0; then the slip state is zeroed.
__global__ void newton_init_kernel(int64_t Ntot, const int *inst_of, const Inst *inst, const double *a,
                                   const double *b, const double *f0, const double *V0, const unsigned char *fake,
                                   const double *P, double *Y, double *tau0, double *wlast)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= Ntot) return;
    const Inst &I = inst[inst_of[e]];
    const int64_t N = I.N, k = e - I.eoff;
    double *y = Y + 3 * I.eoff;
    const double V = y[k], psi = y[N + k], sig = y[2 * N + k];
    double t0 = 0.0, w = 0.0;
    if (!fake[e]) {
        const double C = exp((f0[e] + b[e] * psi) / a[e]);
        w = asinh(V * C / (2.0 * V0[e]));
        t0 = I.mu_2cs * V - (sig + P[e]) * a[e] * w;
    }
    tau0[e] = t0;
    wlast[e] = w;
    y[k] = 0.0;
}

// Element-wise kernels over all instances; k == 0 of an instance also
// updates that instance's scalars.
struct ElemParams {
    int64_t Ntot;
    const Inst *inst;
    const int *inst_of;
    StepCtl *ctl;
};

// ytemp of stage 2 at the start of every attempt (h may have changed).
__global__ void attempt_begin_kernel(ElemParams ep, const double *y, const double *kbuf, double *ytmp, int mask)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ep.Ntot) return;
    const int i = ep.inst_of[e];
    if (!takes_part(ep.ctl, i, mask)) return;
    const Inst &I = ep.inst[i];
    const int64_t N = I.N, k = e - I.eoff;
    const double h = ep.ctl[i].h;
    const double *yi = y + 3 * I.eoff, *kb = kbuf + 18 * I.eoff;
    double *yt = ytmp + 3 * I.eoff;
#pragma unroll
    for (int j = 0; j < 3; j++) yt[j * N + k] = ck_combine(2, h, yi[j * N + k], kb, 3 * N, j * N + k);
    if (k == 0) {
        ep.ctl[i].errmax_bits = 0ull;
        ep.ctl[i].pfail_mask = 0;
        ep.ctl[i].attempts += 1;
    }
}

// Step control after an attempt, one thread per instance:
// src/ode_solver/ode_bs.f90:158-172.
__global__ void decide_kernel(StepCtl *ctl, int B, int mask)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B || !takes_part(ctl, i, mask)) return;
    StepCtl &c = ctl[i];
    const double SAFETY = 0.9, PGROW = -0.2, PSHRNK = -0.25;
    const double ERRCON = (double)1.89e-4f;  // default-real literal in the reference
    double errmax = __longlong_as_double((long long)c.errmax_bits) / c.eps;
    double h = c.h;
    c.step_attempts += 1;
    if (errmax <= 1.0) {
        c.accepted = 1;
        c.hnext = (errmax > ERRCON) ? SAFETY * h * pow(errmax, PGROW) : 5.0 * h;
        c.hdid = h;
    } else {
        c.accepted = 0;
        c.rejected += 1;
        double htemp = SAFETY * h * pow(errmax, PSHRNK);
        h = copysign(fmax(fabs(htemp), 0.1 * fabs(h)), h);
        c.h = h;
        if (c.x + h == c.x) atomicCAS(&c.status, 0, 2);
        else if (c.step_attempts >= c.max_attempts) atomicCAS(&c.status, 0, 8);
    }
}

// Start of one pass of solve() for instances beginning a step:
// src/solver.f90:60-77.
__global__ void step_begin_kernel(StepCtl *ctl, const Inst *inst, int B, const double *src_tb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B || ctl[i].phase != PH_NEW) return;
    StepCtl &c = ctl[i];
    c.it_count += 1;
    c.accepted = 0;
    c.probe_ier = 0;
    c.step_attempts = 0;
    c.commit_bad = 0;
    c.x = 0.0;
    if (c.t_try > 10.0) {
        const Inst &I = inst[i];
        for (int64_t s = 0; s < I.nsrc; s++) {
            const double tb = src_tb[I.soff + s];
            if (c.time < tb && c.time + c.t_try > tb) c.t_try = 10.0;
        }
    }
    // runs to a target time (dfn_solve_batch with t_end > 0; the reference
    // stops by step count only) land on it: the last step is shortened
    if (c.t_end > 0.0 && c.time + c.t_try > c.t_end) c.t_try = c.t_end - c.time;
}

__global__ void set_h_kernel(StepCtl *ctl, int B)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B || ctl[i].phase != PH_NEW) return;
    ctl[i].h = ctl[i].t_try;
}

// ---------------------------------------------------------------------------
// Permeability evolution (permeability_coupling = 1). k* is fixed from the
// initial state (src/initialisation.f90:256-261),
//   k* = kmin + (k - kmin) exp(|sigmaN + P| / |Snk|),
// and before every pressure solve the permeability and the face values
// follow the committed sigmaN and P (src/fluid_diffusion.f90:68-70, 74-75):
//   k = (k* - kmin) exp(-|sigmaN + P| / |Snk|) + kmin,
//   k_x(face j) = 2 k(j-1) k(j) / (k(j-1) + k(j)),  j = 1 .. N-1.
__device__ __forceinline__ double perm_coupled(double kstar, double kmin, double Snk, double sig, double P)
{
    return add_(mul_(kstar - kmin, exp(-(fabs(sig + P) / fabs(Snk)))), kmin);
}

__global__ void perm_init_kernel(ElemParams ep, const double *Y, const double *P, const double *perm,
                                 const double *kmin, const double *Snk, double *kstar)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ep.Ntot) return;
    const Inst &I = ep.inst[ep.inst_of[e]];
    const double sig = Y[3 * I.eoff + 2 * I.N + (e - I.eoff)];
    kstar[e] = add_(kmin[e], mul_(perm[e] - kmin[e], exp(fabs(sig + P[e]) / fabs(Snk[e]))));
}

// Networks in `mask` (with accepted_only, those whose attempt of this round
// was accepted: the state is the new one, P still the old).
__global__ void perm_update_kernel(ElemParams ep, int mask, int accepted_only, const double *Y, const double *P,
                                   const double *kstar, const double *kmin, const double *Snk, double *perm,
                                   double *permx)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ep.Ntot) return;
    const int i = ep.inst_of[e];
    if (!takes_part(ep.ctl, i, mask)) return;
    if (accepted_only && (!ep.ctl[i].accepted || ep.ctl[i].status != 0)) return;
    const Inst &I = ep.inst[i];
    const int64_t N = I.N, k = e - I.eoff;
    const double *sg = Y + 3 * I.eoff + 2 * N;
    const double pk = perm_coupled(kstar[e], kmin[e], Snk[e], sg[k], P[e]);
    perm[e] = pk;
    if (k >= 1) {
        const double pl = perm_coupled(kstar[e - 1], kmin[e - 1], Snk[e - 1], sg[k - 1], P[e - 1]);
        permx[I.eoff + i + k] = __ddiv_rn(mul_(mul_(2.0, pl), pk), add_(pl, pk));
    }
}

// The commit of the coupled pressure: P of the commit solve (system slot 5,
// dt = hdid) where it converged.
__global__ void commit_p_kernel(ElemParams ep, double *P, double *Pdot, const double *Ptemp, const double *Pdot_s)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ep.Ntot) return;
    const int i = ep.inst_of[e];
    const StepCtl &c = ep.ctl[i];
    if (!takes_part(ep.ctl, i, M_ACTIVE) || !c.accepted || c.status != 0 || (c.pfail_mask & (1 << 6))) return;
    const Inst &I = ep.inst[i];
    const int64_t N = I.N, k = e - I.eoff;
    P[e] = Ptemp[6 * I.eoff + 5 * N + k];
    Pdot[e] = Pdot_s[6 * I.eoff + 5 * N + k];
}

// Accepted attempts: Y = yout, and the pressure commit compute_P(t_did),
// which equals the stage-5 solve of the accepted attempt (dt = 0 + 1.0*h).
// The whole state is committed before the stop rules look at it, as the
// reference commits Y, P and time before check_errors (src/solver.f90:
// 170-197): an extensional or non-finite component only raises a flag here,
// which finish_kernel turns into the status after the time update.
__global__ void commit_kernel(ElemParams ep, double *y, const double *yout, double *P, double *Pdot,
                              const double *Ptemp, const double *Pdot_s, double *slip, const double *slip_out,
                              int commit_p)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ep.Ntot) return;
    const int i = ep.inst_of[e];
    const StepCtl &c = ep.ctl[i];
    if (!takes_part(ep.ctl, i, M_ACTIVE) || !c.accepted || c.status != 0) return;
    const Inst &I = ep.inst[i];
    const int64_t N = I.N, k = e - I.eoff;
    double *yi = y + 3 * I.eoff;
    const double *yo = yout + 3 * I.eoff;
    int bad = 0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const double v = yo[j * N + k];
        yi[j * N + k] = v;
        if (j == 2 && v > 0.0) bad |= 1;
        if (!isfinite(v)) bad |= 2;
    }
    if (bad) atomicOr(&ep.ctl[i].commit_bad, bad);
    if (slip) slip[e] = slip_out[e];
    if (commit_p && !(c.pfail_mask & (1 << 4))) {
        P[e] = Ptemp[6 * I.eoff + 4 * N + k];
        Pdot[e] = Pdot_s[6 * I.eoff + 4 * N + k];
    }
}

// End of one pass of solve() per instance (src/solver.f90:117-196): time,
// t_try with the 1-day cap, the stop rules on the committed state
// (check_errors, src/solver.f90:412-418; non-finite values too) and the
// instance's next phase.
__global__ void finish_kernel(StepCtl *ctl, int B, double t_cap)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B || !takes_part(ctl, i, M_ACTIVE)) return;
    StepCtl &c = ctl[i];
    if (c.status != 0) { c.phase = PH_DONE; return; }
    if (!c.accepted) { c.phase = PH_RETRY; return; }
    c.time = c.time + c.hdid;
    double tn = c.hnext;
    if (tn > t_cap) tn = t_cap;
    c.t_try = tn;
    c.steps_done += 1;
    if (c.commit_bad) {
        c.status = (c.commit_bad & 1) ? 3 : 4;
        c.phase = PH_DONE;
        return;
    }
    bool done = (c.steps_done >= c.target_steps) || (c.t_end > 0.0 && c.time >= c.t_end * (1.0 - 1e-14));
    c.phase = done ? PH_DONE : PH_NEW;
}

// Arms every instance for `nsteps` more accepted steps (or until t_end).
__global__ void arm_kernel(StepCtl *ctl, int B, long long nsteps, double t_end, int max_attempts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    StepCtl &c = ctl[i];
    c.steps_done = 0;
    c.target_steps = nsteps;
    c.t_end = t_end;
    c.max_attempts = max_attempts;
    c.phase = (c.status == 0 && nsteps > 0 && !(t_end > 0.0 && c.time >= t_end)) ? PH_NEW : PH_DONE;
}

// K.V output for the operator entry point: sum the chunks and scale.
__global__ void kv_finish_kernel(int64_t N, int mode, int nchunk, double pref, const double *partT,
                                 const double *partN, double *sT, double *sN)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= N) return;
    double T = 0.0, Nn = 0.0;
    for (int c = 0; c < nchunk; c++) T += partT[(int64_t)c * N + k];
    sT[k] = pref * T;
    if (sN) {
        if (mode == 2) {
            for (int c = 0; c < nchunk; c++) Nn += partN[(int64_t)c * N + k];
            sN[k] = pref * Nn;
        } else {
            sN[k] = 0.0;
        }
    }
}
