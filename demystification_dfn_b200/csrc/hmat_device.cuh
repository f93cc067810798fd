// hmat_device.cuh — H-matrix K.V on the GPU (replaces Hgemv_right,
// src/hmatrix/calculation_hmat.f90:3-165, and the permutations of
// hmatII/hmatIII, src/kernel_calculation/hmatrixModeII.f90:46-69).
//
// The reference recurses over the block tree and calls ZGEMV on each leaf
// with complex(8) storage (16 bytes per real entry). Here the leaves are a
// flat list and every K.V is five launches over task lists:
//   0. xp = x in cluster order (one gather, so that the leaf kernels read
//      their columns contiguously);
//   1. z_b = B_b^T xp for every low-rank block b, split in column chunks
//      (partial sums per chunk, added in fixed order in step 2);
//   2. the rows: F xp over the dense leaves of a row cluster (one output
//      slot per (group, row)) and A_b z_b of the low-rank leaves (one output
//      slot per (leaf, row));
//   3. y(row) = sum of the row's slots in a fixed order, written in the
//      original element order (y[perm[pos]]).
// Small whole low-rank leaves go one warp each, larger ones one CTA each,
// those wider than HM_COLS columns through split z partials and row tasks.
// Factors are stored in FP64 or FP32 with rows padded to whole 16-byte
// vectors and 16-byte aligned: dense F row-major (nr x ldf), low-rank A and
// B transposed, rank-major (r x lda, r x ldb), so that every factor streams
// as coalesced 16-byte loads. Sums are FP64. Every launch is predicated on
// the network's phase like the dense K.V, and covers all networks of a batch.
#pragma once
#include "dfn_device.cuh"
#include "hmat_build.h"

struct HBlk {
    int inst, comp, dense, rank;
    int r0, nr, c0, nc;        // positions in cluster order (within the network)
    int64_t foff;              // dense: F offset; low-rank: A^T offset (values)
    int64_t goff;              // low-rank: B^T offset (values)
    int64_t zoff;              // low-rank: first z partial (ntask1 x rank doubles)
    int64_t outoff;            // first output slot of the leaf's rows
    int ntask1;                // column chunks of the low-rank product
    int ld;                    // padded row length: dense F, or low-rank B^T
    int lda;                   // low-rank A^T padded row length
    int pad;
};

struct HTask { int blk, start, count, chunk; };

constexpr int HM_COLS = 1024;  // columns per step-1 task
constexpr int HM_ROWS = 64;    // rows per step-2 task of a dense leaf
constexpr int HM_LROWS = 1024; // rows per step-2 task of a low-rank leaf (a 16-byte vector per thread)
constexpr int HM_XPAD = 8;     // zero doubles after xp (padded columns read them)

template <typename T> struct HVec;
template <> struct HVec<float> {
    using V = float4;
    static constexpr int W = 4;
    __device__ static void unpack(const float4 &v, double *o) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
};
template <> struct HVec<double> {
    using V = double2;
    static constexpr int W = 2;
    __device__ static void unpack(const double2 &v, double *o) { o[0] = v.x; o[1] = v.y; }
};

// xp[eoff + pos] = x of network i at its element perm[pos]
__global__ void hm_permute_kernel(int64_t Ntot, const int *__restrict__ inst_of, const Inst *__restrict__ inst,
                                  const StepCtl *__restrict__ ctl, int mask, const int *__restrict__ perm,
                                  const double *__restrict__ Vbase, int vmul, double *__restrict__ xp)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= Ntot) return;
    const int i = inst_of[e];
    if (!takes_part(ctl, i, mask)) return;
    const Inst &I = inst[i];
    xp[e] = Vbase[(int64_t)vmul * I.eoff + perm[e]];
}

// z partial of one column chunk: the chunk's x staged once in shared memory;
// warp w takes rank rows q = w, w+8, ... two at a time (independent sums, so
// their loads overlap); lanes stream a row's columns in 16-byte vectors.
template <typename T>
__global__ void __launch_bounds__(256) hm_lowrank_kernel(const HTask *__restrict__ tasks, const HBlk *__restrict__ blks,
                                                         const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                                                         int mask, const T *__restrict__ vals,
                                                         const double *__restrict__ xp, double *__restrict__ zpart)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    __shared__ __align__(16) double xs[HM_COLS + HM_XPAD];
    const HTask t = tasks[blockIdx.x];
    const HBlk b = blks[t.blk];
    if (!takes_part(ctl, b.inst, mask)) return;   // CTA-uniform: before the barrier
    const Inst &I = inst[b.inst];
    const double *x = xp + I.eoff + b.c0 + t.start;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nv = (t.count + W - 1) / W;    // vectors of the chunk (padding columns are zero)
    for (int j = threadIdx.x; j < nv * W; j += blockDim.x) xs[j] = x[j];
    __syncthreads();
    for (int q = w; q < b.rank; q += 16) {
        const bool two = q + 8 < b.rank;
        const VT *row0 = reinterpret_cast<const VT *>(vals + b.goff + (int64_t)q * b.ld + t.start);
        const VT *row1 = reinterpret_cast<const VT *>(vals + b.goff + (int64_t)(two ? q + 8 : q) * b.ld + t.start);
        double s0 = 0.0, s1 = 0.0;
        for (int v = lane; v < nv; v += 32) {
            double f0[W], f1[W];
            HVec<T>::unpack(row0[v], f0);
            HVec<T>::unpack(row1[v], f1);
#pragma unroll
            for (int j = 0; j < W; j++) {
                const double xv = xs[v * W + j];
                s0 = fma(f0[j], xv, s0);
                s1 = fma(f1[j], xv, s1);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        }
        if (lane == 0) {
            zpart[b.zoff + (int64_t)t.chunk * b.rank + q] = s0;
            if (two) zpart[b.zoff + (int64_t)t.chunk * b.rank + q + 8] = s1;
        }
    }
}

// Rows of dense leaves. The dense leaves that share a row cluster form a
// group; one CTA takes up to HM_ROWS rows of a group and walks all of its
// leaves, so one accumulator per row sums the row over every dense leaf of
// the group (one output slot per row of the group, not per leaf) and each
// task streams the group's bytes behind one chain of dependent loads
// (task, group, network phase). A half-warp per row, 16-byte vectors of F
// against xp, four rows per half-warp in flight; each row summed over the
// group's leaves in order, each leaf's vectors by lane, then a fixed
// half-warp tree.
struct HDLeaf {
    int64_t foff;   // values of F (row-major, rows of ld values)
    int64_t xoff;   // xp index of the leaf's first column
    int ld, nv;     // padded row length, 16-byte vectors covering the columns
};
struct HDGroup {
    int64_t outoff;            // output slot of the group's first row
    int first, count, inst, pad;   // its leaves dl[first .. first + count), network
};

template <typename T>
__device__ __forceinline__ void hm_dense_task(const HTask t, const HDGroup *__restrict__ groups,
                                              const HDLeaf *__restrict__ dl, const StepCtl *__restrict__ ctl,
                                              int mask, const T *__restrict__ vals, const double *__restrict__ xp,
                                              double *__restrict__ out)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    constexpr int U = 4;
    const HDGroup g = groups[t.blk];
    if (!takes_part(ctl, g.inst, mask)) return;
    const int hl = threadIdx.x & 15, w = threadIdx.x >> 5, half = (threadIdx.x >> 4) & 1;
    const VT zero{};
    // the loop runs the same trips in both half-warps (shuffles below)
    for (int wb = w * 2 * U; wb < t.count; wb += 8 * 2 * U) {
        const int i0 = wb + half * U;
        double s[U];
#pragma unroll
        for (int u = 0; u < U; u++) s[u] = 0.0;
        for (int j = 0; j < g.count; j++) {
            const HDLeaf L = dl[g.first + j];
            const double *x = xp + L.xoff;
            for (int v = hl; v < L.nv; v += 16) {
                double xv[W];
#pragma unroll
                for (int q = 0; q < W; q++) xv[q] = x[v * W + q];
                VT fv[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int row = t.start + i0 + u;
                    fv[u] = (i0 + u < t.count) ? reinterpret_cast<const VT *>(vals + L.foff + (int64_t)row * L.ld)[v]
                                               : zero;
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    double a[W];
                    HVec<T>::unpack(fv[u], a);
#pragma unroll
                    for (int q = 0; q < W; q++) s[u] = fma(a[q], xv[q], s[u]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], o);
            if (hl == 0 && i0 + u < t.count) out[g.outoff + t.start + i0 + u] = s[u];
        }
    }
}

// one CTA per task
template <typename T>
__global__ void __launch_bounds__(256, 5) hm_dense_kernel(const HTask *__restrict__ tasks,
                                                          const HDGroup *__restrict__ groups,
                                                          const HDLeaf *__restrict__ dl,
                                                          const StepCtl *__restrict__ ctl, int mask,
                                                          const T *__restrict__ vals, const double *__restrict__ xp,
                                                          double *__restrict__ out)
{
    hm_dense_task<T>(tasks[blockIdx.x], groups, dl, ctl, mask, vals, xp, out);
}

// The same rows on a persistent grid: CTA c takes tasks c, c + gridDim.x,
// ... (each row's arithmetic is that of hm_dense_kernel).
template <typename T>
__global__ void __launch_bounds__(256, 5) hm_dense_persistent_kernel(const HTask *__restrict__ tasks, int64_t ntasks,
                                                                     const HDGroup *__restrict__ groups,
                                                                     const HDLeaf *__restrict__ dl,
                                                                     const StepCtl *__restrict__ ctl, int mask,
                                                                     const T *__restrict__ vals,
                                                                     const double *__restrict__ xp,
                                                                     double *__restrict__ out)
{
    for (int64_t tk = blockIdx.x; tk < ntasks; tk += gridDim.x)
        hm_dense_task<T>(tasks[tk], groups, dl, ctl, mask, vals, xp, out);
}

// Low-rank leaves of at most HM_COLS columns, whole: x staged in shared
// memory, z = B^T xp into shared memory (warp per rank row, two rows at a
// time), then the rows y = A z (a 16-byte vector of A rows per thread, the
// rank rows split over groups of threads when the leaf has fewer than 1024
// rows); one CTA per leaf, no partial sums in global memory.
template <typename T>
__global__ void __launch_bounds__(256) hm_lowrank_fused_kernel(const int *__restrict__ leaves,
                                                               const HBlk *__restrict__ blks,
                                                               const Inst *__restrict__ inst,
                                                               const StepCtl *__restrict__ ctl, int mask,
                                                               const T *__restrict__ vals,
                                                               const double *__restrict__ xp, double *__restrict__ out)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    __shared__ double z[hmat::kMaxRank];
    __shared__ __align__(16) double xs[HM_COLS + HM_XPAD];
    const HBlk b = blks[leaves[blockIdx.x]];
    if (!takes_part(ctl, b.inst, mask)) return;   // CTA-uniform: before the barriers
    const Inst &I = inst[b.inst];
    const double *x = xp + I.eoff + b.c0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nv = (b.nc + W - 1) / W;
    for (int j = threadIdx.x; j < nv * W; j += blockDim.x) xs[j] = x[j];
    __syncthreads();
    for (int q = w; q < b.rank; q += 16) {
        const bool two = q + 8 < b.rank;
        const VT *row0 = reinterpret_cast<const VT *>(vals + b.goff + (int64_t)q * b.ld);
        const VT *row1 = reinterpret_cast<const VT *>(vals + b.goff + (int64_t)(two ? q + 8 : q) * b.ld);
        double s0 = 0.0, s1 = 0.0;
        for (int v = lane; v < nv; v += 32) {
            double f0[W], f1[W];
            HVec<T>::unpack(row0[v], f0);
            HVec<T>::unpack(row1[v], f1);
#pragma unroll
            for (int j = 0; j < W; j++) {
                const double xv = xs[v * W + j];
                s0 = fma(f0[j], xv, s0);
                s1 = fma(f1[j], xv, s1);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        }
        if (lane == 0) {
            z[q] = s0;
            if (two) z[q + 8] = s1;
        }
    }
    __syncthreads();
    // y = A z: nav2 threads (a power of two, at most 256) over the vectors
    // of leaf rows, 256 / nav2 groups of them over the rank rows (group g
    // takes rows g, g + 256 / nav2, ... in order); the groups' sums added in
    // group order through shared memory (xs, no longer needed). Leaves of
    // 1024 rows or more keep one group.
    const int nav = (b.nr + W - 1) / W, avl = b.lda / W;
    const VT *Av = reinterpret_cast<const VT *>(vals + b.foff);
    const int lgv = nav >= 256 ? 8 : 32 - __clz(nav - 1);
    const int nav2 = 1 << lgv, hq = 256 >> lgv;   // 256 threads
    const int v0 = threadIdx.x & (nav2 - 1), qg = threadIdx.x >> lgv;
    double *red = xs;   // 256 x W doubles at most
    for (int rb = 0; rb < nav; rb += nav2) {   // the same trips in every thread (barriers)
        const int iv = rb + v0;
        double acc[W];
#pragma unroll
        for (int c = 0; c < W; c++) acc[c] = 0.0;
        if (iv < nav) {
#pragma unroll 4
            for (int q = qg; q < b.rank; q += hq) {
                double a[W];
                HVec<T>::unpack(Av[(int64_t)q * avl + iv], a);
                const double zq = z[q];
#pragma unroll
                for (int c = 0; c < W; c++) acc[c] = fma(a[c], zq, acc[c]);
            }
        }
        if (hq > 1) {   // CTA-uniform
#pragma unroll
            for (int c = 0; c < W; c++) red[(qg * nav2 + v0) * W + c] = acc[c];
            __syncthreads();
            if (qg == 0)
                for (int g = 1; g < hq; g++)
#pragma unroll
                    for (int c = 0; c < W; c++) acc[c] += red[(g * nav2 + v0) * W + c];
            __syncthreads();
        }
        if (qg == 0 && iv < nav) {
#pragma unroll
            for (int c = 0; c < W; c++)
                if (iv * W + c < b.nr) out[b.outoff + iv * W + c] = acc[c];
        }
    }
}

// Small low-rank leaves, one warp each (four per 128-thread CTA), from a
// compact descriptor list (one load per leaf before its factors): z = B^T xp
// with lanes in groups of the B^T row's vector count (several rank rows per
// pass when the rows are short; the lane's x vectors held in registers),
// then y = A z with a 16-byte vector of A rows per lane (rows summed over
// the rank in order, as in hm_lowrank_fused_kernel), written to the leaf's
// output slots. Leaves qualify when their factors take at most
// HM_WARP_LEAF_BYTES and their B^T rows at most 32 * HM_WARP_XV vectors.
// These leaves are a few KB each and latency-bound: a SM holds the loads of
// dozens of them in flight, against 8 with one CTA per leaf. The kernel is
// held to 40 registers (12 CTAs of four warps per SM, a few spills to L1)
// and the dense-row kernel to 48 (five CTAs of 256): K.V 0.840 -> 0.823 ms
// at N = 81 750 (8 CTAs and 64 registers each before).
constexpr int HM_WARP_LEAF_BYTES = 32 * 1024;
constexpr int HM_WARP_XV = 2;

struct HLeafW {
    int64_t aoff;     // A^T offset (values); B^T follows at aoff + rank * lda
    int64_t xoff;     // first column of the leaf in xp
    int64_t outoff;   // first output slot of the leaf's rows
    int inst, rank, lda, ld, nr, blk;
};

// y = A z of a small leaf by one warp: nav2 lanes (a power of two, at most
// 32) over the vectors of leaf rows, 32 / nav2 groups of them over the rank
// rows (group g takes rows g, g + 32 / nav2, ... in order), the groups
// added by a fixed butterfly. Leaves of 128 rows or more keep one group
// (each lane sums all rank rows of its vectors in order).
template <typename T>
__device__ __forceinline__ void hm_warp_az(const HLeafW &d, const T *__restrict__ A, const double *z,
                                           double *__restrict__ out, int lane)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    const int nav = (d.nr + W - 1) / W;   // vectors of an A row (padding rows are zero)
    const int avl = d.lda / W;
    const VT *Av = reinterpret_cast<const VT *>(A);
    const int lgv = nav >= 32 ? 5 : 32 - __clz(nav - 1);
    const int nav2 = 1 << lgv, hq = 32 >> lgv;
    const int v0 = lane & (nav2 - 1), qg = lane >> lgv;
    for (int rb = 0; rb < nav; rb += nav2) {   // the same trips in every lane (shuffles)
        const int rv = rb + v0;
        double acc[W];
#pragma unroll
        for (int c = 0; c < W; c++) acc[c] = 0.0;
        if (rv < nav) {
#pragma unroll 4
            for (int q = qg; q < d.rank; q += hq) {
                double a[W];
                HVec<T>::unpack(Av[(int64_t)q * avl + rv], a);
                const double zq = z[q];
#pragma unroll
                for (int c = 0; c < W; c++) acc[c] = fma(a[c], zq, acc[c]);
            }
        }
        for (int o = nav2; o < 32; o <<= 1)
#pragma unroll
            for (int c = 0; c < W; c++) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
        if (qg == 0 && rv < nav) {
#pragma unroll
            for (int c = 0; c < W; c++)
                if (rv * W + c < d.nr) out[d.outoff + rv * W + c] = acc[c];
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(128, 12) hm_lowrank_warp_kernel(const HLeafW *__restrict__ leaves, int64_t n,
                                                                  const StepCtl *__restrict__ ctl, int mask,
                                                                  const T *__restrict__ vals,
                                                                  const double *__restrict__ xp,
                                                                  double *__restrict__ out)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    __shared__ double zs[4][hmat::kMaxRank];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t k = (int64_t)blockIdx.x * 4 + warp;
    if (k >= n) return;   // warp-uniform; the kernel has no block barrier
    const HLeafW d = leaves[k];
    if (!takes_part(ctl, d.inst, mask)) return;
    const int rank = d.rank, nv = d.ld / W;
    int g = 1;
    while (g < nv && g < 32) g <<= 1;
    const int sub = lane / g, v0 = lane % g, rp = 32 / g;
    double xv[HM_WARP_XV][W];
#pragma unroll
    for (int m = 0; m < HM_WARP_XV; m++) {
        const int v = v0 + m * g;
#pragma unroll
        for (int c = 0; c < W; c++) xv[m][c] = (v < nv) ? __ldg(xp + d.xoff + v * W + c) : 0.0;
    }
    const T *A = vals + d.aoff;
    const VT *Bt = reinterpret_cast<const VT *>(A + (int64_t)rank * d.lda);
    double *z = zs[warp];
#pragma unroll 4
    for (int q0 = 0; q0 < rank; q0 += rp) {
        const int q = q0 + sub;
        double acc = 0.0;
        if (q < rank) {
#pragma unroll
            for (int m = 0; m < HM_WARP_XV; m++) {
                const int v = v0 + m * g;
                if (v < nv) {
                    double f[W];
                    HVec<T>::unpack(Bt[(int64_t)q * nv + v], f);
#pragma unroll
                    for (int c = 0; c < W; c++) acc = fma(f[c], xv[m][c], acc);
                }
            }
        }
        for (int o = g >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (v0 == 0 && q < rank) z[q] = acc;
    }
    __syncwarp();
    hm_warp_az<T>(d, A, z, out, lane);
}

template <typename T>
__device__ __forceinline__ void hm_lowrank_warp_leaf(const HLeafW &d, const T *__restrict__ vals,
                                                     const double *__restrict__ xp, double *__restrict__ out,
                                                     double *z)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    const int lane = threadIdx.x & 31;
    const int rank = d.rank, nv = d.ld / W;
    int g = 1;
    while (g < nv && g < 32) g <<= 1;
    const int sub = lane / g, v0 = lane % g, rp = 32 / g;
    double xv[HM_WARP_XV][W];
#pragma unroll
    for (int m = 0; m < HM_WARP_XV; m++) {
        const int v = v0 + m * g;
#pragma unroll
        for (int c = 0; c < W; c++) xv[m][c] = (v < nv) ? __ldg(xp + d.xoff + v * W + c) : 0.0;
    }
    const T *A = vals + d.aoff;
    const VT *Bt = reinterpret_cast<const VT *>(A + (int64_t)rank * d.lda);
#pragma unroll 4
    for (int q0 = 0; q0 < rank; q0 += rp) {
        const int q = q0 + sub;
        double acc = 0.0;
        if (q < rank) {
#pragma unroll
            for (int m = 0; m < HM_WARP_XV; m++) {
                const int v = v0 + m * g;
                if (v < nv) {
                    double f[W];
                    HVec<T>::unpack(Bt[(int64_t)q * nv + v], f);
#pragma unroll
                    for (int c = 0; c < W; c++) acc = fma(f[c], xv[m][c], acc);
                }
            }
        }
        for (int o = g >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (v0 == 0 && q < rank) z[q] = acc;
    }
    __syncwarp();
    hm_warp_az<T>(d, A, z, out, lane);
    __syncwarp();   // z is rewritten by the warp's next leaf
}

// The same leaves on a persistent grid: warp w of CTA c takes leaves
// 4c + w, 4c + w + 4 gridDim.x, ... (each leaf's arithmetic is that of
// hm_lowrank_warp_kernel).
template <typename T>
__global__ void __launch_bounds__(128, 12) hm_lowrank_warp_persistent_kernel(const HLeafW *__restrict__ leaves, int64_t n,
                                                                  const StepCtl *__restrict__ ctl, int mask,
                                                                  const T *__restrict__ vals,
                                                                  const double *__restrict__ xp,
                                                                  double *__restrict__ out)
{
    __shared__ double zs[4][hmat::kMaxRank];
    const int warp = threadIdx.x >> 5;
    for (int64_t k = (int64_t)blockIdx.x * 4 + warp; k < n; k += (int64_t)gridDim.x * 4) {
        const HLeafW d = leaves[k];
        if (!takes_part(ctl, d.inst, mask)) continue;   // warp-uniform; the kernel has no block barrier
        hm_lowrank_warp_leaf<T>(d, vals, xp, out, zs[warp]);
    }
}

// Rows of low-rank leaves: a 16-byte vector of A rows per thread (rows of a
// task start at a multiple of HM_LROWS), each row the sum over the rank of
// A^T[q][row] z[q] in order.
template <typename T>
__global__ void __launch_bounds__(256) hm_rows_kernel(const HTask *__restrict__ tasks, const HBlk *__restrict__ blks,
                                                      const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                                                      int mask, const T *__restrict__ vals,
                                                      const double *__restrict__ zpart, double *__restrict__ out)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    __shared__ double z[hmat::kMaxRank];
    const HTask t = tasks[blockIdx.x];
    const HBlk b = blks[t.blk];
    if (!takes_part(ctl, b.inst, mask)) return;
    const int r = b.rank;
    if (threadIdx.x < r) {
        double s = 0.0;
        for (int j = 0; j < b.ntask1; j++) s += zpart[b.zoff + (int64_t)j * r + threadIdx.x];
        z[threadIdx.x] = s;
    }
    __syncthreads();
    const int nav = (t.count + W - 1) / W, avl = b.lda / W, v0 = t.start / W;
    const VT *Av = reinterpret_cast<const VT *>(vals + b.foff);
    for (int iv = threadIdx.x; iv < nav; iv += blockDim.x) {
        double acc[W];
#pragma unroll
        for (int c = 0; c < W; c++) acc[c] = 0.0;
#pragma unroll 8
        for (int q = 0; q < r; q++) {
            double a[W];
            HVec<T>::unpack(Av[(int64_t)q * avl + v0 + iv], a);
            const double zq = z[q];
#pragma unroll
            for (int c = 0; c < W; c++) acc[c] = fma(a[c], zq, acc[c]);
        }
#pragma unroll
        for (int c = 0; c < W; c++)
            if (iv * W + c < t.count) out[b.outoff + t.start + iv * W + c] = acc[c];
    }
}

// Setup: the entries of the dense leaves, evaluated on the device (the same
// formulas as the dense assembly), rows [start, start+count) of a task.
template <typename T>
__global__ void __launch_bounds__(256) hm_fill_dense_kernel(const HTask *__restrict__ tasks,
                                                            const HBlk *__restrict__ blks,
                                                            const Inst *__restrict__ inst, int mode,
                                                            const int *__restrict__ perm,
                                                            const double *__restrict__ node,
                                                            const double *__restrict__ elem,
                                                            const double *__restrict__ tan,
                                                            const double *__restrict__ nrm, T *__restrict__ vals)
{
    const HTask t = tasks[blockIdx.x];
    const HBlk b = blks[t.blk];
    const Inst &I = inst[b.inst];
    const int64_t e0 = I.eoff;
    const double *E = elem + 2 * e0, *Tn = tan + 2 * e0, *R = nrm + 2 * e0, *D = node + 2 * (e0 + b.inst);
    const int *pm = perm + e0;
    const int64_t n = (int64_t)t.count * b.nc;
    for (int64_t q = threadIdx.x; q < n; q += blockDim.x) {
        const int i = t.start + (int)(q / b.nc), j = (int)(q % b.nc);
        const int64_t k = pm[b.r0 + i], l = pm[b.c0 + j];
        double v;
        if (mode == 3) {
            v = entry_mode3(E[2 * k], E[2 * k + 1], Tn[2 * k], Tn[2 * k + 1], D[2 * l], D[2 * l + 1], D[2 * l + 2],
                            D[2 * l + 3]);
        } else {
            double kt, kn;
            entry_mode2(E[2 * k], E[2 * k + 1], R[2 * k], R[2 * k + 1], D[2 * l], D[2 * l + 1], D[2 * l + 2],
                        D[2 * l + 3], R[2 * l], R[2 * l + 1], kt, kn);
            v = b.comp == 0 ? kt : kn;
        }
        vals[b.foff + (int64_t)i * b.ld + j] = (T)v;
    }
}

// ---------------------------------------------------------------------------
// Low-rank leaves built on the device: one 128-thread CTA per admissible
// leaf runs the partial-pivot ACA (the reference's unused `ACA` routine,
// src/hmatrix/ACA_algorithm.f90:12-260, with the relative Frobenius stopping
// rule of its full-pivot ACA) and the recompression of
// src/hmatrix/H_matrix_recompression.f90:145-301 (QR of both factors, SVD of
// R_A R_B^T, truncation), in these steps:
//   partial-pivot ACA: residual row at the pivot row, pivot column = the
//     largest unused |entry| (lowest index on ties), scaled row into B, the
//     residual column into A, ||S_k||_F^2 updated by 2 sum_q (a_q.a_k)(b_q.b_k)
//     + |a_k|^2 |b_k|^2, stop at |a_k||b_k| <= eps ||S_k||_F, next pivot row
//     = the largest unused |a_k(i)|; -1 beyond HM_KMAX terms (stored dense);
//   recompression (when 0 < k < min(m, n) and k <= HM_KSVD; blocks of more
//     terms keep their ACA factors): Householder QR of A and B in
//     place (reflectors below the diagonal, R above it, R's diagonal and the
//     reflector scales in shared memory), one-sided Jacobi SVD of
//     R_A R_B^T (k x k, shared memory; rotations of a sweep in parallel
//     rounds of disjoint column pairs), truncation at the first singular
//     value <= eps * sigma_1 (kept), A' = Q_A U_r S_r and B' = Q_B W_r formed
//     by applying the reflectors to [U_r S_r; 0] and [W_r; 0].
// Results: rank[b] (-1 dense, 0 zero block) and the factors A' (m x r) and
// B' (n x r), column-major by rank, in the leaf's X regions of the scratch.
// Sums are block reductions in a fixed order (deterministic).
#define HM_KMAX 128   // ACA terms at most
#define HM_KSVD 64    // recompression up to this rank (its k x k matrices in shared memory)
#define HM_BT 128

struct AcaLeaf {
    int r0, c0, nr, nc;
    int64_t soff;     // scratch doubles: A, B, XA, XB (nr, nc, nr, nc x HM_KMAX)
    int64_t foff;     // char flags: nr row flags, nc column flags
};

// Dynamic shared memory of hm_aca_kernel: G/U and W (HM_KSVD^2 each), five
// HM_KSVD arrays, three HM_KMAX arrays and 64 doubles of reductions.
constexpr size_t hm_aca_smem_bytes()
{
    return (size_t)(2 * HM_KSVD * HM_KSVD + 5 * HM_KSVD + 3 * HM_KMAX + 64) * sizeof(double);
}

__device__ __forceinline__ double hm_block_sum(double v, double *red)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < HM_BT / 32; q++) t += red[q];
    return t;
}

// max |v| over the CTA with the lowest index on ties (idx -1: none > 0)
__device__ __forceinline__ void hm_block_argmax(double v, int idx, double *redv, int *redi, double &best, int &bi)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi >= 0 && (idx < 0 || oi < idx))) { v = ov; idx = oi; }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) { redv[w] = v; redi[w] = idx; }
    __syncthreads();
    best = redv[0];
    bi = redi[0];
#pragma unroll
    for (int q = 1; q < HM_BT / 32; q++)
        if (redv[q] > best || (redv[q] == best && redi[q] >= 0 && (bi < 0 || redi[q] < bi))) { best = redv[q]; bi = redi[q]; }
}

struct AcaGeom {
    int mode, comp;
    const int *perm;                                  // cluster order of the network
    const double *E, *T, *R, *D;                      // midpoints, tangents, normals, nodes of the network
};

__device__ __forceinline__ double aca_entry(const AcaGeom &g, int64_t k, int64_t l)
{
    if (g.mode == 3)
        return entry_mode3(g.E[2 * k], g.E[2 * k + 1], g.T[2 * k], g.T[2 * k + 1], g.D[2 * l], g.D[2 * l + 1],
                           g.D[2 * l + 2], g.D[2 * l + 3]);
    double kt, kn;
    entry_mode2(g.E[2 * k], g.E[2 * k + 1], g.R[2 * k], g.R[2 * k + 1], g.D[2 * l], g.D[2 * l + 1], g.D[2 * l + 2],
                g.D[2 * l + 3], g.R[2 * l], g.R[2 * l + 1], kt, kn);
    return g.comp == 0 ? kt : kn;
}

// Householder QR of M (m x k, column-major, ld m) in place; tau[j] and the
// diagonal of R (alpha[j]) into shared memory.
__device__ void hm_qr(double *M, int m, int k, double *tau, double *alpha, double *red)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = 0; j < k; j++) {
        double *v = M + (int64_t)j * m;
        double l2 = 0.0;
        for (int i = j + threadIdx.x; i < m; i += HM_BT) l2 += v[i] * v[i];
        const double nrm = sqrt(hm_block_sum(l2, red));
        if (nrm == 0.0) {
            if (threadIdx.x == 0) { tau[j] = 0.0; alpha[j] = 0.0; }
            __syncthreads();
            continue;
        }
        const double a0 = v[j];
        const double al = a0 > 0 ? -nrm : nrm;
        __syncthreads();
        if (threadIdx.x == 0) { v[j] = a0 - al; alpha[j] = al; }
        __syncthreads();
        double vl = 0.0;
        for (int i = j + threadIdx.x; i < m; i += HM_BT) vl += v[i] * v[i];
        const double tj = 2.0 / hm_block_sum(vl, red);
        if (threadIdx.x == 0) tau[j] = tj;
        // the remaining columns, one warp per column
        for (int c = j + 1 + w; c < k; c += HM_BT / 32) {
            double *mc = M + (int64_t)c * m;
            double s = 0.0;
            for (int i = j + lane; i < m; i += 32) s += v[i] * mc[i];
            s = warp_sum(s) * tj;
            for (int i = j + lane; i < m; i += 32) mc[i] -= s * v[i];
        }
        __syncthreads();
    }
}

// X (m x r, column-major, ld m) = Q [Y; 0] with Q = H_0 ... H_{k-1} from hm_qr;
// column c of Y is ycol(c)[0..k).
template <class YF>
__device__ void hm_apply_q(const double *M, int m, int k, const double *tau, double *X, int r, YF ycol)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c = w; c < r; c += HM_BT / 32) {
        double *xc = X + (int64_t)c * m;
        for (int i = lane; i < m; i += 32) xc[i] = (i < k) ? ycol(c, i) : 0.0;
        __syncwarp();
        for (int j = k - 1; j >= 0; j--) {
            if (tau[j] == 0.0) continue;
            const double *v = M + (int64_t)j * m;
            double s = 0.0;
            for (int i = j + lane; i < m; i += 32) s += v[i] * xc[i];
            s = warp_sum(s) * tau[j];
            for (int i = j + lane; i < m; i += 32) xc[i] -= s * v[i];
            __syncwarp();
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(HM_BT) hm_aca_kernel(const AcaLeaf *__restrict__ leaves, AcaGeom g, double eps,
                                                       double *__restrict__ scratch, char *__restrict__ flags,
                                                       int *__restrict__ rank_out)
{
    extern __shared__ __align__(16) double hm_sm[];
    double *U = hm_sm;                          // k x k, column-major (G, then U)
    double *W = U + HM_KSVD * HM_KSVD;          // k x k
    double *tauA = W + HM_KSVD * HM_KSVD, *tauB = tauA + HM_KSVD, *alA = tauB + HM_KSVD, *alB = alA + HM_KSVD;
    double *Sv = alB + HM_KSVD, *aq = Sv + HM_KSVD, *bq = aq + HM_KMAX, *cache = bq + HM_KMAX;
    double *red = cache + HM_KMAX;              // 64 doubles: reductions
    __shared__ int redi[HM_BT / 32];
    __shared__ int ord[HM_KSVD];
    __shared__ int s_i, s_k, s_done;
    __shared__ double s_norm2;

    const AcaLeaf L = leaves[blockIdx.x];
    const int m = L.nr, n = L.nc;
    double *A = scratch + L.soff, *B = A + (int64_t)m * HM_KMAX;
    double *XA = B + (int64_t)n * HM_KMAX, *XB = XA + (int64_t)m * HM_KMAX;
    char *rused = flags + L.foff, *cused = rused + m;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    auto ent = [&](int ii, int jj) { return aca_entry(g, g.perm[L.r0 + ii], g.perm[L.c0 + jj]); };

    // ---- partial-pivot ACA ----
    if (tid == 0) { s_i = 0; s_k = 0; s_done = 0; s_norm2 = 0.0; }
    int zero_rows = 0;
    int result = 0;
    __syncthreads();
    const int kcap = min(m, n);
    while (true) {
        const int k = s_k, is = s_i;
        if (k >= kcap) { result = k; break; }
        if (k >= HM_KMAX) { result = -1; break; }
        if (tid == 0) rused[is] = 1;
        for (int q = tid; q < k; q += HM_BT) cache[q] = A[(int64_t)q * m + is];
        __syncthreads();
        double *row = B + (int64_t)k * n;
        double bv = 0.0;
        int bj = -1;
        for (int j = tid; j < n; j += HM_BT) {
            double v = ent(is, j);
            for (int q = 0; q < k; q++) v -= cache[q] * B[(int64_t)q * n + j];
            row[j] = v;
            if (!cused[j] && fabs(v) > bv) { bv = fabs(v); bj = j; }
        }
        double best;
        int js;
        hm_block_argmax(bv, bj, red, redi, best, js);
        if (js < 0 || best <= 1e-300) {
            // zero residual row: try another unused row
            if (++zero_rows > 3) { result = k; break; }
            __syncthreads();
            if (tid == 0) {
                int nxt = -1;
                for (int i = 0; i < m; i++)
                    if (!rused[i]) { nxt = i; break; }
                s_i = nxt;
            }
            __syncthreads();
            if (s_i < 0) { result = k; break; }
            continue;
        }
        const double piv = row[js];
        __syncthreads();
        if (tid == 0) cused[js] = 1;
        for (int q = tid; q < k; q += HM_BT) cache[q] = B[(int64_t)q * n + js];
        __syncthreads();
        for (int j = tid; j < n; j += HM_BT) row[j] /= piv;
        double *col = A + (int64_t)k * m;
        double bc = -1.0;
        int bi = -1;
        for (int i = tid; i < m; i += HM_BT) {
            double v = ent(i, js);
            for (int q = 0; q < k; q++) v -= cache[q] * A[(int64_t)q * m + i];
            col[i] = v;
        }
        __syncthreads();
        double la = 0.0, lb = 0.0;
        for (int i = tid; i < m; i += HM_BT) {
            la += col[i] * col[i];
            if (!rused[i] && fabs(col[i]) > bc) { bc = fabs(col[i]); bi = i; }
        }
        for (int j = tid; j < n; j += HM_BT) lb += row[j] * row[j];
        const double an = hm_block_sum(la, red);
        const double bn = hm_block_sum(lb, red);
        // a_q.a_k and b_q.b_k, one warp per q
        for (int q = w; q < k; q += HM_BT / 32) {
            double sa = 0.0, sb = 0.0;
            for (int i = lane; i < m; i += 32) sa += A[(int64_t)q * m + i] * col[i];
            for (int j = lane; j < n; j += 32) sb += B[(int64_t)q * n + j] * row[j];
            sa = warp_sum(sa);
            sb = warp_sum(sb);
            if (lane == 0) { aq[q] = sa; bq[q] = sb; }
        }
        double nb;
        int ni;
        hm_block_argmax(bc, bi, red + 8, redi, nb, ni);   // next pivot row (after aq/bq: the sync inside orders them)
        if (tid == 0) {
            double cross = 0.0;
            for (int q = 0; q < k; q++) cross += aq[q] * bq[q];
            s_norm2 += 2.0 * cross + an * bn;
            s_k = k + 1;
            s_done = (sqrt(an * bn) <= eps * sqrt(fabs(s_norm2))) ? 1 : (ni < 0 ? 1 : 0);
            s_i = ni;
        }
        __syncthreads();
        if (s_done) { result = s_k; break; }
    }
    __syncthreads();
    int k = result;
    if (k <= 0) {
        if (tid == 0) rank_out[blockIdx.x] = k;
        return;
    }
    if (k >= min(m, n) || k > HM_KSVD) {
        // no recompression: the ACA factors as they are
        for (int64_t q = tid; q < (int64_t)m * k; q += HM_BT) XA[q] = A[q];
        for (int64_t q = tid; q < (int64_t)n * k; q += HM_BT) XB[q] = B[q];
        if (tid == 0) rank_out[blockIdx.x] = k;
        return;
    }
    // ---- recompression ----
    hm_qr(A, m, k, tauA, alA, red);
    hm_qr(B, n, k, tauB, alB, red);
    // G = R_A R_B^T into U (column-major), W = identity
    for (int e = tid; e < k * k; e += HM_BT) {
        const int r = e % k, c = e / k;
        double sg = 0.0;
        for (int q = max(r, c); q < k; q++) {
            const double ra = (q == r) ? alA[r] : A[(int64_t)q * m + r];
            const double rb = (q == c) ? alB[c] : B[(int64_t)q * n + c];
            sg += ra * rb;
        }
        U[c * k + r] = sg;
        W[c * k + r] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    // one-sided Jacobi: sweeps of k' - 1 rounds (k' = k rounded up to even;
    // the extra column, if any, is a bye), k'/2 disjoint pairs per round
    const int kp = (k + 1) & ~1;
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0;
        for (int rd = 0; rd < kp - 1; rd++) {
            for (int pr = w; pr < kp / 2; pr += HM_BT / 32) {
                // round-robin pairing: position 0 fixed, the others rotate
                int a = (pr == 0) ? 0 : 1 + (pr - 1 + rd) % (kp - 1);
                int b = 1 + (kp - 2 - pr + rd) % (kp - 1);
                int p = min(a, b), q = max(a, b);
                if (q >= k || p == q) continue;
                double sa = 0.0, sb = 0.0, sg = 0.0;
                for (int i = lane; i < k; i += 32) {
                    const double up = U[p * k + i], uq = U[q * k + i];
                    sa += up * up;
                    sb += uq * uq;
                    sg += up * uq;
                }
                sa = warp_sum(sa);
                sb = warp_sum(sb);
                sg = warp_sum(sg);
                if (fabs(sg) <= 1e-300) continue;
                off = fmax(off, fabs(sg) / sqrt(sa * sb));
                const double zeta = (sb - sa) / (2.0 * sg);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
                for (int i = lane; i < k; i += 32) {
                    const double up = U[p * k + i], uq = U[q * k + i];
                    U[p * k + i] = cs * up - sn * uq;
                    U[q * k + i] = sn * up + cs * uq;
                    const double wp = W[p * k + i], wq = W[q * k + i];
                    W[p * k + i] = cs * wp - sn * wq;
                    W[q * k + i] = sn * wp + cs * wq;
                }
            }
            __syncthreads();
        }
        // largest off-diagonal measure of the sweep over the warps
        off = fmax(off, __shfl_xor_sync(0xffffffffu, off, 16));
        __syncthreads();
        if (lane == 0) red[w] = off;
        __syncthreads();
        double mo = 0.0;
        for (int q = 0; q < HM_BT / 32; q++) mo = fmax(mo, red[q]);
        __syncthreads();
        if (mo < 1e-15) break;
    }
    // singular values (column norms), normalised U, order by decreasing value
    for (int j = w; j < k; j += HM_BT / 32) {
        double sn = 0.0;
        for (int i = lane; i < k; i += 32) sn += U[j * k + i] * U[j * k + i];
        sn = sqrt(warp_sum(sn));
        if (lane == 0) Sv[j] = sn;
        __syncwarp();
        if (sn > 0)
            for (int i = lane; i < k; i += 32) U[j * k + i] /= sn;
    }
    __syncthreads();
    for (int j = tid; j < k; j += HM_BT) {
        int pos = 0;
        for (int q = 0; q < k; q++) pos += (Sv[q] > Sv[j]) || (Sv[q] == Sv[j] && q < j);
        ord[pos] = j;
    }
    __syncthreads();
    if (tid == 0) {
        int r = 0;
        for (int i = 0; i < k; i++) {
            r = i + 1;
            if (Sv[ord[i]] <= eps * Sv[ord[0]]) break;
        }
        s_k = r;
    }
    __syncthreads();
    const int r = s_k;
    hm_apply_q(A, m, k, tauA, XA, r, [&](int c, int i) { return U[ord[c] * k + i] * Sv[ord[c]]; });
    hm_apply_q(B, n, k, tauB, XB, r, [&](int c, int i) { return W[ord[c] * k + i]; });
    if (tid == 0) rank_out[blockIdx.x] = r;
}

// Factors of rank r > 0 from the scratch X regions into the stored layout
// (A'^T rank x lda and B'^T rank x ld, rank-major, padding left as it is):
// dst offsets relative to the start of the batch's segment.
struct AcaPlace {
    int64_t foff, goff;   // A'^T and B'^T offsets in the segment
    int lda, ld, rank;
};

template <typename T>
__global__ void __launch_bounds__(256) hm_aca_place_kernel(const AcaLeaf *__restrict__ leaves,
                                                           const AcaPlace *__restrict__ place,
                                                           const double *__restrict__ scratch, T *__restrict__ dst)
{
    const AcaLeaf L = leaves[blockIdx.x];
    const AcaPlace P = place[blockIdx.x];
    if (P.rank <= 0) return;
    const double *XA = scratch + L.soff + (int64_t)(L.nr + L.nc) * HM_KMAX;
    const double *XB = XA + (int64_t)L.nr * HM_KMAX;
    for (int64_t e = threadIdx.x; e < (int64_t)P.rank * L.nr; e += blockDim.x) {
        const int q = (int)(e / L.nr), i = (int)(e % L.nr);
        dst[P.foff + (int64_t)q * P.lda + i] = (T)XA[(int64_t)q * L.nr + i];
    }
    for (int64_t e = threadIdx.x; e < (int64_t)P.rank * L.nc; e += blockDim.x) {
        const int q = (int)(e / L.nc), j = (int)(e % L.nc);
        dst[P.goff + (int64_t)q * P.ld + j] = (T)XB[(int64_t)q * L.nc + j];
    }
}

// y(pos) = sum of the slots of row pos (fixed order: the leaves of its
// segment of rows in block order; a warp's rows mostly share a segment, so
// the bases are broadcast and the slot reads coalesced), stored at the
// original element index in the K.V result arrays (partials with one chunk).
__global__ void hm_gather_kernel(int64_t Ntot, int ncomp, const int *__restrict__ inst_of,
                                 const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl, int mask,
                                 const int *__restrict__ perm, const int32_t *__restrict__ segof,
                                 const int64_t *__restrict__ segptr, const int64_t *__restrict__ segbase,
                                 const double *__restrict__ out, double *partT, double *partN)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= Ntot) return;
    const int i = inst_of[e];
    if (!takes_part(ctl, i, mask)) return;
    const Inst &I = inst[i];
    const int64_t orig = perm[e];   // perm[eoff + pos], a network-local index
    for (int c = 0; c < ncomp; c++) {
        const int sg = segof[(int64_t)c * Ntot + e];
        double s = 0.0;
        for (int64_t j = segptr[sg]; j < segptr[sg + 1]; j++) s += out[segbase[j] + e];
        (c == 0 ? partT : partN)[I.poff + orig] = s;
    }
}
