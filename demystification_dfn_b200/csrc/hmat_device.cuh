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
//   2. the rows of every leaf: F_b xp (dense leaves) and A_b z_b (low-rank
//      leaves), two launches, one output slot per (leaf, row);
//   3. y(row) = sum of the row's slots in a fixed order, written in the
//      original element order (y[perm[pos]]).
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
constexpr int HM_LROWS = 256;  // rows per step-2 task of a low-rank leaf
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

// z partial of one column chunk: warp w takes rank rows q = w, w+8, ...;
// lanes stream the row's columns in 16-byte vectors.
template <typename T>
__global__ void __launch_bounds__(256) hm_lowrank_kernel(const HTask *__restrict__ tasks, const HBlk *__restrict__ blks,
                                                         const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                                                         int mask, const T *__restrict__ vals,
                                                         const double *__restrict__ xp, double *__restrict__ zpart)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    const HTask t = tasks[blockIdx.x];
    const HBlk b = blks[t.blk];
    if (!takes_part(ctl, b.inst, mask)) return;
    const Inst &I = inst[b.inst];
    const double *x = xp + I.eoff + b.c0 + t.start;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nv = (t.count + W - 1) / W;    // vectors of the chunk (padding columns are zero)
    for (int q = w; q < b.rank; q += 8) {
        const VT *row = reinterpret_cast<const VT *>(vals + b.goff + (int64_t)q * b.ld + t.start);
        double s = 0.0;
        for (int v = lane; v < nv; v += 32) {
            double f[W];
            HVec<T>::unpack(row[v], f);
#pragma unroll
            for (int j = 0; j < W; j++) s = fma(f[j], x[v * W + j], s);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) zpart[b.zoff + (int64_t)t.chunk * b.rank + q] = s;
    }
}

// Rows of dense leaves: a half-warp per row, 16-byte vectors of F against
// xp; four rows per half-warp in flight (their loads issued together).
template <typename T>
__global__ void __launch_bounds__(256) hm_dense_kernel(const HTask *__restrict__ tasks, const HBlk *__restrict__ blks,
                                                       const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                                                       int mask, const T *__restrict__ vals,
                                                       const double *__restrict__ xp, double *__restrict__ out)
{
    using VT = typename HVec<T>::V;
    constexpr int W = HVec<T>::W;
    constexpr int U = 4;
    const HTask t = tasks[blockIdx.x];
    const HBlk b = blks[t.blk];
    if (!takes_part(ctl, b.inst, mask)) return;
    const Inst &I = inst[b.inst];
    const double *x = xp + I.eoff + b.c0;
    const int hl = threadIdx.x & 15, w = threadIdx.x >> 5, half = (threadIdx.x >> 4) & 1;
    const int nv = (b.nc + W - 1) / W;
    const VT zero{};
    // the loop runs the same trips in both half-warps (shuffles below)
    for (int wb = w * 2 * U; wb < t.count; wb += 8 * 2 * U) {
        const int i0 = wb + half * U;
        double s[U];
#pragma unroll
        for (int u = 0; u < U; u++) s[u] = 0.0;
        for (int v = hl; v < nv; v += 16) {
            double xv[W];
#pragma unroll
            for (int j = 0; j < W; j++) xv[j] = x[v * W + j];
            VT fv[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int row = t.start + i0 + u;
                fv[u] = (i0 + u < t.count) ? reinterpret_cast<const VT *>(vals + b.foff + (int64_t)row * b.ld)[v]
                                           : zero;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                double a[W];
                HVec<T>::unpack(fv[u], a);
#pragma unroll
                for (int j = 0; j < W; j++) s[u] = fma(a[j], xv[j], s[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], o);
            if (hl == 0 && i0 + u < t.count) out[b.outoff + t.start + i0 + u] = s[u];
        }
    }
}

// Low-rank leaves of at most HM_COLS columns, whole: z = B^T xp into shared
// memory (warp per rank row), then the rows y = A z (thread per row); one
// CTA per leaf, no partial sums in global memory.
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
    const HBlk b = blks[leaves[blockIdx.x]];
    if (!takes_part(ctl, b.inst, mask)) return;
    const Inst &I = inst[b.inst];
    const double *x = xp + I.eoff + b.c0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nv = (b.nc + W - 1) / W;
    for (int q = w; q < b.rank; q += 8) {
        const VT *row = reinterpret_cast<const VT *>(vals + b.goff + (int64_t)q * b.ld);
        double s = 0.0;
        for (int v = lane; v < nv; v += 32) {
            double f[W];
            HVec<T>::unpack(row[v], f);
#pragma unroll
            for (int j = 0; j < W; j++) s = fma(f[j], x[v * W + j], s);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) z[q] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < b.nr; i += blockDim.x) {
        const T *a = vals + b.foff + i;
        double s = 0.0;
        for (int q = 0; q < b.rank; q++) s = fma((double)a[(int64_t)q * b.lda], z[q], s);
        out[b.outoff + i] = s;
    }
}

// Rows of low-rank leaves: one thread per row, sum over the rank of
// A^T[q][row] z[q] (coalesced across the threads for each q).
template <typename T>
__global__ void __launch_bounds__(256) hm_rows_kernel(const HTask *__restrict__ tasks, const HBlk *__restrict__ blks,
                                                      const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                                                      int mask, const T *__restrict__ vals,
                                                      const double *__restrict__ zpart, double *__restrict__ out)
{
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
    for (int i = threadIdx.x; i < t.count; i += blockDim.x) {
        const int row = t.start + i;
        const T *a = vals + b.foff + row;
        double s = 0.0;
        for (int q = 0; q < r; q++) s = fma((double)a[(int64_t)q * b.lda], z[q], s);
        out[b.outoff + row] = s;
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

// y(pos) = sum of the slots of row pos (fixed order), stored at the
// original element index in the K.V result arrays (partials with one chunk).
__global__ void hm_gather_kernel(int64_t Ntot, int ncomp, const int *__restrict__ inst_of,
                                 const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl, int mask,
                                 const int *__restrict__ perm, const int64_t *__restrict__ rowptr,
                                 const int64_t *__restrict__ slots, const double *__restrict__ out, double *partT,
                                 double *partN)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= Ntot) return;
    const int i = inst_of[e];
    if (!takes_part(ctl, i, mask)) return;
    const Inst &I = inst[i];
    const int64_t orig = perm[e];   // perm[eoff + pos], a network-local index
    for (int c = 0; c < ncomp; c++) {
        const int64_t q = (int64_t)c * Ntot + e;
        double s = 0.0;
        for (int64_t j = rowptr[q]; j < rowptr[q + 1]; j++) s += out[slots[j]];
        (c == 0 ? partT : partN)[I.poff + orig] = s;
    }
}
