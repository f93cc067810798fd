// hmat_device.cuh — H-matrix K.V on the GPU (replaces Hgemv_right,
// src/hmatrix/calculation_hmat.f90:3-165, and the permutations of
// hmatII/hmatIII, src/kernel_calculation/hmatrixModeII.f90:46-69).
//
// The reference recurses over the block tree and calls ZGEMV on each leaf
// with complex(8) storage (16 bytes per real entry). Here the leaves are a
// flat list and every K.V is three launches over task lists:
//   1. z_b = B_b^T x for every low-rank block b, split in column chunks
//      (partial sums per chunk, added in fixed order in step 2);
//   2. the rows of every leaf: F_b x (dense leaves) or A_b z_b (low-rank),
//      one output slot per (leaf, row);
//   3. y(row) = sum of the row's slots in a fixed order, written in the
//      original element order (y[perm[pos]]).
// x is the slip-rate vector read through the cluster permutation. Factors are
// stored row-major (F: nr x nc, A: nr x rank, B: nc x rank) in FP64 or FP32;
// sums are FP64. Every launch is predicated on the network's phase like the
// dense K.V, and covers all networks of a batch.
#pragma once
#include "dfn_device.cuh"
#include "hmat_build.h"

struct HBlk {
    int inst, comp, dense, rank;
    int r0, nr, c0, nc;        // positions in cluster order (within the network)
    int64_t foff;              // dense: F offset; low-rank: A offset (values)
    int64_t goff;              // low-rank: B offset (values)
    int64_t zoff;              // low-rank: first z partial (ntask1 x rank doubles)
    int64_t outoff;            // first output slot of the leaf's rows
    int ntask1;                // column chunks of the low-rank product
    int pad;
};

struct HTask { int blk, start, count, chunk; };

constexpr int HM_COLS = 1024;  // columns per step-1 task
constexpr int HM_ROWS = 64;    // rows per step-2 task

template <typename T>
__global__ void __launch_bounds__(256) hm_lowrank_kernel(const HTask *__restrict__ tasks, const HBlk *__restrict__ blks,
                                                         const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                                                         int mask, const T *__restrict__ vals,
                                                         const int *__restrict__ perm, const double *__restrict__ Vbase,
                                                         int vmul, double *__restrict__ zpart)
{
    __shared__ double red[8][hmat::kMaxRank];
    const HTask t = tasks[blockIdx.x];
    const HBlk b = blks[t.blk];
    if (!takes_part(ctl, b.inst, mask)) return;
    const Inst &I = inst[b.inst];
    const double *V = Vbase + (int64_t)vmul * I.eoff;
    const int *pm = perm + I.eoff;
    // warp w takes columns start+w, start+w+8, ...; lane q accumulates rank
    // components q and q+32 (the r values of a column are contiguous)
    static_assert(hmat::kMaxRank <= 64, "two rank components per lane");
    const int r = b.rank;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double acc0 = 0.0, acc1 = 0.0;
    for (int l = t.start + w; l < t.start + t.count; l += 8) {
        const double x = V[pm[b.c0 + l]];
        const T *row = vals + b.goff + (int64_t)l * r;
        if (lane < r) acc0 = fma((double)row[lane], x, acc0);
        if (lane + 32 < r) acc1 = fma((double)row[lane + 32], x, acc1);
    }
    red[w][lane] = acc0;
    red[w][lane + 32] = acc1;
    __syncthreads();
    if (threadIdx.x < r) {
        double s = 0.0;
        for (int ww = 0; ww < 8; ww++) s += red[ww][threadIdx.x];
        zpart[b.zoff + (int64_t)t.chunk * r + threadIdx.x] = s;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) hm_rows_kernel(const HTask *__restrict__ tasks, const HBlk *__restrict__ blks,
                                                      const Inst *__restrict__ inst, const StepCtl *__restrict__ ctl,
                                                      int mask, const T *__restrict__ vals,
                                                      const int *__restrict__ perm, const double *__restrict__ Vbase,
                                                      int vmul, const double *__restrict__ zpart,
                                                      double *__restrict__ out)
{
    __shared__ double z[hmat::kMaxRank];
    const HTask t = tasks[blockIdx.x];
    const HBlk b = blks[t.blk];
    if (!takes_part(ctl, b.inst, mask)) return;
    const Inst &I = inst[b.inst];
    if (b.dense) {
        const double *V = Vbase + (int64_t)vmul * I.eoff;
        const int *pm = perm + I.eoff;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int i = w; i < t.count; i += 8) {
            const int row = t.start + i;
            const T *f = vals + b.foff + (int64_t)row * b.nc;
            double s = 0.0;
            for (int l = lane; l < b.nc; l += 32) s = fma((double)f[l], V[pm[b.c0 + l]], s);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) out[b.outoff + row] = s;
        }
    } else {
        const int r = b.rank;
        if (threadIdx.x < r) {
            double s = 0.0;
            for (int j = 0; j < b.ntask1; j++) s += zpart[b.zoff + (int64_t)j * r + threadIdx.x];
            z[threadIdx.x] = s;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < t.count; i += blockDim.x) {
            const int row = t.start + i;
            const T *a = vals + b.foff + (int64_t)row * r;
            double s = 0.0;
            for (int q = 0; q < r; q++) s = fma((double)a[q], z[q], s);
            out[b.outoff + row] = s;
        }
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
