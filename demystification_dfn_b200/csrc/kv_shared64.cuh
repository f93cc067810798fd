// kv_shared64.cuh — FP64 K.V of a batch whose networks share one kernel
// matrix (DFN_STORE_FP64_SHARED). The R slip-rate vectors of a stage meet the
// same K, so K.V is a GEMM, C[k][m] = sum_l K[k][l] V_m[l] (rows k with their
// shear and normal entries, members m), computed in FP64 on the CUDA cores
// with K streamed from HBM once for all members. It is the FP64 counterpart
// of the tensor-core batch (tc_gemm.cuh): same K sharing, FP64 products and
// sums, so that the two isolate what the BF16 hi+lo tensor-core arithmetic
// itself gains. (The reference has one network per process and no batch.)
//
// K is stored row-major, N rows of Np columns (Np = N padded to S64_COLS with
// zero columns), {K_T, K_N} per column in mode II; the V of all members is
// packed per stage into vt[l][m] (RP members padded to S64_MEM with zeros).
// CTA tile: S64_ROWS rows x S64_MEM members; the columns of the CTA's split
// pass through a two-buffer shared-memory pipeline (cp.async, 16 bytes per
// copy) in chunks of S64_COLS. Thread (ty, tx) owns rows 2ty, 2ty+1 and
// members 2tx, 2tx+1, 32+2tx, 33+2tx of the tile (so that a half-warp reads
// 256 contiguous bytes of V): 8 shear (and 8 normal) accumulators. K rows
// in shared memory are padded by 16 bytes, so the two rows a warp reads at
// once fall in different banks.
// Each split writes its partial sums to part[poff_m + split*N + k] (the
// layout the stage kernel sums in fixed order), so results are
// deterministic.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

constexpr int S64_ROWS = 32;
constexpr int S64_MEM = 64;
constexpr int S64_COLS = 32;
constexpr int S64_THREADS = 256;

// dynamic shared memory of one CTA: two buffers of K (rows x cols x {T,N})
// and V (cols x members)
__host__ __device__ constexpr size_t s64_smem_bytes(int mode)
{
    return 2 * sizeof(double) * ((size_t)S64_ROWS * (S64_COLS * (mode == 2 ? 2 : 1) + 2) + (size_t)S64_COLS * S64_MEM);
}

__device__ __forceinline__ void s64_cp16(void *smem_dst, const void *gmem_src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(
                     __cvta_generic_to_shared(smem_dst))),
                 "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void s64_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void s64_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// vt[l * RP + m] = V of member m at column l (zero beyond N and R); V of
// member m is Vbase[vmul * eoff_m + l].
__global__ void s64_pack_v_kernel(const double *__restrict__ Vbase, int vmul, const Inst *__restrict__ inst,
                                  int64_t N, int R, int RP, int64_t Np, double *__restrict__ vt)
{
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= Np * RP) return;
    const int64_t l = idx / RP;
    const int m = (int)(idx % RP);
    vt[idx] = (l < N && m < R) ? Vbase[(int64_t)vmul * inst[m].eoff + l] : 0.0;
}

// grid (row tiles, member tiles, splits); split s covers column chunks
// [s * kc_per_split, min(nkc, (s + 1) * kc_per_split)).
template <int MODE>
__global__ void __launch_bounds__(S64_THREADS) s64_gemm_kernel(const double *__restrict__ K,
                                                               const double *__restrict__ vt,
                                                               const Inst *__restrict__ inst, int64_t N, int64_t Np,
                                                               int R, int RP, int kc_per_split, int nkc,
                                                               double *__restrict__ partT,
                                                               double *__restrict__ partN)
{
    constexpr int CPE = (MODE == 2) ? 2 : 1;            // doubles per stored entry
    constexpr int KROW = S64_COLS * CPE;                 // doubles per K row of a chunk
    constexpr int KLD = KROW + 2;                        // padded row in shared memory
    constexpr int KSZ = S64_ROWS * KLD, VSZ = S64_COLS * S64_MEM;
    extern __shared__ __align__(16) double s64_smem[];
    double *Ks = s64_smem;                // [2][S64_ROWS][KLD]
    double *Vs = s64_smem + 2 * KSZ;      // [2][S64_COLS][S64_MEM]

    const int tid = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * S64_ROWS;
    const int m0 = blockIdx.y * S64_MEM;
    const int split = blockIdx.z;
    const int kc0 = split * kc_per_split;
    const int kc1 = (kc0 + kc_per_split < nkc) ? kc0 + kc_per_split : nkc;
    const int ty = tid >> 4, tx = tid & 15;

    double aT[2][4], aN[2][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) { aT[i][j] = 0.0; aN[i][j] = 0.0; }

    // one chunk of K rows and V columns into buffer b (16-byte copies; rows
    // beyond N are zeros written directly)
    auto load = [&](int b, int kc) {
        const int64_t c0 = (int64_t)kc * S64_COLS;
        double *kd = Ks + b * KSZ;
        for (int p = tid; p < S64_ROWS * KROW / 2; p += S64_THREADS) {
            const int row = p / (KROW / 2), q = p % (KROW / 2);
            const int64_t gr = r0 + row;
            double *dst = kd + row * KLD + 2 * q;
            if (gr < N) s64_cp16(dst, K + (gr * Np + c0) * CPE + 2 * q);
            else { dst[0] = 0.0; dst[1] = 0.0; }
        }
        double *vd = Vs + b * VSZ;
        for (int p = tid; p < VSZ / 2; p += S64_THREADS) {
            const int col = p / (S64_MEM / 2), q = p % (S64_MEM / 2);
            s64_cp16(vd + col * S64_MEM + 2 * q, vt + (c0 + col) * RP + m0 + 2 * q);
        }
        s64_commit();
    };

    if (kc0 < kc1) load(0, kc0);
    for (int kc = kc0; kc < kc1; kc++) {
        const int b = (kc - kc0) & 1;
        if (kc + 1 < kc1) {
            load(b ^ 1, kc + 1);
            s64_wait<1>();
        } else {
            s64_wait<0>();
        }
        __syncthreads();
        const double *kb = Ks + b * KSZ + (2 * ty) * KLD;
        const double *vb = Vs + b * VSZ + 2 * tx;
#pragma unroll 8
        for (int c = 0; c < S64_COLS; c++) {
            const double2 v01 = *reinterpret_cast<const double2 *>(vb + c * S64_MEM);
            const double2 v23 = *reinterpret_cast<const double2 *>(vb + c * S64_MEM + 32);
            const double v[4] = {v01.x, v01.y, v23.x, v23.y};
#pragma unroll
            for (int i = 0; i < 2; i++) {
                double kT, kN = 0.0;
                if (MODE == 2) {
                    const double2 kk = *reinterpret_cast<const double2 *>(kb + i * KLD + 2 * c);
                    kT = kk.x;
                    kN = kk.y;
                } else {
                    kT = kb[i * KLD + c];
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    aT[i][j] = fma(kT, v[j], aT[i][j]);
                    if (MODE == 2) aN[i][j] = fma(kN, v[j], aN[i][j]);
                }
            }
        }
        __syncthreads();   // the buffer is refilled by the next iteration's copies
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int64_t row = r0 + 2 * ty + i;
        if (row >= N) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int m = m0 + (j < 2 ? 2 * tx + j : 32 + 2 * tx + (j - 2));
            if (m >= R) continue;
            const int64_t o = inst[m].poff + (int64_t)split * N + row;
            partT[o] = aT[i][j];
            if (MODE == 2) partN[o] = aN[i][j];
        }
    }
}
