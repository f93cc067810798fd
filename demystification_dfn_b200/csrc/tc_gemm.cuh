// tc_gemm.cuh — K·V of a batch of networks that share one geometry, as a
// GEMM on the 5th-generation tensor cores (tcgen05, accumulators in TMEM).
//
// When R networks share their fault geometry (a parameter or initial-state
// ensemble of one network), the R slip-rate vectors of a stage meet the same
// kernel matrix: D[m, r] = sum_l K[m, l] V_r[l], a GEMM with M = rows of K
// (shear rows, then normal rows in mode II), N = R, and the source elements
// as the reduction dimension. K is streamed from HBM once for all R vectors.
//
// Precision: K and V are split into BF16 hi + lo parts (x = hi + lo to 16
// mantissa bits); D = Khi Vhi + Khi Vlo + Klo Vhi, three kind::f16 MMAs per
// K step into one FP32 accumulator in TMEM (the lo x lo term is below the
// BF16 rounding of the others).
//
// Layout in HBM: K (hi and lo) and the packed V rows are stored tile by
// tile (128 x 64 for K, BN x 64 for V, tiles of one row block consecutive
// along the reduction), each tile already in the 128-byte-swizzled order the
// tensor cores read from shared memory (16-byte chunk c of row r at chunk
// position c ^ (r mod 8) within 1024-byte groups of 8 rows). A stage is then
// four contiguous bulk copies (16 KiB for a K tile), which streams HBM at
// full page locality instead of 128-byte row pieces 2N bytes apart.
//
// Work unit: one 128-row tile of K and one split of the reduction range (the
// splits spread the 128-row tiles over the 148 SMs; their partial sums go to
// part[s][row] and the friction kernel adds them in a fixed order, so the
// result is deterministic). One CTA of 4 warps per unit:
//   warp 0, one lane   producer: cp.async.bulk copies of the Khi, Klo and
//                      Vhi, Vlo tiles of a stage into a ring of 2-4 stages,
//                      completed on mbarriers;
//   warp 1, one lane   MMA issuer: 4 x 3 tcgen05.mma per stage, then
//                      tcgen05.commit to the stage's "empty" mbarrier;
//   all 4 warps        epilogue: tcgen05.ld of the warp's 32 TMEM lanes
//                      (rows) x BN columns, stores of the partial sums.
// Every wait is bounded; on expiry the CTA raises the error flag, the
// producer waits (bounded) for the copies it issued, TMEM is freed and the
// CTA returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define TC_BM 128          // rows of K per tile (TMEM lanes)
#define TC_BK 64           // reduction elements per stage (128 bytes of BF16)
#define TC_THREADS 128

__host__ __device__ constexpr size_t tc_stage_bytes(int bn) { return (size_t)2 * TC_BM * TC_BK * 2 + (size_t)2 * bn * TC_BK * 2; }
// deepest ring that keeps the stages within 192 KiB of shared memory (one
// CTA per SM); the autotuner may pick a 2-stage ring instead (two CTAs per
// SM for BN <= 64, one's fill and epilogue overlapping the other's stream)
__host__ __device__ constexpr int tc_stages(int bn) { return bn <= 64 ? 4 : (bn <= 128 ? 3 : 2); }
__host__ __device__ constexpr size_t tc_smem_bytes(int bn, int stages) { return stages * tc_stage_bytes(bn) + 1024 + 256; }

// Element offset of (row r, column j < 64) inside a swizzled tile of 128-byte rows.
__host__ __device__ inline int64_t tc_swz(int64_t r, int64_t j)
{
    return (r >> 3) * 512 + (r & 7) * 64 + ((((j >> 3) ^ (r & 7))) << 3) + (j & 7);
}

struct TcOut {
    double *partT, *partN;     // per network at inst[r].poff: [splits][N]
    const Inst *inst;
    int64_t N;                 // elements per network
    int64_t mrows;             // rows of K (N, or 2N in mode II)
    int R;                     // networks
    int kb_per_split;          // reduction stages per split
    int nkb;                   // reduction stages in total
    int nmt;                   // 128-row tiles
    int nsplit;                // reduction splits (work units = nmt * nsplit)
};

// Shared-memory matrix descriptor (tcgen05): K-major operand, 128-byte
// swizzle, rows of 128 bytes, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                          // leading byte offset (unused with swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                          // 128-byte swizzle
    return d;
}

// Instruction descriptor: D F32, A and B BF16, both K-major, M = 128, N = bn.
__host__ __device__ constexpr uint32_t tc_idesc(int bn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Bounded wait that also gives up once another role of the CTA raised the
// abort flag.
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity, const int *abort_flag)
{
    for (int it = 0; it < (1 << 22); it++) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(smem_u32(bar)), "r"(parity)
                     : "memory");
        if (ok) return true;
        if ((it & 63) == 63 && *(volatile const int *)abort_flag) return false;
    }
    return false;
}

// Epilogue of one work unit for one warp: TMEM lanes 32q..32q+31 (rows of
// the 128-row tile) x BN columns (networks), read from accumulator columns
// starting at tmem_acc, stored as part[split][row] of each network; zeros
// when the unit had no reduction stages (have = false).
template <int BN>
__device__ __forceinline__ void tc_store_unit(uint32_t tmem_acc, const TcOut &out, int mt, int split, int q, int lane,
                                              bool have)
{
    const int64_t row = (int64_t)mt * TC_BM + q * 32 + lane;
    const bool shear = row < out.N;
    const int64_t k = shear ? row : row - out.N;
    const bool live = row < out.mrows;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 16) {
        uint32_t v[16];
        if (have) {
            const uint32_t taddr = tmem_acc + ((uint32_t)(q * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                           "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] = 0u;
        }
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int r = c0 + j;
            if (live && r < out.R) {
                double *dst = (shear ? out.partT : out.partN) + out.inst[r].poff + (int64_t)split * out.N + k;
                *dst = (double)__uint_as_float(v[j]);
            }
        }
    }
}

template <int BN, int STAGES>
__global__ void __launch_bounds__(TC_THREADS, 1)
    tc_gemm_kernel(const __nv_bfloat16 *__restrict__ Ah, const __nv_bfloat16 *__restrict__ Al,
                   const __nv_bfloat16 *__restrict__ Bh, const __nv_bfloat16 *__restrict__ Bl, TcOut out,
                   int *err_flag)
{
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "N of an M=128 MMA is a multiple of 16 up to 256");
    static_assert(STAGES >= 2 && STAGES * tc_stage_bytes(BN) <= 196608, "ring within 192 KiB");
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    // 1024-byte alignment of the stage ring (128-byte swizzle atoms)
    unsigned char *ring = reinterpret_cast<unsigned char *>(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + STAGES * tc_stage_bytes(BN));
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x % out.nmt, split = blockIdx.x / out.nmt;
    const int kb0 = split * out.kb_per_split;
    const int kb1 = min(kb0 + out.kb_per_split, out.nkb);
    const int nk = max(kb1 - kb0, 0);   // a trailing split may be empty
    constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2;
    constexpr uint32_t TX = 2 * A_BYTES + 2 * B_BYTES;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        // TMEM: BN columns of 32-bit accumulators for the 128 lanes
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)(BN < 32 ? 32 : BN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0 && nk > 0) {
        // producer
        int issued = 0;
        for (int i = 0; i < nk; i++) {
            const int s = i % STAGES, use = i / STAGES;
            if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1)) { *abort_flag = 1; break; }
            if (*(volatile int *)abort_flag) break;
            unsigned char *st = ring + s * tc_stage_bytes(BN);
            mbar_expect_tx(&full[s], TX);
            const int64_t kb = kb0 + i;
            const int64_t at = ((int64_t)mt * out.nkb + kb) * (TC_BM * TC_BK), bt = kb * (BN * TC_BK);
            tma_bulk_g2s(st, Ah + at, A_BYTES, &full[s]);
            tma_bulk_g2s(st + A_BYTES, Al + at, A_BYTES, &full[s]);
            tma_bulk_g2s(st + 2 * A_BYTES, Bh + bt, B_BYTES, &full[s]);
            tma_bulk_g2s(st + 2 * A_BYTES + B_BYTES, Bl + bt, B_BYTES, &full[s]);
            issued = i + 1;
        }
        // the copies this thread issued complete before the CTA may exit
        for (int i = (issued > STAGES ? issued - STAGES : 0); i < issued; i++)
            if (!mbar_wait(&full[i % STAGES], (i / STAGES) & 1)) *abort_flag = 1;
    } else if (warp == 1 && lane == 0 && nk > 0) {
        // MMA issuer
        const uint32_t idesc = tc_idesc(BN);
        for (int i = 0; i < nk; i++) {
            const int s = i % STAGES, use = i / STAGES;
            if (!mbar_wait(&full[s], use & 1)) { *abort_flag = 1; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = smem_u32(ring + s * tc_stage_bytes(BN));
            const uint64_t ah = tc_desc(base), al = tc_desc(base + A_BYTES);
            const uint64_t bh = tc_desc(base + 2 * A_BYTES), bl = tc_desc(base + 2 * A_BYTES + B_BYTES);
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; kk++) {
                // 16 BF16 = 32 bytes further along K inside the swizzle atom
                const uint64_t o = (uint64_t)(kk * 32 >> 4);
                tc_mma(tmem, ah + o, bh + o, idesc, (i > 0 || kk > 0) ? 1u : 0u);
                tc_mma(tmem, ah + o, bl + o, idesc, 1u);
                tc_mma(tmem, al + o, bh + o, idesc, 1u);
            }
            tc_commit(&empty[s]);   // the stage is free once these MMAs have read it
        }
        tc_commit(done);            // all MMAs issued so far have completed
    }
    __syncwarp();
    // epilogue: warp w holds rows 32w..32w+31 of the tile (TMEM lanes)
    bool ok = (nk > 0);
    if (ok) ok = mbar_wait(done, 0);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && nk > 0) *abort_flag = 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    const bool good = ok && !*(volatile int *)abort_flag;
    if (good || nk == 0) {
        tc_store_unit<BN>(tmem, out, mt, split, warp, lane, nk > 0);
    } else if (threadIdx.x == 0) {
        atomicExch(err_flag, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"((uint32_t)(BN < 32 ? 32 : BN)));
}

// Persistent form of the same GEMM: one CTA per SM walks the work units
// u = blockIdx.x, blockIdx.x + gridDim.x, ... (unit u = row tile u % nmt,
// split u / nmt, as above). The producer streams the stages of consecutive
// units through the ring without a break, the MMA issuer alternates between
// two TMEM accumulators (2 x BN columns), and four epilogue warps drain one
// accumulator while the MMAs of the next unit fill the other, so the per-unit
// start-up (TMEM allocation, barrier set-up, first copy latency) and the
// epilogue leave the HBM stream. Every unit is summed exactly as in
// tc_gemm_kernel: the results are identical bit for bit.
//   warp 0, one lane   producer;  warp 1, one lane   MMA issuer;
//   warps 2-5          epilogue (TMEM lane quarter warp % 4).
#define TC_PTHREADS 192

template <int BN, int STAGES>
__global__ void __launch_bounds__(TC_PTHREADS, 1)
    tc_gemm_persistent_kernel(const __nv_bfloat16 *__restrict__ Ah, const __nv_bfloat16 *__restrict__ Al,
                              const __nv_bfloat16 *__restrict__ Bh, const __nv_bfloat16 *__restrict__ Bl, TcOut out,
                              int *err_flag)
{
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "N of an M=128 MMA is a multiple of 16 up to 256");
    static_assert(STAGES >= 2 && STAGES * tc_stage_bytes(BN) <= 196608, "ring within 192 KiB");
    constexpr uint32_t TCOLS = 2 * BN < 32 ? 32 : 2 * BN;   // two accumulators, a power of two >= 32
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    unsigned char *ring = reinterpret_cast<unsigned char *>(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + STAGES * tc_stage_bytes(BN));
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;    // accumulator a holds a finished unit
    uint64_t *tempty = tfull + 2;        // accumulator a has been read out
    uint64_t *done = tempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int units = out.nmt * out.nsplit;
    constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2;
    constexpr uint32_t TX = 2 * A_BYTES + 2 * B_BYTES;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int a = 0; a < 2; a++) { mbar_init(&tfull[a], 1); mbar_init(&tempty[a], 4); }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // producer: stage g of this CTA goes to ring slot g % STAGES
            uint32_t g = 0;
            bool stop = false;
            for (int u = blockIdx.x; u < units && !stop; u += gridDim.x) {
                const int mt = u % out.nmt, split = u / out.nmt;
                const int kb0 = split * out.kb_per_split, kb1 = min(kb0 + out.kb_per_split, out.nkb);
                for (int kb = kb0; kb < kb1; kb++, g++) {
                    const uint32_t s = g % STAGES, use = g / STAGES;
                    if (use > 0 && !tc_wait(&empty[s], (use - 1) & 1, abort_flag)) {
                        *abort_flag = 1;
                        stop = true;
                        break;
                    }
                    unsigned char *st = ring + s * tc_stage_bytes(BN);
                    mbar_expect_tx(&full[s], TX);
                    const int64_t at = ((int64_t)mt * out.nkb + kb) * (TC_BM * TC_BK), bt = (int64_t)kb * (BN * TC_BK);
                    tma_bulk_g2s(st, Ah + at, A_BYTES, &full[s]);
                    tma_bulk_g2s(st + A_BYTES, Al + at, A_BYTES, &full[s]);
                    tma_bulk_g2s(st + 2 * A_BYTES, Bh + bt, B_BYTES, &full[s]);
                    tma_bulk_g2s(st + 2 * A_BYTES + B_BYTES, Bl + bt, B_BYTES, &full[s]);
                }
            }
            // the copies this thread issued complete before the CTA may exit
            for (uint32_t i = (g > STAGES ? g - STAGES : 0); i < g; i++)
                if (!mbar_wait(&full[i % STAGES], (i / STAGES) & 1)) *abort_flag = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer: unit j of this CTA accumulates in TMEM columns (j & 1) * BN
            const uint32_t idesc = tc_idesc(BN);
            uint32_t g = 0;
            bool stop = false;
            int j = 0;
            for (int u = blockIdx.x; u < units && !stop; u += gridDim.x, j++) {
                const int split = u / out.nmt;
                const int kb0 = split * out.kb_per_split, kb1 = min(kb0 + out.kb_per_split, out.nkb);
                const int a = j & 1;
                const uint32_t acc = tmem + (uint32_t)(a * BN);
                if (j >= 2 && !tc_wait(&tempty[a], ((j >> 1) - 1) & 1, abort_flag)) {
                    *abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int kb = kb0; kb < kb1; kb++, g++) {
                    const uint32_t s = g % STAGES, use = g / STAGES;
                    if (!tc_wait(&full[s], use & 1, abort_flag)) {
                        *abort_flag = 1;
                        stop = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = smem_u32(ring + s * tc_stage_bytes(BN));
                    const uint64_t ah = tc_desc(base), al = tc_desc(base + A_BYTES);
                    const uint64_t bh = tc_desc(base + 2 * A_BYTES), bl = tc_desc(base + 2 * A_BYTES + B_BYTES);
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 16; kk++) {
                        const uint64_t o = (uint64_t)(kk * 32 >> 4);
                        tc_mma(acc, ah + o, bh + o, idesc, (kb > kb0 || kk > 0) ? 1u : 0u);
                        tc_mma(acc, ah + o, bl + o, idesc, 1u);
                        tc_mma(acc, al + o, bh + o, idesc, 1u);
                    }
                    tc_commit(&empty[s]);
                }
                if (!stop) tc_commit(&tfull[a]);   // arrives once the unit's MMAs have completed
            }
            tc_commit(done);
            if (!mbar_wait(done, 0)) *abort_flag = 1;
        }
    } else {
        // epilogue warps
        const int q = warp & 3;
        int j = 0;
        for (int u = blockIdx.x; u < units; u += gridDim.x, j++) {
            const int mt = u % out.nmt, split = u / out.nmt;
            const int kb0 = split * out.kb_per_split, kb1 = min(kb0 + out.kb_per_split, out.nkb);
            const int a = j & 1;
            bool ok = tc_wait(&tfull[a], (j >> 1) & 1, abort_flag);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) {
                if (lane == 0) *(volatile int *)abort_flag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            tc_store_unit<BN>(tmem + (uint32_t)(a * BN), out, mt, split, q, lane, kb1 > kb0);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[a]);
        }
    }
    __syncwarp();
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0 && *(volatile int *)abort_flag) atomicExch(err_flag, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

// V of the R networks of a stage -> BF16 hi/lo, swizzled tiles of rpad rows
// per 64 reduction elements (zero padded); V of network r is
// Vbase[vmul * r * N + l]. One thread per (row, element).
__global__ void tc_pack_v_kernel(const double *__restrict__ Vbase, int vmul, int64_t N, int R, int rpad,
                                 int64_t kpad, __nv_bfloat16 *__restrict__ Bh, __nv_bfloat16 *__restrict__ Bl)
{
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)rpad * kpad) return;
    const int r = (int)(idx / kpad);
    const int64_t l = idx - (int64_t)r * kpad;
    double x = (r < R && l < N) ? Vbase[(int64_t)vmul * r * N + l] : 0.0;
    const __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    const __nv_bfloat16 lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    const int64_t o = (l / TC_BK) * ((int64_t)rpad * TC_BK) + tc_swz(r, l % TC_BK);
    Bh[o] = h;
    Bl[o] = lo;
}

// Kernel matrix of the shared geometry as BF16 hi/lo swizzled tiles (row
// block mt, reduction block kb at tile mt * nkb + kb): shear rows 0..N-1,
// normal rows N..2N-1 (mode II); padding stays zero.
__device__ __forceinline__ int64_t tc_a_index(int64_t m, int64_t l, int64_t nkb)
{
    return ((m / TC_BM) * nkb + l / TC_BK) * (TC_BM * TC_BK) + tc_swz(m % TC_BM, l % TC_BK);
}

template <int MODE>
__global__ void tc_assemble_kernel(int64_t N, int64_t kpad, const double *__restrict__ node,
                                   const double *__restrict__ elem, const double *__restrict__ tan,
                                   const double *__restrict__ nrm, __nv_bfloat16 *__restrict__ Ah,
                                   __nv_bfloat16 *__restrict__ Al)
{
    const int64_t k = blockIdx.x;
    const int64_t l = blockIdx.y * (int64_t)blockDim.x + threadIdx.x;
    if (k >= N || l >= N) return;
    const double e1 = elem[2 * k], e2 = elem[2 * k + 1];
    const double xl = node[2 * l], yl = node[2 * l + 1], xr = node[2 * l + 2], yr = node[2 * l + 3];
    double T = 0.0, Nn = 0.0;
    if (MODE == 3) T = entry_mode3(e1, e2, tan[2 * k], tan[2 * k + 1], xl, yl, xr, yr);
    else entry_mode2(e1, e2, nrm[2 * k], nrm[2 * k + 1], xl, yl, xr, yr, nrm[2 * l], nrm[2 * l + 1], T, Nn);
    const int64_t nkb = kpad / TC_BK;
    __nv_bfloat16 h, lo;
    split_bf16(T, h, lo);
    Ah[tc_a_index(k, l, nkb)] = h;
    Al[tc_a_index(k, l, nkb)] = lo;
    if (MODE == 2) {
        split_bf16(Nn, h, lo);
        Ah[tc_a_index(N + k, l, nkb)] = h;
        Al[tc_a_index(N + k, l, nkb)] = lo;
    }
}
