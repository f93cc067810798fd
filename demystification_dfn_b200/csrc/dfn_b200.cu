// dfn_b200.cu — C ABI (include/dfn_b200.h) over the sm_100a kernels of
// dfn_device.cuh. Host code here only sequences launches on the handle's
// stream and moves caller buffers; every arithmetic step of the hot path runs
// on the GPU. There is no CPU fallback: without a usable CUDA device,
// dfn_create fails with DFN_ERR_CUDA.
//
// A handle holds a batch of independent networks (a single network is a
// batch of one). Each "round" gives every active network one RK attempt:
// networks starting a step do the probe and the scaling RHS first, networks
// whose last attempt was rejected retry with their new step. Every kernel is
// predicated on the network's phase, so the host launches rounds back to back
// and reads the controllers only between groups of rounds.
#include "../../include/dfn_b200.h"
#include "dfn_device.cuh"
#include "hmat_device.cuh"
#include "newton.cuh"
#include "tc_gemm.cuh"
#include "kv_shared64.cuh"

#include <algorithm>
#include <cmath>
#include <unordered_map>
#include <array>
#include <deque>
#include <map>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

void set_err(const char *what, cudaError_t e, const char *file, int line)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_err = buf;
}

#define CK(x)                                                                                       \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) {                                                                    \
            set_err(#x, e_, __FILE__, __LINE__);                                                    \
            return (e_ == cudaErrorMemoryAllocation) ? DFN_ERR_NOMEM : DFN_ERR_CUDA;                \
        }                                                                                           \
    } while (0)

#define CKL()                                                                                       \
    do {                                                                                            \
        cudaError_t e_ = cudaGetLastError();                                                        \
        if (e_ != cudaSuccess) {                                                                    \
            set_err("kernel launch", e_, __FILE__, __LINE__);                                       \
            return DFN_ERR_CUDA;                                                                    \
        }                                                                                           \
    } while (0)

#define TRY(x)                       \
    do {                             \
        int s_ = (x);                \
        if (s_ != DFN_OK) return s_; \
    } while (0)

unsigned blocks_of(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int bytes_per_col(int mode, int store)
{
    const bool f64 = store == DFN_STORE_FP64 || store == DFN_STORE_FP64_SHARED;
    if (mode == DFN_MODE_II) return f64 ? 16 : 8;
    return f64 ? 8 : 4;
}

}  // namespace

struct dfn_handle {
    int dev = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // CUDA graph of kGraphRounds rounds of the solve loop, replayed on the
    // handle's stream (captured on cap_stream: capture needs a stream other
    // than the legacy default one a caller may have set)
    cudaStream_t cap_stream = nullptr;
    // H-matrix K.V: the low-rank leaves run on side_stream beside the dense
    // rows (fork after the permutation, join before the row sums)
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_pfork = nullptr, ev_pjoin = nullptr;   // pressure solves beside a K.V
    cudaStream_t side_lo = nullptr;       // lowest priority: tiled pressure filling around the tensor-core GEMM
    cudaGraphExec_t graph_exec = nullptr;
    int64_t graph_kernels = 0;
    bool use_graphs = true;
    int B = 1;                    // networks in the batch
    int mode = 2, store = 0, pressure = 0, gemv_impl = 0, max_attempts = 64;
    int64_t Ntot = 0;             // elements of all networks
    std::vector<Inst> hinst;      // host copy of the instance table
    Inst *inst = nullptr;
    int *inst_of = nullptr;
    int4 *tiles = nullptr;
    int64_t ntiles = 0, ntiles0 = 0;      // all tiles / tiles of network 0
    int64_t *seg_start = nullptr;
    int *seg_inst = nullptr;
    int64_t nseg = 0, nseg0 = 0;
    int *long_seg = nullptr;              // segments longer than TRI_SHORT_MAX
    int64_t nlong = 0, nlong0 = 0;
    int *short_seg = nullptr;             // the others
    int64_t nshort = 0, nshort0 = 0;
    int tri_shape = 0;                    // short segments: 0 a warp each, 1 a thread each, 2 tiles
    int2 *tri_tiles = nullptr;            // tiles of consecutive short segments (first in short_seg, count)
    int64_t ntri_tiles = 0, ntri_tiles0 = 0;
    int64_t nsrc_tot = 0, part_tot = 0;
    // geometry and parameters (concatenated)
    double *node = nullptr, *elem = nullptr, *ds = nullptr, *tan = nullptr, *nrm = nullptr, *permx = nullptr;
    double *a = nullptr, *b = nullptr, *Dc = nullptr, *f0 = nullptr, *V0 = nullptr, *nload = nullptr,
           *sload = nullptr, *perm = nullptr;
    unsigned char *fake = nullptr;
    int64_t *src_fault = nullptr, *src_elem = nullptr;
    double *src_Q = nullptr, *src_tb = nullptr, *src_te = nullptr;
    // state and work
    double *Y = nullptr, *P = nullptr, *Pdot = nullptr, *yout = nullptr, *yscal = nullptr, *ytmp = nullptr;
    double *kbuf = nullptr, *SigT = nullptr, *SigN = nullptr, *partT = nullptr, *partN = nullptr;
    double *Ptemp = nullptr, *Pdot_s = nullptr, *pwork = nullptr, *vin = nullptr, *vout = nullptr, *snap = nullptr;
    double *pcoef = nullptr;              // CG row coefficients [6][3N] per network
    // slip of the V formulation, integrated by the same Cash-Karp stages
    // outside the error norm: committed, the attempt's 5th-order value, and
    // the partial stage sum C1 V1 + C3 V3 + C4 V4
    double *slip = nullptr, *slip_out = nullptr, *slip_acc = nullptr;
    // permeability evolution (permeability_coupling = 1): k*, kmin, Snk
    bool pcoup = false;
    double *kstar = nullptr, *kmin = nullptr, *Snk = nullptr;
    int *err_flag = nullptr;
    int wait_polls = MBAR_POLLS;          // polls of the TMA K.V pipeline's bounded waits
    void *K = nullptr;
    size_t K_bytes = 0;
    int64_t kv_bytes = 0;         // algorithmic bytes of one K.V over the batch
    // shared-geometry batch on tensor cores (DFN_STORE_BF16X2_TC)
    bool tc = false;
    int tc_bn = 0, tc_nmt = 0, tc_split = 1, tc_kps = 0, tc_nkb = 0;
    int tc_variant = 0;                   // 0 persistent, 1 unit per CTA deepest ring, 2 unit per CTA 2-stage ring
    int sms = 148;                        // streaming multiprocessors of the device
    int pcl = 0, pcl_n = 0, pcl_max = 0;  // cluster CG: CTAs per cluster, largest range, clusters at once
    int pcl_mode = -1;                    // -1: clusters when they all fit at once, 0: one CTA on global memory,
                                          // 1: clusters, 2: one CTA with shared-memory vectors (autotuner)
    bool pcl_lean = false;                // x in global memory, M p recomputed (long ranges)
    bool pcl_ok = false;                  // the shared-memory CG forms can be launched
    int64_t ncross = 0;                   // fault crossings over the batch
    int64_t *xptr = nullptr;              // [Ntot + 1] crossing rows of the pressure system
    XCon *xcon = nullptr;
    int64_t *xrows = nullptr, *xrows_ptr = nullptr;
    double *tcoef = nullptr;              // tridiagonal row factors (3 per element; tridiagonal handles)
    int64_t tc_kpad = 0, tc_mpad = 0, tc_mrows = 0;
    __nv_bfloat16 *tc_A = nullptr, *tc_B = nullptr;   // [hi | lo] each, swizzled tiles
    // shared-geometry batch in FP64 (DFN_STORE_FP64_SHARED): one K, splits of
    // the columns, packed V of all members per stage
    bool s64 = false;
    int s64_split = 1, s64_kps = 0, s64_nkc = 0, s64_rp = S64_MEM;
    double *s64_vt = nullptr;
    StepCtl *ctl = nullptr;
    StepCtl *h_ctl = nullptr;     // pinned mirror, B entries
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;
    PressGlobal pg{};
    // H-matrix representation (static_kernel = hmatrix)
    bool hmat = false;
    int ncomp = 1;                        // 2 in mode II (shear and normal), 1 in mode III
    HBlk *hblk = nullptr;
    HTask *ht1 = nullptr, *ht2 = nullptr;
    int64_t hn1 = 0, hn2 = 0, hn1_0 = 0, hn2_0 = 0;   // low-rank column tasks, low-rank row tasks
    int64_t hn3 = 0, hn3_0 = 0;                        // dense row tasks
    HTask *ht3 = nullptr;                              // dense leaf rows (setup: filling the values)
    HTask *htg = nullptr;                              // dense row tasks: (group, rows)
    HDGroup *hdg = nullptr;                            // dense leaves sharing a row cluster
    HDLeaf *hdl = nullptr;                             // their leaves
    int64_t hn4 = 0, hn4_0 = 0;                        // low-rank leaves done whole
    int *hl4 = nullptr;
    int64_t hn5 = 0, hn5_0 = 0;                        // small low-rank leaves done whole, one warp each
    int *hl5 = nullptr;                                // their blocks (one CTA each when small_form = 1)
    HLeafW *hlw = nullptr;                             // their descriptors (one warp each)
    int small_form = 0;                                // small leaves: 0 one warp each, 1 one CTA each
    int64_t hm_dense_grid = 0, hm_warp_grid = 0;       // CTAs of the dense-row and small-leaf kernels (0: one
                                                       // per task / per four leaves; else a persistent grid)
    void *hvals = nullptr;
    int *hperm = nullptr;
    int32_t *hsegof = nullptr;            // row sums: segment of every (component, row)
    int64_t *hsegptr = nullptr, *hsegbase = nullptr;   // a segment's slot bases
    double *hz = nullptr, *hout = nullptr, *hxp = nullptr;
    std::vector<int> hranks;              // rank of every low-rank leaf (report)
    int64_t hdense_vals = 0, hlr_vals = 0, hblocks = 0;
    // Newton formulation and the learned guess
    int form = 0, guess = 0, newton_maxit = 50;
    double newton_tol = 1e-13;
    double max_step = 86400.0;            // cap on t_try after an accepted step (the reference's one day)
    double *tau0 = nullptr, *wlast = nullptr, *vnow = nullptr;
    MlpTC *mlp = nullptr;                 // tensor-core image of the learned guess
    double mlp_gate = 1e-1;               // relative residual of the analytic start that calls for it
    float *rec_x = nullptr, *rec_t = nullptr;
    unsigned long long *rec_n = nullptr;
    long long rec_cap = 0;
    // K.V launch timing
    bool prof = false;
    std::vector<cudaEvent_t> pev;
    int pcount = 0;
};

static const int kProfMax = 16384;

// ---------------------------------------------------------------------------
// launch helpers

typedef void (*gemv_fn)(const int4 *, const Inst *, const StepCtl *, int, const uint4 *, const double *, int,
                        double *, double *);
typedef void (*gemv_tma_fn)(const int4 *, const Inst *, const StepCtl *, int, const uint4 *, const double *, int,
                            double *, double *, int, int *);

static gemv_fn pick_gemv(int mode, int store)
{
    if (mode == 2) {
        if (store == 0) return gemv_kernel<2, 0>;
        if (store == 1) return gemv_kernel<2, 1>;
        return gemv_kernel<2, 2>;
    }
    if (store == 0) return gemv_kernel<3, 0>;
    if (store == 1) return gemv_kernel<3, 1>;
    return gemv_kernel<3, 2>;
}
static gemv_tma_fn pick_gemv_tma(int mode, int store)
{
    if (mode == 2) {
        if (store == 0) return gemv_tma_kernel<2, 0>;
        if (store == 1) return gemv_tma_kernel<2, 1>;
        return gemv_tma_kernel<2, 2>;
    }
    if (store == 0) return gemv_tma_kernel<3, 0>;
    if (store == 1) return gemv_tma_kernel<3, 1>;
    return gemv_tma_kernel<3, 2>;
}

static const size_t kTmaSmem = TMA_STAGES * GEMV_CHUNK_BYTES + 2 * TMA_STAGES * sizeof(uint64_t);

// H-matrix K.V: low-rank products, leaf rows, fixed-order row gather.
static int launch_hmat(dfn_handle *h, int mask, const double *Vbase, int vmul, bool only0)
{
    const int64_t n1 = only0 ? h->hn1_0 : h->hn1, n2 = only0 ? h->hn2_0 : h->hn2;
    const int64_t n3 = only0 ? h->hn3_0 : h->hn3, n4 = only0 ? h->hn4_0 : h->hn4;
    const int64_t n5 = only0 ? h->hn5_0 : h->hn5;
    const int64_t ne = only0 ? h->hinst[0].N : h->Ntot;
    hm_permute_kernel<<<blocks_of(ne, 256), 256, 0, h->stream>>>(ne, h->inst_of, h->inst, h->ctl, mask, h->hperm,
                                                                 Vbase, vmul, h->hxp);
    h->launches++;
    CKL();

    // the low-rank leaves (latency-bound; the rows of the wide ones after
    // their z partials) on the side stream, issued first, beside the dense
    // rows (bandwidth-bound) on the handle's stream
    const bool fork = (n1 > 0 || n2 > 0 || n4 > 0 || n5 > 0) && n3 > 0 && h->side_stream;
    cudaStream_t ls = fork ? h->side_stream : h->stream;
    if (fork) {
        CK(cudaEventRecord(h->ev_fork, h->stream));
        CK(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
    }
    if (n5 > 0 && h->small_form == 1) {
        if (h->store == 0)
            hm_lowrank_fused_kernel<double><<<(unsigned)n5, 256, 0, ls>>>(
                h->hl5, h->hblk, h->inst, h->ctl, mask, (const double *)h->hvals, h->hxp, h->hout);
        else
            hm_lowrank_fused_kernel<float><<<(unsigned)n5, 256, 0, ls>>>(
                h->hl5, h->hblk, h->inst, h->ctl, mask, (const float *)h->hvals, h->hxp, h->hout);
        h->launches++;
        CKL();
    } else if (n5 > 0) {
        const int64_t gfull = (n5 + 3) / 4;
        if (h->hm_warp_grid > 0 && h->hm_warp_grid < gfull) {
            const unsigned g = (unsigned)h->hm_warp_grid;
            if (h->store == 0)
                hm_lowrank_warp_persistent_kernel<double><<<g, 128, 0, ls>>>(
                    h->hlw, n5, h->ctl, mask, (const double *)h->hvals, h->hxp, h->hout);
            else
                hm_lowrank_warp_persistent_kernel<float><<<g, 128, 0, ls>>>(
                    h->hlw, n5, h->ctl, mask, (const float *)h->hvals, h->hxp, h->hout);
        } else {
            if (h->store == 0)
                hm_lowrank_warp_kernel<double><<<(unsigned)gfull, 128, 0, ls>>>(
                    h->hlw, n5, h->ctl, mask, (const double *)h->hvals, h->hxp, h->hout);
            else
                hm_lowrank_warp_kernel<float><<<(unsigned)gfull, 128, 0, ls>>>(
                    h->hlw, n5, h->ctl, mask, (const float *)h->hvals, h->hxp, h->hout);
        }
        h->launches++;
        CKL();
    }
    if (n4 > 0) {
        if (h->store == 0)
            hm_lowrank_fused_kernel<double><<<(unsigned)n4, 256, 0, ls>>>(
                h->hl4, h->hblk, h->inst, h->ctl, mask, (const double *)h->hvals, h->hxp, h->hout);
        else
            hm_lowrank_fused_kernel<float><<<(unsigned)n4, 256, 0, ls>>>(
                h->hl4, h->hblk, h->inst, h->ctl, mask, (const float *)h->hvals, h->hxp, h->hout);
        h->launches++;
        CKL();
    }
    if (n1 > 0) {
        if (h->store == 0)
            hm_lowrank_kernel<double><<<(unsigned)n1, 256, 0, ls>>>(
                h->ht1, h->hblk, h->inst, h->ctl, mask, (const double *)h->hvals, h->hxp, h->hz);
        else
            hm_lowrank_kernel<float><<<(unsigned)n1, 256, 0, ls>>>(
                h->ht1, h->hblk, h->inst, h->ctl, mask, (const float *)h->hvals, h->hxp, h->hz);
        h->launches++;
        CKL();
    }
    if (n2 > 0) {
        if (h->store == 0)
            hm_rows_kernel<double><<<(unsigned)n2, 256, 0, ls>>>(h->ht2, h->hblk, h->inst, h->ctl, mask,
                                                                        (const double *)h->hvals, h->hz, h->hout);
        else
            hm_rows_kernel<float><<<(unsigned)n2, 256, 0, ls>>>(h->ht2, h->hblk, h->inst, h->ctl, mask,
                                                                       (const float *)h->hvals, h->hz, h->hout);
        h->launches++;
        CKL();
    }
    if (n3 > 0) {
        if (h->hm_dense_grid > 0 && h->hm_dense_grid < n3) {
            const unsigned g3 = (unsigned)h->hm_dense_grid;
            if (h->store == 0)
                hm_dense_persistent_kernel<double><<<g3, 256, 0, h->stream>>>(
                    h->htg, n3, h->hdg, h->hdl, h->ctl, mask, (const double *)h->hvals, h->hxp, h->hout);
            else
                hm_dense_persistent_kernel<float><<<g3, 256, 0, h->stream>>>(
                    h->htg, n3, h->hdg, h->hdl, h->ctl, mask, (const float *)h->hvals, h->hxp, h->hout);
        } else {
            if (h->store == 0)
                hm_dense_kernel<double><<<(unsigned)n3, 256, 0, h->stream>>>(
                    h->htg, h->hdg, h->hdl, h->ctl, mask, (const double *)h->hvals, h->hxp, h->hout);
            else
                hm_dense_kernel<float><<<(unsigned)n3, 256, 0, h->stream>>>(
                    h->htg, h->hdg, h->hdl, h->ctl, mask, (const float *)h->hvals, h->hxp, h->hout);
        }
        h->launches++;
        CKL();
    }
    if (fork) {
        CK(cudaEventRecord(h->ev_join, h->side_stream));
        CK(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    }
    hm_gather_kernel<<<blocks_of(ne, 256), 256, 0, h->stream>>>(ne, h->ncomp, h->inst_of, h->inst, h->ctl, mask,
                                                                h->hperm, h->hsegof, h->hsegptr, h->hsegbase, h->hout,
                                                                h->partT,
                                                                h->partN);
    h->launches++;
    CKL();
    return DFN_OK;
}

// Shared-geometry K.V on tensor cores: V of every network to BF16 hi/lo rows,
// then one GEMM over (128-row tile, reduction split) work units.
template <int BN>
static void tc_launch_bn(dfn_handle *h, const TcOut &o)
{
    const int64_t na = h->tc_mpad * h->tc_kpad, nb = (int64_t)h->tc_bn * h->tc_kpad;
    const unsigned units = (unsigned)(h->tc_nmt * h->tc_split);
    if (h->tc_variant == 0) {
        const unsigned grid = std::min(units, (unsigned)h->sms);
        tc_gemm_persistent_kernel<BN, tc_stages(BN)><<<grid, TC_PTHREADS, tc_smem_bytes(BN, tc_stages(BN)),
                                                       h->stream>>>(h->tc_A, h->tc_A + na, h->tc_B, h->tc_B + nb, o,
                                                                    h->err_flag);
        return;
    }
    const unsigned grid = units;
    if (h->tc_variant == 2 && tc_stages(BN) > 2)
        tc_gemm_kernel<BN, 2><<<grid, TC_THREADS, tc_smem_bytes(BN, 2), h->stream>>>(
            h->tc_A, h->tc_A + na, h->tc_B, h->tc_B + nb, o, h->err_flag);
    else
        tc_gemm_kernel<BN, tc_stages(BN)><<<grid, TC_THREADS, tc_smem_bytes(BN, tc_stages(BN)), h->stream>>>(
            h->tc_A, h->tc_A + na, h->tc_B, h->tc_B + nb, o, h->err_flag);
}

static int launch_tc(dfn_handle *h, const double *Vbase, int vmul)
{
    const Inst &I = h->hinst[0];
    const int64_t nb = (int64_t)h->tc_bn * h->tc_kpad;
    tc_pack_v_kernel<<<blocks_of(nb, 256), 256, 0, h->stream>>>(Vbase, vmul, I.N, h->B, h->tc_bn, h->tc_kpad,
                                                                h->tc_B, h->tc_B + nb);
    h->launches++;
    CKL();
    TcOut o;
    o.partT = h->partT; o.partN = h->partN; o.inst = h->inst; o.N = I.N; o.mrows = h->tc_mrows; o.R = h->B;
    o.kb_per_split = h->tc_kps; o.nkb = h->tc_nkb; o.nmt = h->tc_nmt; o.nsplit = h->tc_split;
    switch (h->tc_bn) {
    case 16: tc_launch_bn<16>(h, o); break;
    case 32: tc_launch_bn<32>(h, o); break;
    case 64: tc_launch_bn<64>(h, o); break;
    case 128: tc_launch_bn<128>(h, o); break;
    default: tc_launch_bn<256>(h, o); break;
    }
    return DFN_OK;
}

// Shared-geometry K.V in FP64: V of every member packed per column, then one
// GEMM over (row tile, member tile, column split).
static int launch_s64(dfn_handle *h, const double *Vbase, int vmul)
{
    const Inst &I = h->hinst[0];
    const int64_t nv = I.Np * h->s64_rp;
    s64_pack_v_kernel<<<blocks_of(nv, 256), 256, 0, h->stream>>>(Vbase, vmul, h->inst, I.N, h->B, h->s64_rp, I.Np,
                                                                 h->s64_vt);
    h->launches++;
    CKL();
    dim3 grid((unsigned)((I.N + S64_ROWS - 1) / S64_ROWS), (unsigned)(h->s64_rp / S64_MEM), (unsigned)h->s64_split);
    const double *K = static_cast<const double *>(h->K);
    if (h->mode == DFN_MODE_II)
        s64_gemm_kernel<2><<<grid, S64_THREADS, s64_smem_bytes(2), h->stream>>>(
            K, h->s64_vt, h->inst, I.N, I.Np, h->B, h->s64_rp, h->s64_kps, h->s64_nkc, h->partT, h->partN);
    else
        s64_gemm_kernel<3><<<grid, S64_THREADS, s64_smem_bytes(3), h->stream>>>(
            K, h->s64_vt, h->inst, I.N, I.Np, h->B, h->s64_rp, h->s64_kps, h->s64_nkc, h->partT, h->partN);
    return DFN_OK;
}

// K.V of all networks (only0 = false) or of network 0 (only0 = true);
// V of network i is Vbase[vmul*eoff_i + l].
static int launch_gemv(dfn_handle *h, int mask, const double *Vbase, int vmul, bool only0)
{
    const bool rec = h->prof && h->pcount < kProfMax;
    if (rec) CK(cudaEventRecord(h->pev[2 * h->pcount], h->stream));
    const uint4 *K = static_cast<const uint4 *>(h->K);
    const int64_t ntiles = only0 ? h->ntiles0 : h->ntiles;
    if (h->hmat) {
        TRY(launch_hmat(h, mask, Vbase, vmul, only0));
    } else if (h->tc) {
        TRY(launch_tc(h, Vbase, vmul));
    } else if (h->s64) {
        TRY(launch_s64(h, Vbase, vmul));
    } else if (h->gemv_impl == 0) {
        gemv_tma_fn fn = pick_gemv_tma(h->mode, h->store);
        fn<<<(unsigned)ntiles, (TMA_CONSUMERS + 1) * 32, kTmaSmem, h->stream>>>(
            h->tiles, h->inst, h->ctl, mask, K, Vbase, vmul, h->partT, h->partN, h->wait_polls, h->err_flag);
    } else {
        gemv_fn fn = pick_gemv(h->mode, h->store);
        fn<<<(unsigned)ntiles, GEMV_WARPS * 32, 0, h->stream>>>(h->tiles, h->inst, h->ctl, mask, K, Vbase, vmul,
                                                                h->partT, h->partN);
    }
    h->launches++;
    CKL();
    if (rec) {
        CK(cudaEventRecord(h->pev[2 * h->pcount + 1], h->stream));
        h->pcount++;
    }
    return DFN_OK;
}

// Pressure systems sys0..sys0+nsys-1 of the first `ninst` networks.
static void pcl_config(cudaLaunchConfig_t &cfg, cudaLaunchAttribute *at, int cl, int n, bool lean, unsigned gx,
                       unsigned gy, cudaStream_t stream)
{
    cfg = cudaLaunchConfig_t{};
    cfg.gridDim = dim3(gx, gy);
    cfg.blockDim = dim3(PCL_THREADS);
    cfg.dynamicSmemBytes = cl == 1 ? (size_t)PCL_SMEM_CAP : pcl_smem_bytes(n, lean);
    cfg.stream = stream;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
}

static int launch_pressure(dfn_handle *h, int mask, int kind, int sys0, int nsys, double dt_explicit, int ninst)
{
    const bool clusters = h->pcl > 0 && (h->pcl_mode == 1 || (h->pcl_mode < 0 && nsys * ninst <= h->pcl_max));
    const int cl = h->pcl_mode == 2 ? 1 : (clusters ? h->pcl : 0);
    if (h->pressure == DFN_PRESSURE_CG && cl > 0) {
        // one cluster of cl CTAs per system, vectors in shared memory
        cudaLaunchConfig_t cfg;
        cudaLaunchAttribute at[1];
        pcl_config(cfg, at, cl, h->pcl_n, h->pcl_lean, (unsigned)(nsys * cl), (unsigned)ninst, h->stream);
        CK(cudaLaunchKernelEx(&cfg, pressure_cg_cluster_kernel, h->pg, (const Inst *)h->inst, h->ctl, mask, kind,
                              sys0, dt_explicit, h->Ptemp, h->Pdot_s, h->pwork, h->pcl_lean ? 1 : 0, h->pcoef));
    } else if (h->pressure != DFN_PRESSURE_TRIDIAG) {
        dim3 grid((unsigned)nsys, (unsigned)ninst);
        const int exact = h->pressure == DFN_PRESSURE_CG_EXACT ? 1 : 0;
        if (h->ncross > 0)
            pressure_cg_batch_kernel<true><<<grid, 1024, 0, h->stream>>>(
                h->pg, h->inst, h->ctl, mask, kind, sys0, dt_explicit, h->Ptemp, h->Pdot_s, h->pwork, exact, h->pcoef);
        else
            pressure_cg_batch_kernel<false><<<grid, 1024, 0, h->stream>>>(
                h->pg, h->inst, h->ctl, mask, kind, sys0, dt_explicit, h->Ptemp, h->Pdot_s, h->pwork, exact, h->pcoef);
    } else {
        const int64_t nshort = (ninst == h->B) ? h->nshort : h->nshort0;
        const int64_t nlong = (ninst == h->B) ? h->nlong : h->nlong0;
        if (nshort > 0 && h->tri_shape == 2) {
            const int64_t nt = (ninst == h->B) ? h->ntri_tiles : h->ntri_tiles0;
            dim3 grid((unsigned)nt, (unsigned)nsys);
            pressure_tridiag_tile_kernel<<<grid, 128, 0, h->stream>>>(h->pg, h->inst, h->ctl, mask, kind, sys0,
                                                                      dt_explicit, h->seg_start, h->seg_inst,
                                                                      h->short_seg, h->tri_tiles, h->Ptemp,
                                                                      h->Pdot_s);
            if (nlong > 0) {
                h->launches++;
                CKL();
            }
        } else if (nshort > 0 && h->tri_shape == 1) {
            dim3 grid((unsigned)((nshort + 127) / 128), (unsigned)nsys);
            pressure_tridiag_thread_kernel<<<grid, 128, 0, h->stream>>>(h->pg, h->inst, h->ctl, mask, kind, sys0,
                                                                        dt_explicit, h->seg_start, h->seg_inst,
                                                                        h->short_seg, nshort, h->Ptemp, h->Pdot_s,
                                                                        h->pwork);
            if (nlong > 0) {
                h->launches++;
                CKL();
            }
        } else if (nshort > 0) {
            dim3 grid((unsigned)((nshort + 7) / 8), (unsigned)nsys);
            pressure_tridiag_kernel<<<grid, 256, 0, h->stream>>>(h->pg, h->inst, h->ctl, mask, kind, sys0,
                                                                 dt_explicit, h->seg_start, h->seg_inst,
                                                                 h->short_seg, nshort, h->Ptemp, h->Pdot_s, h->pwork);
            if (nlong > 0) {
                h->launches++;
                CKL();
            }
        }
        if (nlong > 0) {
            dim3 lgrid((unsigned)nlong, (unsigned)nsys);
            pressure_tridiag_long_kernel<<<lgrid, TRI_NT, 0, h->stream>>>(
                h->pg, h->inst, h->ctl, mask, kind, sys0, dt_explicit, h->seg_start, h->seg_inst, h->long_seg,
                h->Ptemp, h->Pdot_s, h->pwork);
        }
    }
    h->launches++;
    CKL();
    return DFN_OK;
}

static FricParams fric_params(dfn_handle *h, int64_t nelem)
{
    FricParams f;
    f.Ntot = nelem; f.mode = h->mode; f.inst = h->inst; f.inst_of = h->inst_of;
    f.a = h->a; f.b = h->b; f.Dc = h->Dc; f.f0 = h->f0; f.V0 = h->V0; f.nload = h->nload; f.sload = h->sload;
    f.fake = h->fake; f.partT = h->partT; f.partN = h->partN; f.SigT = h->SigT; f.SigN = h->SigN;
    f.Ptemp = h->Ptemp; f.Pdot = h->Pdot_s; f.Pc = h->P; f.y = h->Y; f.ytmp = h->ytmp; f.kbuf = h->kbuf; f.yscal = h->yscal;
    f.yout = h->yout; f.ctl = h->ctl;
    f.form = h->form; f.guess = h->guess; f.maxit = h->newton_maxit; f.tol = h->newton_tol; f.off_explicit = 0.0;
    f.tau0 = h->tau0; f.wlast = h->wlast; f.vnow = h->vnow; f.mlp = h->mlp; f.mlp_gate = h->mlp_gate;
    f.slip = h->slip; f.slip_out = h->slip_out; f.slip_acc = h->slip_acc;
    f.rec_x = h->rec_x; f.rec_t = h->rec_t; f.rec_n = h->rec_n; f.rec_cap = h->rec_cap;
    return f;
}

static int launch_friction(dfn_handle *h, int stage, int sys, int mask, int64_t nelem, double off_explicit = 0.0)
{
    FricParams f = fric_params(h, nelem);
    f.off_explicit = off_explicit;
    // 128-thread blocks: five per SM at the register count (two of 256)
    if (h->form == DFN_FORM_NEWTON && h->guess == DFN_GUESS_MLP)
        friction_kernel<true><<<(unsigned)((nelem + 127) / 128), 128, 0, h->stream>>>(f, stage, sys, mask);
    else
        friction_kernel<false><<<(unsigned)((nelem + 127) / 128), 128, 0, h->stream>>>(f, stage, sys, mask);
    h->launches++;
    CKL();
    return DFN_OK;
}

static ElemParams elem_params(dfn_handle *h)
{
    ElemParams ep;
    ep.Ntot = h->Ntot; ep.inst = h->inst; ep.inst_of = h->inst_of; ep.ctl = h->ctl;
    return ep;
}


// Pressure solves beside the K.V that follows them (they depend only on the
// stage times, not on the stage state); the stage kernel that reads them
// waits for the join. Returns the stream: the high-priority one for the CG on
// a few thread-block clusters (at most half the SMs: placed first, the K.V
// streams on the others), the lowest-priority one for the tiled tridiagonal
// solve of a tensor-core batch (one tile CTA fits beside each persistent GEMM
// CTA; issued after the GEMM, so that the GEMM's CTAs are placed first and the
// tiles fill around them), or none (in line). The fork event is recorded
// before the K.V in both cases.
static cudaStream_t pressure_beside(dfn_handle *h, int nsys, int ninst)
{
    if (!h->side_stream) return nullptr;
    if (h->pressure == DFN_PRESSURE_TRIDIAG)
        return (h->tc && h->tc_variant == 0 && h->tri_shape == 2 && h->nlong == 0) ? h->side_lo : nullptr;
    if (h->pressure != DFN_PRESSURE_CG || h->pcl <= 0 || h->pcl_mode == 0 || h->pcl_mode == 2) return nullptr;
    if (h->pcl_mode < 0 && (int64_t)nsys * ninst > h->pcl_max) return nullptr;
    return ((int64_t)nsys * ninst * h->pcl <= h->sms / 2) ? h->side_stream : nullptr;
}

static int launch_pressure_side(dfn_handle *h, cudaStream_t side, int mask, int kind, int sys0, int nsys, int ninst)
{
    CK(cudaStreamWaitEvent(side, h->ev_pfork, 0));
    cudaStream_t main = h->stream;
    h->stream = side;
    const int st = launch_pressure(h, mask, kind, sys0, nsys, 0.0, ninst);
    h->stream = main;
    TRY(st);
    CK(cudaEventRecord(h->ev_pjoin, side));
    return DFN_OK;
}

// One RK attempt (stages 2..6 and the error test) of every network in `mask`.
static int run_attempt(dfn_handle *h, int mask)
{
    attempt_begin_kernel<<<blocks_of(h->Ntot, 256), 256, 0, h->stream>>>(elem_params(h), h->Y, h->kbuf, h->ytmp,
                                                                         mask);
    h->launches++;
    CKL();
    // the Newton formulation interpolates the stage pressure in time and
    // needs only the full-step system (c = 1)
    const int sys0 = h->form == DFN_FORM_NEWTON ? 4 : 1, nsys = h->form == DFN_FORM_NEWTON ? 1 : 5;
    cudaStream_t side = pressure_beside(h, nsys, h->B);
    const bool beside = side != nullptr, after = side == h->side_lo;
    if (beside) CK(cudaEventRecord(h->ev_pfork, h->stream));
    if (beside && !after) TRY(launch_pressure_side(h, side, mask, 1, sys0, nsys, h->B));
    else if (!beside) TRY(launch_pressure(h, mask, 1, sys0, nsys, 0.0, h->B));
    for (int s = 2; s <= 6; s++) {
        TRY(launch_gemv(h, mask, h->ytmp, 3, false));
        if (s == 2 && after) TRY(launch_pressure_side(h, side, mask, 1, sys0, nsys, h->B));
        if (s == 2 && beside) CK(cudaStreamWaitEvent(h->stream, h->ev_pjoin, 0));
        TRY(launch_friction(h, s, s - 1, mask, h->Ntot));
    }
    decide_kernel<<<blocks_of(h->B, 128), 128, 0, h->stream>>>(h->ctl, h->B, mask);
    h->launches++;
    CKL();
    return DFN_OK;
}

// Permeability coupling: the permeability and face values of the networks
// in `mask` from their committed sigmaN and P (accepted_only: those whose
// attempt of this round was accepted), then the tridiagonal row factors.
static int perm_refresh(dfn_handle *h, int mask, int accepted_only)
{
    perm_update_kernel<<<blocks_of(h->Ntot, 256), 256, 0, h->stream>>>(elem_params(h), mask, accepted_only, h->Y,
                                                                        h->P, h->kstar, h->kmin, h->Snk, h->perm,
                                                                        h->permx);
    h->launches++;
    CKL();
    if (h->tcoef) {
        tri_coef_kernel<<<blocks_of(h->Ntot, 256), 256, 0, h->stream>>>(h->pg, h->inst, h->inst_of, h->Ntot,
                                                                        h->tcoef);
        h->launches++;
        CKL();
    }
    return DFN_OK;
}

// One round of the solve() loop for every network of the batch.
static int run_round(dfn_handle *h)
{
    const unsigned bb = blocks_of(h->B, 128);
    step_begin_kernel<<<bb, 128, 0, h->stream>>>(h->ctl, h->inst, h->B, h->src_tb);
    h->launches++;
    CKL();
    // coupled permeability of a new step: from sigmaN and P committed
    if (h->pcoup) TRY(perm_refresh(h, M_NEW, 0));
    // CG probe at t_try (halving on non-convergence); its solution is the
    // pressure of the scaling RHS evaluated at dt = t_try (src/solver.f90:81-101).
    cudaStream_t side = pressure_beside(h, 1, h->B);
    const bool beside = side != nullptr, after = side == h->side_lo;
    if (beside) CK(cudaEventRecord(h->ev_pfork, h->stream));
    if (beside && !after) TRY(launch_pressure_side(h, side, M_NEW, 0, 0, 1, h->B));
    else if (!beside) TRY(launch_pressure(h, M_NEW, 0, 0, 1, 0.0, h->B));
    TRY(launch_gemv(h, M_NEW, h->Y, 3, false));
    if (after) TRY(launch_pressure_side(h, side, M_NEW, 0, 0, 1, h->B));
    if (beside) CK(cudaStreamWaitEvent(h->stream, h->ev_pjoin, 0));
    TRY(launch_friction(h, 1, 0, M_NEW, h->Ntot));
    set_h_kernel<<<bb, 128, 0, h->stream>>>(h->ctl, h->B);
    h->launches++;
    CKL();
    TRY(run_attempt(h, M_ACTIVE));
    commit_kernel<<<blocks_of(h->Ntot, 256), 256, 0, h->stream>>>(
        elem_params(h), h->Y, h->yout, h->P, h->Pdot, h->Ptemp, h->Pdot_s,
        h->form == DFN_FORM_NEWTON ? nullptr : h->slip, h->slip_out, h->pcoup ? 0 : 1);
    h->launches++;
    CKL();
    if (h->pcoup) {
        // the reference's commit compute_P(t_did) sees the new sigmaN and the
        // old P (src/solver.f90:174 after rkqs): its own solve, not the
        // stage-5 one, then P committed where it converged
        TRY(perm_refresh(h, M_ACTIVE, 1));
        TRY(launch_pressure(h, M_ACTIVE, 3, 5, 1, 0.0, h->B));
        commit_p_kernel<<<blocks_of(h->Ntot, 256), 256, 0, h->stream>>>(elem_params(h), h->P, h->Pdot, h->Ptemp,
                                                                        h->Pdot_s);
        h->launches++;
        CKL();
    }
    finish_kernel<<<bb, 128, 0, h->stream>>>(h->ctl, h->B, h->max_step);
    h->launches++;
    CKL();
    return DFN_OK;
}

static int sync_ctl(dfn_handle *h)
{
    CK(cudaMemcpyAsync(h->h_ctl, h->ctl, sizeof(StepCtl) * h->B, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int flag = 0;
    CK(cudaMemcpy(&flag, h->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        // reported once: the flag is cleared so that the handle can be
        // reused after the caller has restored its state
        CK(cudaMemsetAsync(h->err_flag, 0, sizeof(int), h->stream));
        g_err = "a bounded wait of a K.V pipeline expired (its partial sums are incomplete)";
        return DFN_ERR_TIMEOUT;
    }
    return DFN_OK;
}

static int put_ctl(dfn_handle *h)
{
    CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(StepCtl) * h->B, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DFN_OK;
}

// Advances every network by `nsteps` accepted steps, or until its time
// reaches t_end (> 0). Rounds are launched in groups; the controllers are
// read between groups only.
static const int64_t kGraphRounds = 8;

static void drop_graph(dfn_handle *h)
{
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
}

// Capture kGraphRounds rounds into an executable graph. Every kernel of a
// round reads the step controllers on the device, so the same graph serves
// every later replay; rounds of networks that are done are no-ops.
static int build_graph(dfn_handle *h)
{
    cudaStream_t saved = h->stream;
    const int64_t l0 = h->launches;
    cudaGraph_t g = nullptr;
    h->stream = h->cap_stream;
    cudaError_t e = cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal);
    int st = (e == cudaSuccess) ? DFN_OK : DFN_ERR_CUDA;
    for (int64_t r = 0; r < kGraphRounds && st == DFN_OK; r++) st = run_round(h);
    cudaError_t e2 = cudaStreamEndCapture(h->cap_stream, &g);
    h->stream = saved;
    h->graph_kernels = h->launches - l0;
    h->launches = l0;
    if (st == DFN_OK && e2 == cudaSuccess && g) {
        e = cudaGraphInstantiate(&h->graph_exec, g, cudaGraphInstantiateFlagUseNodePriority);
        if (e != cudaSuccess) {
            h->graph_exec = nullptr;
            st = DFN_ERR_CUDA;
        }
    } else if (st == DFN_OK) {
        st = DFN_ERR_CUDA;
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();   // a failed capture leaves nothing behind: direct launches follow
    return st;
}

// n rounds: whole graphs while possible (not while K.V launches are being
// timed one by one), then single launches.
static int run_rounds(dfn_handle *h, int64_t n)
{
    if (h->use_graphs && !h->prof && n >= kGraphRounds) {
        if (!h->graph_exec && build_graph(h) != DFN_OK) h->use_graphs = false;
        if (h->graph_exec) {
            for (; n >= kGraphRounds; n -= kGraphRounds) {
                CK(cudaGraphLaunch(h->graph_exec, h->stream));
                h->launches += h->graph_kernels;
            }
        }
    }
    for (int64_t r = 0; r < n; r++) TRY(run_round(h));
    return DFN_OK;
}

static int solve_impl(dfn_handle *h, int64_t nsteps, double t_end)
{
    arm_kernel<<<blocks_of(h->B, 128), 128, 0, h->stream>>>(h->ctl, h->B, (long long)nsteps, t_end,
                                                            h->max_attempts);
    h->launches++;
    CKL();
    int64_t group = (t_end > 0.0) ? 8 : std::max<int64_t>(nsteps, 1);
    for (int64_t guard = 0; guard < 1000000; guard++) {
        TRY(run_rounds(h, group));
        TRY(sync_ctl(h));
        int64_t remaining = 0;
        bool active = false;
        for (int i = 0; i < h->B; i++) {
            const StepCtl &c = h->h_ctl[i];
            if (c.phase == PH_DONE) continue;
            active = true;
            remaining = std::max<int64_t>(remaining, c.target_steps - c.steps_done);
        }
        if (!active) return DFN_OK;
        group = (t_end > 0.0) ? 8 : std::max<int64_t>(remaining, 1);
    }
    g_err = "solve did not finish";
    return DFN_ERR_ATTEMPTS;
}

static __global__ void snapshot_kernel(int64_t N, const double *Y, const double *Dc, const double *V0,
                                       const double *P, const double *SigT, double *out)
{
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= N) return;
    out[k] = Y[k];
    out[N + k] = Dc[k] / V0[k] * exp(Y[N + k]);
    out[2 * N + k] = P[k];
    out[3 * N + k] = SigT[k];
    out[4 * N + k] = Y[2 * N + k];
}

static void fill_report(const StepCtl &c, dfn_report *r)
{
    if (!r) return;
    r->it_count = c.it_count; r->attempts = c.attempts; r->rejected = c.rejected; r->rhs_evals = c.rhs_evals;
    r->cg_iterations = c.cg_iters; r->probe_halvings = c.halvings; r->time = c.time; r->t_try = c.t_try;
    r->last_hdid = c.hdid; r->status = c.status; r->pad = 0; r->stage_cg_failures = c.stage_noconv;
    r->newton_solves = c.newton_solves; r->newton_iters = c.newton_iters; r->newton_fail = c.newton_fail;
    r->mlp_warps = c.mlp_warps;
}

// ---------------------------------------------------------------------------
// H-matrix construction on the host (setup) and upload: hmat_build.h builds
// the cluster tree, the block leaves and the factors of each network from
// the element geometry the device computed; entries are the same formulas
// as the dense assembly (entry_mode2/entry_mode3).
struct HostLeaf {
    int dense, rank;
    int64_t foff, goff;         // low-rank: A'^T and B'^T offsets in the low-rank value region
};

// Device buffer owned by the build (freed on every return path).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    int reserve(size_t b)
    {
        if (b <= bytes) return DFN_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, b) != cudaSuccess) return DFN_ERR_NOMEM;
        bytes = b;
        return DFN_OK;
    }
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};
struct LrSegment {
    int64_t start, len;   // values of the low-rank region
    DevBuf buf;
};

// find_fault_crossing (src/initialisation.f90:279-344) for every network
// of the batch: node pairs of two faults closer than 0.01 times the smaller
// of the two faults' smallest element length. Each crossing couples the (up
// to) two elements around the node on one fault with those on the other;
// the pressure rows store, in crossing order, each coupling's partner
// elements and harmonic-mean permeabilities (XCon). Returns the crossings.
static int64_t build_crossings(const dfn_problem *probs, int count, const std::vector<Inst> &hinst,
                               std::vector<int64_t> &xptr, std::vector<XCon> &xcon)
{
    int64_t Ntot = 0;
    for (int i = 0; i < count; i++) Ntot += hinst[i].N;
    std::vector<std::vector<XCon>> rows((size_t)Ntot);
    int64_t ncross = 0;
    auto harm = [](double k1, double k2) { return (k1 + k2 > 0.0) ? 2.0 * k1 * k2 / (k1 + k2) : 0.0; };
    for (int i = 0; i < count; i++) {
        const dfn_problem &p = probs[i];
        const int64_t F = p.nb_fault, e0 = hinst[i].eoff;
        const double *nd = p.node, *perm = p.permeability;
        std::vector<int64_t> first((size_t)F), nel((size_t)F);
        std::vector<double> minds((size_t)F);
        int64_t cnt = 0;
        for (int64_t f = 0; f < F; f++) {
            first[f] = cnt;
            nel[f] = p.fault_nb_element[f];
            double m = INFINITY;
            for (int64_t e = cnt; e < cnt + nel[f]; e++) {
                const double dx = nd[2 * e + 2] - nd[2 * e], dy = nd[2 * e + 3] - nd[2 * e + 1];
                m = std::min(m, std::sqrt(dx * dx + dy * dy));
            }
            minds[f] = m;
            cnt += nel[f] + 1;
        }
        // candidate node pairs from a hashed grid whose cells are as large as
        // the largest pair threshold (a pair within its threshold lies in the
        // same or a neighbouring cell); crossings then in the reference's
        // loop order (fault 1, fault 2, node of fault 1, node of fault 2)
        double maxthr = 0.0;
        for (int64_t f = 0; f < F; f++) maxthr = std::max(maxthr, 0.01 * minds[f]);
        std::vector<std::array<int64_t, 4>> found;   // f1, f2, a, b (local 0-based nodes)
        if (maxthr > 0.0 && F > 1) {
            std::unordered_map<uint64_t, std::vector<std::pair<int64_t, int64_t>>> grid;   // cell -> (fault, node)
            auto cell = [&](double x, double y, int64_t dx, int64_t dy) {
                const int64_t cx = (int64_t)std::floor(x / maxthr) + dx, cy = (int64_t)std::floor(y / maxthr) + dy;
                return ((uint64_t)cx * 0x9E3779B97F4A7C15ull) ^ (uint64_t)cy;
            };
            for (int64_t f = 0; f < F; f++)
                for (int64_t a = 0; a <= nel[f]; a++) {
                    const double *q = nd + 2 * (first[f] + a);
                    grid[cell(q[0], q[1], 0, 0)].push_back({f, a});
                }
            for (int64_t f1 = 0; f1 < F; f1++)
                for (int64_t a = 0; a <= nel[f1]; a++) {
                    const double *p1 = nd + 2 * (first[f1] + a);
                    for (int64_t dx = -1; dx <= 1; dx++)
                        for (int64_t dy = -1; dy <= 1; dy++) {
                            auto it = grid.find(cell(p1[0], p1[1], dx, dy));
                            if (it == grid.end()) continue;
                            for (const auto &fb : it->second) {
                                const int64_t f2 = fb.first, b = fb.second;
                                if (f2 <= f1) continue;
                                const double *p2 = nd + 2 * (first[f2] + b);
                                // the same criterion as the reference's double loop
                                const double thr = 0.01 * std::min(minds[f1], minds[f2]);
                                const double d = std::sqrt((p1[0] - p2[0]) * (p1[0] - p2[0]) +
                                                           (p1[1] - p2[1]) * (p1[1] - p2[1]));
                                if (d < thr) found.push_back({f1, f2, a, b});
                            }
                        }
                }
            std::sort(found.begin(), found.end());
            found.erase(std::unique(found.begin(), found.end()), found.end());
        }
        for (const auto &c : found) {
            const int64_t f1 = c[0], f2 = c[1], a = c[2], b = c[3];
            ncross++;
            const int64_t e1[2] = {a >= 1 ? first[f1] + a - 1 : -1, a < nel[f1] ? first[f1] + a : -1};
            const int64_t e2[2] = {b >= 1 ? first[f2] + b - 1 : -1, b < nel[f2] ? first[f2] + b : -1};
            for (int side = 0; side < 2; side++)
                for (int j = 0; j < 2; j++) {
                    const int64_t row = side == 0 ? e1[j] : e2[j];
                    if (row < 0) continue;
                    const int64_t *o = side == 0 ? e2 : e1;
                    XCon x;
                    x.a = o[0] >= 0 ? o[0] : row;
                    x.b = o[1] >= 0 ? o[1] : row;
                    // harmonic means with the first fault's element first
                    if (side == 0) {
                        x.kl = o[0] >= 0 ? harm(perm[row], perm[o[0]]) : 0.0;
                        x.kr = o[1] >= 0 ? harm(perm[row], perm[o[1]]) : 0.0;
                    } else {
                        x.kl = o[0] >= 0 ? harm(perm[o[0]], perm[row]) : 0.0;
                        x.kr = o[1] >= 0 ? harm(perm[o[1]], perm[row]) : 0.0;
                    }
                    rows[(size_t)(e0 + row)].push_back(x);
                }
        }
    }
    xptr.assign((size_t)Ntot + 1, 0);
    xcon.clear();
    for (int64_t k = 0; k < Ntot; k++) {
        xcon.insert(xcon.end(), rows[(size_t)k].begin(), rows[(size_t)k].end());
        xptr[(size_t)k + 1] = (int64_t)xcon.size();
    }
    return ncross;
}

static int build_hmatrix(dfn_handle *h, const dfn_problem *probs, const dfn_options &opt)
{
    const int leaf = opt.hmat_leaf > 0 ? opt.hmat_leaf : 100;
    const double eta = opt.hmat_eta > 0 ? opt.hmat_eta : 3.0;
    const double eps = opt.hmat_eps > 0 ? opt.hmat_eps : 1e-8;
    const int B = h->B, nc = h->ncomp;
    const int64_t Nt = h->Ntot;
    std::vector<double> el(2 * Nt);   // midpoints: cluster tree and admissibility on the host
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(el.data(), h->elem, sizeof(double) * 2 * Nt, cudaMemcpyDeviceToHost));

    // values per 16-byte vector of the stored type; factor rows padded to it
    const int VW = h->store == DFN_STORE_FP64 ? 2 : 4;
    auto rup = [VW](int64_t n) { return (n + VW - 1) / VW * VW; };
    std::vector<int> perm(Nt);
    std::vector<HBlk> blks;
    std::vector<HTask> t1, t2, t3, tg;
    std::vector<HDGroup> dgroups;   // dense leaves by row cluster, and their row tasks
    std::vector<HDLeaf> dleaves;
    std::vector<int> l4;
    std::vector<int> l5;     // small whole low-rank leaves (one warp each), and their descriptors
    std::vector<HLeafW> lw;
    int64_t dense_off = 0;   // values of the dense region (first in the device array)
    int64_t lr_off = 0;      // values of the low-rank region (after it)
    const size_t vsz = h->store == DFN_STORE_FP64 ? 8 : 4;
    const size_t kAcaScratch = (size_t)2 << 30;   // device ACA scratch per batch of leaves
    DevBuf scratch, flagbuf, leafbuf, rankbuf, placebuf, dperm;
    std::deque<LrSegment> segs;
    CK(cudaFuncSetAttribute(hm_aca_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hm_aca_smem_bytes()));
    int64_t zoff = 0, slot = 0;
    // row contributions: per component, per global position, slot indices
    std::vector<std::vector<int64_t>> rows((size_t)nc * Nt);
    std::map<std::pair<int, int>, std::vector<int>> dgrp;   // dense leaves by row cluster (r0, nr)
    for (int i = 0; i < B; i++) {
        const Inst &I = h->hinst[i];
        const int64_t e0 = I.eoff, N = I.N;
        const double *E = el.data() + 2 * e0;
        hmat::Tree tree = hmat::build_tree(E, (int)N, leaf);
        for (int64_t p = 0; p < N; p++) perm[e0 + p] = tree.perm[p];
        TRY(dperm.reserve(sizeof(int) * (size_t)N));
        CK(cudaMemcpyAsync(dperm.p, tree.perm.data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice, h->stream));
        std::vector<hmat::Block> leaves;
        hmat::build_blocks(tree, hmat::boxes(tree, E), eta, 0, 0, leaves);
        for (int c = 0; c < nc; c++) {
            // admissible leaves: partial-pivot ACA and recompression on the
            // device (hm_aca_kernel), in batches whose scratch stays within
            // kAcaScratch; factors placed in leaf order into segments of the
            // low-rank value region
            std::vector<HostLeaf> host(leaves.size());
            std::vector<int> lr;
            for (size_t b = 0; b < leaves.size(); b++) {
                host[b] = HostLeaf{1, 0, 0, 0};
                if (!leaves[b].dense) lr.push_back((int)b);
            }
            AcaGeom geo;
            geo.mode = h->mode == DFN_MODE_III ? 3 : 2;
            geo.comp = c;
            geo.perm = static_cast<const int *>(dperm.p);
            geo.E = h->elem + 2 * e0; geo.T = h->tan + 2 * e0; geo.R = h->nrm + 2 * e0; geo.D = h->node + 2 * (e0 + i);
            for (size_t q0 = 0; q0 < lr.size();) {
                std::vector<AcaLeaf> al;
                int64_t soff = 0, foff = 0;
                size_t q1 = q0;
                while (q1 < lr.size()) {
                    const hmat::Block &L = leaves[lr[q1]];
                    const int64_t need = 2LL * (L.nr + L.nc) * HM_KMAX;
                    if (!al.empty() && (size_t)(soff + need) * sizeof(double) > kAcaScratch) break;
                    al.push_back(AcaLeaf{L.r0, L.c0, L.nr, L.nc, soff, foff});
                    soff += need;
                    foff += L.nr + L.nc;
                    q1++;
                }
                TRY(scratch.reserve((size_t)soff * sizeof(double)));
                TRY(flagbuf.reserve((size_t)foff));
                TRY(leafbuf.reserve(al.size() * sizeof(AcaLeaf)));
                TRY(rankbuf.reserve(al.size() * sizeof(int)));
                TRY(placebuf.reserve(al.size() * sizeof(AcaPlace)));
                CK(cudaMemcpyAsync(leafbuf.p, al.data(), al.size() * sizeof(AcaLeaf), cudaMemcpyHostToDevice,
                                   h->stream));
                CK(cudaMemsetAsync(flagbuf.p, 0, (size_t)foff, h->stream));
                hm_aca_kernel<<<(unsigned)al.size(), HM_BT, hm_aca_smem_bytes(), h->stream>>>(
                    static_cast<const AcaLeaf *>(leafbuf.p), geo, eps, static_cast<double *>(scratch.p),
                    static_cast<char *>(flagbuf.p), static_cast<int *>(rankbuf.p));
                h->launches++;
                CK(cudaGetLastError());
                std::vector<int> ranks(al.size());
                CK(cudaMemcpyAsync(ranks.data(), rankbuf.p, al.size() * sizeof(int), cudaMemcpyDeviceToHost,
                                   h->stream));
                CK(cudaStreamSynchronize(h->stream));
                // offsets in leaf order (16-byte aligned starts, rows padded)
                std::vector<AcaPlace> pl(al.size());
                const int64_t seg0 = lr_off;
                for (size_t t = 0; t < al.size(); t++) {
                    HostLeaf &H = host[lr[q0 + t]];
                    // dense where the ACA did not converge, or where its factors
                    // would not be smaller than the block
                    int rk = ranks[t] > hmat::kMaxRank ? -1 : ranks[t];
                    if (rk > 0 && (int64_t)(al[t].nr + al[t].nc) * rk >= (int64_t)al[t].nr * al[t].nc) rk = -1;
                    pl[t] = AcaPlace{0, 0, 0, 0, 0};
                    if (rk < 0) continue;   // did not converge: stored dense
                    H.dense = 0;
                    H.rank = rk;
                    if (rk == 0) continue;  // zero block
                    const int lda = (int)rup(al[t].nr), ld = (int)rup(al[t].nc);
                    lr_off = rup(lr_off);
                    H.foff = lr_off;
                    lr_off += (int64_t)rk * lda;
                    H.goff = lr_off;
                    lr_off += (int64_t)rk * ld;
                    pl[t] = AcaPlace{H.foff - seg0, H.goff - seg0, lda, ld, rk};
                }
                if (lr_off > seg0) {
                    segs.emplace_back();
                    LrSegment &sg = segs.back();
                    sg.start = seg0;
                    sg.len = lr_off - seg0;
                    TRY(sg.buf.reserve((size_t)sg.len * vsz));
                    CK(cudaMemsetAsync(sg.buf.p, 0, (size_t)sg.len * vsz, h->stream));
                    CK(cudaMemcpyAsync(placebuf.p, pl.data(), pl.size() * sizeof(AcaPlace), cudaMemcpyHostToDevice,
                                       h->stream));
                    if (h->store == DFN_STORE_FP64)
                        hm_aca_place_kernel<double><<<(unsigned)al.size(), 256, 0, h->stream>>>(
                            static_cast<const AcaLeaf *>(leafbuf.p), static_cast<const AcaPlace *>(placebuf.p),
                            static_cast<const double *>(scratch.p), static_cast<double *>(sg.buf.p));
                    else
                        hm_aca_place_kernel<float><<<(unsigned)al.size(), 256, 0, h->stream>>>(
                            static_cast<const AcaLeaf *>(leafbuf.p), static_cast<const AcaPlace *>(placebuf.p),
                            static_cast<const double *>(scratch.p), static_cast<float *>(sg.buf.p));
                    h->launches++;
                    CK(cudaGetLastError());
                    CK(cudaStreamSynchronize(h->stream));   // scratch and place list are reused by the next batch
                }
                q0 = q1;
            }
            for (size_t b = 0; b < leaves.size(); b++) {
                const hmat::Block &L = leaves[b];
                HostLeaf &H = host[b];
                if (H.rank == 0 && !H.dense) continue;   // zero block
                HBlk hb{};
                hb.inst = i; hb.comp = c; hb.dense = H.dense; hb.rank = H.rank;
                hb.r0 = L.r0; hb.nr = L.nr; hb.c0 = L.c0; hb.nc = L.nc;
                hb.outoff = H.dense ? -1 : slot;
                if (H.dense) {
                    // F row-major, rows padded with zeros, in the dense region
                    // (filled on the device)
                    hb.ld = (int)rup(L.nc);
                    hb.foff = dense_off;
                    dense_off += rup((int64_t)L.nr * hb.ld);
                    h->hdense_vals += (int64_t)L.nr * L.nc;
                } else {
                    // A'^T (rank x nr) and B'^T (rank x nc), rank-major, rows
                    // padded, placed by the device build
                    hb.lda = (int)rup(L.nr);
                    hb.ld = (int)rup(L.nc);
                    hb.foff = H.foff;
                    hb.goff = H.goff;
                    hb.zoff = zoff;
                    hb.ntask1 = (L.nc + HM_COLS - 1) / HM_COLS;
                    zoff += (int64_t)hb.ntask1 * H.rank;
                    h->hlr_vals += (int64_t)(L.nr + L.nc) * H.rank;
                    h->hranks.push_back(H.rank);
                }
                const int bi = (int)blks.size();
                blks.push_back(hb);
                if (H.dense) {
                    for (int r = 0; r < L.nr; r += HM_ROWS) t3.push_back(HTask{bi, r, std::min(HM_ROWS, L.nr - r), 0});
                } else if (L.nc <= HM_COLS) {
                    // whole leaf: one warp when small, else one CTA
                    if ((int64_t)H.rank * (hb.lda + hb.ld) * (int64_t)vsz <= HM_WARP_LEAF_BYTES &&
                        hb.ld / VW <= 32 * HM_WARP_XV) {
                        l5.push_back(bi);
                        lw.push_back(HLeafW{hb.foff, e0 + L.c0, slot, i, H.rank, hb.lda, hb.ld, L.nr, bi});
                    } else {
                        l4.push_back(bi);
                    }
                } else {
                    for (int j = 0; j < hb.ntask1; j++)
                        t1.push_back(HTask{bi, j * HM_COLS, std::min(HM_COLS, L.nc - j * HM_COLS), j});
                    for (int r = 0; r < L.nr; r += HM_LROWS) t2.push_back(HTask{bi, r, std::min(HM_LROWS, L.nr - r), 0});
                }
                if (H.dense) {
                    dgrp[std::make_pair(L.r0, L.nr)].push_back(bi);
                    continue;
                }
                for (int r = 0; r < L.nr; r++) rows[(size_t)c * Nt + e0 + L.r0 + r].push_back(slot + r);
                slot += L.nr;
            }
            // the dense leaves of each row cluster: one group, one slot per row
            for (const auto &kv : dgrp) {
                const int r0 = kv.first.first, nr = kv.first.second;
                const int gi = (int)dgroups.size();
                dgroups.push_back(HDGroup{slot, (int)dleaves.size(), (int)kv.second.size(), i, 0});
                for (int bi : kv.second) {
                    const HBlk &b = blks[bi];
                    dleaves.push_back(HDLeaf{b.foff, e0 + b.c0, b.ld, (b.nc + VW - 1) / VW});
                }
                for (int r = 0; r < nr; r += HM_ROWS) tg.push_back(HTask{gi, r, std::min(HM_ROWS, nr - r), 0});
                for (int r = 0; r < nr; r++) rows[(size_t)c * Nt + e0 + r0 + r].push_back(slot + r);
                slot += nr;
            }
            dgrp.clear();
        }
        if (i == 0) {
            h->hn1_0 = (int64_t)t1.size();
            h->hn2_0 = (int64_t)t2.size();
            h->hn3_0 = (int64_t)tg.size();
            h->hn4_0 = (int64_t)l4.size();
            h->hn5_0 = (int64_t)l5.size();
        }
    }
    // tasks must list network 0 first for the operator entry points; they
    // do, since networks are built in order. Row sums: leaf b's result for
    // the row at position e sits in slot base_b + e (base_b = its first slot
    // minus its first row), so consecutive rows with the same blocks share
    // one list of bases (a segment), in block order.
    std::vector<int32_t> segof((size_t)nc * Nt);
    std::vector<int64_t> segptr(1, 0), segbase;
    for (size_t q = 0; q < rows.size(); q++) {
        const int64_t e = (int64_t)(q % (size_t)Nt);
        bool same = e > 0 && rows[q].size() == rows[q - 1].size();
        for (size_t k = 0; same && k < rows[q].size(); k++)
            if (rows[q][k] - e != rows[q - 1][k] - (e - 1)) same = false;
        if (!same) {
            for (int64_t v : rows[q]) segbase.push_back(v - e);
            segptr.push_back((int64_t)segbase.size());
        }
        segof[q] = (int32_t)(segptr.size() - 2);
    }
    rows.clear();
    h->hn1 = (int64_t)t1.size();
    h->hn2 = (int64_t)t2.size();
    h->hn3 = (int64_t)tg.size();
    h->hn4 = (int64_t)l4.size();
    h->hn5 = (int64_t)l5.size();
    h->hblocks = (int64_t)blks.size();
    h->kv_bytes = (h->hdense_vals + h->hlr_vals) * (int64_t)vsz;   // stored entries, padding excluded
    // device values: [dense leaves | low-rank factors]
    for (HBlk &hb : blks)
        if (!hb.dense) { hb.foff += dense_off; hb.goff += dense_off; }
    const size_t ntot = (size_t)(dense_off + lr_off);
    CK(cudaMalloc(&h->hvals, std::max<size_t>(ntot, 1) * vsz));
    CK(cudaMemsetAsync(h->hvals, 0, (size_t)dense_off * vsz, h->stream));   // padding of the dense rows
    for (LrSegment &sg : segs)
        CK(cudaMemcpyAsync(static_cast<char *>(h->hvals) + (size_t)(dense_off + sg.start) * vsz, sg.buf.p,
                           (size_t)sg.len * vsz, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    segs.clear();
    CK(cudaMalloc((void **)&h->hblk, std::max<size_t>(blks.size(), 1) * sizeof(HBlk)));
    CK(cudaMemcpyAsync(h->hblk, blks.data(), blks.size() * sizeof(HBlk), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->ht1, std::max<size_t>(t1.size(), 1) * sizeof(HTask)));
    if (!t1.empty()) CK(cudaMemcpyAsync(h->ht1, t1.data(), t1.size() * sizeof(HTask), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->ht2, std::max<size_t>(t2.size(), 1) * sizeof(HTask)));
    if (!t2.empty()) CK(cudaMemcpyAsync(h->ht2, t2.data(), t2.size() * sizeof(HTask), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hl4, std::max<size_t>(l4.size(), 1) * sizeof(int)));
    if (!l4.empty()) CK(cudaMemcpyAsync(h->hl4, l4.data(), l4.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hl5, std::max<size_t>(l5.size(), 1) * sizeof(int)));
    if (!l5.empty()) CK(cudaMemcpyAsync(h->hl5, l5.data(), l5.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    for (HLeafW &w : lw) w.aoff += dense_off;   // low-rank values follow the dense region
    CK(cudaMalloc((void **)&h->hlw, std::max<size_t>(lw.size(), 1) * sizeof(HLeafW)));
    if (!lw.empty()) CK(cudaMemcpyAsync(h->hlw, lw.data(), lw.size() * sizeof(HLeafW), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->htg, std::max<size_t>(tg.size(), 1) * sizeof(HTask)));
    if (!tg.empty()) CK(cudaMemcpyAsync(h->htg, tg.data(), tg.size() * sizeof(HTask), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hdg, std::max<size_t>(dgroups.size(), 1) * sizeof(HDGroup)));
    if (!dgroups.empty())
        CK(cudaMemcpyAsync(h->hdg, dgroups.data(), dgroups.size() * sizeof(HDGroup), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hdl, std::max<size_t>(dleaves.size(), 1) * sizeof(HDLeaf)));
    if (!dleaves.empty())
        CK(cudaMemcpyAsync(h->hdl, dleaves.data(), dleaves.size() * sizeof(HDLeaf), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->ht3, std::max<size_t>(t3.size(), 1) * sizeof(HTask)));
    if (!t3.empty()) CK(cudaMemcpyAsync(h->ht3, t3.data(), t3.size() * sizeof(HTask), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hperm, sizeof(int) * Nt));
    CK(cudaMemcpyAsync(h->hperm, perm.data(), sizeof(int) * Nt, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hsegof, sizeof(int32_t) * segof.size()));
    CK(cudaMemcpyAsync(h->hsegof, segof.data(), sizeof(int32_t) * segof.size(), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hsegptr, sizeof(int64_t) * segptr.size()));
    CK(cudaMemcpyAsync(h->hsegptr, segptr.data(), sizeof(int64_t) * segptr.size(), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMalloc((void **)&h->hsegbase, sizeof(int64_t) * std::max<size_t>(segbase.size(), 1)));
    CK(cudaMemcpyAsync(h->hsegbase, segbase.data(), sizeof(int64_t) * segbase.size(), cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));   // the host vectors go out of scope
    if (!t3.empty()) {
        if (h->store == DFN_STORE_FP64)
            hm_fill_dense_kernel<double><<<(unsigned)t3.size(), 256, 0, h->stream>>>(
                h->ht3, h->hblk, h->inst, h->mode, h->hperm, h->node, h->elem, h->tan, h->nrm,
                static_cast<double *>(h->hvals));
        else
            hm_fill_dense_kernel<float><<<(unsigned)t3.size(), 256, 0, h->stream>>>(
                h->ht3, h->hblk, h->inst, h->mode, h->hperm, h->node, h->elem, h->tan, h->nrm,
                static_cast<float *>(h->hvals));
        h->launches++;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaMalloc((void **)&h->hz, sizeof(double) * std::max<int64_t>(zoff, 1)));
    CK(cudaMalloc((void **)&h->hxp, sizeof(double) * (Nt + HM_XPAD)));
    CK(cudaMemsetAsync(h->hxp, 0, sizeof(double) * (Nt + HM_XPAD), h->stream));
    CK(cudaMalloc((void **)&h->hout, sizeof(double) * std::max<int64_t>(slot, 1)));
    return DFN_OK;
}

static int single_only(const dfn_handle *h)
{
    if (h->B != 1) {
        g_err = "this entry point works on a handle holding one network";
        return DFN_ERR_UNSUPPORTED;
    }
    return DFN_OK;
}
// ---------------------------------------------------------------------------
extern "C" {

int32_t dfn_abi_version(void) { return DFN_ABI_VERSION; }
int64_t dfn_problem_struct_size(void) { return (int64_t)sizeof(dfn_problem); }
int64_t dfn_options_struct_size(void) { return (int64_t)sizeof(dfn_options); }
int64_t dfn_report_struct_size(void) { return (int64_t)sizeof(dfn_report); }
const char *dfn_last_error(void) { return g_err.c_str(); }

const char *dfn_status_string(int32_t s)
{
    switch (s) {
    case DFN_OK: return "ok";
    case DFN_ERR_NOCONV: return "pressure CG did not converge (ier=1)";
    case DFN_ERR_UNDERFLOW: return "stepsize underflow in rkqs";
    case DFN_ERR_EXTENSIONAL: return "normal traction became extensional";
    case DFN_ERR_NONFINITE: return "non-finite value in the state or pressure";
    case DFN_ERR_ARG: return "invalid argument";
    case DFN_ERR_CUDA: return "CUDA error";
    case DFN_ERR_UNSUPPORTED: return "unsupported feature";
    case DFN_ERR_ATTEMPTS: return "too many rejected attempts in one step";
    case DFN_ERR_NOMEM: return "device allocation failed";
    case DFN_ERR_TIMEOUT: return "a bounded device wait expired";
    default: return "unknown status";
    }
}

void dfn_default_options(dfn_options *o)
{
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->kernel_storage = DFN_STORE_FP64;
    o->pressure_solver = DFN_PRESSURE_CG;
    o->device = 0;
    o->max_attempts = 64;
    o->gemv_impl = 0;
}

int32_t dfn_destroy(dfn_handle *h)
{
    if (!h) return DFN_OK;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void *ptrs[] = {h->kstar, h->kmin, h->Snk, h->s64_vt, h->slip, h->slip_out, h->slip_acc, h->tau0, h->wlast, h->vnow, h->mlp, h->rec_x, h->rec_t, h->rec_n,
                    h->hblk, h->ht1, h->ht2, h->hvals, h->hperm, h->hsegof, h->hsegptr, h->hsegbase, h->hz, h->hout, h->hxp, h->ht3, h->htg, h->hdg, h->hdl, h->hl4, h->hl5, h->hlw, h->xptr, h->xcon, h->xrows, h->xrows_ptr, h->tri_tiles, h->tcoef,
                    h->inst, h->inst_of, h->tiles, h->seg_start, h->seg_inst, h->long_seg, h->short_seg, h->tc_A, h->tc_B, h->node, h->elem, h->ds, h->tan,
                    h->nrm, h->permx, h->a, h->b, h->Dc, h->f0, h->V0, h->nload, h->sload, h->perm, h->fake,
                    h->src_fault, h->src_elem, h->src_Q, h->src_tb, h->src_te, h->Y, h->P, h->Pdot, h->yout,
                    h->yscal, h->ytmp, h->kbuf, h->SigT, h->SigN, h->partT, h->partN, h->Ptemp, h->Pdot_s,
                    h->pwork, h->pcoef, h->vin, h->vout, h->snap, h->err_flag, h->K, h->ctl};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (h->h_ctl) cudaFreeHost(h->h_ctl);
    for (cudaEvent_t e : h->pev) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->side_stream) cudaStreamDestroy(h->side_stream);
    if (h->side_lo) cudaStreamDestroy(h->side_lo);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->ev_pfork) cudaEventDestroy(h->ev_pfork);
    if (h->ev_pjoin) cudaEventDestroy(h->ev_pjoin);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return DFN_OK;
}

static bool all_finite(const double *x, int64_t n)
{
    for (int64_t i = 0; i < n; i++)
        if (!std::isfinite(x[i])) return false;
    return true;
}

static int check_problem(const dfn_problem *p)
{
    const int64_t N = p->nb_element, F = p->nb_fault;
    if (N < 2 || F < 1 || !p->fault_nb_element || !p->node) { g_err = "need nb_element >= 2 and nb_fault >= 1"; return DFN_ERR_ARG; }
    int64_t cnt = 0;
    for (int64_t f = 0; f < F; f++) {
        if (p->fault_nb_element[f] < 1) { g_err = "every fault needs at least one element"; return DFN_ERR_ARG; }
        cnt += p->fault_nb_element[f] + 1;
    }
    if (cnt - 1 != N) { g_err = "nb_element must equal sum(fault_nb_element) + nb_fault - 1"; return DFN_ERR_ARG; }
    if (p->fracture_mode != DFN_MODE_II && p->fracture_mode != DFN_MODE_III) { g_err = "fracture_mode must be 2 or 3"; return DFN_ERR_ARG; }
    if (!(p->tol_solver > 0)) { g_err = "tol_solver must be positive"; return DFN_ERR_ARG; }
    if (!p->a || !p->b || !p->Dc || !p->f0 || !p->V0 || !p->V || !p->theta || !p->sigmaN || !p->P ||
        !p->normal_loading_dot || !p->shear_loading_dot || !p->permeability) { g_err = "null array in dfn_problem"; return DFN_ERR_ARG; }
    for (int64_t s = 0; s < p->nb_source; s++) {
        int64_t f = p->src_fault[s];
        if (f < 1 || f > F || p->src_index[s] < 1 || p->src_index[s] > p->fault_nb_element[f - 1]) {
            g_err = "source fault/index out of range";
            return DFN_ERR_ARG;
        }
    }
    if (p->permeability_coupling != 0 && p->permeability_coupling != 1) {
        g_err = "permeability_coupling must be 0 or 1";
        return DFN_ERR_ARG;
    }
    if (p->permeability_coupling == 1) {
        if (!p->kmin || !p->Snk) { g_err = "permeability_coupling = 1 needs kmin and Snk"; return DFN_ERR_ARG; }
        for (int64_t k = 0; k < N; k++)
            if (!(p->Snk[k] != 0.0) || !std::isfinite(p->Snk[k]) || !std::isfinite(p->kmin[k])) {
                g_err = "permeability coupling: Snk must be finite and nonzero, kmin finite";
                return DFN_ERR_ARG;
            }
    }
    // the initial state must be finite (the reference would carry a NaN
    // into every right-hand side and reject every attempt)
    const double *st[4] = {p->V, p->theta, p->sigmaN, p->P};
    for (int j = 0; j < 4; j++)
        if (!all_finite(st[j], N)) {
            g_err = "non-finite value in the initial state (V, theta, sigmaN or P)";
            return DFN_ERR_NONFINITE;
        }
    return DFN_OK;
}

#define DALLOC(ptr, count)                                                \
    do {                                                                  \
        cudaError_t e_ = cudaMalloc((void **)&(ptr), sizeof(*(ptr)) * (size_t)std::max<int64_t>((count), 1)); \
        if (e_ != cudaSuccess) {                                          \
            set_err("cudaMalloc " #ptr, e_, __FILE__, __LINE__);          \
            dfn_destroy(h);                                               \
            return e_ == cudaErrorMemoryAllocation ? DFN_ERR_NOMEM : DFN_ERR_CUDA; \
        }                                                                 \
    } while (0)

#define HCOPY(dst, src, count)                                                                          \
    do {                                                                                                \
        if ((count) > 0) {                                                                              \
            cudaError_t e_ = cudaMemcpyAsync((dst), (src), sizeof(*(dst)) * (size_t)(count), cudaMemcpyHostToDevice, h->stream); \
            if (e_ != cudaSuccess) {                                                                    \
                set_err("cudaMemcpy " #dst, e_, __FILE__, __LINE__);                                    \
                dfn_destroy(h);                                                                         \
                return DFN_ERR_CUDA;                                                                    \
            }                                                                                           \
        }                                                                                               \
    } while (0)

#define CKC(x)                                                 \
    do {                                                       \
        cudaError_t e_ = (x);                                  \
        if (e_ != cudaSuccess) {                               \
            set_err(#x, e_, __FILE__, __LINE__);               \
            dfn_destroy(h);                                    \
            return DFN_ERR_CUDA;                               \
        }                                                      \
    } while (0)

int32_t dfn_create_batch(const dfn_problem *probs, int32_t count, const dfn_options *opt_in, dfn_handle **out)
{
    if (!probs || !out || count < 1) { g_err = "null argument or empty batch"; return DFN_ERR_ARG; }
    *out = nullptr;
    dfn_options opt;
    if (opt_in) opt = *opt_in; else dfn_default_options(&opt);
    if (opt.kernel_storage < 0 || opt.kernel_storage > 4) { g_err = "bad kernel_storage"; return DFN_ERR_ARG; }
    if (opt.pressure_solver < 0 || opt.pressure_solver > 2) { g_err = "bad pressure_solver"; return DFN_ERR_ARG; }
    for (int i = 0; i < count; i++) {
        TRY(check_problem(&probs[i]));
        if (probs[i].fracture_mode != probs[0].fracture_mode) { g_err = "all networks of a batch need the same fracture_mode"; return DFN_ERR_ARG; }
        if (probs[i].permeability_coupling != probs[0].permeability_coupling) {
            g_err = "all networks of a batch need the same permeability_coupling";
            return DFN_ERR_ARG;
        }
    }
    if (probs[0].permeability_coupling == 1 && opt.formulation == DFN_FORM_NEWTON) {
        g_err = "permeability coupling follows the state's sigmaN: the V formulation only";
        return DFN_ERR_UNSUPPORTED;
    }
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev <= opt.device) {
        g_err = std::string("no usable CUDA device: ") + cudaGetErrorString(ce);
        return DFN_ERR_CUDA;
    }

    dfn_handle *h = new dfn_handle();
    h->dev = opt.device;
    CKC(cudaSetDevice(h->dev));
    CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    CKC(cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
    h->B = count;
    h->mode = probs[0].fracture_mode; h->store = opt.kernel_storage;
    h->pressure = opt.pressure_solver; h->gemv_impl = opt.gemv_impl;
    if (cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->dev) != cudaSuccess || h->sms <= 0)
        h->sms = 148;
    h->max_attempts = opt.max_attempts > 0 ? opt.max_attempts : 64;
    h->form = opt.formulation == DFN_FORM_NEWTON ? DFN_FORM_NEWTON : DFN_FORM_V;
    h->guess = (opt.newton_guess >= 0 && opt.newton_guess <= 3) ? opt.newton_guess : 0;
    h->newton_maxit = opt.newton_maxit > 0 ? opt.newton_maxit : 50;
    h->newton_tol = opt.newton_tol > 0 ? opt.newton_tol : 1e-13;
    h->max_step = opt.max_step > 0 ? opt.max_step : 86400.0;
    const int bpc = bytes_per_col(h->mode, h->store);
    const int64_t CW = GEMV_CHUNK_BYTES / bpc;
    // static_kernel selects the dense kernel ("direct") or the H-matrix
    // ("hmatrix"), as kernel_ptr does in src/initialisation.f90:105-128
    h->hmat = probs[0].static_kernel == DFN_KERNEL_HMATRIX;
    for (int i = 1; i < count; i++)
        if ((probs[i].static_kernel == DFN_KERNEL_HMATRIX) != h->hmat) {
            g_err = "all networks of a batch need the same static_kernel";
            dfn_destroy(h);
            return DFN_ERR_ARG;
        }
    if (h->hmat && (h->store == DFN_STORE_BF16X2 || h->store == DFN_STORE_FP64_SHARED)) {
        g_err = "the H-matrix path stores FP64 or FP32 factors";
        dfn_destroy(h);
        return DFN_ERR_UNSUPPORTED;
    }
    h->ncomp = (h->mode == DFN_MODE_II) ? 2 : 1;
    h->tc = h->store == DFN_STORE_BF16X2_TC;
    h->s64 = h->store == DFN_STORE_FP64_SHARED;
    if (h->tc || h->s64) {
        const dfn_problem &p0 = probs[0];
        std::string why;
        if (h->hmat) why = "the H-matrix path has its own storage";
        if (count > 256) why = "at most 256 networks share one kernel matrix";
        for (int i = 1; i < count && why.empty(); i++) {
            const dfn_problem &q = probs[i];
            if (q.nb_element != p0.nb_element || q.nb_fault != p0.nb_fault || q.fracture_mode != p0.fracture_mode ||
                q.mu != p0.mu || q.cp != p0.cp || q.cs != p0.cs ||
                memcmp(q.node, p0.node, sizeof(double) * 2 * (p0.nb_element + 1)) != 0)
                why = "networks of a tensor-core batch must share nb_element, nodes, fracture mode and mu, cp, cs";
        }
        if (!why.empty()) {
            g_err = why;
            dfn_destroy(h);
            return DFN_ERR_ARG;
        }
        const int64_t N0 = p0.nb_element;
        if (h->s64) {
            // column splits: the fewest that fill whole waves (three CTAs per SM)
            h->s64_rp = ((count + S64_MEM - 1) / S64_MEM) * S64_MEM;
            h->s64_nkc = (int)((N0 + S64_COLS - 1) / S64_COLS);
            const int64_t tiles = ((N0 + S64_ROWS - 1) / S64_ROWS) * (h->s64_rp / S64_MEM);
            const int64_t slots = (int64_t)h->sms * 3;
            double best = -1.0;
            for (int sp = 1; sp <= 16 && sp <= h->s64_nkc; sp++) {
                const int64_t units = tiles * sp;
                const double eff = (double)units / (double)(((units + slots - 1) / slots) * slots);
                if (eff > best + 0.02) { best = eff; h->s64_split = sp; }
            }
            h->s64_kps = (h->s64_nkc + h->s64_split - 1) / h->s64_split;
        }
    }
    if (h->tc) {
        const dfn_problem &p0 = probs[0];
        const int64_t N0 = p0.nb_element;
        h->tc_mrows = h->ncomp * N0;
        h->tc_nmt = (int)((h->tc_mrows + TC_BM - 1) / TC_BM);
        h->tc_mpad = (int64_t)h->tc_nmt * TC_BM;
        h->tc_nkb = (int)((N0 + TC_BK - 1) / TC_BK);
        h->tc_kpad = (int64_t)h->tc_nkb * TC_BK;
        h->tc_bn = count <= 16 ? 16 : count <= 32 ? 32 : count <= 64 ? 64 : count <= 128 ? 128 : 256;
        // reduction splits: the fewest that fill whole waves of the SMs well
        const int sms = h->sms;
        double best = -1.0;
        for (int s = 1; s <= 8 && s <= h->tc_nkb; s++) {
            const int64_t units = (int64_t)h->tc_nmt * s;
            const double eff = (double)units / (double)(((units + sms - 1) / sms) * sms);
            if (eff > best + 0.05) { best = eff; h->tc_split = s; }
        }
        h->tc_kps = (h->tc_nkb + h->tc_split - 1) / h->tc_split;
    }

    // instance table
    int64_t eoff = 0, kvec = 0, poff = 0, soff = 0;
    h->hinst.resize(count);
    for (int i = 0; i < count; i++) {
        const dfn_problem &p = probs[i];
        Inst &I = h->hinst[i];
        I.N = p.nb_element;
        I.Np = (h->hmat || h->tc) ? I.N : (h->s64 ? ((I.N + S64_COLS - 1) / S64_COLS) * S64_COLS
                                                 : ((I.N + CW - 1) / CW) * CW);
        I.eoff = eoff;
        I.nchunk = h->hmat ? 1 : (h->tc ? h->tc_split : (h->s64 ? h->s64_split : I.Np / CW));
        I.kvec = h->s64 ? 0 : kvec;   // a shared-geometry batch has one matrix
        I.poff = poff;
        I.soff = soff;
        I.nsrc = p.nb_source;
        // prefactors: src/kernel_calculation/hmatrixModeII.f90:67-68, hmatrixModeIII.f90:55
        I.prefT = (h->mode == DFN_MODE_II) ? p.mu / DFN_PI * (1.0 - p.cs * p.cs / (p.cp * p.cp)) : p.mu / (2.0 * DFN_PI);
        I.mu_2cs = p.mu / (2.0 * p.cs);
        I.porosity = p.porosity; I.dyn_visc = p.dyn_viscosity; I.comp = p.fluid_comp + p.rock_comp;
        I.tol = p.tol_solver;
        I.t0 = p.time0;
        eoff += I.N;
        if (!h->hmat && !h->tc && !h->s64) kvec += I.N * I.Np * bpc / 16;
        if (h->s64 && i == 0) kvec = I.N * I.Np * bpc / 16;
        poff += I.nchunk * I.N;
        soff += I.nsrc;
        if (!h->hmat && !h->tc && (!h->s64 || i == 0)) h->kv_bytes += I.N * I.N * bpc;
    }
    const int64_t Nt = eoff;
    h->Ntot = Nt;
    h->part_tot = poff;
    h->nsrc_tot = soff;
    const int64_t Nnode = Nt + count;   // every network has N_i + 1 nodes and faces

    DALLOC(h->inst, count); DALLOC(h->inst_of, Nt);
    DALLOC(h->node, 2 * Nnode); DALLOC(h->elem, 2 * Nt); DALLOC(h->ds, Nt); DALLOC(h->tan, 2 * Nt);
    DALLOC(h->nrm, 2 * Nt); DALLOC(h->permx, Nnode);
    DALLOC(h->a, Nt); DALLOC(h->b, Nt); DALLOC(h->Dc, Nt); DALLOC(h->f0, Nt); DALLOC(h->V0, Nt);
    DALLOC(h->nload, Nt); DALLOC(h->sload, Nt); DALLOC(h->perm, Nt); DALLOC(h->fake, Nt);
    DALLOC(h->Y, 3 * Nt); DALLOC(h->P, Nt); DALLOC(h->Pdot, Nt); DALLOC(h->yout, 3 * Nt); DALLOC(h->yscal, 3 * Nt);
    DALLOC(h->ytmp, 3 * Nt); DALLOC(h->kbuf, 18 * Nt); DALLOC(h->SigT, Nt); DALLOC(h->SigN, Nt);
    DALLOC(h->partT, poff); DALLOC(h->partN, poff);
    DALLOC(h->Ptemp, 6 * Nt); DALLOC(h->Pdot_s, 6 * Nt); DALLOC(h->pwork, 24 * Nt);
    if (h->pressure != DFN_PRESSURE_TRIDIAG) DALLOC(h->pcoef, 18 * Nt);
    DALLOC(h->vin, 3 * h->hinst[0].N); DALLOC(h->vout, 3 * h->hinst[0].N); DALLOC(h->snap, 5 * Nt);
    DALLOC(h->err_flag, 1); DALLOC(h->ctl, count);
    DALLOC(h->slip, Nt); DALLOC(h->slip_out, Nt); DALLOC(h->slip_acc, Nt);
    CKC(cudaMemsetAsync(h->slip, 0, sizeof(double) * Nt, h->stream));
    DALLOC(h->src_fault, soff); DALLOC(h->src_elem, soff); DALLOC(h->src_Q, soff); DALLOC(h->src_tb, soff);
    DALLOC(h->src_te, soff);
    CKC(cudaMemsetAsync(h->err_flag, 0, sizeof(int), h->stream));
    CKC(cudaMemsetAsync(h->partN, 0, sizeof(double) * std::max<int64_t>(poff, 1), h->stream));
    CKC(cudaMemsetAsync(h->Pdot, 0, sizeof(double) * Nt, h->stream));
    CKC(cudaMemsetAsync(h->SigT, 0, sizeof(double) * Nt, h->stream));
    CKC(cudaMemsetAsync(h->SigN, 0, sizeof(double) * Nt, h->stream));
    CKC(cudaMallocHost((void **)&h->h_ctl, sizeof(StepCtl) * count));
    HCOPY(h->inst, h->hinst.data(), count);

    std::vector<int> inst_of(Nt);
    std::vector<unsigned char> fake(Nt, 0);
    for (int i = 0; i < count; i++) {
        const dfn_problem &p = probs[i];
        const Inst &I = h->hinst[i];
        const int64_t N = I.N, e0 = I.eoff, F = p.nb_fault;
        for (int64_t k = 0; k < N; k++) inst_of[e0 + k] = i;
        HCOPY(h->node + 2 * (e0 + i), p.node, 2 * (N + 1));
        HCOPY(h->a + e0, p.a, N); HCOPY(h->b + e0, p.b, N); HCOPY(h->Dc + e0, p.Dc, N); HCOPY(h->f0 + e0, p.f0, N);
        HCOPY(h->V0 + e0, p.V0, N); HCOPY(h->nload + e0, p.normal_loading_dot, N);
        HCOPY(h->sload + e0, p.shear_loading_dot, N); HCOPY(h->perm + e0, p.permeability, N);
        HCOPY(h->Y + 3 * e0, p.V, N); HCOPY(h->Y + 3 * e0 + N, p.theta, N); HCOPY(h->Y + 3 * e0 + 2 * N, p.sigmaN, N);
        HCOPY(h->P + e0, p.P, N);
        // fake elements (src/friction/RateStateAgingModeII.f90:81-89) and
        // 0-based fault starts (src/configuration.f90:245-246)
        std::vector<int64_t> first(F);
        int64_t idx = 0, c2 = 0;
        for (int64_t f = 0; f < F; f++) {
            first[f] = c2;
            c2 += p.fault_nb_element[f] + 1;
            idx += p.fault_nb_element[f] + 1;
            if (idx <= N) fake[e0 + idx - 1] = 1;
        }
        if (p.nb_source > 0) {
            std::vector<int64_t> se(p.nb_source);
            for (int64_t s = 0; s < p.nb_source; s++) se[s] = first[p.src_fault[s] - 1] + p.src_index[s] - 1;
            HCOPY(h->src_fault + I.soff, p.src_fault, p.nb_source); HCOPY(h->src_elem + I.soff, se.data(), p.nb_source);
            HCOPY(h->src_Q + I.soff, p.src_Q, p.nb_source); HCOPY(h->src_tb + I.soff, p.src_t_beg, p.nb_source);
            HCOPY(h->src_te + I.soff, p.src_t_end, p.nb_source);
        }
        // geometry (device), src/initialisation.f90:145-205
        geometry_kernel<<<blocks_of(N + 1, 256), 256, 0, h->stream>>>(
            N, h->mode, h->node + 2 * (e0 + i), h->elem + 2 * e0, h->ds + e0, h->tan + 2 * e0, h->nrm + 2 * e0,
            h->nload + e0, h->sload + e0, h->Y + 3 * e0 + 2 * N, h->perm + e0, h->permx + e0 + i, p.Sigma11_dot,
            p.Sigma12_dot, p.Sigma22_dot, p.Sigma31_dot, p.Sigma32_dot);
        h->launches++;
        CKC(cudaGetLastError());
    }
    HCOPY(h->inst_of, inst_of.data(), Nt);
    h->pcoup = probs[0].permeability_coupling == 1;
    if (h->pcoup) {
        DALLOC(h->kstar, Nt); DALLOC(h->kmin, Nt); DALLOC(h->Snk, Nt);
        for (int i = 0; i < count; i++) {
            const Inst &I = h->hinst[i];
            HCOPY(h->kmin + I.eoff, probs[i].kmin, I.N);
            HCOPY(h->Snk + I.eoff, probs[i].Snk, I.N);
        }
        // k* from the state after the geometry's loading projection
        // (src/initialisation.f90:256-261)
        perm_init_kernel<<<blocks_of(Nt, 256), 256, 0, h->stream>>>(elem_params(h), h->Y, h->P, h->perm, h->kmin,
                                                                   h->Snk, h->kstar);
        h->launches++;
        CKC(cudaGetLastError());
    }
    CKC(cudaMalloc((void **)&h->mlp, kMlpImgBytes));
    CKC(cudaMemsetAsync(h->mlp, 0, kMlpImgBytes, h->stream));
    DALLOC(h->rec_n, 1);
    CKC(cudaMemsetAsync(h->rec_n, 0, sizeof(unsigned long long), h->stream));
    if (h->form == DFN_FORM_NEWTON) {
        DALLOC(h->tau0, Nt); DALLOC(h->wlast, Nt); DALLOC(h->vnow, Nt);
        CKC(cudaMemsetAsync(h->vnow, 0, sizeof(double) * Nt, h->stream));
        HCOPY(h->fake, fake.data(), Nt);
        newton_init_kernel<<<blocks_of(Nt, 256), 256, 0, h->stream>>>(Nt, h->inst_of, h->inst, h->a, h->b, h->f0,
                                                                       h->V0, h->fake, h->P, h->Y, h->tau0,
                                                                       h->wlast);
        h->launches++;
        CKC(cudaGetLastError());
    }
    HCOPY(h->fake, fake.data(), Nt);

    // decoupled pressure segments from the face permeabilities
    {
        std::vector<double> px(Nnode);
        CKC(cudaMemcpyAsync(px.data(), h->permx, sizeof(double) * Nnode, cudaMemcpyDeviceToHost, h->stream));
        CKC(cudaStreamSynchronize(h->stream));
        std::vector<int64_t> seg;
        std::vector<int> sinst;
        for (int i = 0; i < count; i++) {
            const Inst &I = h->hinst[i];
            seg.push_back(I.eoff);
            sinst.push_back(i);
            for (int64_t k = 1; k < I.N; k++)
                if (px[I.eoff + i + k] == 0.0) { seg.push_back(I.eoff + k); sinst.push_back(i); }
            if (i == 0) h->nseg0 = (int64_t)seg.size();
        }
        seg.push_back(Nt);
        h->nseg = (int64_t)seg.size() - 1;
        DALLOC(h->seg_start, seg.size());
        DALLOC(h->seg_inst, sinst.size());
        HCOPY(h->seg_start, seg.data(), seg.size());
        HCOPY(h->seg_inst, sinst.data(), sinst.size());
        // long segments go to the CTA-parallel solve; networks in order, so
        // those of network 0 come first
        std::vector<int> lg, sh;
        for (int64_t q = 0; q < h->nseg; q++) {
            if (seg[q + 1] - seg[q] > TRI_SHORT_MAX) lg.push_back((int)q);
            else sh.push_back((int)q);
            if (q + 1 == h->nseg0) {
                h->nlong0 = (int64_t)lg.size();
                h->nshort0 = (int64_t)sh.size();
            }
        }
        h->nlong = (int64_t)lg.size();
        h->nshort = (int64_t)sh.size();
        // default launch shape of the short segments (dfn_autotune measures
        // instead): warps while the segments fill few waves of warps, threads
        // once there are tens of thousands
        h->tri_shape = h->nshort >= 16384 ? 2 : 0;
        // tiles: runs of consecutive short segments of one network, at most
        // TRI_TILE elements and 128 segments each; network 0's first
        std::vector<int2> tl;
        for (size_t q = 0; q < sh.size();) {
            size_t r = q + 1;
            int64_t ne = seg[sh[q] + 1] - seg[sh[q]];
            while (r < sh.size() && r - q < 128 && sh[r] == sh[r - 1] + 1 && sinst[sh[r]] == sinst[sh[q]] &&
                   ne + (seg[sh[r] + 1] - seg[sh[r]]) <= TRI_TILE) {
                ne += seg[sh[r] + 1] - seg[sh[r]];
                r++;
            }
            tl.push_back(make_int2((int)q, (int)(r - q)));
            if (sinst[sh[q]] == 0) h->ntri_tiles0 = (int64_t)tl.size();
            q = r;
        }
        h->ntri_tiles = (int64_t)tl.size();
        if (!tl.empty()) {
            DALLOC(h->tri_tiles, tl.size());
            HCOPY(h->tri_tiles, tl.data(), tl.size());
        }
        if (h->nlong) {
            DALLOC(h->long_seg, lg.size());
            HCOPY(h->long_seg, lg.data(), lg.size());
        }
        if (h->nshort) {
            DALLOC(h->short_seg, sh.size());
            HCOPY(h->short_seg, sh.data(), sh.size());
        }
    }

    {
        // side stream at the highest priority (its CTAs are placed first):
        // the H-matrix's low-rank leaves beside its dense rows, and pressure
        // solves on a few thread-block clusters beside a K.V
        int lo_pri = 0, hi_pri = 0;
        CKC(cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri));
        CKC(cudaStreamCreateWithPriority(&h->side_stream, cudaStreamNonBlocking, hi_pri));
        CKC(cudaStreamCreateWithPriority(&h->side_lo, cudaStreamNonBlocking, lo_pri));
        CKC(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&h->ev_pfork, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&h->ev_pjoin, cudaEventDisableTiming));
    }
    if (h->hmat) {
        const int st = build_hmatrix(h, probs, opt);
        if (st != DFN_OK) {
            dfn_destroy(h);
            return st;
        }
    }
    if (h->tc) {
        // one kernel matrix for the batch: BF16 hi and lo, rows padded to
        // 128, reduction to 64 with zeros; V rows of all networks likewise
        const int64_t na = h->tc_mpad * h->tc_kpad, nb = (int64_t)h->tc_bn * h->tc_kpad;
        DALLOC(h->tc_A, 2 * na);
        DALLOC(h->tc_B, 2 * nb);
        CKC(cudaMemsetAsync(h->tc_A, 0, sizeof(__nv_bfloat16) * 2 * na, h->stream));
        CKC(cudaMemsetAsync(h->tc_B, 0, sizeof(__nv_bfloat16) * 2 * nb, h->stream));
        const Inst &I = h->hinst[0];
        dim3 grid((unsigned)I.N, (unsigned)((I.N + 255) / 256));
        if (h->mode == 2)
            tc_assemble_kernel<2><<<grid, 256, 0, h->stream>>>(I.N, h->tc_kpad, h->node, h->elem, h->tan, h->nrm,
                                                              h->tc_A, h->tc_A + na);
        else
            tc_assemble_kernel<3><<<grid, 256, 0, h->stream>>>(I.N, h->tc_kpad, h->node, h->elem, h->tan, h->nrm,
                                                              h->tc_A, h->tc_A + na);
        h->launches++;
        CKC(cudaGetLastError());
        h->kv_bytes = 4 * h->tc_mrows * I.N;   // hi + lo, 2 bytes each, per stored entry
#define TC_SMEM_ATTR(BN, ST) \
    CKC(cudaFuncSetAttribute(tc_gemm_kernel<BN, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_bytes(BN, ST)))
        TC_SMEM_ATTR(16, 4); TC_SMEM_ATTR(32, 4); TC_SMEM_ATTR(64, 4); TC_SMEM_ATTR(128, 3); TC_SMEM_ATTR(256, 2);
        TC_SMEM_ATTR(16, 2); TC_SMEM_ATTR(32, 2); TC_SMEM_ATTR(64, 2); TC_SMEM_ATTR(128, 2);
#undef TC_SMEM_ATTR
#define TC_SMEM_ATTR(BN, ST)                                                                                       \
    CKC(cudaFuncSetAttribute(tc_gemm_persistent_kernel<BN, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                             (int)tc_smem_bytes(BN, ST)))
        TC_SMEM_ATTR(16, 4); TC_SMEM_ATTR(32, 4); TC_SMEM_ATTR(64, 4); TC_SMEM_ATTR(128, 3); TC_SMEM_ATTR(256, 2);
#undef TC_SMEM_ATTR
        if (opt.gemv_impl < 0 || opt.gemv_impl > 2) {
            g_err = "gemv_impl of a tensor-core handle is 0 (persistent), 1 (deepest ring) or 2 (2-stage ring)";
            dfn_destroy(h);
            return DFN_ERR_ARG;
        }
        h->tc_variant = opt.gemv_impl;
    }
    // dense kernel matrices, one per network (one for a shared-geometry batch)
    h->K_bytes = (size_t)std::max<int64_t>(kvec, 1) * 16;
    if (!h->hmat && !h->tc) {
        cudaError_t e = cudaMalloc(&h->K, h->K_bytes);
        if (e != cudaSuccess) {
            set_err("cudaMalloc K", e, __FILE__, __LINE__);
            dfn_destroy(h);
            return DFN_ERR_NOMEM;
        }
    }
    if (h->s64) {
        const Inst &I = h->hinst[0];
        dim3 grid((unsigned)I.N, (unsigned)((I.Np + 255) / 256));
        if (h->mode == 2)
            assemble_kernel<2, 0><<<grid, 256, 0, h->stream>>>(I.N, I.Np, h->node, h->elem, h->tan, h->nrm, h->K);
        else
            assemble_kernel<3, 0><<<grid, 256, 0, h->stream>>>(I.N, I.Np, h->node, h->elem, h->tan, h->nrm, h->K);
        h->launches++;
        CKC(cudaGetLastError());
        DALLOC(h->s64_vt, I.Np * h->s64_rp);
        CKC(cudaFuncSetAttribute(s64_gemm_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)s64_smem_bytes(2)));
        CKC(cudaFuncSetAttribute(s64_gemm_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)s64_smem_bytes(3)));
    }
    std::vector<int4> tiles;
    for (int i = 0; i < count && !h->hmat && !h->tc && !h->s64; i++) {
        const Inst &I = h->hinst[i];
        const int64_t e0 = I.eoff;
        void *Ki = static_cast<unsigned char *>(h->K) + I.kvec * 16;
        dim3 grid((unsigned)I.N, (unsigned)((I.Np + 255) / 256));
#define ASM(MODE, STORE) \
    assemble_kernel<MODE, STORE><<<grid, 256, 0, h->stream>>>(I.N, I.Np, h->node + 2 * (e0 + i), h->elem + 2 * e0, h->tan + 2 * e0, h->nrm + 2 * e0, Ki)
        if (h->mode == 2) {
            if (h->store == 0) ASM(2, 0); else if (h->store == 1) ASM(2, 1); else ASM(2, 2);
        } else {
            if (h->store == 0) ASM(3, 0); else if (h->store == 1) ASM(3, 1); else ASM(3, 2);
        }
#undef ASM
        h->launches++;
        CKC(cudaGetLastError());
        const int64_t nrb = (I.N + GEMV_ROWS - 1) / GEMV_ROWS;
        for (int64_t rb = 0; rb < nrb; rb++)
            for (int64_t c = 0; c < I.nchunk; c++) tiles.push_back(make_int4(i, (int)c, (int)rb, 0));
        if (i == 0) h->ntiles0 = (int64_t)tiles.size();
    }
    h->ntiles = (int64_t)tiles.size();
    DALLOC(h->tiles, tiles.size());
    if (!tiles.empty()) HCOPY(h->tiles, tiles.data(), tiles.size());
    // TMA pipeline needs the dynamic shared memory opt-in
    {
        gemv_tma_fn fns[6] = {gemv_tma_kernel<2, 0>, gemv_tma_kernel<2, 1>, gemv_tma_kernel<2, 2>,
                              gemv_tma_kernel<3, 0>, gemv_tma_kernel<3, 1>, gemv_tma_kernel<3, 2>};
        for (auto fn : fns) CKC(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaSmem));
    }

    PressGlobal &pg = h->pg;
    pg.P = h->P; pg.permx = h->permx; pg.ds = h->ds; pg.src_fault = h->src_fault; pg.src_elem = h->src_elem;
    pg.src_Q = h->src_Q; pg.src_tb = h->src_tb; pg.src_te = h->src_te;
    pg.xptr = nullptr;
    pg.xcon = nullptr;
    pg.xrows = nullptr;
    pg.xrows_ptr = nullptr;
    pg.tcoef = nullptr;
    {
        std::vector<int64_t> xp;
        std::vector<XCon> xc;
        h->ncross = build_crossings(probs, count, h->hinst, xp, xc);
        if (h->ncross > 0 && h->pcoup) {
            g_err = "permeability coupling of networks with fault crossings is not supported (the crossing "
                    "coefficients hold the permeabilities of set-up)";
            dfn_destroy(h);
            return DFN_ERR_UNSUPPORTED;
        }
        if (h->ncross > 0) {
            if (h->pressure == DFN_PRESSURE_TRIDIAG) {
                g_err = "the network has fault crossings, which couple pressure rows outside the three diagonals: "
                        "use a CG pressure solver";
                dfn_destroy(h);
                return DFN_ERR_ARG;
            }
            CKC(cudaMalloc((void **)&h->xptr, sizeof(int64_t) * xp.size()));
            CKC(cudaMemcpyAsync(h->xptr, xp.data(), sizeof(int64_t) * xp.size(), cudaMemcpyHostToDevice, h->stream));
            CKC(cudaMalloc((void **)&h->xcon, sizeof(XCon) * std::max<size_t>(xc.size(), 1)));
            if (!xc.empty()) CKC(cudaMemcpyAsync(h->xcon, xc.data(), sizeof(XCon) * xc.size(), cudaMemcpyHostToDevice, h->stream));
            // per network, its rows that have crossings (network-local indices)
            std::vector<int64_t> rows, rptr(1, 0);
            for (int i = 0; i < count; i++) {
                const Inst &I = h->hinst[i];
                for (int64_t k = 0; k < I.N; k++)
                    if (xp[(size_t)(I.eoff + k) + 1] > xp[(size_t)(I.eoff + k)]) rows.push_back(k);
                rptr.push_back((int64_t)rows.size());
            }
            CKC(cudaMalloc((void **)&h->xrows, sizeof(int64_t) * std::max<size_t>(rows.size(), 1)));
            if (!rows.empty()) CKC(cudaMemcpyAsync(h->xrows, rows.data(), sizeof(int64_t) * rows.size(), cudaMemcpyHostToDevice, h->stream));
            CKC(cudaMalloc((void **)&h->xrows_ptr, sizeof(int64_t) * rptr.size()));
            CKC(cudaMemcpyAsync(h->xrows_ptr, rptr.data(), sizeof(int64_t) * rptr.size(), cudaMemcpyHostToDevice, h->stream));
            pg.xptr = h->xptr;
            pg.xcon = h->xcon;
            pg.xrows = h->xrows;
            pg.xrows_ptr = h->xrows_ptr;
        }
    }
    if (h->pressure == DFN_PRESSURE_TRIDIAG) {
        CKC(cudaMalloc((void **)&h->tcoef, sizeof(double) * 3 * (size_t)h->Ntot));
        tri_coef_kernel<<<blocks_of(h->Ntot, 256), 256, 0, h->stream>>>(pg, h->inst, h->inst_of, h->Ntot, h->tcoef);
        h->launches++;
        CKC(cudaGetLastError());
        pg.tcoef = h->tcoef;
    }

    // cluster CG (CG mode): the fewest CTAs per cluster (2 to 16) whose
    // ranges hold at most PCL_NTARGET elements, else the first of 8 roomy,
    // 16 roomy, 16 lean, 8 lean whose ranges fit in shared memory, taking
    // the first shape the device can schedule; systems under 2048 elements
    // keep the one-CTA solver
    bool attrs_ok = false;
    // (networks with fault crossings keep the one-CTA solver: their rows
    // couple elements of other faults, anywhere in the system)
    if (h->pressure == DFN_PRESSURE_CG && h->ncross == 0) {
        int64_t nmax = 0;
        for (int i = 0; i < count; i++) nmax = std::max<int64_t>(nmax, h->hinst[i].N);
        struct Shape { int cl; bool lean; };
        std::vector<Shape> cand;
        if (nmax >= 2048) {
            for (int c = 2; c <= 16; c *= 2)
                if ((nmax + c - 1) / c <= PCL_NTARGET) cand.push_back({c, false});
            const Shape more[4] = {{8, false}, {16, false}, {16, true}, {8, true}};
            for (const Shape &sh : more)
                if (pcl_smem_bytes((int)((nmax + sh.cl - 1) / sh.cl), sh.lean) <= (size_t)PCL_SMEM_CAP)
                    cand.push_back(sh);
        }
        // the attributes are per function, shared by every handle: set to
        // the largest values any handle may use
        attrs_ok =
            cudaFuncSetAttribute(pressure_cg_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
                cudaSuccess &&
            cudaFuncSetAttribute(pressure_cg_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 PCL_SMEM_CAP) == cudaSuccess;
        for (size_t q = 0; attrs_ok && q < cand.size(); q++) {
            const Shape &sh = cand[q];
            const int n = (int)((nmax + sh.cl - 1) / sh.cl);
            int nc = 0;
            cudaLaunchConfig_t cfg;
            cudaLaunchAttribute at[1];
            pcl_config(cfg, at, sh.cl, n, sh.lean, (unsigned)sh.cl, 1, h->stream);
            if (cudaOccupancyMaxActiveClusters(&nc, pressure_cg_cluster_kernel, &cfg) == cudaSuccess && nc > 0) {
                h->pcl = sh.cl;
                h->pcl_n = n;
                h->pcl_lean = sh.lean;
                h->pcl_max = nc;
                break;
            }
        }
        if (attrs_ok) {
            // one CTA per system with shared-memory vectors (autotuner's choice)
            int nc = 0;
            cudaLaunchConfig_t cfg;
            cudaLaunchAttribute at[1];
            pcl_config(cfg, at, 1, 0, false, 1, 1, h->stream);
            h->pcl_ok = cudaOccupancyMaxActiveClusters(&nc, pressure_cg_cluster_kernel, &cfg) == cudaSuccess && nc > 0;
        }
        cudaGetLastError();   // an unsupported shape leaves the one-CTA solver in place
    }

    // controllers: solve() entry, src/solver.f90:50-56
    for (int i = 0; i < count; i++) {
        StepCtl &c = h->h_ctl[i];
        memset(&c, 0, sizeof(c));
        c.time = probs[i].time0; c.t_try = 100.0; c.eps = probs[i].tol_solver; c.h = 100.0;
        c.phase = PH_DONE; c.max_attempts = h->max_attempts;
    }
    CKC(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(StepCtl) * count, cudaMemcpyHostToDevice, h->stream));
    CKC(cudaEventCreate(&h->ev0));
    CKC(cudaEventCreate(&h->ev1));
    CKC(cudaStreamSynchronize(h->stream));
    *out = h;
    return DFN_OK;
}

int32_t dfn_create(const dfn_problem *p, const dfn_options *opt, dfn_handle **out)
{
    return dfn_create_batch(p, 1, opt, out);
}

// Times the interchangeable launch shapes on this handle's own data and
// keeps the fastest: K.V through TMA bulk copies or 128-bit loads (bitwise
// identical results), and, with the tridiagonal pressure solve, short
// segments one thread or one warp each (equal to rounding). The timing
// launches write only per-attempt work buffers; the state is untouched.
int32_t dfn_autotune(dfn_handle *h, dfn_tuning *t)
{
    if (!h) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    dfn_tuning r;
    memset(&r, 0, sizeof(r));
    const bool prof = h->prof;
    h->prof = false;
    auto time_it = [&](auto &&launch, int reps, double &ms) -> int {
        TRY(launch());   // warm-up
        CK(cudaEventRecord(h->ev0, h->stream));
        for (int q = 0; q < reps; q++) TRY(launch());
        CK(cudaEventRecord(h->ev1, h->stream));
        CK(cudaEventSynchronize(h->ev1));
        float f = 0.0f;
        CK(cudaEventElapsedTime(&f, h->ev0, h->ev1));
        ms = f / reps;
        return DFN_OK;
    };
    r.gemv_impl = h->gemv_impl;
    if (!h->hmat && !h->tc && !h->s64) {
        const int keep = h->gemv_impl;
        for (int impl = 0; impl < 2; impl++) {
            h->gemv_impl = impl;
            TRY(time_it([&]() { return launch_gemv(h, M_ALL, h->Y, 3, false); }, 5, r.ms[impl]));
        }
        h->gemv_impl = (r.ms[1] < r.ms[0]) ? 1 : 0;
        r.gemv_impl = h->gemv_impl;
        (void)keep;
    }
    if (h->hmat) {
        // grids of the dense-row and small-leaf kernels: one CTA per task
        // (0) or persistent grids of 4 or 8 CTAs per SM; identical results
        const int64_t opts[3] = {0, 4 * (int64_t)h->sms, 8 * (int64_t)h->sms};
        double best = 1e300;
        int64_t bd = 0, bw = 0;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                h->hm_dense_grid = opts[a];
                h->hm_warp_grid = 2 * opts[b];
                double ms = 0.0;
                TRY(time_it([&]() { return launch_gemv(h, M_ALL, h->Y, 3, false); }, 5, ms));
                if (ms < best) { best = ms; bd = opts[a]; bw = 2 * opts[b]; }
                if (a == 0 && b == 0) r.ms[1] = ms;
            }
        h->hm_dense_grid = bd;
        h->hm_warp_grid = bw;
        r.ms[0] = best;
        r.hm_dense_grid = bd;
        r.hm_warp_grid = bw;
    }
    if (h->tc) {
        // persistent -> ms[0], unit per CTA with the deepest ring -> ms[1],
        // unit per CTA with a 2-stage ring -> ms[4] (when that is another shape)
        const int nv = tc_stages(h->tc_bn) > 2 ? 3 : 2;
        double msv[3] = {0.0, 0.0, 0.0};
        for (int v = 0; v < nv; v++) {
            h->tc_variant = v;
            TRY(time_it([&]() { return launch_gemv(h, M_ALL, h->Y, 3, false); }, 5, msv[v]));
        }
        int best = 0;
        for (int v = 1; v < nv; v++)
            if (msv[v] < msv[best]) best = v;
        h->tc_variant = best;
        r.ms[0] = msv[0];
        r.ms[1] = msv[1];
        r.ms[4] = msv[2];
        r.gemv_impl = best;
    }
    r.tri_thread = h->tri_shape;
    if (h->pressure == DFN_PRESSURE_CG && h->pcl_ok) {
        // one CTA on global memory -> ms[2], clusters -> ms[3] (when this
        // handle has a cluster form), one CTA on shared memory -> ms[5]
        double msv[3] = {0.0, 0.0, 0.0};
        for (int v = 0; v < 3; v++) {
            if (v == 1 && h->pcl == 0) continue;
            h->pcl_mode = v;
            TRY(time_it([&]() { return launch_pressure(h, M_ALL, 2, 1, 5, 100.0, h->B); }, 3, msv[v]));
        }
        int best = 0;
        for (int v = 1; v < 3; v++)
            if (msv[v] > 0.0 && msv[v] < msv[best]) best = v;
        h->pcl_mode = best;
        r.ms[2] = msv[0];
        r.ms[3] = msv[1];
        r.ms[5] = msv[2];
    }
    r.cg_cluster_ctas = h->pressure == DFN_PRESSURE_CG ? h->pcl : 0;
    r.cg_cluster = 0;
    if (h->pressure == DFN_PRESSURE_CG) {
        if (h->pcl_mode == 2) r.cg_cluster = 2;
        else if (h->pcl > 0 && (h->pcl_mode == 1 || (h->pcl_mode < 0 && 5 * h->B <= h->pcl_max))) r.cg_cluster = 1;
    }
    if (h->pressure == DFN_PRESSURE_TRIDIAG && h->nshort > 0) {
        // warps -> ms[2], threads -> ms[3], tiles -> ms[5]
        double msv[3];
        for (int v = 0; v < 3; v++) {
            h->tri_shape = v;
            TRY(time_it([&]() { return launch_pressure(h, M_ALL, 2, 1, 5, 100.0, h->B); }, 3, msv[v]));
        }
        int best = 0;
        for (int v = 1; v < 3; v++)
            if (msv[v] < msv[best]) best = v;
        h->tri_shape = best;
        r.ms[2] = msv[0];
        r.ms[3] = msv[1];
        r.ms[5] = msv[2];
        r.tri_thread = best;
    }
    h->prof = prof;
    drop_graph(h);
    CK(cudaStreamSynchronize(h->stream));
    if (t) *t = r;
    return DFN_OK;
}

int32_t dfn_set_graphs(dfn_handle *h, int32_t enable)
{
    if (!h) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    h->use_graphs = enable != 0;
    drop_graph(h);
    return DFN_OK;
}

int32_t dfn_set_wait_limit(dfn_handle *h, int32_t polls)
{
    if (!h) return DFN_ERR_ARG;
    h->wait_polls = polls < 0 ? MBAR_POLLS : polls;
    drop_graph(h);   // a captured graph holds the old limit in its kernel parameters
    return DFN_OK;
}

int64_t dfn_crossing_count(const dfn_handle *h) { return h ? h->ncross : -1; }

int32_t dfn_set_hmat_grids(dfn_handle *h, int64_t dense_ctas, int64_t warp_ctas)
{
    if (!h || dense_ctas < 0 || warp_ctas < 0) return DFN_ERR_ARG;
    if (!h->hmat) return DFN_ERR_UNSUPPORTED;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    h->hm_dense_grid = dense_ctas;
    h->hm_warp_grid = warp_ctas;
    drop_graph(h);
    return DFN_OK;
}

int32_t dfn_set_tri_shape(dfn_handle *h, int32_t shape)
{
    if (!h) return DFN_ERR_ARG;
    if (shape < 0 || shape > 2 || h->pressure != DFN_PRESSURE_TRIDIAG) {
        g_err = "short-segment shape is 0, 1 or 2 on a tridiagonal-pressure handle";
        return DFN_ERR_ARG;
    }
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    h->tri_shape = shape;
    drop_graph(h);
    return DFN_OK;
}

int32_t dfn_set_cg_form(dfn_handle *h, int32_t form)
{
    if (!h) return DFN_ERR_ARG;
    if (form < -1 || form > 2 || h->pressure != DFN_PRESSURE_CG || (form >= 1 && !h->pcl_ok) ||
        (form == 1 && h->pcl == 0)) {
        g_err = "CG form not available on this handle (CG pressure; 1 needs systems of 2048 elements or more)";
        return DFN_ERR_ARG;
    }
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    h->pcl_mode = form;
    drop_graph(h);
    return DFN_OK;
}

int32_t dfn_set_hmat_small_leaves(dfn_handle *h, int32_t form)
{
    if (!h) return DFN_ERR_ARG;
    if (!h->hmat) { g_err = "handle uses the dense kernel"; return DFN_ERR_UNSUPPORTED; }
    if (form < 0 || form > 1) { g_err = "form must be 0 (one warp per leaf) or 1 (one CTA per leaf)"; return DFN_ERR_ARG; }
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    h->small_form = form;
    drop_graph(h);
    return DFN_OK;
}

int32_t dfn_set_stream(dfn_handle *h, void *s)
{
    if (!h) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->own_stream = false;
    h->stream = (cudaStream_t)s;
    return DFN_OK;
}

int32_t dfn_batch_size(const dfn_handle *h) { return h ? h->B : -1; }
int64_t dfn_nb_element(const dfn_handle *h) { return h ? h->hinst[0].N : -1; }
int64_t dfn_kernel_bytes(const dfn_handle *h) { return h ? h->kv_bytes : -1; }
int64_t dfn_launch_count(const dfn_handle *h) { return h ? h->launches : -1; }

int32_t dfn_kernel_device(dfn_handle *h, const double *d_slip, double *d_sT, double *d_sN)
{
    if (!h || !d_slip || !d_sT) return DFN_ERR_ARG;
    TRY(single_only(h));
    CK(cudaSetDevice(h->dev));
    const Inst &I = h->hinst[0];
    TRY(launch_gemv(h, M_ALL, d_slip, 1, true));
    kv_finish_kernel<<<blocks_of(I.N, 256), 256, 0, h->stream>>>(I.N, h->mode, (int)I.nchunk, I.prefT, h->partT,
                                                                 h->partN, d_sT, d_sN);
    h->launches++;
    CKL();
    return DFN_OK;
}

int32_t dfn_kernel_batch(dfn_handle *h, const double *slip, double *sT, double *sN)
{
    if (!h || !slip || !sT) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    const int64_t Nt = h->Ntot;
    double *d = nullptr;
    CK(cudaMalloc((void **)&d, sizeof(double) * 3 * Nt));
    int st = DFN_OK;
    cudaError_t e = cudaMemcpyAsync(d, slip, sizeof(double) * Nt, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) st = launch_gemv(h, M_ALL, d, 1, false);
    for (int i = 0; i < h->B && e == cudaSuccess && st == DFN_OK; i++) {
        const Inst &I = h->hinst[i];
        kv_finish_kernel<<<blocks_of(I.N, 256), 256, 0, h->stream>>>(I.N, h->mode, (int)I.nchunk, I.prefT,
                                                                     h->partT + I.poff, h->partN + I.poff,
                                                                     d + Nt + I.eoff, d + 2 * Nt + I.eoff);
        h->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && st == DFN_OK)
        e = cudaMemcpyAsync(sT, d + Nt, sizeof(double) * Nt, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && st == DFN_OK && sN)
        e = cudaMemcpyAsync(sN, d + 2 * Nt, sizeof(double) * Nt, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) {
        set_err("dfn_kernel_batch", e, __FILE__, __LINE__);
        return DFN_ERR_CUDA;
    }
    if (st != DFN_OK) return st;
    int flag = 0;
    CK(cudaMemcpy(&flag, h->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        CK(cudaMemsetAsync(h->err_flag, 0, sizeof(int), h->stream));
        g_err = "a bounded wait of a K.V pipeline expired (its partial sums are incomplete)";
        return DFN_ERR_TIMEOUT;
    }
    return DFN_OK;
}

int32_t dfn_kernel(dfn_handle *h, const double *slip, double *sT, double *sN)
{
    if (!h || !slip || !sT) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t N = h->hinst[0].N;
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(h->vin, slip, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
    TRY(dfn_kernel_device(h, h->vin, h->vout, h->vout + N));
    CK(cudaMemcpyAsync(sT, h->vout, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    if (sN) CK(cudaMemcpyAsync(sN, h->vout + N, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    return DFN_OK;
}

static int reset_status0(dfn_handle *h)
{
    CK(cudaMemsetAsync(&h->ctl[0].status, 0, sizeof(int), h->stream));
    return DFN_OK;
}

int32_t dfn_compute_P(dfn_handle *h, double dt, double *P_temp, double *P_dot, int32_t *ier)
{
    if (!h || !P_temp || !P_dot) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t N = h->hinst[0].N;
    CK(cudaSetDevice(h->dev));
    TRY(reset_status0(h));
    if (h->pcoup) TRY(perm_refresh(h, M_ALL, 0));
    TRY(launch_pressure(h, M_ALL, 2, 0, 1, dt, 1));
    TRY(sync_ctl(h));
    int st = h->h_ctl[0].status;
    if (ier) *ier = (st == 1) ? 1 : 0;
    if (st == 1) { TRY(reset_status0(h)); return DFN_OK; }
    if (st) return st;
    CK(cudaMemcpy(P_temp, h->Ptemp, sizeof(double) * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(P_dot, h->Pdot_s, sizeof(double) * N, cudaMemcpyDeviceToHost));
    return DFN_OK;
}

int32_t dfn_friction_law(dfn_handle *h, double x, int64_t nv, const double *Y, double *Ydot)
{
    if (!h || !Y || !Ydot) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t N = h->hinst[0].N;
    if (nv != 3 * N) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    TRY(reset_status0(h));
    CK(cudaMemcpyAsync(h->ytmp, Y, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, h->stream));
    if (h->pcoup) TRY(perm_refresh(h, M_ALL, 0));
    TRY(launch_pressure(h, M_ALL, 2, 0, 1, x, 1));
    TRY(launch_gemv(h, M_ALL, h->ytmp, 3, true));
    TRY(launch_friction(h, 0, 0, M_ALL, N, x));
    CK(cudaMemcpyAsync(Ydot, h->kbuf, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    int st = h->h_ctl[0].status;
    TRY(reset_status0(h));
    return st;
}

int32_t dfn_rkqs(dfn_handle *h, double *y, const double *dydx, int64_t nv, double *x, double htry, double eps,
                 const double *yscal, double *hdid, double *hnext)
{
    if (!h || !y || !dydx || !x || !yscal || !hdid || !hnext) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t n3 = 3 * h->hinst[0].N;
    if (nv != n3) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(h->Y, y, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->kbuf, dydx, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->yscal, yscal, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
    TRY(sync_ctl(h));
    StepCtl saved = h->h_ctl[0];
    StepCtl &c = h->h_ctl[0];
    c.x = *x; c.h = htry; c.eps = eps; c.accepted = 0; c.status = 0; c.phase = PH_RETRY; c.step_attempts = 0;
    c.max_attempts = h->max_attempts;
    TRY(put_ctl(h));
    if (h->pcoup) TRY(perm_refresh(h, M_ALL, 0));
    for (;;) {
        TRY(run_attempt(h, M_ACTIVE));
        TRY(sync_ctl(h));
        if (h->h_ctl[0].status) return h->h_ctl[0].status;
        if (h->h_ctl[0].accepted) break;
    }
    CK(cudaMemcpyAsync(h->Y, h->yout, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(y, h->yout, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    *hdid = h->h_ctl[0].hdid;
    *hnext = h->h_ctl[0].hnext;
    *x = *x + *hdid;
    StepCtl &d = h->h_ctl[0];
    d.eps = saved.eps; d.x = 0.0; d.phase = PH_DONE;
    TRY(put_ctl(h));
    return DFN_OK;
}

int32_t dfn_solve_steps(dfn_handle *h, int64_t n_steps, dfn_report *rep)
{
    if (!h || n_steps < 0) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    int st = solve_impl(h, n_steps, 0.0);
    int st2 = sync_ctl(h);
    if (st == DFN_OK) st = st2;
    if (st == DFN_OK) {
        for (int i = 0; i < h->B; i++)
            if (h->h_ctl[i].status) { st = h->h_ctl[i].status; break; }
    }
    fill_report(h->h_ctl[0], rep);
    return st;
}

int32_t dfn_solve_batch(dfn_handle *h, int64_t n_steps, double t_end, dfn_report *reps)
{
    if (!h || n_steps < 0 || !(t_end >= 0.0)) return DFN_ERR_ARG;
    if (t_end > 0.0 && n_steps == 0) n_steps = (int64_t)1 << 62;
    CK(cudaSetDevice(h->dev));
    int st = solve_impl(h, n_steps, t_end);
    int st2 = sync_ctl(h);
    if (st == DFN_OK) st = st2;
    if (reps)
        for (int i = 0; i < h->B; i++) fill_report(h->h_ctl[i], &reps[i]);
    return st;
}

int32_t dfn_get_state_instance(dfn_handle *h, int32_t i, double *Y, double *P, double *time, double *t_try,
                               int64_t *it_count)
{
    if (!h || i < 0 || i >= h->B) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    TRY(sync_ctl(h));
    const Inst &I = h->hinst[i];
    if (Y) CK(cudaMemcpy(Y, h->Y + 3 * I.eoff, sizeof(double) * 3 * I.N, cudaMemcpyDeviceToHost));
    if (P) CK(cudaMemcpy(P, h->P + I.eoff, sizeof(double) * I.N, cudaMemcpyDeviceToHost));
    if (time) *time = h->h_ctl[i].time;
    if (t_try) *t_try = h->h_ctl[i].t_try;
    if (it_count) *it_count = h->h_ctl[i].it_count;
    return DFN_OK;
}

int32_t dfn_get_slip(dfn_handle *h, int32_t i, double *slip)
{
    if (!h || !slip || i < 0 || i >= h->B) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    const Inst &I = h->hinst[i];
    const double *src = (h->form == DFN_FORM_NEWTON) ? h->Y + 3 * I.eoff : h->slip + I.eoff;
    CK(cudaMemcpyAsync(slip, src, sizeof(double) * I.N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DFN_OK;
}

int32_t dfn_set_slip(dfn_handle *h, int32_t i, const double *slip)
{
    if (!h || !slip || i < 0 || i >= h->B) return DFN_ERR_ARG;
    const Inst &I = h->hinst[i];
    if (!all_finite(slip, I.N)) {
        g_err = "dfn_set_slip: non-finite slip";
        return DFN_ERR_NONFINITE;
    }
    CK(cudaSetDevice(h->dev));
    double *dst = (h->form == DFN_FORM_NEWTON) ? h->Y + 3 * I.eoff : h->slip + I.eoff;
    CK(cudaMemcpyAsync(dst, slip, sizeof(double) * I.N, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DFN_OK;
}

int32_t dfn_get_report(dfn_handle *h, int32_t i, dfn_report *rep)
{
    if (!h || !rep || i < 0 || i >= h->B) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    TRY(sync_ctl(h));
    fill_report(h->h_ctl[i], rep);
    return DFN_OK;
}

int32_t dfn_get_state(dfn_handle *h, double *Y, double *P, double *time, double *t_try, int64_t *it_count)
{
    return dfn_get_state_instance(h, 0, Y, P, time, t_try, it_count);
}

int32_t dfn_set_state(dfn_handle *h, const double *Y, const double *P, double time, double t_try, int64_t it_count)
{
    if (!h) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t N = h->hinst[0].N;
    if ((Y && !all_finite(Y, 3 * N)) || (P && !all_finite(P, N)) || !std::isfinite(time) || !std::isfinite(t_try)) {
        g_err = "dfn_set_state: non-finite value in the state";
        return DFN_ERR_NONFINITE;
    }
    CK(cudaSetDevice(h->dev));
    if (Y) CK(cudaMemcpyAsync(h->Y, Y, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, h->stream));
    if (P) CK(cudaMemcpyAsync(h->P, P, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
    TRY(sync_ctl(h));
    StepCtl &c = h->h_ctl[0];
    c.time = time; c.t_try = t_try; c.it_count = it_count; c.status = 0;
    TRY(put_ctl(h));
    return DFN_OK;
}

int32_t dfn_get_snapshot(dfn_handle *h, double *V, double *theta, double *P, double *tT, double *tN,
                         double *permeability, double *time)
{
    if (!h) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t N = h->hinst[0].N;
    CK(cudaSetDevice(h->dev));
    snapshot_kernel<<<blocks_of(N, 256), 256, 0, h->stream>>>(N, h->Y, h->Dc, h->V0, h->P, h->SigT, h->snap);
    h->launches++;
    CKL();
    double *dst[5] = {V, theta, P, tT, tN};
    for (int i = 0; i < 5; i++)
        if (dst[i]) CK(cudaMemcpyAsync(dst[i], h->snap + i * N, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    if (permeability) CK(cudaMemcpyAsync(permeability, h->perm, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    if (time) *time = h->h_ctl[0].time;
    return DFN_OK;
}

int32_t dfn_step_host(dfn_handle *h, const double *Y_in, const double *P_in, double time_in, double t_try_in,
                      double *V_out, double *theta_out, double *P_out, double *tT_out, double *tN_out,
                      dfn_report *rep)
{
    if (!h || !Y_in || !P_in) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t N = h->hinst[0].N;
    if (!all_finite(Y_in, 3 * N) || !all_finite(P_in, N) || !std::isfinite(time_in) || !std::isfinite(t_try_in)) {
        g_err = "dfn_step_host: non-finite value in the state";
        return DFN_ERR_NONFINITE;
    }
    CK(cudaSetDevice(h->dev));
    TRY(sync_ctl(h));
    CK(cudaMemcpyAsync(h->Y, Y_in, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->P, P_in, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
    StepCtl &c = h->h_ctl[0];
    c.time = time_in; c.t_try = t_try_in; c.status = 0;
    CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice, h->stream));
    int st = solve_impl(h, 1, 0.0);
    if (st != DFN_OK) { sync_ctl(h); fill_report(h->h_ctl[0], rep); return st; }
    TRY(dfn_get_snapshot(h, V_out, theta_out, P_out, tT_out, tN_out, nullptr, nullptr));
    fill_report(h->h_ctl[0], rep);
    return h->h_ctl[0].status;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free pressure step. The CG work vectors of dfn_compute_P_noalloc
// live in this fixed device array: the first 32 doubles (256 bytes) hold the
// step controller the CG kernel reports into, then 4 vectors of
// DFN_NOALLOC_MAX_ELEMENTS doubles (x, r, p, M.p). In host code the symbol is
// only a handle for cudaGetSymbolAddress, never a device address.
static const int64_t kNoAllocCtlDoubles = 32;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocCtlDoubles + 4 * (int64_t)DFN_NOALLOC_MAX_ELEMENTS];
static_assert(sizeof(StepCtl) <= kNoAllocCtlDoubles * sizeof(double), "controller does not fit the scratch header");

// Device address of the scratch array in the context current on the
// calling thread. Looked up on every call (cheap next to the call's own
// stream synchronisation): the address belongs to the context that loaded
// the module, so a cached value would go stale after cudaDeviceReset or
// under another context of the same device.
static int noalloc_scratch(double **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        set_err("cudaGetSymbolAddress(g_noalloc_scratch)", e, __FILE__, __LINE__);
        return DFN_ERR_CUDA;
    }
    *out = static_cast<double *>(p);
    return DFN_OK;
}

// Clears the shared controller (status, counters) and sets time and tol:
// the array keeps the previous call's contents.
static __global__ void noalloc_reset_kernel(StepCtl *ctl, double time, double tol)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    StepCtl c;
    memset(&c, 0, sizeof(c));
    c.time = time;
    c.eps = tol;
    *ctl = c;
}

extern "C" {

int32_t dfn_compute_P_noalloc(int64_t N, double dt, double time, const double *d_P, const double *d_permx,
                              const double *d_ds, double porosity, double dyn_viscosity, double fluid_comp,
                              double rock_comp, double tol_solver, int64_t nsrc, const int64_t *d_src_fault,
                              const int64_t *d_src_elem, const double *d_src_Q, const double *d_src_tb,
                              const double *d_src_te, double *d_P_temp, double *d_P_dot, int32_t *ier,
                              void *stream)
{
    if (N > DFN_NOALLOC_MAX_ELEMENTS) {
        g_err = "nb_element exceeds DFN_NOALLOC_MAX_ELEMENTS (65536) of the allocation-free pressure step";
        return DFN_ERR_ARG;
    }
    if (N < 2 || !d_P || !d_permx || !d_ds || !d_P_temp || !d_P_dot || !ier || !(tol_solver > 0) ||
        nsrc < 0 || (nsrc > 0 && (!d_src_fault || !d_src_elem || !d_src_Q || !d_src_tb || !d_src_te))) {
        g_err = "dfn_compute_P_noalloc: invalid argument";
        return DFN_ERR_ARG;
    }
    double *scratch = nullptr;
    TRY(noalloc_scratch(&scratch));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    StepCtl *ctl = reinterpret_cast<StepCtl *>(scratch);
    double *work = scratch + kNoAllocCtlDoubles;

    PressParams pp{};
    pp.N = N; pp.P = d_P; pp.permx = d_permx; pp.ds = d_ds;
    pp.porosity = porosity; pp.dyn_visc = dyn_viscosity; pp.comp = fluid_comp + rock_comp;
    pp.tol = tol_solver; pp.nsrc = nsrc; pp.src_fault = d_src_fault; pp.src_elem = d_src_elem;
    pp.src_Q = d_src_Q; pp.src_tb = d_src_tb; pp.src_te = d_src_te; pp.ctl_time = &ctl->time;

    noalloc_reset_kernel<<<1, 32, 0, s>>>(ctl, time, tol_solver);
    CKL();
    pressure_cg_kernel<<<1, 1024, 0, s>>>(pp, ctl, 2, 0, dt, d_P_temp, d_P_dot, work);
    CKL();
    StepCtl c;
    CK(cudaMemcpyAsync(&c, ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // ier = 1 for the CG cap (outputs untouched) and for a non-finite
    // solution (outputs written, as the reference's maxval test after the
    // update, src/fluid_diffusion.f90:146-148); the latter also returns
    // DFN_ERR_NONFINITE
    *ier = (c.status == 1 || c.status == 4) ? 1 : 0;
    if (c.status != 0 && c.status != 1) return c.status;
    return DFN_OK;
}

int32_t dfn_set_mlp(dfn_handle *h, const float *weights)
{
    if (!h || !weights) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    // FP32 weights in, the kernels' FP16 tensor-core image out
    float *w = nullptr;
    CK(cudaMalloc((void **)&w, sizeof(float) * MLP_NPAR));
    cudaError_t e = cudaMemcpyAsync(w, weights, sizeof(float) * MLP_NPAR, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        mlp_image_kernel<<<1, 256, 0, h->stream>>>(w, h->mlp);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(w);
    if (e != cudaSuccess) {
        set_err("dfn_set_mlp", e, __FILE__, __LINE__);
        return DFN_ERR_CUDA;
    }
    return DFN_OK;
}

int32_t dfn_set_mlp_gate(dfn_handle *h, double rel)
{
    if (!h || !(rel >= 0.0)) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    h->mlp_gate = rel;
    drop_graph(h);   // a captured graph holds the old gate in its kernel parameters
    return DFN_OK;
}

int32_t dfn_record(dfn_handle *h, int64_t capacity)
{
    if (!h || capacity < 0) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    if (h->rec_x) { cudaFree(h->rec_x); h->rec_x = nullptr; }
    if (h->rec_t) { cudaFree(h->rec_t); h->rec_t = nullptr; }
    h->rec_cap = 0;
    drop_graph(h);        // the friction launches carry the recording buffers
    CK(cudaMemsetAsync(h->rec_n, 0, sizeof(unsigned long long), h->stream));
    if (capacity > 0) {
        CK(cudaMalloc((void **)&h->rec_x, sizeof(float) * MLP_IN * capacity));
        CK(cudaMalloc((void **)&h->rec_t, sizeof(float) * capacity));
        h->rec_cap = capacity;
    }
    return DFN_OK;
}

int32_t dfn_record_read(dfn_handle *h, float *x, float *t, int64_t max, int64_t *count)
{
    if (!h || !count) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    unsigned long long n = 0;
    CK(cudaMemcpy(&n, h->rec_n, sizeof(n), cudaMemcpyDeviceToHost));
    int64_t m = std::min<int64_t>((int64_t)n, h->rec_cap);
    m = std::min<int64_t>(m, max);
    if (m > 0 && x) CK(cudaMemcpy(x, h->rec_x, sizeof(float) * MLP_IN * m, cudaMemcpyDeviceToHost));
    if (m > 0 && t) CK(cudaMemcpy(t, h->rec_t, sizeof(float) * m, cudaMemcpyDeviceToHost));
    *count = m;
    return DFN_OK;
}

// Gradient (and optionally an Adam step) over samples [0, n) of device
// arrays in batches; returns the summed squared error.
static int mlp_pass(const float *dX, const float *dT, int64_t n, int64_t n_total, float *dW, float *dm, float *dv,
                    float *dg, float *dgp, float *dlp, float *dls, int step, float lr, float *loss_sum,
                    cudaStream_t s)
{
    const int nblk = (int)((n + MLP_SB - 1) / MLP_SB);
    const size_t smem = sizeof(MlpSmem);
    CK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mlp_grad_kernel<<<nblk, 256, smem, s>>>(dX, dT, n, n_total, dW, dgp, dlp);
    CKL();
    mlp_reduce_adam_kernel<<<(MLP_NPAR + 255) / 256, 256, 0, s>>>(dgp, nblk, dW, dm, dv, dg, step, lr);
    CKL();
    sum_kernel<<<1, 32, 0, s>>>(dlp, nblk, dls);
    CKL();
    float l = 0.0f;
    CK(cudaMemcpyAsync(&l, dls, sizeof(float), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *loss_sum = l;
    return DFN_OK;
}

struct MlpBuffers {
    float *X = nullptr, *T = nullptr, *W = nullptr, *m = nullptr, *v = nullptr, *g = nullptr, *gp = nullptr,
          *lp = nullptr, *ls = nullptr;
    ~MlpBuffers()
    {
        float *p[] = {X, T, W, m, v, g, gp, lp, ls};
        for (float *q : p)
            if (q) cudaFree(q);
    }
};

static int mlp_alloc(MlpBuffers &b, int64_t n, int64_t batch)
{
    const int64_t nblk = (batch + MLP_SB - 1) / MLP_SB;
    CK(cudaMalloc((void **)&b.X, sizeof(float) * MLP_IN * std::max<int64_t>(n, 1)));
    CK(cudaMalloc((void **)&b.T, sizeof(float) * std::max<int64_t>(n, 1)));
    CK(cudaMalloc((void **)&b.W, sizeof(float) * MLP_NPAR));
    CK(cudaMalloc((void **)&b.m, sizeof(float) * MLP_NPAR));
    CK(cudaMalloc((void **)&b.v, sizeof(float) * MLP_NPAR));
    CK(cudaMalloc((void **)&b.g, sizeof(float) * MLP_NPAR));
    CK(cudaMalloc((void **)&b.gp, sizeof(float) * MLP_NPAR * nblk));
    CK(cudaMalloc((void **)&b.lp, sizeof(float) * nblk));
    CK(cudaMalloc((void **)&b.ls, sizeof(float)));
    CK(cudaMemset(b.m, 0, sizeof(float) * MLP_NPAR));
    CK(cudaMemset(b.v, 0, sizeof(float) * MLP_NPAR));
    return DFN_OK;
}

int32_t dfn_mlp_loss_grad(const float *x, const float *t, int64_t n, const float *weights, float *loss, float *grad)
{
    if (!x || !t || n < 1 || !weights || !loss || !grad) return DFN_ERR_ARG;
    MlpBuffers b;
    TRY(mlp_alloc(b, n, n));
    CK(cudaMemcpy(b.X, x, sizeof(float) * MLP_IN * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.T, t, sizeof(float) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.W, weights, sizeof(float) * MLP_NPAR, cudaMemcpyHostToDevice));
    float ls = 0.0f;
    TRY(mlp_pass(b.X, b.T, n, n, b.W, b.m, b.v, b.g, b.gp, b.lp, b.ls, 1, 0.0f, &ls, nullptr));
    *loss = ls / (float)n;
    CK(cudaMemcpy(grad, b.g, sizeof(float) * MLP_NPAR, cudaMemcpyDeviceToHost));
    return DFN_OK;
}

int32_t dfn_mlp_infer(const float *x, int64_t n, const float *weights, float *y)
{
    if (!x || n < 1 || !weights || !y) return DFN_ERR_ARG;
    MlpBuffers b;
    CK(cudaMalloc((void **)&b.X, sizeof(float) * MLP_IN * n));
    CK(cudaMalloc((void **)&b.T, sizeof(float) * n));
    CK(cudaMalloc((void **)&b.W, sizeof(float) * MLP_NPAR));
    CK(cudaMemcpy(b.X, x, sizeof(float) * MLP_IN * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.W, weights, sizeof(float) * MLP_NPAR, cudaMemcpyHostToDevice));
    mlp_infer_kernel<<<(unsigned)((n + 255) / 256), 256, sizeof(MlpTC)>>>(b.X, n, b.W, b.T);
    CK(cudaGetLastError());
    CK(cudaMemcpy(y, b.T, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return DFN_OK;
}

int32_t dfn_mlp_train(const float *x, const float *t, int64_t n, float *weights, int32_t epochs, int32_t batch,
                      float lr, uint64_t seed, float *loss)
{
    if (!x || !t || n < 1 || !weights || epochs < 1 || batch < 1 || !(lr > 0)) return DFN_ERR_ARG;
    // seeded shuffle of the samples (host), then epochs over fixed minibatches
    std::vector<int64_t> order(n);
    for (int64_t i = 0; i < n; i++) order[i] = i;
    uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
    for (int64_t i = n - 1; i > 0; i--) {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        const int64_t j = (int64_t)((st >> 33) % (uint64_t)(i + 1));
        std::swap(order[i], order[j]);
    }
    std::vector<float> xs((size_t)MLP_IN * n), ts(n);
    for (int64_t i = 0; i < n; i++) {
        for (int q = 0; q < MLP_IN; q++) xs[(size_t)i * MLP_IN + q] = x[order[i] * MLP_IN + q];
        ts[i] = t[order[i]];
    }
    MlpBuffers b;
    TRY(mlp_alloc(b, n, batch));
    CK(cudaMemcpy(b.X, xs.data(), sizeof(float) * xs.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.T, ts.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.W, weights, sizeof(float) * MLP_NPAR, cudaMemcpyHostToDevice));
    int step = 0;
    for (int ep = 0; ep < epochs; ep++) {
        double esum = 0.0;
        for (int64_t s0 = 0; s0 < n; s0 += batch) {
            const int64_t m = std::min<int64_t>(batch, n - s0);
            float ls = 0.0f;
            TRY(mlp_pass(b.X + s0 * MLP_IN, b.T + s0, m, m, b.W, b.m, b.v, nullptr, b.gp, b.lp, b.ls, ++step, lr,
                         &ls, nullptr));
            esum += ls;
        }
        if (loss && ep == 0) loss[0] = (float)(esum / n);
        if (loss && ep == epochs - 1) loss[1] = (float)(esum / n);
    }
    CK(cudaMemcpy(weights, b.W, sizeof(float) * MLP_NPAR, cudaMemcpyDeviceToHost));
    return DFN_OK;
}

int32_t dfn_velocity(dfn_handle *h, double *V)
{
    if (!h || !V) return DFN_ERR_ARG;
    TRY(single_only(h));
    const int64_t N = h->hinst[0].N;
    CK(cudaSetDevice(h->dev));
    if (h->form != DFN_FORM_NEWTON) {
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaMemcpy(V, h->Y, sizeof(double) * N, cudaMemcpyDeviceToHost));
        return DFN_OK;
    }
    // stresses of the committed slip, pressure at dt = 0 (the committed P),
    // then the friction law for V
    TRY(reset_status0(h));
    CK(cudaMemcpyAsync(h->ytmp, h->Y, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, h->stream));
    TRY(launch_pressure(h, M_ALL, 2, 0, 1, 0.0, 1));
    TRY(launch_gemv(h, M_ALL, h->ytmp, 3, true));
    TRY(launch_friction(h, 0, 0, M_ALL, N, 0.0));
    CK(cudaMemcpyAsync(V, h->vnow, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    return DFN_OK;
}

int32_t dfn_hmat_stats(const dfn_handle *h, int64_t *st)
{
    if (!h || !st) return DFN_ERR_ARG;
    if (!h->hmat) { g_err = "handle uses the dense kernel"; return DFN_ERR_UNSUPPORTED; }
    const int64_t nlr = (int64_t)h->hranks.size();
    int64_t mx = 0, sum = 0;
    for (int r : h->hranks) { mx = std::max<int64_t>(mx, r); sum += r; }
    st[0] = h->hblocks; st[1] = h->hblocks - nlr; st[2] = nlr; st[3] = mx;
    st[4] = nlr ? (1000 * sum) / nlr : 0;
    st[5] = h->hdense_vals + h->hlr_vals; st[6] = h->hdense_vals; st[7] = h->hlr_vals;
    return DFN_OK;
}

int32_t dfn_hmat_perm(const dfn_handle *h, int32_t *perm)
{
    if (!h || !perm) return DFN_ERR_ARG;
    if (!h->hmat) { g_err = "handle uses the dense kernel"; return DFN_ERR_UNSUPPORTED; }
    CK(cudaMemcpy(perm, h->hperm, sizeof(int) * h->hinst[0].N, cudaMemcpyDeviceToHost));
    return DFN_OK;
}

int32_t dfn_profile_kv(dfn_handle *h, int32_t enable)
{
    if (!h) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    if (enable && h->pev.empty()) {
        h->pev.resize(2 * kProfMax);
        for (auto &e : h->pev) CK(cudaEventCreate(&e));
    }
    h->prof = enable != 0;
    h->pcount = 0;
    return DFN_OK;
}

int32_t dfn_profile_kv_read(dfn_handle *h, double *total_ms, int64_t *n)
{
    if (!h || !total_ms || !n) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    double t = 0.0;
    for (int i = 0; i < h->pcount; i++) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, h->pev[2 * i], h->pev[2 * i + 1]));
        t += ms;
    }
    *total_ms = t;
    *n = h->pcount;
    return DFN_OK;
}

int32_t dfn_time_kernel(dfn_handle *h, int32_t reps, double *ms)
{
    if (!h || reps < 1 || !ms) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    TRY(launch_gemv(h, M_ALL, h->Y, 3, false));
    CK(cudaEventRecord(h->ev0, h->stream));
    for (int i = 0; i < reps; i++) TRY(launch_gemv(h, M_ALL, h->Y, 3, false));
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    *ms = (double)t / reps;
    return DFN_OK;
}

}  // extern "C"
