// dfn_b200.cu — C ABI (include/dfn_b200.h) over the sm_100a kernels of
// dfn_device.cuh. Host code here only sequences launches on the handle's
// stream and moves caller buffers; every arithmetic step of the hot path runs
// on the GPU. There is no CPU fallback: without a usable CUDA device,
// dfn_create fails with DFN_ERR_CUDA.
#include "../../include/dfn_b200.h"
#include "dfn_device.cuh"

#include <cstdio>
#include <cstring>
#include <mutex>
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

int bytes_per_col(int mode, int store)
{
    if (mode == DFN_MODE_II) return store == DFN_STORE_FP64 ? 16 : 8;
    return store == DFN_STORE_FP64 ? 8 : 4;
}

}  // namespace

struct dfn_handle {
    int dev = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int64_t N = 0, F = 0, Np = 0;
    int mode = 2, store = 0, pressure = 0, gemv_impl = 0, max_attempts = 64;
    int nchunk = 0;
    double tol = 0, prefT = 0, mu_2cs = 0;
    int64_t nsrc = 0, nseg = 0;
    // geometry and parameters
    double *node = nullptr, *elem = nullptr, *ds = nullptr, *tan = nullptr, *nrm = nullptr, *permx = nullptr;
    double *a = nullptr, *b = nullptr, *Dc = nullptr, *f0 = nullptr, *V0 = nullptr, *nload = nullptr,
           *sload = nullptr, *perm = nullptr;
    unsigned char *fake = nullptr;
    int64_t *src_fault = nullptr, *src_elem = nullptr, *seg_start = nullptr;
    double *src_Q = nullptr, *src_tb = nullptr, *src_te = nullptr;
    std::vector<double> h_src_tb;
    // state and work
    double *Y = nullptr, *P = nullptr, *Pdot = nullptr, *yout = nullptr, *yscal = nullptr, *ytmp = nullptr;
    double *kbuf = nullptr, *SigT = nullptr, *SigN = nullptr, *partT = nullptr, *partN = nullptr;
    double *Ptemp = nullptr, *Pdot_s = nullptr, *pwork = nullptr, *vin = nullptr, *vout = nullptr, *snap = nullptr;
    int *err_flag = nullptr;
    void *K = nullptr;
    size_t K_bytes = 0;
    StepCtl *ctl = nullptr;
    StepCtl *h_ctl = nullptr;  // pinned mirror
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;
    PressParams pp{};
    // K.V launch timing
    bool prof = false;
    std::vector<cudaEvent_t> pev;
    int pcount = 0;
};

static const int kProfMax = 16384;

// ---------------------------------------------------------------------------
// launch helpers

typedef void (*gemv_fn)(int64_t, int64_t, const uint4 *, const double *, double *, double *);
typedef void (*gemv_tma_fn)(int64_t, int64_t, const uint4 *, const double *, double *, double *, int *);

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

static int launch_gemv(dfn_handle *h, const double *Vin)
{
    const bool rec = h->prof && h->pcount < kProfMax;
    if (rec) CK(cudaEventRecord(h->pev[2 * h->pcount], h->stream));
    dim3 grid((unsigned)h->nchunk, (unsigned)((h->N + GEMV_ROWS - 1) / GEMV_ROWS));
    if (h->gemv_impl == 0) {
        gemv_tma_fn fn = pick_gemv_tma(h->mode, h->store);
        fn<<<grid, (TMA_CONSUMERS + 1) * 32, kTmaSmem, h->stream>>>(h->N, h->Np, (const uint4 *)h->K, Vin, h->partT,
                                                                     h->partN, h->err_flag);
    } else {
        gemv_fn fn = pick_gemv(h->mode, h->store);
        fn<<<grid, GEMV_WARPS * 32, 0, h->stream>>>(h->N, h->Np, (const uint4 *)h->K, Vin, h->partT, h->partN);
    }
    h->launches++;
    CKL();
    if (rec) {
        CK(cudaEventRecord(h->pev[2 * h->pcount + 1], h->stream));
        h->pcount++;
    }
    return DFN_OK;
}

static int launch_pressure(dfn_handle *h, int kind, int sys0, int nsys, double dt_explicit)
{
    if (h->pressure == DFN_PRESSURE_CG) {
        pressure_cg_kernel<<<nsys, 1024, 0, h->stream>>>(h->pp, h->ctl, kind, sys0, dt_explicit, h->Ptemp, h->Pdot_s,
                                                         h->pwork);
    } else {
        dim3 grid((unsigned)((h->nseg + 127) / 128), (unsigned)nsys);
        pressure_tridiag_kernel<<<grid, 128, 0, h->stream>>>(h->pp, h->ctl, kind, sys0, dt_explicit, h->seg_start,
                                                             h->nseg, h->Ptemp, h->Pdot_s, h->pwork);
    }
    h->launches++;
    CKL();
    return DFN_OK;
}

static FricParams fric_params(dfn_handle *h, int sys, double *yin_tmp)
{
    FricParams f;
    f.N = h->N; f.mode = h->mode; f.nchunk = h->nchunk; f.prefT = h->prefT; f.mu_2cs = h->mu_2cs;
    f.a = h->a; f.b = h->b; f.Dc = h->Dc; f.f0 = h->f0; f.V0 = h->V0; f.nload = h->nload; f.sload = h->sload;
    f.fake = h->fake; f.partT = h->partT; f.partN = h->partN; f.SigT = h->SigT; f.SigN = h->SigN;
    f.Ptemp = h->Ptemp + (int64_t)sys * h->N; f.Pdot = h->Pdot_s + (int64_t)sys * h->N;
    f.y = h->Y; f.ytmp = yin_tmp; f.kbuf = h->kbuf; f.yscal = h->yscal; f.yout = h->yout; f.ctl = h->ctl;
    return f;
}

static int launch_friction(dfn_handle *h, int stage, int sys, double *ytmp)
{
    FricParams f = fric_params(h, sys, ytmp);
    unsigned nb = (unsigned)((h->N + 255) / 256);
    friction_kernel<<<nb, 256, 0, h->stream>>>(f, stage);
    h->launches++;
    CKL();
    return DFN_OK;
}

#define TRY(x)                       \
    do {                             \
        int s_ = (x);                \
        if (s_ != DFN_OK) return s_; \
    } while (0)

// One RK attempt (stages 2..6 and the error test) with the current ctl->h.
static int run_attempt(dfn_handle *h)
{
    const int64_t n3 = 3 * h->N;
    attempt_begin_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, h->stream>>>(h->N, h->Y, h->kbuf, h->ytmp, h->ctl);
    h->launches++;
    CKL();
    TRY(launch_pressure(h, 1, 1, 5, 0.0));
    for (int s = 2; s <= 6; s++) {
        TRY(launch_gemv(h, h->ytmp));
        TRY(launch_friction(h, s, s - 1, h->ytmp));
    }
    decide_kernel<<<1, 32, 0, h->stream>>>(h->ctl);
    h->launches++;
    CKL();
    return DFN_OK;
}

static int sync_ctl(dfn_handle *h)
{
    CK(cudaMemcpyAsync(h->h_ctl, h->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int flag = 0;
    CK(cudaMemcpy(&flag, h->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        g_err = "bounded wait expired in the TMA K.V pipeline";
        return DFN_ERR_CUDA;
    }
    return DFN_OK;
}

// Attempt loop of rkqs (src/ode_solver/ode_bs.f90:155-165) with k1 and
// yscal already on the device and ctl->h set.
static int rkqs_device(dfn_handle *h)
{
    for (int att = 0;; att++) {
        TRY(run_attempt(h));
        TRY(sync_ctl(h));
        if (h->h_ctl->status) return h->h_ctl->status;
        if (h->h_ctl->accepted) return DFN_OK;
        if (att + 1 >= h->max_attempts) return DFN_ERR_ATTEMPTS;
    }
}

static int solve_one_step(dfn_handle *h)
{
    step_begin_kernel<<<1, 32, 0, h->stream>>>(h->ctl, h->nsrc, h->src_tb);
    h->launches++;
    CKL();
    // CG probe at t_try (halving on non-convergence); its solution is the
    // pressure of the scaling RHS evaluated at dt = t_try (src/solver.f90:81-101).
    TRY(launch_pressure(h, 0, 0, 1, 0.0));
    TRY(launch_gemv(h, h->Y));
    TRY(launch_friction(h, 1, 0, h->ytmp));
    set_h_kernel<<<1, 32, 0, h->stream>>>(h->ctl);
    h->launches++;
    CKL();
    TRY(rkqs_device(h));
    commit_kernel<<<(unsigned)((3 * h->N + 255) / 256), 256, 0, h->stream>>>(
        h->N, h->Y, h->yout, h->P, h->Pdot, h->Ptemp + 4 * h->N, h->Pdot_s + 4 * h->N, h->ctl, 86400.0);
    h->launches++;
    CKL();
    return DFN_OK;
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
    void *ptrs[] = {h->node, h->elem, h->ds, h->tan, h->nrm, h->permx, h->a, h->b, h->Dc, h->f0, h->V0,
                    h->nload, h->sload, h->perm, h->fake, h->src_fault, h->src_elem, h->seg_start, h->src_Q,
                    h->src_tb, h->src_te, h->Y, h->P, h->Pdot, h->yout, h->yscal, h->ytmp, h->kbuf, h->SigT,
                    h->SigN, h->partT, h->partN, h->Ptemp, h->Pdot_s, h->pwork, h->vin, h->vout, h->snap,
                    h->err_flag, h->K, h->ctl};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (h->h_ctl) cudaFreeHost(h->h_ctl);
    for (cudaEvent_t e : h->pev) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return DFN_OK;
}

#define DALLOC(ptr, count)                                                \
    do {                                                                  \
        cudaError_t e_ = cudaMalloc((void **)&(ptr), sizeof(*(ptr)) * (size_t)(count)); \
        if (e_ != cudaSuccess) {                                          \
            set_err("cudaMalloc " #ptr, e_, __FILE__, __LINE__);          \
            dfn_destroy(h);                                               \
            return e_ == cudaErrorMemoryAllocation ? DFN_ERR_NOMEM : DFN_ERR_CUDA; \
        }                                                                 \
    } while (0)

#define HCOPY(dst, src, count)                                                                          \
    do {                                                                                                \
        cudaError_t e_ = cudaMemcpy((dst), (src), sizeof(*(dst)) * (size_t)(count), cudaMemcpyHostToDevice); \
        if (e_ != cudaSuccess) {                                                                        \
            set_err("cudaMemcpy " #dst, e_, __FILE__, __LINE__);                                        \
            dfn_destroy(h);                                                                             \
            return DFN_ERR_CUDA;                                                                        \
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

int32_t dfn_create(const dfn_problem *p, const dfn_options *opt_in, dfn_handle **out)
{
    if (!p || !out) { g_err = "null argument"; return DFN_ERR_ARG; }
    *out = nullptr;
    dfn_options opt;
    if (opt_in) opt = *opt_in; else dfn_default_options(&opt);
    const int64_t N = p->nb_element, F = p->nb_fault;
    if (N < 2 || F < 1 || !p->fault_nb_element || !p->node) { g_err = "need nb_element >= 2 and nb_fault >= 1"; return DFN_ERR_ARG; }
    int64_t cnt = 0;
    for (int64_t f = 0; f < F; f++) {
        if (p->fault_nb_element[f] < 1) { g_err = "every fault needs at least one element"; return DFN_ERR_ARG; }
        cnt += p->fault_nb_element[f] + 1;
    }
    if (cnt - 1 != N) { g_err = "nb_element must equal sum(fault_nb_element) + nb_fault - 1"; return DFN_ERR_ARG; }
    if (p->fracture_mode != DFN_MODE_II && p->fracture_mode != DFN_MODE_III) { g_err = "fracture_mode must be 2 or 3"; return DFN_ERR_ARG; }
    if (opt.kernel_storage < 0 || opt.kernel_storage > 2) { g_err = "bad kernel_storage"; return DFN_ERR_ARG; }
    if (opt.pressure_solver < 0 || opt.pressure_solver > 1) { g_err = "bad pressure_solver"; return DFN_ERR_ARG; }
    if (p->tol_solver <= 0) { g_err = "tol_solver must be positive"; return DFN_ERR_ARG; }
    for (int64_t s = 0; s < p->nb_source; s++) {
        int64_t f = p->src_fault[s];
        if (f < 1 || f > F || p->src_index[s] < 1 || p->src_index[s] > p->fault_nb_element[f - 1]) {
            g_err = "source fault/index out of range";
            return DFN_ERR_ARG;
        }
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
    h->N = N; h->F = F; h->mode = p->fracture_mode; h->store = opt.kernel_storage;
    h->pressure = opt.pressure_solver; h->gemv_impl = opt.gemv_impl;
    h->max_attempts = opt.max_attempts > 0 ? opt.max_attempts : 64;
    h->tol = p->tol_solver;
    const int bpc = bytes_per_col(h->mode, h->store);
    const int64_t CW = GEMV_CHUNK_BYTES / bpc;
    h->Np = ((N + CW - 1) / CW) * CW;
    h->nchunk = (int)(h->Np / CW);
    // prefactors: src/kernel_calculation/hmatrixModeII.f90:67-68, hmatrixModeIII.f90:55
    if (h->mode == DFN_MODE_II) h->prefT = p->mu / DFN_PI * (1.0 - p->cs * p->cs / (p->cp * p->cp));
    else h->prefT = p->mu / (2.0 * DFN_PI);
    h->mu_2cs = p->mu / (2.0 * p->cs);

    DALLOC(h->node, 2 * (N + 1)); DALLOC(h->elem, 2 * N); DALLOC(h->ds, N); DALLOC(h->tan, 2 * N);
    DALLOC(h->nrm, 2 * N); DALLOC(h->permx, N + 1);
    DALLOC(h->a, N); DALLOC(h->b, N); DALLOC(h->Dc, N); DALLOC(h->f0, N); DALLOC(h->V0, N);
    DALLOC(h->nload, N); DALLOC(h->sload, N); DALLOC(h->perm, N); DALLOC(h->fake, N);
    DALLOC(h->Y, 3 * N); DALLOC(h->P, N); DALLOC(h->Pdot, N); DALLOC(h->yout, 3 * N); DALLOC(h->yscal, 3 * N);
    DALLOC(h->ytmp, 3 * N); DALLOC(h->kbuf, 18 * N); DALLOC(h->SigT, N); DALLOC(h->SigN, N);
    DALLOC(h->partT, (int64_t)h->nchunk * N); DALLOC(h->partN, (int64_t)h->nchunk * N);
    DALLOC(h->Ptemp, 6 * N); DALLOC(h->Pdot_s, 6 * N); DALLOC(h->pwork, 24 * N);
    DALLOC(h->vin, 3 * N); DALLOC(h->vout, 3 * N); DALLOC(h->snap, 5 * N);
    DALLOC(h->err_flag, 1); DALLOC(h->ctl, 1);
    CKC(cudaMemset(h->err_flag, 0, sizeof(int)));
    CKC(cudaMemset(h->partN, 0, sizeof(double) * h->nchunk * N));
    CKC(cudaMemset(h->Pdot, 0, sizeof(double) * N));
    CKC(cudaMemset(h->SigT, 0, sizeof(double) * N));
    CKC(cudaMemset(h->SigN, 0, sizeof(double) * N));
    CKC(cudaMallocHost((void **)&h->h_ctl, sizeof(StepCtl)));

    HCOPY(h->node, p->node, 2 * (N + 1));
    HCOPY(h->a, p->a, N); HCOPY(h->b, p->b, N); HCOPY(h->Dc, p->Dc, N); HCOPY(h->f0, p->f0, N);
    HCOPY(h->V0, p->V0, N); HCOPY(h->nload, p->normal_loading_dot, N); HCOPY(h->sload, p->shear_loading_dot, N);
    HCOPY(h->perm, p->permeability, N);
    HCOPY(h->Y, p->V, N); HCOPY(h->Y + N, p->theta, N); HCOPY(h->Y + 2 * N, p->sigmaN, N); HCOPY(h->P, p->P, N);

    // fake elements (src/friction/RateStateAgingModeII.f90:81-89) and
    // 0-based fault starts (src/configuration.f90:245-246)
    std::vector<unsigned char> fake(N, 0);
    std::vector<int64_t> first(F);
    {
        int64_t idx = 0, c2 = 0;
        for (int64_t f = 0; f < F; f++) {
            first[f] = c2;
            c2 += p->fault_nb_element[f] + 1;
            idx += p->fault_nb_element[f] + 1;
            if (idx <= N) fake[idx - 1] = 1;
        }
    }
    HCOPY(h->fake, fake.data(), N);

    h->nsrc = p->nb_source;
    int64_t ns = h->nsrc > 0 ? h->nsrc : 1;
    DALLOC(h->src_fault, ns); DALLOC(h->src_elem, ns); DALLOC(h->src_Q, ns); DALLOC(h->src_tb, ns); DALLOC(h->src_te, ns);
    if (h->nsrc > 0) {
        std::vector<int64_t> se(h->nsrc);
        for (int64_t s = 0; s < h->nsrc; s++) se[s] = first[p->src_fault[s] - 1] + p->src_index[s] - 1;
        HCOPY(h->src_fault, p->src_fault, h->nsrc); HCOPY(h->src_elem, se.data(), h->nsrc);
        HCOPY(h->src_Q, p->src_Q, h->nsrc); HCOPY(h->src_tb, p->src_t_beg, h->nsrc); HCOPY(h->src_te, p->src_t_end, h->nsrc);
        h->h_src_tb.assign(p->src_t_beg, p->src_t_beg + h->nsrc);
    }

    // geometry (device)
    geometry_kernel<<<(unsigned)((N + 1 + 255) / 256), 256, 0, h->stream>>>(
        N, h->mode, h->node, h->elem, h->ds, h->tan, h->nrm, h->nload, h->sload, h->Y + 2 * N, h->perm, h->permx,
        p->Sigma11_dot, p->Sigma12_dot, p->Sigma22_dot, p->Sigma31_dot, p->Sigma32_dot);
    h->launches++;
    CKC(cudaGetLastError());

    // decoupled pressure segments from the face permeabilities
    {
        std::vector<double> px(N + 1);
        CKC(cudaMemcpyAsync(px.data(), h->permx, sizeof(double) * (N + 1), cudaMemcpyDeviceToHost, h->stream));
        CKC(cudaStreamSynchronize(h->stream));
        std::vector<int64_t> seg;
        seg.push_back(0);
        for (int64_t k = 1; k < N; k++)
            if (px[k] == 0.0) seg.push_back(k);
        seg.push_back(N);
        h->nseg = (int64_t)seg.size() - 1;
        DALLOC(h->seg_start, seg.size());
        HCOPY(h->seg_start, seg.data(), seg.size());
    }

    // dense kernel matrix
    h->K_bytes = (size_t)N * (size_t)h->Np * (size_t)bpc;
    {
        cudaError_t e = cudaMalloc(&h->K, h->K_bytes);
        if (e != cudaSuccess) {
            set_err("cudaMalloc K", e, __FILE__, __LINE__);
            dfn_destroy(h);
            return DFN_ERR_NOMEM;
        }
    }
    {
        dim3 grid((unsigned)N, (unsigned)((h->Np + 255) / 256));
#define ASM(MODE, STORE) assemble_kernel<MODE, STORE><<<grid, 256, 0, h->stream>>>(N, h->Np, h->node, h->elem, h->tan, h->nrm, h->K)
        if (h->mode == 2) {
            if (h->store == 0) ASM(2, 0); else if (h->store == 1) ASM(2, 1); else ASM(2, 2);
        } else {
            if (h->store == 0) ASM(3, 0); else if (h->store == 1) ASM(3, 1); else ASM(3, 2);
        }
#undef ASM
        h->launches++;
        CKC(cudaGetLastError());
    }
    // TMA pipeline needs the dynamic shared memory opt-in
    {
        gemv_tma_fn fns[6] = {gemv_tma_kernel<2, 0>, gemv_tma_kernel<2, 1>, gemv_tma_kernel<2, 2>,
                              gemv_tma_kernel<3, 0>, gemv_tma_kernel<3, 1>, gemv_tma_kernel<3, 2>};
        for (auto fn : fns) CKC(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaSmem));
    }

    // pressure parameters
    PressParams &pp = h->pp;
    pp.N = N; pp.P = h->P; pp.permx = h->permx; pp.ds = h->ds;
    pp.porosity = p->porosity; pp.dyn_visc = p->dyn_viscosity; pp.comp = p->fluid_comp + p->rock_comp;
    pp.tol = p->tol_solver; pp.nsrc = h->nsrc; pp.src_fault = h->src_fault; pp.src_elem = h->src_elem;
    pp.src_Q = h->src_Q; pp.src_tb = h->src_tb; pp.src_te = h->src_te; pp.ctl_time = &h->ctl->time;

    // controller: solve() entry, src/solver.f90:50-56
    StepCtl c;
    memset(&c, 0, sizeof(c));
    c.time = p->time0; c.t_try = 100.0; c.eps = p->tol_solver; c.h = 100.0;
    CKC(cudaMemcpy(h->ctl, &c, sizeof(c), cudaMemcpyHostToDevice));
    CKC(cudaEventCreate(&h->ev0));
    CKC(cudaEventCreate(&h->ev1));
    CKC(cudaStreamSynchronize(h->stream));
    *out = h;
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

int64_t dfn_nb_element(const dfn_handle *h) { return h ? h->N : -1; }
int64_t dfn_kernel_bytes(const dfn_handle *h)
{
    if (!h) return -1;
    return (int64_t)h->N * (int64_t)h->N * bytes_per_col(h->mode, h->store);
}
int64_t dfn_launch_count(const dfn_handle *h) { return h ? h->launches : -1; }

int32_t dfn_kernel_device(dfn_handle *h, const double *d_slip, double *d_sT, double *d_sN)
{
    if (!h || !d_slip || !d_sT) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    TRY(launch_gemv(h, d_slip));
    kv_finish_kernel<<<(unsigned)((h->N + 255) / 256), 256, 0, h->stream>>>(h->N, h->mode, h->nchunk, h->prefT,
                                                                             h->partT, h->partN, d_sT, d_sN);
    h->launches++;
    CKL();
    return DFN_OK;
}

int32_t dfn_kernel(dfn_handle *h, const double *slip, double *sT, double *sN)
{
    if (!h || !slip || !sT) return DFN_ERR_ARG;
    const int64_t N = h->N;
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(h->vin, slip, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
    TRY(dfn_kernel_device(h, h->vin, h->vout, h->vout + N));
    CK(cudaMemcpyAsync(sT, h->vout, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    if (sN) CK(cudaMemcpyAsync(sN, h->vout + N, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int flag = 0;
    CK(cudaMemcpy(&flag, h->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) { g_err = "bounded wait expired in the TMA K.V pipeline"; return DFN_ERR_CUDA; }
    return DFN_OK;
}

static int reset_status(dfn_handle *h)
{
    CK(cudaMemsetAsync(&h->ctl->status, 0, sizeof(int), h->stream));
    return DFN_OK;
}

int32_t dfn_compute_P(dfn_handle *h, double dt, double *P_temp, double *P_dot, int32_t *ier)
{
    if (!h || !P_temp || !P_dot) return DFN_ERR_ARG;
    const int64_t N = h->N;
    CK(cudaSetDevice(h->dev));
    TRY(reset_status(h));
    TRY(launch_pressure(h, 2, 0, 1, dt));
    TRY(sync_ctl(h));
    int st = h->h_ctl->status;
    if (ier) *ier = (st == 1) ? 1 : 0;
    if (st == 1) { TRY(reset_status(h)); return DFN_OK; }
    if (st) return st;
    CK(cudaMemcpy(P_temp, h->Ptemp, sizeof(double) * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(P_dot, h->Pdot_s, sizeof(double) * N, cudaMemcpyDeviceToHost));
    return DFN_OK;
}

int32_t dfn_friction_law(dfn_handle *h, double x, int64_t nv, const double *Y, double *Ydot)
{
    if (!h || !Y || !Ydot || nv != 3 * h->N) return DFN_ERR_ARG;
    const int64_t N = h->N;
    CK(cudaSetDevice(h->dev));
    TRY(reset_status(h));
    CK(cudaMemcpyAsync(h->ytmp, Y, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, h->stream));
    TRY(launch_pressure(h, 2, 0, 1, x));
    TRY(launch_gemv(h, h->ytmp));
    TRY(launch_friction(h, 0, 0, h->ytmp));
    CK(cudaMemcpyAsync(Ydot, h->kbuf, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    int st = h->h_ctl->status;
    TRY(reset_status(h));
    return st;
}

int32_t dfn_rkqs(dfn_handle *h, double *y, const double *dydx, int64_t nv, double *x, double htry, double eps,
                 const double *yscal, double *hdid, double *hnext)
{
    if (!h || !y || !dydx || !x || !yscal || !hdid || !hnext || nv != 3 * h->N) return DFN_ERR_ARG;
    const int64_t n3 = 3 * h->N;
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(h->Y, y, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->kbuf, dydx, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->yscal, yscal, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
    TRY(sync_ctl(h));
    StepCtl c = *h->h_ctl;
    double eps_saved = c.eps;
    c.x = *x; c.h = htry; c.eps = eps; c.accepted = 0; c.status = 0;
    CK(cudaMemcpyAsync(h->ctl, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
    int st = rkqs_device(h);
    if (st != DFN_OK) return st;
    CK(cudaMemcpyAsync(h->Y, h->yout, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(y, h->yout, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    *hdid = h->h_ctl->hdid;
    *hnext = h->h_ctl->hnext;
    *x = *x + *hdid;
    c = *h->h_ctl;
    c.eps = eps_saved; c.x = 0.0;
    CK(cudaMemcpy(h->ctl, &c, sizeof(c), cudaMemcpyHostToDevice));
    return DFN_OK;
}

static void fill_report(dfn_handle *h, dfn_report *r)
{
    if (!r) return;
    const StepCtl &c = *h->h_ctl;
    r->it_count = c.it_count; r->attempts = c.attempts; r->rejected = c.rejected; r->rhs_evals = c.rhs_evals;
    r->cg_iterations = c.cg_iters; r->probe_halvings = c.halvings; r->time = c.time; r->t_try = c.t_try;
    r->last_hdid = c.hdid; r->status = c.status; r->pad = 0;
}

int32_t dfn_solve_steps(dfn_handle *h, int64_t n_steps, dfn_report *rep)
{
    if (!h || n_steps < 0) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    int st = DFN_OK;
    for (int64_t s = 0; s < n_steps; s++) {
        st = solve_one_step(h);
        if (st != DFN_OK) break;
    }
    int st2 = sync_ctl(h);
    if (st == DFN_OK) st = st2;
    if (st == DFN_OK && h->h_ctl->status) st = h->h_ctl->status;
    fill_report(h, rep);
    return st;
}

int32_t dfn_get_state(dfn_handle *h, double *Y, double *P, double *time, double *t_try, int64_t *it_count)
{
    if (!h) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    TRY(sync_ctl(h));
    if (Y) CK(cudaMemcpy(Y, h->Y, sizeof(double) * 3 * h->N, cudaMemcpyDeviceToHost));
    if (P) CK(cudaMemcpy(P, h->P, sizeof(double) * h->N, cudaMemcpyDeviceToHost));
    if (time) *time = h->h_ctl->time;
    if (t_try) *t_try = h->h_ctl->t_try;
    if (it_count) *it_count = h->h_ctl->it_count;
    return DFN_OK;
}

int32_t dfn_set_state(dfn_handle *h, const double *Y, const double *P, double time, double t_try, int64_t it_count)
{
    if (!h) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    if (Y) CK(cudaMemcpyAsync(h->Y, Y, sizeof(double) * 3 * h->N, cudaMemcpyHostToDevice, h->stream));
    if (P) CK(cudaMemcpyAsync(h->P, P, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->stream));
    TRY(sync_ctl(h));
    StepCtl c = *h->h_ctl;
    c.time = time; c.t_try = t_try; c.it_count = it_count; c.status = 0;
    CK(cudaMemcpyAsync(h->ctl, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DFN_OK;
}

int32_t dfn_get_snapshot(dfn_handle *h, double *V, double *theta, double *P, double *tT, double *tN,
                         double *permeability, double *time)
{
    if (!h) return DFN_ERR_ARG;
    const int64_t N = h->N;
    CK(cudaSetDevice(h->dev));
    snapshot_kernel<<<(unsigned)((N + 255) / 256), 256, 0, h->stream>>>(N, h->Y, h->Dc, h->V0, h->P, h->SigT, h->snap);
    h->launches++;
    CKL();
    double *dst[5] = {V, theta, P, tT, tN};
    for (int i = 0; i < 5; i++)
        if (dst[i]) CK(cudaMemcpyAsync(dst[i], h->snap + i * N, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    if (permeability) CK(cudaMemcpyAsync(permeability, h->perm, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync_ctl(h));
    if (time) *time = h->h_ctl->time;
    return DFN_OK;
}

int32_t dfn_step_host(dfn_handle *h, const double *Y_in, const double *P_in, double time_in, double t_try_in,
                      double *V_out, double *theta_out, double *P_out, double *tT_out, double *tN_out,
                      dfn_report *rep)
{
    if (!h || !Y_in || !P_in) return DFN_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    TRY(sync_ctl(h));
    StepCtl c = *h->h_ctl;
    CK(cudaMemcpyAsync(h->Y, Y_in, sizeof(double) * 3 * h->N, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->P, P_in, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->stream));
    c.time = time_in; c.t_try = t_try_in; c.status = 0;
    *h->h_ctl = c;
    CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(c), cudaMemcpyHostToDevice, h->stream));
    int st = solve_one_step(h);
    if (st != DFN_OK) { sync_ctl(h); fill_report(h, rep); return st; }
    TRY(dfn_get_snapshot(h, V_out, theta_out, P_out, tT_out, tN_out, nullptr, nullptr));
    fill_report(h, rep);
    return h->h_ctl->status;
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

static const int kNoAllocMaxDevices = 128;
static double *g_noalloc_addr[kNoAllocMaxDevices];  // device address per device ordinal, set once
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device, looked up
// once per device with that device current.
static int noalloc_scratch(double **out)
{
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        g_err = "device ordinal out of range for the allocation-free scratch table";
        return DFN_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_err("cudaGetSymbolAddress(g_noalloc_scratch)", e, __FILE__, __LINE__);
            return DFN_ERR_CUDA;
        }
        g_noalloc_addr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_addr[dev];
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
    *ier = (c.status == 1) ? 1 : 0;
    if (c.status != 0 && c.status != 1) return c.status;
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
    TRY(launch_gemv(h, h->Y));
    CK(cudaEventRecord(h->ev0, h->stream));
    for (int i = 0; i < reps; i++) TRY(launch_gemv(h, h->Y));
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    *ms = (double)t / reps;
    return DFN_OK;
}

}  // extern "C"
