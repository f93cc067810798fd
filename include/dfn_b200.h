/*
 * dfn_b200.h — C ABI of the B200 earthquake-cycle hot path.
 *
 * The hot path is one right-hand-side evaluation of the rate-and-state
 * earthquake-cycle ODE and the adaptive Cash-Karp RK45 driver around it:
 *   - elastostatic stress-rate transfer K.V (shear and, in mode II, normal),
 *   - rate-and-state friction with radiation damping (closed-form dV/dt),
 *   - implicit pore-pressure diffusion along the concatenated fault chain.
 *
 * Every entry point takes plain pointers and sizes. Host buffers belong to
 * the caller; device memory is owned by the handle. A handle is bound to one
 * CUDA device and one stream and must not be shared between host threads.
 * All functions return a dfn_status code; nothing here falls back to the CPU.
 *
 * State layout (identical to the reference's Y vector,
 * src/configuration.f90:185-187,235-237):
 *   Y[0:N)    slip rate V            (m/s)
 *   Y[N:2N)   log-state psi = ln(theta*V0/Dc)
 *   Y[2N:3N)  normal traction sigmaN (Pa, compression negative)
 * N counts one "fake" element between consecutive faults
 * (src/configuration.f90:126,136); its derivatives are held at zero.
 */
#ifndef DFN_B200_H
#define DFN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFN_ABI_VERSION 1

/* Status codes. DFN_ERR_NOCONV plays the role of the reference's ier=1. */
typedef enum dfn_status {
    DFN_OK = 0,
    DFN_ERR_NOCONV = 1,      /* pressure CG hit its 200-iteration cap (src/fluid_diffusion.f90:120-125) */
    DFN_ERR_UNDERFLOW = 2,   /* "stepsize underflow in rkqs" (src/ode_solver/ode_bs.f90:164) */
    DFN_ERR_EXTENSIONAL = 3, /* sigmaN > 0 after a step (src/solver.f90:412-418) */
    DFN_ERR_NONFINITE = 4,   /* NaN/Inf in the state or in a pressure solve */
    DFN_ERR_ARG = 5,         /* invalid argument or size */
    DFN_ERR_CUDA = 6,        /* a CUDA runtime call failed */
    DFN_ERR_UNSUPPORTED = 7, /* feature not available in this library */
    DFN_ERR_ATTEMPTS = 8,    /* more rejected RK attempts in one step than the device budget */
    DFN_ERR_NOMEM = 9,       /* device allocation failed */
    DFN_ERR_TIMEOUT = 10     /* a bounded wait inside a kernel expired (the kernel stopped early) */
} dfn_status;

enum { DFN_MODE_II = 2, DFN_MODE_III = 3 };                    /* hyperparameter/fracture_mode */
enum { DFN_KERNEL_DIRECT = 0, DFN_KERNEL_HMATRIX = 1 };        /* hyperparameter/static_kernel */
/* Stored K entries. DFN_STORE_BF16X2_TC: for a batch whose networks share
 * one geometry (same nb_element, nodes, fracture mode and elastic constants;
 * up to 256 networks), K is stored once as BF16 hi + lo matrices and the
 * K.V of all networks of a stage is one tcgen05 tensor-core GEMM (BF16
 * products, FP32 accumulation). DFN_STORE_FP64_SHARED: the same shared K
 * in FP64 and an FP64 GEMM on the CUDA cores (K streamed once per stage for
 * all networks, products and sums in FP64), the counterpart that isolates
 * the tensor-core arithmetic from the sharing. No counterpart in the
 * reference. */
enum { DFN_STORE_FP64 = 0, DFN_STORE_FP32 = 1, DFN_STORE_BF16X2 = 2, DFN_STORE_BF16X2_TC = 3,
       DFN_STORE_FP64_SHARED = 4 };
/* Pressure solver: DFN_PRESSURE_CG is the reference's CG with tree-reduced
 * dot products (systems of 2048 elements or more, when a launch has few of
 * them, are solved by a cluster of 2 to 16 CTAs holding the vectors in shared
 * memory: a tree of another shape, so such a network's results can differ
 * in rounding between a batch and a handle of its own; networks with fault
 * crossings always use one CTA per system); DFN_PRESSURE_CG_EXACT sums them sequentially as the reference
 * does, reproducing its rounding and iteration counts bit for bit (slower
 * for large N); DFN_PRESSURE_TRIDIAG solves the same implicit step exactly
 * (networks without fault crossings: dfn_create rejects the others).
 * Fault crossings (node pairs of two faults closer than 0.01 times the
 * smaller of their smallest element lengths, as find_fault_crossing,
 * src/initialisation.f90:279-344) couple the pressure of the elements around
 * the crossing node (src/fluid_diffusion.f90:213-295, 338-405), with every
 * coefficient using its own row's element length and every term divided by
 * the diagonal (the reference uses ds(1) and a stale ds(k-1), and divides
 * one row by the element index). */
enum { DFN_PRESSURE_CG = 0, DFN_PRESSURE_TRIDIAG = 1, DFN_PRESSURE_CG_EXACT = 2 };

/*
 * Problem description: the reference's in-memory state after read_config
 * (src/configuration.f90:70-379), fake elements included. Per-element arrays
 * have N entries; the node array has N+1 nodes stored x,y,x,y,... (the
 * Fortran node(2,nb_node) array). Fake elements carry the reader's presets
 * (a=b=Dc=f0=V0=1) and zeros elsewhere.
 */
typedef struct dfn_problem {
    int64_t nb_element;              /* N (fake elements included) */
    int64_t nb_fault;                /* F */
    const int64_t *fault_nb_element; /* [F] elements of each fault */
    int32_t fracture_mode;           /* DFN_MODE_II or DFN_MODE_III */
    int32_t static_kernel;           /* DFN_KERNEL_* */
    const double *node;              /* [2*(N+1)] */
    const double *a, *b, *Dc, *f0, *V0;        /* [N] friction parameters */
    const double *V, *theta, *sigmaN, *P;      /* [N] initial state, theta is psi */
    const double *normal_loading_dot;          /* [N] */
    const double *shear_loading_dot;           /* [N] */
    const double *permeability;                /* [N] */
    double mu, cp, cs;
    double Sigma11_dot, Sigma12_dot, Sigma22_dot, Sigma31_dot, Sigma32_dot;
    double rock_comp, fluid_comp, fluid_density, porosity, dyn_viscosity;
    int64_t nb_source;               /* total sources over all faults */
    const int64_t *src_fault;        /* [nb_source] 1-based fault id, grouped by fault */
    const int64_t *src_index;        /* [nb_source] 1-based element index within the fault */
    const double *src_Q;             /* [nb_source] m/s */
    const double *src_t_beg, *src_t_end;       /* [nb_source] s */
    double tol_solver;
    double time0;
    int64_t max_it, stride_time, freq_writing_file;
    /* Permeability evolution (hyperparameter/permeability_coupling = 1,
     * src/fluid_diffusion.f90:68-70): before every pressure solve,
     *   permeability = (k* - kmin) exp(-|sigmaN + P| / |Snk|) + kmin
     * from the committed sigmaN and P, with k* = kmin + (k - kmin)
     * exp(|sigmaN + P| / |Snk|) fixed from the initial state
     * (src/initialisation.f90:256-261), and the face permeabilities follow.
     * V formulation, networks without fault crossings. kmin and Snk may be
     * NULL when the coupling is 0. */
    int64_t permeability_coupling;
    const double *kmin, *Snk;                  /* [N] */
} dfn_problem;

/* Options of this implementation (no counterpart in the reference). */
typedef struct dfn_options {
    int32_t kernel_storage;   /* DFN_STORE_*; FP64 is the plain path */
    int32_t pressure_solver;  /* DFN_PRESSURE_* */
    int32_t device;           /* CUDA device ordinal */
    int32_t max_attempts;     /* RK attempts per step scheduled on the device before the host looks (>=1) */
    int32_t gemv_impl;        /* 0 = TMA bulk-copy pipeline, 1 = direct 128-bit loads;
                                 tensor-core storage: 0 persistent GEMM, 1 / 2 one unit
                                 per CTA with the deepest / a 2-stage ring */
    /* H-matrix parameters for static_kernel = hmatrix (0 = the reference's
     * defaults nleaf=100, eta=3, eps_ACA=1e-8, src/variables.f90:122-124).
     * Admissible blocks get a partial-pivot ACA of at most 128 terms to
     * eps_ACA (recompressed when at most 64); a block whose ACA does not
     * converge within 128 terms, or whose factors would not be smaller than
     * the block, is stored dense (the reference truncates at rank 20,
     * src/hmatrix/H_matrix_construction.f90:59). */
    int32_t hmat_leaf;
    /* DFN_FORM_V integrates V as the reference does; DFN_FORM_NEWTON
     * integrates slip and psi and solves the friction law for V by Newton
     * at every stage (no counterpart in the reference, see below). */
    int32_t formulation;
    double hmat_eta;
    double hmat_eps;
    int32_t newton_guess;     /* DFN_GUESS_* initial guess of the Newton solve */
    int32_t newton_maxit;     /* Newton iteration cap (0 = 50) */
    double newton_tol;        /* |residual| <= tol * (|tau| + sigma_eff*a*|w|) (0 = 1e-13) */
    double max_step;          /* cap on the next trial step after each accepted step, s
                                 (0 = the reference's one day, src/solver.f90:117-120) */
} dfn_options;

/* Newton formulation (options.formulation = DFN_FORM_NEWTON). The state is
 * Y = [slip | psi | sigmaN0] (the third block keeps its initial value; its
 * derivative is zero). Shear and normal traction are algebraic:
 *   tau   = tau0 + K_T.slip + shear_loading_dot*(t - time0)
 *   sigma = sigmaN0 + K_N.slip + normal_loading_dot*(t - time0)
 * with tau0 chosen so that the initial V satisfies the friction law. Each
 * stage solves tau - eta*V + (sigma+P)*a*asinh(V*C/(2 V0)) = 0 for V in
 * w = asinh(V*C/(2 V0)), C = exp((f0 + b psi)/a), eta = mu/(2 cs); the
 * derivative of this law in time is the reference's dV/dt
 * (src/friction/RateStateAgingModeII.f90:54-68). */
enum { DFN_FORM_V = 0, DFN_FORM_NEWTON = 1 };
/* Initial guesses (w = asinh(V C / 2 V0), C = exp((f0 + b psi)/a)):
 * QUASISTATIC neglects radiation damping, w0 = tau/(sigma_eff a), exact when
 * eta*V << tau; ANALYTIC takes whichever of w0 and the radiation-only root
 * wr (eta V(wr) = tau) is nearer zero: both bound the root from the same
 * side, so Newton converges monotonically from it; MLP adds the correction
 * predicted by the learned network (dfn_set_mlp) to the ANALYTIC start and
 * Newton starts from whichever of the two has the smaller FP64 residual (the
 * network is evaluated only where the ANALYTIC start misses the tolerance);
 * WARM starts from the last solution of the element. Convergence is always
 * decided on the FP64 residual. With sigma_eff <= 0 there is no frictional
 * strength and V = tau/eta without a solve. */
enum { DFN_GUESS_ANALYTIC = 0, DFN_GUESS_MLP = 1, DFN_GUESS_WARM = 2, DFN_GUESS_QUASISTATIC = 3 };
/* The learned guess: an MLP 7 -> 64 -> 64 -> 1 with SiLU activations,
 * trained in FP32; the friction kernel evaluates it with FP16 tensor-core
 * MMAs and FP32 accumulation. Weights, flat, in this order: W1[7][64],
 * b1[64], W2[64][64], b2[64], W3[64], b3[1]. Inputs, from tau, psi,
 * sigma_eff = -(sigmaN + P), P, a, b:
 *   x = [wa/100, psi/30, ln(sigma_eff)/20 - 0.85, P/(sigma_eff + |P|),
 *        100a - 1, 100b - 1, clamp(|wr| - |w0|, -30, 30)/10]
 * with wa the ANALYTIC start; output y, guess w = wa + 10 y. Recorded
 * training samples (dfn_record) are these inputs and the target
 * (w* - wa)/10 of converged solves whose ANALYTIC start missed the
 * tolerance. */
#define DFN_MLP_PARAMS 4737
#define DFN_MLP_IN 7
#define DFN_MLP_HIDDEN 64

/* Per-call report of the solve driver. */
typedef struct dfn_report {
    int64_t it_count;         /* accepted steps since the start (reference it_count) */
    int64_t attempts;         /* RK attempts, accepted and rejected */
    int64_t rejected;
    int64_t rhs_evals;
    int64_t cg_iterations;    /* pressure CG iterations summed over all solves */
    int64_t probe_halvings;   /* t_try halvings forced by CG non-convergence */
    double time;              /* simulated time after the last step */
    double t_try;             /* next trial step */
    double last_hdid;
    int32_t status;
    int32_t pad;
    int64_t stage_cg_failures; /* stage pressure solves that hit the CG cap (the stage then uses the last
                                  CG iterate; the reference would use an uninitialised P_temp) */
    int64_t newton_solves;     /* element Newton solves (Newton formulation) */
    int64_t newton_iters;      /* Newton iterations summed over the solves */
    int64_t newton_fail;       /* solves that hit the iteration cap */
    int64_t mlp_warps;         /* warps (32 elements) that evaluated the learned guess */
} dfn_report;

typedef struct dfn_handle dfn_handle;

/* ---- lifecycle ------------------------------------------------------- */
int32_t dfn_abi_version(void);
int64_t dfn_problem_struct_size(void);
int64_t dfn_options_struct_size(void);
int64_t dfn_report_struct_size(void);
const char *dfn_status_string(int32_t status);
const char *dfn_last_error(void);
void dfn_default_options(dfn_options *opt);

/* Reads the problem, builds geometry (src/initialisation.f90:139-272),
 * assembles the kernel matrices on the device and sets time/t_try/it_count
 * as solve() does at entry (src/solver.f90:47-56). */
int32_t dfn_create(const dfn_problem *prob, const dfn_options *opt, dfn_handle **out);
/* Autotuner: times the interchangeable launch shapes on the handle's own
 * data and keeps the fastest. K.V: TMA bulk copies or 128-bit loads
 * (gemv_impl 0/1, bitwise identical results); tridiagonal pressure: short
 * segments (<= 64 elements) solved by one warp each (scans; tri_thread 0,
 * ms[2]), one thread each (sequential Thomas; 1, ms[3]) or one thread each
 * in tiles staged through shared memory (the same recurrence, identical to
 * the threads; 2, ms[5]), the warps equal to the others to rounding.
 * ms[0] and ms[1] = milliseconds per launch of K.V TMA and LDG (0 = not
 * timed).
 * For DFN_STORE_BF16X2_TC handles the K.V choices are instead the
 * tensor-core GEMM as a persistent kernel (one CTA per SM walking the work
 * units, epilogue overlapped with the next unit; gemv_impl 0, ms[0]), one
 * unit per CTA with the deepest shared-memory ring (gemv_impl 1, ms[1]) or
 * with a 2-stage ring (two CTAs per SM; gemv_impl 2, ms[4], timed when it
 * differs from the deepest ring); all give identical results.
 * CG pressure (DFN_PRESSURE_CG): the stage systems of the batch solved by one
 * CTA each on global memory (ms[2]), by a cluster of CTAs each with the
 * vectors in shared memory (ms[3]; handles with systems of 2048 elements or
 * more) or by one CTA each with the vectors in shared memory (ms[5]; larger
 * systems of the batch on global memory); cg_cluster = 0, 1 or 2 names the
 * form kept, cg_cluster_ctas = CTAs per cluster of this handle's cluster
 * form (2 to 16; 0 when it has none). The forms differ in the order of the
 * dot-product sums (equal to rounding).
 * H-matrix handles: the dense-row and small-leaf kernels on one CTA per
 * task or on persistent grids of 4 or 8 CTAs per SM (identical results);
 * ms[0] the fastest combination, ms[1] one CTA per task.
 * Without a call, K.V uses options.gemv_impl (0..2 for tensor-core handles),
 * the short segments use tiles once a launch has at least 16384 of them,
 * and the CG uses clusters when all of a launch's clusters fit on the GPU at
 * once. No counterpart in the reference. */
typedef struct dfn_tuning {
    int32_t gemv_impl;
    int32_t tri_thread;
    double ms[6];
    int32_t cg_cluster;
    int32_t cg_cluster_ctas;
    int64_t hm_dense_grid;    /* H-matrix handles: CTAs of the dense-row kernel kept (0: one per task) */
    int64_t hm_warp_grid;     /* and of the small-leaf kernel (0: one per four leaves) */
} dfn_tuning;
int32_t dfn_autotune(dfn_handle *h, dfn_tuning *t);

/* Solve loops (dfn_solve_steps, dfn_solve_batch) replay a CUDA graph of 8
 * rounds of the solve() loop when at least 8 rounds remain (on by default;
 * captured at the first such call, on a private stream, and replayed on the
 * handle's stream). Results are identical either way; enable = 0 launches
 * every kernel on its own. While dfn_profile_kv is on, kernels are launched
 * one by one so that each K.V launch is timed. No counterpart in the
 * reference (a host loop of subroutine calls). */
int32_t dfn_set_graphs(dfn_handle *h, int32_t enable);
/* Polls of the bounded waits in the TMA K.V pipeline (gemv_impl 0 of the
 * dense storages) before a kernel gives up: it then stops streaming, waits
 * with the full limit for its own copies in flight, raises an error flag
 * and returns; the next call that reads the step controllers returns
 * DFN_ERR_TIMEOUT once (the partial sums of that K.V are incomplete, so the
 * state must be restored, e.g. with dfn_set_state). polls < 0 restores the
 * default (2^22 polls, far beyond any copy's latency); 0 gives up at the
 * first wait, which tests the error path. No counterpart in the reference. */
int32_t dfn_set_wait_limit(dfn_handle *h, int32_t polls);
/* Form of the CG pressure solves (DFN_PRESSURE_CG handles): -1 the default
 * rule (clusters when a launch's clusters all fit on the GPU at once, else
 * one CTA per system on global memory), 0 one CTA per system on global
 * memory, 1 one thread-block cluster per system with shared-memory vectors
 * (systems of 2048 elements or more), 2 one CTA per system with shared-memory
 * vectors (systems too large for them on global memory). The forms agree to
 * the solver tolerance. dfn_autotune sets the fastest. No counterpart in the
 * reference. */
int32_t dfn_set_cg_form(dfn_handle *h, int32_t form);
/* H-matrix handles: the whole low-rank leaves of at most 32 KiB of factors
 * by one warp each, four per CTA (form 0, the default: the loads of many
 * leaves in flight per SM), or by one CTA each (form 1, like the larger
 * leaves). The forms sum each leaf in another order (agreement to
 * rounding). No counterpart in the reference (ZGEMV per leaf,
 * src/hmatrix/calculation_hmat.f90:3-165). */
int32_t dfn_set_hmat_small_leaves(dfn_handle *h, int32_t form);
/* Launch shape of the short tridiagonal segments (DFN_PRESSURE_TRIDIAG
 * handles): 0 one warp per segment (scans), 1 one thread per segment, 2 one
 * thread per segment in tiles staged through shared memory (identical to 1).
 * dfn_autotune sets the fastest. No counterpart in the reference. */
int32_t dfn_set_tri_shape(dfn_handle *h, int32_t shape);
/* H-matrix handles: CTAs of the dense-row kernel and of the small-leaf
 * kernel (one warp per leaf); 0 = one CTA per task (per four leaves), n > 0
 * = a grid of n CTAs looping over the tasks (leaves). Same arithmetic per
 * row, identical results. dfn_autotune sets the fastest. No counterpart in
 * the reference. */
int32_t dfn_set_hmat_grids(dfn_handle *h, int64_t dense_ctas, int64_t warp_ctas);
/* A batch of independent networks in one handle (no counterpart in the
 * reference, which runs one network per process). All networks share the
 * fracture mode and the options; each keeps its own state, step size,
 * controller and done flag, and every kernel launch covers the whole batch.
 * dfn_create(p, ...) is dfn_create_batch(p, 1, ...). The per-network
 * operator entry points below (kernel, compute_P, friction_law, rkqs,
 * set_state, snapshot, step_host) need a batch of one. */
int32_t dfn_create_batch(const dfn_problem *probs, int32_t count, const dfn_options *opt, dfn_handle **out);
int32_t dfn_batch_size(const dfn_handle *h);
int32_t dfn_destroy(dfn_handle *h);
int32_t dfn_set_stream(dfn_handle *h, void *cuda_stream);
int64_t dfn_nb_element(const dfn_handle *h);
/* Fault crossings found over the batch (see the pressure solver notes). */
int64_t dfn_crossing_count(const dfn_handle *h);
/* Bytes of stored kernel matrices (K.V algorithmic bytes per evaluation). */
int64_t dfn_kernel_bytes(const dfn_handle *h);

/* ---- operators (host buffers) ---------------------------------------- */
/* K.V of every network of a batch: slip, sT and sN hold the networks'
 * vectors back to back (host memory, sum of nb_element doubles each; sN may
 * be NULL). Allocates a device buffer per call (a utility, not a stage of the
 * solve loop). No counterpart in the reference, whose kernel_ptr serves one
 * network (src/variables.f90:17-26). */
int32_t dfn_kernel_batch(dfn_handle *h, const double *slip, double *sT, double *sN);
/* Replaces kernel_ptr => directII/directIII/hmatII/hmatIII,
 * interface src/variables.f90:17-26: stressT/stressN = K.slip (stress rates
 * when slip holds V). stressN may be NULL in mode III. */
int32_t dfn_kernel(dfn_handle *h, const double *slip, double *stressT, double *stressN);

/* Replaces compute_P(dt,P_temp,P_dot_temp,ier), src/fluid_diffusion.f90:24-152:
 * implicit step of length dt from the committed pressure. On *ier==1 the
 * outputs are left untouched, as in the reference. */
int32_t dfn_compute_P(dfn_handle *h, double dt, double *P_temp, double *P_dot, int32_t *ier);

/* Replaces fric_law_ptr => ode_RateStateAgingModeII/III, interface
 * src/variables.f90:9-14: Y_dot = f(x, Y) with x the offset from the step start. */
int32_t dfn_friction_law(dfn_handle *h, double x, int64_t nv, const double *Y, double *Y_dot);

/* Replaces rkqs (src/ode_solver/ode_bs.f90:125-174): one adaptive Cash-Karp
 * step of the handle's ODE from y, with dydx = f(x, y) supplied. */
int32_t dfn_rkqs(dfn_handle *h, double *y, const double *dydx, int64_t nv, double *x,
                 double htry, double eps, const double *yscal, double *hdid, double *hnext);

/* ---- solve driver ----------------------------------------------------- */
/* Advances the solve() loop (src/solver.f90:59-198) by n_steps accepted steps
 * on the device: injection clamp, CG probe, scaling RHS, rkqs, 1-day cap,
 * pressure commit, time update, save_data and the sigmaN>0 check. */
int32_t dfn_solve_steps(dfn_handle *h, int64_t n_steps, dfn_report *rep);

/* One step with host buffers on both sides: uploads Y/P/time/t_try from
 * pinned or pageable host memory, advances one accepted step and downloads
 * the save_data snapshot (V, theta, P, tractionT, tractionN). */
int32_t dfn_step_host(dfn_handle *h, const double *Y_in, const double *P_in, double time_in,
                      double t_try_in, double *V_out, double *theta_out, double *P_out,
                      double *tractionT_out, double *tractionN_out, dfn_report *rep);

/* Advances every network of the batch by n_steps accepted steps of its own
 * solve() loop, or, when t_end > 0, until its simulated time reaches t_end
 * (n_steps = 0 then means no step limit). Networks that finish or fail stop
 * while the others go on. reps (may be NULL) receives one report per network. */
int32_t dfn_solve_batch(dfn_handle *h, int64_t n_steps, double t_end, dfn_report *reps);
int32_t dfn_get_state_instance(dfn_handle *h, int32_t i, double *Y, double *P, double *time, double *t_try,
                               int64_t *it_count);
/* Slip of network i (m). The reference allocates slip
 * (src/configuration.f90:190) but never updates it; here, in the V
 * formulation, it is the integral of V carried by the same Cash-Karp stages
 * as a passive component outside the error norm, slip + h (C1 V1 + C3 V3 +
 * C4 V4 + C6 V6) with V_s the slip rate of stage s (src/ode_solver/
 * ode_bs.f90:223), zero at dfn_create and committed with the state; in the
 * Newton formulation it is the first block of the state. dfn_set_slip
 * overwrites it (e.g. after dfn_set_state). */
int32_t dfn_get_slip(dfn_handle *h, int32_t i, double *slip);
int32_t dfn_set_slip(dfn_handle *h, int32_t i, const double *slip);
/* Counters and status of network i since the handle was created. */
int32_t dfn_get_report(dfn_handle *h, int32_t i, dfn_report *rep);

/* State access. Y has 3N entries. */
int32_t dfn_get_state(dfn_handle *h, double *Y, double *P, double *time, double *t_try,
                      int64_t *it_count);
int32_t dfn_set_state(dfn_handle *h, const double *Y, const double *P, double time, double t_try,
                      int64_t it_count);

/* The save_data snapshot of the last accepted step (src/solver.f90:211-222):
 * V, theta=Dc/V0*exp(psi), P, tractionTel=SigmaT_dot of the last RHS
 * evaluation, tractionNel=sigmaN, permeability, time. Any pointer may be NULL. */
int32_t dfn_get_snapshot(dfn_handle *h, double *V, double *theta, double *P, double *tractionT,
                         double *tractionN, double *permeability, double *time);

/* ---- device-pointer entry points (same stream as the handle) ---------- */
int32_t dfn_kernel_device(dfn_handle *h, const double *d_slip, double *d_stressT,
                          double *d_stressN);

/* ---- allocation-free pressure step ------------------------------------ */
/* No counterpart in the reference: an extra entry point of this library.
 *
 * The implicit pressure step of dfn_compute_P (the reference's CG, with its
 * 200-iteration cap) for networks WITHOUT fault crossings, for callers that
 * must not allocate device memory: host programs that give all device
 * memory to their own pool allocator at start-up (so a cudaMalloc would fail
 * or fight the pool), and time-stepping loops that cannot afford the
 * device-wide synchronisation cudaMalloc and cudaFree may cause. It needs no
 * handle and allocates nothing; the caller passes every input and output as
 * device pointers. It takes no crossing arrays, so for a network with fault
 * crossings it solves the uncoupled chain; use dfn_compute_P there.
 *
 * Its CG work vectors live in one fixed device array inside this library,
 * sized for DFN_NOALLOC_MAX_ELEMENTS elements (about 2 MiB); every GPU that
 * loads the library holds that array until the process exits. Larger
 * problems are rejected with DFN_ERR_ARG. Work runs in the calling thread's
 * current context and on `stream` (NULL = legacy default stream); every
 * call looks up the array's address in that context, copies the solver's
 * status to host memory and synchronises `stream`, so it must not be issued
 * while `stream` (or a stream the legacy default stream waits on) is being
 * captured into a CUDA graph. All calls share the one array, so calls that
 * overlap on the GPU (other threads or streams) race; serialise them.
 *
 * Inputs: d_P (committed pressure), d_permeability_x (N+1 face values as
 * built by the reference, src/initialisation.f90:252-269), d_ds (element
 * lengths), the fluid constants, tol_solver, and the sources (fault id
 * 1-based, element index 0-based into the concatenated element arrays).
 * Outputs: d_P_temp, d_P_dot. *ier = 1 when CG hits its iteration cap (the
 * outputs are left untouched and the call returns DFN_OK, as the
 * reference's compute_P returns early) and when the solution is not finite
 * (the outputs are written, as in the reference, src/fluid_diffusion.f90:
 * 146-148, and the call returns DFN_ERR_NONFINITE). */
#define DFN_NOALLOC_MAX_ELEMENTS 65536
int32_t dfn_compute_P_noalloc(int64_t nb_element, double dt, double time, const double *d_P,
                              const double *d_permeability_x, const double *d_ds, double porosity,
                              double dyn_viscosity, double fluid_comp, double rock_comp, double tol_solver,
                              int64_t nb_source, const int64_t *d_src_fault, const int64_t *d_src_element,
                              const double *d_src_Q, const double *d_src_t_beg, const double *d_src_t_end,
                              double *d_P_temp, double *d_P_dot, int32_t *ier, void *stream);

/* ---- learned Newton guess (no counterpart in the reference) ------------- */
/* Sets the MLP weights (DFN_MLP_PARAMS floats, host memory) used by
 * DFN_GUESS_MLP. */
int32_t dfn_set_mlp(dfn_handle *h, const float *weights);
/* The gate of the learned guess: a warp evaluates the network only when one
 * of its elements' analytic start leaves a residual above rel * (|tau| +
 * sigma_eff a |w|) (default 1e-1: Newton from such a start takes four or
 * more iterations; closer starts converge in a few, which an FP16 network's
 * guess cannot beat); the warp then offers the guess to every element whose
 * start misses the tolerance. 0 evaluates it wherever a start misses. */
int32_t dfn_set_mlp_gate(dfn_handle *h, double rel);
/* Records converged Newton solves: for every solve, the 6 MLP inputs and the
 * training target (w* - wa)/10, FP32, in a device buffer of `capacity`
 * samples (capacity 0 stops recording). dfn_record_read copies up to `max`
 * samples to host memory (x: DFN_MLP_IN per sample, t: 1) and returns the
 * count. */
int32_t dfn_record(dfn_handle *h, int64_t capacity);
int32_t dfn_record_read(dfn_handle *h, float *x, float *t, int64_t max, int64_t *count);
/* Trains the MLP on the GPU with the library's own forward/backward kernels
 * (Adam, mean squared error, minibatches drawn in a seeded order) on n
 * samples in host memory; weights (in/out) are DFN_MLP_PARAMS floats.
 * loss[0]/loss[1] receive the mean loss of the first and the last epoch.
 * Standalone: no handle, runs on the current device. */
int32_t dfn_mlp_train(const float *x, const float *t, int64_t n, float *weights, int32_t epochs, int32_t batch,
                      float lr, uint64_t seed, float *loss);
/* Mean-squared-error loss and its gradient over n samples (host buffers),
 * computed by the same device kernels as training; grad has
 * DFN_MLP_PARAMS floats. */
int32_t dfn_mlp_loss_grad(const float *x, const float *t, int64_t n, const float *weights, float *loss,
                          float *grad);
/* Network outputs y[n] for n input rows (host buffers) by the inference path
 * of the friction kernel: one warp per 32 rows, FP16 tensor-core MMAs with
 * FP32 accumulation. */
int32_t dfn_mlp_infer(const float *x, int64_t n, const float *weights, float *y);
/* Slip rate of network 0 at its current state (Newton formulation: solves
 * the friction law; V formulation: copies V). */
int32_t dfn_velocity(dfn_handle *h, double *V);

/* ---- H-matrix introspection (static_kernel = hmatrix) ------------------ */
/* stats[0..7]: leaves, dense leaves, low-rank leaves, max rank, mean rank x 1000,
 * stored values, dense values, low-rank values (all networks, all components).
 * Returns DFN_ERR_UNSUPPORTED for a dense-kernel handle. */
int32_t dfn_hmat_stats(const dfn_handle *h, int64_t *stats);
/* Cluster order of network 0: perm[pos] = element index (the reference's mat_corr). */
int32_t dfn_hmat_perm(const dfn_handle *h, int32_t *perm);

/* ---- timing helpers (CUDA events on the handle's stream) --------------- */
/* Times `reps` K.V launches of the handle's storage on its stream and
 * returns the mean duration of one launch in milliseconds. */
int32_t dfn_time_kernel(dfn_handle *h, int32_t reps, double *ms_per_launch);
/* Number of kernels this library launched since the handle was created. */
int64_t dfn_launch_count(const dfn_handle *h);
/* Per-launch CUDA-event timing of the K.V kernel inside the solve driver.
 * enable!=0 clears the record and starts recording (up to 16384 launches);
 * read returns the summed duration (ms) and the number of recorded launches. */
int32_t dfn_profile_kv(dfn_handle *h, int32_t enable);
int32_t dfn_profile_kv_read(dfn_handle *h, double *total_ms, int64_t *launches);

#ifdef __cplusplus
}
#endif
#endif /* DFN_B200_H */
