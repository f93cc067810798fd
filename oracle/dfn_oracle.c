/*
 * dfn_oracle.c — CPU FP64 restatement of DemystiFicatioN's earthquake-cycle
 * hot path. TEST INFRASTRUCTURE ONLY: it is the checker for the CUDA library
 * (tests, smoke, and the cpu_baseline / reference arm of bench.py). The
 * product path never calls it.
 *
 * PARITY UNPINNED: the reference is Fortran with no compiler in this image
 * and ships no golden outputs, so this restatement is checked against
 * known answers (telescoping sums, steady state, exact ODE solutions, direct
 * tridiagonal solves) instead of reference outputs.
 *
 * Each routine cites the reference file:line it restates. Arithmetic follows
 * the Fortran expression order; this file is compiled with
 * -ffp-contract=off so no FMA is formed (the reference's x86-64 -O1 build
 * has none either).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/dfn_b200.h"

#define PI_F90 3.141592653589793238 /* src/variables.f90:44 */

typedef struct orc {
    int64_t N, F;
    int mode, static_kernel;
    int64_t *fault_n, *fault_first; /* fault_first: 0-based first element */
    double *node;                   /* 2*(N+1) */
    double *elem, *ds, *tan, *nrm;  /* ini_value geometry */
    double *a, *b, *Dc, *f0, *V0, *nload, *sload, *perm, *permx;
    unsigned char *fake;
    double mu, cp, cs;
    double S11d, S12d, S22d, S31d, S32d;
    double rock_comp, fluid_comp, porosity, dyn_visc;
    int64_t nsrc;
    int64_t *src_fault, *src_index;
    double *src_Q, *src_tb, *src_te;
    double tol;
    /* mutable state */
    double time, t_try;
    int64_t it_count;
    double *Y, *P, *Pdot, *SigmaT_dot, *SigmaN_dot;
    /* dense kernel (optional) */
    double *KT, *KN;
    int kernel_impl; /* 0 matrix-free reference routine, 1 dense stored K, 2 H-matrix */
    void *hmat;      /* orc_hmat */
    int nthreads;
    /* counters */
    int64_t cg_iters, rhs_evals, attempts, rejected, halvings, stage_noconv;
    int last_status;
    /* fault crossings: per element row, xptr[k]..xptr[k+1] contributions
     * (partner elements xa, xb; harmonic permeabilities xkl, xkr) */
    int64_t ncross, nxc;
    int64_t *xptr, *xa, *xb;
    double *xkl, *xkr;
    /* slip: integrated as a passive component (dslip/dt = V) of the V
     * formulation, outside the error norm; the reference allocates it
     * (src/configuration.f90:190) but never updates it */
    double *slip;
    /* Newton slip formulation (the library's DFN_FORM_NEWTON): form 1 means
     * Y = [slip | psi | sigmaN0] and V solved from the friction law */
    int form, nguess, nmaxit;
    double ntol, time0;
    double max_step; /* cap on t_try after a step (the reference's one day) */
    /* permeability evolution (permeability_coupling = 1) */
    int pcoup;
    double *kstar, *kmin, *Snk;
    double *tau0;
    int64_t newton_solves, newton_iters, newton_fail;
} orc;

static void *xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

struct orc_hmat;
static void orc_hmat_free(struct orc_hmat *H);

/* ---------------------------------------------------------------------- */
/* Geometry and loading projection: src/initialisation.f90:145-153,159-205,
 * permeability_x: src/initialisation.f90:252-269.                         */
static void orc_ini_value(orc *o)
{
    int64_t N = o->N;
    for (int64_t k = 0; k < N; k++) {
        double x0 = o->node[2 * k], y0 = o->node[2 * k + 1];
        double x1 = o->node[2 * k + 2], y1 = o->node[2 * k + 3];
        o->elem[2 * k] = (x1 + x0) * 0.5;
        o->elem[2 * k + 1] = (y1 + y0) * 0.5;
        o->ds[k] = sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0));
        o->tan[2 * k] = (x1 - x0) / o->ds[k];
        o->tan[2 * k + 1] = (y1 - y0) / o->ds[k];
        o->nrm[2 * k] = -o->tan[2 * k + 1];
        o->nrm[2 * k + 1] = o->tan[2 * k];
    }
    double *sig = o->Y + 2 * N;
    for (int64_t k = 0; k < N; k++) {
        double n1 = o->nrm[2 * k], n2 = o->nrm[2 * k + 1];
        double t1 = o->tan[2 * k], t2 = o->tan[2 * k + 1];
        if (o->mode == DFN_MODE_III) {
            o->sload[k] = o->sload[k] - t2 * o->S31d + t1 * o->S32d;
            sig[k] = sig[k] + n1 * (n1 * o->S11d + n2 * o->S12d) + n2 * (n1 * o->S12d + n2 * o->S22d);
        } else {
            /* Sigma11/12/22 (not _dot) are never read and stay zero. */
            sig[k] = sig[k] + n1 * (n1 * 0.0 + n2 * 0.0) + n2 * (n1 * 0.0 + n2 * 0.0);
            o->nload[k] = o->nload[k] + n1 * (n1 * o->S11d + n2 * o->S12d) + n2 * (n1 * o->S12d + n2 * o->S22d);
            o->sload[k] = o->sload[k] + t1 * (n1 * o->S11d + n2 * o->S12d) + t2 * (n1 * o->S12d + n2 * o->S22d);
        }
    }
    for (int64_t j = 0; j <= N; j++) o->permx[j] = 0.0;
    for (int64_t k = 1; k < N; k++)
        o->permx[k] = 2.0 * o->perm[k - 1] * o->perm[k] / (o->perm[k - 1] + o->perm[k]);
}

/* find_fault_crossing (src/initialisation.f90:279-344): node pairs of two
 * faults closer than 0.01 * the smaller of the two faults' smallest element
 * length. Each crossing couples the (up to) two elements around the node on
 * one fault with those on the other (src/fluid_diffusion.f90:213-295,
 * 338-405), here with the corrections of that model: every coefficient uses
 * the element length of its own row (the reference uses ds(1) in the
 * diagonal and a stale ds(k-1) in the product), every row divides by the
 * diagonal (one reference row divides by the element index), and elements
 * outside the fault (fake elements, or none before the first fault) are not
 * coupled. Contributions of a row are kept in crossing order, each crossing
 * updating its rows in the order element1(node-1), element1(node),
 * element2(node-1), element2(node). */
static double orc_harm(double k1, double k2) { return (k1 + k2 > 0.0) ? 2.0 * k1 * k2 / (k1 + k2) : 0.0; }

static void orc_find_crossings(orc *o)
{
    int64_t N = o->N, F = o->F;
    double *minds = (double *)xcalloc(F, 8);
    for (int64_t f = 0; f < F; f++) {
        double m = INFINITY;
        for (int64_t e = 0; e < o->fault_n[f]; e++) m = fmin(m, o->ds[o->fault_first[f] + e]);
        minds[f] = m;
    }
    /* pass 1: crossings; pass 2: contributions per row */
    int64_t cap = 0, n = 0;
    int64_t *cr = NULL;   /* (f1, f2, a, b) with a, b 0-based local nodes */
    /* bounding boxes of the faults' nodes: pairs farther apart than the
     * threshold are skipped (the loop order is the reference's) */
    double *bb = (double *)xcalloc(4 * F, 8);
    for (int64_t f = 0; f < F; f++) {
        bb[4 * f] = bb[4 * f + 2] = INFINITY;
        bb[4 * f + 1] = bb[4 * f + 3] = -INFINITY;
        for (int64_t a = 0; a <= o->fault_n[f]; a++) {
            const double *q = o->node + 2 * (o->fault_first[f] + a);
            bb[4 * f] = fmin(bb[4 * f], q[0]); bb[4 * f + 1] = fmax(bb[4 * f + 1], q[0]);
            bb[4 * f + 2] = fmin(bb[4 * f + 2], q[1]); bb[4 * f + 3] = fmax(bb[4 * f + 3], q[1]);
        }
    }
    for (int64_t f1 = 0; f1 < F; f1++)
        for (int64_t f2 = f1 + 1; f2 < F; f2++) {
            double thr = 0.01 * fmin(minds[f1], minds[f2]);
            if (bb[4 * f1] > bb[4 * f2 + 1] + thr || bb[4 * f2] > bb[4 * f1 + 1] + thr ||
                bb[4 * f1 + 2] > bb[4 * f2 + 3] + thr || bb[4 * f2 + 2] > bb[4 * f1 + 3] + thr)
                continue;
            for (int64_t a = 0; a <= o->fault_n[f1]; a++) {
                const double *p1 = o->node + 2 * (o->fault_first[f1] + a);
                for (int64_t b = 0; b <= o->fault_n[f2]; b++) {
                    const double *p2 = o->node + 2 * (o->fault_first[f2] + b);
                    double d = sqrt((p1[0] - p2[0]) * (p1[0] - p2[0]) + (p1[1] - p2[1]) * (p1[1] - p2[1]));
                    if (!(d < thr)) continue;
                    if (n == cap) { cap = cap ? 2 * cap : 16; cr = (int64_t *)realloc(cr, sizeof(int64_t) * 4 * cap); }
                    cr[4 * n] = f1; cr[4 * n + 1] = f2; cr[4 * n + 2] = a; cr[4 * n + 3] = b;
                    n++;
                }
            }
        }
    o->ncross = n;
    /* rows and partners per crossing: element left (a-1) and right (a) of
     * the node, -1 where outside the fault */
    int64_t *rows = (int64_t *)xcalloc(4 * n, 8), *pa = (int64_t *)xcalloc(4 * n, 8), *pb = (int64_t *)xcalloc(4 * n, 8);
    double *kl = (double *)xcalloc(4 * n, 8), *kr = (double *)xcalloc(4 * n, 8);
    int64_t m = 0;
    for (int64_t c = 0; c < n; c++) {
        int64_t f1 = cr[4 * c], f2 = cr[4 * c + 1], a = cr[4 * c + 2], b = cr[4 * c + 3];
        int64_t e1[2] = {a >= 1 ? o->fault_first[f1] + a - 1 : -1, a < o->fault_n[f1] ? o->fault_first[f1] + a : -1};
        int64_t e2[2] = {b >= 1 ? o->fault_first[f2] + b - 1 : -1, b < o->fault_n[f2] ? o->fault_first[f2] + b : -1};
        for (int side = 0; side < 2; side++)
            for (int j = 0; j < 2; j++) {
                int64_t row = side == 0 ? e1[j] : e2[j];
                if (row < 0) continue;
                const int64_t *other = side == 0 ? e2 : e1;
                rows[m] = row;
                pa[m] = other[0] >= 0 ? other[0] : row;
                pb[m] = other[1] >= 0 ? other[1] : row;
                /* harmonic means with the fault-1 element first */
                if (side == 0) {
                    kl[m] = other[0] >= 0 ? orc_harm(o->perm[row], o->perm[other[0]]) : 0.0;
                    kr[m] = other[1] >= 0 ? orc_harm(o->perm[row], o->perm[other[1]]) : 0.0;
                } else {
                    kl[m] = other[0] >= 0 ? orc_harm(o->perm[other[0]], o->perm[row]) : 0.0;
                    kr[m] = other[1] >= 0 ? orc_harm(o->perm[other[1]], o->perm[row]) : 0.0;
                }
                m++;
            }
    }
    /* CSR by row, crossing order kept within a row */
    o->nxc = m;
    o->xptr = (int64_t *)xcalloc(N + 1, 8);
    for (int64_t q = 0; q < m; q++) o->xptr[rows[q] + 1]++;
    for (int64_t k = 0; k < N; k++) o->xptr[k + 1] += o->xptr[k];
    o->xa = (int64_t *)xcalloc(m, 8); o->xb = (int64_t *)xcalloc(m, 8);
    o->xkl = (double *)xcalloc(m, 8); o->xkr = (double *)xcalloc(m, 8);
    int64_t *fill = (int64_t *)xcalloc(N, 8);
    for (int64_t q = 0; q < m; q++) {
        int64_t r = rows[q], at = o->xptr[r] + fill[r]++;
        o->xa[at] = pa[q]; o->xb[at] = pb[q]; o->xkl[at] = kl[q]; o->xkr[at] = kr[q];
    }
    free(fill); free(rows); free(pa); free(pb); free(kl); free(kr); free(cr); free(minds); free(bb);
}

int64_t orc_crossings(const orc *o) { return o->ncross; }

orc *orc_create(const dfn_problem *p)
{
    if (!p || p->nb_element < 2 || p->nb_fault < 1) return NULL;
    orc *o = (orc *)xcalloc(1, sizeof(orc));
    int64_t N = p->nb_element, F = p->nb_fault;
    o->N = N; o->F = F;
    o->mode = p->fracture_mode; o->static_kernel = p->static_kernel;
    o->fault_n = (int64_t *)xcalloc(F, 8); o->fault_first = (int64_t *)xcalloc(F, 8);
    int64_t cnt = 0;
    for (int64_t f = 0; f < F; f++) {
        o->fault_n[f] = p->fault_nb_element[f];
        o->fault_first[f] = cnt;
        cnt += p->fault_nb_element[f] + 1;
    }
    if (cnt - 1 != N) { free(o->fault_n); free(o->fault_first); free(o); return NULL; }
    o->node = (double *)xcalloc(2 * (N + 1), 8);
    memcpy(o->node, p->node, sizeof(double) * 2 * (N + 1));
    o->elem = (double *)xcalloc(2 * N, 8); o->ds = (double *)xcalloc(N, 8);
    o->tan = (double *)xcalloc(2 * N, 8); o->nrm = (double *)xcalloc(2 * N, 8);
#define CP(dst, src) do { dst = (double *)xcalloc(N, 8); memcpy(dst, src, 8 * N); } while (0)
    CP(o->a, p->a); CP(o->b, p->b); CP(o->Dc, p->Dc); CP(o->f0, p->f0); CP(o->V0, p->V0);
    CP(o->nload, p->normal_loading_dot); CP(o->sload, p->shear_loading_dot);
    CP(o->perm, p->permeability);
    o->permx = (double *)xcalloc(N + 1, 8);
    o->fake = (unsigned char *)xcalloc(N, 1);
    /* src/friction/RateStateAgingModeII.f90:81-89: element idx after each fault */
    int64_t idx = 0;
    for (int64_t f = 0; f < F; f++) {
        idx += o->fault_n[f] + 1;
        if (idx <= N) o->fake[idx - 1] = 1;
    }
    o->mu = p->mu; o->cp = p->cp; o->cs = p->cs;
    o->S11d = p->Sigma11_dot; o->S12d = p->Sigma12_dot; o->S22d = p->Sigma22_dot;
    o->S31d = p->Sigma31_dot; o->S32d = p->Sigma32_dot;
    o->rock_comp = p->rock_comp; o->fluid_comp = p->fluid_comp;
    o->porosity = p->porosity; o->dyn_visc = p->dyn_viscosity;
    o->nsrc = p->nb_source;
    o->src_fault = (int64_t *)xcalloc(o->nsrc, 8); o->src_index = (int64_t *)xcalloc(o->nsrc, 8);
    o->src_Q = (double *)xcalloc(o->nsrc, 8); o->src_tb = (double *)xcalloc(o->nsrc, 8);
    o->src_te = (double *)xcalloc(o->nsrc, 8);
    for (int64_t s = 0; s < o->nsrc; s++) {
        o->src_fault[s] = p->src_fault[s]; o->src_index[s] = p->src_index[s];
        o->src_Q[s] = p->src_Q[s]; o->src_tb[s] = p->src_t_beg[s]; o->src_te[s] = p->src_t_end[s];
    }
    o->tol = p->tol_solver;
    o->Y = (double *)xcalloc(3 * N, 8);
    memcpy(o->Y, p->V, 8 * N); memcpy(o->Y + N, p->theta, 8 * N); memcpy(o->Y + 2 * N, p->sigmaN, 8 * N);
    CP(o->P, p->P);
#undef CP
    o->Pdot = (double *)xcalloc(N, 8);
    o->SigmaT_dot = (double *)xcalloc(N, 8); o->SigmaN_dot = (double *)xcalloc(N, 8);
    o->slip = (double *)xcalloc(N, 8);
    o->tau0 = (double *)xcalloc(N, 8);
    o->time0 = p->time0;
    o->nmaxit = 50; o->ntol = 1e-13;
    o->max_step = 24 * 60 * 60;
    o->pcoup = p->permeability_coupling == 1;
    o->kstar = (double *)xcalloc(N, 8); o->kmin = (double *)xcalloc(N, 8); o->Snk = (double *)xcalloc(N, 8);
    if (o->pcoup) { memcpy(o->kmin, p->kmin, 8 * N); memcpy(o->Snk, p->Snk, 8 * N); }
    orc_ini_value(o);
    /* src/initialisation.f90:256-261, from the state after ini_value */
    if (o->pcoup)
        for (int64_t k = 0; k < N; k++)
            o->kstar[k] = o->kmin[k] + (o->perm[k] - o->kmin[k]) * exp(fabs(o->Y[2 * N + k] + o->P[k]) / fabs(o->Snk[k]));
    orc_find_crossings(o);
    /* solve() entry: src/solver.f90:50-56 */
    o->time = p->time0; o->t_try = 100.0; o->it_count = 0;
    o->kernel_impl = 0;
    o->nthreads = 1;
    return o;
}

void orc_destroy(orc *o)
{
    if (!o) return;
    void *ptrs[] = {o->fault_n, o->fault_first, o->node, o->elem, o->ds, o->tan, o->nrm, o->a, o->b,
                    o->Dc, o->f0, o->V0, o->nload, o->sload, o->perm, o->permx, o->fake, o->src_fault,
                    o->src_index, o->src_Q, o->src_tb, o->src_te, o->Y, o->P, o->Pdot, o->SigmaT_dot,
                    o->SigmaN_dot, o->KT, o->KN, o->xptr, o->xa, o->xb, o->xkl, o->xkr, o->slip, o->tau0,
                    o->kstar, o->kmin, o->Snk};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    orc_hmat_free((struct orc_hmat *)o->hmat);
    free(o);
}

void orc_set_threads(orc *o, int n) { o->nthreads = n < 1 ? 1 : n; }
/* cap on t_try after each step (src/solver.f90:117-120 uses one day) */
void orc_set_max_step(orc *o, double s) { o->max_step = s > 0.0 ? s : 24 * 60 * 60; }
void orc_set_kernel_impl(orc *o, int impl) { o->kernel_impl = impl; }
int64_t orc_n(const orc *o) { return o->N; }

/* ---------------------------------------------------------------------- */
/* Matrix-free kernels, the reference's "direct" routines.                 */

/* directII: src/kernel_calculation/directModeII.f90:33-103 */
static void orc_directII(const orc *o, const double *slip, double *sT, double *sN)
{
    int64_t N = o->N;
    const double *el = o->elem, *nd = o->node, *nr = o->nrm;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(o->nthreads)
#endif
    for (int64_t k = 0; k < N; k++) {
        double T = 0.0, Nn = 0.0;
        double e1 = el[2 * k], e2 = el[2 * k + 1];
        double n1 = nr[2 * k], n2 = nr[2 * k + 1];
        for (int64_t l = 0; l < N; l++) {
            double dxl = e1 - nd[2 * l], dyl = e2 - nd[2 * l + 1];
            double dxr = e1 - nd[2 * l + 2], dyr = e2 - nd[2 * l + 3];
            double rl = sqrt(dxl * dxl + dyl * dyl);
            double rr = sqrt(dxr * dxr + dyr * dyr);
            double g1l = dxl / rl, g2l = dyl / rl, g1r = dxr / rr, g2r = dyr / rr;
            double I1tl = (4.0 * n1 * n2 * g1l * g2l + (n2 * n2 - n1 * n1) * (g2l * g2l - g1l * g1l)) * g1l / rl;
            double I2tl = (4.0 * n1 * n2 * g1l * g2l + (n2 * n2 - n1 * n1) * (g2l * g2l - g1l * g1l)) * g2l / rl;
            double I1tr = (4.0 * n1 * n2 * g1r * g2r + (n2 * n2 - n1 * n1) * (g2r * g2r - g1r * g1r)) * g1r / rr;
            double I2tr = (4.0 * n1 * n2 * g1r * g2r + (n2 * n2 - n1 * n1) * (g2r * g2r - g1r * g1r)) * g2r / rr;
            double I1nl = g1l / rl - g2l / rl * (2.0 * n1 * n2 * (g2l * g2l - g1l * g1l) - (n2 * n2 - n1 * n1) * 2.0 * g1l * g2l);
            double I2nl = g2l / rl + g1l / rl * (2.0 * n1 * n2 * (g2l * g2l - g1l * g1l) - (n2 * n2 - n1 * n1) * 2.0 * g1l * g2l);
            double I1nr = g1r / rr - g2r / rr * (2.0 * n1 * n2 * (g2r * g2r - g1r * g1r) - (n2 * n2 - n1 * n1) * 2.0 * g1r * g2r);
            double I2nr = g2r / rr + g1r / rr * (2.0 * n1 * n2 * (g2r * g2r - g1r * g1r) - (n2 * n2 - n1 * n1) * 2.0 * g1r * g2r);
            /* normal_left = normal_right = normal (src/initialisation.f90:203-204) */
            double nl1 = nr[2 * l], nl2 = nr[2 * l + 1];
            T = T + slip[l] * (nl2 * I1tl - nl2 * I1tr - nl1 * I2tl + nl1 * I2tr);
            Nn = Nn + slip[l] * (nl1 * I1nl - nl1 * I1nr + nl2 * I2nl - nl2 * I2nr);
        }
        sT[k] = T; sN[k] = Nn;
    }
    double pref = o->mu / PI_F90 * (1.0 - o->cs * o->cs / (o->cp * o->cp));
    for (int64_t k = 0; k < N; k++) { sN[k] = pref * sN[k]; sT[k] = pref * sT[k]; }
}

/* directIII: src/kernel_calculation/directModeIII.f:35-80, with its own
 * element/tangent (node + 0.5*(dnode), real 0.5 literal). */
static void orc_directIII(const orc *o, const double *slip, double *sT)
{
    int64_t N = o->N;
    const double *nd = o->node;
    double *el = (double *)malloc(16 * N), *t = (double *)malloc(16 * N);
    for (int64_t k = 0; k < N; k++) {
        t[2 * k] = nd[2 * k + 2] - nd[2 * k];
        t[2 * k + 1] = nd[2 * k + 3] - nd[2 * k + 1];
        double nt = sqrt(t[2 * k] * t[2 * k] + t[2 * k + 1] * t[2 * k + 1]);
        t[2 * k] = t[2 * k] / nt; t[2 * k + 1] = t[2 * k + 1] / nt;
        el[2 * k] = nd[2 * k] + 0.5 * (nd[2 * k + 2] - nd[2 * k]);
        el[2 * k + 1] = nd[2 * k + 1] + 0.5 * (nd[2 * k + 3] - nd[2 * k + 1]);
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(o->nthreads)
#endif
    for (int64_t k = 0; k < N; k++) {
        double acc = 0.0;
        for (int64_t l = 1; l <= N + 1; l++) { /* 1-based node index */
            double dx = el[2 * k] - nd[2 * (l - 1)], dy = el[2 * k + 1] - nd[2 * (l - 1) + 1];
            double r1 = sqrt(dx * dx + dy * dy);
            double I1 = t[2 * k] / (r1 * r1) * dx + t[2 * k + 1] / (r1 * r1) * dy;
            if (l - 1 >= 1 && l <= N) acc = acc - (slip[l - 1] - slip[l - 2]) * I1;
            else if (l == 1) acc = acc - slip[l - 1] * I1;
            else acc = acc + slip[l - 2] * I1;
        }
        sT[k] = acc;
    }
    for (int64_t k = 0; k < N; k++) sT[k] = sT[k] * o->mu / (2 * PI_F90);
    free(el); free(t);
}

/* ---------------------------------------------------------------------- */
/* Kernel entries: src/hmatrix/eval_kernel_hmatrix.f90:7-199 with
 * node_left=node(l), node_right=node(l+1) (src/initialisation.f90:212-213).
 * which: 0 = mode III, 1 = mode II shear (T), 2 = mode II normal (N).     */
double orc_kernel_entry(const orc *o, int64_t k, int64_t l, int which)
{
    const double *el = o->elem, *nd = o->node;
    double e1 = el[2 * k], e2 = el[2 * k + 1];
    if (which == 0) {
        double t1 = o->tan[2 * k], t2 = o->tan[2 * k + 1];
        double ax = nd[2 * l] - e1, ay = nd[2 * l + 1] - e2;
        double bx = nd[2 * l + 2] - e1, by = nd[2 * l + 3] - e2;
        double r1 = sqrt(ax * ax + ay * ay);
        double r2 = sqrt(bx * bx + by * by);
        double I1 = t1 / (r1 * r1) * (e1 - nd[2 * l]) + t2 / (r1 * r1) * (e2 - nd[2 * l + 1]);
        double I2 = t1 / (r2 * r2) * (e1 - nd[2 * l + 2]) + t2 / (r2 * r2) * (e2 - nd[2 * l + 3]);
        return -I1 + I2;
    }
    double n1 = o->nrm[2 * k], n2 = o->nrm[2 * k + 1];
    double dxl = e1 - nd[2 * l], dyl = e2 - nd[2 * l + 1];
    double dxr = e1 - nd[2 * l + 2], dyr = e2 - nd[2 * l + 3];
    double rl = sqrt(dxl * dxl + dyl * dyl);
    double rr = sqrt(dxr * dxr + dyr * dyr);
    double g1l = dxl / rl, g2l = dyl / rl, g1r = dxr / rr, g2r = dyr / rr;
    double nl1 = o->nrm[2 * l], nl2 = o->nrm[2 * l + 1];
    if (which == 1) {
        double I1tl = (4.0 * n1 * n2 * g1l * g2l + (n2 * n2 - n1 * n1) * (g2l * g2l - g1l * g1l)) * g1l / rl;
        double I2tl = (4.0 * n1 * n2 * g1l * g2l + (n2 * n2 - n1 * n1) * (g2l * g2l - g1l * g1l)) * g2l / rl;
        double I1tr = (4.0 * n1 * n2 * g1r * g2r + (n2 * n2 - n1 * n1) * (g2r * g2r - g1r * g1r)) * g1r / rr;
        double I2tr = (4.0 * n1 * n2 * g1r * g2r + (n2 * n2 - n1 * n1) * (g2r * g2r - g1r * g1r)) * g2r / rr;
        return nl2 * I1tl - nl2 * I1tr - nl1 * I2tl + nl1 * I2tr;
    }
    double I1nl = g1l / rl - g2l / rl * (2.0 * n1 * n2 * (g2l * g2l - g1l * g1l) - (n2 * n2 - n1 * n1) * 2.0 * g1l * g2l);
    double I2nl = g2l / rl + g1l / rl * (2.0 * n1 * n2 * (g2l * g2l - g1l * g1l) - (n2 * n2 - n1 * n1) * 2.0 * g1l * g2l);
    double I1nr = g1r / rr - g2r / rr * (2.0 * n1 * n2 * (g2r * g2r - g1r * g1r) - (n2 * n2 - n1 * n1) * 2.0 * g1r * g2r);
    double I2nr = g2r / rr + g1r / rr * (2.0 * n1 * n2 * (g2r * g2r - g1r * g1r) - (n2 * n2 - n1 * n1) * 2.0 * g1r * g2r);
    return nl1 * I1nl - nl1 * I1nr + nl2 * I2nl - nl2 * I2nr;
}

/* Dense unscaled K (row-major, K[k*N+l]); KN only in mode II. */
int orc_assemble_dense(orc *o)
{
    int64_t N = o->N;
    free(o->KT); free(o->KN); o->KT = o->KN = NULL;
    o->KT = (double *)malloc(sizeof(double) * N * N);
    if (!o->KT) return -1;
    if (o->mode == DFN_MODE_II) {
        o->KN = (double *)malloc(sizeof(double) * N * N);
        if (!o->KN) return -1;
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(o->nthreads)
#endif
    for (int64_t k = 0; k < N; k++)
        for (int64_t l = 0; l < N; l++) {
            if (o->mode == DFN_MODE_II) {
                o->KT[k * N + l] = orc_kernel_entry(o, k, l, 1);
                o->KN[k * N + l] = orc_kernel_entry(o, k, l, 2);
            } else {
                o->KT[k * N + l] = orc_kernel_entry(o, k, l, 0);
            }
        }
    return 0;
}

void orc_copy_dense(const orc *o, double *KT, double *KN)
{
    int64_t NN = o->N * o->N;
    if (KT && o->KT) memcpy(KT, o->KT, 8 * NN);
    if (KN && o->KN) memcpy(KN, o->KN, 8 * NN);
}

/* K.V with the stored dense K, sequential sums per row, then the reference
 * prefactor (hmatII src/kernel_calculation/hmatrixModeII.f90:65-69,
 * hmatIII src/kernel_calculation/hmatrixModeIII.f90:53-56). */
static void orc_dense_kv(const orc *o, const double *slip, double *sT, double *sN)
{
    int64_t N = o->N;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(o->nthreads)
#endif
    for (int64_t k = 0; k < N; k++) {
        double t = 0.0, n = 0.0;
        const double *rt = o->KT + k * N;
        for (int64_t l = 0; l < N; l++) t = t + rt[l] * slip[l];
        if (o->KN) {
            const double *rn = o->KN + k * N;
            for (int64_t l = 0; l < N; l++) n = n + rn[l] * slip[l];
        }
        sT[k] = t; if (sN) sN[k] = n;
    }
    if (o->mode == DFN_MODE_II) {
        double pref = o->mu / PI_F90 * (1.0 - o->cs * o->cs / (o->cp * o->cp));
        for (int64_t k = 0; k < N; k++) { sT[k] = pref * sT[k]; if (sN) sN[k] = pref * sN[k]; }
    } else {
        for (int64_t k = 0; k < N; k++) { sT[k] = o->mu / (2.0 * PI_F90) * sT[k]; if (sN) sN[k] = 0.0; }
    }
}

static void orc_hmat_kv(const orc *o, const double *slip, double *sT, double *sN);

/* kernel_ptr dispatch (src/initialisation.f90:105-128). */
void orc_kernel(orc *o, const double *slip, double *sT, double *sN)
{
    if (o->kernel_impl == 2 && o->hmat) { orc_hmat_kv(o, slip, sT, sN); return; }
    if (o->kernel_impl == 1 && o->KT) { orc_dense_kv(o, slip, sT, sN); return; }
    if (o->mode == DFN_MODE_II) orc_directII(o, slip, sT, sN);
    else { orc_directIII(o, slip, sT); if (sN) memset(sN, 0, 8 * o->N); }
}

/* ---------------------------------------------------------------------- */
/* Pore pressure: src/fluid_diffusion.f90, with the fault-crossing coupling
 * of orc_find_crossings.                                                   */
static inline double orc_coef(const orc *o, double kx, double dt, double dsv)
{
    /* kx*dt/(porosity*dyn_viscosity*(fluid_comp+rock_comp)*ds**2) */
    return kx * dt / (o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp) * (dsv * dsv));
}

/* compute_diag: src/fluid_diffusion.f90:308-334 */
static void orc_diag(const orc *o, double dt, double *diag)
{
    int64_t N = o->N;
    const double *px = o->permx, *ds = o->ds;
    diag[0] = 1.0 + orc_coef(o, px[1], dt, ds[0]);
    diag[N - 1] = 1.0 + orc_coef(o, px[N - 1], dt, ds[N - 1]);
    for (int64_t k = 1; k < N - 1; k++)
        diag[k] = 1.0 + (px[k] + px[k + 1]) * dt /
                            (o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp) * (ds[k] * ds[k]));
    /* crossing terms (src/fluid_diffusion.f90:338-405, own-row ds) */
    for (int64_t k = 0; k < N; k++)
        for (int64_t q = o->xptr[k]; q < o->xptr[k + 1]; q++)
            diag[k] = diag[k] + orc_coef(o, o->xkl[q], dt, ds[k]) + orc_coef(o, o->xkr[q], dt, ds[k]);
}

/* compute_MatrixVector: src/fluid_diffusion.f90:163-204 */
static void orc_matvec(const orc *o, const double *v, double dt, const double *diag, double *out)
{
    int64_t N = o->N;
    const double *px = o->permx, *ds = o->ds;
    double A1, A2, A3;
    A2 = 1.0 + orc_coef(o, px[1], dt, ds[0]);
    A3 = -px[1] * dt / (o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp) * (ds[0] * ds[0]));
    out[0] = (A2 * v[0] + A3 * v[1]) / diag[0];
    A1 = -px[N - 1] * dt / (o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp) * (ds[N - 1] * ds[N - 1]));
    A2 = 1.0 + orc_coef(o, px[N - 1], dt, ds[N - 1]);
    out[N - 1] = (A1 * v[N - 2] + A2 * v[N - 1]) / diag[N - 1];
    for (int64_t k = 1; k < N - 1; k++) {
        A1 = -px[k] * dt / (o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp) * (ds[k - 1] * ds[k - 1]));
        A2 = 1.0 + (px[k] + px[k + 1]) * dt /
                       (o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp) * (ds[k] * ds[k]));
        A3 = -px[k + 1] * dt / (o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp) * (ds[k + 1] * ds[k + 1]));
        out[k] = (A1 * v[k - 1] + A2 * v[k] + A3 * v[k + 1]) / diag[k];
    }
    /* crossing terms (src/fluid_diffusion.f90:213-295, own-row ds, / diag) */
    for (int64_t k = 0; k < N; k++)
        for (int64_t q = o->xptr[k]; q < o->xptr[k + 1]; q++) {
            double cl = orc_coef(o, o->xkl[q], dt, ds[k]), cr = orc_coef(o, o->xkr[q], dt, ds[k]);
            double X1 = -cl, X2 = cl + cr, X3 = -cr;
            out[k] = out[k] + (X1 * v[o->xa[q]] + X2 * v[k] + X3 * v[o->xb[q]]) / diag[k];
        }
}

/* Right-hand side b1 with the injection sources (src/fluid_diffusion.f90:44-64).
 * Sources are vector subscripts in the reference: when source s of a fault
 * is active, every source of that fault is added once more. */
static void orc_rhs_b1(const orc *o, double dt, const double *diag, double *b1)
{
    int64_t N = o->N;
    for (int64_t k = 0; k < N; k++) b1[k] = o->P[k] / diag[k];
    for (int64_t s = 0; s < o->nsrc; s++) {
        double t = o->time + dt;
        if (!(t >= o->src_tb[s] && t < o->src_te[s])) continue;
        int64_t f = o->src_fault[s] - 1;
        for (int64_t j = 0; j < o->nsrc; j++) {
            if (o->src_fault[j] != o->src_fault[s]) continue;
            int64_t e = o->fault_first[f] + o->src_index[j] - 1;
            b1[e] = b1[e] + (dt * o->src_Q[j] / (o->porosity * (o->fluid_comp + o->rock_comp)) / o->ds[e]) / diag[e];
        }
    }
}

/* compute_P: src/fluid_diffusion.f90:24-152. Returns ier. With stage != 0
 * (a pressure solve inside a right-hand-side evaluation) a solve that hits
 * the cap still writes its last iterate: the reference would go on with an
 * uninitialised P_temp there (undefined), this restatement and the GPU path
 * both use the last iterate and count the event. */
static int orc_compute_P_mode(orc *o, double dt, double *P_temp, double *P_dot, int stage);

int orc_compute_P(orc *o, double dt, double *P_temp, double *P_dot)
{
    return orc_compute_P_mode(o, dt, P_temp, P_dot, 0);
}

/* permeability_coupling = 1: permeability from the committed sigmaN and P,
 * and the face values (src/fluid_diffusion.f90:68-70, 74-75). The
 * reference updates them after compute_diag, so its Jacobi scaling uses the
 * previous call's faces; the scaling cancels from the solved system
 * (M x / d = b / d), and here the diagonal follows the updated faces. */
static void orc_perm_update(orc *o)
{
    int64_t N = o->N;
    for (int64_t k = 0; k < N; k++)
        o->perm[k] = (o->kstar[k] - o->kmin[k]) * exp(-(fabs(o->Y[2 * N + k] + o->P[k]) / fabs(o->Snk[k]))) + o->kmin[k];
    for (int64_t k = 1; k < N; k++) o->permx[k] = 2.0 * o->perm[k - 1] * o->perm[k] / (o->perm[k - 1] + o->perm[k]);
}

static int orc_compute_P_mode(orc *o, double dt, double *P_temp, double *P_dot, int stage)
{
    int64_t N = o->N;
    double *w = (double *)malloc(sizeof(double) * 7 * N);
    double *pk = w, *rk = w + N, *rk1 = w + 2 * N, *xk = w + 3 * N, *b1 = w + 4 * N, *diag = w + 5 * N,
           *Mp = w + 6 * N;
    int ier = 0;
    if (o->pcoup) orc_perm_update(o);
    orc_diag(o, dt, diag);
    orc_rhs_b1(o, dt, diag, b1);
    /* permeability_coupling == 0: permeability_x is recomputed from the
     * unchanged permeability (src/fluid_diffusion.f90:74-75) */
    for (int64_t k = 0; k < N; k++) xk[k] = o->P[k];
    orc_matvec(o, xk, dt, diag, Mp);
    for (int64_t k = 0; k < N; k++) { rk[k] = b1[k] - Mp[k]; pk[k] = rk[k]; }
    int64_t it = 0;
    double errmax = 0.0;
    for (int64_t k = 0; k < N; k++) errmax = fmax(errmax, fabs(rk[k] / 1.0));
    errmax = errmax / o->tol;
    while (errmax >= 1.0) {
        it++;
        orc_matvec(o, pk, dt, diag, Mp);
        double s_rr = 0.0, s_pAp = 0.0;
        for (int64_t k = 0; k < N; k++) s_rr = s_rr + rk[k] * rk[k];
        for (int64_t k = 0; k < N; k++) s_pAp = s_pAp + pk[k] * Mp[k];
        double alpha = s_rr / s_pAp;
        for (int64_t k = 0; k < N; k++) xk[k] = xk[k] + alpha * pk[k];
        for (int64_t k = 0; k < N; k++) rk1[k] = rk[k] - alpha * Mp[k];
        double s_r1 = 0.0;
        for (int64_t k = 0; k < N; k++) s_r1 = s_r1 + rk1[k] * rk1[k];
        double beta = s_r1 / s_rr;
        for (int64_t k = 0; k < N; k++) pk[k] = rk1[k] + beta * pk[k];
        for (int64_t k = 0; k < N; k++) rk[k] = rk1[k];
        if (it > 200) {
            ier = 1;
            o->cg_iters += it;
            if (stage) {
                o->stage_noconv++;
                for (int64_t k = 0; k < N; k++) {
                    P_dot[k] = (dt < 1e-9) ? 0.0 : (xk[k] - o->P[k]) / dt;
                    P_temp[k] = xk[k];
                }
            }
            free(w);
            return ier;
        }
        errmax = 0.0;
        for (int64_t k = 0; k < N; k++) errmax = fmax(errmax, fabs(rk[k] / 1.0));
        errmax = errmax / o->tol;
    }
    o->cg_iters += it;
    if (dt < 1e-9) for (int64_t k = 0; k < N; k++) P_dot[k] = 0.0;
    else for (int64_t k = 0; k < N; k++) P_dot[k] = (xk[k] - o->P[k]) / dt;
    double mx = 0.0;
    for (int64_t k = 0; k < N; k++) { P_temp[k] = xk[k]; mx = fmax(mx, fabs(P_temp[k])); }
    if (mx > DBL_MAX) ier = 1;
    free(w);
    return ier;
}

/* Exact solve of the same implicit step with the unscaled tridiagonal
 * system (Thomas algorithm); used by tests to check both CG and the GPU
 * tridiagonal solver. Not a reference routine. */
/* Exact tridiagonal solve of the same implicit step (networks without
 * fault crossings: a crossing couples rows outside the three diagonals). */
void orc_pressure_exact(orc *o, double dt, double *P_temp)
{
    int64_t N = o->N;
    if (o->pcoup) orc_perm_update(o);
    double *diag = (double *)malloc(8 * N), *b1 = (double *)malloc(8 * N);
    double *lo = (double *)malloc(8 * N), *di = (double *)malloc(8 * N), *up = (double *)malloc(8 * N);
    orc_diag(o, dt, diag);
    orc_rhs_b1(o, dt, diag, b1);
    double c = o->porosity * o->dyn_visc * (o->fluid_comp + o->rock_comp);
    const double *px = o->permx, *ds = o->ds;
    for (int64_t k = 0; k < N; k++) {
        b1[k] *= diag[k];
        double dsm = ds[k > 0 ? k - 1 : 0], dsp = ds[k < N - 1 ? k + 1 : N - 1];
        if (k == 0) { lo[k] = 0; di[k] = 1.0 + px[1] * dt / (c * ds[0] * ds[0]); up[k] = -px[1] * dt / (c * ds[0] * ds[0]); }
        else if (k == N - 1) { lo[k] = -px[k] * dt / (c * ds[k] * ds[k]); di[k] = 1.0 + px[k] * dt / (c * ds[k] * ds[k]); up[k] = 0; }
        else { lo[k] = -px[k] * dt / (c * dsm * dsm); di[k] = 1.0 + (px[k] + px[k + 1]) * dt / (c * ds[k] * ds[k]); up[k] = -px[k + 1] * dt / (c * dsp * dsp); }
    }
    for (int64_t k = 1; k < N; k++) {
        double m = lo[k] / di[k - 1];
        di[k] -= m * up[k - 1];
        b1[k] -= m * b1[k - 1];
    }
    P_temp[N - 1] = b1[N - 1] / di[N - 1];
    for (int64_t k = N - 2; k >= 0; k--) P_temp[k] = (b1[k] - up[k] * P_temp[k + 1]) / di[k];
    free(diag); free(b1); free(lo); free(di); free(up);
}

/* ---------------------------------------------------------------------- */
/* Friction RHS: src/friction/RateStateAgingModeII.f90:19-92 and
 * src/friction/RateStateAgingModeIII.f90:112-214. Returns compute_P's ier. */
int orc_rhs(orc *o, double dt, const double *Y1, double *Y1dot)
{
    int64_t N = o->N;
    double *Pt = (double *)malloc(8 * N);
    memset(Pt, 0, 8 * N);
    orc_kernel(o, Y1, o->SigmaT_dot, o->SigmaN_dot);
    int ier = orc_compute_P_mode(o, dt, Pt, o->Pdot, 1);
    o->rhs_evals++;
    const double *V = Y1, *psi = Y1 + N, *sig = Y1 + 2 * N;
    for (int64_t k = 0; k < N; k++) {
        double dsig = (o->mode == DFN_MODE_II) ? o->SigmaN_dot[k] + o->nload[k] : o->nload[k];
        Y1dot[2 * N + k] = dsig;
        double B = V[k] / (2.0 * o->V0[k]);
        double C = exp((o->f0[k] + o->b[k] * psi[k]) / o->a[k]);
        double D = 1.0 / (C * C) + B * B;
        D = 1.0 / sqrt(D);
        double num = o->sload[k] + o->SigmaT_dot[k] + (Y1dot[2 * N + k] + o->Pdot[k]) * o->a[k] * asinh(B * C) +
                     B * D * (sig[k] + Pt[k]) * o->b[k] * (o->V0[k] / o->Dc[k] * exp(-psi[k]) - fabs(V[k]) / o->Dc[k]);
        double den = o->mu / (2.0 * o->cs) - D * (sig[k] + Pt[k]) * o->a[k] / (2.0 * o->V0[k]);
        Y1dot[k] = num / den;
        Y1dot[N + k] = o->V0[k] / o->Dc[k] * exp(-psi[k]) - fabs(V[k]) / o->Dc[k];
    }
    for (int64_t k = 0; k < N; k++)
        if (o->fake[k]) { Y1dot[k] = 0.0; Y1dot[N + k] = 0.0; Y1dot[2 * N + k] = 0.0; }
    free(Pt);
    return ier;
}

/* ---------------------------------------------------------------------- */
/* Cash-Karp tableau and step control: src/ode_solver/ode_bs.f90:125-226. */
static const double A2 = 0.2, A3 = 0.3, A4 = 0.6, A5 = 1.0, A6 = 0.875;
static const double B21 = 0.2, B31 = 3.0 / 40.0, B32 = 9.0 / 40.0, B41 = 0.3, B42 = -0.9, B43 = 1.2;
static const double B51 = -11.0 / 54.0, B52 = 2.5, B53 = -70.0 / 27.0, B54 = 35.0 / 27.0;
static const double B61 = 1631.0 / 55296.0, B62 = 175.0 / 512.0, B63 = 575.0 / 13824.0,
                    B64 = 44275.0 / 110592.0, B65 = 253.0 / 4096.0;
static const double C1 = 37.0 / 378.0, C3 = 250.0 / 621.0, C4 = 125.0 / 594.0, C6 = 512.0 / 1771.0;
#define DC1 (C1 - 2825.0 / 27648.0)
#define DC3 (C3 - 18575.0 / 48384.0)
#define DC4 (C4 - 13525.0 / 55296.0)
#define DC5 (-277.0 / 14336.0)
#define DC6 (C6 - 0.25)

/* derivs callback: the friction RHS of the handle, or a user function. */
typedef void (*orc_derivs_fn)(double x, int64_t n, const double *y, double *dydx, void *ctx);

static void orc_rhs_cb(double x, int64_t n, const double *y, double *dydx, void *ctx)
{
    (void)n;
    orc_rhs((orc *)ctx, x, y, dydx);
}

/* rkck: src/ode_solver/ode_bs.f90:177-226 */
static void orc_rkck_cb(orc_derivs_fn derivs, void *ctx, const double *y, const double *dydx, int64_t n, double x,
                        double h, double *yout, double *yerr)
{
    double *w = (double *)malloc(sizeof(double) * 6 * n);
    double *ak2 = w, *ak3 = w + n, *ak4 = w + 2 * n, *ak5 = w + 3 * n, *ak6 = w + 4 * n, *yt = w + 5 * n;
    for (int64_t i = 0; i < n; i++) yt[i] = y[i] + B21 * h * dydx[i];
    derivs(x + A2 * h, n, yt, ak2, ctx);
    for (int64_t i = 0; i < n; i++) yt[i] = y[i] + h * (B31 * dydx[i] + B32 * ak2[i]);
    derivs(x + A3 * h, n, yt, ak3, ctx);
    for (int64_t i = 0; i < n; i++) yt[i] = y[i] + h * (B41 * dydx[i] + B42 * ak2[i] + B43 * ak3[i]);
    derivs(x + A4 * h, n, yt, ak4, ctx);
    for (int64_t i = 0; i < n; i++) yt[i] = y[i] + h * (B51 * dydx[i] + B52 * ak2[i] + B53 * ak3[i] + B54 * ak4[i]);
    derivs(x + A5 * h, n, yt, ak5, ctx);
    for (int64_t i = 0; i < n; i++)
        yt[i] = y[i] + h * (B61 * dydx[i] + B62 * ak2[i] + B63 * ak3[i] + B64 * ak4[i] + B65 * ak5[i]);
    derivs(x + A6 * h, n, yt, ak6, ctx);
    for (int64_t i = 0; i < n; i++) yout[i] = y[i] + h * (C1 * dydx[i] + C3 * ak3[i] + C4 * ak4[i] + C6 * ak6[i]);
    for (int64_t i = 0; i < n; i++)
        yerr[i] = h * (DC1 * dydx[i] + DC3 * ak3[i] + DC4 * ak4[i] + DC5 * ak5[i] + DC6 * ak6[i]);
    free(w);
}

/* rkqs: src/ode_solver/ode_bs.f90:125-174. Returns 0 or DFN_ERR_UNDERFLOW.
 * counters (attempts, rejected) may be NULL. The error norm runs over the
 * first nerr components (the others are integrated passively). */
static int orc_rkqs_nerr(orc_derivs_fn derivs, void *ctx, int64_t *counters, double *y, const double *dydx,
                         int64_t n, int64_t nerr, double *x, double htry, double eps, const double *yscal,
                         double *hdid, double *hnext);

int orc_rkqs_cb(orc_derivs_fn derivs, void *ctx, int64_t *counters, double *y, const double *dydx, int64_t n,
                double *x, double htry, double eps, const double *yscal, double *hdid, double *hnext)
{
    return orc_rkqs_nerr(derivs, ctx, counters, y, dydx, n, n, x, htry, eps, yscal, hdid, hnext);
}

static int orc_rkqs_nerr(orc_derivs_fn derivs, void *ctx, int64_t *counters, double *y, const double *dydx,
                         int64_t n, int64_t nerr, double *x, double htry, double eps, const double *yscal,
                         double *hdid, double *hnext)
{
    const double SAFETY = 0.9, PGROW = -0.2, PSHRNK = -0.25;
    const double ERRCON = (double)1.89e-4f; /* default-real literal in the reference */
    double *yerr = (double *)malloc(8 * n), *ytemp = (double *)malloc(8 * n);
    double h = htry, errmax;
    for (;;) {
        if (counters) counters[0]++;
        orc_rkck_cb(derivs, ctx, y, dydx, n, *x, h, ytemp, yerr);
        errmax = 0.0;
        for (int64_t i = 0; i < nerr; i++) errmax = fmax(errmax, fabs(yerr[i] / yscal[i]));
        errmax = errmax / eps;
        if (errmax <= 1.0) break;
        if (counters) counters[1]++;
        double htemp = SAFETY * h * pow(errmax, PSHRNK);
        h = copysign(fmax(fabs(htemp), 0.1 * fabs(h)), h);
        double xnew = *x + h;
        if (xnew == *x) { free(yerr); free(ytemp); return DFN_ERR_UNDERFLOW; }
    }
    if (errmax > ERRCON) *hnext = SAFETY * h * pow(errmax, PGROW);
    else *hnext = 5.0 * h;
    *hdid = h;
    *x = *x + h;
    for (int64_t i = 0; i < n; i++) y[i] = ytemp[i];
    free(yerr); free(ytemp);
    return 0;
}

int orc_rkqs(orc *o, double *y, const double *dydx, int64_t n, double *x, double htry, double eps,
             const double *yscal, double *hdid, double *hnext)
{
    int64_t c[2] = {0, 0};
    int st = orc_rkqs_cb(orc_rhs_cb, o, c, y, dydx, n, x, htry, eps, yscal, hdid, hnext);
    o->attempts += c[0];
    o->rejected += c[1];
    return st;
}

/* derivs of the V formulation with slip appended: [V psi sigma slip]' =
 * [friction RHS, V] (slip is passive: nothing reads it back). */
static void orc_rhs_slip_cb(double x, int64_t n, const double *y, double *dydx, void *ctx)
{
    orc *o = (orc *)ctx;
    int64_t N = o->N;
    (void)n;
    orc_rhs(o, x, y, dydx);
    for (int64_t k = 0; k < N; k++) dydx[3 * N + k] = y[k];
}

static int orc_newton_solve_step(orc *o);

/* ---------------------------------------------------------------------- */
/* One pass of the solve() loop: src/solver.f90:59-198 (printing and file
 * output excluded). Returns 0, or a dfn_status code. Slip rides along as a
 * fourth block outside the error norm. */
int orc_solve_step(orc *o)
{
    if (o->form == 1) return orc_newton_solve_step(o);
    int64_t N = o->N, n = 3 * N;
    o->it_count++;
    if (o->t_try > 10.0) {
        for (int64_t s = 0; s < o->nsrc; s++)
            if (o->time < o->src_tb[s] && o->time + o->t_try > o->src_tb[s]) o->t_try = 10.0;
    }
    double *Pt = (double *)malloc(8 * N);
    int ier = orc_compute_P(o, o->t_try, Pt, o->Pdot);
    int guard = 0;
    while (ier == 1) {
        o->t_try = o->t_try / 2.0;
        o->halvings++;
        ier = orc_compute_P(o, o->t_try, Pt, o->Pdot);
        if (++guard > 2000) { free(Pt); return DFN_ERR_NOCONV; }
    }
    double *y4 = (double *)malloc(8 * 4 * N), *Ydot = (double *)malloc(8 * 4 * N), *yscal = (double *)malloc(8 * n);
    memcpy(y4, o->Y, 8 * n);
    memcpy(y4 + n, o->slip, 8 * N);
    double time_temp = 0.0;
    orc_rhs_slip_cb(o->t_try, 4 * N, y4, Ydot, o);
    for (int64_t i = 0; i < n; i++) yscal[i] = fabs(o->Y[i]) + fabs(Ydot[i] * o->t_try) + o->tol;
    double t_did = 0, t_next = 0;
    int64_t c[2] = {0, 0};
    int st = orc_rkqs_nerr(orc_rhs_slip_cb, o, c, y4, Ydot, 4 * N, n, &time_temp, o->t_try, o->tol, yscal, &t_did,
                           &t_next);
    o->attempts += c[0];
    o->rejected += c[1];
    free(Ydot); free(yscal);
    if (st) { free(Pt); free(y4); return st; }
    memcpy(o->Y, y4, 8 * n);
    memcpy(o->slip, y4 + n, 8 * N);
    free(y4);
    o->t_try = t_next;
    if (o->t_try > o->max_step) o->t_try = o->max_step;
    ier = orc_compute_P(o, t_did, o->P, o->Pdot);
    free(Pt);
    o->time = o->time + t_did;
    for (int64_t k = 0; k < N; k++)
        if (o->Y[2 * N + k] > 0) return DFN_ERR_EXTENSIONAL;
    for (int64_t i = 0; i < n; i++)
        if (!isfinite(o->Y[i])) return DFN_ERR_NONFINITE;
    return 0;
}

int orc_solve_steps(orc *o, int64_t nsteps, double *hdid_log)
{
    for (int64_t s = 0; s < nsteps; s++) {
        double t0 = o->time;
        int st = orc_solve_step(o);
        if (hdid_log) hdid_log[s] = o->time - t0;
        if (st) { o->last_status = st; return st; }
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Newton slip formulation: the library's DFN_FORM_NEWTON restated. It has
 * no counterpart in the reference, which integrates V; the friction law it
 * solves is the reference's (src/friction/RateStateAgingModeII.f90:54-68,
 * whose time derivative is the reference's dV/dt):
 *   state Y = [slip | psi | sigmaN0]   (slip 0 and tau0 set at entry)
 *   tau   = tau0 + prefactor K_T.slip + shear_loading_dot (t - time0)
 *   sigma = sigmaN0 + prefactor K_N.slip + normal_loading_dot (t - time0)
 *           (mode III: no K_N term)
 *   g(w)  = tau - eta V(w) - s a w = 0,  s = -(sigma + P),
 *           V(w) = (2 V0/C) sinh w,  C = exp((f0 + b psi)/a),  eta = mu/(2 cs)
 * Newton on w from the bounded start (the friction-only root w0 = tau/(s a)
 * or the radiation-only root wr, eta V(wr) = tau, whichever is nearer
 * zero; guess 3 takes w0), steps limited to |dw| <= 10, converged when
 * |g| <= tol (|tau| + s a |w|); s <= 0: V = tau/eta. dslip/dt = V,
 * dpsi/dt = the aging law, dsigmaN0/dt = 0. The stage pressure is linear
 * in the stage time between the committed P (c = 0) and the implicit-Euler
 * pressure over the whole step (c = 1), which is what is committed. */
static const double ORC_LN2 = 0.6931471805599453;

static double orc_w_radiation(double tau, double eta, double lnA)
{
    double at = fabs(tau);
    if (at == 0.0) return 0.0;
    double lz = log(at / eta) - lnA;
    double wr = (lz > 20.0) ? lz + ORC_LN2 : asinh(exp(lz));
    return copysign(wr, tau);
}

static void orc_eta_v(double w, double lnA, double eta, double *ev, double *edv)
{
    double aw = fabs(w);
    double e = exp(lnA + aw - ORC_LN2);
    double q = exp(-2.0 * aw);
    *ev = eta * copysign(e * (1.0 - q), w);
    *edv = eta * e * (1.0 + q);
}

static double orc_v_of_w(double w, double lnA)
{
    double aw = fabs(w);
    return copysign(exp(lnA + aw - ORC_LN2) * (1.0 - exp(-2.0 * aw)), w);
}

static double orc_newton_w(double tau, double s, double a, double lnA, double eta, double w, double tol, int maxit,
                           int *iters, int *ok)
{
    *iters = 0;
    *ok = 0;
    for (int it = 0; it <= maxit; it++) {
        double ev, edv;
        orc_eta_v(w, lnA, eta, &ev, &edv);
        double g = tau - ev - s * a * w;
        if (fabs(g) <= tol * (fabs(tau) + s * a * fabs(w) + 1e-300)) { *ok = 1; break; }
        if (it == maxit) break;
        double dw = g / (edv + s * a);
        dw = fmax(fmin(dw, 10.0), -10.0);
        w += dw;
        (*iters)++;
    }
    return w;
}

/* Switches the formulation (0: V, the reference's; 1: Newton). Newton:
 * tau0 such that the current V satisfies the friction law at slip 0 with
 * the committed P, then slip = 0. guess 0 bounded start, 3 friction-only
 * start; maxit 0 = 50, tol 0 = 1e-13. */
int orc_set_formulation(orc *o, int form, int guess, int maxit, double tol)
{
    if (form != 0 && form != 1) return DFN_ERR_ARG;
    if (guess != 0 && guess != 3) return DFN_ERR_UNSUPPORTED;
    o->form = form;
    o->nguess = guess;
    o->nmaxit = maxit > 0 ? maxit : 50;
    o->ntol = tol > 0.0 ? tol : 1e-13;
    if (form == 0) return 0;
    int64_t N = o->N;
    double eta = o->mu / (2.0 * o->cs);
    for (int64_t k = 0; k < N; k++) {
        double V = o->Y[k], psi = o->Y[N + k], sig = o->Y[2 * N + k];
        double t0 = 0.0;
        if (!o->fake[k]) {
            double C = exp((o->f0[k] + o->b[k] * psi) / o->a[k]);
            double w = asinh(V * C / (2.0 * o->V0[k]));
            t0 = eta * V - (sig + o->P[k]) * o->a[k] * w;
        }
        o->tau0[k] = t0;
        o->Y[k] = 0.0;
    }
    o->time0 = o->time;
    return 0;
}

/* Right-hand side of the Newton formulation at offset `off` from the step
 * start with the stage pressure Pt; V of the evaluation into Vout (may be
 * NULL). */
static void orc_newton_rhs(orc *o, double off, const double *Pt, const double *Y, double *Yd, double *Vout)
{
    int64_t N = o->N;
    orc_kernel(o, Y, o->SigmaT_dot, o->SigmaN_dot);
    o->rhs_evals++;
    double eta = o->mu / (2.0 * o->cs);
    double tt = (o->time - o->time0) + off;
    const double *psi = Y + N, *sig0 = Y + 2 * N;
    for (int64_t k = 0; k < N; k++) {
        Yd[2 * N + k] = 0.0;
        if (o->fake[k]) { Yd[k] = 0.0; Yd[N + k] = 0.0; if (Vout) Vout[k] = 0.0; continue; }
        double tau = o->tau0[k] + o->SigmaT_dot[k] + o->sload[k] * tt;
        double sig = ((o->mode == DFN_MODE_II) ? sig0[k] + o->SigmaN_dot[k] : sig0[k]) + o->nload[k] * tt;
        double s = -(sig + Pt[k]);
        double a = o->a[k], V;
        if (s > 0.0) {
            double lnA = log(2.0 * o->V0[k]) - (o->f0[k] + o->b[k] * psi[k]) / a;
            double w0 = tau / (s * a);
            double wr = orc_w_radiation(tau, eta, lnA);
            double w = (o->nguess != 3 && fabs(wr) < fabs(w0)) ? wr : w0;
            int it, ok;
            w = orc_newton_w(tau, s, a, lnA, eta, w, o->ntol, o->nmaxit, &it, &ok);
            o->newton_solves++;
            o->newton_iters += it;
            if (!ok) o->newton_fail++;
            V = orc_v_of_w(w, lnA);
        } else {
            V = tau / eta;
        }
        if (Vout) Vout[k] = V;
        Yd[k] = V;
        Yd[N + k] = o->V0[k] / o->Dc[k] * exp(-psi[k]) - fabs(V) / o->Dc[k];
    }
}

/* One pass of solve() in the Newton formulation: the V formulation's loop
 * (probe with halving, scaling right-hand side, rkqs, 1-day cap, pressure
 * commit, time, stop rules), with the stage pressures above. */
static int orc_newton_solve_step(orc *o)
{
    static const double A[7] = {0.0, 0.0, 0.2, 0.3, 0.6, 1.0, 0.875};
    const double SAFETY = 0.9, PGROW = -0.2, PSHRNK = -0.25;
    const double ERRCON = (double)1.89e-4f;
    int64_t N = o->N, n = 3 * N;
    o->it_count++;
    if (o->t_try > 10.0) {
        for (int64_t s = 0; s < o->nsrc; s++)
            if (o->time < o->src_tb[s] && o->time + o->t_try > o->src_tb[s]) o->t_try = 10.0;
    }
    double *w = (double *)malloc(8 * (13 * n + 3 * N));
    double *k1 = w, *k2 = w + n, *k3 = w + 2 * n, *k4 = w + 3 * n, *k5 = w + 4 * n, *k6 = w + 5 * n;
    double *yt = w + 6 * n, *yout = w + 7 * n, *yscal = w + 8 * n, *yerr = w + 9 * n;
    double *Pfull = w + 13 * n, *Pdf = Pfull + N, *Pst = Pdf + N;
    double **ks[7] = {NULL, NULL, &k2, &k3, &k4, &k5, &k6};
    /* the probe: src/solver.f90:81-92 (its solution is not used here) */
    int ier = orc_compute_P(o, o->t_try, Pst, Pdf);
    int guard = 0;
    while (ier == 1) {
        o->t_try = o->t_try / 2.0;
        o->halvings++;
        ier = orc_compute_P(o, o->t_try, Pst, Pdf);
        if (++guard > 2000) { free(w); return DFN_ERR_NOCONV; }
    }
    orc_newton_rhs(o, 0.0, o->P, o->Y, k1, NULL);
    for (int64_t i = 0; i < n; i++) yscal[i] = fabs(o->Y[i]) + fabs(k1[i] * o->t_try) + o->tol;
    double h = o->t_try, errmax, hnext;
    int ier_full;
    for (;;) {
        o->attempts++;
        ier_full = orc_compute_P_mode(o, 0.0 + A[5] * h, Pfull, Pdf, 1);
        const double *y = o->Y;
        for (int st = 2; st <= 6; st++) {
            for (int64_t i = 0; i < n; i++) {
                switch (st) {
                case 2: yt[i] = y[i] + 0.2 * h * k1[i]; break;
                case 3: yt[i] = y[i] + h * (B31 * k1[i] + B32 * k2[i]); break;
                case 4: yt[i] = y[i] + h * (B41 * k1[i] + B42 * k2[i] + B43 * k3[i]); break;
                case 5: yt[i] = y[i] + h * (B51 * k1[i] + B52 * k2[i] + B53 * k3[i] + B54 * k4[i]); break;
                default:
                    yt[i] = y[i] + h * (B61 * k1[i] + B62 * k2[i] + B63 * k3[i] + B64 * k4[i] + B65 * k5[i]);
                }
            }
            for (int64_t k = 0; k < N; k++) Pst[k] = o->P[k] + A[st] * (Pfull[k] - o->P[k]);
            orc_newton_rhs(o, 0.0 + A[st] * h, Pst, yt, *ks[st], NULL);
        }
        for (int64_t i = 0; i < n; i++) yout[i] = y[i] + h * (C1 * k1[i] + C3 * k3[i] + C4 * k4[i] + C6 * k6[i]);
        for (int64_t i = 0; i < n; i++)
            yerr[i] = h * (DC1 * k1[i] + DC3 * k3[i] + DC4 * k4[i] + DC5 * k5[i] + DC6 * k6[i]);
        errmax = 0.0;
        for (int64_t i = 0; i < n; i++) errmax = fmax(errmax, fabs(yerr[i] / yscal[i]));
        errmax = errmax / o->tol;
        if (errmax <= 1.0) break;
        o->rejected++;
        double htemp = SAFETY * h * pow(errmax, PSHRNK);
        h = copysign(fmax(fabs(htemp), 0.1 * fabs(h)), h);
        if (0.0 + h == 0.0) { free(w); return DFN_ERR_UNDERFLOW; }
    }
    hnext = (errmax > ERRCON) ? SAFETY * h * pow(errmax, PGROW) : 5.0 * h;
    memcpy(o->Y, yout, 8 * n);
    o->t_try = hnext;
    if (o->t_try > o->max_step) o->t_try = o->max_step;
    /* the commit compute_P(t_did) is the full-step solve of the accepted
     * attempt; a capped solve keeps P, as the reference's early return */
    if (ier_full == 0) {
        memcpy(o->Pdot, Pdf, 8 * N);
        memcpy(o->P, Pfull, 8 * N);
    }
    o->time = o->time + h;
    free(w);
    for (int64_t k = 0; k < N; k++)
        if (o->Y[2 * N + k] > 0) return DFN_ERR_EXTENSIONAL;
    for (int64_t i = 0; i < n; i++)
        if (!isfinite(o->Y[i])) return DFN_ERR_NONFINITE;
    return 0;
}

/* Slip rate at the current state (Newton: the friction law solved with the
 * committed P; V formulation: the state itself). */
void orc_velocity(orc *o, double *V)
{
    int64_t N = o->N;
    if (o->form != 1) { memcpy(V, o->Y, 8 * N); return; }
    double *Yd = (double *)malloc(8 * 3 * N);
    int64_t c[4] = {o->rhs_evals, o->newton_solves, o->newton_iters, o->newton_fail};
    orc_newton_rhs(o, 0.0, o->P, o->Y, Yd, V);
    o->rhs_evals = c[0]; o->newton_solves = c[1]; o->newton_iters = c[2]; o->newton_fail = c[3];
    free(Yd);
}

/* Slip (V formulation: the passive integral of V; Newton: the state). */
void orc_get_slip(const orc *o, double *slip)
{
    memcpy(slip, o->form == 1 ? o->Y : o->slip, 8 * o->N);
}
void orc_set_slip(orc *o, const double *slip)
{
    memcpy(o->form == 1 ? o->Y : o->slip, slip, 8 * o->N);
}
void orc_newton_counters(const orc *o, int64_t *c)
{
    c[0] = o->newton_solves; c[1] = o->newton_iters; c[2] = o->newton_fail;
}

/* ---------------------------------------------------------------------- */
/* Accessors */
/* ---------------------------------------------------------------------- */
/* H-matrix (static_kernel = hmatrix): the src/hmatrix/ sources.           */

typedef struct { int first, last, son1, son2; } orc_clus;
typedef struct { int r0, nr, c0, nc, dense, rank; double *A, *B, *F; } orc_leaf;

struct orc_hmat {
    int N, ncl, nleaf_blocks, cap;
    int *perm;              /* mat_corr: perm[pos] = element */
    orc_clus *cl;
    orc_leaf *lv[2];        /* per component (T, N) */
    int nlv;
    int failed;             /* an ACA needed more than 20 terms (the reference STOPs) */
};
typedef struct orc_hmat orc_hmat;

/* cluster_tree.f90: bisection of the bounding box along its longer side
 * (ties: second coordinate), points >= midpoint form one son, order kept,
 * the son holding the smallest current position placed first. */
static void orc_split(double *x, double *y, int *perm, int first, int last, int nleaf, orc_hmat *H)
{
    int me = H->ncl++;
    H->cl[me].first = first; H->cl[me].last = last; H->cl[me].son1 = -1; H->cl[me].son2 = -1;
    if (last - first + 1 <= nleaf) return;
    double bx0 = x[first], bx1 = x[first], by0 = y[first], by1 = y[first];
    for (int i = first; i <= last; i++) {
        bx0 = fmin(bx0, x[i]); bx1 = fmax(bx1, x[i]); by0 = fmin(by0, y[i]); by1 = fmax(by1, y[i]);
    }
    double box[2] = {bx1 - bx0, by1 - by0};
    int dir = 0;
    for (int d = 0; d < 2; d++) if (box[d] >= box[dir]) dir = d;
    const double *c = dir == 0 ? x : y;
    double lo = dir == 0 ? bx0 : by0, hi = dir == 0 ? bx1 : by1;
    double mid = lo + (hi - lo) / 2;
    int n = last - first + 1, n1 = 0, n2 = 0;
    int *s1 = (int *)malloc(sizeof(int) * n), *s2 = (int *)malloc(sizeof(int) * n);
    for (int i = first; i <= last; i++) { if (c[i] >= mid) s1[n1++] = i; else s2[n2++] = i; }
    if (n1 == 0 || n2 == 0) { free(s1); free(s2); return; }
    int *A = s1[0] <= s2[0] ? s1 : s2, *B = s1[0] <= s2[0] ? s2 : s1;
    int nA = s1[0] <= s2[0] ? n1 : n2, nB = n - nA;
    double *nx = (double *)malloc(8 * n), *ny = (double *)malloc(8 * n);
    int *np = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < nA; i++) { nx[i] = x[A[i]]; ny[i] = y[A[i]]; np[i] = perm[A[i]]; }
    for (int i = 0; i < nB; i++) { nx[nA + i] = x[B[i]]; ny[nA + i] = y[B[i]]; np[nA + i] = perm[B[i]]; }
    for (int i = 0; i < n; i++) { x[first + i] = nx[i]; y[first + i] = ny[i]; perm[first + i] = np[i]; }
    free(nx); free(ny); free(np); free(s1); free(s2);
    int a = H->ncl;
    orc_split(x, y, perm, first, first + nA - 1, nleaf, H);
    int b = H->ncl;
    orc_split(x, y, perm, first + nA, last, nleaf, H);
    H->cl[me].son1 = a; H->cl[me].son2 = b;
}

static void orc_bbox(const orc *o, const orc_hmat *H, int k, double *b)
{
    b[0] = 1e300; b[1] = -1e300; b[2] = 1e300; b[3] = -1e300;
    for (int p = H->cl[k].first; p <= H->cl[k].last; p++) {
        int e = H->perm[p];
        b[0] = fmin(b[0], o->elem[2 * e]); b[1] = fmax(b[1], o->elem[2 * e]);
        b[2] = fmin(b[2], o->elem[2 * e + 1]); b[3] = fmax(b[3], o->elem[2 * e + 1]);
    }
}

/* block_cluster_tree.f90:342-476 (admissibility eta*dist >= max(diam)) */
static void orc_blocks(const orc *o, orc_hmat *H, double eta, int r, int c)
{
    double R[4], C[4];
    orc_bbox(o, H, r, R);
    orc_bbox(o, H, c, C);
    double dr = sqrt((R[1] - R[0]) * (R[1] - R[0]) + (R[3] - R[2]) * (R[3] - R[2]));
    double dc = sqrt((C[1] - C[0]) * (C[1] - C[0]) + (C[3] - C[2]) * (C[3] - C[2]));
    double d = 0.0;
    d = d + pow(fmax(0.0, R[0] - C[1]), 2) + pow(fmax(0.0, C[0] - R[1]), 2);
    d = d + pow(fmax(0.0, R[2] - C[3]), 2) + pow(fmax(0.0, C[2] - R[3]), 2);
    d = sqrt(d);
    orc_clus cr = H->cl[r], cc = H->cl[c];
    int dense;
    if (eta * d >= fmax(dr, dc)) dense = 0;
    else if (cr.son1 >= 0 && cc.son1 >= 0) {
        orc_blocks(o, H, eta, cr.son1, cc.son1); orc_blocks(o, H, eta, cr.son1, cc.son2);
        orc_blocks(o, H, eta, cr.son2, cc.son1); orc_blocks(o, H, eta, cr.son2, cc.son2);
        return;
    } else dense = 1;
    if (H->nlv == H->cap) {
        H->cap *= 2;
        H->lv[0] = (orc_leaf *)realloc(H->lv[0], sizeof(orc_leaf) * H->cap);
        H->lv[1] = (orc_leaf *)realloc(H->lv[1], sizeof(orc_leaf) * H->cap);
    }
    for (int q = 0; q < 2; q++) {
        orc_leaf *L = &H->lv[q][H->nlv];
        memset(L, 0, sizeof(*L));
        L->r0 = cr.first; L->nr = cr.last - cr.first + 1; L->c0 = cc.first; L->nc = cc.last - cc.first + 1;
        L->dense = dense;
    }
    H->nlv++;
}

/* compute_full_ACA: src/hmatrix/ACA_algorithm.f90:665-826, on the fully
 * evaluated block; pivot = first maximum of |R| in column-major order,
 * stop when |pivot| <= 10.0**(-14) (a default-real literal) or
 * ||R||_F <= eps*||A||_F; more than 20 terms is the reference's STOP. */
static int orc_full_aca(int m, int n, double *R, double eps, int maxr, double *A, double *B)
{
    double nA = 0.0;
    for (int64_t q = 0; q < (int64_t)m * n; q++) nA += R[q] * R[q];
    nA = sqrt(nA);
    int rank = 0;
    for (int k = 1; k <= (m < n ? m : n); k++) {
        if (k > maxr) return -1;
        int pi = 0, pj = 0;
        double best = -1.0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) {
                double v = fabs(R[(int64_t)j * m + i]);
                if (v > best) { best = v; pi = i; pj = j; }
            }
        if (best <= (double)1e-14f) return k - 1;
        double piv = R[(int64_t)pj * m + pi];
        for (int i = 0; i < m; i++) A[(int64_t)(k - 1) * m + i] = R[(int64_t)pj * m + i];
        for (int j = 0; j < n; j++) B[(int64_t)(k - 1) * n + j] = R[(int64_t)j * m + pi] / piv;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++)
                R[(int64_t)j * m + i] = R[(int64_t)j * m + i] - A[(int64_t)(k - 1) * m + i] * B[(int64_t)(k - 1) * n + j];
        double nR = 0.0;
        for (int64_t q = 0; q < (int64_t)m * n; q++) nR += R[q] * R[q];
        nR = sqrt(nR);
        rank = k;
        if (nR <= eps * nA) return k;
    }
    return rank;
}

static void orc_hmat_free(orc_hmat *H)
{
    if (!H) return;
    for (int q = 0; q < 2; q++) {
        if (!H->lv[q]) continue;
        for (int b = 0; b < H->nlv; b++) { free(H->lv[q][b].A); free(H->lv[q][b].B); free(H->lv[q][b].F); }
        free(H->lv[q]);
    }
    free(H->perm); free(H->cl); free(H);
}

/* initiate_hmat: src/hmatrix/initialisation_hmat.f90:13-100 (no
 * recompression: it only lowers the ranks, within eps). Returns 0, or -1
 * when an ACA needed more than 20 terms. */
int orc_hmat_build(orc *o, int nleaf, double eta, double eps)
{
    int N = (int)o->N;
    orc_hmat *H = (orc_hmat *)calloc(1, sizeof(orc_hmat));
    H->N = N;
    H->perm = (int *)malloc(sizeof(int) * N);
    H->cl = (orc_clus *)malloc(sizeof(orc_clus) * 2 * N);
    double *x = (double *)malloc(8 * N), *y = (double *)malloc(8 * N);
    for (int i = 0; i < N; i++) { x[i] = o->elem[2 * i]; y[i] = o->elem[2 * i + 1]; H->perm[i] = i; }
    orc_split(x, y, H->perm, 0, N - 1, nleaf, H);
    free(x); free(y);
    H->cap = 64;
    H->lv[0] = (orc_leaf *)malloc(sizeof(orc_leaf) * H->cap);
    H->lv[1] = (orc_leaf *)malloc(sizeof(orc_leaf) * H->cap);
    orc_blocks(o, H, eta, 0, 0);
    int ncomp = o->mode == DFN_MODE_II ? 2 : 1;
    for (int q = 0; q < ncomp; q++) {
        int which = o->mode == DFN_MODE_II ? 1 + q : 0;
        for (int b = 0; b < H->nlv; b++) {
            orc_leaf *L = &H->lv[q][b];
            double *R = (double *)malloc(sizeof(double) * (size_t)L->nr * L->nc);
            for (int j = 0; j < L->nc; j++)
                for (int i = 0; i < L->nr; i++)
                    R[(int64_t)j * L->nr + i] = orc_kernel_entry(o, H->perm[L->r0 + i], H->perm[L->c0 + j], which);
            if (L->dense) { L->F = R; continue; }
            L->A = (double *)malloc(sizeof(double) * (size_t)L->nr * 20);
            L->B = (double *)malloc(sizeof(double) * (size_t)L->nc * 20);
            double *Rc = (double *)malloc(sizeof(double) * (size_t)L->nr * L->nc);
            memcpy(Rc, R, sizeof(double) * (size_t)L->nr * L->nc);
            int r = orc_full_aca(L->nr, L->nc, Rc, eps, 20, L->A, L->B);
            free(Rc);
            if (r < 0) { H->failed = 1; L->dense = 1; L->F = R; continue; }
            L->rank = r;
            free(R);
        }
    }
    orc_hmat_free((orc_hmat *)o->hmat);
    o->hmat = H;
    o->kernel_impl = 2;
    return H->failed ? -1 : 0;
}

/* hmatII/hmatIII + Hgemv_right: y_perm = H x_perm, then back to element
 * order and the prefactor (src/kernel_calculation/hmatrixModeII.f90:46-69). */
static void orc_hmat_kv(const orc *o, const double *slip, double *sT, double *sN)
{
    const orc_hmat *H = (const orc_hmat *)o->hmat;
    int N = H->N, ncomp = o->mode == DFN_MODE_II ? 2 : 1;
    double *x = (double *)malloc(8 * N), *y = (double *)malloc(8 * N), *z = (double *)malloc(8 * 64);
    for (int p = 0; p < N; p++) x[p] = slip[H->perm[p]];
    for (int q = 0; q < ncomp; q++) {
        for (int p = 0; p < N; p++) y[p] = 0.0;
        for (int b = 0; b < H->nlv; b++) {
            const orc_leaf *L = &H->lv[q][b];
            if (L->dense) {
                for (int i = 0; i < L->nr; i++) {
                    double s = 0.0;
                    for (int j = 0; j < L->nc; j++) s += L->F[(int64_t)j * L->nr + i] * x[L->c0 + j];
                    y[L->r0 + i] += s;
                }
            } else {
                for (int k = 0; k < L->rank; k++) {
                    double s = 0.0;
                    for (int j = 0; j < L->nc; j++) s += L->B[(int64_t)k * L->nc + j] * x[L->c0 + j];
                    z[k] = s;
                }
                for (int i = 0; i < L->nr; i++) {
                    double s = 0.0;
                    for (int k = 0; k < L->rank; k++) s += L->A[(int64_t)k * L->nr + i] * z[k];
                    y[L->r0 + i] += s;
                }
            }
        }
        double *out = q == 0 ? sT : sN;
        double pref = o->mode == DFN_MODE_II ? o->mu / PI_F90 * (1.0 - o->cs * o->cs / (o->cp * o->cp))
                                             : o->mu / (2.0 * PI_F90);
        for (int p = 0; p < N; p++) out[H->perm[p]] = pref * y[p];
    }
    if (ncomp == 1 && sN) memset(sN, 0, 8 * N);
    free(x); free(y); free(z);
}

void orc_hmat_perm(const orc *o, int *perm)
{
    const orc_hmat *H = (const orc_hmat *)o->hmat;
    if (H) memcpy(perm, H->perm, sizeof(int) * H->N);
}

void orc_hmat_stats(const orc *o, int64_t *st)
{
    const orc_hmat *H = (const orc_hmat *)o->hmat;
    st[0] = st[1] = st[2] = st[3] = 0;
    if (!H) return;
    st[0] = H->nlv;
    for (int b = 0; b < H->nlv; b++) {
        if (H->lv[0][b].dense) st[1]++;
        else if (H->lv[0][b].rank > st[2]) st[2] = H->lv[0][b].rank;
    }
    st[3] = H->ncl;
}

void orc_get_state(const orc *o, double *Y, double *P, double *scal)
{
    if (Y) memcpy(Y, o->Y, 8 * 3 * o->N);
    if (P) memcpy(P, o->P, 8 * o->N);
    if (scal) { scal[0] = o->time; scal[1] = o->t_try; scal[2] = (double)o->it_count; }
}
void orc_set_state(orc *o, const double *Y, const double *P, double time, double t_try, int64_t it)
{
    if (Y) memcpy(o->Y, Y, 8 * 3 * o->N);
    if (P) memcpy(o->P, P, 8 * o->N);
    o->time = time; o->t_try = t_try; o->it_count = it;
}
void orc_get_geometry(const orc *o, double *elem, double *ds, double *tan, double *nrm, double *permx)
{
    int64_t N = o->N;
    if (elem) memcpy(elem, o->elem, 16 * N);
    if (ds) memcpy(ds, o->ds, 8 * N);
    if (tan) memcpy(tan, o->tan, 16 * N);
    if (nrm) memcpy(nrm, o->nrm, 16 * N);
    if (permx) memcpy(permx, o->permx, 8 * (N + 1));
}
/* Current permeability (the last solve's, with the coupling). */
void orc_get_permeability(const orc *o, double *perm) { memcpy(perm, o->perm, 8 * o->N); }
void orc_get_loads(const orc *o, double *nload, double *sload, unsigned char *fake)
{
    if (nload) memcpy(nload, o->nload, 8 * o->N);
    if (sload) memcpy(sload, o->sload, 8 * o->N);
    if (fake) memcpy(fake, o->fake, o->N);
}
void orc_get_last_stress(const orc *o, double *sT, double *sN, double *Pdot)
{
    if (sT) memcpy(sT, o->SigmaT_dot, 8 * o->N);
    if (sN) memcpy(sN, o->SigmaN_dot, 8 * o->N);
    if (Pdot) memcpy(Pdot, o->Pdot, 8 * o->N);
}
void orc_counters(const orc *o, int64_t *c)
{
    c[0] = o->cg_iters; c[1] = o->rhs_evals; c[2] = o->attempts; c[3] = o->rejected; c[4] = o->halvings;
    c[5] = o->it_count; c[6] = o->stage_noconv;
}
