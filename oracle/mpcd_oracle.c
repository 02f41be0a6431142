/*
 * mpcd_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C, serial, FP64
 * restatement of the reference's solvent timestep (NIAMH-MPCD,
 * mpcd/subroutines/mpc.c:4496-4954 and the helpers it calls), used by the
 * tests, smoke() and the benchmark's CPU baseline as the checker for the GPU
 * library.  The product never links or calls this file.
 *
 * Random numbers come from niamh-mpcd_b200/csrc/mpcd_rng.h keyed by
 * (seed, replica, step, stream, cell or particle id), the same values the GPU
 * uses and the reference harness (oracle/ref/ref_harness.c) injects into the
 * reference, so all three consume identical draws.
 *
 * Stage order follows timestep() for the paths without MD, swimmers,
 * thermostats or moving walls:
 *   grid shift        ranshift + gridShift_all     mpc.c:4567-4575, 720-766
 *   bin (shifted)     bin(...,1)                   mpc.c:4596, 948-992
 *   acceleration      acc_all                      mpc.c:4621, 697-700
 *   cell moments      localPROP                    mpc.c:4630, 64-216
 *   phantom particles ghostPart                    mpc.c:4634, 351-567
 *   nematic           LCcollision, jefferysTorque  mpc.c:4640-4678
 *   collision         MPCcollision per cell        mpc.c:4699-4714
 *   globals           avVel, TEMP                  mpc.c:4738-4752
 *   shift back        gridShift_all(...,1)         mpc.c:4793-4799
 *   stream            stream_all                   mpc.c:4815-4817
 *   walls             MPC_BCcollision              mpc.c:4834, bc.c:1363
 *   re-bin            bin(...,0) + localPROP       mpc.c:4936-4942
 * Within a cell, particles are visited in ascending particle index; the
 * reference visits them in linked-list order, so sums differ only by
 * rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mpcd_gpu.h"
#include "mpcd_rng.h"
#include "mpcd_oracle.h"

#define TOL 1e-8    /* definitions.h:56 */
#define NBOUNCE 50  /* definitions.h:62 */
#define MPCD_PI 3.14159265358979323846 /* pi = MPCD_PI, definitions.h:72 */

struct oracle {
    mpcd_config cfg;
    int dim, n;
    int L[3], N1[3], ncells;
    int pbc[3];
    double vol, gndnst;
    double *Q, *V, *U, *T;
    int *spid;
    int *key, *start, *list, *cnt;
    int *pop;
    double *mass, *vcm, *cm, *I, *S, *dir, *E;
    double wallQ[MPCD_MAX_WALLS][3];
    double avnow[3], kbtnow;
    long escaped, bounce_limit;
    int vdist[MPCD_MAX_SPECIES];  /* VDIST per species, for re-thermalisation */
    uint32_t step;                /* the step being taken                     */
};

/* ------------------------------------------------------------ small math */
static double dot3(const double *a, const double *b, int n) {
    double r = 0.0;
    for (int i = 0; i < n; i++) r += a[i] * b[i];
    return r;
}
static void cross3(const double *x, const double *y, double *r) {
    r[0] = x[1] * y[2] - x[2] * y[1];
    r[1] = x[2] * y[0] - x[0] * y[2];
    r[2] = x[0] * y[1] - x[1] * y[0];
}
/* inverse of a 3x3 matrix through its adjugate and determinant (the
 * method of invert3x3, mtools.c:1031-1038) */
static void inv3(const double m[9], double r[9]) {
    double c00 = m[4] * m[8] - m[5] * m[7];
    double c01 = m[3] * m[8] - m[5] * m[6];
    double c02 = m[3] * m[7] - m[4] * m[6];
    double det = m[0] * c00 - m[1] * c01 + m[2] * c02;
    double c10 = m[1] * m[8] - m[2] * m[7];
    double c11 = m[0] * m[8] - m[2] * m[6];
    double c12 = m[0] * m[7] - m[1] * m[6];
    double c20 = m[1] * m[5] - m[2] * m[4];
    double c21 = m[0] * m[5] - m[2] * m[3];
    double c22 = m[0] * m[4] - m[1] * m[3];
    /* r[j][i] = (-1)^(i+j) minor(i,j) / det */
    r[0] = c00 / det;
    r[3] = -c01 / det;
    r[6] = c02 / det;
    r[1] = -c10 / det;
    r[4] = c11 / det;
    r[7] = -c12 / det;
    r[2] = c20 / det;
    r[5] = -c21 / det;
    r[8] = c22 / det;
}

static int cell_index(const oracle_t *o, int a, int b, int c) {
    return (a * o->N1[1] + b) * o->N1[2] + c;
}

static double wall_W(const oracle_t *o, int w, const double *q) {
    /* calcW_PLANE, bc.c:306-316 */
    const mpcd_wall *wl = &o->cfg.walls[w];
    double W = 0.0;
    for (int i = 0; i < o->dim; i++) W += wl->A[i] * (q[i] - o->wallQ[w][i]);
    W -= wl->R;
    if (wl->inv) W *= -1.0;
    return W;
}

/* ----------------------------------------------------------- create/free */
void oracle_destroy(oracle_t *o) {
    if (!o) return;
    free(o->Q);
    free(o->V);
    free(o->U);
    free(o->T);
    free(o->spid);
    free(o->key);
    free(o->start);
    free(o->list);
    free(o->cnt);
    free(o->pop);
    free(o->mass);
    free(o->vcm);
    free(o->cm);
    free(o->I);
    free(o->S);
    free(o->dir);
    free(o->E);
    free(o);
}

static void bin_cells(oracle_t *o, int shifted);
static void local_prop(oracle_t *o);
static void vel_grad_2d(oracle_t *o);
static void order_param_2d(oracle_t *o, int c);

oracle_t *oracle_create(const mpcd_config *cfg, int n, const double *Q,
                        const double *V, const double *U, const int *spid) {
    oracle_t *o = (oracle_t *)calloc(1, sizeof(oracle_t));
    if (!o) return NULL;
    o->cfg = *cfg;
    o->dim = cfg->dim;
    o->n = n;
    for (int d = 0; d < 3; d++) {
        o->L[d] = d < o->dim ? cfg->L[d] : 1;
        o->N1[d] = o->L[d] + 1; /* (L+1)^D grid, read.c:1053 */
    }
    o->ncells = o->N1[0] * o->N1[1] * o->N1[2];
    o->vol = 1.0;
    for (int d = 0; d < o->dim; d++) o->vol *= o->L[d];
    /* periodic axes as setPBC (read.c:584-603) */
    for (int w = 0; w < cfg->n_walls; w++) {
        const mpcd_wall *wl = &cfg->walls[w];
        for (int d = 0; d < 3; d++) {
            o->wallQ[w][d] = wl->Q[d];
            if (fabs(fabs(wl->A[d]) - 1.0) <= TOL && wl->MVN > 0.0 &&
                wl->MVT > 0.0 && (fabs(wl->DN) >= TOL || fabs(wl->DT) >= TOL))
                o->pbc[d] = 1;
        }
    }
    size_t n3 = (size_t)3 * (size_t)(n > 0 ? n : 1);
    o->Q = (double *)malloc(n3 * sizeof(double));
    o->V = (double *)malloc(n3 * sizeof(double));
    o->U = (double *)calloc(n3, sizeof(double));
    o->T = (double *)calloc(n3, sizeof(double));
    o->spid = (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int));
    o->key = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    o->list = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    o->start = (int *)malloc((size_t)(o->ncells + 1) * sizeof(int));
    o->cnt = (int *)malloc((size_t)o->ncells * sizeof(int));
    o->pop = (int *)calloc((size_t)o->ncells, sizeof(int));
    o->mass = (double *)calloc((size_t)o->ncells, sizeof(double));
    o->vcm = (double *)calloc((size_t)o->ncells * 3, sizeof(double));
    o->cm = (double *)calloc((size_t)o->ncells * 3, sizeof(double));
    o->I = (double *)calloc((size_t)o->ncells * 9, sizeof(double));
    o->S = (double *)calloc((size_t)o->ncells, sizeof(double));
    o->dir = (double *)calloc((size_t)o->ncells * 3, sizeof(double));
    o->E = (double *)calloc((size_t)o->ncells * 9, sizeof(double));
    memcpy(o->Q, Q, (size_t)3 * n * sizeof(double));
    memcpy(o->V, V, (size_t)3 * n * sizeof(double));
    if (U) memcpy(o->U, U, (size_t)3 * n * sizeof(double));
    if (spid) memcpy(o->spid, spid, (size_t)n * sizeof(int));
    /* initial binning + localPROP + globalDensities (init.c:2114-2127) */
    bin_cells(o, 0);
    local_prop(o);
    if (cfg->gndnst > 0.0) {
        o->gndnst = cfg->gndnst;
    } else {
        /* globalDensities, init.c:1002-1018: mean POPSRD over occupied cells
         * of the L^D box (the extra layer excluded) */
        double cnt = 0.0, sumN = 0.0;
        for (int a = 0; a < o->L[0]; a++)
            for (int b = 0; b < o->L[1]; b++)
                for (int c = 0; c < o->L[2]; c++) {
                    int ci = cell_index(o, a, b, c);
                    if (o->pop[ci] > 0) {
                        cnt += 1.0;
                        sumN += (double)o->pop[ci];
                    }
                }
        o->gndnst = cnt > 0.0 ? sumN / cnt : 0.0;
    }
    return o;
}

double oracle_gndnst(const oracle_t *o) { return o->gndnst; }
int oracle_ncells(const oracle_t *o) { return o->ncells; }

/* -------------------------------------------------------------- binning */
/* Cell key by truncation; on shifted grids periodic axes map index L to 0
 * (bin, mpc.c:958-968).  A particle outside the grid here is counted as
 * escaped and clamped; the end-of-step re-bin's re-placement
 * (mpc.c:969-982) is replace_escaped's, before the unshifted binning. */
static void bin_cells(oracle_t *o, int shifted) {
    int n = o->n;
    memset(o->cnt, 0, (size_t)o->ncells * sizeof(int));
    for (int i = 0; i < n; i++) {
        int idx[3];
        for (int d = 0; d < 3; d++) {
            int a = (int)o->Q[3 * i + d];
            if (shifted && o->pbc[d] && a == o->L[d]) a = 0;
            if (a < 0 || a > o->L[d]) {
                o->escaped++;
                a = a < 0 ? 0 : o->L[d];
            }
            idx[d] = a;
        }
        int k = cell_index(o, idx[0], idx[1], idx[2]);
        o->key[i] = k;
        o->cnt[k]++;
    }
    o->start[0] = 0;
    for (int c = 0; c < o->ncells; c++) o->start[c + 1] = o->start[c] + o->cnt[c];
    memset(o->cnt, 0, (size_t)o->ncells * sizeof(int));
    for (int i = 0; i < n; i++) {
        int k = o->key[i];
        o->list[o->start[k] + o->cnt[k]++] = i;
    }
}

static int compute_cm(int op, int lc) {
    /* localPROP, mpc.c:75 */
    return op == MPCD_COLL_RAT || lc != 0 || op == 15 || op == 16 || op == 17;
}

/* localPROP (mpc.c:64-216) for MPCD particles: POP, MASS, VCM, CM and the
 * moment of inertia about CM (localMomInertiaTensor, mpc.c:4209-4299). */
static void local_prop(oracle_t *o) {
    int dim = o->dim, op = o->cfg.coll_op, lc = o->cfg.lc;
    int ccm = compute_cm(op, lc);
    for (int c = 0; c < o->ncells; c++) {
        int s = o->start[c], e = o->start[c + 1];
        double M = 0.0, v[3] = {0, 0, 0}, q[3] = {0, 0, 0};
        for (int j = s; j < e; j++) {
            int i = o->list[j];
            double m = o->cfg.species[o->spid[i]].mass;
            M += m;
            for (int d = 0; d < dim; d++) v[d] += o->V[3 * i + d] * m;
            if (ccm)
                for (int d = 0; d < dim; d++) q[d] += o->Q[3 * i + d] * m;
        }
        o->pop[c] = e - s;
        o->mass[c] = M;
        for (int d = 0; d < dim; d++) {
            if (M > 0.0) {
                v[d] /= M;
                if (ccm) q[d] /= M;
            }
            o->vcm[3 * c + d] = v[d];
            if (ccm) o->cm[3 * c + d] = q[d];
        }
        if (op == MPCD_COLL_RAT || lc != 0) {
            double I[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int j = s; j < e; j++) {
                int i = o->list[j];
                double m = o->cfg.species[o->spid[i]].mass;
                double r[3] = {0, 0, 0};
                for (int d = 0; d < dim; d++) r[d] = o->Q[3 * i + d] - o->cm[3 * c + d];
                I[0] += m * (r[1] * r[1] + r[2] * r[2]);
                I[4] += m * (r[0] * r[0] + r[2] * r[2]);
                I[8] += m * (r[0] * r[0] + r[1] * r[1]);
                I[1] += m * r[0] * r[1];
                I[2] += m * r[0] * r[2];
                I[5] += m * r[1] * r[2];
            }
            I[1] = -I[1];
            I[2] = -I[2];
            I[5] = -I[5];
            I[3] = I[1];
            I[6] = I[2];
            I[7] = I[5];
            memcpy(&o->I[9 * c], I, sizeof(I));
        }
    }
    if (lc != 0) {
        for (int c = 0; c < o->ncells; c++)
            if (o->start[c + 1] - o->start[c] > 1) order_param_2d(o, c);
        vel_grad_2d(o);
    }
}


/* ---------------------------------------------------------------- nematic */
static double len3(const double *v, int n) { return sqrt(dot3(v, v, n)); }
static void norm_n(double *v, int n) {
    /* norm, mtools.c:246-251 */
    double l = len3(v, n);
    if (fabs(l) >= TOL)
        for (int i = 0; i < n; i++) v[i] = v[i] / l;
}
/* rodriguesRotation, mtools.c:1572-1585 (renormalises to the old length) */
static void rodrigues(double *vec, double *ax, double th) {
    double cp[3], dp, old, nw;
    norm_n(ax, 3);
    old = len3(vec, 3);
    cross3(ax, vec, cp);
    dp = dot3(ax, vec, 3);
    for (int i = 0; i < 3; i++)
        vec[i] = vec[i] * cos(th) + cp[i] * sin(th) + ax[i] * dp * (1.0 - cos(th));
    nw = len3(vec, 3);
    for (int i = 0; i < 3; i++) vec[i] *= (old / nw);
}

/* 2x2 eigen-decomposition of the order tensor, eigenvalues2x2 and
 * eigenvectors2x2 (mtools.c:1225-1300), including their special cases.
 * Returns the largest eigenvalue; dir receives eigenvector 0. */
static double eigen2(const double m[4], double dir[2]) {
    double det = m[0] * m[3] - m[2] * m[1];
    double tr = m[0] + m[3];
    double sq = sqrt(tr * tr * 0.25 - det);
    double ev0 = tr * 0.5 + sq, ev1 = tr * 0.5 - sq;
    double e0[2] = {0, 0}, e1[2] = {0, 0};
    (void)ev1;
    if (fabs(m[2] - 0.0) >= TOL) {
        e0[0] = ev0 - m[3];
        e0[1] = m[2];
        norm_n(e0, 2);
    } else if (fabs(m[1] - 0.0) >= TOL) {
        e0[0] = m[1];
        e0[1] = ev0 - m[0];
        norm_n(e0, 2);
    } else {
        if (fabs(m[0] - m[3]) <= TOL) {
            e0[0] = sqrt(2.);
            e0[1] = e0[0];
        } else if (fabs(m[0] - ev0) <= TOL) {
            e0[0] = 1.0;
            e0[1] = 0.0;
        } else if (fabs(m[3] - ev0) <= TOL) {
            /* the reference writes row 0 twice here, ending at (1, 0) */
            e0[0] = 1.0;
            e0[1] = 0.0;
        }
    }
    (void)e1;
    dir[0] = e0[0];
    dir[1] = e0[1];
    return ev0;
}

/* velGradD2Q9, lc.c:2130-2162: E_ij = 3 sum_k w_k e_kj VCM_i(x + e_k) on
 * bulk cells 1..L-1, then edges copied from their neighbour in the
 * reference's order; corner (L, L) keeps its old value. */
static void vel_grad_2d(oracle_t *o) {
    static const int ev[8][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
    const double w[8] = {1. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
    int Lx = o->L[0], Ly = o->L[1];
    for (int a = 1; a < Lx; a++)
        for (int b = 1; b < Ly; b++) {
            double *E = &o->E[9 * cell_index(o, a, b, 0)];
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++) {
                    double e = 0.0;
                    for (int k = 0; k < 8; k++)
                        e += w[k] * ev[k][j] *
                             o->vcm[3 * cell_index(o, a + ev[k][0], b + ev[k][1], 0) + i];
                    e *= 3.;
                    E[3 * i + j] = e;
                }
        }
#define COPYE(dst, src)                                                       \
    for (int i = 0; i < 2; i++)                                                \
        for (int j = 0; j < 2; j++) o->E[9 * (dst) + 3 * i + j] = o->E[9 * (src) + 3 * i + j];
    for (int b = 0; b < Ly; b++) COPYE(cell_index(o, 0, b, 0), cell_index(o, 1, b, 0));
    for (int b = 0; b < Ly; b++) COPYE(cell_index(o, Lx, b, 0), cell_index(o, Lx - 1, b, 0));
    for (int a = 0; a < Lx; a++) COPYE(cell_index(o, a, 0, 0), cell_index(o, a, 1, 0));
    for (int a = 0; a < Lx; a++) COPYE(cell_index(o, a, Ly, 0), cell_index(o, a, Ly - 1, 0));
#undef COPYE
}

/* order tensor, director and scalar order parameter of a cell with more
 * than one particle (tensOrderParam lc.c:1125-1148, localPROP mpc.c:176-213),
 * 2D */
static void order_param_2d(oracle_t *o, int c) {
    int s = o->start[c], e = o->start[c + 1];
    double Sm[4] = {0, 0, 0, 0};
    double cc = 1. / (2.0 - 1.), popinv = 1. / (double)(e - s);
    for (int j = s; j < e; j++) {
        const double *u = &o->U[3 * o->list[j]];
        Sm[0] += u[0] * u[0];
        Sm[1] += u[0] * u[1];
        Sm[3] += u[1] * u[1];
    }
    Sm[0] *= cc * 2.0 * popinv;
    Sm[1] *= cc * 2.0 * popinv;
    Sm[3] *= cc * 2.0 * popinv;
    Sm[0] -= cc;
    Sm[3] -= cc;
    Sm[2] = Sm[1];
    double dir[2];
    double S = eigen2(Sm, dir);
    o->dir[3 * c + 0] = dir[0];
    o->dir[3 * c + 1] = dir[1];
    o->dir[3 * c + 2] = 0.0;
    if (S > 1.0) S = 1.0;
    o->S[c] = S;
}

/* ------------------------------------------------------------ phantoms */
/* ghostPart (mpc.c:351-567), momentum part: a cell cut by a phantom wall
 * (some corner with W < 0, walls at their shifted position) holding
 * 0 < POP < GnDNST gets VCM <- (VCM + N(0, kT (GnDNST-POP))) / GnDNST. */
static void ghost_part(oracle_t *o, uint32_t step) {
    int dim = o->dim, nc = 1 << dim;
    int any = 0;
    for (int w = 0; w < o->cfg.n_walls; w++) any |= o->cfg.walls[w].phantom;
    if (!any) return;
    for (int a = 0; a <= o->L[0]; a++)
        for (int b = 0; b <= o->L[1]; b++)
            for (int c = 0; c <= o->L[2]; c++) {
                int ci = cell_index(o, a, b, c);
                if (o->pop[ci] <= 0) continue;
                int cut = 0;
                for (int w = 0; w < o->cfg.n_walls; w++) {
                    if (!o->cfg.walls[w].phantom) continue;
                    for (int j = 0; j < nc; j++) {
                        double q[3] = {(double)a + (double)(j & 1),
                                       (double)b + (double)((j >> 1) & 1),
                                       (double)c + (double)((j >> 2) & 1)};
                        if (wall_W(o, w, q) < 0.0) cut = 1;
                    }
                }
                if (cut && o->pop[ci] < o->gndnst) {
                    double invN = 1.0 / (o->gndnst - (double)o->pop[ci]);
                    double sig = sqrt(o->cfg.kbt / invN);
                    for (int d = 0; d < dim; d++) {
                        float g = mpcd_rng_normal(o->cfg.seed, o->cfg.replica, step,
                                                  MPCD_STREAM_GHOST, (uint32_t)ci,
                                                  (uint32_t)d);
                        o->vcm[3 * ci + d] += sig * (double)g;
                        o->vcm[3 * ci + d] /= o->gndnst;
                    }
                }
            }
}

/* ------------------------------------------------------------ collisions */
/* The active part of active SRD (activeSRD, mpc.c:2055-2076) after the
 * rotation: turn v toward the cell's VCM u by ACT times their angle (absAngle,
 * mtools.c:325-367) about v x u by Rodrigues' formula with the length kept
 * (rodriguesRotation, mtools.c:1572-1585); skipped for |ACT| < 1e-8 (fneq)
 * and for angles not above ROTTOL = 1e-5.  The cell's activity is the last
 * listed particle's ACT in the reference; the library admits only species
 * of one activity, for which that is every particle's own. */
static void active_turn(double act, const double *u, double *v) {
    if (!(fabs(act) >= 1e-8)) return;
    double cosa = dot3(v, u, 3);
    cosa /= len3(v, 3);
    cosa /= len3(u, 3);
    double theta = acos(cosa), ax[3], cp[3];
    cross3(v, u, ax);
    if (!(fabs(theta) > 1e-5)) return;
    double l = len3(ax, 3);
    if (fabs(l) >= 1e-8)
        for (int d = 0; d < 3; d++) ax[d] = ax[d] / l;
    double old = len3(v, 3);
    cross3(ax, v, cp);
    double dp = dot3(ax, v, 3), t = act * theta;
    for (int d = 0; d < 3; d++) v[d] = v[d] * cos(t) + cp[d] * sin(t) + ax[d] * dp * (1.0 - cos(t));
    double now = len3(v, 3);
    for (int d = 0; d < 3; d++) v[d] *= (old / now);
}

/* SRD (stochrotMPC, mpc.c:1275-1333 with rotate, mpc.c:1181-1257): the
 * rotation sign draw (long)genrand_real() is always 0, so the angle is
 * always -RA; in 2D the random axis is unused.  The orthogonal-axis form
 * (RTECH ORTHAXIS) rotates about Cartesian axis CA = (int)DIM*u
 * (mpc.c:1289); rotate's x-axis matrix has -.1*S in row 2, column 1
 * (mpc.c:1215), kept as the reference has it. */
static void collide_srd(oracle_t *o, int c, uint32_t step) {
    int dim = o->dim;
    double Cs = cos(o->cfg.rot_ang), Sn = -1.0 * sin(o->cfg.rot_ang);
    double R[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int op = o->cfg.coll_op;
    const int active = op == MPCD_COLL_ACT_ARBAXIS || op == MPCD_COLL_ACT_ORTHAXIS;
    if (dim == 3 && (op == MPCD_COLL_ORTHAXIS || op == MPCD_COLL_ACT_ORTHAXIS)) {
        int ca = mpcd_rng_orth_axis(o->cfg.seed, o->cfg.replica, step, (uint32_t)c, dim);
        if (ca == 0) {
            R[0] = 1.;
            R[4] = Cs;
            R[5] = Sn;
            R[7] = -.1 * Sn;
            R[8] = Cs;
        } else if (ca == 1) {
            R[0] = Cs;
            R[2] = Sn;
            R[4] = 1.;
            R[6] = -1. * Sn;
            R[8] = Cs;
        } else {
            R[0] = Cs;
            R[1] = Sn;
            R[3] = -1. * Sn;
            R[4] = Cs;
            R[8] = 1.;
        }
    } else if (dim == 3) {
        double L[3];
        mpcd_rng_axis3(o->cfg.seed, o->cfg.replica, step, (uint32_t)c, L);
        R[0] = L[0] * L[0] + (1. - L[0] * L[0]) * Cs;
        R[1] = L[0] * L[1] * (1. - Cs) - L[2] * Sn;
        R[2] = L[0] * L[2] * (1. - Cs) + L[1] * Sn;
        R[3] = L[0] * L[1] * (1. - Cs) + L[2] * Sn;
        R[4] = L[1] * L[1] + (1. - L[1] * L[1]) * Cs;
        R[5] = L[1] * L[2] * (1. - Cs) - L[0] * Sn;
        R[6] = L[0] * L[2] * (1. - Cs) - L[1] * Sn;
        R[7] = L[1] * L[2] * (1. - Cs) + L[0] * Sn;
        R[8] = L[2] * L[2] + (1. - L[2] * L[2]) * Cs;
    } else {
        R[0] = Cs;
        R[1] = -1. * Sn;
        R[3] = Sn;
        R[4] = Cs;
    }
    const double *u = &o->vcm[3 * c];
    for (int j = o->start[c]; j < o->start[c + 1]; j++) {
        int i = o->list[j];
        double w[3] = {0, 0, 0}, t[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) w[d] = o->V[3 * i + d] - u[d];
        for (int a = 0; a < dim; a++)
            for (int b = 0; b < dim; b++) t[a] += R[a * 3 + b] * w[b];
        for (int d = 0; d < dim; d++) o->V[3 * i + d] = u[d] + t[d];
        if (active) active_turn(o->cfg.species[o->spid[i]].act, u, &o->V[3 * i]);
    }
}

static void thermal_draw(const oracle_t *o, int i, uint32_t step, double *rv) {
    double m = o->cfg.species[o->spid[i]].mass;
    double sig = sqrt(o->cfg.kbt / m); /* genrand_gaussMB, rand.c:510-513 */
    for (int d = 0; d < o->dim; d++)
        rv[d] = sig * (double)mpcd_rng_normal(o->cfg.seed, o->cfg.replica, step,
                                              MPCD_STREAM_THERMAL, (uint32_t)i,
                                              (uint32_t)d);
}

/* Andersen MPC-AT (andersenMPC, mpc.c:1353-1444):
 * v' = VCM + RV - RS - DAMP*VCM/POP, RS = sum(m RV)/M. */
/* Vicsek (vicsek, mpc.c:2098-2135): every particle keeps its speed (length
 * over DIM) and takes a direction uniform on the cone of half-angle
 * pi (1 - ACT) that genrand_cone (rand.c:438-454) builds about
 * VCMdir = VCM/|VCM| (normCopy over 3 components): a draw on the cone about
 * the x axis (genrand_coneNP, rand.c:397-425), then Rodrigues' rotation
 * about VCMdir x x-hat by the angle between them.  The reference leaves
 * VCMdir unset for |VCM| < 1e-8; the draw keeps the x axis here. */
static void rodrigues_keep(double *v, double *ax, double t) {
    double l = len3(ax, 3);
    if (fabs(l - 0.0) >= 1e-8)
        for (int d = 0; d < 3; d++) ax[d] = ax[d] / l;
    double old = len3(v, 3), cp[3];
    cross3(ax, v, cp);
    double dp = dot3(ax, v, 3);
    for (int d = 0; d < 3; d++) v[d] = v[d] * cos(t) + cp[d] * sin(t) + ax[d] * dp * (1.0 - cos(t));
    double now = len3(v, 3);
    for (int d = 0; d < 3; d++) v[d] *= (old / now);
}
/* genrand_cone (rand.c:438-454) with particle i's own uniforms
 * (MPCD_STREAM_VICSEK from index 0): a draw on the cone of half-angle t
 * about x (genrand_coneNP, rand.c:397-425), then, when `rotate`, Rodrigues'
 * rotation about axis x x-hat by the angle between them. */
static void cone_draw(const oracle_t *o, int i, uint32_t step, double t, const double *axis,
                      int rotate, double *r) {
    double u0 = mpcd_rng_uniform(o->cfg.seed, o->cfg.replica, step, MPCD_STREAM_VICSEK,
                                 (uint32_t)i, 0u);
    r[0] = r[1] = r[2] = 0.0;
    if (o->dim == 3) {
        double ct = cos(t), z = u0 * (1.0 - ct) + ct;
        double phi = mpcd_rng_uniform(o->cfg.seed, o->cfg.replica, step, MPCD_STREAM_VICSEK,
                                      (uint32_t)i, 1u) * 2.0 * MPCD_PI;
        r[0] = z;
        r[1] = sqrt(1.0 - z * z) * cos(phi);
        r[2] = sqrt(1.0 - z * z) * sin(phi);
    } else {
        double phi = t * (1. - 2. * u0);
        r[0] = cos(phi);
        r[1] = sin(phi);
    }
    if (rotate) {
        double x[3] = {1.0, 0.0, 0.0}, ax[3];
        cross3(axis, x, ax);
        double cosa = dot3(axis, x, 3);
        cosa /= len3(axis, 3);
        cosa /= len3(x, 3);
        rodrigues_keep(r, ax, acos(cosa));
    }
}

static void collide_vicsek(oracle_t *o, int c, uint32_t step) {
    int dim = o->dim;
    double u[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) u[d] = o->vcm[3 * c + d];
    double l = len3(u, 3);
    int dir = fabs(l - 0.0) >= 1e-8;
    if (dir)
        for (int d = 0; d < 3; d++) u[d] = u[d] / l;
    for (int j = o->start[c]; j < o->start[c + 1]; j++) {
        int i = o->list[j];
        double *v = &o->V[3 * i], r[3];
        double speed = len3(v, dim), theta = MPCD_PI * (1.0 - o->cfg.species[o->spid[i]].act);
        cone_draw(o, i, step, theta, u, dir, r);
        for (int d = 0; d < dim; d++) v[d] = r[d] * speed;
    }
}

/* Chate (chate, mpc.c:2151-2186), 2D: the cell's director is the leading
 * eigenvector of the order tensor of the normalised velocities
 * (tensOrderParam with addToTensOrderParamVel, lc.c:1103-1148; localPROP,
 * mpc.c:176-206; normCopy leaves a velocity shorter than 1e-8 unset, zero
 * here); each particle keeps its speed and takes a direction on the cone of
 * half-angle pi/2 (1 - ACT) about the director, times genrand_pmOne
 * (rand.c:378-382), its next uniform. */
static void chate_dir(const oracle_t *o, int c, double *dir) {
    int s = o->start[c], e = o->start[c + 1];
    double Sm[4] = {0, 0, 0, 0}, cc = 1. / (2.0 - 1.), popinv = 1. / (double)(e - s);
    for (int j = s; j < e; j++) {
        const double *v = &o->V[3 * o->list[j]];
        double l = len3(v, 2), U[2] = {0.0, 0.0};
        if (fabs(l - 0.0) >= 1e-8) {
            U[0] = v[0] / l;
            U[1] = v[1] / l;
        }
        Sm[0] += U[0] * U[0];
        Sm[1] += U[0] * U[1];
        Sm[3] += U[1] * U[1];
    }
    Sm[0] *= cc * 2.0 * popinv;
    Sm[1] *= cc * 2.0 * popinv;
    Sm[3] *= cc * 2.0 * popinv;
    Sm[0] -= cc;
    Sm[3] -= cc;
    Sm[2] = Sm[1];
    dir[0] = dir[1] = dir[2] = 0.0;
    eigen2(Sm, dir);
}

static void collide_chate(oracle_t *o, int c, uint32_t step) {
    int s = o->start[c], e = o->start[c + 1];
    double dir[3];
    chate_dir(o, c, dir);
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double *v = &o->V[3 * i], r[3];
        double speed = len3(v, 2);
        cone_draw(o, i, step, 0.5 * MPCD_PI * (1.0 - o->cfg.species[o->spid[i]].act), dir, 1, r);
        double pm = mpcd_rng_uniform(o->cfg.seed, o->cfg.replica, step, MPCD_STREAM_VICSEK,
                                     (uint32_t)i, 1u) <= 0.5 ? -1.0 : 1.0;
        for (int d = 0; d < 2; d++) v[d] = r[d] * (pm * speed);
    }
}

/* The Vicsek alignment of vicsekAndersenMPC (mpc.c:2204-2290) and
 * vicsekLangevinMPC (mpc.c:2409-2480): a particle whose species has
 * |ACT| > 1e-8 (not feq) gains RELAX (ACT VCMdir - V), VCMdir = VCM/|VCM|
 * (normCopy, mtools.c:262-267; the reference leaves VCMdir unset for
 * |VCM| < 1e-8, taken as zero here).  Neither operator applies DAMP. */
static int vicsek_op(int op) {
    return op == MPCD_COLL_VICSEK_MPCAT || op == MPCD_COLL_VICSEK_LANG;
}
static void vicsek_dir(int dim, const double *u, double *dir) {
    double l = len3(u, dim);
    for (int d = 0; d < 3; d++) dir[d] = 0.0;
    if (fabs(l - 0.0) >= 1e-8)
        for (int d = 0; d < dim; d++) dir[d] = u[d] / l;
}

/* The active velocity of MPC-AT with Chate alignment (chateAndersenMPC,
 * mpc.c:2300-2408), 2D: for |ACT| >= 1e-8 (fneq), AV = pmOne RELAX
 * (ACT - |V|) DIR with pmOne the particle's uniform (genrand_pmOne,
 * rand.c:378-382); returns whether the particle is active.  The update is
 * VCM + RV - RS + AV - AS with AS the cell's mass-weighted mean of AV, and
 * no damping. */
static int chate_av(const oracle_t *o, int i, uint32_t step, const double *dir, double *av) {
    double act = o->cfg.species[o->spid[i]].act;
    av[0] = av[1] = av[2] = 0.0;
    if (!(fabs(act - 0.0) >= 1e-8)) return 0;
    double speed = len3(&o->V[3 * i], 2);
    double pm = mpcd_rng_uniform(o->cfg.seed, o->cfg.replica, step, MPCD_STREAM_VICSEK,
                                 (uint32_t)i, 0u) <= 0.5 ? -1.0 : 1.0;
    for (int d = 0; d < 2; d++) av[d] = pm * o->cfg.relax * (act - speed) * dir[d];
    return 1;
}

static void collide_mpcat(oracle_t *o, int c, uint32_t step) {
    int dim = o->dim, s = o->start[c], e = o->start[c + 1];
    double RS[3] = {0, 0, 0};
    const double *u = &o->vcm[3 * c];
    const int vic = vicsek_op(o->cfg.coll_op);
    const int cha = o->cfg.coll_op == MPCD_COLL_CHATE_MPCAT;
    double dir[3], cdir[3] = {0, 0, 0}, AS[3] = {0, 0, 0};
    vicsek_dir(dim, u, dir);
    if (cha) chate_dir(o, c, cdir);
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double rv[3], av[3];
        thermal_draw(o, i, step, rv);
        double m = o->cfg.species[o->spid[i]].mass;
        for (int d = 0; d < dim; d++) RS[d] += m * rv[d];
        if (cha && chate_av(o, i, step, cdir, av))
            for (int d = 0; d < dim; d++) AS[d] += m * av[d];
    }
    for (int d = 0; d < dim; d++) RS[d] /= o->mass[c];
    for (int d = 0; d < dim; d++) AS[d] /= o->mass[c];
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double rv[3];
        thermal_draw(o, i, step, rv);
        const mpcd_species *sp = &o->cfg.species[o->spid[i]];
        double av[3] = {0, 0, 0};
        if (cha) {
            chate_av(o, i, step, cdir, av);
            for (int d = 0; d < dim; d++) o->V[3 * i + d] = u[d] + rv[d] - RS[d] + av[d] - AS[d];
        } else if (vic && fabs(sp->act - 0.0) > 1e-8) {
            for (int d = 0; d < dim; d++)
                o->V[3 * i + d] = u[d] + o->cfg.relax * (sp->act * dir[d] - o->V[3 * i + d]) +
                                  rv[d] - RS[d];
        } else if (vic) {
            for (int d = 0; d < dim; d++) o->V[3 * i + d] = u[d] + rv[d] - RS[d];
        } else {
            for (int d = 0; d < dim; d++)
                o->V[3 * i + d] = u[d] + rv[d] - RS[d] - sp->damp * u[d] / (double)(e - s);
        }
    }
}

/* Langevin MPC (langevinMPC, mpc.c:1674-1780): the noise WN of every
 * particle (its thermal draw), its plain mean WNS over the cell, and
 * V' = VCM + a (V - VCM) + b (WN - WNS) - DAMP VCM / POP with
 * a = (m - F dt / 2) / (m + F dt / 2), b = sqrt(F dt) / (m + F dt / 2). */
static void collide_lang(oracle_t *o, int c, uint32_t step) {
    int dim = o->dim, s = o->start[c], e = o->start[c + 1];
    double WNS[3] = {0, 0, 0};
    const double *u = &o->vcm[3 * c];
    const double F = o->cfg.fricco, dt = o->cfg.dt;
    const int vic = vicsek_op(o->cfg.coll_op);
    double dir[3];
    vicsek_dir(dim, u, dir);
    for (int j = s; j < e; j++) {
        double rv[3];
        thermal_draw(o, o->list[j], step, rv);
        for (int d = 0; d < dim; d++) WNS[d] += rv[d];
    }
    for (int d = 0; d < dim; d++) WNS[d] /= (double)(e - s);
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double rv[3];
        thermal_draw(o, i, step, rv);
        const mpcd_species *sp = &o->cfg.species[o->spid[i]];
        const double M = sp->mass;
        const double a = (M - F * dt * 0.5) / (M + 0.5 * F * dt);
        const double b = sqrt(F * dt) / (M + 0.5 * F * dt);
        if (vic && fabs(sp->act - 0.0) > 1e-8) {
            for (int d = 0; d < dim; d++) {
                const double v = o->V[3 * i + d];
                o->V[3 * i + d] = u[d] + o->cfg.relax * (sp->act * dir[d] - v) + a * (v - u[d]) +
                                  b * (rv[d] - WNS[d]);
            }
        } else if (vic) {
            for (int d = 0; d < dim; d++)
                o->V[3 * i + d] = u[d] + a * (o->V[3 * i + d] - u[d]) + b * (rv[d] - WNS[d]);
        } else {
            for (int d = 0; d < dim; d++)
                o->V[3 * i + d] = u[d] + a * (o->V[3 * i + d] - u[d]) + b * (rv[d] - WNS[d]) -
                                  sp->damp * u[d] / (double)(e - s);
        }
    }
}

/* Andersen MPC-AT+a (andersenROT, mpc.c:1461-1657): as MPC-AT with the
 * damping not divided by POP, plus the angular-momentum restoring term
 * W x (r - CM), W = I^-1 sum (r-CM) x m(v - RV).  3D: I inverted by
 * adjugate, zero for POP < 3; 2D: only 1/I_zz. */
static void collide_rat(oracle_t *o, int c, uint32_t step) {
    int dim = o->dim, s = o->start[c], e = o->start[c + 1];
    int pop = e - s;
    double RS[3] = {0, 0, 0}, Lm[3] = {0, 0, 0}, W[3] = {0, 0, 0};
    double II[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double *u = &o->vcm[3 * c], *cm = &o->cm[3 * c];
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double rv[3];
        thermal_draw(o, i, step, rv);
        double m = o->cfg.species[o->spid[i]].mass;
        for (int d = 0; d < dim; d++) RS[d] += m * rv[d];
    }
    for (int d = 0; d < dim; d++) RS[d] /= o->mass[c];
    if (dim == 3) {
        if (pop >= 3) inv3(&o->I[9 * c], II);
    } else {
        II[8] = 1. / o->I[9 * c + 8];
    }
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double rv[3] = {0, 0, 0}, r[3] = {0, 0, 0}, dv[3] = {0, 0, 0}, am[3];
        thermal_draw(o, i, step, rv);
        double m = o->cfg.species[o->spid[i]].mass;
        for (int d = 0; d < dim; d++) {
            r[d] = o->Q[3 * i + d] - cm[d];
            dv[d] = m * (o->V[3 * i + d] - rv[d]);
        }
        cross3(r, dv, am);
        for (int d = 0; d < 3; d++) Lm[d] += am[d];
    }
    for (int a = 0; a < 3; a++) {
        W[a] = 0.0;
        for (int b = 0; b < 3; b++) W[a] += II[a * 3 + b] * Lm[b];
    }
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double rv[3] = {0, 0, 0}, r[3] = {0, 0, 0}, ang[3];
        thermal_draw(o, i, step, rv);
        double damp = o->cfg.species[o->spid[i]].damp;
        for (int d = 0; d < dim; d++) r[d] = o->Q[3 * i + d] - cm[d];
        cross3(W, r, ang);
        for (int d = 0; d < dim; d++)
            o->V[3 * i + d] = u[d] + rv[d] - RS[d] - damp * u[d] + ang[d];
    }
}


/* LCcollision (lc.c:427-544) with genrand_maierSaupeMetropolis_2D
 * (lc.c:341-411): Metropolis sampling of each orientation in the cell's
 * mean-field potential, rotated onto the director; torque T = rfc U x dU/dt.
 * Uniforms: the particle's own sequence of the LC stream. */
static void lc_collision_cell(oracle_t *o, int c, uint32_t step) {
    const double KBT = o->cfg.kbt, dt = o->cfg.dt;
    int s = o->start[c], e = o->start[c + 1], pop = e - s;
    double S = o->S[c];
    double DIR[3] = {o->dir[3 * c], o->dir[3 * c + 1], 0.0};
    double xaxis[3] = {1.0, 0.0, 0.0}, rotAx[3];
    cross3(DIR, xaxis, rotAx);
    double ca = dot3(DIR, xaxis, 2) / len3(DIR, 2) / len3(xaxis, 2);
    double rotAngle = -1. * acos(ca);
    norm_n(rotAx, 3);
    double av = 0.0;
    for (int j = s; j < e; j++) av += o->cfg.species[o->spid[o->list[j]]].mfpot;
    if (pop > 1) av /= (float)pop;
    double effM = av * 0.5 * 2.0;
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double *U = &o->U[3 * i], *T = &o->T[3 * i];
        double rfc = o->cfg.species[o->spid[i]].rfc;
        double dU[3] = {U[0], U[1], 0.0};
        for (int d = 0; d < 3; d++) T[d] = 0.;
        uint32_t k = 0;
        /* genrand_maierSaupeMetropolis_2D */
        double newU[3] = {U[0], U[1], 0.0};
        double A[3] = {DIR[0], DIR[1], 0}, B[3] = {U[0], U[1], 0}, cr[3];
        cross3(A, B, cr);
        double ang0 = atan2(len3(cr, 3), dot3(A, B, 2));
        if (fabs(ang0 - 0.5 * MPCD_PI) <= TOL || fabs(ang0 + 0.5 * MPCD_PI) <= TOL)
            ang0 = MPCD_PI * (0.5 - mpcd_rng_uniform(o->cfg.seed, o->cfg.replica, step,
                                                  MPCD_STREAM_LC, (uint32_t)i, k++));
        double uz0 = dot3(DIR, U, 2);
        int anneal = (int)(5 + 0.1 * effM * S / KBT);
        int cnt = 0;
        for (int a = 0; a < anneal; a++) {
            int acc = 0;
            double w0 = effM * S * uz0 * uz0 / KBT;
            double ang1 = MPCD_PI * (0.5 - mpcd_rng_uniform(o->cfg.seed, o->cfg.replica, step,
                                                        MPCD_STREAM_LC, (uint32_t)i, k++));
            double uz1 = cos(ang1);
            double w1 = effM * S * uz1 * uz1 / KBT;
            double dw = w1 - w0;
            if (dw >= 0.) {
                acc = 1;
            } else {
                double R = mpcd_rng_uniform(o->cfg.seed, o->cfg.replica, step, MPCD_STREAM_LC,
                                            (uint32_t)i, k++);
                if (R <= exp(dw)) acc = 1;
            }
            if (acc) {
                cnt += 1;
                ang0 = ang1;
                uz0 = uz1;
            }
        }
        newU[0] = uz0;
        newU[1] = sin(ang0);
        if (cnt > 0) {
            double ax[3] = {rotAx[0], rotAx[1], rotAx[2]};
            rodrigues(newU, ax, rotAngle);
            U[0] = newU[0];
            U[1] = newU[1];
        }
        for (int d = 0; d < 2; d++) dU[d] = (U[d] - dU[d]) / dt;
        cross3(U, dU, T);
        for (int d = 0; d < 3; d++) T[d] *= rfc;
    }
}

/* jefferysTorque (lc.c:559-607) with larsonRotRate (lc.c:622-718):
 * du/dt = u.W + lambda (u.D - u u u:D), rotation by chi dt |u x du/dt|. */
static void jeffery_cell(oracle_t *o, int c) {
    const double *E = &o->E[9 * c];
    for (int j = o->start[c]; j < o->start[c + 1]; j++) {
        int p = o->list[j];
        double tumble = o->cfg.species[o->spid[p]].tumble;
        double chihi = o->cfg.species[o->spid[p]].chihi;
        double *U = &o->U[3 * p];
        double u[3] = {U[0], U[1], U[2]};
        double D[3][3], W[3][3], uuuD[3] = {0, 0, 0}, uw[3] = {0, 0, 0}, uD[3] = {0, 0, 0};
        double dudt[3], w[3];
        for (int i = 0; i < 3; i++)
            for (int jj = 0; jj < 3; jj++) {
                D[jj][i] = 0.5 * (E[3 * i + jj] + E[3 * jj + i]);
                W[jj][i] = 0.5 * (E[3 * i + jj] - E[3 * jj + i]);
            }
        for (int jj = 0; jj < 3; jj++) {
            for (int i = 0; i < 3; i++) {
                for (int k = 0; k < 3; k++) uuuD[jj] += u[jj] * (u[i] * D[i][k] * u[k]);
                uD[jj] += u[i] * D[i][jj];
                uw[jj] += u[i] * W[i][jj];
            }
            dudt[jj] = uw[jj] + tumble * (uD[jj] - uuuD[jj]);
        }
        cross3(u, dudt, w);
        for (int i = 0; i < 3; i++) w[i] *= chihi;
        for (int i = 0; i < 3; i++) w[i] *= o->cfg.dt;
        double theta = len3(w, 3);
        norm_n(w, 3);
        rodrigues(U, w, theta);
    }
}

/* Andersen-ROT for nematic fluids: andersenROT_LC (lc.c:1515-1728) and
 * dipoleAndersenROT_LC (lc.c:1749-2043, collOp 16/17/20/21: active dipole
 * kick +-ACT dt DIR by the side of the plane through CM normal to DIR).
 * Angular momentum includes the orientational torques sum T dt. */
static void collide_lc(oracle_t *o, int c, uint32_t step) {
    int op = o->cfg.coll_op, s = o->start[c], e = o->start[c + 1], pop = e - s;
    int dipole = (op == 16 || op == 17 || op == 20 || op == 21);
    const double dt = o->cfg.dt;
    double RS[3] = {0, 0, 0}, AS[3] = {0, 0, 0}, Llm[3] = {0, 0, 0}, Lnm[3] = {0, 0, 0};
    double W[3] = {0, 0, 0}, II[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double *u = &o->vcm[3 * c], *cm = &o->cm[3 * c], *dir = &o->dir[3 * c];
    double ACT = 0.0, sigW = 0.0, sigP = 0.0;
    if (dipole) {
        int spcnt[MPCD_MAX_SPECIES] = {0};
        for (int j = s; j < e; j++) spcnt[o->spid[o->list[j]]]++;
        for (int j = s; j < e; j++) {
            const mpcd_species *sp = &o->cfg.species[o->spid[o->list[j]]];
            if (sp->minactratio == 0.0 ||
                sp->minactratio * o->gndnst < (double)spcnt[o->spid[o->list[j]]]) {
                ACT += sp->act / sp->mass;
                sigW += sp->sigwidth;
                sigP += sp->sigpos;
            }
        }
        if (op == 17 || op == 20) ACT *= o->gndnst / ((double)pop);
        if (op == 20 || op == 21) {
            sigW /= (double)pop;
            sigP /= (double)pop;
            double fall = (1 - tanh(((double)pop - o->gndnst * (1 + sigP)) / (o->gndnst * sigW)));
            ACT *= fall / 2;
        }
        ACT *= dt;
    }
    int act_on = dipole && fabs(ACT - 0.0) >= TOL;
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double m = o->cfg.species[o->spid[i]].mass;
        double rv[3];
        thermal_draw(o, i, step, rv);
        for (int d = 0; d < 2; d++) RS[d] += m * rv[d];
        if (act_on) {
            double pW = 0.0;
            for (int d = 0; d < 2; d++) pW += dir[d] * (o->Q[3 * i + d] - cm[d]);
            pW -= 0.0;
            double pm = pW <= 0 ? -1. : 1.;
            for (int d = 0; d < 2; d++) AS[d] += m * (pm * ACT * dir[d]);
        }
    }
    for (int d = 0; d < 2; d++) {
        RS[d] /= o->mass[c];
        AS[d] /= o->mass[c];
    }
    II[8] = 1. / o->I[9 * c + 8];
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double m = o->cfg.species[o->spid[i]].mass;
        double rv[3] = {0, 0, 0}, r[3] = {0, 0, 0}, dv[3] = {0, 0, 0}, am[3], av[3] = {0, 0, 0};
        thermal_draw(o, i, step, rv);
        if (act_on) {
            double pW = 0.0;
            for (int d = 0; d < 2; d++) pW += dir[d] * (o->Q[3 * i + d] - cm[d]);
            pW -= 0.0;
            double pm = pW <= 0 ? -1. : 1.;
            for (int d = 0; d < 2; d++) av[d] = pm * ACT * dir[d];
        }
        for (int d = 0; d < 2; d++) {
            r[d] = o->Q[3 * i + d] - cm[d];
            dv[d] = dipole ? m * (o->V[3 * i + d] - rv[d] - av[d]) : m * (o->V[3 * i + d] - rv[d]);
        }
        cross3(r, dv, am);
        for (int d = 0; d < 3; d++) Llm[d] += am[d];
        for (int d = 0; d < 3; d++) Lnm[d] += o->T[3 * i + d] * dt;
    }
    double L[3];
    for (int d = 0; d < 3; d++) L[d] = Llm[d] + Lnm[d];
    for (int a = 0; a < 3; a++) {
        W[a] = 0.0;
        for (int b = 0; b < 3; b++) W[a] += II[a * 3 + b] * L[b];
    }
    for (int j = s; j < e; j++) {
        int i = o->list[j];
        double rv[3] = {0, 0, 0}, r[3] = {0, 0, 0}, ang[3], av[3] = {0, 0, 0};
        thermal_draw(o, i, step, rv);
        double damp = o->cfg.species[o->spid[i]].damp;
        for (int d = 0; d < 2; d++) r[d] = o->Q[3 * i + d] - cm[d];
        cross3(W, r, ang);
        if (dipole) {
            if (act_on) {
                double pW = 0.0;
                for (int d = 0; d < 2; d++) pW += dir[d] * (o->Q[3 * i + d] - cm[d]);
                pW -= 0.0;
                double pm = pW <= 0 ? -1. : 1.;
                for (int d = 0; d < 2; d++) av[d] = pm * ACT * dir[d];
            }
            for (int d = 0; d < 2; d++)
                o->V[3 * i + d] = u[d] + rv[d] - RS[d] + ang[d] + av[d] - AS[d] - damp * u[d];
        } else {
            for (int d = 0; d < 2; d++) o->V[3 * i + d] = u[d] + rv[d] - RS[d] + ang[d];
        }
    }
}

/* oriBC (lc.c:1290-1405) for a static wall: orientation made unit, turned to
 * point out of the wall, its normal/tangential parts scaled by MUN/MUT (or
 * replaced by DUxyz when both are 0), scaled by MUxyz and renormalised. */
static void ori_bc(oracle_t *o, int i, const mpcd_wall *wl, const double *n) {
    int dim = o->dim;
    double *U = &o->U[3 * i], UN[3] = {0, 0, 0}, UT[3] = {0, 0, 0};
    norm_n(U, dim);
    if (dot3(U, n, dim) >= 0.0)
        for (int d = 0; d < dim; d++) U[d] *= 1.;
    else
        for (int d = 0; d < dim; d++) U[d] *= -1.;
    double x = dot3(U, n, dim);
    for (int d = 0; d < dim; d++) UN[d] = x * n[d];
    for (int d = 0; d < dim; d++) UT[d] = U[d] - UN[d];
    if (fabs(wl->MUN - 0.0) <= TOL && fabs(wl->MUT - 0.0) <= TOL) {
        for (int d = 0; d < dim; d++) U[d] = wl->DUxyz[d];
    } else {
        for (int d = 0; d < dim; d++) {
            UN[d] *= wl->MUN;
            UT[d] *= wl->MUT;
        }
        for (int d = 0; d < dim; d++) U[d] = UN[d] + UT[d];
        U[0] *= wl->MUxyz[0];
        if (dim >= 2) U[1] *= wl->MUxyz[1];
        if (dim >= 3) U[2] *= wl->MUxyz[2];
    }
    norm_n(U, dim);
}

/* ----------------------------------------------------------------- walls */
/* MPC_BCcollision (bc.c:1363-1496) for static planar walls with rule-based
 * collisions (COLL_TYPE 1): repeatedly find the wall crossed earliest
 * (chooseBC, bc.c:1252-1334), rewind to it, transform velocity (velBC,
 * bc.c:598-746) and position (posBC, bc.c:760-774), stream the rest. */
static void push_velocity(const mpcd_config *c, int dim, uint32_t step, uint32_t stream,
                          uint32_t id, uint32_t k0, int PL, double MASS, double *V);

static void wall_collisions(oracle_t *o, int i) {
    int dim = o->dim, nw = o->cfg.n_walls;
    double *q = &o->Q[3 * i], *v = &o->V[3 * i];
    double dt = o->cfg.dt, t_left = dt, t_coll = 0.0;
    int chosen = 0, cnt = 0, cnt2 = 0, flagged = 0;
    double m = o->cfg.species[o->spid[i]].mass;
    for (;;) {
        double t_min = t_left, W = 1.0;
        for (int w = 0; w < nw; w++) {
            const mpcd_wall *wl = &o->cfg.walls[w];
            if (!wl->inter[o->spid[i]]) continue;
            double tw = wall_W(o, w, q);
            if (tw < 0.0) {
                /* crosstimeReverse, planar branch (bc.c:257-262) */
                double t1 = wl->R;
                for (int d = 0; d < dim; d++) t1 += wl->A[d] * (o->wallQ[w][d] - q[d]);
                t1 /= (wl->A[0] * (-v[0]) + wl->A[1] * (-v[1]) + wl->A[2] * (-v[2]));
                double tc = t_left - t1;
                if (tc < t_min) {
                    t_min = tc;
                    chosen = w;
                    W = tw;
                }
            }
        }
        t_coll = t_min;
        if (W > -TOL) break;
        cnt++;
        const mpcd_wall *wl = &o->cfg.walls[chosen];
        if (t_coll > -TOL) {
            double n[3] = {0, 0, 0}, vn[3] = {0, 0, 0}, vt[3] = {0, 0, 0};
            double V[3] = {0, 0, 0};
            for (int d = 0; d < dim; d++) q[d] = q[d] - (t_left - t_coll) * v[d];
            for (int d = 0; d < dim; d++) n[d] = wl->A[d];
            double len = sqrt(dot3(n, n, dim));
            if (fabs(len) >= TOL)
                for (int d = 0; d < dim; d++) n[d] = n[d] / len;
            /* velBC, rule branch: walls at rest, no spin */
            for (int d = 0; d < dim; d++) V[d] = v[d] - 0.0 - 0.0;
            double x = dot3(V, n, dim);
            for (int d = 0; d < dim; d++) vn[d] = x * n[d];
            for (int d = 0; d < dim; d++) vt[d] = V[d] - vn[d];
            for (int d = 0; d < dim; d++) {
                vn[d] *= wl->MVN;
                vn[d] += wl->DVN * n[d];
                vt[d] *= wl->MVT;
                vt[d] += wl->DVT;
            }
            for (int d = 0; d < dim; d++) V[d] = vn[d] + vt[d];
            for (int d = 0; d < dim; d++) V[d] += wl->DVxyz[d];
            for (int d = 0; d < dim; d++) V[d] += 0.0 + 0.0;
            for (int d = 0; d < dim; d++) {
                V[d] -= v[d];
                V[d] *= m;
            }
            double imp = 1.0 / m;
            for (int d = 0; d < dim; d++) v[d] += V[d] * 1.0 * imp;
            /* posBC */
            double pn[3], pt[3];
            double xq = dot3(q, n, dim);
            for (int d = 0; d < dim; d++) pn[d] = xq * n[d];
            for (int d = 0; d < dim; d++) pt[d] = q[d] - pn[d];
            for (int d = 0; d < dim; d++) {
                pn[d] += wl->DN * n[d] * (1. - 2. * TOL);
                pt[d] += wl->DT;
            }
            for (int d = 0; d < dim; d++) q[d] = pn[d] + pt[d];
            if (o->cfg.lc != 0) ori_bc(o, i, wl, n);
            t_left -= t_coll;
            for (int d = 0; d < dim; d++) q[d] = q[d] + t_left * v[d];
            if (wall_W(o, chosen, q) < -TOL)
                for (int d = 0; d < dim; d++) q[d] = q[d] - t_left * v[d];
        } else {
            for (int d = 0; d < dim; d++) q[d] = q[d] - (t_left - t_coll) * v[d];
        }
        if (cnt > NBOUNCE) {
            flagged = 1; /* bcCNT, bc.c:1462 */
            if (cnt < 2 * NBOUNCE && cnt2 == 0) {
                if (t_left > TOL) {
                    t_left *= 1.1;
                } else {
                    t_left = 0.9 * dt;
                    t_coll = 0.1 * dt;
                }
            } else {
                /* re-thermalise: a fresh velocity of the species'
                 * distribution and a whole step to stream (bc.c:1477-1488);
                 * at most 16 times (the reference tries for ever) */
                if (cnt2 >= 16) break;
                push_velocity(&o->cfg, dim, o->step, MPCD_STREAM_RETHERM, (uint32_t)i,
                              4u * (uint32_t)cnt2, o->vdist[o->spid[i]], m, v);
                t_left = dt;
                t_coll = 0.0;
                cnt2++;
                cnt = 0;
            }
        }
    }
    if (flagged) o->bounce_limit++;
}

/* ------------------------------------------------------------------ step */
int oracle_set_vdist(oracle_t *o, const int *vdist) {
    for (int s = 0; s < o->cfg.n_species; s++) o->vdist[s] = vdist[s];
    return 0;
}

/* The end-of-step re-bin (bin, mpc.c:969-982, unshifted): a particle whose
 * truncated index on some axis lies outside [0, L] left the grid and is
 * re-placed: replacePos_WithCheck (init.c:1462-1483) draws the uniform
 * position L u (replace, init.c:1240-1243) until no wall has W <= TOL there
 * (every wall, as the reference loops over all of them), then bin() gives it
 * a Maxwell-Boltzmann velocity (genrand_gaussMB per component) and, for a
 * nematic, the orientation genrand_coneNP(U, pi, DIM) (rand.c:397-425, 2D
 * branch).  The reference keeps the particle in its old cell list until the
 * next bin(); here it is binned at its new position.  Draws: the particle's
 * counter-based streams of the step; placement attempt a takes uniforms
 * DIM a .. DIM a + DIM - 1, at most 64 attempts (the reference tries for
 * ever). */
static void replace_escaped(oracle_t *o, int i, uint32_t step) {
    const int dim = o->dim;
    double *q = &o->Q[3 * i];
    int out = 0;
    for (int d = 0; d < dim; d++) {
        const int a = (int)q[d];
        if (a < 0 || a > o->L[d]) out = 1;
    }
    if (!out) return;
    o->escaped++;
    const mpcd_config *c = &o->cfg;
    for (uint32_t a = 0; a < 64u; a++) {
        for (int d = 0; d < dim; d++)
            q[d] = (double)o->L[d] * mpcd_rng_uniform(c->seed, c->replica, step,
                                                      MPCD_STREAM_ESCAPE_POS, (uint32_t)i,
                                                      a * (uint32_t)dim + (uint32_t)d);
        int in_wall = 0;
        for (int w = 0; w < c->n_walls; w++)
            if (wall_W(o, w, q) <= TOL) in_wall = 1;
        if (!in_wall) break;
    }
    const double sig = sqrt(c->kbt / c->species[o->spid[i]].mass);
    for (int d = 0; d < dim; d++)
        o->V[3 * i + d] = sig * (double)mpcd_rng_normal(c->seed, c->replica, step,
                                                        MPCD_STREAM_ESCAPE_VEL, (uint32_t)i,
                                                        (uint32_t)d);
    if (c->lc != 0 && dim == 2) {
        const double u = mpcd_rng_uniform(c->seed, c->replica, step, MPCD_STREAM_ESCAPE_ORI,
                                          (uint32_t)i, 0u);
        const double phi = MPCD_PI * (1. - 2. * u);
        o->U[3 * i] = cos(phi);
        o->U[3 * i + 1] = sin(phi);
    }
}

int oracle_step(oracle_t *o, uint32_t step) {
    o->step = step;
    int dim = o->dim, n = o->n, op = o->cfg.coll_op;
    double s[3] = {0, 0, 0};
    if (o->cfg.lc != 0 && dim != 2) return MPCD_ERR_UNSUPPORTED;
    if (o->cfg.galinv) mpcd_rng_shift(o->cfg.seed, o->cfg.replica, step, dim, s);
    /* gridShift_all(...,0), mpc.c:728-736 and walls :765 */
    for (int i = 0; i < n; i++)
        for (int d = 0; d < dim; d++) {
            double *q = &o->Q[3 * i + d];
            *q += s[d];
            if (*q > o->L[d] && *q <= o->L[d] + s[d]) *q -= o->L[d];
        }
    for (int w = 0; w < o->cfg.n_walls; w++)
        for (int d = 0; d < dim; d++) o->wallQ[w][d] += s[d];
    bin_cells(o, 1);
    /* acc_all, mpc.c:697-700 (GRAV_FLAG as initializeSIM, init.c:2059) */
    const double *g = o->cfg.grav;
    if (fabs(g[0]) >= TOL || fabs(g[1]) >= TOL || fabs(g[2]) >= TOL)
        for (int i = 0; i < n; i++)
            for (int d = 0; d < dim; d++) o->V[3 * i + d] = o->V[3 * i + d] + o->cfg.dt * g[d];
    local_prop(o);
    ghost_part(o, step);
    if (o->cfg.lc != 0) {
        /* mpc.c:4640-4678 */
        for (int c = 0; c < o->ncells; c++)
            if (o->pop[c] > 1) lc_collision_cell(o, c, step);
        for (int c = 0; c < o->ncells; c++)
            if (o->pop[c] > 1) jeffery_cell(o, c);
    }
    for (int c = 0; c < o->ncells; c++) {
        if (o->pop[c] <= 1) continue;
        if (o->cfg.lc != 0)
            collide_lc(o, c, step);
        else if (op == MPCD_COLL_ARBAXIS || op == MPCD_COLL_ORTHAXIS ||
                 op == MPCD_COLL_ACT_ARBAXIS || op == MPCD_COLL_ACT_ORTHAXIS)
            collide_srd(o, c, step);
        else if (op == MPCD_COLL_VICSEK)
            collide_vicsek(o, c, step);
        else if (op == MPCD_COLL_CHATE && dim == 2)
            collide_chate(o, c, step);
        else if (op == MPCD_COLL_MPCAT || op == MPCD_COLL_VICSEK_MPCAT ||
                 (op == MPCD_COLL_CHATE_MPCAT && dim == 2))
            collide_mpcat(o, c, step);
        else if (op == MPCD_COLL_LANG || op == MPCD_COLL_VICSEK_LANG)
            collide_lang(o, c, step);
        else if (op == MPCD_COLL_RAT)
            collide_rat(o, c, step);
        else
            return MPCD_ERR_UNSUPPORTED;
    }
    /* avVel (therm.c:362-367) over every cell; TEMP (therm.c:209-235) */
    for (int d = 0; d < 3; d++) o->avnow[d] = 0.0;
    for (int c = 0; c < o->ncells; c++)
        for (int d = 0; d < dim; d++) o->avnow[d] += o->vcm[3 * c + d];
    for (int d = 0; d < dim; d++) o->avnow[d] /= o->vol;
    double kbt = 0.0;
    for (int i = 0; i < n; i++) {
        const double *v = &o->V[3 * i];
        double t = (v[0] - 0.0) * (v[0] - 0.0);
        t += (v[1] - 0.0) * (v[1] - 0.0);
        t += (v[2] - 0.0) * (v[2] - 0.0);
        kbt += o->cfg.species[o->spid[i]].mass * t;
    }
    o->kbtnow = kbt / (double)(n * dim);
    /* gridShift_all(...,1) */
    for (int i = 0; i < n; i++)
        for (int d = 0; d < dim; d++) {
            double *q = &o->Q[3 * i + d];
            *q += -1.0 * s[d];
            if (*q < 0.0 && *q >= -1.0 * s[d]) *q += o->L[d];
        }
    for (int w = 0; w < o->cfg.n_walls; w++)
        for (int d = 0; d < dim; d++) o->wallQ[w][d] += -1.0 * s[d];
    /* stream_all, mpc.c:680-687 */
    for (int i = 0; i < n; i++)
        for (int d = 0; d < dim; d++) o->Q[3 * i + d] = o->Q[3 * i + d] + o->cfg.dt * o->V[3 * i + d];
    for (int i = 0; i < n; i++) wall_collisions(o, i);
    /* the re-bin's escape rule (bin, mpc.c:969-982) */
    for (int i = 0; i < n; i++) replace_escaped(o, i, step);
    /* re-bin on the unshifted grid + localPROP, mpc.c:4936-4942 */
    bin_cells(o, 0);
    local_prop(o);
    return 0;
}

int oracle_get_particles(const oracle_t *o, double *Q, double *V, double *U) {
    if (Q) memcpy(Q, o->Q, (size_t)3 * o->n * sizeof(double));
    if (V) memcpy(V, o->V, (size_t)3 * o->n * sizeof(double));
    if (U) memcpy(U, o->U, (size_t)3 * o->n * sizeof(double));
    return 0;
}

int oracle_get_globals(const oracle_t *o, double *kbtnow, double *avnow) {
    *kbtnow = o->kbtnow;
    for (int d = 0; d < 3; d++) avnow[d] = o->avnow[d];
    return 0;
}

int oracle_get_cells(const oracle_t *o, int *pop, double *mass, double *vcm,
                     double *cm) {
    for (int c = 0; c < o->ncells; c++) {
        if (pop) pop[c] = o->pop[c];
        if (mass) mass[c] = o->mass[c];
        for (int d = 0; d < 3; d++) {
            if (vcm) vcm[3 * c + d] = o->vcm[3 * c + d];
            if (cm) cm[3 * c + d] = o->cm[3 * c + d];
        }
    }
    return 0;
}

long oracle_escaped(const oracle_t *o) { return o->escaped; }

/* Populations of the cells of step 'step's shifted grid from the current
 * positions, without changing the state: the shift (ranshift,
 * rand.c:678-696), gridShift_all's forward wrap (mpc.c:728-736) and bin's
 * truncation, periodic L -> 0 and clamping (mpc.c:958-982) -- the cell lists
 * the next oracle_step(o, step) collides. */
int oracle_shifted_counts(const oracle_t *o, uint32_t step, int *pop) {
    double s[3] = {0, 0, 0};
    if (o->cfg.galinv) mpcd_rng_shift(o->cfg.seed, o->cfg.replica, step, o->dim, s);
    memset(pop, 0, (size_t)o->ncells * sizeof(int));
    for (int i = 0; i < o->n; i++) {
        int idx[3] = {0, 0, 0};
        for (int d = 0; d < o->dim; d++) {
            double q = o->Q[3 * i + d] + s[d];
            if (q > o->L[d] && q <= o->L[d] + s[d]) q -= o->L[d];
            int a = (int)q;
            if (o->pbc[d] && a == o->L[d]) a = 0;
            if (a < 0) a = 0;
            if (a > o->L[d]) a = o->L[d];
            idx[d] = a;
        }
        pop[cell_index(o, idx[0], idx[1], idx[2])]++;
    }
    return 0;
}

/* ============================================================ initial state
 * initializeSIM's particle set-up (init.c:2092-2170) for QDIST = PRF:
 * setcoord (init.c:1565-1600) with place, push and orient per particle and
 * the mean velocity AVV; checkplaceMPC/replace (init.c:1240-1246, 1428-1449)
 * per particle; galileantrans (mtools.c:673-711) when RFRAME and GPOP > 2;
 * TEMP about AVV and the VSC scaling (scaleT, therm.c:106-143).  Draws: the
 * counter-based generator at step 0, per particle, in the streams
 * MPCD_STREAM_INIT_POS (attempt a: uniforms 4a + d), MPCD_STREAM_INIT_VEL and
 * MPCD_STREAM_INIT_ORI.  Sums run serially in particle order, as the
 * reference's loops do. */
static double init_u(const mpcd_config *c, uint32_t stream, int i, uint32_t k) {
    return mpcd_rng_uniform(c->seed, c->replica, 0u, stream, (uint32_t)i, k);
}

/* norm (mtools.c:246-251) with fneq (mtools.c:74-76) */
static void init_norm(double *x, int dim) {
    double l = 0.0;
    for (int i = 0; i < dim; i++) l += x[i] * x[i];
    l = sqrt(l);
    if (fabs(l - 0.0) >= TOL)
        for (int i = 0; i < dim; i++) x[i] = x[i] / l;
}

/* genrand_coneNP(vec, pi, dim), rand.c:397-425 */
static void init_cone(const mpcd_config *c, int i, uint32_t *k, double *vec, int dim) {
    const double theta = MPCD_PI;
    double ct = cos(theta);
    if (dim == 3) {
        double z = init_u(c, MPCD_STREAM_INIT_ORI, i, (*k)++) * (1.0 - ct) + ct;
        double phi = init_u(c, MPCD_STREAM_INIT_ORI, i, (*k)++) * 2.0 * MPCD_PI;
        vec[0] = z;
        vec[1] = sqrt(1.0 - z * z) * cos(phi);
        vec[2] = sqrt(1.0 - z * z) * sin(phi);
    } else {
        double phi = theta * (1. - 2. * init_u(c, MPCD_STREAM_INIT_ORI, i, (*k)++));
        vec[0] = cos(phi);
        vec[1] = sin(phi);
    }
}

/* orient, init.c:1307-1405 */
static void init_orient(const mpcd_config *c, int dim, const int *XYZ, int i, int PL,
                        const double *Q, double *U) {
    uint32_t k = 0;
    double noise;
    int d;
    if (PL == MPCD_ODIST_RANDORIENT) {
        init_cone(c, i, &k, U, dim);
    } else if (PL == MPCD_ODIST_ALIGNX) {
        noise = 1.0 + 0.02 * (init_u(c, MPCD_STREAM_INIT_ORI, i, k++) - 0.5);
        U[0] = 0.9999 * noise;
        U[1] = 0.01414178 * noise;
        if (dim >= 3) U[2] = 0.000008 * noise;
    } else if (PL == MPCD_ODIST_ALIGNY) {
        noise = 1.0 + 0.02 * (init_u(c, MPCD_STREAM_INIT_ORI, i, k++) - 0.5);
        U[1] = 0.9999 * noise;
        U[0] = 0.01414178 * noise;
        if (dim >= 3) U[2] = 0.000008 * noise;
    } else if (PL == MPCD_ODIST_ALIGNZ) {
        noise = 1.0 + 0.02 * (init_u(c, MPCD_STREAM_INIT_ORI, i, k++) - 0.5);
        U[2] = 0.9999 * noise;
        U[0] = 0.007071 * noise;
        U[1] = 0.007071 * noise;
    } else if (PL == MPCD_ODIST_ALIGN45) {
        if (dim == 2)
            for (d = 0; d < dim; d++) U[d] = 1. / sqrt(2.);
        else
            for (d = 0; d < dim; d++) U[d] = 1. / sqrt(3.);
    } else if (PL == MPCD_ODIST_PLANEZ) {
        init_cone(c, i, &k, U, 2);
    } else if (PL == MPCD_ODIST_PLANEY) {
        init_cone(c, i, &k, U, 2);
        U[2] = U[1];
        U[1] = 0.0;
    } else if (PL == MPCD_ODIST_PLANEX) {
        init_cone(c, i, &k, U, 2);
        U[2] = U[0];
        U[0] = 0.0;
    } else if (PL == MPCD_ODIST_ALIGNTR) {
        double L2 = 0.0;
        for (d = 0; d < dim; d++) L2 += XYZ[d] * XYZ[d];
        L2 = sqrt(L2);
        for (d = 0; d < dim; d++) U[d] = XYZ[d] / L2;
    } else if (PL == MPCD_ODIST_ALIGNDEFECTPAIR) {
        double QP[2], QM[2], UP[2], UM[2], kP = 0.5, kM = -0.5, phiP, phiM, wP, wM, wY, r, R;
        R = 0.5 * sqrt(2.25 * ((double)XYZ[0]) * ((double)XYZ[0]) +
                       ((double)XYZ[1]) * ((double)XYZ[1]));
        QP[0] = ((double)XYZ[0]) * 0.25;
        QP[1] = ((double)XYZ[1]) * 0.5;
        phiP = atan2(QP[1] - Q[1], QP[0] - Q[0]);
        UP[0] = cos(kP * phiP);
        UP[1] = sin(kP * phiP);
        r = sqrt(pow(QP[0] - Q[0], 2.0) + pow(QP[1] - Q[1], 2.0));
        wP = 1.0 - r / R;
        QM[0] = ((double)XYZ[0]) * 0.75;
        QM[1] = ((double)XYZ[1]) * 0.5;
        phiM = atan2(-QM[1] + Q[1], -QM[0] + Q[0]);
        UM[0] = cos(kM * phiM);
        UM[1] = sin(kM * phiM);
        r = sqrt(pow(QM[0] - Q[0], 2.0) + pow(QM[1] - Q[1], 2.0));
        wM = 1.0 - r / R;
        if (Q[1] <= 0.5 * ((double)XYZ[1]))
            wY = 1.0 - 2.0 * Q[1] / (double)XYZ[1];
        else
            wY = 1.0 - 2.0 * ((double)XYZ[1] - Q[1]) / (double)XYZ[1];
        U[0] = wP * UP[0] + wM * UM[0] + wY;
        U[1] = wP * UP[1] + wM * UM[1];
        if (dim > 2) U[2] = 0.0;
        init_norm(U, dim);
    }
}

/* push, init.c:1261-1291, drawing from (step, stream, id): uniforms or
 * normals k0 + d */
static void push_velocity(const mpcd_config *c, int dim, uint32_t step, uint32_t stream,
                          uint32_t id, uint32_t k0, int PL, double MASS, double *V) {
    const double KBT = c->kbt;
    int d;
    for (d = 0; d < 3; d++) V[d] = 0.0;
    if (PL == MPCD_VDIST_RANDVEL) {
        for (d = 0; d < dim; d++)
            V[d] = sqrt(KBT / MASS) *
                   (2. * mpcd_rng_uniform(c->seed, c->replica, step, stream, id, k0 + d) - 1.);
    } else if (PL == MPCD_VDIST_HOMOAXIS) {
        for (d = 0; d < dim; d++) {
            V[d] = sqrt(dim * KBT / MASS);
            V[d] *= mpcd_rng_uniform(c->seed, c->replica, step, stream, id, k0 + d) <= 0.5
                        ? -1.0
                        : 1.0;
        }
    } else {
        /* genrand_gaussMB (rand.c:510-513): sqrt(KBT/M) times a float normal */
        for (d = 0; d < dim; d++)
            V[d] = sqrt(KBT / MASS) *
                   mpcd_rng_normal(c->seed, c->replica, step, stream, id, k0 + (uint32_t)d);
        if (PL == MPCD_VDIST_HOMO) {
            init_norm(V, dim);
            double normalize = sqrt((double)dim * KBT / MASS);
            for (d = 0; d < dim; d++) V[d] *= normalize;
        }
    }
}

/* Q, V, U (3 doubles per particle) and spid of the initial state; returns
 * 0, or -1 for bad arguments or a particle not placed within max_attempts. */
int oracle_init_state(const mpcd_config *cfg, const mpcd_init_params *p, int max_attempts,
                      double *Q, double *V, double *U, int *spid, double *kbtnow) {
    const int dim = cfg->dim;
    int XYZ[3], i, j, d, s, n = 0;
    for (d = 0; d < 3; d++) XYZ[d] = d < dim ? cfg->L[d] : 1;
    for (s = 0; s < cfg->n_species; s++) n += p->population[s];
    /* setcoord: species in order, then place/push/orient */
    double AVV[3] = {0.0, 0.0, 0.0};
    int k = 0;
    for (s = 0; s < cfg->n_species; s++)
        for (j = 0; j < p->population[s]; j++) spid[k++] = s;
    for (i = 0; i < n; i++) {
        double *q = Q + 3 * i, *v = V + 3 * i, *u = U ? U + 3 * i : NULL;
        for (d = 0; d < 3; d++) {
            q[d] = 0.0;
            v[d] = 0.0;
            if (u) u[d] = 0.0;
        }
        for (d = 0; d < dim; d++) q[d] = init_u(cfg, MPCD_STREAM_INIT_POS, i, d) * XYZ[d];
        push_velocity(cfg, dim, 0u, MPCD_STREAM_INIT_VEL, (uint32_t)i, 0u, p->vdist[spid[i]],
                      cfg->species[spid[i]].mass, v);
        for (d = 0; d < dim; d++) AVV[d] += v[d];
        if (u && cfg->lc) init_orient(cfg, dim, XYZ, i, p->odist[spid[i]], q, u);
    }
    for (d = 0; d < dim; d++) AVV[d] /= (double)n;
    /* checkplace for every particle: re-place while an interacting wall has
     * W <= TOL */
    for (i = 0; i < n; i++) {
        double *q = Q + 3 * i;
        int a, inside = 1;
        for (a = 0; a < max_attempts && inside; a++) {
            if (a > 0)
                for (d = 0; d < dim; d++)
                    q[d] = (double)XYZ[d] * init_u(cfg, MPCD_STREAM_INIT_POS, i, 4u * a + d);
            inside = 0;
            for (j = 0; j < cfg->n_walls && !inside; j++) {
                const mpcd_wall *wl = &cfg->walls[j];
                if (!wl->inter[spid[i]]) continue;
                double W = 0.0;
                for (d = 0; d < dim; d++) W += wl->A[d] * (q[d] - wl->Q[d]);
                W -= wl->R;
                if (wl->inv) W *= -1.0;
                if (W <= TOL) inside = 1;
            }
        }
        if (inside) return -1;
    }
    /* galileantrans with VEL = AVV */
    if (p->rframe && n > 2) {
        double NET[3] = {0.0, 0.0, 0.0}, totM = 0.0;
        for (i = 0; i < n; i++) {
            double M = cfg->species[spid[i]].mass;
            totM += M;
            for (d = 0; d < dim; d++) NET[d] += M * V[3 * i + d];
        }
        for (d = 0; d < dim; d++) NET[d] /= totM;
        for (d = 0; d < dim; d++) NET[d] -= AVV[d];
        for (i = 0; i < n; i++)
            for (d = 0; d < dim; d++) V[3 * i + d] -= NET[d];
    }
    /* TEMP about AVV (therm.c:209-235), then VSC: V *= sqrt(KBT/KBTNOW) */
    for (int pass = 0; pass < 2; pass++) {
        double KBT = 0.0;
        for (i = 0; i < n; i++) {
            const double *v = V + 3 * i;
            double t = (v[0] - AVV[0]) * (v[0] - AVV[0]);
            t += (v[1] - AVV[1]) * (v[1] - AVV[1]);
            t += (v[2] - AVV[2]) * (v[2] - AVV[2]);
            KBT += cfg->species[spid[i]].mass * t;
        }
        KBT /= (double)(n * dim);
        if (pass == 1) {
            if (kbtnow) *kbtnow = KBT;
            break;
        }
        if (KBT > 0.0) {
            double TSC = sqrt(cfg->kbt / KBT);
            for (i = 0; i < n; i++)
                for (d = 0; d < dim; d++) V[3 * i + d] *= TSC;
        }
    }
    return 0;
}

long oracle_bounce_limit(const oracle_t *o) { return o->bounce_limit; }
