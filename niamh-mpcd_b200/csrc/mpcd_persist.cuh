// mpcd_persist.cuh -- the FP64 solvent timestep of a small box in one
// persistent kernel launch: every step of an mpcd_step call, the particles
// held in shared memory throughout (MPCD_KERNEL_PERSIST).
//
// A box of some ten thousand particles is too small to keep a B200 busy
// kernel by kernel: a step of the other families is a handful of launches of
// a few microseconds each, so such a box is bound by launch latency.  Here
// one cooperative launch of G blocks (at most one per SM, all resident at
// once) loads the box, runs nsteps steps, and writes it back:
//   - block b holds particles [b*chunk, (b+1)*chunk) of the state in its
//     shared memory (positions, velocities, id, species, and per step the
//     cell, the shifted position and the thermal velocities of this step and
//     the next);
//   - the cells' moment sums and collision records are small global arrays
//     that stay in L2; cell k is turned from sums into a record by block
//     k % G;
//   - each step is three phases between two grid barriers:
//       cells      localPROP, ghostPart and the operator's cell parameters
//                  (mpc.c:64-216, 351-567, 1181-1657), avVel; the blocks'
//                  other threads draw their particles' thermal velocities of
//                  the next step meanwhile;
//       particles  the collision, TEMP, shift back, stream, walls
//                  (MPC_BCcollision), then the next step's shift
//                  (gridShift_all), binning, acc_all and the particle's raw
//                  moments added to its cell's sums with FP64 reductions in
//                  L2 (mpc.c:4567-4621).
// The moments are taken about the corner of the particle's shifted cell
// (position minus the integer cell index, an exact subtraction), so the
// centre of mass, the inertia tensor about it and the angular momentum follow
// from them with little cancellation; they agree with localPROP's two-pass
// sums over absolute positions to rounding.
// The grid barrier is a counter in global memory; each wait on it is bounded
// (kBarrierSpins), after which the block counts a sync timeout in the status
// words and carries on (the step's results are then invalid, and reported
// so).  The cooperative launch guarantees that every block is resident, so
// in normal operation every wait ends.
// Every draw is the counter-based one of the other families (keyed by the
// particle's original index and the step), so the trajectory is theirs.
#pragma once

#include "mpcd_tile.cuh"

namespace mpcd {

#ifndef MPCD_PER_THREADS
#define MPCD_PER_THREADS 256
#endif
constexpr int kPerThreads = MPCD_PER_THREADS;
constexpr long long kBarrierSpins = 1ll << 24;  // each ~0.1 us or more: seconds in all

// Moment sums per cell (index into the sum rows), by operator:
//   SRD:      M, P[D]
//   MPC-AT:   M, P[D], R[D]                 (R = sum m RV)
//   MPC-AT+a: M, P[D], R[D], Q1[D], Q2, Lr  (Q1 = sum m q, Q2 = sum m q q
//             (3D: xx, yy, zz, xy, xz, yz; 2D: xx + yy), Lr = sum q x m (v - RV)
//             (3D: 3 components; 2D: z))
// with q the position relative to the shifted cell's corner.
template <int DIM>
struct PerQ {
    static constexpr int M = 0, P = 1, R = 1 + DIM, Q1 = 1 + 2 * DIM, Q2 = 1 + 3 * DIM;
    static constexpr int NQ2 = DIM == 3 ? 6 : 1;
    static constexpr int Lr = Q2 + NQ2;
    static constexpr int NL = DIM == 3 ? 3 : 1;
    static __host__ __device__ constexpr int nq(int op) {
        return is_vcm_op(op)
                   ? 1 + DIM
                   : (is_mpcat_op(op) || is_lang_op(op) ? 1 + 2 * DIM : Lr + NL);
    }
    // record: u[D], then SRD 3D: R[9]; Andersen: RS[D]; MPC-AT+a: CM[D], W[NL]
    static constexpr int U = 0, ROT = DIM, RS = DIM, CM = 2 * DIM, W = 3 * DIM;
    static __host__ __device__ constexpr int nr(int op) {
        return is_vcm_op(op) ? (DIM == 3 ? DIM + 9 : DIM)
                                       : (is_mpcat_op(op) || is_lang_op(op)
                                              ? 2 * DIM
                                              : 3 * DIM + NL);
    }
    // the most rows any operator uses (compile-time bounds of the unrolled
    // loads, so that the rows stay in registers and load together)
    static constexpr int NQMAX = Lr + NL;
    static constexpr int NRMAX = 3 * DIM + NL;
};
// rows of the largest operator (3D MPC-AT+a): the size of the global arrays
constexpr int kPerRowsMax = PerQ<3>::Lr + PerQ<3>::NL;
constexpr int kPerRecMax = 3 * 3 + PerQ<3>::NL;

// Shared-memory layout of one block (offsets in bytes).
struct PerLayout {
    int blocks;  // blocks of the launch
    int chunk;   // particles per block (the last may hold fewer)
    int nq, nr;  // sum and record rows of the operator
    int off_q, off_v, off_rv, off_rvn, off_k, off_ix, off_pid, off_sp;
    int off_red;
    int bytes;
};

template <int DIM>
inline PerLayout per_layout(int n, int op, int n_species, int blocks) {
    PerLayout l;
    l.blocks = blocks;
    l.chunk = (n + blocks - 1) / blocks;
    l.nq = PerQ<DIM>::nq(op);
    l.nr = PerQ<DIM>::nr(op);
    const bool andersen = !is_vcm_op(op);
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const int at = (int)o;
        o += (bytes + 15) / 16 * 16;
        return at;
    };
    const size_t ch = (size_t)l.chunk;
    l.off_q = take(ch * DIM * 8);
    l.off_v = take(ch * DIM * 8);
    l.off_rv = andersen ? take(ch * DIM * 8) : -1;
    l.off_rvn = andersen ? take(ch * DIM * 8) : -1;
    l.off_k = take(ch * 4);
    l.off_ix = take(ch * 4);
    l.off_pid = take(ch * 4);
    l.off_sp = n_species > 1 ? take(ch) : -1;
    l.off_red = take(64 * 8);
    l.bytes = (int)o;
    return l;
}

// The global working arrays: nq rows of ncells sums, the populations, nr
// rows of ncells record values and the records' populations, the barrier
// counter.
struct PerGlobal {
    double *sum;
    int *pop;
    double *rec;
    int *rpop;
    unsigned long long *bar;
    int ncells;
};

__device__ __forceinline__ double per_block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int j = 0; j < (int)(blockDim.x >> 5); j++) t += red[j];
    return t;  // thread 0 holds the block's sum
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier number `epoch` (1, 2, ...) of G blocks on a counter that was
// zero at the launch: every block's writes before it are visible to every
// block after it.  The wait is bounded; on timeout the block counts a sync
// timeout and carries on.
__device__ __forceinline__ void per_grid_sync(unsigned long long *bar, unsigned long long epoch,
                                              int blocks, unsigned long long *status) {
    __syncthreads();
    if (threadIdx.x == 0) {
        // arrival with release semantics: the block's writes before it (made
        // visible to this thread by the block barrier) are ordered before it
        asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(bar) : "memory");
        const unsigned long long target = epoch * (unsigned long long)blocks;
        long long spins = 0;
        while (ld_acquire_u64(bar) < target) {
            if (++spins > kBarrierSpins) {
                atomicAdd(&status[ST_SYNC], 1ull);
                break;
            }
            __nanosleep(32);
        }
    }
    __syncthreads();
}

// The thermal velocity of local particle j for `step` (Andersen), into
// `dst` (the rv or rvn rows).
template <int DIM>
__device__ __forceinline__ void per_draw(const DevCfg &c, const PerLayout &l, unsigned char *sm,
                                         int j, uint32_t step, double *dst) {
    const int *pid = (const int *)(sm + l.off_pid);
    const unsigned char *spa = l.off_sp >= 0 ? sm + l.off_sp : nullptr;
    double rv[3];
    thermal<DIM>(c, step, (uint32_t)pid[j], spa ? spa[j] : 0, rv);
    for (int d = 0; d < DIM; d++) dst[d * l.chunk + j] = rv[d];
}

// Entry of local particle j into a step: the shifted position and cell
// (gridShift_all + bin, mpc.c:720-766, 948-992), the gravity kick (acc_all,
// mpc.c:697-700), and the particle's raw moments (with its thermal velocity
// of the step, drawn already) added to its cell's sums.
template <int DIM>
__device__ __forceinline__ void per_enter(const DevCfg &c, const PerLayout &l, const PerGlobal &g,
                                          unsigned char *sm, int j, const double s[3],
                                          const double *rvrow, int &esc) {
    double *q = (double *)(sm + l.off_q), *v = (double *)(sm + l.off_v);
    int *kk = (int *)(sm + l.off_k), *ix = (int *)(sm + l.off_ix);
    const unsigned char *spa = l.off_sp >= 0 ? sm + l.off_sp : nullptr;
    const int sp = spa ? spa[j] : 0;
    const double m = c.mass[sp];
    using Q = PerQ<DIM>;
    double qs[3] = {0, 0, 0}, vv[3] = {0, 0, 0}, rel[3] = {0, 0, 0}, rv[3] = {0, 0, 0};
    int idx[3] = {0, 0, 0};
    for (int d = 0; d < DIM; d++) {
        qs[d] = shift_fwd(q[d * l.chunk + j], s[d], c.L[d]);
        idx[d] = bin_axis(qs[d], c.L[d], c.pbc[d], 1, esc);
        rel[d] = qs[d] - (double)idx[d];
        q[d * l.chunk + j] = qs[d];
        vv[d] = v[d * l.chunk + j];
        if (c.grav_flag) vv[d] = vv[d] + c.dt * c.grav[d];
        v[d * l.chunk + j] = vv[d];
        if (rvrow) rv[d] = rvrow[d * l.chunk + j];
    }
    const int k = cell_lin(c, idx[0], idx[1], idx[2]);
    kk[j] = k;
    ix[j] = idx[0] | (idx[1] << 10) | (idx[2] << 20);
    auto add = [&](int row, double x) { atomicAdd(g.sum + (size_t)row * g.ncells + k, x); };
    atomicAdd(g.pop + k, 1);
    add(Q::M, m);
    for (int d = 0; d < DIM; d++) add(Q::P + d, vv[d] * m);
    if (is_vcm_op(c.op)) return;
    // Langevin: the plain sum of the noise (langevinMPC, mpc.c:1707-1710)
    for (int d = 0; d < DIM; d++) add(Q::R + d, is_lang_op(c.op) ? rv[d] : rv[d] * m);
    if (c.op != MPCD_COLL_RAT) return;
    for (int d = 0; d < DIM; d++) add(Q::Q1 + d, rel[d] * m);
    double dv[3] = {0, 0, 0};
    for (int d = 0; d < DIM; d++) dv[d] = m * (vv[d] - rv[d]);
    if (DIM == 3) {
        add(Q::Q2 + 0, m * rel[0] * rel[0]);
        add(Q::Q2 + 1, m * rel[1] * rel[1]);
        add(Q::Q2 + 2, m * rel[2] * rel[2]);
        add(Q::Q2 + 3, m * rel[0] * rel[1]);
        add(Q::Q2 + 4, m * rel[0] * rel[2]);
        add(Q::Q2 + 5, m * rel[1] * rel[2]);
        double am[3];
        cross3(rel, dv, am);
        for (int d = 0; d < 3; d++) add(Q::Lr + d, am[d]);
    } else {
        add(Q::Q2, m * (rel[0] * rel[0] + rel[1] * rel[1]));
        add(Q::Lr, rel[0] * dv[1] - rel[1] * dv[0]);
    }
}

// Cell phase for cell k: the record from the sums, which are cleared;
// returns the cell's centre-of-mass velocity (avVel term).
template <int DIM>
__device__ __forceinline__ void per_cell(const DevCfg &c, const PerLayout &l, const PerGlobal &g,
                                         int k, uint32_t step, const double s[3], double u[3]) {
    using Q = PerQ<DIM>;
    // the sums, read from L2 (every SM added to them), then cleared for the
    // next step
    double x[Q::NQMAX];
#pragma unroll
    for (int r = 0; r < Q::NQMAX; r++) x[r] = r < l.nq ? __ldcg(g.sum + (size_t)r * g.ncells + k) : 0.0;
    const int n = __ldcg(g.pop + k);
#pragma unroll
    for (int r = 0; r < Q::NQMAX; r++)
        if (r < l.nq) g.sum[(size_t)r * g.ncells + k] = 0.0;
    g.pop[k] = 0;
    g.rpop[k] = n;
    auto put = [&](int row, double val) { g.rec[(size_t)row * g.ncells + k] = val; };
    const double M = x[Q::M];
    for (int d = 0; d < 3; d++) u[d] = 0.0;
    if (M > 0.0)
        for (int d = 0; d < DIM; d++) u[d] = x[Q::P + d] / M;
    int cc[3] = {0, 0, 0};
    if (c.any_phantom) cell_coords(c, k, cc[0], cc[1], cc[2]);
    // ghostPart's phantom fill (mpc.c:549-557, quirk Q4)
    if (c.any_phantom && n > 0 && n < c.gndnst &&
        cell_cut_by_phantom<DIM>(c, cc[0], cc[1], cc[2], s)) {
        const double invN = 1.0 / (c.gndnst - (double)n);
        const double sig = sqrt(c.kbt / invN);
        for (int d = 0; d < DIM; d++) {
            const float gd = mpcd_rng_normal(c.seed, c.replica, step, MPCD_STREAM_GHOST,
                                             (uint32_t)k, (uint32_t)d);
            u[d] += sig * (double)gd;
            u[d] /= c.gndnst;
        }
    }
    for (int d = 0; d < DIM; d++) put(Q::U + d, u[d]);
    if (is_vcm_op(c.op)) {
        if (DIM == 3) {
            double R[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (n > 1 && c.op != MPCD_COLL_VICSEK)
                srd_cell_matrix<DIM, double>(c, step, (uint32_t)k, R);
            for (int r = 0; r < 9; r++) put(Q::ROT + r, R[r]);
        }
        return;
    }
    double rs[3] = {0, 0, 0};
    if (n > 1)
        for (int d = 0; d < DIM; d++)
            rs[d] = x[Q::R + d] / (is_lang_op(c.op) ? (double)n : M);
    for (int d = 0; d < DIM; d++) put(Q::RS + d, rs[d]);
    if (c.op != MPCD_COLL_RAT) return;
    double cm[3] = {0, 0, 0}, W[3] = {0, 0, 0};
    if (M > 0.0)
        for (int d = 0; d < DIM; d++) cm[d] = x[Q::Q1 + d] / M;
    if (n > 1) {
        // angular momentum about the centre of mass: sum (q - cm) x m (v - RV)
        double pr[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) pr[d] = x[Q::P + d] - x[Q::R + d];
        if (DIM == 3) {
            double cx[3];
            cross3(cm, pr, cx);
            double Lm[3];
            for (int d = 0; d < 3; d++) Lm[d] = x[Q::Lr + d] - cx[d];
            if (n >= 3) {
                // moment of inertia about the centre of mass
                // (localMomInertiaTensor, mpc.c:4209-4299)
                const double sxx = x[Q::Q2 + 0] - M * cm[0] * cm[0];
                const double syy = x[Q::Q2 + 1] - M * cm[1] * cm[1];
                const double szz = x[Q::Q2 + 2] - M * cm[2] * cm[2];
                const double sxy = x[Q::Q2 + 3] - M * cm[0] * cm[1];
                const double sxz = x[Q::Q2 + 4] - M * cm[0] * cm[2];
                const double syz = x[Q::Q2 + 5] - M * cm[1] * cm[2];
                const double I[9] = {syy + szz, -sxy, -sxz, -sxy, sxx + szz, -syz,
                                     -sxz, -syz, sxx + syy};
                double II[9];
                inv3(I, II);
                for (int a = 0; a < 3; a++) {
                    double w = 0.0;
                    for (int b = 0; b < 3; b++) w += II[a * 3 + b] * Lm[b];
                    W[a] = w;
                }
            }
        } else {
            const double Lz = x[Q::Lr] - (cm[0] * pr[1] - cm[1] * pr[0]);
            const double Izz = x[Q::Q2] - M * (cm[0] * cm[0] + cm[1] * cm[1]);
            W[0] = (1. / Izz) * Lz;
        }
    }
    for (int d = 0; d < DIM; d++) put(Q::CM + d, cm[d]);
    for (int d = 0; d < Q::NL; d++) put(Q::W + d, W[d]);
}

// Collision of local particle j with its cell's record (rvv: the rows of
// this step's thermal velocities), then TEMP, shift back, streaming and
// walls (F64T::finish); the state is left unshifted.  Returns the particle's
// m v^2.
template <int DIM>
__device__ __forceinline__ double per_collide(const DevCfg &c, const PerLayout &l,
                                              const PerGlobal &g, unsigned char *sm, int j,
                                              const double s[3], const double *rvv,
                                              uint32_t step, int &bounce, int &esc) {
    using Q = PerQ<DIM>;
    double *q = (double *)(sm + l.off_q), *v = (double *)(sm + l.off_v);
    const int k = ((const int *)(sm + l.off_k))[j];
    const unsigned char *spa = l.off_sp >= 0 ? sm + l.off_sp : nullptr;
    const int sp = spa ? spa[j] : 0;
    // the record (written by another block): from L2
    double rc[Q::NRMAX];
#pragma unroll
    for (int r = 0; r < Q::NRMAX; r++) rc[r] = r < l.nr ? __ldcg(g.rec + (size_t)r * g.ncells + k) : 0.0;
    const int n = __ldcg(g.rpop + k);
    double vv[3] = {0, 0, 0}, qs[3] = {0, 0, 0};
    for (int d = 0; d < DIM; d++) {
        vv[d] = v[d * l.chunk + j];
        qs[d] = q[d * l.chunk + j];
    }
    if (n > 1) {
        double u[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) u[d] = rc[Q::U + d];
        if (c.op == MPCD_COLL_VICSEK) {
            const uint32_t pid = (uint32_t)((const int *)(sm + l.off_pid))[j];
            const double3 t = vicsek_cone(c.act[sp], DIM, c.seed, c.replica, step, pid,
                                          make_double3(u[0], u[1], u[2]),
                                          make_double3(vv[0], vv[1], vv[2]));
            vv[0] = t.x;
            vv[1] = t.y;
            vv[2] = t.z;
        } else if (is_vcm_op(c.op)) {
            double R[9];
            if (DIM == 3) {
                for (int r = 0; r < 9; r++) R[r] = rc[Q::ROT + r];
            } else {
                const double uu[3] = {0.0, 0.0, 1.0};
                srd_matrix<DIM, double>(c, uu, R);
            }
            double w[3] = {0, 0, 0}, t[3] = {0, 0, 0};
            for (int d = 0; d < DIM; d++) w[d] = vv[d] - u[d];
            for (int a = 0; a < DIM; a++)
                for (int b = 0; b < DIM; b++) t[a] += R[a * 3 + b] * w[b];
            for (int d = 0; d < DIM; d++) vv[d] = u[d] + t[d];
            if (c.act_srd) {
                const double3 t = active_srd_turn(c.act[sp], make_double3(u[0], u[1], u[2]),
                                                  make_double3(vv[0], vv[1], vv[2]));
                vv[0] = t.x;
                vv[1] = t.y;
                vv[2] = t.z;
            }
        } else {
            const double damp = c.damp[sp];
            double rv[3] = {0, 0, 0};
            for (int d = 0; d < DIM; d++) rv[d] = rvv[d * l.chunk + j];
            const double3 v0 = make_double3(vv[0], vv[1], vv[2]);
            if (is_lang_op(c.op) || is_vicsek_op(c.op)) {
                // the Vicsek-aligned MPC-AT takes this update with a = 0, b = 1
                // langevinMPC, mpc.c:1739-1750
                const double a = c.lang_a[sp], b = c.lang_b[sp];
                for (int d = 0; d < DIM; d++)
                    vv[d] = u[d] + a * (vv[d] - u[d]) + b * (rv[d] - rc[Q::RS + d]) -
                            damp * u[d] / (double)n;
                if (is_vicsek_op(c.op)) {
                    const double3 t = vicsek_term(c.relax, c.act[sp], DIM,
                                                  make_double3(u[0], u[1], u[2]), v0);
                    vv[0] += t.x;
                    vv[1] += t.y;
                    if (DIM == 3) vv[2] += t.z;
                }
            } else if (is_mpcat_op(c.op)) {
                // andersenMPC, mpc.c:1353-1444 (damping over POP)
                for (int d = 0; d < DIM; d++)
                    vv[d] = u[d] + rv[d] - rc[Q::RS + d] - damp * u[d] / (double)n;
            } else {
                // andersenROT, mpc.c:1461-1657 (damping not over POP)
                const int pix = ((const int *)(sm + l.off_ix))[j];
                const int idx[3] = {pix & 1023, (pix >> 10) & 1023, (pix >> 20) & 1023};
                double rr[3] = {0, 0, 0}, W[3] = {0, 0, 0}, ang[3];
                for (int d = 0; d < DIM; d++) rr[d] = (qs[d] - (double)idx[d]) - rc[Q::CM + d];
                if (DIM == 3)
                    for (int d = 0; d < 3; d++) W[d] = rc[Q::W + d];
                else
                    W[2] = rc[Q::W];
                cross3(W, rr, ang);
                for (int d = 0; d < DIM; d++)
                    vv[d] = u[d] + rv[d] - rc[Q::RS + d] - damp * u[d] + ang[d];
            }
        }
    }
    double t = vv[0] * vv[0];
    t += vv[1] * vv[1];
    t += vv[2] * vv[2];
    const double ke = c.mass[sp] * t;
    // shift back, stream, walls (F64T::finish)
    double qq[3] = {0, 0, 0};
    for (int d = 0; d < DIM; d++) {
        qq[d] = shift_back(qs[d], s[d], c.L[d]);
        qq[d] = qq[d] + c.dt * vv[d];
    }
    const uint32_t pid = (uint32_t)((const int *)(sm + l.off_pid))[j];
    bounce += wall_collisions<DIM, false>(c, qq, vv, sp, false, step, pid);
    if (left_grid(c, qq, DIM)) {
        // the reference's end-of-step re-bin re-places it (mpc.c:969-982)
        replace_escaped<DIM>(c, qq, vv, nullptr, sp, step, pid);
        esc++;
    }
    for (int d = 0; d < DIM; d++) {
        q[d * l.chunk + j] = qq[d];
        v[d * l.chunk + j] = vv[d];
    }
    return ke;
}

// nsteps steps from step0 of the whole box (n particles of state st, which
// is read at the start and written back in place at the end), as a
// cooperative launch of l.blocks blocks.  Per step: acc_ring[step % ring]
// gets the step's sum m v^2 and sum VCM.  At the end pop_out (zero at the
// launch) receives the populations of the cells of step step0 + nsteps's
// shifted grid.  Escapes are counted once per binning, as the other families
// count them: the binning of the next step at the end of each step, and the
// first step's own binning when count_first is set (no earlier launch
// counted it).  g.sum, g.pop and g.bar are zero at the launch; g.sum and
// g.pop are zero again at its end.
template <int DIM>
__global__ void __launch_bounds__(kPerThreads)
    k_persist(const __grid_constant__ DevCfg c, Fp64State st, int n, PerLayout l, PerGlobal g,
              uint32_t step0, int nsteps, double *acc_ring, int ring, int *pop_out,
              unsigned long long *status, int count_first) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int b = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const int p0 = b * l.chunk;
    const int np = max(0, min(l.chunk, n - p0));
    double *red = (double *)(sm + l.off_red);
    double *rv = l.off_rv >= 0 ? (double *)(sm + l.off_rv) : nullptr;
    double *rvn = l.off_rvn >= 0 ? (double *)(sm + l.off_rvn) : nullptr;
    unsigned long long epoch = 0;
    {
        double *q = (double *)(sm + l.off_q), *v = (double *)(sm + l.off_v);
        int *pid = (int *)(sm + l.off_pid);
        unsigned char *spa = l.off_sp >= 0 ? sm + l.off_sp : nullptr;
        for (int j = tid; j < np; j += nt) {
            for (int d = 0; d < DIM; d++) {
                q[d * l.chunk + j] = st.q[d][p0 + j];
                v[d * l.chunk + j] = st.v[d][p0 + j];
            }
            pid[j] = st.pid[p0 + j];
            if (spa) spa[j] = (unsigned char)(st.sp ? st.sp[p0 + j] : 0);
        }
        if (b == 0 && tid < ACC_WORDS)
            acc_ring[(size_t)(step0 % (uint32_t)ring) * ACC_WORDS + tid] = 0.0;
    }
    __syncthreads();
    int esc = 0, bounce = 0;
    double s[3] = {0, 0, 0};
    if (c.galinv) mpcd_rng_shift(c.seed, c.replica, step0, DIM, s);
    {
        int esc0 = 0;
        for (int j = tid; j < np; j += nt) {
            if (rv) per_draw<DIM>(c, l, sm, j, step0, rv);
            per_enter<DIM>(c, l, g, sm, j, s, rv, esc0);
        }
        if (count_first) esc += esc0;
    }
    per_grid_sync(g.bar, ++epoch, l.blocks, status);
    for (int it = 0; it < nsteps; it++) {
        const uint32_t step = step0 + (uint32_t)it;
        double *acc = acc_ring + (size_t)(step % (uint32_t)ring) * ACC_WORDS;
        const bool last = it + 1 == nsteps;
        // cells of this block; its particles' thermal velocities of the next
        // step meanwhile
        double av[3] = {0, 0, 0};
        for (int k = b + tid * l.blocks; k < c.ncells; k += nt * l.blocks) {
            double u[3];
            per_cell<DIM>(c, l, g, k, step, s, u);
            for (int d = 0; d < DIM; d++) av[d] += u[d];
        }
        if (rvn && !last)
            for (int j = tid; j < np; j += nt) per_draw<DIM>(c, l, sm, j, step + 1u, rvn);
        if (b == 0 && tid < ACC_WORDS)
            acc_ring[(size_t)((step + 1u) % (uint32_t)ring) * ACC_WORDS + tid] = 0.0;
        for (int d = 0; d < DIM; d++) {
            const double t = per_block_sum(av[d], red);
            if (tid == 0) atomicAdd(&acc[ACC_VCM + d], t);
        }
        per_grid_sync(g.bar, ++epoch, l.blocks, status);
        // particles: collide, stream, walls; then enter the next step
        double sn[3] = {0, 0, 0};
        if (c.galinv) mpcd_rng_shift(c.seed, c.replica, step + 1u, DIM, sn);
        double ke = 0.0;
        for (int j = tid; j < np; j += nt) {
            ke += per_collide<DIM>(c, l, g, sm, j, s, rv, step, bounce, esc);
            if (!last) per_enter<DIM>(c, l, g, sm, j, sn, rvn, esc);
        }
        const double t = per_block_sum(ke, red);
        if (tid == 0) atomicAdd(&acc[ACC_KE], t);
        for (int d = 0; d < 3; d++) s[d] = sn[d];
        double *sw = rv;  // the next step's draws become this step's
        rv = rvn;
        rvn = sw;
        if (!last) per_grid_sync(g.bar, ++epoch, l.blocks, status);
    }
    // the populations of the next step's cells, counted on the final state
    // (no kick or draw: the next launch enters that step itself)
    for (int j = tid; j < np; j += nt) {
        int idx[3] = {0, 0, 0};
        const double *q = (const double *)(sm + l.off_q);
        for (int d = 0; d < DIM; d++)
            idx[d] = bin_axis(shift_fwd(q[d * l.chunk + j], s[d], c.L[d]), c.L[d], c.pbc[d], 1,
                              esc);
        atomicAdd(&pop_out[cell_lin(c, idx[0], idx[1], idx[2])], 1);
    }
    // write the particles back in place
    {
        const double *q = (const double *)(sm + l.off_q), *v = (const double *)(sm + l.off_v);
        for (int j = tid; j < np; j += nt)
            for (int d = 0; d < DIM; d++) {
                st.q[d][p0 + j] = q[d * l.chunk + j];
                st.v[d][p0 + j] = v[d * l.chunk + j];
            }
    }
    if (esc) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc);
    if (bounce) atomicAdd(&status[ST_BOUNCE], (unsigned long long)bounce);
}

}  // namespace mpcd
