// mpcd_resident64.cuh -- SRD step of the FP64 form with the particles
// resident in place (MPCD_KERNEL_RESIDENT for MPCD_PREC_FP64).
//
// The same two-pass structure as the mixed resident family
// (mpcd_resident.cuh), with the FP64 form's arithmetic:
//   k_r64_cells  one thread per cell: u = (sum m v) / (sum m) from the FP64
//                sums of the previous particle pass, the random axis
//                (stochrotMPC, mpc.c:1275-1333), the avVel term; writes a
//                64-byte record {u, pop, axis} and clears the sums.
//   k_r64_parts  one thread per particle (one wave of blocks, each thread
//                striding over the particles): its cell on this step's grid
//                (recomputed from its position exactly as the split family
//                does), the rotation matrix from the record's axis (rotate,
//                mpc.c:1181-1257, the split family's srd_matrix), v' = u +
//                R (v - u), TEMP term, finish() (shift back,
//                stream, walls, next step's cell), the particle written back
//                in place, and its mass and momentum (with the next step's
//                gravity kick) added to its cell of the next step with FP64
//                atomics.
// The sums are FP64 additions in the order the atomics arrive, so they
// agree with the split family's sorted-order sums to rounding (about 1e-16
// relative); the state is re-sorted every few steps for locality only.
#pragma once

#include "mpcd_split.cuh"

namespace mpcd {

// FP64 cell sums: mass, mass-weighted momentum (with the step's gravity
// kick) and, with several species, population, one array each, so that the atomics of one cell's
// particles fall on different sectors (the L2 serialises atomics on one
// sector).  Each array holds nc entries.
struct R64Sums {
    double *M, *p[3];
    int *pop;
};

// A cell's record: two 32-byte sectors.  The particle pass builds the
// rotation matrix from the axis (the 9 doubles of the matrix would double
// the bytes every particle gathers).
struct __align__(64) R64Rec {
    double u[3];
    double pop;
    double L[3];
    double pad_;
};

template <int DIM>
__global__ void __launch_bounds__(256) k_r64_cells(const __grid_constant__ DevCfg c,
                                                   R64Sums sums, R64Rec *crec, StepArgs sa,
                                                   double *acc, double *acc_next) {
    __shared__ double red[8];
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    pdl_trigger();
    // the axis depends on the step and the cell only: drawn while the
    // particle pass before this kernel may still be running
    double Lx[3] = {0.0, 0.0, 1.0};
    if (DIM == 3 && cell < c.ncells) mpcd_rng_axis3(c.seed, c.replica, sa.step, (uint32_t)cell, Lx);
    pdl_wait();  // the sums are complete from here on
    if (blockIdx.x == 0 && threadIdx.x < ACC_WORDS) acc_next[threadIdx.x] = 0.0;
    double av[3] = {0.0, 0.0, 0.0};
    if (cell < c.ncells) {
        const double M = sums.M[cell];
        double p[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < DIM; d++) p[d] = sums.p[d][cell];
        // one species: the population is the mass sum over the mass (exact:
        // n equal terms, far below 2^52); several: the counted population
        const bool one = c.n_species == 1;
        const int pop = one ? (int)llrint(M / c.mass[0]) : sums.pop[cell];
        sums.M[cell] = 0.0;
        for (int d = 0; d < DIM; d++) sums.p[d][cell] = 0.0;
        if (!one) sums.pop[cell] = 0;
        double u[3] = {0.0, 0.0, 0.0};
        if (M > 0.0) {
            const double iM = 1.0 / M;
            for (int d = 0; d < DIM; d++) u[d] = p[d] * iM;
        }
        for (int d = 0; d < DIM; d++) av[d] = u[d];
        R64Rec rec;
        for (int d = 0; d < 3; d++) {
            rec.u[d] = u[d];
            rec.L[d] = Lx[d];
        }
        rec.pop = (double)pop;
        rec.pad_ = 0.0;
        crec[cell] = rec;
    }
    for (int d = 0; d < DIM; d++) {
        const double t = block_sum256(av[d], red);
        if (threadIdx.x == 0) atomicAdd(&acc[ACC_VCM + d], t);
    }
}

// RES_STEP: collide, stream, write back, add to the next step's sums.
// RES_SUM:  only add each particle to this step's sums (bootstrap).
// Four blocks of 256 threads per SM (64 registers, no spills).
#ifndef R64_MINB
#define R64_MINB 4
#endif
// OPEN: the box has a side without a periodic wall (see F64T::finish).
template <int DIM, int MODE, bool OPEN>
__global__ void __launch_bounds__(256, R64_MINB) k_r64_parts(const __grid_constant__ DevCfg c,
                                                   Fp64State a, int n, const R64Rec *crec,
                                                   R64Sums sums, double *acc,
                                                   unsigned long long *status, StepArgs sa) {
    __shared__ double red[8];
    pdl_trigger();
    pdl_wait();  // records, sums and particles are complete from here on
    double ke = 0.0;
    int bounce = 0, esc = 0;
    // one wave of blocks striding over the particles: the block-end
    // reduction and the block turnover are paid once per resident block
    // rather than once per 256 particles
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        // the particle stays in place, so its id is not written, and read
        // where walls may re-thermalise it or it may leave the grid (the
        // draws are keyed by the
        // id); otherwise as F64T::load: the shifted position and the
        // velocity with this step's kick
        F64Rec r;
        r.pid = (MODE == RES_STEP && !c.all_periodic) ? a.pid[i] : 0;
        for (int d = 0; d < 3; d++) {
            r.q[d] = d < DIM ? shift_fwd(a.q[d][i], sa.s[d], c.L[d]) : 0.0;
            r.v[d] = d < DIM ? a.v[d][i] : 0.0;
            if (d < DIM && c.grav_flag) r.v[d] = r.v[d] + c.dt * c.grav[d];
        }
        const int sp = F64T<DIM>::sp(a, i);
        int k;
        double v[3] = {0.0, 0.0, 0.0};
        if (MODE == RES_STEP) {
            const int kc = cur_key<DIM>(c, r, sa);
            const R64Rec cr = crec[kc];
            if (cr.pop > 1.0) {
                double R[9];
                srd_matrix<DIM, double>(c, cr.L, R);
                double w[3] = {0, 0, 0}, tt[3] = {0, 0, 0};
                for (int d = 0; d < DIM; d++) w[d] = r.v[d] - cr.u[d];
                for (int x = 0; x < DIM; x++)
                    for (int y = 0; y < DIM; y++) tt[x] += R[x * 3 + y] * w[y];
                for (int d = 0; d < DIM; d++) r.v[d] = cr.u[d] + tt[d];
            }
            double t = r.v[0] * r.v[0];
            t += r.v[1] * r.v[1];
            t += r.v[2] * r.v[2];
            ke += c.mass[sp] * t;
            k = F64T<DIM>::template finish<OPEN>(c, r, sp, sa, bounce, esc);
            for (int d = 0; d < DIM; d++) {
                a.q[d][i] = r.q[d];
                a.v[d][i] = r.v[d];
            }
            // the next step's cell pass sees the velocity with its kick
            for (int d = 0; d < DIM; d++)
                v[d] = c.grav_flag ? r.v[d] + c.dt * c.grav[d] : r.v[d];
        } else {
            k = cur_key<DIM>(c, r, sa);
            for (int d = 0; d < DIM; d++) v[d] = r.v[d];
        }
        const double m = c.mass[sp];
        atomicAdd(sums.M + k, m);
        for (int d = 0; d < DIM; d++) atomicAdd(sums.p[d] + k, v[d] * m);
        if (c.n_species > 1) atomicAdd(sums.pop + k, 1);
    }
    if (MODE == RES_STEP) {
        const double t = block_sum256(ke, red);
        if (threadIdx.x == 0) atomicAdd(&acc[ACC_KE], t);
        if (bounce) atomicAdd(&status[ST_BOUNCE], (unsigned long long)bounce);
    }
    if (esc) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc);
}

}  // namespace mpcd
