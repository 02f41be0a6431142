// mpcd_fp64.cuh -- the plain-FP64 form of the solvent timestep.
//
// State: structure-of-arrays doubles (q[3], v[3]) plus the particle's
// original index (pid, keys every per-particle draw and the download order)
// and its species.  Each step is a counting sort of the particles by cell of
// the randomly shifted grid followed by one warp per cell:
//
//   k_bin      grid shift + key + per-cell count (+ acceleration)
//   k_scan_*   exclusive scan of the counts -> cell start offsets
//   k_scatter  reorder the state into cell order (second buffer)
//   k_cell     per cell: moments, phantom particles, collision, global sums,
//              shift back, stream, walls
#pragma once

#include "mpcd_device.cuh"

namespace mpcd {

struct Fp64State {
    double *q[3];
    double *v[3];
    int *pid;
    int *sp;  // species (nullptr when there is one species)
};

constexpr int kScanTile = 2048;  // cells per scan block (256 threads x 8)

template <int DIM>
__global__ void __launch_bounds__(256) k_bin_fp64(const __grid_constant__ DevCfg c,
                                                  Fp64State st, int n, int *key,
                                                  int *rank, int *count, uint32_t step,
                                                  unsigned long long *status) {
    double s[3] = {0, 0, 0};
    if (c.galinv) mpcd_rng_shift(c.seed, c.replica, step, DIM, s);
    int esc_local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int idx[3] = {0, 0, 0};
        int esc = 0;
        for (int d = 0; d < DIM; d++) {
            double q = shift_fwd(st.q[d][i], s[d], c.L[d]);
            st.q[d][i] = q;
            idx[d] = bin_axis(q, c.L[d], c.pbc[d], 1, esc);
        }
        esc_local += esc;
        int k = cell_lin(c, idx[0], idx[1], idx[2]);
        key[i] = k;
        rank[i] = atomicAdd(&count[k], 1);
        if (c.grav_flag)
            for (int d = 0; d < DIM; d++) st.v[d][i] = st.v[d][i] + c.dt * c.grav[d];
    }
    if (esc_local) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc_local);
}

// Block-wide exclusive scan of one int per thread (256 threads).
__device__ __forceinline__ int block_excl_scan256(int x, int &total) {
    __shared__ int warp_tot[8];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    int wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        int t = warp_tot[w];
        if (w < wid) wpre += t;
        tot += t;
    }
    __syncthreads();
    total = tot;
    return wpre + incl - x;
}

// Sum of each tile of counts.
__global__ void __launch_bounds__(256) k_scan_partial(const int *count, int ncells,
                                                      int *part) {
    int base = blockIdx.x * kScanTile;
    int local = 0;
    for (int j = threadIdx.x; j < kScanTile; j += 256) {
        int idx = base + j;
        if (idx < ncells) local += count[idx];
    }
    int tot;
    block_excl_scan256(local, tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// Exclusive scan of the counts into start[0..ncells]; zeroes the counts for
// the next step and the per-step accumulators.
__global__ void __launch_bounds__(256) k_scan_apply(int *count, int ncells,
                                                    const int *part, int *start,
                                                    double *acc) {
    __shared__ int s_off;
    if (threadIdx.x == 0) {
        int off = 0;
        for (int b = 0; b < (int)blockIdx.x; b++) off += part[b];
        s_off = off;
    }
    if (blockIdx.x == 0 && threadIdx.x < ACC_WORDS) acc[threadIdx.x] = 0.0;
    __syncthreads();
    int base = blockIdx.x * kScanTile + threadIdx.x * 8;
    int v[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        int idx = base + j;
        v[j] = idx < ncells ? count[idx] : 0;
        sum += v[j];
    }
    int tot;
    int pre = block_excl_scan256(sum, tot) + s_off;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        int idx = base + j;
        if (idx < ncells) {
            start[idx] = pre;
            count[idx] = 0;
        }
        pre += v[j];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 255) start[ncells] = pre;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_scatter_fp64(Fp64State a, Fp64State b, int n,
                                                      const int *key, const int *rank,
                                                      const int *start) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int dst = start[key[i]] + rank[i];
        for (int d = 0; d < DIM; d++) {
            b.q[d][dst] = a.q[d][i];
            b.v[d][dst] = a.v[d][i];
        }
        b.pid[dst] = a.pid[i];
        if (a.sp) b.sp[dst] = a.sp[i];
    }
}

// One warp per cell of the shifted grid.
template <int DIM>
__global__ void __launch_bounds__(256) k_cell_fp64(const __grid_constant__ DevCfg c,
                                                   Fp64State st, const int *start,
                                                   uint32_t step, double *acc,
                                                   unsigned long long *status) {
    __shared__ double s_acc[ACC_WORDS];
    if (threadIdx.x < ACC_WORDS) s_acc[threadIdx.x] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    double s[3] = {0, 0, 0};
    if (c.galinv) mpcd_rng_shift(c.seed, c.replica, step, DIM, s);
    double ke = 0.0;
    int bounce = 0;
    if (cell < c.ncells) {
        const int b0 = start[cell], e0 = start[cell + 1], pop = e0 - b0;
        const bool need_cm = (c.op == MPCD_COLL_RAT);
        // ---- moments (localPROP) ----
        double M = 0.0, pv[3] = {0, 0, 0}, pq[3] = {0, 0, 0};
        for (int j = b0 + lane; j < e0; j += 32) {
            int sp = st.sp ? st.sp[j] : 0;
            double m = c.mass[sp];
            M += m;
            for (int d = 0; d < DIM; d++) {
                pv[d] += st.v[d][j] * m;
                if (need_cm) pq[d] += st.q[d][j] * m;
            }
        }
        M = warp_sum(M);
        double u[3] = {0, 0, 0}, cm[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) {
            u[d] = warp_sum(pv[d]);
            if (need_cm) cm[d] = warp_sum(pq[d]);
            if (M > 0.0) {
                u[d] /= M;
                if (need_cm) cm[d] /= M;
            }
        }
        // ---- phantom particles (ghostPart momentum) ----
        if (c.any_phantom && pop > 0 && pop < c.gndnst) {
            int a, b, z;
            cell_coords(c, cell, a, b, z);
            if (cell_cut_by_phantom<DIM>(c, a, b, z, s)) {
                double invN = 1.0 / (c.gndnst - (double)pop);
                double sig = sqrt(c.kbt / invN);
                for (int d = 0; d < DIM; d++) {
                    float g = mpcd_rng_normal(c.seed, c.replica, step, MPCD_STREAM_GHOST,
                                              (uint32_t)cell, (uint32_t)d);
                    u[d] += sig * (double)g;
                    u[d] /= c.gndnst;
                }
            }
        }
        if (lane == 0)
            for (int d = 0; d < DIM; d++) atomicAdd(&s_acc[ACC_VCM + d], u[d]);
        // ---- collision ----
        if (pop > 1) {
            if (c.op == MPCD_COLL_ARBAXIS) {
                double L[3] = {0, 0, 1}, R[9];
                if (DIM == 3) mpcd_rng_axis3(c.seed, c.replica, step, (uint32_t)cell, L);
                srd_matrix<DIM, double>(c, L, R);
                for (int j = b0 + lane; j < e0; j += 32) {
                    double w[3] = {0, 0, 0}, t[3] = {0, 0, 0};
                    for (int d = 0; d < DIM; d++) w[d] = st.v[d][j] - u[d];
                    for (int x = 0; x < DIM; x++)
                        for (int y = 0; y < DIM; y++) t[x] += R[x * 3 + y] * w[y];
                    for (int d = 0; d < DIM; d++) st.v[d][j] = u[d] + t[d];
                }
            } else {
                // Andersen (MPCAT / RAT): RS = sum m RV / M
                double rs[3] = {0, 0, 0};
                for (int j = b0 + lane; j < e0; j += 32) {
                    int sp = st.sp ? st.sp[j] : 0;
                    double rv[3];
                    thermal<DIM>(c, step, (uint32_t)st.pid[j], sp, rv);
                    for (int d = 0; d < DIM; d++) rs[d] += c.mass[sp] * rv[d];
                }
                for (int d = 0; d < DIM; d++) rs[d] = warp_sum(rs[d]) / M;
                double W[3] = {0, 0, 0};
                if (c.op == MPCD_COLL_RAT) {
                    // inertia about CM and angular momentum of (v - RV)
                    double I6[6] = {0, 0, 0, 0, 0, 0}, Lm[3] = {0, 0, 0};
                    for (int j = b0 + lane; j < e0; j += 32) {
                        int sp = st.sp ? st.sp[j] : 0;
                        double m = c.mass[sp];
                        double r[3] = {0, 0, 0}, rv[3], dv[3] = {0, 0, 0}, am[3];
                        thermal<DIM>(c, step, (uint32_t)st.pid[j], sp, rv);
                        for (int d = 0; d < DIM; d++) {
                            r[d] = st.q[d][j] - cm[d];
                            dv[d] = m * (st.v[d][j] - rv[d]);
                        }
                        I6[0] += m * (r[1] * r[1] + r[2] * r[2]);
                        I6[1] += m * (r[0] * r[0] + r[2] * r[2]);
                        I6[2] += m * (r[0] * r[0] + r[1] * r[1]);
                        I6[3] += m * r[0] * r[1];
                        I6[4] += m * r[0] * r[2];
                        I6[5] += m * r[1] * r[2];
                        cross3(r, dv, am);
                        for (int d = 0; d < 3; d++) Lm[d] += am[d];
                    }
                    for (int k = 0; k < 6; k++) I6[k] = warp_sum(I6[k]);
                    for (int d = 0; d < 3; d++) Lm[d] = warp_sum(Lm[d]);
                    double II[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                    if (DIM == 3) {
                        if (pop >= 3) {
                            double I[9] = {I6[0], -I6[3], -I6[4], -I6[3], I6[1],
                                           -I6[5], -I6[4], -I6[5], I6[2]};
                            inv3(I, II);
                        }
                    } else {
                        II[8] = 1. / I6[2];
                    }
                    for (int x = 0; x < 3; x++)
                        for (int y = 0; y < 3; y++) W[x] += II[x * 3 + y] * Lm[y];
                }
                for (int j = b0 + lane; j < e0; j += 32) {
                    int sp = st.sp ? st.sp[j] : 0;
                    double rv[3];
                    thermal<DIM>(c, step, (uint32_t)st.pid[j], sp, rv);
                    double damp = c.damp[sp];
                    if (c.op == MPCD_COLL_MPCAT) {
                        for (int d = 0; d < DIM; d++)
                            st.v[d][j] = u[d] + rv[d] - rs[d] - damp * u[d] / (double)pop;
                    } else {
                        double r[3] = {0, 0, 0}, ang[3];
                        for (int d = 0; d < DIM; d++) r[d] = st.q[d][j] - cm[d];
                        cross3(W, r, ang);
                        for (int d = 0; d < DIM; d++)
                            st.v[d][j] = u[d] + rv[d] - rs[d] - damp * u[d] + ang[d];
                    }
                }
            }
        }
        // ---- TEMP, shift back, stream, walls ----
        for (int j = b0 + lane; j < e0; j += 32) {
            int sp = st.sp ? st.sp[j] : 0;
            double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
            for (int d = 0; d < DIM; d++) {
                v[d] = st.v[d][j];
                q[d] = shift_back(st.q[d][j], s[d], c.L[d]);
            }
            double t = v[0] * v[0];
            t += v[1] * v[1];
            t += v[2] * v[2];
            ke += c.mass[sp] * t;
            for (int d = 0; d < DIM; d++) q[d] = q[d] + c.dt * v[d];
            bounce += wall_collisions<DIM>(c, q, v, sp, false);
            for (int d = 0; d < DIM; d++) {
                st.q[d][j] = q[d];
                st.v[d][j] = v[d];
            }
        }
    }
    ke = warp_sum(ke);
    if (lane == 0) atomicAdd(&s_acc[ACC_KE], ke);
    if (bounce) atomicAdd(&status[ST_BOUNCE], (unsigned long long)bounce);
    __syncthreads();
    if (threadIdx.x < ACC_WORDS) atomicAdd(&acc[threadIdx.x], s_acc[threadIdx.x]);
}

}  // namespace mpcd
