// mpcd_xfer.cuh -- device-side conversions between the caller's layout and
// the handle's state, and the per-cell quantities read back for output.
//
//   k_f64_from_aos (k_mix_from_f64 in mpcd_mixed.cuh for the mixed form)
//        the reference's particle arrays (3 doubles per vector, original
//        particle order, SRDclss.h:34-44) to the state;
//   k_inv_pid_* + k_*_gather_aos  back: the inverse of the state's order,
//        then a gather in the original order (coalesced writes; components
//        beyond DIM and the orientation's third are 0; species ids on
//        request);
//   k_pop_unshifted + k_gndnst_reduce  the initial binning on the unshifted
//        grid and the global number density GnDNST (globalDensities,
//        init.c:1002-1018): the mean population of the occupied cells of the
//        L^D box (the extra layer excluded), as integer counts.
//   k_props_*  the end-of-step re-bin on the unshifted grid and localPROP's
//        POP, MASS, VCM, CM and per-species populations per cell
//        (mpc.c:4936-4942, 64-216), which the reference's output writers
//        read (pout.c:640-1757); k_flow_add the flow field's running sum.
//   k_counts_*  the populations of the cells of the next step's shifted grid
//        exactly as the step's own kernels hold them (the sort's starts, the
//        resident families' population sums), for parity checks.
#pragma once

#include "mpcd_fp64.cuh"
#include "mpcd_mixed.cuh"

namespace mpcd {

// Caller arrays (AoS) -> FP64 state.  A non-finite position or velocity or
// a species id out of range counts in *err and leaves that particle
// unwritten (the upload is then rejected).  Without U, a nematic state
// starts every orientation at (1, 0).
template <int DIM>
__global__ void __launch_bounds__(256) k_f64_from_aos(Fp64State s, const __grid_constant__ DevCfg c,
                                                      int n, const double *Q, const double *V,
                                                      const double *U, const int *spid,
                                                      int *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        bool ok = true;
        double q[3], v[3];
        for (int d = 0; d < DIM; d++) {
            q[d] = Q[3 * (size_t)i + d];
            v[d] = V[3 * (size_t)i + d];
            ok = ok && isfinite(q[d]) && isfinite(v[d]);
        }
        const int sp = spid ? spid[i] : 0;
        if (sp < 0 || sp >= c.n_species) ok = false;
        if (!ok) {
            atomicAdd(err, 1);
            continue;
        }
        for (int d = 0; d < DIM; d++) {
            s.q[d][i] = q[d];
            s.v[d][i] = v[d];
        }
        s.pid[i] = i;
        if (s.sp) s.sp[i] = sp;
        if (s.u[0]) {
            s.u[0][i] = U ? U[3 * (size_t)i] : 1.0;
            s.u[1][i] = U ? U[3 * (size_t)i + 1] : 0.0;
        }
    }
}

// The inverse of the state's order: inv[pid] = slot for every slot (a
// scatter of 4-byte indices), so that a download can gather each caller-order
// record and write the caller's arrays with coalesced stores.  An original
// index out of range counts in *err.
__global__ void __launch_bounds__(256) k_inv_pid_f64(const int *pid, int n, int *inv, int *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = pid[i];
        if (p < 0 || p >= n) {
            atomicAdd(err, 1);
            continue;
        }
        inv[p] = i;
    }
}
__global__ void __launch_bounds__(256) k_inv_pid_mix(const float4 *W, int n, int *inv, int *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = __float_as_int(W[i].w);
        if (p < 0 || p >= n) {
            atomicAdd(err, 1);
            continue;
        }
        inv[p] = i;
    }
}

// FP64 state -> caller arrays (AoS), gathered through inv (caller index ->
// slot; a slot outside [0, n), which only a corrupted state leaves, counts
// in *err).
template <int DIM>
__global__ void __launch_bounds__(256) k_f64_gather_aos(Fp64State s, int n, const int *inv,
                                                        double *Q, double *V, double *U,
                                                        int *spo, int *err) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int i = inv[p];
        if (i < 0 || i >= n) {
            atomicAdd(err, 1);
            continue;
        }
        const size_t o = 3 * (size_t)p;
        for (int d = 0; d < 3; d++) {
            Q[o + d] = d < DIM ? s.q[d][i] : 0.0;
            V[o + d] = d < DIM ? s.v[d][i] : 0.0;
        }
        if (U) {
            U[o] = s.u[0] ? s.u[0][i] : 0.0;
            U[o + 1] = s.u[0] ? s.u[1][i] : 0.0;
            U[o + 2] = 0.0;
        }
        if (spo) spo[p] = s.sp ? s.sp[i] : 0;
    }
}

// Mixed state -> caller arrays (AoS, FP64), gathered through inv.
__global__ void __launch_bounds__(256) k_mix_gather_aos(MixState s, const __grid_constant__ DevCfg c,
                                                        int n, const int *inv, double *Q,
                                                        double *V, double *U, int *spo,
                                                        int *err) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int i = inv[p];
        if (i < 0 || i >= n) {
            atomicAdd(err, 1);
            continue;
        }
        int ci[3];
        uint32_t f[3];
        pos_unpack(s.P[i], ci, f);
        const float4 w = s.W[i];
        const float v[3] = {w.x, w.y, w.z};
        const size_t o = 3 * (size_t)p;
        for (int d = 0; d < 3; d++) {
            Q[o + d] = d < c.dim ? (double)ci[d] + (double)f[d] * kFxInv : 0.0;
            V[o + d] = d < c.dim ? (double)v[d] : 0.0;
        }
        if (U) {
            const float2 u = s.U ? s.U[i] : make_float2(0.f, 0.f);
            U[o] = (double)u.x;
            U[o + 1] = (double)u.y;
            U[o + 2] = 0.0;
        }
        if (spo) spo[p] = s.sp ? s.sp[i] : 0;
    }
}

// Unshifted cell of a caller position (truncation, clamped to the grid, as
// the initial binning that globalDensities reads), from the staged FP64
// positions of an upload, counted into count[] (zero at rest).
__global__ void __launch_bounds__(256) k_pop_unshifted(const __grid_constant__ DevCfg c, int n,
                                                       const double *Q, int *count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int idx[3] = {0, 0, 0};
        for (int d = 0; d < c.dim; d++) {
            int a = (int)Q[3 * (size_t)i + d];
            if (a < 0) a = 0;
            if (a > c.L[d]) a = c.L[d];
            idx[d] = a;
        }
        atomicAdd(&count[cell_lin(c, idx[0], idx[1], idx[2])], 1);
    }
}

// Occupied cells of the L^D box and their particles (out[0], out[1]); the
// counts are cleared again for the sort that shares them.
__global__ void __launch_bounds__(256) k_gndnst_reduce(const __grid_constant__ DevCfg c,
                                                       int *count, unsigned long long *out) {
    __shared__ unsigned long long red[2][8];
    unsigned long long occ = 0, sum = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c.ncells; k += gridDim.x * blockDim.x) {
        const int p = count[k];
        count[k] = 0;
        int a, b, z;
        cell_coords(c, k, a, b, z);
        if (a < c.L[0] && b < c.L[1] && z < c.L[2] && p > 0) {
            occ += 1ull;
            sum += (unsigned long long)p;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        occ += __shfl_xor_sync(0xffffffffu, occ, o);
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = occ;
        red[1][w] = sum;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        unsigned long long t = 0;
        for (int j = 0; j < 8; j++) t += red[threadIdx.x][j];
        atomicAdd(&out[threadIdx.x], t);
    }
}

// One particle's m v^2 / 2 (E = sum v_d^2, then times m/2, as enout).
__device__ __forceinline__ double kinetic_of(const DevCfg &c, const Fp64State &s, int i) {
    double e = 0.0;
    for (int d = 0; d < c.dim; d++) e += s.v[d][i] * s.v[d][i];
    return e * 0.5 * c.mass[s.sp ? s.sp[i] : 0];
}
__device__ __forceinline__ double kinetic_of(const DevCfg &c, const MixState &s, int i) {
    const float4 w = s.W[i];
    const double v[3] = {(double)w.x, (double)w.y, (double)w.z};
    double e = 0.0;
    for (int d = 0; d < c.dim; d++) e += v[d] * v[d];
    return e * 0.5 * c.mass[s.sp ? s.sp[i] : 0];
}

// Per-cell output properties on the unshifted grid: the accumulators.
struct CellProps {
    int *pop;
    double *mass;  // [nc]
    double *sv;    // [3 nc]: sum m v, then VCM
    double *sq;    // [3 nc]: sum m Q, then CM
    int *spc;      // [n_species nc]: populations per species (null: one species)
};

// One particle's contribution: its cell by truncation (clamped), as bin(...,
// 0) (mpc.c:958-982, no periodic L -> 0 on the unshifted grid).
template <int DIM>
__device__ __forceinline__ void props_add(const DevCfg &c, CellProps p, const double q[3],
                                          const double v[3], int sp) {
    const double m = c.mass[sp];
    int idx[3] = {0, 0, 0};
    for (int d = 0; d < DIM; d++) {
        int a = (int)q[d];
        if (a < 0) a = 0;
        if (a > c.L[d]) a = c.L[d];
        idx[d] = a;
    }
    const int k = cell_lin(c, idx[0], idx[1], idx[2]);
    atomicAdd(&p.pop[k], 1);
    if (p.spc) atomicAdd(&p.spc[(size_t)sp * c.ncells + k], 1);
    atomicAdd(&p.mass[k], m);
    for (int d = 0; d < DIM; d++) {
        atomicAdd(&p.sv[3 * (size_t)k + d], v[d] * m);
        atomicAdd(&p.sq[3 * (size_t)k + d], q[d] * m);
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_props_f64(const __grid_constant__ DevCfg c, Fp64State s,
                                                   int n, CellProps p) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) {
            q[d] = s.q[d][i];
            v[d] = s.v[d][i];
        }
        props_add<DIM>(c, p, q, v, s.sp ? s.sp[i] : 0);
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_props_mix(const __grid_constant__ DevCfg c, MixState s,
                                                   int n, CellProps p) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int ci[3];
        uint32_t f[3];
        pos_unpack(s.P[i], ci, f);
        const float4 w = s.W[i];
        const float wv[3] = {w.x, w.y, w.z};
        double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) {
            // the position the download returns (exact in FP64)
            q[d] = (double)ci[d] + (double)f[d] * kFxInv;
            v[d] = (double)wv[d];
        }
        props_add<DIM>(c, p, q, v, s.sp ? s.sp[i] : 0);
    }
}

// VCM = sum m v / M and CM = sum m Q / M in place (localPROP's divisions);
// empty cells keep zeros.
__global__ void __launch_bounds__(256) k_props_finish(const __grid_constant__ DevCfg c,
                                                      CellProps p) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c.ncells; k += gridDim.x * blockDim.x) {
        const double M = p.mass[k];
        if (!(M > 0.0)) continue;
        for (int d = 0; d < c.dim; d++) {
            p.sv[3 * (size_t)k + d] /= M;
            p.sq[3 * (size_t)k + d] /= M;
        }
    }
}

// FLOW += VCM over every cell of the (L+1)^D grid (sumFLOW, mpc.c:241-246,
// after localFLOW's per-cell centre-of-mass velocity, mpc.c:226-231 and
// 3889-3910, which equals localPROP's VCM for MPCD particles alone).
__global__ void __launch_bounds__(256) k_flow_add(const __grid_constant__ DevCfg c,
                                                  const double *vcm, double *flow) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c.ncells; k += gridDim.x * blockDim.x)
        for (int d = 0; d < c.dim; d++) flow[3 * (size_t)k + d] += vcm[3 * (size_t)k + d];
}

// Sum of m v^2 / 2 over the particles (per-block sums, one FP64 atomic per
// block).
template <class S>
__global__ void __launch_bounds__(256) k_kinetic(const __grid_constant__ DevCfg c, S s, int n,
                                                 double *out) {
    __shared__ double red[8];
    double e = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        e += kinetic_of(c, s, i);
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        atomicAdd(out, t);
    }
}

// Populations of the cells of a step's shifted grid from the counting
// sort's starts.
__global__ void __launch_bounds__(256) k_counts_start(const int *start, int nc, int *out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x)
        out[k] = start[k + 1] - start[k];
}
// ... from the mixed resident family's population plane (64-bit words).
__global__ void __launch_bounds__(256) k_counts_plane(const long long *n_plane, int nc, int *out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x)
        out[k] = (int)n_plane[k];
}
// ... from the FP64 resident family's sums: the counted populations
// (several species), or, as its cell pass takes them with one species, the
// mass sum over the mass.
__global__ void __launch_bounds__(256) k_counts_r64(const double *M, const int *pop, double mass,
                                                    int nc, int *out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x)
        out[k] = pop ? pop[k] : (int)llrint(M[k] / mass);
}

}  // namespace mpcd
