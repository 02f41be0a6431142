// mpcd_split.cuh -- SRD step as a cell pass and a particle pass.
//
// For the stochastic-rotation operator the collision of a particle needs only
// two per-cell quantities: the centre-of-mass velocity u and the rotation R.
// So the step is split into two simple, fully parallel kernels:
//   k_srd_cells  one thread per cell of the sorted order: FP64 mass/momentum
//                sums over its particles (localPROP, mpc.c:64-216), u, the
//                random axis and rotation matrix (stochrotMPC + rotate,
//                mpc.c:1181-1333), avVel term; writes a 64-byte (mixed) or
//                128-byte (FP64) cell record, which stays in L2.
//   k_srd_parts  one thread per particle: its cell key on this step's grid
//                (recomputed exactly from its position; it equals the key the
//                particles were sorted by), v' = u + R (v - u), TEMP term,
//                then finish() (shift back, stream, walls, next step's key)
//                and the write-out of the chosen strategy (MODE_*).
// No shared-memory staging and no block-wide phases: both kernels run at
// full occupancy and overlap memory latency across many warps.
#pragma once

#include "mpcd_tile.cuh"

namespace mpcd {

template <class T>
struct SrdCell;
// mixed: {u.x, u.y, u.z, pop} + R[9] (+3 pad) as four float4
template <int DIM>
struct SrdCell<MixT<DIM>> {
    struct Rec {
        float4 a, b, c, d;
    };
    static __device__ __forceinline__ void vel(const MixState &st, int i, const DevCfg &cf,
                                               double v[3]) {
        float4 w = st.W[i];
        if (cf.grav_flag) {
            w.x += (float)(cf.dt * cf.grav[0]);
            w.y += (float)(cf.dt * cf.grav[1]);
            if (DIM == 3) w.z += (float)(cf.dt * cf.grav[2]);
        }
        v[0] = w.x;
        v[1] = w.y;
        v[2] = DIM == 3 ? (double)w.z : 0.0;
    }
    static __device__ __forceinline__ void put(Rec *r, int c, const double *u, int pop,
                                               const float *R) {
        Rec x;
        x.a = make_float4((float)u[0], (float)u[1], (float)u[2], __int_as_float(pop));
        x.b = make_float4(R[0], R[1], R[2], R[3]);
        x.c = make_float4(R[4], R[5], R[6], R[7]);
        x.d = make_float4(R[8], 0.f, 0.f, 0.f);
        r[c] = x;
    }
};
// FP64: u[3], pop, R[9] (+pad) as doubles
template <int DIM>
struct SrdCell<F64T<DIM>> {
    struct Rec {
        double u[3];
        double pop;
        double R[9];
        double pad_[3];
    };
    static __device__ __forceinline__ void vel(const Fp64State &st, int i, const DevCfg &cf,
                                               double v[3]) {
        for (int d = 0; d < 3; d++) {
            v[d] = d < DIM ? st.v[d][i] : 0.0;
            if (d < DIM && cf.grav_flag) v[d] = v[d] + cf.dt * cf.grav[d];
        }
    }
    static __device__ __forceinline__ void put(Rec *r, int c, const double *u, int pop,
                                               const double *R) {
        for (int d = 0; d < 3; d++) r[c].u[d] = u[d];
        r[c].pop = (double)pop;
        for (int k = 0; k < 9; k++) r[c].R[k] = R[k];
    }
};

template <int DIM, class T>
__global__ void __launch_bounds__(256) k_srd_cells(const __grid_constant__ DevCfg c,
                                                   typename T::State a, const int *start,
                                                   typename SrdCell<T>::Rec *crec,
                                                   StepArgs sa, double *acc) {
    using VT = typename T::VT;
    __shared__ double red[8];
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    double av[3] = {0, 0, 0};
    if (cell < c.ncells) {
        const int j0 = start[cell], j1 = start[cell + 1], pop = j1 - j0;
        double M = 0.0, pv[3] = {0, 0, 0};
        for (int j = j0; j < j1; j++) {
            double m = c.mass[T::sp(a, j)];
            double v[3];
            SrdCell<T>::vel(a, j, c, v);
            M += m;
            for (int d = 0; d < DIM; d++) pv[d] += v[d] * m;
        }
        double u[3] = {0, 0, 0};
        if (M > 0.0) {
            const double iM = 1.0 / M;
            for (int d = 0; d < DIM; d++) u[d] = pv[d] * iM;
        }
        for (int d = 0; d < DIM; d++) av[d] = u[d];
        VT R[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (pop > 1) {
            double Lx[3] = {0, 0, 1};
            if (DIM == 3) mpcd_rng_axis3(c.seed, c.replica, sa.step, (uint32_t)cell, Lx);
            srd_matrix<DIM, VT>(c, Lx, R);
        }
        SrdCell<T>::put(crec, cell, u, pop, R);
    }
    for (int d = 0; d < DIM; d++) {
        double t = block_sum256(av[d], red);
        if (threadIdx.x == 0) atomicAdd(&acc[ACC_VCM + d], t);
    }
}

// Current-step cell key of a particle from its stored position, and its
// per-axis indices.
template <int DIM>
__device__ __forceinline__ int cur_key_idx(const DevCfg &c, const MixRec &r,
                                           const StepArgs &sa, int idx[3]) {
    if (c.all_periodic) {
        fx_cur_idx_periodic<DIM>(r.P, c.L, sa.ks, idx);
    } else {
        int ci[3], e = 0;
        uint32_t f[3], t;
        pos_unpack(r.P, ci, f);
        idx[0] = fx_shift_axis(ci[0], f[0], sa.ks[0], c.L[0], c.pbc[0], t, e);
        idx[1] = fx_shift_axis(ci[1], f[1], sa.ks[1], c.L[1], c.pbc[1], t, e);
        idx[2] = DIM == 3 ? fx_shift_axis(ci[2], f[2], sa.ks[2], c.L[2], c.pbc[2], t, e) : 0;
    }
    return cell_lin(c, idx[0], idx[1], idx[2]);
}
template <int DIM>
__device__ __forceinline__ int cur_key(const DevCfg &c, const MixRec &r, const StepArgs &sa) {
    int idx[3];
    return cur_key_idx<DIM>(c, r, sa, idx);
}
template <int DIM>
__device__ __forceinline__ int cur_key(const DevCfg &c, const F64Rec &r, const StepArgs &sa) {
    int idx[3] = {0, 0, 0}, e = 0;
    for (int d = 0; d < DIM; d++) idx[d] = bin_axis(r.q[d], c.L[d], c.pbc[d], 1, e);
    return cell_lin(c, idx[0], idx[1], idx[2]);
}

#ifndef MPCD_SPLIT_MINB
#define MPCD_SPLIT_MINB 4  // minimum resident blocks per SM of the particle pass
#endif

template <int DIM, class T, int MODE>
__global__ void __launch_bounds__(256, MPCD_SPLIT_MINB) k_srd_parts(const __grid_constant__ DevCfg c,
                                                   typename T::State a, typename T::State b,
                                                   int n, const typename SrdCell<T>::Rec *crec,
                                                   TileBufs tb, StepArgs sa) {
    using Rec = typename T::Rec;
    __shared__ double red[8];
    double ke = 0.0;
    int bounce = 0, esc = 0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        Rec r;
        T::load(c, a, i, sa, r);
        const int sp = T::sp(a, i);
        const int kc = cur_key<DIM>(c, r, sa);
        if constexpr (sizeof(typename T::VT) == 4) {
            const typename SrdCell<T>::Rec cr = crec[kc];
            MixRec &m = *(MixRec *)&r;
            if (__float_as_int(cr.a.w) > 1) {
                const float ux = cr.a.x, uy = cr.a.y, uz = cr.a.z;
                float w0 = m.W.x - ux, w1 = m.W.y - uy, w2 = DIM == 3 ? m.W.z - uz : 0.f;
                if (DIM == 3) {
                    m.W.x = ux + (cr.b.x * w0 + cr.b.y * w1 + cr.b.z * w2);
                    m.W.y = uy + (cr.b.w * w0 + cr.c.x * w1 + cr.c.y * w2);
                    m.W.z = uz + (cr.c.z * w0 + cr.c.w * w1 + cr.d.x * w2);
                } else {
                    m.W.x = ux + (cr.b.x * w0 + cr.b.y * w1);
                    m.W.y = uy + (cr.b.w * w0 + cr.c.x * w1);
                }
            }
            if (MODE != MODE_COUNT) {
                float t = m.W.x * m.W.x + m.W.y * m.W.y;
                if (DIM == 3) t += m.W.z * m.W.z;
                ke = c.mass[sp] * (double)t;
            }
        } else {
            const typename SrdCell<T>::Rec &cr = crec[kc];
            F64Rec &f = *(F64Rec *)&r;
            if (cr.pop > 1.0) {
                double w[3] = {0, 0, 0}, tt[3] = {0, 0, 0};
                for (int d = 0; d < DIM; d++) w[d] = f.v[d] - cr.u[d];
                for (int x = 0; x < DIM; x++)
                    for (int y = 0; y < DIM; y++) tt[x] += cr.R[x * 3 + y] * w[y];
                for (int d = 0; d < DIM; d++) f.v[d] = cr.u[d] + tt[d];
            }
            if (MODE != MODE_COUNT) {
                double t = f.v[0] * f.v[0];
                t += f.v[1] * f.v[1];
                t += f.v[2] * f.v[2];
                ke = c.mass[sp] * t;
            }
        }
        const int k = T::finish(c, r, sp, sa, bounce, esc);
        // one atomic per particle on its next cell's counter (L2 resolves
        // same-cell contention; a warp-level match of equal cells first
        // measured far slower on this GPU)
        if (MODE == MODE_COUNT) {
            atomicAdd(&tb.count_next[k], 1);
        } else {
            const int base =
                atomicAdd(MODE == MODE_INPLACE ? &tb.count_next[k] : &tb.fill[k], 1);
            if (MODE == MODE_INPLACE) {
                T::store(a, i, r);
                tb.key[i] = k;
                tb.rank[i] = base;
            } else {
                const int dst = tb.start_next[k] + base;
                T::store(b, dst, r);
                T::store_sp(b, dst, sp);
            }
        }
    }
    if (MODE != MODE_COUNT) {
        double t = block_sum256(ke, red);
        if (threadIdx.x == 0) atomicAdd(&tb.acc[ACC_KE], t);
        if (bounce) atomicAdd(&tb.status[ST_BOUNCE], (unsigned long long)bounce);
    }
    if (esc && MODE != MODE_FINAL) atomicAdd(&tb.status[ST_ESCAPED], (unsigned long long)esc);
}

}  // namespace mpcd
