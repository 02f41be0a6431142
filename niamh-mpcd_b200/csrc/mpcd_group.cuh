// mpcd_group.cuh -- warp-autonomous SRD step ("one warp per cell group").
//
// For the stochastic-rotation operator the per-cell work is small (sums of
// mass and momentum, a random axis, a 3x3 rotation), so a warp owns a group
// of 32 consecutive cells of the sorted order and runs the whole collision
// for them without block-wide barriers:
//   1. stage the group's particle velocities in warp-private shared memory
//      (coalesced 16-byte loads; the group's particles are contiguous);
//   2. lane l = cell l: FP64 mass/momentum sums over its particles, centre of
//      mass velocity (localPROP, mpc.c:64-216), random axis and rotation
//      matrix (stochrotMPC + rotate, mpc.c:1181-1333), avVel term;
//   3. lane = particle: v' = u + R (v - u), TEMP term, then the same
//      finish() as the tile kernel (shift back, stream, walls, next key).
// A group larger than the staging area is split into sub-groups of cells; a
// single cell larger than the staging area is streamed without collision and
// counted (status.overflow), as in the tile kernel.
#pragma once

#include "mpcd_tile.cuh"

#ifndef MPCD_GROUP_BATCH
#define MPCD_GROUP_BATCH 2  // particles per lane in flight
#endif
#ifndef MPCD_GROUP_MINB
#define MPCD_GROUP_MINB 1  // minimum resident blocks per SM (register cap)
#endif

namespace mpcd {

template <class T>
struct GroupVel;
#ifndef MPCD_GROUP_STAGE_FULL
#define MPCD_GROUP_STAGE_FULL 1  // mixed: stage position and velocity records
#endif
#if MPCD_GROUP_STAGE_FULL
// mixed: the whole 32-byte record is staged, so the per-particle phase
// reads only shared memory
template <int DIM>
struct GroupVel<MixT<DIM>> {
    using S = MixRec;
    static __device__ __forceinline__ S load(const DevCfg &c, const MixState &st, int i) {
        MixRec r;
        r.P = st.P[i];
        r.W = st.W[i];
        if (c.grav_flag) {
            r.W.x += (float)(c.dt * c.grav[0]);
            r.W.y += (float)(c.dt * c.grav[1]);
            if (DIM == 3) r.W.z += (float)(c.dt * c.grav[2]);
        }
        return r;
    }
    static __device__ __forceinline__ void vel(const S &s, double v[3]) {
        v[0] = s.W.x;
        v[1] = s.W.y;
        v[2] = DIM == 3 ? (double)s.W.z : 0.0;
    }
    static __device__ __forceinline__ void compose(const DevCfg &c, const MixState &st, int i,
                                                   const StepArgs &sa, const S &s, MixRec &r) {
        r = s;
    }
};
#else
// mixed: only the velocity record is staged; positions are read in the
// per-particle phase
template <int DIM>
struct GroupVel<MixT<DIM>> {
    using S = float4;
    static __device__ __forceinline__ S load(const DevCfg &c, const MixState &st, int i) {
        float4 w = st.W[i];
        if (c.grav_flag) {
            w.x += (float)(c.dt * c.grav[0]);
            w.y += (float)(c.dt * c.grav[1]);
            if (DIM == 3) w.z += (float)(c.dt * c.grav[2]);
        }
        return w;
    }
    static __device__ __forceinline__ void vel(const S &s, double v[3]) {
        v[0] = s.x;
        v[1] = s.y;
        v[2] = DIM == 3 ? (double)s.z : 0.0;
    }
    static __device__ __forceinline__ void compose(const DevCfg &c, const MixState &st, int i,
                                                   const StepArgs &sa, const S &s, MixRec &r) {
        r.P = st.P[i];
        r.W = s;
    }
};
#endif
template <int DIM>
struct GroupVel<F64T<DIM>> {
    struct S {
        double v[3];
    };
    static __device__ __forceinline__ S load(const DevCfg &c, const Fp64State &st, int i) {
        S s;
        for (int d = 0; d < 3; d++) {
            s.v[d] = d < DIM ? st.v[d][i] : 0.0;
            if (d < DIM && c.grav_flag) s.v[d] = s.v[d] + c.dt * c.grav[d];
        }
        return s;
    }
    static __device__ __forceinline__ void vel(const S &s, double v[3]) {
        v[0] = s.v[0];
        v[1] = s.v[1];
        v[2] = s.v[2];
    }
    static __device__ __forceinline__ void compose(const DevCfg &c, const Fp64State &st, int i,
                                                   const StepArgs &sa, const S &s, F64Rec &r) {
        for (int d = 0; d < 3; d++) {
            r.q[d] = d < DIM ? shift_fwd(st.q[d][i], sa.s[d], c.L[d]) : 0.0;
            r.v[d] = s.v[d];
        }
        r.pid = st.pid[i];
    }
};

template <class T>
struct GroupLayout {
    using GV = GroupVel<T>;
    using VT = typename T::VT;
    static constexpr int kWarps = 4;  // warps per block
    static __host__ __device__ int per_warp_bytes(int capw) {
        int b = capw * (int)sizeof(typename GV::S);
        b = (b + 15) / 16 * 16;
        b += 32 * 12 * (int)sizeof(VT);  // u[3] + R[9] per cell
        b = (b + 15) / 16 * 16;
        b += capw;  // cell of particle
        b = (b + 15) / 16 * 16;
        b += 32 * 4;  // population of each cell
        return b;
    }
};

template <int DIM, class T, int MODE>
__global__ void __launch_bounds__(128, MPCD_GROUP_MINB) k_group(const __grid_constant__ DevCfg c,
                                               typename T::State a, typename T::State b,
                                               TileBufs tb, StepArgs sa, int capw) {
    using GV = GroupVel<T>;
    using VS = typename GV::S;
    using VT = typename T::VT;
    using Rec = typename T::Rec;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *my = smem + (size_t)wib * GroupLayout<T>::per_warp_bytes(capw);
    VS *sV = (VS *)my;
    int off = (capw * (int)sizeof(VS) + 15) / 16 * 16;
    VT *sUR = (VT *)(my + off);  // per cell: u[0..2], R[0..8]
    off += 32 * 12 * (int)sizeof(VT);
    off = (off + 15) / 16 * 16;
    unsigned char *sCell = my + off;
    off += capw;
    off = (off + 15) / 16 * 16;
    int *sPop = (int *)(my + off);

    const int group = blockIdx.x * GroupLayout<T>::kWarps + wib;
    const int g0 = group * 32;
    double ke = 0.0, av[3] = {0, 0, 0};
    int bounce = 0, esc = 0, overflow = 0;
    if (g0 < c.ncells) {
        const int ncg = min(32, c.ncells - g0);
        const int my_s = lane < ncg ? tb.start[g0 + lane] : 0;
        const int my_e = lane < ncg ? tb.start[g0 + lane + 1] : 0;
        int la = 0;
        while (la < ncg) {
            const int base = __shfl_sync(0xffffffffu, my_s, la);
            // cells [la, lb) whose particles fit the staging area
            unsigned fit = __ballot_sync(0xffffffffu, lane >= la && lane < ncg &&
                                                          my_e - base <= capw);
            // fit is a contiguous run of lanes starting at la (ends are
            // monotonic in the lane): count its trailing ones
            const unsigned run = fit >> la;
            int lb = la + (~run ? (int)__ffs(~run) - 1 : 32);
            if (lb > ncg) lb = ncg;
            const bool huge = (lb == la);
            if (huge) lb = la + 1;
            const int pend = __shfl_sync(0xffffffffu, my_e, lb - 1);
            const int np = pend - base;
            if (huge) {
                if (lane == 0) overflow += np;
                for (int j = lane; j < np; j += 32) {
                    Rec r;
                    T::load(c, a, base + j, sa, r);
                    int sp = T::sp(a, base + j);
                    double v[3];
                    T::vel(r, v);
                    ke += c.mass[sp] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                    int k = T::finish(c, r, sp, sa, bounce, esc);
                    if (MODE == MODE_INPLACE) {
                        T::store(a, base + j, r);
                        tb.key[base + j] = k;
                        tb.rank[base + j] = atomicAdd(&tb.count_next[k], 1);
                    } else if (MODE == MODE_COUNT) {
                        atomicAdd(&tb.count_next[k], 1);
                    } else {
                        int dst = tb.start_next[k] + atomicAdd(&tb.fill[k], 1);
                        T::store(b, dst, r);
                        T::store_sp(b, dst, sp);
                    }
                }
                la = lb;
                continue;
            }
            // ---- stage velocities ----
            for (int j = lane; j < np; j += 32) sV[j] = GV::load(c, a, base + j);
            __syncwarp();
            // ---- lane = cell ----
            if (lane >= la && lane < lb) {
                const int cell = g0 + lane;
                const int j0 = my_s - base, j1 = my_e - base, pop = j1 - j0;
                double M = 0.0, pv[3] = {0, 0, 0};
                for (int j = j0; j < j1; j++) {
                    double m = c.mass[T::sp(a, base + j)];
                    double v[3];
                    GV::vel(sV[j], v);
                    M += m;
                    for (int d = 0; d < DIM; d++) pv[d] += v[d] * m;
                    sCell[j] = (unsigned char)lane;
                }
                double u[3] = {0, 0, 0};
                if (M > 0.0) {
                    const double iM = 1.0 / M;
                    for (int d = 0; d < DIM; d++) u[d] = pv[d] * iM;
                }
                for (int d = 0; d < DIM; d++) av[d] += u[d];
                VT *ur = &sUR[12 * lane];
                for (int d = 0; d < 3; d++) ur[d] = (VT)u[d];
                sPop[lane] = pop;
                if (pop > 1) {
                    double Lx[3] = {0, 0, 1};
                    if (DIM == 3) mpcd_rng_axis3(c.seed, c.replica, sa.step, (uint32_t)cell, Lx);
                    srd_matrix<DIM, VT>(c, Lx, ur + 3);
                }
            }
            __syncwarp();
            // ---- lane = particle, kBatch particles per lane in flight ----
            constexpr int kBatch = MPCD_GROUP_BATCH;
            for (int j0 = lane; j0 < np; j0 += 32 * kBatch) {
                Rec r[kBatch];
                int k[kBatch], spv[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; u++) {
                    const int j = j0 + 32 * u;
                    k[u] = -1;
                    if (j >= np) continue;
                    const int gi = base + j;
                    const int lc = sCell[j];
                    const VT *ur = &sUR[12 * lc];
                    const int sp = T::sp(a, gi);
                    spv[u] = sp;
                    GV::compose(c, a, gi, sa, sV[j], r[u]);
                    if (sPop[lc] > 1) {
                        if constexpr (sizeof(VT) == 4) {
                            MixRec &m = *(MixRec *)&r[u];
                            float w0 = m.W.x - ur[0], w1 = m.W.y - ur[1];
                            float w2 = DIM == 3 ? m.W.z - ur[2] : 0.f;
                            const float *R = ur + 3;
                            if (DIM == 3) {
                                m.W.x = ur[0] + (R[0] * w0 + R[1] * w1 + R[2] * w2);
                                m.W.y = ur[1] + (R[3] * w0 + R[4] * w1 + R[5] * w2);
                                m.W.z = ur[2] + (R[6] * w0 + R[7] * w1 + R[8] * w2);
                            } else {
                                m.W.x = ur[0] + (R[0] * w0 + R[1] * w1);
                                m.W.y = ur[1] + (R[3] * w0 + R[4] * w1);
                            }
                        } else {
                            double v[3], w[3] = {0, 0, 0}, t[3] = {0, 0, 0}, nv[3];
                            T::vel(r[u], v);
                            for (int d = 0; d < DIM; d++) w[d] = v[d] - (double)ur[d];
                            for (int x = 0; x < DIM; x++)
                                for (int y = 0; y < DIM; y++)
                                    t[x] += (double)ur[3 + x * 3 + y] * w[y];
                            for (int d = 0; d < DIM; d++) nv[d] = (double)ur[d] + t[d];
                            T::set_vel(r[u], nv);
                        }
                    }
                    if (MODE != MODE_COUNT) {
                        if constexpr (sizeof(VT) == 4) {
                            const MixRec &m = *(const MixRec *)&r[u];
                            float t = m.W.x * m.W.x + m.W.y * m.W.y;
                            if (DIM == 3) t += m.W.z * m.W.z;
                            ke += c.mass[sp] * (double)t;
                        } else {
                            double v[3];
                            T::vel(r[u], v);
                            double t = v[0] * v[0];
                            t += v[1] * v[1];
                            t += v[2] * v[2];
                            ke += c.mass[sp] * t;
                        }
                    }
                    k[u] = T::finish(c, r[u], sp, sa, bounce, esc);
                }
                if (MODE == MODE_COUNT) {
#pragma unroll
                    for (int u = 0; u < kBatch; u++)
                        if (k[u] >= 0) atomicAdd(&tb.count_next[k[u]], 1);
                } else if (MODE == MODE_INPLACE) {
                    int rk[kBatch];
#pragma unroll
                    for (int u = 0; u < kBatch; u++)
                        if (k[u] >= 0) rk[u] = atomicAdd(&tb.count_next[k[u]], 1);
#pragma unroll
                    for (int u = 0; u < kBatch; u++)
                        if (k[u] >= 0) {
                            const int gi = base + j0 + 32 * u;
                            T::store(a, gi, r[u]);
                            tb.key[gi] = k[u];
                            tb.rank[gi] = rk[u];
                        }
                } else {
                    int slot[kBatch];
#pragma unroll
                    for (int u = 0; u < kBatch; u++)
                        if (k[u] >= 0) slot[u] = atomicAdd(&tb.fill[k[u]], 1);
#pragma unroll
                    for (int u = 0; u < kBatch; u++)
                        if (k[u] >= 0) {
                            const int dst = tb.start_next[k[u]] + slot[u];
                            T::store(b, dst, r[u]);
                            T::store_sp(b, dst, spv[u]);
                        }
                }
            }
            __syncwarp();
            la = lb;
        }
    }
    if (MODE != MODE_COUNT) {
        ke = warp_sum(ke);
        for (int d = 0; d < DIM; d++) av[d] = warp_sum(av[d]);
        if (lane == 0) {
            atomicAdd(&tb.acc[ACC_KE], ke);
            for (int d = 0; d < DIM; d++) atomicAdd(&tb.acc[ACC_VCM + d], av[d]);
            if (overflow) atomicAdd(&tb.status[ST_OVERFLOW], (unsigned long long)overflow);
        }
        if (bounce) atomicAdd(&tb.status[ST_BOUNCE], (unsigned long long)bounce);
    }
    if (esc && MODE != MODE_FINAL) atomicAdd(&tb.status[ST_ESCAPED], (unsigned long long)esc);
}

}  // namespace mpcd
