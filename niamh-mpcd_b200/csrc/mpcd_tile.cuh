// mpcd_tile.cuh -- the fused per-step kernel of the solvent timestep.
//
// Particles are kept sorted by cell of the current step's shifted grid
// (counting sort, cell start offsets in 'start').  One CTA owns a tile of
// consecutive cells; it stages the tile's particles in shared memory, then
//   - one thread per cell: moments (localPROP), phantom particles
//     (ghostPart), the cell's collision parameters (SRD axis and rotation
//     matrix; Andersen sums; MPC-AT+a inertia tensor, its FP64 inverse and
//     the angular-momentum term), avVel;
//   - one thread per particle: the collision (MPCcollision), TEMP, shift
//     back, streaming, walls, and the particle's cell key on the NEXT step's
//     shifted grid (whose shift is known: draws are counter-based), counted
//     into the next step's histogram.
// Three variants of the write-out (MODE_*):
//   INPLACE  write the state back in place + key/rank (a scatter kernel then
//            reorders it);
//   COUNT    write nothing, only count the next keys;
//   FINAL    recompute and write each particle straight to its slot of the
//            next step's order (needs the scan of COUNT's histogram).
// INPLACE+scatter moves 144 B/particle (mixed), COUNT+FINAL 96 B, at twice
// the arithmetic.  The default is COUNT+FINAL for SRD and INPLACE+scatter for
// the Andersen operators; mpcd_autotune times both (and the tile sizes) on the
// live state and applies the faster.
#pragma once

#include "mpcd_device.cuh"
#include "mpcd_fp64.cuh"
#include "mpcd_mixed.cuh"

namespace mpcd {

enum { MODE_INPLACE = 0, MODE_COUNT = 1, MODE_FINAL = 2 };

enum { ST_OVERFLOW = 3 };  // status word: cells too large for a tile

struct StepArgs {
    uint32_t step;
    int pad_;
    double s[3];     // shift of this step
    double sn[3];    // shift of the next step
    uint32_t ks[3];  // the same shifts as 32-bit fractions (s = k * 2^-32)
    uint32_t ksn[3];
};

struct TileBufs {
    const int *start;       // this step's cell starts
    const int *start_next;  // next step's cell starts (FINAL)
    int *count_next;        // next step's histogram (INPLACE, COUNT)
    int *fill;              // next step's fill cursors (FINAL)
    int *key;               // INPLACE: next key per particle
    int *rank;              // INPLACE: rank within next cell
    double *acc;
    unsigned long long *status;
};

// ------------------------------------------------------- precision traits
struct MixRec {
    uint4 P;
    float4 W;
};
struct F64Rec {
    double q[3];  // position on the shifted grid
    double v[3];
    int pid, pad_;
};

template <int DIM>
struct MixT {
    using State = MixState;
    using Rec = MixRec;
    using VT = float;
    static __device__ __forceinline__ void load(const DevCfg &c, const State &st, int i,
                                                const StepArgs &sa, Rec &r) {
        r.P = st.P[i];
        r.W = st.W[i];
        if (c.grav_flag) {
            r.W.x += (float)(c.dt * c.grav[0]);
            r.W.y += (float)(c.dt * c.grav[1]);
            if (DIM == 3) r.W.z += (float)(c.dt * c.grav[2]);
        }
    }
    static __device__ __forceinline__ int sp(const State &st, int i) {
        return st.sp ? st.sp[i] : 0;
    }
    static __device__ __forceinline__ uint32_t pid(const Rec &r) {
        return (uint32_t)__float_as_int(r.W.w);
    }
    static __device__ __forceinline__ void vel(const Rec &r, double v[3]) {
        v[0] = r.W.x;
        v[1] = r.W.y;
        v[2] = DIM == 3 ? (double)r.W.z : 0.0;
    }
    static __device__ __forceinline__ void velf(const Rec &r, float v[3]) {
        v[0] = r.W.x;
        v[1] = r.W.y;
        v[2] = DIM == 3 ? r.W.z : 0.f;
    }
    // position relative to the origin of its shifted cell
    static __device__ __forceinline__ void rel(const DevCfg &c, const Rec &r,
                                               const StepArgs &sa, const int *cc,
                                               double q[3]) {
        mix_rel<DIM>(c, r.P, sa.ks, q);
    }
    static __device__ __forceinline__ void set_vel(Rec &r, const double v[3]) {
        r.W.x = (float)v[0];
        r.W.y = (float)v[1];
        if (DIM == 3) r.W.z = (float)v[2];
    }
    static __device__ __forceinline__ void set_velf(Rec &r, const float v[3]) {
        r.W.x = v[0];
        r.W.y = v[1];
        if (DIM == 3) r.W.z = v[2];
    }
    // stream (fixed point), walls (FP64, solid only), exact periodic wrap;
    // returns the particle's cell key on the next step's grid; 'bounce' set
    // when the wall loop hit its limit.
    static __device__ __forceinline__ int finish(const DevCfg &c, Rec &r, int sp,
                                                 const StepArgs &sa, int &bounce, int &esc) {
        int idx[3];
        return finish_idx(c, r, sp, sa, bounce, esc, idx);
    }
    // finish(), also returning the next cell's per-axis indices
    static __device__ __forceinline__ int finish_idx(const DevCfg &c, Rec &r, int sp,
                                                     const StepArgs &sa, int &bounce, int &esc,
                                                     int idx[3]) {
        const float dtf = (float)c.dt;
        if (c.all_periodic) {
            // periodic box: exact wrap and the short form of the next key
            fx_finish_periodic<DIM>(r.P, r.W, dtf, c.L, sa.ksn, idx);
            return cell_lin(c, idx[0], idx[1], idx[2]);
        }
        int ci[3];
        uint32_t f[3];
        pos_unpack(r.P, ci, f);
        float vv[3] = {r.W.x, r.W.y, r.W.z};
        for (int d = 0; d < DIM; d++) fx_stream(f[d], ci[d], dtf * vv[d]);
        if (c.n_solid > 0) {
            double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
            for (int d = 0; d < DIM; d++) {
                q[d] = (double)ci[d] + (double)f[d] * kFxInv;
                v[d] = (double)vv[d];
            }
            bool inside = false;
            for (int wi = 0; wi < c.n_walls; wi++) {
                const DevWall &wl = c.walls[wi];
                if (!wl.periodic && wall_W(wl, q, wl.Q, DIM) < 0.0) inside = true;
            }
            if (inside) {
                bounce += wall_collisions_rare<DIM>(c, q, v, sp, sa.step, pid(r));
                for (int d = 0; d < DIM; d++) {
                    fx_from_double(q[d], ci[d], f[d]);
                    vv[d] = (float)v[d];
                }
            }
        }
        if (left_grid_fx(c, ci, f, DIM)) {
            // the reference's end-of-step re-bin re-places it (mpc.c:969-982)
            double q[3] = {0, 0, 0}, v[3] = {vv[0], vv[1], vv[2]};
            replace_escaped<DIM>(c, q, v, nullptr, sp, sa.step, pid(r));
            for (int d = 0; d < DIM; d++) {
                fx_from_double(q[d], ci[d], f[d]);
                vv[d] = (float)v[d];
            }
            esc++;
        }
        for (int d = 0; d < DIM; d++) {
            if (c.pbc[d]) {
                if (ci[d] < 0 || ci[d] >= c.L[d])
                    ci[d] = ((ci[d] % c.L[d]) + c.L[d]) % c.L[d];
            } else if (ci[d] < 0) {
                ci[d] = 0;
                f[d] = 0u;
            } else if (ci[d] > c.L[d]) {
                ci[d] = c.L[d];
            }
        }
        if (DIM == 2) {
            ci[2] = 0;
            f[2] = 0u;
        }
        r.P = pos_pack(ci, f);
        r.W.x = vv[0];
        r.W.y = vv[1];
        if (DIM == 3) r.W.z = vv[2];
        uint32_t t;
        int a = fx_shift_axis(ci[0], f[0], sa.ksn[0], c.L[0], c.pbc[0], t, esc);
        int b = fx_shift_axis(ci[1], f[1], sa.ksn[1], c.L[1], c.pbc[1], t, esc);
        int z = 0;
        if (DIM == 3) z = fx_shift_axis(ci[2], f[2], sa.ksn[2], c.L[2], c.pbc[2], t, esc);
        idx[0] = a;
        idx[1] = b;
        idx[2] = z;
        return cell_lin(c, a, b, z);
    }
    static __device__ __forceinline__ void store(const State &st, int i, const Rec &r) {
        st.P[i] = r.P;
        st.W[i] = r.W;
    }
    static __device__ __forceinline__ void store_sp(const State &st, int i, int sp) {
        if (st.sp) st.sp[i] = sp;
    }
};

template <int DIM>
struct F64T {
    using State = Fp64State;
    using Rec = F64Rec;
    using VT = double;
    static __device__ __forceinline__ void load(const DevCfg &c, const State &st, int i,
                                                const StepArgs &sa, Rec &r) {
        for (int d = 0; d < 3; d++) {
            r.q[d] = d < DIM ? shift_fwd(st.q[d][i], sa.s[d], c.L[d]) : 0.0;
            r.v[d] = d < DIM ? st.v[d][i] : 0.0;
            if (d < DIM && c.grav_flag) r.v[d] = r.v[d] + c.dt * c.grav[d];
        }
        r.pid = st.pid[i];
    }
    static __device__ __forceinline__ int sp(const State &st, int i) {
        return st.sp ? st.sp[i] : 0;
    }
    static __device__ __forceinline__ uint32_t pid(const Rec &r) { return (uint32_t)r.pid; }
    static __device__ __forceinline__ void vel(const Rec &r, double v[3]) {
        v[0] = r.v[0];
        v[1] = r.v[1];
        v[2] = r.v[2];
    }
    static __device__ __forceinline__ void rel(const DevCfg &c, const Rec &r,
                                               const StepArgs &sa, const int *cc,
                                               double q[3]) {
        // the reference uses absolute shifted positions (localPROP, mpc.c:103)
        q[0] = r.q[0];
        q[1] = r.q[1];
        q[2] = r.q[2];
    }
    static __device__ __forceinline__ void set_vel(Rec &r, const double v[3]) {
        for (int d = 0; d < DIM; d++) r.v[d] = v[d];
    }
    // OPEN: the box may have an open side, so that particles can leave the
    // grid (a box periodic on every axis cannot: its kernels compile the
    // re-placement out)
    template <bool OPEN = true>
    static __device__ __forceinline__ int finish(const DevCfg &c, Rec &r, int sp,
                                                 const StepArgs &sa, int &bounce, int &esc) {
        double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) {
            v[d] = r.v[d];
            q[d] = shift_back(r.q[d], sa.s[d], c.L[d]);
            q[d] = q[d] + c.dt * v[d];
        }
        bounce += wall_collisions<DIM>(c, q, v, sp, false, sa.step, (uint32_t)r.pid);
        if (OPEN && left_grid(c, q, DIM)) {
            // the reference's end-of-step re-bin re-places it (mpc.c:969-982)
            replace_escaped<DIM>(c, q, v, nullptr, sp, sa.step, (uint32_t)r.pid);
            esc++;
        }
        int idx[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) {
            r.q[d] = q[d];
            r.v[d] = v[d];
            double qs = shift_fwd(q[d], sa.sn[d], c.L[d]);
            idx[d] = bin_axis(qs, c.L[d], c.pbc[d], 1, esc);
        }
        return cell_lin(c, idx[0], idx[1], idx[2]);
    }
    static __device__ __forceinline__ void store(const State &st, int i, const Rec &r) {
        for (int d = 0; d < DIM; d++) {
            st.q[d][i] = r.q[d];
            st.v[d][i] = r.v[d];
        }
        st.pid[i] = r.pid;
    }
    static __device__ __forceinline__ void store_sp(const State &st, int i, int sp) {
        if (st.sp) st.sp[i] = sp;
    }
};

// Lanes per cell in the tile kernel's per-cell phase, and the sum over such
// a group of lanes (a power of two within a warp; every lane of the warp
// calls it, and each ends with its own group's total).
constexpr int kCellLanes = 8;
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = kCellLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// --------------------------------------------------------- smem layout
struct TileLayout {
    int ct;   // cells per tile
    int cap;  // particle capacity of the staging area
    int off_rec, off_sp, off_cell, off_rv;
    int off_start, off_u, off_R, off_cm, off_rs, off_W;
    int bytes;
};

template <class T>
static inline TileLayout tile_layout(int ct, int cap, int op, int nspecies) {
    TileLayout L;
    L.ct = ct;
    L.cap = cap;
    int o = 0;
    auto take = [&](int bytes, int align) {
        o = (o + align - 1) / align * align;
        int r = o;
        o += bytes;
        return r;
    };
    L.off_rec = take(cap * (int)sizeof(typename T::Rec), 16);
    bool and_ = !is_vcm_op(op);
    L.off_rv = and_ ? take(cap * 3 * (int)sizeof(typename T::VT), 16) : -1;
    L.off_start = take((ct + 1) * 4, 16);
    L.off_u = take(ct * 3 * 8, 16);
    L.off_R = is_vcm_op(op) ? take(ct * 9 * (int)sizeof(typename T::VT), 16) : -1;
    L.off_cm = op == MPCD_COLL_RAT ? take(ct * 3 * 8, 16) : -1;
    L.off_rs = and_ ? take(ct * 3 * 8, 16) : -1;
    L.off_W = op == MPCD_COLL_RAT ? take(ct * 3 * 8, 16) : -1;
    L.off_sp = nspecies > 1 ? take(cap, 4) : -1;
    L.off_cell = take(cap, 4);
    L.bytes = (o + 15) / 16 * 16;
    return L;
}

__device__ __forceinline__ double block_sum256(double v, double *red) {
    v = warp_sum(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        t = warp_sum(t);
    }
    return t;  // valid in thread 0
}

// Chate's cell director, 2D (tensOrderParam with addToTensOrderParamVel,
// lc.c:1103-1148; localPROP, mpc.c:176-206): the order tensor of the
// normalised velocities, summed by the cell's lane group (every lane of the
// warp calls it), its leading eigenvector written by the lead lane to
// R[0..1].  normCopy leaves a velocity shorter than 1e-8 unset in the
// reference, zero here.  Out of line: only Chate reaches it.
template <class T>
static __device__ __noinline__ double2 chate_director(const typename T::Rec *rec, int j, int j1,
                                                     int pop) {
    double s00 = 0.0, s01 = 0.0, s11 = 0.0;
    for (; j < j1; j += kCellLanes) {
        double v[3] = {0, 0, 0};
        T::vel(rec[j], v);
        const double l = sqrt(v[0] * v[0] + v[1] * v[1]);
        const double o0 = fabs(l) >= 1e-8 ? v[0] / l : 0.0;
        const double o1 = fabs(l) >= 1e-8 ? v[1] / l : 0.0;
        s00 += o0 * o0;
        s01 += o0 * o1;
        s11 += o1 * o1;
    }
    s00 = group_sum(s00);
    s01 = group_sum(s01);
    s11 = group_sum(s11);
    const double cc = 1. / (2.0 - 1.), pinv = 1. / (double)pop;
    double e0, e1;
    order_eigen2(s00 * (cc * 2.0 * pinv) - cc, s01 * (cc * 2.0 * pinv), s11 * (cc * 2.0 * pinv) - cc,
                 e0, e1);
    return make_double2(e0, e1);
}

// The active velocities of MPC-AT with Chate alignment (chateAndersenMPC,
// mpc.c:2300-2408), 2D: a particle whose species has |ACT| >= 1e-8 (fneq)
// takes AV = pmOne RELAX (ACT - |V|) DIR, pmOne from its own uniform
// (genrand_pmOne, rand.c:378-382; MPCD_STREAM_VICSEK, index 0); AV joins its
// thermal velocity, so that the cell's mass-weighted mean of the two is
// RS + AS and the update VCM + RV - RS + AV - AS is the MPC-AT one.  Every
// lane of the warp calls it; each lane touches only its own particles.
template <class T>
static __device__ __noinline__ void chate_active(const DevCfg &c, const typename T::Rec *rec,
                                                 const unsigned char *spv, typename T::VT *rv,
                                                 int j, int j1, int pop, uint32_t step) {
    const double2 dir = chate_director<T>(rec, j, j1, pop);
    for (; j < j1; j += kCellLanes) {
        const int sp = spv ? spv[j] : 0;
        const double act = c.act[sp];
        if (!(fabs(act - 0.0) >= 1e-8)) continue;
        double v[3] = {0, 0, 0};
        T::vel(rec[j], v);
        const double speed = sqrt(v[0] * v[0] + v[1] * v[1]);
        const double pm = mpcd_rng_uniform(c.seed, c.replica, step, MPCD_STREAM_VICSEK,
                                           T::pid(rec[j]), 0u) <= 0.5 ? -1.0 : 1.0;
        const double f = pm * c.relax * (act - speed);
        rv[3 * j] = (typename T::VT)((double)rv[3 * j] + f * dir.x);
        rv[3 * j + 1] = (typename T::VT)((double)rv[3 * j + 1] + f * dir.y);
    }
}

template <int DIM, class T, int MODE>
__global__ void __launch_bounds__(256) k_tile(const __grid_constant__ DevCfg c,
                                              typename T::State a, typename T::State b,
                                              TileBufs tb, StepArgs sa, TileLayout lay) {
    using Rec = typename T::Rec;
    using VT = typename T::VT;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[8];
    __shared__ int s_sub[2];
    Rec *s_rec = (Rec *)(smem + lay.off_rec);
    unsigned char *s_cell = smem + lay.off_cell;
    unsigned char *s_sp = lay.off_sp >= 0 ? smem + lay.off_sp : nullptr;
    VT *s_rv = lay.off_rv >= 0 ? (VT *)(smem + lay.off_rv) : nullptr;
    int *s_start = (int *)(smem + lay.off_start);
    double *s_u = (double *)(smem + lay.off_u);
    VT *s_R = lay.off_R >= 0 ? (VT *)(smem + lay.off_R) : nullptr;
    double *s_cm = lay.off_cm >= 0 ? (double *)(smem + lay.off_cm) : nullptr;
    double *s_rs = lay.off_rs >= 0 ? (double *)(smem + lay.off_rs) : nullptr;
    double *s_W = lay.off_W >= 0 ? (double *)(smem + lay.off_W) : nullptr;

    const int tid = threadIdx.x, nth = blockDim.x;
    const int c0 = blockIdx.x * lay.ct;
    const int c1 = min(c0 + lay.ct, c.ncells);
    const int nct = c1 - c0;
    for (int k = tid; k <= nct; k += nth) s_start[k] = tb.start[c0 + k];
    __syncthreads();

    const bool andersen = !is_vcm_op(c.op);
    const bool rat = c.op == MPCD_COLL_RAT;
    // Langevin: the cell's plain mean of the noise instead of the
    // mass-weighted one (langevinMPC, mpc.c:1689-1736)
    const bool plain = is_lang_op(c.op);
    // the Vicsek-aligned MPC-AT takes the Langevin update with a = 0, b = 1
    const bool vic = is_vicsek_op(c.op);
    const bool lang = plain || vic;
    double ke = 0.0, av[3] = {0, 0, 0};
    int bounce = 0, esc = 0, overflow = 0;

    int cl_a = 0;
    while (cl_a < nct) {
        // largest sub-tile [cl_a, cl_b) that fits the staging area
        if (tid == 0) {
            const int base = s_start[cl_a];
            int cl_b = nct;
            if (s_start[nct] - base > lay.cap) {  // rare: tile above capacity
                cl_b = cl_a;
                while (cl_b < nct && s_start[cl_b + 1] - base <= lay.cap) cl_b++;
            }
            s_sub[0] = cl_b;
        }
        __syncthreads();
        int cl_b = s_sub[0];
        const bool huge = (cl_b == cl_a);  // one cell larger than the tile
        if (huge) cl_b = cl_a + 1;
        const int p0 = s_start[cl_a];
        const int np = s_start[cl_b] - p0;
        if (huge) {
            // no collision for a cell beyond capacity (counted); particles
            // still stream and are re-binned
            if (tid == 0) overflow += np;
            for (int j = tid; j < np; j += nth) {
                Rec r;
                T::load(c, a, p0 + j, sa, r);
                int sp = T::sp(a, p0 + j);
                double v[3];
                T::vel(r, v);
                ke += c.mass[sp] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                int k = T::finish(c, r, sp, sa, bounce, esc);
                if (MODE == MODE_INPLACE) {
                    T::store(a, p0 + j, r);
                    tb.key[p0 + j] = k;
                    tb.rank[p0 + j] = atomicAdd(&tb.count_next[k], 1);
                } else if (MODE == MODE_COUNT) {
                    atomicAdd(&tb.count_next[k], 1);
                } else {
                    int dst = tb.start_next[k] + atomicAdd(&tb.fill[k], 1);
                    T::store(b, dst, r);
                    T::store_sp(b, dst, sp);
                }
            }
            __syncthreads();
            cl_a = cl_b;
            continue;
        }
        // ---- stage ----
        for (int j = tid; j < np; j += nth) {
            T::load(c, a, p0 + j, sa, s_rec[j]);
            if (s_sp) s_sp[j] = (unsigned char)T::sp(a, p0 + j);
        }
        for (int cl = cl_a + tid; cl < cl_b; cl += nth)
            for (int j = s_start[cl] - p0; j < s_start[cl + 1] - p0; j++)
                s_cell[j] = (unsigned char)(cl - cl_a);
        __syncthreads();
        // ---- thermal draws (Andersen), one per particle ----
        if (andersen) {
            for (int j = tid; j < np; j += nth) {
                int sp = s_sp ? s_sp[j] : 0;
                double rv[3];
                thermal<DIM>(c, sa.step, T::pid(s_rec[j]), sp, rv);
                for (int d = 0; d < 3; d++) s_rv[3 * j + d] = (VT)rv[d];
            }
            __syncthreads();
        }
        // ---- per cell: a group of kCellLanes lanes per cell, its lanes
        // taking the cell's particles in turn; the groups of a warp step
        // through their cells together, so every shuffle has all 32 lanes
        // (a group without a cell adds zeros) ----
        const int sub = tid & (kCellLanes - 1);
        const int groups = nth / kCellLanes;
        for (int base = cl_a + (tid >> 5) * (32 / kCellLanes); base < cl_b;
             base += groups) {
            const int cl = base + ((tid & 31) / kCellLanes);
            const bool have = cl < cl_b;
            const int lc = cl - cl_a;
            const int j0 = have ? s_start[cl] - p0 : 0;
            const int j1 = have ? s_start[cl + 1] - p0 : 0;
            const int pop = j1 - j0;
            const int cell = c0 + cl;
            int cc[3] = {0, 0, 0};
            if (have && (c.any_phantom || rat)) cell_coords(c, cell, cc[0], cc[1], cc[2]);
            double M = 0.0, pv[3] = {0, 0, 0}, pq[3] = {0, 0, 0};
            for (int j = j0 + sub; j < j1; j += kCellLanes) {
                double m = c.mass[s_sp ? s_sp[j] : 0];
                double v[3];
                T::vel(s_rec[j], v);
                M += m;
                for (int d = 0; d < DIM; d++) pv[d] += v[d] * m;
                if (rat) {
                    double q[3];
                    T::rel(c, s_rec[j], sa, cc, q);
                    for (int d = 0; d < DIM; d++) pq[d] += q[d] * m;
                }
            }
            M = group_sum(M);
            for (int d = 0; d < DIM; d++) {
                pv[d] = group_sum(pv[d]);
                if (rat) pq[d] = group_sum(pq[d]);
            }
            double u[3] = {0, 0, 0}, cm[3] = {0, 0, 0};
            if (M > 0.0)
                for (int d = 0; d < DIM; d++) {
                    u[d] = pv[d] / M;
                    if (rat) cm[d] = pq[d] / M;
                }
            if (have && c.any_phantom && pop > 0 && pop < c.gndnst &&
                cell_cut_by_phantom<DIM>(c, cc[0], cc[1], cc[2], sa.s)) {
                double invN = 1.0 / (c.gndnst - (double)pop);
                double sig = sqrt(c.kbt / invN);
                for (int d = 0; d < DIM; d++) {
                    float g = mpcd_rng_normal(c.seed, c.replica, sa.step, MPCD_STREAM_GHOST,
                                              (uint32_t)cell, (uint32_t)d);
                    u[d] += sig * (double)g;
                    u[d] /= c.gndnst;
                }
            }
            const bool lead = have && sub == 0;
            if (lead) {
                for (int d = 0; d < DIM; d++) av[d] += u[d];
                for (int d = 0; d < 3; d++) s_u[3 * lc + d] = u[d];
            }
            if (!andersen) {
                if (DIM == 2 && c.op == MPCD_COLL_CHATE) {
                    const double2 dir = chate_director<T>(s_rec, j0 + sub, j1, pop);
                    if (lead && pop > 1) {
                        s_R[9 * lc] = (VT)dir.x;
                        s_R[9 * lc + 1] = (VT)dir.y;
                    }
                } else if (lead && pop > 1 && c.op != MPCD_COLL_VICSEK)
                    srd_cell_matrix<DIM, VT>(c, sa.step, (uint32_t)cell, &s_R[9 * lc]);
                continue;
            }
            // Andersen: the cell's sum of thermal velocities (every group of
            // the warp takes part in the shuffles; a group's own cell may
            // have fewer than two particles and ignore the result)
            if (DIM == 2 && c.op == MPCD_COLL_CHATE_MPCAT)
                chate_active<T>(c, s_rec, s_sp, s_rv, j0 + sub, j1, pop, sa.step);
            double rs[3] = {0, 0, 0};
            for (int j = j0 + sub; j < j1; j += kCellLanes) {
                double m = plain ? 1.0 : c.mass[s_sp ? s_sp[j] : 0];
                for (int d = 0; d < DIM; d++) rs[d] += m * (double)s_rv[3 * j + d];
            }
            for (int d = 0; d < DIM; d++) rs[d] = group_sum(rs[d]);
            if (lead && pop > 1)
                for (int d = 0; d < 3; d++)
                    s_rs[3 * lc + d] = d < DIM ? rs[d] / (plain ? (double)pop : M) : 0.0;
            if (!rat) continue;
            double I6[6] = {0, 0, 0, 0, 0, 0}, Lm[3] = {0, 0, 0};
            for (int j = j0 + sub; j < j1; j += kCellLanes) {
                double m = c.mass[s_sp ? s_sp[j] : 0];
                double q[3], v[3], r[3] = {0, 0, 0}, dv[3] = {0, 0, 0}, am[3];
                T::rel(c, s_rec[j], sa, cc, q);
                T::vel(s_rec[j], v);
                for (int d = 0; d < DIM; d++) {
                    r[d] = q[d] - cm[d];
                    dv[d] = m * (v[d] - (double)s_rv[3 * j + d]);
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
            for (int k = 0; k < 6; k++) I6[k] = group_sum(I6[k]);
            for (int d = 0; d < 3; d++) Lm[d] = group_sum(Lm[d]);
            if (lead && pop > 1) {
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
                for (int x = 0; x < 3; x++) {
                    double w = 0.0;
                    for (int y = 0; y < 3; y++) w += II[x * 3 + y] * Lm[y];
                    s_W[3 * lc + x] = w;
                    s_cm[3 * lc + x] = cm[x];
                }
            }
        }
        __syncthreads();
        // ---- per particle ----
        for (int j = tid; j < np; j += nth) {
            const int lc = s_cell[j];
            const int cl = cl_a + lc;
            const int pop = s_start[cl + 1] - s_start[cl];
            const int sp = s_sp ? s_sp[j] : 0;
            Rec r = s_rec[j];
            if (pop > 1) {
                if (!andersen && c.op == MPCD_COLL_VICSEK) {
                    double v[3] = {0, 0, 0};
                    T::vel(r, v);
                    const double3 t = vicsek_cone(
                        c.act[sp], DIM, c.seed, c.replica, sa.step, T::pid(r),
                        make_double3(s_u[3 * lc], s_u[3 * lc + 1], s_u[3 * lc + 2]),
                        make_double3(v[0], v[1], v[2]));
                    const double nv[3] = {t.x, t.y, t.z};
                    T::set_vel(r, nv);
                } else if (DIM == 2 && !andersen && c.op == MPCD_COLL_CHATE) {
                    double v[3] = {0, 0, 0};
                    T::vel(r, v);
                    const double3 t = chate_cone(
                        c.act[sp], DIM, c.seed, c.replica, sa.step, T::pid(r),
                        make_double3((double)s_R[9 * lc], (double)s_R[9 * lc + 1], 0.0),
                        make_double3(v[0], v[1], v[2]));
                    const double nv[3] = {t.x, t.y, t.z};
                    T::set_vel(r, nv);
                } else if (!andersen) {
                    const VT *R = &s_R[9 * lc];
                    if constexpr (sizeof(VT) == 4) {
                        float ux = (float)s_u[3 * lc], uy = (float)s_u[3 * lc + 1],
                              uz = (float)s_u[3 * lc + 2];
                        float v[3];
                        MixT<DIM>::velf(*(const MixRec *)&r, v);
                        float wx = v[0] - ux, wy = v[1] - uy, wz = DIM == 3 ? v[2] - uz : 0.f;
                        float nv[3];
                        if (DIM == 3) {
                            nv[0] = ux + ((float)R[0] * wx + (float)R[1] * wy + (float)R[2] * wz);
                            nv[1] = uy + ((float)R[3] * wx + (float)R[4] * wy + (float)R[5] * wz);
                            nv[2] = uz + ((float)R[6] * wx + (float)R[7] * wy + (float)R[8] * wz);
                        } else {
                            nv[0] = ux + ((float)R[0] * wx + (float)R[1] * wy);
                            nv[1] = uy + ((float)R[3] * wx + (float)R[4] * wy);
                            nv[2] = 0.f;
                        }
                        if (c.act_srd) {
                            const double3 t = active_srd_turn(
                                c.act[sp], make_double3(s_u[3 * lc], s_u[3 * lc + 1], s_u[3 * lc + 2]),
                                make_double3(nv[0], nv[1], nv[2]));
                            nv[0] = (float)t.x;
                            nv[1] = (float)t.y;
                            nv[2] = (float)t.z;
                        }
                        MixT<DIM>::set_velf(*(MixRec *)&r, nv);
                    } else {
                        double v[3], w[3] = {0, 0, 0}, t[3] = {0, 0, 0}, nv[3] = {0, 0, 0};
                        T::vel(r, v);
                        const double *u = &s_u[3 * lc];
                        for (int d = 0; d < DIM; d++) w[d] = v[d] - u[d];
                        for (int x = 0; x < DIM; x++)
                            for (int y = 0; y < DIM; y++) t[x] += (double)R[x * 3 + y] * w[y];
                        for (int d = 0; d < DIM; d++) nv[d] = u[d] + t[d];
                        if (c.act_srd) {
                            const double3 t = active_srd_turn(c.act[sp], make_double3(u[0], u[1], u[2]),
                                                              make_double3(nv[0], nv[1], nv[2]));
                            nv[0] = t.x;
                            nv[1] = t.y;
                            nv[2] = t.z;
                        }
                        T::set_vel(r, nv);
                    }
                } else {
                    const double *u = &s_u[3 * lc], *rs = &s_rs[3 * lc];
                    double damp = c.damp[sp];
                    double nv[3];
                    if (lang) {
                        // V' = VCM + a (V - VCM) + b (WN - WNS) - DAMP VCM / POP
                        double v[3];
                        T::vel(r, v);
                        const double a = c.lang_a[sp], b = c.lang_b[sp];
                        for (int d = 0; d < DIM; d++)
                            nv[d] = u[d] + a * (v[d] - u[d]) +
                                    b * ((double)s_rv[3 * j + d] - rs[d]) -
                                    damp * u[d] / (double)pop;
                        if (vic) {
                            const double3 t = vicsek_term(c.relax, c.act[sp], DIM,
                                                          make_double3(u[0], u[1], u[2]),
                                                          make_double3(v[0], v[1], v[2]));
                            nv[0] += t.x;
                            nv[1] += t.y;
                            if (DIM == 3) nv[2] += t.z;
                        }
                    } else if (!rat) {
                        for (int d = 0; d < DIM; d++)
                            nv[d] = u[d] + (double)s_rv[3 * j + d] - rs[d] -
                                    damp * u[d] / (double)pop;
                    } else {
                        int cc[3];
                        cell_coords(c, c0 + cl, cc[0], cc[1], cc[2]);
                        double q[3], rr[3] = {0, 0, 0}, ang[3];
                        T::rel(c, r, sa, cc, q);
                        for (int d = 0; d < DIM; d++) rr[d] = q[d] - s_cm[3 * lc + d];
                        cross3(&s_W[3 * lc], rr, ang);
                        for (int d = 0; d < DIM; d++)
                            nv[d] = u[d] + (double)s_rv[3 * j + d] - rs[d] - damp * u[d] + ang[d];
                    }
                    T::set_vel(r, nv);
                }
            }
            {
                double v[3];
                T::vel(r, v);
                double t = v[0] * v[0];
                t += v[1] * v[1];
                t += v[2] * v[2];
                ke += c.mass[sp] * t;
            }
            int k = T::finish(c, r, sp, sa, bounce, esc);
            const int gi = p0 + j;
            if (MODE == MODE_INPLACE && andersen) {
                // the rank is fetched after the loop, several at once (the
                // particle's thermal-velocity slots are free by now)
                T::store(a, gi, r);
                tb.key[gi] = k;
                *(int *)(s_rv + 3 * j) = k;
            } else if (MODE == MODE_INPLACE) {
                T::store(a, gi, r);
                tb.key[gi] = k;
                tb.rank[gi] = atomicAdd(&tb.count_next[k], 1);
            } else if (MODE == MODE_COUNT) {
                atomicAdd(&tb.count_next[k], 1);
            } else {
                int dst = tb.start_next[k] + atomicAdd(&tb.fill[k], 1);
                T::store(b, dst, r);
                T::store_sp(b, dst, sp);
            }
        }
        if (MODE == MODE_INPLACE && andersen) {
            // the ranks in the next step's cells, four atomics in flight at
            // a time (each thread fetches those of its own particles)
            for (int j0 = tid; j0 < np; j0 += 4 * nth) {
                int kk[4], rk[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int j = j0 + u * nth;
                    kk[u] = j < np ? *(const int *)(s_rv + 3 * j) : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; u++)
                    rk[u] = j0 + u * nth < np ? atomicAdd(&tb.count_next[kk[u]], 1) : 0;
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (j0 + u * nth < np) tb.rank[p0 + j0 + u * nth] = rk[u];
            }
        }
        __syncthreads();
        cl_a = cl_b;
    }
    // ---- block reductions ----
    if (MODE != MODE_COUNT) {
        double t = block_sum256(ke, red);
        if (tid == 0) atomicAdd(&tb.acc[ACC_KE], t);
        for (int d = 0; d < DIM; d++) {
            t = block_sum256(av[d], red);
            if (tid == 0) atomicAdd(&tb.acc[ACC_VCM + d], t);
        }
        if (bounce) atomicAdd(&tb.status[ST_BOUNCE], (unsigned long long)bounce);
        if (overflow) atomicAdd(&tb.status[ST_OVERFLOW], (unsigned long long)overflow);
    }
    if (esc && MODE != MODE_FINAL) atomicAdd(&tb.status[ST_ESCAPED], (unsigned long long)esc);
}

// Keys on the shifted grid of a step from the stored (unshifted) state:
// establishes the cell order before the first step.
template <int DIM>
__global__ void __launch_bounds__(256) k_key_mix(const __grid_constant__ DevCfg c, MixState a,
                                                 int n, int *key, int *rank, int *count,
                                                 StepArgs sa, unsigned long long *status) {
    int esc_local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int ci[3], e = 0;
        uint32_t f[3], t;
        pos_unpack(a.P[i], ci, f);
        int x = fx_shift_axis(ci[0], f[0], sa.ks[0], c.L[0], c.pbc[0], t, e);
        int y = fx_shift_axis(ci[1], f[1], sa.ks[1], c.L[1], c.pbc[1], t, e);
        int z = DIM == 3 ? fx_shift_axis(ci[2], f[2], sa.ks[2], c.L[2], c.pbc[2], t, e) : 0;
        esc_local += e;
        int k = cell_lin(c, x, y, z);
        key[i] = k;
        rank[i] = atomicAdd(&count[k], 1);
    }
    if (esc_local) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc_local);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_key_f64(const __grid_constant__ DevCfg c, Fp64State a,
                                                 int n, int *key, int *rank, int *count,
                                                 StepArgs sa, unsigned long long *status) {
    int esc_local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int idx[3] = {0, 0, 0}, e = 0;
        for (int d = 0; d < DIM; d++) {
            double qs = shift_fwd(a.q[d][i], sa.s[d], c.L[d]);
            idx[d] = bin_axis(qs, c.L[d], c.pbc[d], 1, e);
        }
        esc_local += e;
        int k = cell_lin(c, idx[0], idx[1], idx[2]);
        key[i] = k;
        rank[i] = atomicAdd(&count[k], 1);
    }
    if (esc_local) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc_local);
}

// Reorder into the other buffer as a gather: destination j reads the
// particle perm[j] (k_perm), so the writes are coalesced.
template <int DIM>
__global__ void __launch_bounds__(256) k_gather_f64(Fp64State a, Fp64State b, int n,
                                                    const int *perm) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int i = __ldg(perm + j);
        for (int d = 0; d < DIM; d++) {
            b.q[d][j] = a.q[d][i];
            b.v[d][j] = a.v[d][i];
        }
        b.pid[j] = a.pid[i];
        if (a.sp) b.sp[j] = a.sp[i];
        if (a.u[0]) {
            b.u[0][j] = a.u[0][i];
            b.u[1][j] = a.u[1][i];
        }
    }
}

// Reorder by (key, rank) into the other buffer.
template <int DIM>
__global__ void __launch_bounds__(256) k_scatter_f64v(Fp64State a, Fp64State b, int n,
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
        if (a.u[0]) {
            b.u[0][dst] = a.u[0][i];
            b.u[1][dst] = a.u[1][i];
        }
    }
}

}  // namespace mpcd
