// mpcd_lc.cuh -- the nematic (liquid-crystal) solvent step, 2D.
//
// Per step, on particles sorted by cell of the shifted grid:
//   k_lc_moments  one thread per cell: mass, centre-of-mass velocity and
//                 position, moment of inertia about the centre of mass, and,
//                 for cells with more than one particle, the order tensor,
//                 its 2x2 eigen-decomposition, scalar order S and director
//                 (localPROP mpc.c:64-216, localMomInertiaTensor
//                 mpc.c:4209-4299, tensOrderParam lc.c:1125-1148,
//                 eigenvalues2x2/eigenvectors2x2 mtools.c:1225-1300).  S and
//                 the director persist in cells with fewer particles, as in
//                 the reference.
//   k_lc_grad     D2Q9 velocity gradient of the bulk cells, then the edge
//                 copies in the reference's order (velGradD2Q9,
//                 lc.c:2130-2162).
//   k_lc_tile     one block per tile of cells, staged in shared memory:
//                 per particle the Maier-Saupe Metropolis orientation
//                 update and rotational torque (LCcollision lc.c:427-544,
//                 genrand_maierSaupeMetropolis_2D lc.c:341-411), the
//                 Jeffery rotation by the cell's velocity gradient
//                 (jefferysTorque lc.c:559-607, larsonRotRate lc.c:622-718)
//                 and the thermal and active velocities; per cell the
//                 Andersen sums and the angular-momentum term including the
//                 torques; per particle the collision (andersenROT_LC
//                 lc.c:1515-1728, dipoleAndersenROT_LC lc.c:1749-2043), TEMP,
//                 streaming, walls with oriBC, and the next step's key.
#pragma once

#include "mpcd_tile.cuh"

namespace mpcd {

constexpr double kPi = 3.14159265358979323846;

struct LcCells {
    double *vcm;  // 2 per cell (the step's centre-of-mass velocity)
    double *cm;   // 2 per cell
    double *izz;  // moment of inertia about the centre of mass
    double *mass;
    double *S;    // scalar order parameter (persists)
    double *dir;  // 2 per cell (persists)
    double *E;    // 4 per cell, E[i][j] = dv_i/dx_j (persists)
};

// precision adaptors: position relative to a reference point of its shifted
// cell (F64: absolute shifted coordinates, as the reference; mixed: within
// the shifted cell), velocity, orientation
template <class T>
struct LcIO;
template <>
struct LcIO<F64T<2>> {
    static __device__ __forceinline__ void pos(const DevCfg &c, const Fp64State &st, int i,
                                               const StepArgs &sa, double q[2]) {
        for (int d = 0; d < 2; d++) q[d] = shift_fwd(st.q[d][i], sa.s[d], c.L[d]);
    }
    static __device__ __forceinline__ void vel(const DevCfg &c, const Fp64State &st, int i,
                                               double v[2]) {
        for (int d = 0; d < 2; d++) {
            v[d] = st.v[d][i];
            if (c.grav_flag) v[d] = v[d] + c.dt * c.grav[d];
        }
    }
    static __device__ __forceinline__ void ori(const Fp64State &st, int i, double u[2]) {
        u[0] = st.u[0][i];
        u[1] = st.u[1][i];
    }
};
template <>
struct LcIO<MixT<2>> {
    static __device__ __forceinline__ void pos(const DevCfg &c, const MixState &st, int i,
                                               const StepArgs &sa, double q[2]) {
        double r[3];
        mix_rel<2>(c, st.P[i], sa.ks, r);
        q[0] = r[0];
        q[1] = r[1];
    }
    static __device__ __forceinline__ void vel(const DevCfg &c, const MixState &st, int i,
                                               double v[2]) {
        float4 w = st.W[i];
        if (c.grav_flag) {
            w.x += (float)(c.dt * c.grav[0]);
            w.y += (float)(c.dt * c.grav[1]);
        }
        v[0] = w.x;
        v[1] = w.y;
    }
    static __device__ __forceinline__ void ori(const MixState &st, int i, double u[2]) {
        float2 x = st.U[i];
        u[0] = x.x;
        u[1] = x.y;
    }
};

__device__ __forceinline__ void lc_norm(double *v, int n) {
    double l = 0.0;
    for (int i = 0; i < n; i++) l += v[i] * v[i];
    l = sqrt(l);
    if (fabs(l) >= kTol)
        for (int i = 0; i < n; i++) v[i] = v[i] / l;
}

// rodriguesRotation, mtools.c:1572-1585 (renormalised to the old length)
__device__ __forceinline__ void lc_rodrigues(double *vec, double *ax, double th) {
    double cp[3], dp, old, nw;
    lc_norm(ax, 3);
    old = sqrt(vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2]);
    cross3(ax, vec, cp);
    dp = ax[0] * vec[0] + ax[1] * vec[1] + ax[2] * vec[2];
    const double ct = cos(th), st = sin(th);
    for (int i = 0; i < 3; i++) vec[i] = vec[i] * ct + cp[i] * st + ax[i] * dp * (1.0 - ct);
    nw = sqrt(vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2]);
    for (int i = 0; i < 3; i++) vec[i] *= (old / nw);
}

template <class T>
__device__ void lc_cell_moments(const DevCfg &c, const typename T::State &a, const int *start,
                                LcCells &lc, const StepArgs &sa, int cell, double &avx,
                                double &avy);

template <class T>
__global__ void __launch_bounds__(256) k_lc_moments(const __grid_constant__ DevCfg c,
                                                    typename T::State a, const int *start,
                                                    LcCells lc, StepArgs sa, double *acc) {
    __shared__ double red[8];
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    double avx = 0.0, avy = 0.0;
    if (cell < c.ncells) lc_cell_moments<T>(c, a, start, lc, sa, cell, avx, avy);
    double t = block_sum256(avx, red);
    if (threadIdx.x == 0) atomicAdd(&acc[ACC_VCM], t);
    t = block_sum256(avy, red);
    if (threadIdx.x == 0) atomicAdd(&acc[ACC_VCM + 1], t);
}

template <class T>
__device__ void lc_cell_moments(const DevCfg &c, const typename T::State &a, const int *start,
                                LcCells &lc, const StepArgs &sa, int cell, double &avx,
                                double &avy) {
    const int j0 = start[cell], j1 = start[cell + 1], pop = j1 - j0;
    double M = 0.0, pv[2] = {0, 0}, pq[2] = {0, 0};
    for (int j = j0; j < j1; j++) {
        double m = c.mass[T::sp(a, j)];
        double v[2], q[2];
        LcIO<T>::vel(c, a, j, v);
        LcIO<T>::pos(c, a, j, sa, q);
        M += m;
        for (int d = 0; d < 2; d++) {
            pv[d] += v[d] * m;
            pq[d] += q[d] * m;
        }
    }
    double u[2] = {0, 0}, cm[2] = {0, 0};
    if (M > 0.0)
        for (int d = 0; d < 2; d++) {
            u[d] = pv[d] / M;
            cm[d] = pq[d] / M;
        }
    double izz = 0.0;
    for (int j = j0; j < j1; j++) {
        double m = c.mass[T::sp(a, j)];
        double q[2];
        LcIO<T>::pos(c, a, j, sa, q);
        double r0 = q[0] - cm[0], r1 = q[1] - cm[1];
        izz += m * (r0 * r0 + r1 * r1);
    }
    lc.vcm[2 * cell] = u[0];
    lc.vcm[2 * cell + 1] = u[1];
    avx = u[0];
    avy = u[1];
    lc.cm[2 * cell] = cm[0];
    lc.cm[2 * cell + 1] = cm[1];
    lc.izz[cell] = izz;
    lc.mass[cell] = M;
    if (pop > 1) {
        double s00 = 0.0, s01 = 0.0, s11 = 0.0;
        for (int j = j0; j < j1; j++) {
            double o[2];
            LcIO<T>::ori(a, j, o);
            s00 += o[0] * o[0];
            s01 += o[0] * o[1];
            s11 += o[1] * o[1];
        }
        const double cc = 1. / (2.0 - 1.), pinv = 1. / (double)pop;
        s00 *= cc * 2.0 * pinv;
        s01 *= cc * 2.0 * pinv;
        s11 *= cc * 2.0 * pinv;
        s00 -= cc;
        s11 -= cc;
        double e0, e1;
        const double ev0 = order_eigen2(s00, s01, s11, e0, e1);
        lc.dir[2 * cell] = e0;
        lc.dir[2 * cell + 1] = e1;
        lc.S[cell] = ev0 > 1.0 ? 1.0 : ev0;
    }
}

// bulk D2Q9 gradient of cells 1..L-1 in x and y
static __global__ void __launch_bounds__(256) k_lc_grad(const __grid_constant__ DevCfg c, LcCells lc) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = (c.L[0] - 1) * (c.L[1] - 1);
    if (id >= nb) return;
    const int a = 1 + id / (c.L[1] - 1), b = 1 + id % (c.L[1] - 1);
    const int ev[8][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
    const double w[8] = {1. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
    double *E = &lc.E[4 * cell_lin(c, a, b, 0)];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            double e = 0.0;
            for (int k = 0; k < 8; k++)
                e += w[k] * ev[k][j] * lc.vcm[2 * cell_lin(c, a + ev[k][0], b + ev[k][1], 0) + i];
            e *= 3.;
            E[2 * i + j] = e;
        }
}

// edge copies: pass 0 the x-edges (a = 0 and a = L for b < L), pass 1 the
// y-edges (b = 0 and b = L for a < L)
static __global__ void __launch_bounds__(256) k_lc_edges(const __grid_constant__ DevCfg c, LcCells lc,
                                                  int pass) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (pass == 0) {
        if (t >= c.L[1]) return;
        for (int k = 0; k < 4; k++) {
            lc.E[4 * cell_lin(c, 0, t, 0) + k] = lc.E[4 * cell_lin(c, 1, t, 0) + k];
            lc.E[4 * cell_lin(c, c.L[0], t, 0) + k] = lc.E[4 * cell_lin(c, c.L[0] - 1, t, 0) + k];
        }
    } else {
        if (t >= c.L[0]) return;
        for (int k = 0; k < 4; k++) {
            lc.E[4 * cell_lin(c, t, 0, 0) + k] = lc.E[4 * cell_lin(c, t, 1, 0) + k];
            lc.E[4 * cell_lin(c, t, c.L[1], 0) + k] = lc.E[4 * cell_lin(c, t, c.L[1] - 1, 0) + k];
        }
    }
}


// Streaming and walls of a nematic particle; walls (periodic ones included)
// go through the FP64 wall loop so that oriBC acts on the orientation U.
template <class T>
__device__ int lc_finish(const DevCfg &c, typename T::Rec &r, int sp, const StepArgs &sa,
                         int &bounce, int &esc, double *U);
template <>
__device__ int lc_finish<F64T<2>>(const DevCfg &c, F64Rec &r, int sp, const StepArgs &sa,
                                  int &bounce, int &esc, double *U) {
    double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    for (int d = 0; d < 2; d++) {
        v[d] = r.v[d];
        q[d] = shift_back(r.q[d], sa.s[d], c.L[d]);
        q[d] = q[d] + c.dt * v[d];
    }
    bounce += wall_collisions<2, false>(c, q, v, sp, false, sa.step, (uint32_t)r.pid, U);
    if (left_grid(c, q, 2)) {
        // the reference's end-of-step re-bin re-places it (mpc.c:969-982)
        replace_escaped<2>(c, q, v, U, sp, sa.step, (uint32_t)r.pid);
        esc++;
    }
    int idx[3] = {0, 0, 0};
    for (int d = 0; d < 2; d++) {
        r.q[d] = q[d];
        r.v[d] = v[d];
        double qs = shift_fwd(q[d], sa.sn[d], c.L[d]);
        idx[d] = bin_axis(qs, c.L[d], c.pbc[d], 1, esc);
    }
    return cell_lin(c, idx[0], idx[1], 0);
}
template <>
__device__ int lc_finish<MixT<2>>(const DevCfg &c, MixRec &r, int sp, const StepArgs &sa,
                                  int &bounce, int &esc, double *U) {
    int ci[3];
    uint32_t f[3];
    pos_unpack(r.P, ci, f);
    float vv[2] = {r.W.x, r.W.y};
    const float dtf = (float)c.dt;
    for (int d = 0; d < 2; d++) fx_stream(f[d], ci[d], dtf * vv[d]);
    double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    for (int d = 0; d < 2; d++) {
        q[d] = (double)ci[d] + (double)f[d] * kFxInv;
        v[d] = (double)vv[d];
    }
    bool inside = false;
    for (int wi = 0; wi < c.n_walls; wi++)
        if (wall_W(c.walls[wi], q, c.walls[wi].Q, 2) < 0.0) inside = true;
    if (inside) {
        bounce += wall_collisions<2, false>(c, q, v, sp, false, sa.step, MixT<2>::pid(r), U);
        for (int d = 0; d < 2; d++) {
            fx_from_double(q[d], ci[d], f[d]);
            vv[d] = (float)v[d];
        }
    }
    if (left_grid_fx(c, ci, f, 2)) {
        // the reference's end-of-step re-bin re-places it (mpc.c:969-982)
        double qr[3] = {0, 0, 0}, vr[3] = {vv[0], vv[1], 0.0};
        replace_escaped<2>(c, qr, vr, U, sp, sa.step, MixT<2>::pid(r));
        for (int d = 0; d < 2; d++) {
            fx_from_double(qr[d], ci[d], f[d]);
            vv[d] = (float)vr[d];
        }
        esc++;
    }
    for (int d = 0; d < 2; d++) {
        if (c.pbc[d]) {
            if (ci[d] < 0 || ci[d] >= c.L[d]) ci[d] = ((ci[d] % c.L[d]) + c.L[d]) % c.L[d];
        } else if (ci[d] < 0) {
            ci[d] = 0;
            f[d] = 0u;
        } else if (ci[d] > c.L[d]) {
            ci[d] = c.L[d];
        }
    }
    ci[2] = 0;
    f[2] = 0u;
    r.P = pos_pack(ci, f);
    r.W.x = vv[0];
    r.W.y = vv[1];
    uint32_t t;
    int a = fx_shift_axis(ci[0], f[0], sa.ksn[0], c.L[0], c.pbc[0], t, esc);
    int b = fx_shift_axis(ci[1], f[1], sa.ksn[1], c.L[1], c.pbc[1], t, esc);
    return cell_lin(c, a, b, 0);
}

__device__ __forceinline__ void lc_store_ori(const Fp64State &st, int i, const double *U) {
    st.u[0][i] = U[0];
    st.u[1][i] = U[1];
}
__device__ __forceinline__ void lc_store_ori(const MixState &st, int i, const double *U) {
    st.U[i] = make_float2((float)U[0], (float)U[1]);
}

// per-particle staging record of the nematic tile
struct LcPart {
    double q[2];    // position (see LcIO::pos)
    double v[2];    // velocity (incl. acceleration)
    double u[2];    // orientation
    double rv[2];   // thermal velocity
    double tz;      // torque (z) from the orientation update
    double pm;      // active kick sign (+-1, 0 when inactive)
    int pid, sp;
};

struct LcTileLayout {
    int ct, cap, bytes;
};

// The tile kernel's per-cell sums use a group of 8 lanes per cell, 32 cells
// at a time (256 threads): the sum over the group, in every lane.
constexpr int kLcGroups = 32;
__device__ __forceinline__ double lc_group8_sum(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v;
}
__device__ __forceinline__ int lc_group8_sum(int v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v;
}

template <class T>
__global__ void __launch_bounds__(256, 3) k_lc_tile(const __grid_constant__ DevCfg c,
                                                 typename T::State a, LcCells lc, TileBufs tb,
                                                 StepArgs sa, LcTileLayout lay) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[8];
    __shared__ int s_sub[1];
    LcPart *sp_ = (LcPart *)smem;
    int *s_start = (int *)(smem + (size_t)lay.cap * sizeof(LcPart));
    // per cell: rotAx.z, rotAngle, effM, ACT, RS[2], AS[2], Wz
    double *s_c = (double *)(smem + (size_t)lay.cap * sizeof(LcPart) +
                             (size_t)((lay.ct + 1) * 4 + 15) / 16 * 16);
    unsigned char *s_cell =
        (unsigned char *)(s_c + (size_t)lay.ct * 9);
    const int tid = threadIdx.x, nth = blockDim.x;
    const int c0 = blockIdx.x * lay.ct;
    const int c1 = min(c0 + lay.ct, c.ncells);
    const int nct = c1 - c0;
    for (int k = tid; k <= nct; k += nth) s_start[k] = tb.start[c0 + k];
    __syncthreads();
    const int op = c.op;
    const bool dipole = op == 16 || op == 17 || op == 20 || op == 21;
    const double KBT = c.kbt, dt = c.dt;
    double ke = 0.0;
    int bounce = 0, esc = 0, overflow = 0;
    int cl_a = 0;
    while (cl_a < nct) {
        if (tid == 0) {
            const int base = s_start[cl_a];
            int cl_b = nct;
            if (s_start[nct] - base > lay.cap) {
                cl_b = cl_a;
                while (cl_b < nct && s_start[cl_b + 1] - base <= lay.cap) cl_b++;
            }
            s_sub[0] = cl_b;
        }
        __syncthreads();
        int cl_b = s_sub[0];
        if (cl_b == cl_a) {
            // a single cell beyond the staging capacity: counted, streamed
            // without collision
            if (tid == 0) overflow += s_start[cl_a + 1] - s_start[cl_a];
            for (int j = s_start[cl_a] + tid; j < s_start[cl_a + 1]; j += nth) {
                typename T::Rec r;
                T::load(c, a, j, sa, r);
                const int sp = T::sp(a, j);
                double Uo[3] = {0, 0, 0}, v[3];
                LcIO<T>::ori(a, j, Uo);
                T::vel(r, v);
                ke += c.mass[sp] * (v[0] * v[0] + v[1] * v[1]);
                const int k = lc_finish<T>(c, r, sp, sa, bounce, esc, Uo);
                T::store(a, j, r);
                lc_store_ori(a, j, Uo);
                tb.key[j] = k;
                tb.rank[j] = atomicAdd(&tb.count_next[k], 1);
            }
            __syncthreads();
            cl_a = cl_a + 1;
            continue;
        }
        const int p0 = s_start[cl_a];
        const int np = s_start[cl_b] - p0;
        // ---- stage ----
        for (int j = tid; j < np; j += nth) {
            LcPart &P = sp_[j];
            const int gi = p0 + j;
            LcIO<T>::pos(c, a, gi, sa, P.q);
            LcIO<T>::vel(c, a, gi, P.v);
            LcIO<T>::ori(a, gi, P.u);
            P.sp = T::sp(a, gi);
            typename T::Rec r;
            T::load(c, a, gi, sa, r);
            P.pid = (int)T::pid(r);
        }
        for (int cl = cl_a + tid; cl < cl_b; cl += nth)
            for (int j = s_start[cl] - p0; j < s_start[cl + 1] - p0; j++)
                s_cell[j] = (unsigned char)(cl - cl_a);
        __syncthreads();
        // ---- per cell: orientation-collision parameters and activity ----
        // A group of 8 lanes per cell (32 cells at a time): each lane sums
        // every eighth particle of the cell, the group adds its lanes.
        for (int cb = cl_a; cb < cl_b; cb += kLcGroups) {
            const int cl = cb + (tid >> 3), gl = tid & 7;
            const bool has = cl < cl_b;
            const int j0 = has ? s_start[cl] - p0 : 0, j1 = has ? s_start[cl + 1] - p0 : 0;
            const int pop = j1 - j0;
            double avm = 0.0;
            for (int j = j0 + gl; j < j1; j += 8) avm += c.mfpot[sp_[j].sp];
            avm = lc_group8_sum(avm);
            double ACT = 0.0, sw = 0.0, spos = 0.0;
            if (dipole) {
                // species populations of the cell, then the activity of the
                // species that pass the minimum-ratio test
                unsigned elig = 0u;
                for (int sx = 0; sx < c.n_species; sx++) {
                    int n = 0;
                    for (int j = j0 + gl; j < j1; j += 8) n += sp_[j].sp == sx;
                    n = lc_group8_sum(n);
                    if (c.minactratio[sx] == 0.0 || c.minactratio[sx] * c.gndnst < (double)n)
                        elig |= 1u << sx;
                }
                for (int j = j0 + gl; j < j1; j += 8) {
                    const int sx = sp_[j].sp;
                    if ((elig >> sx) & 1u) {
                        ACT += c.act[sx] / c.mass[sx];
                        sw += c.sigwidth[sx];
                        spos += c.sigpos[sx];
                    }
                }
                ACT = lc_group8_sum(ACT);
                sw = lc_group8_sum(sw);
                spos = lc_group8_sum(spos);
            }
            if (!has || gl != 0) continue;
            const int lcx = cl - cl_a, cell = c0 + cl;
            double *C = &s_c[9 * lcx];
            const double d0 = lc.dir[2 * cell], d1 = lc.dir[2 * cell + 1];
            // rotAx = DIR x xhat = (0, 0, -d1), normalised; rotAngle =
            // -acos(cos angle(DIR, xhat))
            double rz = -d1;
            double rl = fabs(rz);
            if (fabs(rl) >= kTol) rz = rz / rl;
            double ca = d0 / sqrt(d0 * d0 + d1 * d1) / 1.0;
            C[0] = rz;
            C[1] = -1. * acos(ca);
            if (pop > 1) avm /= (float)pop;
            C[2] = avm * 0.5 * 2.0;
            if (dipole) {
                if (op == 17 || op == 20) ACT *= c.gndnst / ((double)pop);
                if (op == 20 || op == 21) {
                    sw /= (double)pop;
                    spos /= (double)pop;
                    double fall = (1 - tanh(((double)pop - c.gndnst * (1 + spos)) / (c.gndnst * sw)));
                    ACT *= fall / 2;
                }
                ACT *= dt;
            }
            C[3] = ACT;
        }
        __syncthreads();
        // ---- per particle: Maier-Saupe, torque, Jeffery, draws ----
        for (int j = tid; j < np; j += nth) {
            LcPart &P = sp_[j];
            const int lcx = s_cell[j], cell = c0 + cl_a + lcx;
            const int pop = s_start[cl_a + lcx + 1] - s_start[cl_a + lcx];
            const double *C = &s_c[9 * lcx];
            P.tz = 0.0;
            if (pop > 1) {
                const double S = lc.S[cell];
                const double D0 = lc.dir[2 * cell], D1 = lc.dir[2 * cell + 1];
                const double effM = C[2];
                const double rfc = c.rfc[P.sp];
                const uint32_t pid = (uint32_t)P.pid;
                uint32_t k = 0;
                double U0 = P.u[0], U1 = P.u[1];
                double newU[3] = {U0, U1, 0.0};
                double crz = D0 * U1 - D1 * U0;
                double ang0 = atan2(sqrt(crz * crz), D0 * U0 + D1 * U1);
                if (fabs(ang0 - 0.5 * kPi) <= kTol || fabs(ang0 + 0.5 * kPi) <= kTol)
                    ang0 = kPi * (0.5 - mpcd_rng_uniform(c.seed, c.replica, sa.step,
                                                         MPCD_STREAM_LC, pid, k++));
                double uz0 = D0 * U0 + D1 * U1;
                const int anneal = (int)(5 + 0.1 * effM * S / KBT);
                int cnt = 0;
                for (int it = 0; it < anneal; it++) {
                    bool acc = false;
                    double w0 = effM * S * uz0 * uz0 / KBT;
                    double ang1 = kPi * (0.5 - mpcd_rng_uniform(c.seed, c.replica, sa.step,
                                                                MPCD_STREAM_LC, pid, k++));
                    double uz1 = cos(ang1);
                    double w1 = effM * S * uz1 * uz1 / KBT;
                    double dw = w1 - w0;
                    if (dw >= 0.) {
                        acc = true;
                    } else {
                        double R = mpcd_rng_uniform(c.seed, c.replica, sa.step, MPCD_STREAM_LC,
                                                    pid, k++);
                        if (R <= exp(dw)) acc = true;
                    }
                    if (acc) {
                        cnt += 1;
                        ang0 = ang1;
                        uz0 = uz1;
                    }
                }
                newU[0] = uz0;
                newU[1] = sin(ang0);
                double nU0 = U0, nU1 = U1;
                if (cnt > 0) {
                    double ax[3] = {0.0, 0.0, C[0]};
                    lc_rodrigues(newU, ax, C[1]);
                    nU0 = newU[0];
                    nU1 = newU[1];
                }
                double dU0 = (nU0 - U0) / dt, dU1 = (nU1 - U1) / dt;
                P.tz = (nU0 * dU1 - nU1 * dU0) * rfc;
                // Jeffery rotation with the cell's velocity gradient
                const double *E = &lc.E[4 * cell];
                double Ef[3][3] = {{E[0], E[1], 0.0}, {E[2], E[3], 0.0}, {0.0, 0.0, 0.0}};
                double u[3] = {nU0, nU1, 0.0};
                double Dm[3][3], Wm[3][3], uuuD[3] = {0, 0, 0}, uw[3] = {0, 0, 0},
                                           uD[3] = {0, 0, 0}, dudt[3], w[3];
                for (int x = 0; x < 3; x++)
                    for (int y = 0; y < 3; y++) {
                        Dm[y][x] = 0.5 * (Ef[x][y] + Ef[y][x]);
                        Wm[y][x] = 0.5 * (Ef[x][y] - Ef[y][x]);
                    }
                const double tumble = c.tumble[P.sp];
                for (int y = 0; y < 3; y++) {
                    for (int x = 0; x < 3; x++) {
                        for (int z = 0; z < 3; z++) uuuD[y] += u[y] * (u[x] * Dm[x][z] * u[z]);
                        uD[y] += u[x] * Dm[x][y];
                        uw[y] += u[x] * Wm[x][y];
                    }
                    dudt[y] = uw[y] + tumble * (uD[y] - uuuD[y]);
                }
                cross3(u, dudt, w);
                for (int x = 0; x < 3; x++) w[x] *= c.chihi[P.sp];
                for (int x = 0; x < 3; x++) w[x] *= dt;
                double th = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
                lc_norm(w, 3);
                lc_rodrigues(u, w, th);
                P.u[0] = u[0];
                P.u[1] = u[1];
            }
            double rv[3];
            thermal<2>(c, sa.step, (uint32_t)P.pid, P.sp, rv);
            P.rv[0] = rv[0];
            P.rv[1] = rv[1];
            P.pm = 0.0;
            if (dipole && fabs(C[3] - 0.0) >= kTol) {
                const double D0 = lc.dir[2 * cell], D1 = lc.dir[2 * cell + 1];
                double pW = D0 * (P.q[0] - lc.cm[2 * cell]) + D1 * (P.q[1] - lc.cm[2 * cell + 1]);
                pW -= 0.0;
                P.pm = pW <= 0 ? -1. : 1.;
            }
        }
        __syncthreads();
        // ---- per cell: Andersen sums, angular momentum ----
        // (a group of 8 lanes per cell, as above)
        for (int cb = cl_a; cb < cl_b; cb += kLcGroups) {
            const int cl = cb + (tid >> 3), gl = tid & 7;
            const bool has = cl < cl_b;
            const int lcx = cl - cl_a, cell = c0 + (has ? cl : cl_a);
            const int j0 = has ? s_start[cl] - p0 : 0, j1 = has ? s_start[cl + 1] - p0 : 0;
            const double *C = &s_c[9 * (has ? lcx : 0)];
            const double ACT = C[3];
            const double D0 = lc.dir[2 * cell], D1 = lc.dir[2 * cell + 1];
            const double cm0 = lc.cm[2 * cell], cm1 = lc.cm[2 * cell + 1];
            double RS0 = 0, RS1 = 0, AS0 = 0, AS1 = 0, Llm = 0, Lnm = 0;
            for (int j = j0 + gl; j < j1; j += 8) {
                const LcPart &P = sp_[j];
                double m = c.mass[P.sp];
                RS0 += m * P.rv[0];
                RS1 += m * P.rv[1];
                double a0 = P.pm * ACT * D0, a1 = P.pm * ACT * D1;
                if (P.pm != 0.0) {
                    AS0 += m * a0;
                    AS1 += m * a1;
                }
                double r0 = P.q[0] - cm0, r1 = P.q[1] - cm1;
                double dv0 = dipole ? m * (P.v[0] - P.rv[0] - a0) : m * (P.v[0] - P.rv[0]);
                double dv1 = dipole ? m * (P.v[1] - P.rv[1] - a1) : m * (P.v[1] - P.rv[1]);
                Llm += r0 * dv1 - r1 * dv0;
                Lnm += P.tz * dt;
            }
            RS0 = lc_group8_sum(RS0);
            RS1 = lc_group8_sum(RS1);
            AS0 = lc_group8_sum(AS0);
            AS1 = lc_group8_sum(AS1);
            Llm = lc_group8_sum(Llm);
            Lnm = lc_group8_sum(Lnm);
            if (!has || gl != 0) continue;
            double *Cw = &s_c[9 * lcx];
            const double M = lc.mass[cell];
            Cw[4] = RS0 / M;
            Cw[5] = RS1 / M;
            Cw[6] = AS0 / M;
            Cw[7] = AS1 / M;
            Cw[8] = (1. / lc.izz[cell]) * (Llm + Lnm);
        }
        __syncthreads();
        // ---- per particle: collision, TEMP, stream, walls, next key ----
        for (int j = tid; j < np; j += nth) {
            LcPart &P = sp_[j];
            const int lcx = s_cell[j], cell = c0 + cl_a + lcx;
            const int pop = s_start[cl_a + lcx + 1] - s_start[cl_a + lcx];
            const double *C = &s_c[9 * lcx];
            const int gi = p0 + j;
            double nv0 = P.v[0], nv1 = P.v[1];
            if (pop > 1) {
                const double u0 = lc.vcm[2 * cell], u1 = lc.vcm[2 * cell + 1];
                const double r0 = P.q[0] - lc.cm[2 * cell], r1 = P.q[1] - lc.cm[2 * cell + 1];
                const double Wz = C[8];
                const double ang0 = 0.0 * r0 - Wz * r1, ang1 = Wz * r0 - 0.0 * r0;
                if (dipole) {
                    const double D0 = lc.dir[2 * cell], D1 = lc.dir[2 * cell + 1];
                    const double a0 = P.pm * C[3] * D0, a1 = P.pm * C[3] * D1;
                    const double damp = c.damp[P.sp];
                    nv0 = u0 + P.rv[0] - C[4] + ang0 + a0 - C[6] - damp * u0;
                    nv1 = u1 + P.rv[1] - C[5] + ang1 + a1 - C[7] - damp * u1;
                } else {
                    nv0 = u0 + P.rv[0] - C[4] + ang0;
                    nv1 = u1 + P.rv[1] - C[5] + ang1;
                }
            }
            {
                double t = nv0 * nv0;
                t += nv1 * nv1;
                ke += c.mass[P.sp] * t;
            }
            // stream + walls (+ oriBC) in FP64, then the state's own form
            typename T::Rec r;
            T::load(c, a, gi, sa, r);
            double vv[3] = {nv0, nv1, 0.0};
            T::set_vel(r, vv);
            double Uo[3] = {P.u[0], P.u[1], 0.0};
            const int k = lc_finish<T>(c, r, P.sp, sa, bounce, esc, Uo);
            T::store(a, gi, r);
            lc_store_ori(a, gi, Uo);
            tb.key[gi] = k;
            tb.rank[gi] = atomicAdd(&tb.count_next[k], 1);
        }
        __syncthreads();
        cl_a = cl_b;
    }
    double t = block_sum256(ke, red);
    if (tid == 0) atomicAdd(&tb.acc[ACC_KE], t);
    if (bounce) atomicAdd(&tb.status[ST_BOUNCE], (unsigned long long)bounce);
    if (overflow) atomicAdd(&tb.status[ST_OVERFLOW], (unsigned long long)overflow);
    if (esc) atomicAdd(&tb.status[ST_ESCAPED], (unsigned long long)esc);
}

}  // namespace mpcd
