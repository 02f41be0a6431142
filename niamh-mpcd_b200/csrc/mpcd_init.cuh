// mpcd_init.cuh -- initial particle state on the device, as the reference's
// initialisation builds it (initializeSIM, init.c:2048-2172):
//
//   setcoord (init.c:1565-1600): species in order (the first POP[0]
//     particles are species 0, ...); per particle a uniform position in the
//     box (place, PRF: init.c:1219-1224), a velocity (push, init.c:1261-1291)
//     and, for a nematic, an orientation from the first position (orient,
//     init.c:1307-1405); the mean velocity AVV over all particles; then
//     every particle inside a wall it interacts with (W <= TOL) placed anew
//     until it is not (checkplaceMPC + replace, init.c:1240-1246, 1428-1449);
//   galileantrans (mtools.c:673-711) when RFRAME is set and GPOP > 2
//     (init.c:2140-2152): V -= sum(m V)/sum(m) - AVV;
//   scaleT with VSC (therm.c:106-143, thermostat therm.c:57): V *= sqrt(KBT /
//     TEMP), TEMP about AVV (therm.c:209-235).
//
// Every draw comes from the counter-based generator at step 0: the k-th
// uniform of particle i's position stream (4 per placement attempt: attempt
// a uses k = 4a + d), its velocity stream (uniform k = d, or the d-th
// normal) and its orientation stream.  The arithmetic of each formula is
// written with explicitly rounded operations where the reference's
// x86-64 build (no FMA) rounds every step, so positions and the drawn
// velocities equal the CPU restatement's bit for bit; the sums (AVV, the
// net momentum, TEMP) are per-block trees summed in a fixed order, so the
// state is reproducible run to run and within ~1e-16 of a serial sum.
#pragma once

#include "mpcd_device.cuh"

namespace mpcd {

// velocity distributions (push, init.c:1261-1291; definitions.h RANDVEL,
// HOMO, HOMOAXIS, GAUSS) and orientation distributions (orient,
// init.c:1307-1405; definitions.h:165-183), as the ABI numbers them
struct InitPlan {
    int off[MPCD_MAX_SPECIES + 1];  // first particle of each species
    int vdist[MPCD_MAX_SPECIES];
    int odist[MPCD_MAX_SPECIES];
    int max_attempts[MPCD_MAX_SPECIES];  // placement attempts before an error
    int rframe;
};

__device__ __forceinline__ int init_species(const InitPlan &p, int ns, int i) {
    int s = 0;
    while (s + 1 < ns && i >= p.off[s + 1]) s++;
    return s;
}

__device__ __forceinline__ double init_u(const DevCfg &c, uint32_t stream, int i, uint32_t k) {
    return mpcd_rng_uniform(c.seed, c.replica, 0u, stream, (uint32_t)i, k);
}

// norm (mtools.c:246-251): divide by the length (serial sum of squares)
// when it is at least TOL away from zero (fneq, mtools.c:74-76)
__device__ __forceinline__ void init_norm(double *x, int dim) {
    double l = 0.0;
    for (int d = 0; d < dim; d++) l = __dadd_rn(l, __dmul_rn(x[d], x[d]));
    l = sqrt(l);
    if (fabs(l - 0.0) >= kTol)
        for (int d = 0; d < dim; d++) x[d] = x[d] / l;
}

// genrand_coneNP(vec, pi, dim) (rand.c:397-425): a unit vector uniform on
// the circle (2D) or the sphere (3D, z on [cos pi, 1], azimuth on [0, 2pi))
__device__ __forceinline__ void init_cone(const DevCfg &c, int i, uint32_t &k, double *U,
                                          int dim) {
    const double th = M_PI;
    if (dim == 3) {
        const double ct = cos(th);
        const double z = __dadd_rn(__dmul_rn(init_u(c, MPCD_STREAM_INIT_ORI, i, k), 1.0 - ct), ct);
        const double phi = __dmul_rn(__dmul_rn(init_u(c, MPCD_STREAM_INIT_ORI, i, k + 1), 2.0), th);
        k += 2;
        const double s = sqrt(__dsub_rn(1.0, __dmul_rn(z, z)));
        U[0] = z;
        U[1] = __dmul_rn(s, cos(phi));
        U[2] = __dmul_rn(s, sin(phi));
    } else {
        const double u = init_u(c, MPCD_STREAM_INIT_ORI, i, k++);
        const double phi = __dmul_rn(th, __dsub_rn(1.0, __dmul_rn(2.0, u)));
        U[0] = cos(phi);
        U[1] = sin(phi);
    }
}

// orient (init.c:1307-1405) for particle i at its first position q
__device__ void init_orient(const DevCfg &c, int i, int odist, const double *q, double *U) {
    const int dim = c.dim;
    uint32_t k = 0;
    U[0] = U[1] = U[2] = 0.0;
    switch (odist) {
        case MPCD_ODIST_RANDORIENT:
            init_cone(c, i, k, U, dim);
            break;
        case MPCD_ODIST_ALIGNX:
        case MPCD_ODIST_ALIGNY:
        case MPCD_ODIST_ALIGNZ: {
            // near-alignment with +-1% noise, as the reference gives it
            const double noise = __dadd_rn(
                1.0, __dmul_rn(0.02, __dsub_rn(init_u(c, MPCD_STREAM_INIT_ORI, i, 0), 0.5)));
            if (odist == MPCD_ODIST_ALIGNZ) {
                U[2] = __dmul_rn(0.9999, noise);
                U[0] = __dmul_rn(0.007071, noise);
                U[1] = __dmul_rn(0.007071, noise);
            } else {
                const int a = odist == MPCD_ODIST_ALIGNX ? 0 : 1;
                U[a] = __dmul_rn(0.9999, noise);
                U[1 - a] = __dmul_rn(0.01414178, noise);
                if (dim >= 3) U[2] = __dmul_rn(0.000008, noise);
            }
            break;
        }
        case MPCD_ODIST_ALIGN45:
            for (int d = 0; d < dim; d++) U[d] = 1.0 / sqrt(dim == 2 ? 2.0 : 3.0);
            break;
        case MPCD_ODIST_PLANEZ:
            init_cone(c, i, k, U, 2);
            break;
        case MPCD_ODIST_PLANEY:
            init_cone(c, i, k, U, 2);
            U[2] = U[1];
            U[1] = 0.0;
            break;
        case MPCD_ODIST_PLANEX:
            init_cone(c, i, k, U, 2);
            U[2] = U[0];
            U[0] = 0.0;
            break;
        case MPCD_ODIST_ALIGNTR: {
            int l2 = 0;
            for (int d = 0; d < dim; d++) l2 += c.L[d] * c.L[d];
            const double L2 = sqrt((double)l2);
            for (int d = 0; d < dim; d++) U[d] = (double)c.L[d] / L2;
            break;
        }
        case MPCD_ODIST_ALIGNDEFECTPAIR: {
            // a +1/2 defect at (L/4, Y/2) and a -1/2 defect at (3L/4, Y/2),
            // weighted linearly by distance, plus a wall term along x
            const double X = (double)c.L[0], Y = (double)c.L[1];
            const double R = 0.5 * sqrt(__dadd_rn(__dmul_rn(__dmul_rn(2.25, X), X), __dmul_rn(Y, Y)));
            const double qp0 = X * 0.25, qp1 = Y * 0.5;
            const double phiP = atan2(qp1 - q[1], qp0 - q[0]);
            const double up0 = cos(0.5 * phiP), up1 = sin(0.5 * phiP);
            const double dp0 = qp0 - q[0], dp1 = qp1 - q[1];
            const double wP = 1.0 - sqrt(__dadd_rn(__dmul_rn(dp0, dp0), __dmul_rn(dp1, dp1))) / R;
            const double qm0 = X * 0.75, qm1 = Y * 0.5;
            const double phiM = atan2(-qm1 + q[1], -qm0 + q[0]);
            const double um0 = cos(-0.5 * phiM), um1 = sin(-0.5 * phiM);
            const double dm0 = qm0 - q[0], dm1 = qm1 - q[1];
            const double wM = 1.0 - sqrt(__dadd_rn(__dmul_rn(dm0, dm0), __dmul_rn(dm1, dm1))) / R;
            const double wY = q[1] <= 0.5 * Y ? 1.0 - 2.0 * q[1] / Y : 1.0 - 2.0 * (Y - q[1]) / Y;
            U[0] = __dadd_rn(__dadd_rn(__dmul_rn(wP, up0), __dmul_rn(wM, um0)), wY);
            U[1] = __dadd_rn(__dmul_rn(wP, up1), __dmul_rn(wM, um1));
            U[2] = 0.0;
            init_norm(U, dim);
            break;
        }
        default:
            break;
    }
}

// push (init.c:1261-1291) for particle i of mass m: the velocity stream at
// step 0, uniforms or normals 0..DIM-1
__device__ __forceinline__ void init_push(const DevCfg &c, int i, int vdist, double m, double *v) {
    push_velocity(c, vdist, m, 0u, MPCD_STREAM_INIT_VEL, (uint32_t)i, 0u, v);
}

// Block sums of 'nv' values into part[blockIdx.x * 8 + j], in a fixed order
// (warp trees, then the warps in order).
__device__ __forceinline__ void init_block_sums(double *vals, int nv, double *part) {
    __shared__ double s_w[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = 0; j < nv; j++) {
        const double t = warp_sum(vals[j]);
        if (lane == 0) s_w[j][w] = t;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += s_w[threadIdx.x][k];
        part[blockIdx.x * 8 + threadIdx.x] = t;
    }
}

// Positions, velocities, orientations and species of all n particles into
// the caller-order staging arrays (3 doubles per vector); block sums of V
// (3), m V (3) and m for AVV and the net momentum.  A particle still inside
// a wall after its species' maximum attempts counts in *err.
__global__ void __launch_bounds__(256) k_init_gen(const __grid_constant__ DevCfg c, InitPlan p,
                                                  int n, double *Q, double *V, double *U, int *spid,
                                                  int *err, double *part) {
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const int dim = c.dim;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int sp = init_species(p, c.n_species, i);
        const double m = c.mass[sp];
        double q[3] = {0.0, 0.0, 0.0}, v[3], u[3];
        for (int d = 0; d < dim; d++)
            q[d] = init_u(c, MPCD_STREAM_INIT_POS, i, d) * (double)c.L[d];
        init_push(c, i, p.vdist[sp], m, v);
        if (U) init_orient(c, i, p.odist[sp], q, u);
        // checkplaceMPC: re-place until no interacting wall has W <= TOL
        bool inside = true;
        int a = 0;
        for (; a < p.max_attempts[sp]; a++) {
            if (a > 0)
                for (int d = 0; d < dim; d++)
                    q[d] = (double)c.L[d] * init_u(c, MPCD_STREAM_INIT_POS, i, 4u * a + d);
            inside = false;
            for (int j = 0; j < c.n_walls && !inside; j++) {
                const DevWall &w = c.walls[j];
                if (!((w.inter >> sp) & 1u)) continue;
                if (wall_W(w, q, w.Q, dim) <= kTol) inside = true;
            }
            if (!inside) break;
        }
        if (inside) atomicAdd(err, 1);
        for (int d = 0; d < 3; d++) {
            Q[3 * (size_t)i + d] = q[d];
            V[3 * (size_t)i + d] = v[d];
            if (U) U[3 * (size_t)i + d] = u[d];
        }
        if (spid) spid[i] = sp;
        for (int d = 0; d < 3; d++) {
            acc[d] += v[d];
            acc[3 + d] += m * v[d];
        }
        acc[6] += m;
    }
    init_block_sums(acc, 7, part);
}

// Column sums of nb block partials (fixed order) into out[0..nv).
__global__ void __launch_bounds__(256) k_init_reduce(const double *part, int nb, int nv, double *out) {
    for (int j = 0; j < nv; j++) {
        double t = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) t += part[b * 8 + j];
        t = warp_sum(t);
        __shared__ double s_w[8];
        if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += s_w[k];
            out[j] = s;
        }
        __syncthreads();
    }
}

// AVV = sum(V)/n (setcoord) and, with RFRAME, the shift of galileantrans:
// sum(m V)/sum(m) - AVV, from the sums of k_init_gen
__device__ __forceinline__ void init_frame(const double *sums, int n, int rframe, double *avv,
                                           double *shift) {
    for (int d = 0; d < 3; d++) {
        avv[d] = sums[d] / (double)n;
        shift[d] = rframe ? sums[3 + d] / sums[6] - avv[d] : 0.0;
    }
}

__device__ __forceinline__ double init_temp_term(const double *v, const double *avv, double m) {
    double t = (v[0] - avv[0]) * (v[0] - avv[0]);
    t += (v[1] - avv[1]) * (v[1] - avv[1]);
    t += (v[2] - avv[2]) * (v[2] - avv[2]);
    return m * t;
}

// Pass 2: V -= shift (the Galilean transformation), block sums of m|V-AVV|^2.
// Pass 3 (scale = 1): V *= sqrt(KBT / TEMP) from the pass-2 sum, block sums
// of m|V-AVV|^2 again (the temperature the reference reports after scaling).
__global__ void __launch_bounds__(256) k_init_adjust(const __grid_constant__ DevCfg c, InitPlan p,
                                                     int n, double *V, const double *sums,
                                                     const double *tsum, double *part) {
    double avv[3], shift[3];
    init_frame(sums, n, p.rframe, avv, shift);
    double tsc = 1.0;
    if (tsum) {
        const double kbtnow = tsum[0] / (double)(n * c.dim);
        if (kbtnow > 0.0) tsc = sqrt(c.kbt / kbtnow);
    }
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int sp = init_species(p, c.n_species, i);
        double v[3];
        for (int d = 0; d < 3; d++) v[d] = V[3 * (size_t)i + d];
        for (int d = 0; d < c.dim; d++) v[d] = tsum ? v[d] * tsc : v[d] - shift[d];
        for (int d = 0; d < 3; d++) V[3 * (size_t)i + d] = v[d];
        acc += init_temp_term(v, avv, c.mass[sp]);
    }
    init_block_sums(&acc, 1, part);
}

}  // namespace mpcd
