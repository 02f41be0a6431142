// mpcd_device.cuh -- device-side configuration and per-particle/per-cell
// building blocks of the MPCD solvent timestep (sm_100a).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "mpcd_gpu.h"
#include "mpcd_rng.h"

namespace mpcd {

// Programmatic dependent launch (griddepcontrol, sm_90 and later).  A kernel
// launched with cudaLaunchAttributeProgrammaticStreamSerialization may begin
// while the kernel before it in the stream is still running: pdl_wait()
// returns once that kernel has completed and its memory operations are
// visible (at once for a kernel launched without the attribute), so a kernel
// touches no global memory the previous one uses before it; pdl_trigger()
// lets the next kernel of the stream begin launching.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// L2 eviction priorities (createpolicy + .L2::cache_hint, sm_80 and later).
// A step of the mixed resident family streams the particle state through L2
// once (read, then written in place), while the small per-cell arrays
// (records, sums) are re-read by every block: the stream is marked
// evict_first and the cell arrays evict_last, so that the stream does not
// push the cell arrays out of L2 between the kernel that writes them and the
// one that reads them (64^3 step 55.2 -> 52.7 us on B200; the same hints made
// the FP64 resident pass and the ensemble 2-5% slower, so they have none).
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint4 ld_hint(const uint4 *p, uint64_t pol) {
    uint4 v;
    asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_hint(const float4 *p, uint64_t pol) {
    float4 v;
    asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
// read-only through the non-coherent path (as __ldg)
__device__ __forceinline__ float4 ldg_hint(const float4 *p, uint64_t pol) {
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_hint(uint4 *p, const uint4 &v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v4.u32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p),
                 "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void st_hint(float4 *p, const float4 &v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p),
                 "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void st_hint(long long *p, long long v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.s64 [%0], %1, %2;" ::"l"(p), "l"(v), "l"(pol)
                 : "memory");
}
// Prefetch of [p, p + bytes) from this GPU's global memory into L2 with an
// eviction priority (cp.async.bulk.prefetch.L2, sm_90 and later): one
// instruction that takes no registers or shared memory and has no completion
// to wait for.  p and bytes must be multiples of 16.  A later load of the
// range finds it in L2.
__device__ __forceinline__ void prefetch_l2_bulk_hint(const void *p, uint32_t bytes,
                                                      uint64_t pol) {
    asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(p),
                 "r"(bytes), "l"(pol)
                 : "memory");
}

static inline float __int_as_float_host(int i) {
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}
static inline int __float_as_int_host(float f) {
    int i;
    std::memcpy(&i, &f, 4);
    return i;
}

constexpr double kTol = 1e-8;  // reference TOL, definitions.h:56
constexpr int kNBounce = 50;   // reference NBOUNCE, definitions.h:62
constexpr int kMaxRetherm = 16;  // re-thermalisations of one particle in one step

// Status counters (device, uint64): index into DevStatus words.
// status words (ST_OVERFLOW = 3 is defined with the tile kernels); ST_SYNC
// counts bounded waits inside a kernel that gave up
enum { ST_ESCAPED = 0, ST_BOUNCE = 1, ST_NONFINITE = 2, ST_SYNC = 4, ST_WORDS = 5 };

// Per-step global accumulators: [0] sum m v^2 (TEMP), [1..3] sum VCM (avVel)
enum { ACC_KE = 0, ACC_VCM = 1, ACC_WORDS = 4 };

struct DevWall {
    double A[3], Q[3];
    double R, DN, DT, DVN, DVT, MVN, MVT;
    double DVxyz[3];
    double MUN, MUT, MUxyz[3], DUxyz[3];  // orientation rules (nematic)
    int inv, phantom, periodic, axis;  // axis: the one non-zero component of A
    uint32_t inter;                    // bit s set: species s interacts
    int pad_;
};

struct DevCfg {
    int dim, op, lc, galinv;
    int L[3], N1[3], pbc[3];
    int ncells, n_species, n_walls, any_phantom;
    int n_solid;  // walls that are not periodic (mixed mode loops only these)
    int all_periodic;  // every axis periodic and no solid wall
    int grav_flag;
    // per-axis bit fields of a cell's slot in the resident family's
    // per-block table: slot = sum_d ((idx[d] & res_mask[d]) << res_shift[d])
    int res_shift[3], res_mask[3];
    double dt, kbt, gndnst, vol;
    double cosA, sinA;  // cos(RA) and the sine with the reference's sign (-sin RA)
    double grav[3];
    double mass[MPCD_MAX_SPECIES], damp[MPCD_MAX_SPECIES];
    double sig[MPCD_MAX_SPECIES];  // sqrt(kbt / mass): the thermal draw's width
    // Langevin MPC (langevinMPC, mpc.c:1674-1780): per species
    // a = (m - F dt / 2) / (m + F dt / 2), b = sqrt(F dt) / (m + F dt / 2)
    double lang_a[MPCD_MAX_SPECIES], lang_b[MPCD_MAX_SPECIES];
    double relax;  // in.TAU: RELAX of the Vicsek-aligned operators
    int vdist[MPCD_MAX_SPECIES];   // VDIST: re-thermalisation velocities (push)
    double rfc[MPCD_MAX_SPECIES], tumble[MPCD_MAX_SPECIES], chihi[MPCD_MAX_SPECIES];
    double act[MPCD_MAX_SPECIES], mfpot[MPCD_MAX_SPECIES], sigwidth[MPCD_MAX_SPECIES];
    double sigpos[MPCD_MAX_SPECIES], minactratio[MPCD_MAX_SPECIES];
    uint64_t seed;
    uint32_t replica;
    int act_srd;  // active SRD (collOp 9, 10): turn active particles toward VCM
    DevWall walls[MPCD_MAX_WALLS];
};

__device__ __forceinline__ int cell_lin(const DevCfg &c, int a, int b, int z) {
    return (a * c.N1[1] + b) * c.N1[2] + z;
}

__device__ __forceinline__ void cell_coords(const DevCfg &c, int lin, int &a,
                                            int &b, int &z) {
    z = lin % c.N1[2];
    int t = lin / c.N1[2];
    b = t % c.N1[1];
    a = t / c.N1[1];
}

// ------------------------------------------------------------------ warps
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------- grid shift
// gridShift_all, mpc.c:720-766: forward shift wraps Q > L && Q <= L + s.
__device__ __forceinline__ double shift_fwd(double q, double s, int L) {
    q += s;
    if (q > L && q <= L + s) q -= L;
    return q;
}
__device__ __forceinline__ double shift_back(double q, double s, int L) {
    double ms = -1.0 * s;
    q += ms;
    if (q < 0.0 && q >= ms) q += L;
    return q;
}

// bin, mpc.c:958-982: truncation, periodic index L -> 0 on the shifted grid,
// escapes counted and clamped.
__device__ __forceinline__ int bin_axis(double q, int L, int pbc, int shifted,
                                        int &escaped) {
    int a = (int)q;
    if (shifted && pbc && a == L) a = 0;
    if (a < 0 || a > L) {
        escaped = 1;
        a = a < 0 ? 0 : L;
    }
    return a;
}

// push (init.c:1261-1291): a velocity of distribution vdist for a particle
// of mass m, from the counter-based stream (step, stream, id): uniforms
// k0 + d (RANDVEL, HOMOAXIS) or normals k0 + d (GAUSS, HOMO).  Every step
// is rounded as the reference's x86-64 build rounds it (no contraction).
__device__ __forceinline__ void push_velocity(const DevCfg &c, int vdist, double m,
                                              uint32_t step, uint32_t stream, uint32_t id,
                                              uint32_t k0, double *v) {
    const int dim = c.dim;
    v[0] = v[1] = v[2] = 0.0;
    if (vdist == MPCD_VDIST_RANDVEL) {
        const double s = sqrt(c.kbt / m);
        for (int d = 0; d < dim; d++) {
            const double u = mpcd_rng_uniform(c.seed, c.replica, step, stream, id, k0 + d);
            v[d] = __dmul_rn(s, __dsub_rn(__dmul_rn(2.0, u), 1.0));
        }
    } else if (vdist == MPCD_VDIST_HOMOAXIS) {
        const double s = sqrt((double)dim * c.kbt / m);
        for (int d = 0; d < dim; d++)
            v[d] = mpcd_rng_uniform(c.seed, c.replica, step, stream, id, k0 + d) <= 0.5 ? -s : s;
    } else {  // GAUSS and HOMO: genrand_gaussMB per component
        const double s = sqrt(c.kbt / m);
        for (int d = 0; d < dim; d++)
            v[d] = __dmul_rn(s, (double)mpcd_rng_normal(c.seed, c.replica, step, stream, id,
                                                         k0 + (uint32_t)d));
        if (vdist == MPCD_VDIST_HOMO) {
            double l = 0.0;
            for (int d = 0; d < dim; d++) l = __dadd_rn(l, __dmul_rn(v[d], v[d]));
            l = sqrt(l);
            if (fabs(l - 0.0) >= kTol)
                for (int d = 0; d < dim; d++) v[d] = v[d] / l;
            const double sc = sqrt((double)dim * c.kbt / m);
            for (int d = 0; d < dim; d++) v[d] = __dmul_rn(v[d], sc);
        }
    }
}

// push_velocity out of line.  It runs only when a particle passes the wall
// bounce limit; inlined, its normals and square roots raised the register
// count of the sorted kernels that stream through walls (the channel's tile
// kernel from 80 to 120 registers, two blocks per SM instead of three).  The
// persistent and nematic kernels keep it inline (out of line they measured
// 19% and 1% slower).
static __device__ __noinline__ void push_velocity_outline(const DevCfg &c, int vdist, double m,
                                                          uint32_t step, uint32_t stream,
                                                          uint32_t id, uint32_t k0, double *v) {
    push_velocity(c, vdist, m, step, stream, id, k0, v);
}

// --------------------------------------------------------------- walls
// Surface function of a planar wall (calcW_PLANE, bc.c:306-316) with the
// wall displaced by 'off' (the grid shift during the collision stage).
__device__ __forceinline__ double wall_W(const DevWall &w, const double *q,
                                         const double *wq, int dim) {
    double W = 0.0;
    for (int i = 0; i < dim; i++) W += w.A[i] * (q[i] - wq[i]);
    W -= w.R;
    if (w.inv) W *= -1.0;
    return W;
}

// oriBC (lc.c:1290-1405) for a static wall: the orientation is made unit,
// turned to point out of the wall, its normal and tangential parts scaled by
// MUN/MUT (or replaced by DUxyz when both are 0), scaled by MUxyz and
// renormalised.
template <int DIM>
__device__ void ori_bc(const DevWall &wl, const double *n, double *U) {
    double l = 0.0;
    for (int d = 0; d < DIM; d++) l += U[d] * U[d];
    l = sqrt(l);
    if (fabs(l) >= kTol)
        for (int d = 0; d < DIM; d++) U[d] = U[d] / l;
    double x = 0.0;
    for (int d = 0; d < DIM; d++) x += U[d] * n[d];
    if (x >= 0.0)
        for (int d = 0; d < DIM; d++) U[d] *= 1.;
    else
        for (int d = 0; d < DIM; d++) U[d] *= -1.;
    double un[3], ut[3];
    x = 0.0;
    for (int d = 0; d < DIM; d++) x += U[d] * n[d];
    for (int d = 0; d < DIM; d++) {
        un[d] = x * n[d];
        ut[d] = U[d] - un[d];
    }
    if (fabs(wl.MUN - 0.0) <= kTol && fabs(wl.MUT - 0.0) <= kTol) {
        for (int d = 0; d < DIM; d++) U[d] = wl.DUxyz[d];
    } else {
        for (int d = 0; d < DIM; d++) {
            un[d] *= wl.MUN;
            ut[d] *= wl.MUT;
        }
        for (int d = 0; d < DIM; d++) U[d] = un[d] + ut[d];
        for (int d = 0; d < DIM; d++) U[d] *= wl.MUxyz[d];
    }
    l = 0.0;
    for (int d = 0; d < DIM; d++) l += U[d] * U[d];
    l = sqrt(l);
    if (fabs(l) >= kTol)
        for (int d = 0; d < DIM; d++) U[d] = U[d] / l;
}

// MPC_BCcollision (bc.c:1363-1496) for static planar rule-based walls, in
// FP64, visiting walls in index order.  'only_solid' skips periodic walls
// (the mixed-precision state wraps periodic axes exactly instead).  U, if
// given, is the nematic orientation, transformed by oriBC at each
// collision.  Returns 1 if the particle hit the bounce limit.
template <int DIM, bool OUTLINE = true>
__device__ int wall_collisions(const DevCfg &c, double *q, double *v, int sp,
                               bool only_solid, uint32_t step, uint32_t pid,
                               double *U = nullptr) {
    double t_left = c.dt, t_coll = 0.0;
    int chosen = 0, cnt = 0, cnt2 = 0, flagged = 0;
    const double m = c.mass[sp];
    for (;;) {
        double t_min = t_left, W = 1.0;
        for (int w = 0; w < c.n_walls; w++) {
            const DevWall &wl = c.walls[w];
            if (only_solid && wl.periodic) continue;
            if (!((wl.inter >> sp) & 1u)) continue;
            double tw = wall_W(wl, q, wl.Q, DIM);
            if (tw < 0.0) {
                double t1 = wl.R;
                for (int d = 0; d < DIM; d++) t1 += wl.A[d] * (wl.Q[d] - q[d]);
                double den = wl.A[0] * (-v[0]) + wl.A[1] * (-v[1]);
                den += wl.A[2] * (DIM == 3 ? -v[2] : -0.0);
                t1 /= den;
                double tc = t_left - t1;
                if (tc < t_min) {
                    t_min = tc;
                    chosen = w;
                    W = tw;
                }
            }
        }
        t_coll = t_min;
        if (W > -kTol) return flagged;
        cnt++;
        const DevWall &wl = c.walls[chosen];
        if (t_coll > -kTol) {
            double n[3] = {0, 0, 0}, vn[3], vt[3], V[3];
            for (int d = 0; d < DIM; d++) q[d] = q[d] - (t_left - t_coll) * v[d];
            for (int d = 0; d < DIM; d++) n[d] = wl.A[d];
            double len = 0.0;
            for (int d = 0; d < DIM; d++) len += n[d] * n[d];
            len = sqrt(len);
            if (fabs(len) >= kTol)
                for (int d = 0; d < DIM; d++) n[d] = n[d] / len;
            double x = 0.0;
            for (int d = 0; d < DIM; d++) x += v[d] * n[d];
            for (int d = 0; d < DIM; d++) {
                vn[d] = x * n[d];
                vt[d] = v[d] - vn[d];
            }
            for (int d = 0; d < DIM; d++) {
                vn[d] *= wl.MVN;
                vn[d] += wl.DVN * n[d];
                vt[d] *= wl.MVT;
                vt[d] += wl.DVT;
            }
            for (int d = 0; d < DIM; d++) {
                V[d] = vn[d] + vt[d];
                V[d] += wl.DVxyz[d];
                V[d] -= v[d];
                V[d] *= m;
            }
            double imp = 1.0 / m;
            for (int d = 0; d < DIM; d++) v[d] += V[d] * 1.0 * imp;
            double xq = 0.0, pn[3], pt[3];
            for (int d = 0; d < DIM; d++) xq += q[d] * n[d];
            for (int d = 0; d < DIM; d++) {
                pn[d] = xq * n[d];
                pt[d] = q[d] - pn[d];
                pn[d] += wl.DN * n[d] * (1. - 2. * kTol);
                pt[d] += wl.DT;
                q[d] = pn[d] + pt[d];
            }
            if (U) ori_bc<DIM>(wl, n, U);
            t_left -= t_coll;
            for (int d = 0; d < DIM; d++) q[d] = q[d] + t_left * v[d];
            if (wall_W(wl, q, wl.Q, DIM) < -kTol)
                for (int d = 0; d < DIM; d++) q[d] = q[d] - t_left * v[d];
        } else {
            for (int d = 0; d < DIM; d++) q[d] = q[d] - (t_left - t_coll) * v[d];
        }
        if (cnt > kNBounce) {
            flagged = 1;
            if (cnt < 2 * kNBounce && cnt2 == 0) {
                if (t_left > kTol) {
                    t_left *= 1.1;
                } else {
                    t_left = 0.9 * c.dt;
                    t_coll = 0.1 * c.dt;
                }
            } else {
                // a fresh velocity of the species' distribution and a whole
                // step to stream again (bc.c:1477-1488); the reference tries
                // for ever, here at most kMaxRetherm times
                if (cnt2 >= kMaxRetherm) return flagged;
                if (OUTLINE)
                    push_velocity_outline(c, c.vdist[sp], m, step, MPCD_STREAM_RETHERM, pid,
                                          4u * (uint32_t)cnt2, v);
                else
                    push_velocity(c, c.vdist[sp], m, step, MPCD_STREAM_RETHERM, pid,
                                  4u * (uint32_t)cnt2, v);
                t_left = c.dt;
                t_coll = 0.0;
                cnt2++;
                cnt = 0;
            }
        }
    }
}

// The end-of-step re-bin of the reference (bin(), mpc.c:969-982, on the
// unshifted grid after streaming and the wall collisions): a particle whose
// truncated cell index on some axis lies outside [0, L] has left the grid.
// replacePos_WithCheck (init.c:1462-1483) puts it at the uniform position
// L u (replace, init.c:1240-1243), again while some wall has W <= TOL there,
// and bin() gives it a Maxwell-Boltzmann velocity (genrand_gaussMB per
// component) and, for a nematic, a uniform orientation (genrand_coneNP with
// theta = pi).  The draws come from the particle's counter-based streams of
// the step: placement attempt a takes the uniforms DIM a .. DIM a + DIM - 1.
// The reference tries for ever; here at most kMaxReplace attempts (the
// last position is kept).  Out of line: it runs only for such particles.
__device__ __forceinline__ bool left_grid(const DevCfg &c, const double *q, int dim) {
    for (int d = 0; d < dim; d++) {
        const int a = (int)q[d];
        if (a < 0 || a > c.L[d]) return true;
    }
    return false;
}
constexpr uint32_t kMaxReplace = 64;
// left_grid for a position word pair (cell index, 32-bit offset) per axis:
// (int) Q < 0 when Q <= -1, (int) Q > L when Q >= L + 1
__device__ __forceinline__ bool left_grid_fx(const DevCfg &c, const int *ci, const uint32_t *f,
                                             int dim) {
    for (int d = 0; d < dim; d++)
        if (ci[d] < -1 || (ci[d] == -1 && f[d] == 0u) || ci[d] > c.L[d]) return true;
    return false;
}
template <int DIM>
__device__ __noinline__ void replace_escaped(const DevCfg &c, double *q, double *v, double *U,
                                             int sp, uint32_t step, uint32_t pid) {
    for (uint32_t a = 0; a < kMaxReplace; a++) {
        for (int d = 0; d < DIM; d++)
            q[d] = __dmul_rn((double)c.L[d],
                             mpcd_rng_uniform(c.seed, c.replica, step, MPCD_STREAM_ESCAPE_POS, pid,
                                              a * (uint32_t)DIM + (uint32_t)d));
        bool in_wall = false;
        for (int w = 0; w < c.n_walls; w++)
            if (wall_W(c.walls[w], q, c.walls[w].Q, DIM) <= kTol) in_wall = true;
        if (!in_wall) break;
    }
    for (int d = 0; d < DIM; d++)
        v[d] = __dmul_rn(c.sig[sp], (double)mpcd_rng_normal(c.seed, c.replica, step,
                                                            MPCD_STREAM_ESCAPE_VEL, pid,
                                                            (uint32_t)d));
    if (U && DIM == 2) {
        const double u =
            mpcd_rng_uniform(c.seed, c.replica, step, MPCD_STREAM_ESCAPE_ORI, pid, 0u);
        const double phi = __dmul_rn(M_PI, __dsub_rn(1.0, __dmul_rn(2.0, u)));
        U[0] = cos(phi);
        U[1] = sin(phi);
    }
}

// wall_collisions (solid walls only) out of line, for the mixed form, which
// calls it only for the few particles that ended a step inside a wall: the
// hot path of its kernels then carries none of the wall loop's registers.
template <int DIM>
__device__ __noinline__ int wall_collisions_rare(const DevCfg &c, double *q, double *v, int sp,
                                                 uint32_t step, uint32_t pid) {
    return wall_collisions<DIM>(c, q, v, sp, true, step, pid);
}

// Is the (shifted-grid) cell (a,b,z) cut by a phantom wall at its shifted
// position?  Corner test of ghostPart, mpc.c:380-470.
// The walls are axis-aligned planes (one non-zero component of A), so the
// other axes' terms of W are 0 * (q - Q) = 0 for every corner: the corner
// test reduces to the two corner coordinates along the wall's axis, with the
// same arithmetic for the remaining term.
template <int DIM>
__device__ bool cell_cut_by_phantom(const DevCfg &c, int a, int b, int z,
                                    const double *s) {
    const int cc[3] = {a, b, z};
    for (int w = 0; w < c.n_walls; w++) {
        const DevWall &wl = c.walls[w];
        if (!wl.phantom) continue;
        const int ax = wl.axis;
        const double wq = wl.Q[ax] + (ax < DIM ? s[ax] : 0.0);
        for (int j = 0; j < 2; j++) {
            double W = 0.0;
            W += wl.A[ax] * (((double)cc[ax] + (double)j) - wq);
            W -= wl.R;
            if (wl.inv) W *= -1.0;
            if (W < 0.0) return true;
        }
    }
    return false;
}

// SRD rotation matrix about unit axis L by the reference's angle (rotate,
// mpc.c:1181-1257); in 2D a plane rotation.
template <int DIM, typename T>
__device__ __forceinline__ void srd_matrix(const DevCfg &c, const double *L,
                                           T R[9]) {
    const double Cs = c.cosA, Sn = c.sinA;
    if (DIM == 3) {
        R[0] = (T)(L[0] * L[0] + (1. - L[0] * L[0]) * Cs);
        R[1] = (T)(L[0] * L[1] * (1. - Cs) - L[2] * Sn);
        R[2] = (T)(L[0] * L[2] * (1. - Cs) + L[1] * Sn);
        R[3] = (T)(L[0] * L[1] * (1. - Cs) + L[2] * Sn);
        R[4] = (T)(L[1] * L[1] + (1. - L[1] * L[1]) * Cs);
        R[5] = (T)(L[1] * L[2] * (1. - Cs) - L[0] * Sn);
        R[6] = (T)(L[0] * L[2] * (1. - Cs) - L[1] * Sn);
        R[7] = (T)(L[1] * L[2] * (1. - Cs) + L[0] * Sn);
        R[8] = (T)(L[2] * L[2] + (1. - L[2] * L[2]) * Cs);
    } else {
        R[0] = (T)Cs;
        R[1] = (T)(-1. * Sn);
        R[3] = (T)Sn;
        R[4] = (T)Cs;
        R[2] = R[5] = R[6] = R[7] = R[8] = (T)0;
    }
}

// Orthogonal-axis SRD rotation matrix about Cartesian axis ca (rotate,
// mpc.c:1206-1236, with the angle's sign fixed as for srd_matrix). The
// x-axis matrix carries the reference's -.1*S in row 2, column 1, so that
// rotation about x does not preserve the norm; it is reproduced as written.
// In 2D the axis is unused and the plane rotation of srd_matrix applies.
template <int DIM, typename T>
__device__ __forceinline__ void orth_matrix(const DevCfg &c, int ca, T R[9]) {
    if (DIM != 3) {
        const double L[3] = {0, 0, 1};
        srd_matrix<DIM, T>(c, L, R);
        return;
    }
    const T C = (T)c.cosA, S = (T)c.sinA, one = (T)1, zero = (T)0;
    for (int r = 0; r < 9; r++) R[r] = zero;
    if (ca == 0) {
        R[0] = one;
        R[4] = C;
        R[5] = S;
        R[7] = (T)(-.1 * c.sinA);
        R[8] = C;
    } else if (ca == 1) {
        R[0] = C;
        R[2] = S;
        R[4] = one;
        R[6] = (T)(-1. * c.sinA);
        R[8] = C;
    } else {
        R[0] = C;
        R[1] = S;
        R[3] = (T)(-1. * c.sinA);
        R[4] = C;
        R[8] = one;
    }
}

// A cell's SRD rotation matrix for either rotation operator: a random unit
// axis (MPCD_COLL_ARBAXIS) or a random Cartesian axis (MPCD_COLL_ORTHAXIS).
template <int DIM, typename T>
__device__ __forceinline__ void srd_cell_matrix(const DevCfg &c, uint32_t step,
                                                uint32_t cell, T R[9]) {
    if (c.op == MPCD_COLL_ORTHAXIS || c.op == MPCD_COLL_ACT_ORTHAXIS) {
        const int ca = DIM == 3 ? mpcd_rng_orth_axis(c.seed, c.replica, step, cell, DIM) : 0;
        orth_matrix<DIM, T>(c, ca, R);
        return;
    }
    double Lx[3] = {0, 0, 1};
    if (DIM == 3) mpcd_rng_axis3(c.seed, c.replica, step, cell, Lx);
    srd_matrix<DIM, T>(c, Lx, R);
}

// True for the operators that need only the cell's VCM and no thermal
// draws: the SRD rotations, plain or active, Vicsek and Chate (which also
// takes the cell's velocity director).
__host__ __device__ __forceinline__ bool is_vcm_op(int op) {
    return op == MPCD_COLL_ARBAXIS || op == MPCD_COLL_ORTHAXIS ||
           op == MPCD_COLL_ACT_ARBAXIS || op == MPCD_COLL_ACT_ORTHAXIS ||
           op == MPCD_COLL_VICSEK || op == MPCD_COLL_CHATE;
}

// Andersen MPC-AT and its Vicsek-aligned form (one weighting of the noise).
__host__ __device__ __forceinline__ bool is_mpcat_op(int op) {
    return op == MPCD_COLL_MPCAT || op == MPCD_COLL_VICSEK_MPCAT || op == MPCD_COLL_CHATE_MPCAT;
}
// Langevin MPC and its Vicsek-aligned form (the plain mean of the noise).
__host__ __device__ __forceinline__ bool is_lang_op(int op) {
    return op == MPCD_COLL_LANG || op == MPCD_COLL_VICSEK_LANG;
}
__host__ __device__ __forceinline__ bool is_vicsek_op(int op) {
    return op == MPCD_COLL_VICSEK_MPCAT || op == MPCD_COLL_VICSEK_LANG;
}

// The Vicsek alignment of vicsekAndersenMPC (mpc.c:2204-2290) and
// vicsekLangevinMPC (mpc.c:2409-2480): a particle whose species has
// |ACT| > 1e-8 (not feq) gains RELAX (ACT VCMdir - V), with V its velocity
// before the collision and VCMdir = VCM / |VCM| (normCopy, mtools.c:262-267);
// for |VCM| < 1e-8 the reference leaves VCMdir unset, zero here.  Returns
// the term to add.  Out of line and by value: only these operators reach
// it, and the callers' arrays stay in registers.
static __device__ __noinline__ double3 vicsek_term(double relax, double act, int dim,
                                                   double3 u, double3 v) {
    double3 t = make_double3(0.0, 0.0, 0.0);
    if (!(fabs(act) > 1e-8)) return t;
    double l = u.x * u.x + u.y * u.y;
    if (dim == 3) l += u.z * u.z;
    l = sqrt(l);
    const bool unit = fabs(l) >= 1e-8;
    t.x = relax * (act * (unit ? u.x / l : 0.0) - v.x);
    t.y = relax * (act * (unit ? u.y / l : 0.0) - v.y);
    if (dim == 3) t.z = relax * (act * (unit ? u.z / l : 0.0) - v.z);
    return t;
}

// Length of a 3-vector, summed in index order as the reference's length()
// (mtools.c:230-236), without contraction.
__device__ __forceinline__ double len3_rn(const double *x) {
    double r = __dmul_rn(x[0], x[0]);
    r = __dadd_rn(r, __dmul_rn(x[1], x[1]));
    r = __dadd_rn(r, __dmul_rn(x[2], x[2]));
    return sqrt(r);
}

__device__ __forceinline__ double dot3_rn(const double *x, const double *y) {
    double r = __dmul_rn(x[0], y[0]);
    r = __dadd_rn(r, __dmul_rn(x[1], y[1]));
    return __dadd_rn(r, __dmul_rn(x[2], y[2]));
}

__device__ __forceinline__ void cross3_rn(const double *x, const double *y, double *r) {
    r[0] = __dsub_rn(__dmul_rn(x[1], y[2]), __dmul_rn(x[2], y[1]));
    r[1] = __dsub_rn(__dmul_rn(x[2], y[0]), __dmul_rn(x[0], y[2]));
    r[2] = __dsub_rn(__dmul_rn(x[0], y[1]), __dmul_rn(x[1], y[0]));
}

// Rodrigues' rotation of v about axis ax by t with v's length restored
// (rodriguesRotation, mtools.c:1572-1585): the axis is normalised only when
// its length is at least 1e-8 (norm, mtools.c:246-251), in place.
__device__ __forceinline__ void rodrigues_keep(double *v, double *ax, double t) {
    const double l = len3_rn(ax);
    if (fabs(l) >= 1e-8)
        for (int d = 0; d < 3; d++) ax[d] = __ddiv_rn(ax[d], l);
    const double old = len3_rn(v);
    double cp[3];
    cross3_rn(ax, v, cp);
    const double dp = dot3_rn(ax, v);
    const double ct = cos(t), st = sin(t);
    for (int d = 0; d < 3; d++)
        v[d] = __dadd_rn(__dadd_rn(__dmul_rn(v[d], ct), __dmul_rn(cp[d], st)),
                         __dmul_rn(__dmul_rn(ax[d], dp), __dsub_rn(1.0, ct)));
    const double now = len3_rn(v);
    const double f = __ddiv_rn(old, now);
    for (int d = 0; d < 3; d++) v[d] = __dmul_rn(v[d], f);
}

// The active part of active SRD (activeSRD, mpc.c:2055-2076), after the
// rotation: a particle whose species has ACT != 0 (fneq, |ACT| >= 1e-8) is
// turned toward the cell's centre-of-mass velocity u by ACT times the angle
// between them (absAngle: acos of the cosine, mtools.c:325-367), about the
// normal v x u, by Rodrigues' formula with the length restored
// (rodriguesRotation, mtools.c:1572-1585; the axis is normalised only when
// its length is at least 1e-8).  Turns below 1e-5 rad (ROTTOL) are skipped,
// and so is a NaN angle (a zero v or u).  v and u are 3-vectors (zero z in
// 2D).  Out of line and by value: only the active operators reach it, and
// the callers' arrays stay in registers.
static __device__ __noinline__ double3 active_srd_turn(double act, double3 uu, double3 vv) {
    if (!(fabs(act) >= 1e-8)) return vv;
    const double u[3] = {uu.x, uu.y, uu.z};
    double v[3] = {vv.x, vv.y, vv.z};
    double cosa = dot3_rn(v, u);
    cosa = __ddiv_rn(cosa, len3_rn(v));
    cosa = __ddiv_rn(cosa, len3_rn(u));
    const double theta = acos(cosa);
    double ax[3];
    cross3_rn(v, u, ax);
    if (!(fabs(theta) > 1e-5)) return vv;
    rodrigues_keep(v, ax, __dmul_rn(act, theta));
    return make_double3(v[0], v[1], v[2]);
}

// genrand_cone (rand.c:438-454) with the particle's own uniforms
// (MPCD_STREAM_VICSEK, from index 0): a direction on the cone of half-angle
// t about the x axis (genrand_coneNP, rand.c:397-425: 3D z = u0 (1 - cos t)
// + cos t, phi = 2 pi u1, (z, sqrt(1-z^2) cos phi, sqrt(1-z^2) sin phi); 2D
// phi = t (1 - 2 u0), (cos phi, sin phi)), then, when `rotate`, Rodrigues'
// rotation about axis x x-hat by the angle between them, as the reference
// has it (the cone ends up about the axis mirrored about x).
__device__ __forceinline__ void cone_draw(double t, int dim, uint64_t seed, uint32_t replica,
                                          uint32_t step, uint32_t pid, const double *axis,
                                          bool rotate, double *r) {
    if (dim == 3) {
        const double ct = cos(t);
        const double u0 = mpcd_rng_uniform(seed, replica, step, MPCD_STREAM_VICSEK, pid, 0u);
        const double u1 = mpcd_rng_uniform(seed, replica, step, MPCD_STREAM_VICSEK, pid, 1u);
        const double z = __dadd_rn(__dmul_rn(u0, __dsub_rn(1.0, ct)), ct);
        const double phi = __dmul_rn(__dmul_rn(u1, 2.0), M_PI);
        const double sz = sqrt(__dsub_rn(1.0, __dmul_rn(z, z)));
        r[0] = z;
        r[1] = __dmul_rn(sz, cos(phi));
        r[2] = __dmul_rn(sz, sin(phi));
    } else {
        const double u0 = mpcd_rng_uniform(seed, replica, step, MPCD_STREAM_VICSEK, pid, 0u);
        const double phi = __dmul_rn(t, __dsub_rn(1.0, __dmul_rn(2.0, u0)));
        r[0] = cos(phi);
        r[1] = sin(phi);
        r[2] = 0.0;
    }
    if (rotate) {
        const double x[3] = {1.0, 0.0, 0.0};
        double ax[3];
        cross3_rn(axis, x, ax);
        double cosa = dot3_rn(axis, x);
        cosa = __ddiv_rn(cosa, len3_rn(axis));
        cosa = __ddiv_rn(cosa, len3_rn(x));
        rodrigues_keep(r, ax, acos(cosa));
    }
}

// Speed of a velocity (length over DIM).
__device__ __forceinline__ double speed_dim(double3 v, int dim) {
    double s = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
    if (dim == 3) s = __dadd_rn(s, __dmul_rn(v.z, v.z));
    return sqrt(s);
}

// Vicsek (vicsek, mpc.c:2098-2135): the particle keeps its speed and takes a
// direction on the cone of half-angle pi (1 - ACT) about VCMdir = VCM/|VCM|
// (normCopy over 3 components).  For |VCM| < 1e-8 the reference leaves
// VCMdir unset; here the draw keeps the x axis.  Out of line and by value.
static __device__ __noinline__ double3 vicsek_cone(double act, int dim, uint64_t seed,
                                                   uint32_t replica, uint32_t step,
                                                   uint32_t pid, double3 uu, double3 vv) {
    double u[3] = {uu.x, uu.y, dim == 3 ? uu.z : 0.0};
    const double l = len3_rn(u);
    const bool dir = fabs(l) >= 1e-8;
    if (dir)
        for (int d = 0; d < 3; d++) u[d] = __ddiv_rn(u[d], l);
    const double speed = speed_dim(vv, dim);
    double r[3];
    cone_draw(__dmul_rn(M_PI, __dsub_rn(1.0, act)), dim, seed, replica, step, pid, u, dir, r);
    return make_double3(__dmul_rn(r[0], speed), __dmul_rn(r[1], speed),
                        dim == 3 ? __dmul_rn(r[2], speed) : vv.z);
}

// Chate (chate, mpc.c:2153-2186): the particle keeps its speed and takes a
// direction on the cone of half-angle pi/2 (1 - ACT) about the cell's
// director DIR (used as it is), times a random sign genrand_pmOne
// (rand.c:378-382: -1 for a uniform <= 0.5), the particle's next uniform.
static __device__ __noinline__ double3 chate_cone(double act, int dim, uint64_t seed,
                                                  uint32_t replica, uint32_t step, uint32_t pid,
                                                  double3 dd, double3 vv) {
    const double dir[3] = {dd.x, dd.y, dim == 3 ? dd.z : 0.0};
    const double speed = speed_dim(vv, dim);
    double r[3];
    cone_draw(__dmul_rn(__dmul_rn(0.5, M_PI), __dsub_rn(1.0, act)), dim, seed, replica, step,
              pid, dir, true, r);
    const double pm = mpcd_rng_uniform(seed, replica, step, MPCD_STREAM_VICSEK, pid,
                                       dim == 3 ? 2u : 1u) <= 0.5 ? -1.0 : 1.0;
    const double f = __dmul_rn(pm, speed);
    return make_double3(__dmul_rn(r[0], f), __dmul_rn(r[1], f),
                        dim == 3 ? __dmul_rn(r[2], f) : vv.z);
}

// 2x2 eigen-decomposition of a symmetric order tensor (s00, s01; s01, s11)
// as eigenvalues2x2 and eigenvectors2x2 do it (mtools.c:1225-1300), with
// their special cases: returns the largest eigenvalue, (e0, e1) its
// eigenvector (the director).
__device__ __forceinline__ double order_eigen2(double s00, double s01, double s11, double &e0,
                                              double &e1) {
    const double s10 = s01;
    double det = s00 * s11 - s10 * s01;
    double tr = s00 + s11;
    double sq = sqrt(tr * tr * 0.25 - det);
    double ev0 = tr * 0.5 + sq;
    e0 = 0.0;
    e1 = 0.0;
    if (fabs(s10 - 0.0) >= kTol) {
        e0 = ev0 - s11;
        e1 = s10;
        double l = sqrt(e0 * e0 + e1 * e1);
        if (fabs(l) >= kTol) {
            e0 /= l;
            e1 /= l;
        }
    } else if (fabs(s01 - 0.0) >= kTol) {
        e0 = s01;
        e1 = ev0 - s00;
        double l = sqrt(e0 * e0 + e1 * e1);
        if (fabs(l) >= kTol) {
            e0 /= l;
            e1 /= l;
        }
    } else if (fabs(s00 - s11) <= kTol) {
        e0 = sqrt(2.);
        e1 = e0;
    } else {
        e0 = 1.0;
        e1 = 0.0;
    }
    return ev0;
}

// Inverse of a symmetric-or-not 3x3 matrix by adjugate / determinant.
__device__ __forceinline__ void inv3(const double m[9], double r[9]) {
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

__device__ __forceinline__ void cross3(const double *x, const double *y,
                                       double *r) {
    r[0] = x[1] * y[2] - x[2] * y[1];
    r[1] = x[2] * y[0] - x[0] * y[2];
    r[2] = x[0] * y[1] - x[1] * y[0];
}

// Thermal velocity of particle pid (genrand_gaussMB per component).
template <int DIM>
__device__ __forceinline__ void thermal(const DevCfg &c, uint32_t step,
                                        uint32_t pid, int sp, double *rv) {
    const double sig = c.sig[sp];  // sqrt(kbt / mass), correctly rounded on the host
    float g[2];
    mpcd_rng_normal2(c.seed, c.replica, step, MPCD_STREAM_THERMAL, pid, 0u, g);
    rv[0] = sig * (double)g[0];
    rv[1] = sig * (double)g[1];
    if (DIM == 3) {
        mpcd_rng_normal2(c.seed, c.replica, step, MPCD_STREAM_THERMAL, pid, 1u, g);
        rv[2] = sig * (double)g[0];
    } else {
        rv[2] = 0.0;
    }
}

}  // namespace mpcd
