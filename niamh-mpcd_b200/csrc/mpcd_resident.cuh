// mpcd_resident.cuh -- SRD step with the particles resident in place.
//
// The sorted kernel families move every particle every step (the counting
// sort by next cell).  For the stochastic-rotation operator the sort is not
// needed for the physics: a particle's collision needs only its cell's
// centre-of-mass velocity u and rotation R.  This family keeps the particle
// arrays in place and computes the cell sums by accumulation instead:
//   k_res_cells  one thread per cell: reads the cell's sums (accumulated by
//                the previous particle pass), forms u, the random axis and R
//                (localPROP + stochrotMPC + rotate, mpc.c:64-216,
//                1181-1333), writes the 64-byte cell record and clears the
//                sums for reuse; avVel term.
//   k_res_parts  one thread per particle: v' = u + R (v - u) from its cell's
//                record, TEMP term, shift back / stream / walls / wrap, the
//                new state written back in place, and its mass and momentum
//                (with the next step's gravity kick) added to its cell on the
//                NEXT step's shifted grid.
// One step therefore reads and writes each particle's 32 bytes once.
//
// Sums are 64-bit fixed point (value * 2^32): integer addition is exact and
// order-independent, so the sums -- and the whole step -- are bitwise
// reproducible whatever the order of the atomics and whatever the particle
// order in memory.  Each block first aggregates its chunk of particles in a
// shared-memory hash table keyed by cell (bounded linear probing; a particle
// that finds no slot adds straight to global memory), then adds each table
// entry to global memory once.  Aggregation works because particles that
// are close in memory are close in space: the state is re-sorted by cell
// every few steps (the sort changes no result).
#pragma once

#include "mpcd_split.cuh"

// The table size and occupancy below are compile-time choices of the file
// that includes this header; each such choice gets its own inline
// namespace, so translation units with different choices link together.
#ifndef MPCD_RES_NS
#define MPCD_RES_NS res_s2048_b3
#endif

namespace mpcd {
inline namespace MPCD_RES_NS {

// The resident family's cell record, one 32-byte sector: {u.x, u.y, u.z,
// population (int bits)} and {axis x, y, z, 0}.  The particle pass applies
// the rotation about the axis in its Rodrigues form,
//   R w = cos(a) w + (1 - cos(a)) (L . w) L + s (L x w),
// which is the matrix of stochrotMPC/rotate (mpc.c:1181-1333, the sine s
// with the reference's sign) applied to w.
struct ResRec {
    float4 a, b;
};

// Fixed-point cell sums: p = sum w v * 2^32 with w = 1 for one species
// (the cell's momentum is then m p) and w = m for several species; n =
// population.  In memory the sums of nc cells are four planes of nc words,
// p0, p1, p2 and n (ResPlanes), so that the global additions of one cell
// fall on four sectors rather than one (the L2 serialises atomics on a
// sector); ResSum is a cell's sums in registers, and the 32-byte unit of
// allocation.
struct __align__(16) ResSum {
    long long p[3];
    long long n;
};
struct ResPlanes {
    long long *w;  // word d of cell k at w[d * nc + k]
    int nc;
    __device__ __forceinline__ long long *at(int d, int k) const {
        return w + (size_t)d * (size_t)nc + (size_t)k;
    }
    __device__ __forceinline__ ResSum load(int k) const {
        ResSum s;
        for (int d = 0; d < 3; d++) s.p[d] = *at(d, k);
        s.n = *at(3, k);
        return s;
    }
    __device__ __forceinline__ void clear(int k) const {
        for (int d = 0; d < 4; d++) *at(d, k) = 0ll;
    }
    // clear with an L2 eviction priority (the next particle pass adds to it)
    __device__ __forceinline__ void clear(int k, uint64_t pol) const {
        for (int d = 0; d < 4; d++) st_hint(at(d, k), 0ll, pol);
    }
};
constexpr double kSumFx = 4294967296.0;  // 2^32
constexpr double kSumFxInv = 2.3283064365386963e-10;
constexpr double kSumLimit = 36028797018963968.0;  // 2^55: per-particle bound

#ifndef MPCD_RES_SLOTS
#define MPCD_RES_SLOTS 2048  // table slots per block (power of two)
#endif
#ifndef MPCD_RES_PPT
#define MPCD_RES_PPT 8  // particles per thread
#endif
#ifndef MPCD_RES_MINB
#define MPCD_RES_MINB 3  // minimum resident blocks per SM of the particle pass
#endif
constexpr int kResSlots = MPCD_RES_SLOTS;
constexpr int res_log2(int x) { return x <= 1 ? 0 : 1 + res_log2(x >> 1); }
constexpr int kResBits = res_log2(kResSlots);
static_assert((1 << kResBits) == kResSlots, "hash slots must be a power of two");
constexpr int kResThreads = 256;
constexpr int kResChunk = kResThreads * MPCD_RES_PPT;  // particles per block
static_assert(kResChunk <= 2048, "limb sums are sized for at most 2048 particles");
constexpr int kResProbe = 32;
#ifndef MPCD_RES_BULK_PF
#define MPCD_RES_BULK_PF 1  // bulk L2 prefetch of each block's particles
#endif
static_assert(kResChunk <= 8 * 256, "the prefetch covers eight 256-particle pieces");
// Inside a block the fixed-point values are summed as two signed 32-bit
// limbs, x = hi * 2^20 + lo with |lo| <= 2^19 (fx_limbs), so that the
// shared-memory atomics are native 32-bit integer operations (64-bit and
// floating-point shared atomics are compare-and-swap loops).  For at most
// 2048 particles per entry the limb sums cannot overflow while |x| < 2^40
// (|w v| < 256); a larger value goes straight to the 64-bit global sums.
constexpr int kLimb = 20;
constexpr float kResBigV = 256.0f;

// Per-block accumulation table in dynamic shared memory: keys,
// populations, and per component the momentum limbs (row DIM: the mass
// sum, several species only).  ncomp = DIM for one species, DIM + 1 for
// several.  After them, scratch for the flush's list of used slots (not
// initialised).
struct ResTable {
    int *key;
    unsigned *cnt;
    int *hi;  // [ncomp][kResSlots]
    int *lo;  // [ncomp][kResSlots]
    unsigned short *list;
    __device__ void bind(unsigned char *base, int ncomp) {
        key = (int *)base;
        cnt = (unsigned *)(key + kResSlots);
        hi = (int *)(cnt + kResSlots);
        lo = hi + ncomp * kResSlots;
        list = (unsigned short *)(lo + ncomp * kResSlots);
    }
};
static_assert(kResSlots <= 65536, "slot indices are 16-bit");
// bytes the particle pass sets before use (keys to -1, the rest to 0)
__host__ __device__ constexpr int res_table_init_bytes(int ncomp) {
    return kResSlots * (8 + 8 * ncomp);
}
__host__ __device__ constexpr int res_table_bytes(int ncomp) {
    return res_table_init_bytes(ncomp) + kResSlots * 2;
}

__device__ __forceinline__ long long res_fix(double x, int &bad) {
    if (!(fabs(x) < kSumLimit)) {
        bad = 1;
        return 0ll;
    }
    return __double2ll_rn(x);
}

__device__ __forceinline__ void res_global_add(ResPlanes gs, unsigned long long *gm, int k,
                                               const long long x[4], unsigned cnt, bool multi) {
    for (int d = 0; d < 3; d++)
        if (x[d]) atomicAdd((unsigned long long *)gs.at(d, k), (unsigned long long)x[d]);
    atomicAdd((unsigned long long *)gs.at(3, k), (unsigned long long)cnt);
    if (multi) atomicAdd(&gm[k], (unsigned long long)x[3]);
}

// Slot of key k (per-axis indices idx) in the block's table, inserting it,
// or -1 if the bounded probe found none.  The first slot tried packs the
// low bits of the indices (DevCfg::res_shift/res_mask), the fastest axis in
// the lowest field, rotated by an offset of the other axes' indices so that
// cells adjacent across rows or planes fall in different shared-memory
// banks (a rotation within the field keeps the packing one-to-one).
template <int DIM>
__device__ __forceinline__ int res_slot(ResTable &t, const int *mask, const int *shift, int k,
                                        const int idx[3]) {
    unsigned h;
    if (DIM == 3)
        h = (unsigned)(((idx[2] + 5 * idx[1] + 11 * idx[0]) & mask[2]) |
                       ((idx[1] & mask[1]) << shift[1]) | ((idx[0] & mask[0]) << shift[0]));
    else
        h = (unsigned)(((idx[1] + 5 * idx[0]) & mask[1]) | ((idx[0] & mask[0]) << shift[0]));
    for (int probe = 0; probe < kResProbe; probe++) {
        const int cur = *(volatile int *)&t.key[h];
        if (cur == k) return (int)h;
        if (cur == -1) {
            const int old = atomicCAS(&t.key[h], -1, k);
            if (old == -1 || old == k) return (int)h;
        }
        h = (h + 1u) & (unsigned)(kResSlots - 1);
    }
    return -1;
}

// Add one particle (velocity v, weight w = 1 or its mass) to cell k.
template <int DIM>
__device__ __forceinline__ void res_add(ResTable &t, const int *mask, const int *shift,
                                        ResPlanes sums, unsigned long long *msum, int k,
                                        const int idx[3], const float v[3], double w, bool multi,
                                        int &bad) {
    const int nc = multi ? DIM + 1 : DIM;
    int hi[4] = {0, 0, 0, 0}, lo[4] = {0, 0, 0, 0};
    bool fast = !multi && fabsf(v[0]) < kResBigV && fabsf(v[1]) < kResBigV &&
                (DIM == 2 || fabsf(v[2]) < kResBigV);
    if (fast) {
        fx_limbs_unchecked(v[0], hi[0], lo[0]);
        fx_limbs_unchecked(v[1], hi[1], lo[1]);
        if (DIM == 3) fx_limbs_unchecked(v[2], hi[2], lo[2]);
    } else {
        // several species (w = m) or a large velocity: FP64 conversion
        const double wf = w * kSumFx;
        long long x[4];
        for (int d = 0; d < 3; d++) x[d] = d < DIM ? res_fix((double)v[d] * wf, bad) : 0ll;
        x[3] = multi ? res_fix(wf, bad) : 0ll;
        bool fits = true;
        for (int d = 0; d < 4; d++) fits &= (x[d] < (1ll << 40) && x[d] > -(1ll << 40));
        if (!fits) {
            res_global_add(sums, msum, k, x, 1u, multi);
            return;
        }
        for (int d = 0; d < 4; d++) {
            const long long q = (x[d] + (1ll << 19)) >> kLimb;  // nearest multiple of 2^20
            hi[d] = (int)q;
            lo[d] = (int)(x[d] - q * (1ll << kLimb));
        }
    }
    const int slot = res_slot<DIM>(t, mask, shift, k, idx);
    if (slot >= 0) {
        atomicAdd(&t.cnt[slot], 1u);
        for (int d = 0; d < nc; d++) {
            const int dd = d == DIM ? 3 : d;  // row DIM: the mass limbs
            atomicAdd(&t.hi[d * kResSlots + slot], hi[dd]);
            atomicAdd(&t.lo[d * kResSlots + slot], lo[dd]);
        }
    } else {
        long long x[4];
        for (int d = 0; d < 4; d++) x[d] = (long long)hi[d] * (1ll << kLimb) + lo[d];
        res_global_add(sums, msum, k, x, 1u, multi);
    }
}

// Add every used table entry to the global sums.  Each warp first lists
// the used slots of its share of the table (ballot + prefix count), then
// adds them with all its lanes busy; most slots of a table are unused.
// Requires kResThreads threads.
template <int DIM>
__device__ __forceinline__ void res_flush(const ResTable &t, ResPlanes sums,
                                          unsigned long long *msum, bool multi) {
    const int nc = multi ? DIM + 1 : DIM;
    constexpr int kPer = kResSlots / (kResThreads / 32);
    static_assert(kPer % 32 == 0, "each warp lists whole 32-slot groups");
    const int lane = threadIdx.x & 31;
    const int s0 = (threadIdx.x >> 5) * kPer;
    unsigned short *list = t.list + s0;
    int total = 0;
    for (int j = 0; j < kPer; j += 32) {
        const int s = s0 + j + lane;
        const bool used = t.key[s] >= 0;
        const unsigned m = __ballot_sync(0xffffffffu, used);
        if (used) list[total + __popc(m & ((1u << lane) - 1u))] = (unsigned short)s;
        total += __popc(m);
    }
    __syncwarp();
    for (int j = lane; j < total; j += 32) {
        const int s = list[j];
        long long x[4] = {0, 0, 0, 0};
        for (int d = 0; d < nc; d++) {
            const int dd = d == DIM ? 3 : d;
            x[dd] = (long long)t.hi[d * kResSlots + s] * (1ll << kLimb) +
                    (long long)t.lo[d * kResSlots + s];
        }
        res_global_add(sums, msum, t.key[s], x, t.cnt[s], multi);
    }
}

// A cell's record, both halves: one 32-byte sector, two loads issued
// together (the axis half is loaded whatever the population, so that the
// rotation never waits for a second round trip).
__device__ __forceinline__ void res_load(const ResRec *rec, float4 &ca, float4 &cb) {
    const float4 *q = (const float4 *)rec;
    ca = __ldg(q);
    cb = __ldg(q + 1);
}
__device__ __forceinline__ void res_load(const ResRec *rec, float4 &ca, float4 &cb,
                                         uint64_t pol) {
    const float4 *q = (const float4 *)rec;
    ca = ldg_hint(q, pol);
    cb = ldg_hint(q + 1, pol);
}

// v' = u + R (v - u) from a cell's record (Rodrigues form, see ResRec);
// cells of fewer than two particles leave v unchanged.
template <int DIM>
__device__ __forceinline__ void res_apply(float4 &W, const float4 ca, const float4 cb, float Cs,
                                          float Sn) {
    if (__float_as_int(ca.w) > 1) {
        const float w0 = W.x - ca.x, w1 = W.y - ca.y;
        if (DIM == 3) {
            const float w2 = W.z - ca.z;
            const float ld = (cb.x * w0 + cb.y * w1 + cb.z * w2) * (1.f - Cs);
            W.x = ca.x + (Cs * w0 + ld * cb.x + Sn * (cb.y * w2 - cb.z * w1));
            W.y = ca.y + (Cs * w1 + ld * cb.y + Sn * (cb.z * w0 - cb.x * w2));
            W.z = ca.z + (Cs * w2 + ld * cb.z + Sn * (cb.x * w1 - cb.y * w0));
        } else {
            W.x = ca.x + (Cs * w0 - Sn * w1);
            W.y = ca.y + (Sn * w0 + Cs * w1);
        }
    }
}

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The SRD axis of mpcd_rng_axis3 (same Philox draws, same FP64
// acceptance test of the Marsaglia pair, so the same pair is taken), with
// the square root and the products in FP32: the record holds the axis in
// FP32 anyway.
__device__ __forceinline__ void res_axis3(uint64_t seed, uint32_t replica, uint32_t step,
                                          uint32_t cell, float v[3]) {
    for (uint32_t blk = 0; blk < MPCD_RNG_MAX_BLOCKS; ++blk) {
        const mpcd_u4 r = mpcd_block(seed, replica, step, MPCD_STREAM_AXIS, cell, blk);
        for (int a = 0; a < 2; ++a) {
            const double x = MPCD_DSUB(MPCD_DMUL(2.0, mpcd_u01(a ? r.z : r.x)), 1.0);
            const double y = MPCD_DSUB(MPCD_DMUL(2.0, mpcd_u01(a ? r.w : r.y)), 1.0);
            const double q = MPCD_DADD(MPCD_DMUL(x, x), MPCD_DMUL(y, y));
            if (q <= 1.0) {
                const float f = 2.0f * sqrtf((float)MPCD_DSUB(1.0, q));
                v[0] = f * (float)x;
                v[1] = f * (float)y;
                v[2] = (float)MPCD_DSUB(1.0, MPCD_DMUL(2.0, q));
                return;
            }
        }
    }
    v[0] = 0.f;
    v[1] = 0.f;
    v[2] = 1.f;
}

// Cell pass: sums of this step -> u, axis record; the sums are cleared.
// Each thread takes kResCellsPer cells (their loads issued together); the
// block's records leave through shared memory as one contiguous range.
// Block 0 also clears the next step's accumulators.
constexpr int kResCellsPer = 2;
template <int DIM>
__global__ void __launch_bounds__(256) k_res_cells(const __grid_constant__ DevCfg c,
                                                   ResPlanes sums, unsigned long long *msum,
                                                   ResRec *crec, StepArgs sa, double *acc,
                                                   double *acc_next) {
    __shared__ float4 srec[2 * 256 * kResCellsPer];
    __shared__ double wsum[8][3];
    const int c0 = blockIdx.x * 256 * kResCellsPer;
    pdl_trigger();
    // The axes depend on the step and the cell only: they are drawn while
    // the particle pass before this kernel may still be running (for every
    // cell; cells of fewer than two particles then ignore theirs).
    float Lx[kResCellsPer][3];
#pragma unroll
    for (int q = 0; q < kResCellsPer; q++) {
        const int cell = c0 + q * 256 + threadIdx.x;
        Lx[q][0] = 0.f;
        Lx[q][1] = 0.f;
        Lx[q][2] = 1.f;
        if (DIM == 3 && cell < c.ncells) res_axis3(c.seed, c.replica, sa.step, (uint32_t)cell, Lx[q]);
    }
    pdl_wait();  // the sums are complete from here on
    const uint64_t keep = l2_evict_last();
    double av[3] = {0, 0, 0};
    if (blockIdx.x == 0 && threadIdx.x < ACC_WORDS) acc_next[threadIdx.x] = 0.0;
    ResSum s[kResCellsPer];
    unsigned long long ms[kResCellsPer];
#pragma unroll
    for (int q = 0; q < kResCellsPer; q++) {
        const int cell = c0 + q * 256 + threadIdx.x;
        s[q] = ResSum{{0, 0, 0}, 0};
        ms[q] = 0ull;
        if (cell < c.ncells) {
            s[q] = sums.load(cell);
            if (msum) ms[q] = msum[cell];
        }
    }
#pragma unroll
    for (int q = 0; q < kResCellsPer; q++) {
        const int cell = c0 + q * 256 + threadIdx.x;
        if (cell >= c.ncells) continue;
        sums.clear(cell, keep);
        if (msum) msum[cell] = 0ull;
        const int pop = (int)s[q].n;
        // u = weighted sum / divisor: the population (one species, in FP32:
        // the record is FP32) or the mass sum (several species, in FP64)
        float u[3] = {0.f, 0.f, 0.f};
        if (msum) {
            const double W = (double)(long long)ms[q] * kSumFxInv;
            if (pop > 0 && W > 0.0) {
                const double iW = 1.0 / W;
                for (int d = 0; d < DIM; d++) u[d] = (float)(((double)s[q].p[d] * kSumFxInv) * iW);
            }
        } else if (pop > 0) {
            const float ip = __frcp_rn((float)pop);
            for (int d = 0; d < DIM; d++) u[d] = (float)((double)s[q].p[d] * kSumFxInv) * ip;
        }
        for (int d = 0; d < DIM; d++) av[d] += (double)u[d];
        const bool rot = pop > 1 && DIM == 3;
        float4 *my = srec + 2 * (q * 256 + threadIdx.x);
        my[0] = make_float4(u[0], u[1], u[2], __int_as_float(pop));
        my[1] = make_float4(rot ? Lx[q][0] : 0.f, rot ? Lx[q][1] : 0.f, rot ? Lx[q][2] : 1.f, 0.f);
    }
    __syncthreads();
    {
        const int nrec = min(256 * kResCellsPer, c.ncells - c0);
        float4 *dst = (float4 *)(crec + c0);
        for (int j = threadIdx.x; j < 2 * nrec; j += 256) st_hint(dst + j, srec[j], keep);
    }
    // block sum of the avVel terms: warp shuffles, then one thread per block
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int d = 0; d < DIM; d++) {
        const double t = warp_sum_d(av[d]);
        if (lane == 0) wsum[wid][d] = t;
    }
    __syncthreads();
    if (threadIdx.x < DIM) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += wsum[w][threadIdx.x];
        atomicAdd(&acc[ACC_VCM + threadIdx.x], t);
    }
}

// Sort order of the 3D resident family: bricks of 4x4x4 cells in row-major
// brick order (fastest axis last), row-major inside a brick.  A block's 2048
// consecutive particles (about 3 bricks at 10 per cell) then cover a compact
// region of about 4 x 4 x 13 cells, whose cells on the next step's shifted
// grid (one more on each side) number about 350 instead of the ~550 of a
// row-major slab: fewer table entries per block, so fewer global additions
// in the flush.  The cell arrays stay row-major; only the particle order
// changes.
constexpr int kBrickBits = 2;  // 4 cells per brick side
__host__ __device__ __forceinline__ int res_brick_dim(int n1) {
    return (n1 + (1 << kBrickBits) - 1) >> kBrickBits;
}
__host__ __device__ __forceinline__ int res_brick_keys(const int N1[3]) {
    return res_brick_dim(N1[0]) * res_brick_dim(N1[1]) * res_brick_dim(N1[2]) << (3 * kBrickBits);
}
__host__ __device__ __forceinline__ int res_brick_key(const int N1[3], const int idx[3]) {
    constexpr int m = (1 << kBrickBits) - 1;
    const int b = ((idx[0] >> kBrickBits) * res_brick_dim(N1[1]) + (idx[1] >> kBrickBits)) *
                      res_brick_dim(N1[2]) +
                  (idx[2] >> kBrickBits);
    return (b << (3 * kBrickBits)) | ((idx[0] & m) << (2 * kBrickBits)) |
           ((idx[1] & m) << kBrickBits) | (idx[2] & m);
}

// Sort keys (brick order) and ranks of the mixed state on this step's grid.
static __global__ void __launch_bounds__(256)
    k_key_res3(const __grid_constant__ DevCfg c, MixState a, int n, int *key, int *rank,
               int *count, StepArgs sa, unsigned long long *status) {
    int esc_local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int ci[3], idx[3], e = 0;
        uint32_t f[3], t;
        pos_unpack(a.P[i], ci, f);
        for (int d = 0; d < 3; d++)
            idx[d] = fx_shift_axis(ci[d], f[d], sa.ks[d], c.L[d], c.pbc[d], t, e);
        esc_local += e;
        const int k = res_brick_key(c.N1, idx);
        key[i] = k;
        rank[i] = atomicAdd(&count[k], 1);
    }
    if (esc_local) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc_local);
}

enum { RES_STEP = 0, RES_SUM = 1 };

// Particle pass: block b owns particles [b * kResChunk, (b+1) * kResChunk),
// one per thread at a time (coalesced loads and stores).
//   RES_STEP: collide, stream, write the particle back in place, add it to
//             the next step's sums.
//   RES_SUM:  only add each particle to this step's sums (the first step,
//             or after the state was replaced).
// Both leave in P.w the linear index of the cell each particle was added
// to: the cell whose record it reads at the next RES_STEP (the re-sort
// moves P.w with the particle).
// Accumulation: each particle adds its limbs to its cell's entry in the
// block's table with native 32-bit shared-memory atomics (or, if the table
// has no slot for it, straight to global memory); at the end every table
// entry is added to the global sums once.
// LEAN: the common case of a fully periodic box, one species and no
// gravity, compiled without the general paths (walls, species, gravity).
template <int DIM, int MODE, bool LEAN>
__global__ void __launch_bounds__(kResThreads, MPCD_RES_MINB) k_res_parts(
    const __grid_constant__ DevCfg c, MixState a, int n,
    const ResRec *__restrict__ crec, ResPlanes sums, unsigned long long *msum, double *acc,
    unsigned long long *status, StepArgs sa) {
    extern __shared__ __align__(16) unsigned char res_smem[];
    __shared__ double red[8];
    const int tid = threadIdx.x;
    const bool multi = !LEAN && msum != nullptr;
    const int nc = multi ? DIM + 1 : DIM;
    ResTable t;
    t.bind(res_smem, nc);
    pdl_trigger();
#if MPCD_RES_BULK_PF
    // The block's whole chunk of particle records is requested into L2 at
    // once (16 bulk prefetches of 4 KB by warp 0), so that the loop's loads,
    // one particle ahead of the arithmetic, wait for L2 rather than for
    // DRAM.  A prefetch only moves lines into L2, which stays coherent with
    // the kernel before this one still writing them.  The particle stream
    // (prefetches, loads, stores) is marked evict_first and the cell records
    // evict_last, so that the records, written by the cell pass, are still
    // in L2 when the blocks of the last waves gather them.
    if (tid < 16) {
        const int j0 = blockIdx.x * kResChunk + (tid & 7) * 256;
        const int cnt = min(256, n - j0);
        if (cnt > 0) {
            const void *src = tid < 8 ? (const void *)(a.P + j0) : (const void *)(a.W + j0);
            prefetch_l2_bulk_hint(src, (uint32_t)cnt * 16u, l2_evict_first());
        }
    }
#endif
    {
        // keys to -1, everything after them to 0, in 16-byte stores (while
        // the kernel before this one may still be running)
        uint4 *w = (uint4 *)res_smem;
        const int nkey = kResSlots / 4, nall = res_table_init_bytes(nc) / 16;
        for (int j = tid; j < nall; j += kResThreads)
            w[j] = j < nkey ? make_uint4(~0u, ~0u, ~0u, ~0u) : make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    pdl_wait();  // records, sums and particles are complete from here on
    float ke = 0.f;     // one species: sum of v^2 (times m at the end)
    double ke_m = 0.0;  // several species: sum of m v^2
    int bounce = 0, esc = 0, bad = 0;
    const float gk[3] = {(float)(c.dt * c.grav[0]), (float)(c.dt * c.grav[1]),
                         (float)(c.dt * c.grav[2])};
    const float cosf_a = (float)c.cosA, sinf_a = (float)c.sinA;
    const int base = blockIdx.x * kResChunk;
    // Software pipeline: the next particle is loaded at the top of an
    // iteration, and its cell's record is requested halfway through it
    // (before the accumulation), so neither load is waited for.  The cell
    // is the one the particle was added to at the end of the previous step,
    // which that step left in P.w (clamped only as a guard).
    auto cur_cell = [&](const MixRec &q) { return (int)min(q.P.w, (unsigned)(c.ncells - 1)); };
    // the particle stream leaves L2 first; the records stay
    const uint64_t stream = l2_evict_first(), keep = l2_evict_last();
    // One species (LEAN): odd lanes add each particle to the table one
    // iteration late, so that an atomic instruction carries particles of two
    // different runs of 32 consecutive particles and fewer of its lanes add
    // to the same cell (same-address lanes serialise).
    const bool late = LEAN && (tid & 1);
    int pk = -1, pidx[3] = {0, 0, 0};
    float pv[3] = {0.f, 0.f, 0.f};
    MixRec nx;
    float4 na = make_float4(0.f, 0.f, 0.f, 0.f), nb = na;
    if (base + tid < n) {
        nx.P = ld_hint(a.P + base + tid, stream);
        nx.W = ld_hint(a.W + base + tid, stream);
        if (MODE == RES_STEP) res_load(crec + cur_cell(nx), na, nb, keep);
    }
#pragma unroll 1
    for (int it = 0; it < MPCD_RES_PPT; it++) {
        const int i = base + it * kResThreads + tid;
        if (i >= n) break;
        MixRec r = nx;
        const float4 ca = na, cb = nb;
        const bool more = it + 1 < MPCD_RES_PPT && i + kResThreads < n;
        if (more) {
            nx.P = ld_hint(a.P + i + kResThreads, stream);
            nx.W = ld_hint(a.W + i + kResThreads, stream);
        }
        if (!LEAN && c.grav_flag) {
            r.W.x += gk[0];
            r.W.y += gk[1];
            if (DIM == 3) r.W.z += gk[2];
        }
        const int sp = multi ? MixT<DIM>::sp(a, i) : 0;
        int k, kidx[3];
        if (MODE == RES_STEP) {
            res_apply<DIM>(r.W, ca, cb, cosf_a, sinf_a);
            float tt = r.W.x * r.W.x + r.W.y * r.W.y;
            if (DIM == 3) tt += r.W.z * r.W.z;
            if (multi)
                ke_m += c.mass[sp] * (double)tt;
            else
                ke += tt;
            if (LEAN) {
                fx_finish_periodic<DIM>(r.P, r.W, (float)c.dt, c.L, sa.ksn, kidx);
                k = cell_lin(c, kidx[0], kidx[1], kidx[2]);
            } else {
                k = MixT<DIM>::finish_idx(c, r, sp, sa, bounce, esc, kidx);
            }
            r.P.w = (unsigned)k;  // next step's cell, read back by cur_cell
            st_hint(a.P + i, r.P, stream);
            st_hint(a.W + i, r.W, stream);
            if (more) res_load(crec + cur_cell(nx), na, nb, keep);
            // the next step's load adds the same FP32 gravity kick
            if (!LEAN && c.grav_flag) {
                r.W.x += gk[0];
                r.W.y += gk[1];
                if (DIM == 3) r.W.z += gk[2];
            }
        } else {
            k = cur_key_idx<DIM>(c, r, sa, kidx);
            a.P[i] = make_uint4(r.P.x, r.P.y, r.P.z, (unsigned)k);
        }
        float vs[3] = {r.W.x, r.W.y, DIM == 3 ? r.W.z : 0.f};
        bool go = true;
        if (late) {
            // add the previous iteration's particle, keep this one
            const int tk = k;
            k = pk;
            pk = tk;
            for (int d = 0; d < 3; d++) {
                const int ti = kidx[d];
                kidx[d] = pidx[d];
                pidx[d] = ti;
                const float tv = vs[d];
                vs[d] = pv[d];
                pv[d] = tv;
            }
            go = k >= 0;
        }
        if (go)
            res_add<DIM>(t, c.res_mask, c.res_shift, sums, msum, k, kidx, vs,
                         multi ? c.mass[sp] : 1.0, multi, bad);
    }
    if (late && pk >= 0) res_add<DIM>(t, c.res_mask, c.res_shift, sums, msum, pk, pidx, pv, 1.0,
                                      false, bad);
    __syncthreads();
    res_flush<DIM>(t, sums, msum, multi);
    if (MODE == RES_STEP) {
        const double kt = multi ? ke_m : c.mass[0] * (double)ke;
        const double tk = block_sum256(kt, red);
        if (tid == 0) atomicAdd(&acc[ACC_KE], tk);
        if (bounce) atomicAdd(&status[ST_BOUNCE], (unsigned long long)bounce);
        if (esc) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc);
    }
    if (bad) atomicAdd(&status[ST_NONFINITE], (unsigned long long)bad);
}

// Slot bit fields of the tables for a box of sides L: per-axis low bits of
// the cell indices, so that the cells a block of particles lands in map to
// distinct, mostly consecutive slots (consecutive slots: distinct banks).
// 3D (brick order, k_key_res3): a block's particles span about one brick,
// 4 cells, of the two slower axes and a few bricks of the fastest, and their
// next cells add one on each side: 3 bits for each slower axis, the rest for
// the fastest.  2D (row order): the fastest axis gets up to all but 2 bits.
static inline void res_slot_bits(int dim, const int L[3], int shift[3], int mask[3]) {
    auto clog2 = [](int x) {
        int b = 0;
        while ((1 << b) < x) b++;
        return b;
    };
    int bits[3] = {0, 0, 0};
    if (dim == 3) {
        bits[0] = clog2(L[0]) < 3 ? clog2(L[0]) : 3;
        bits[1] = clog2(L[1]) < 3 ? clog2(L[1]) : 3;
        bits[2] = kResBits - bits[0] - bits[1];
        shift[2] = 0;
        shift[1] = bits[2];
        shift[0] = bits[2] + bits[1];
    } else {
        bits[1] = clog2(L[1]) < kResBits - 2 ? clog2(L[1]) : kResBits - 2;
        bits[0] = kResBits - bits[1];
        shift[1] = 0;
        shift[0] = bits[1];
        shift[2] = 0;
    }
    for (int d = 0; d < 3; d++) mask[d] = (1 << bits[d]) - 1;
}

}  // namespace MPCD_RES_NS
}  // namespace mpcd
