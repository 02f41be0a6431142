// mpcd_mixed.cuh -- the mixed-precision form of the solvent timestep.
//
// Particle state, 32 bytes per particle in two 16-byte records:
//   P = {X, Y, Z, 0} (uint4)         per axis one 32-bit fixed-point word:
//                                    the cell index in the top 10 bits and
//                                    the offset within the cell in the low
//                                    22 bits (X = cell * 2^22 + offset * 2^22)
//   W = {vx, vy, vz, pid} (float4)   FP32 velocity + original particle index
// The sub-cell offset has a uniform resolution of 2^-22 cell whatever the box
// size (an FP32 offset in [0,1) has 2^-24 at best).  Grid shifts are taken
// with 22 fraction bits (the reference draws a 32-bit uniform, rand.c:365-368,
// whose low 10 bits are dropped here), and shifting, wrapping and binning are
// exact integer operations following the reference's gridShift_all/bin rules
// (mpc.c:728-736, 958-968).  The periodic wrap is an exact integer wrap (the
// reference shifts by L(1-2e-8) instead, bc.c:769).  Streaming adds the FP32
// displacement dt*v rounded to the nearest 2^-22.  Cell sums, the MPC-AT+a
// inertia tensor and its inverse are FP64 or exact fixed point; the SRD
// rotation and streaming are FP32.
//
// Helpers that take a (cell index, 32-bit offset f) pair use f = offset word
// << 10, so f always has its low 10 bits zero, as do the shift words.
#pragma once

#include "mpcd_device.cuh"
#include "mpcd_fp64.cuh"

namespace mpcd {

struct MixState {
    uint4 *P;
    float4 *W;
    int *sp;    // species (nullptr for one species)
    float2 *U;  // nematic orientation (2D; nullptr when isotropic)
};

constexpr int kCellBits = 10;
constexpr int kFracBits = 22;                      // offset bits of a position word
constexpr uint32_t kShiftMask = 0xFFFFFC00u;       // 32-bit shift words keep 22 bits
constexpr double kFx = 4294967296.0;               // 2^32
constexpr double kFxInv = 2.3283064365386963e-10;  // 2^-32

// (cell index, 32-bit offset) per axis of a position record, and back.
__host__ __device__ __forceinline__ void pos_unpack(const uint4 &P, int ci[3], uint32_t f[3]) {
    ci[0] = (int)(P.x >> kFracBits);
    ci[1] = (int)(P.y >> kFracBits);
    ci[2] = (int)(P.z >> kFracBits);
    f[0] = P.x << kCellBits;
    f[1] = P.y << kCellBits;
    f[2] = P.z << kCellBits;
}
__host__ __device__ __forceinline__ uint4 pos_pack(const int ci[3], const uint32_t f[3]) {
    uint4 P;
    P.x = ((uint32_t)ci[0] << kFracBits) | (f[0] >> kCellBits);
    P.y = ((uint32_t)ci[1] << kFracBits) | (f[1] >> kCellBits);
    P.z = ((uint32_t)ci[2] << kFracBits) | (f[2] >> kCellBits);
    P.w = 0u;
    return P;
}

static inline int mix_check(const DevCfg &c) {
    for (int d = 0; d < 3; d++)
        if (c.N1[d] > (1 << kCellBits)) return MPCD_ERR_UNSUPPORTED;
    return MPCD_OK;
}

static inline void mix_free(MixState &s) {
    cudaFree(s.P);
    cudaFree(s.W);
    cudaFree(s.sp);
    cudaFree(s.U);
    s.P = nullptr;
    s.W = nullptr;
    s.sp = nullptr;
    s.U = nullptr;
}

static inline int mix_alloc(MixState &s, size_t n, const DevCfg &c) {
    if (cudaMalloc((void **)&s.P, n * sizeof(uint4)) != cudaSuccess) return MPCD_ERR_NOMEM;
    if (cudaMalloc((void **)&s.W, n * sizeof(float4)) != cudaSuccess) return MPCD_ERR_NOMEM;
    if (c.n_species > 1 && cudaMalloc((void **)&s.sp, n * sizeof(int)) != cudaSuccess)
        return MPCD_ERR_NOMEM;
    if (c.lc && cudaMalloc((void **)&s.U, n * sizeof(float2)) != cudaSuccess)
        return MPCD_ERR_NOMEM;
    return MPCD_OK;
}

// Shifted-grid cell index of one axis for the position ci + f*2^-32 and the
// shift k*2^-32, following gridShift_all + bin: with Q' = Q + s, Q' is
// wrapped by -L when L < Q' <= L + s, the cell is trunc(Q'), and index L maps
// to 0 on periodic axes.  'rel' returns the fixed-point position of Q'
// within the returned cell.
__device__ __forceinline__ int fx_shift_axis(int ci, uint32_t f, uint32_t k, int L, int pbc,
                                             uint32_t &rel, int &esc) {
    const uint32_t t = f + k;  // fraction of f + k
    const bool cy = t < f;     // f + k >= 2^32, i.e. o + s >= 1
    int a;
    rel = t;
    if (ci <= L - 2) {
        a = ci + (cy ? 1 : 0);
    } else if (ci == L - 1) {
        if (cy && t != 0u)
            a = 0;  // Q' > L: wrapped into cell 0
        else if (cy)
            a = L;  // Q' == L exactly: not wrapped
        else
            a = L - 1;
    } else {  // ci == L: possible on non-periodic axes only
        if (f == 0u && k != 0u)
            a = 0;  // L < Q' <= L + s: wrapped
        else
            a = L + (cy ? 1 : 0);
    }
    if (pbc && a == L) a = 0;
    if (a < 0 || a > L) {
        esc = 1;
        a = a < 0 ? 0 : L;
    }
    return a;
}

// fx_shift_axis for a periodic axis and a cell index in [0, L): the shifted
// cell is ci + carry, index L wrapping to 0 (both the gridShift wrap and
// bin's L -> 0 rule reduce to this).
__device__ __forceinline__ int fx_shift_axis_pbc(int ci, uint32_t f, uint32_t k, int L) {
    const uint32_t t = f + k;
    const int a = ci + (t < f ? 1 : 0);
    return a == L ? 0 : a;
}

// Position of record p on the shifted grid relative to the origin of its
// shifted cell, in cell units (exact in FP64).
template <int DIM>
__device__ __forceinline__ void mix_rel(const DevCfg &c, const uint4 &p, const uint32_t *k,
                                        double *r) {
    int ci[3], e = 0;
    uint32_t f[3], t;
    pos_unpack(p, ci, f);
    fx_shift_axis(ci[0], f[0], k[0], c.L[0], c.pbc[0], t, e);
    r[0] = (double)t * kFxInv;
    fx_shift_axis(ci[1], f[1], k[1], c.L[1], c.pbc[1], t, e);
    r[1] = (double)t * kFxInv;
    r[2] = 0.0;
    if (DIM == 3) {
        fx_shift_axis(ci[2], f[2], k[2], c.L[2], c.pbc[2], t, e);
        r[2] = (double)t * kFxInv;
    }
}

// rint(v * 2^32) as two signed limbs, hi * 2^20 + lo with |lo| <= 2^19,
// for |v| < 1024, from FP32 adds and multiplies and integer operations only
// (no conversion instructions).  a = v 2^12 is exact; adding 1.5 * 2^23
// rounds it to the nearest integer hi (ties to even), which the sum holds
// in its low mantissa bits; f = a - hi is exact (Sterbenz) and in
// [-1/2, 1/2], g = f 2^20 is exact, and lo = rint(g) by the same addition.
// Since hi 2^20 is an even integer, rint(v 2^32) = hi 2^20 + rint(g), ties
// included.  Returns false (limbs undefined) for |v| >= 1024 or non-finite v.
// fx_limbs without the range check, for |v| < 1024 known to the caller.
__device__ __forceinline__ void fx_limbs_unchecked(float v, int &hi, int &lo) {
    const float kMagic = 12582912.0f;  // 1.5 * 2^23
    const float a = __fmul_rn(v, 4096.0f);
    const float s = __fadd_rn(a, kMagic);
    const float r = __fadd_rn(s, -kMagic);
    const float g = __fmul_rn(__fadd_rn(a, -r), 1048576.0f);
    hi = __float_as_int(s) - 0x4B400000;
    lo = __float_as_int(__fadd_rn(g, kMagic)) - 0x4B400000;
}
__device__ __forceinline__ bool fx_limbs(float v, int &hi, int &lo) {
    const float kMagic = 12582912.0f;  // 1.5 * 2^23
    const float a = __fmul_rn(v, 4096.0f);
    if (!(fabsf(a) < 4194304.0f)) return false;  // 2^22
    const float s = __fadd_rn(a, kMagic);
    const float r = __fadd_rn(s, -kMagic);
    const float g = __fmul_rn(__fadd_rn(a, -r), 1048576.0f);
    hi = __float_as_int(s) - 0x4B400000;
    lo = __float_as_int(__fadd_rn(g, kMagic)) - 0x4B400000;
    return true;
}

// rint(dx * 2^22) for |dx| < 0.999, from one FP32 multiply and one add of
// 1.5 * 2^23 (ties to even), read back from the sum's mantissa bits.
__device__ __forceinline__ int fx_rint22(float dx) {
    return __float_as_int(__fadd_rn(__fmul_rn(dx, 4194304.0f), 12582912.0f)) - 0x4B400000;
}
constexpr float kStreamFast = 0.999f;  // |dx| below this: |rint(dx 2^22)| < 2^22

// Stream one axis by the FP32 displacement dx: exact fixed-point add of
// rint(dx * 2^22) units of 2^-22 cell.
__device__ __forceinline__ void fx_stream(uint32_t &f, int &ci, float dx) {
    if (fabsf(dx) < kStreamFast) {
        const uint32_t nf = f + ((uint32_t)fx_rint22(dx) << kCellBits);
        ci += dx >= 0.0f ? (nf < f ? 1 : 0) : (nf > f ? -1 : 0);
        f = nf;
        return;
    }
    const long long disp = __float2ll_rn(dx * 4194304.0f) * (1ll << kCellBits);
    const long long nq = (long long)f + disp;
    ci += (int)(nq >> 32);
    f = (uint32_t)nq;
}

// Streaming, exact periodic wrap and next-step cell indices of one record
// in a fully periodic box of L cells per axis, the next grid shift ksn (as
// 32-bit fractions).  Shared by every mixed-precision kernel family so that
// they stream identically.
template <int DIM>
__device__ __forceinline__ void fx_finish_periodic(uint4 &P, const float4 &W, float dtf,
                                                   const int L[3], const uint32_t ksn[3],
                                                   int idx[3]) {
    const float dx[3] = {dtf * W.x, dtf * W.y, dtf * W.z};
    idx[0] = idx[1] = idx[2] = 0;
    bool fast = fabsf(dx[0]) < kStreamFast && fabsf(dx[1]) < kStreamFast;
    if (DIM == 3) fast = fast && fabsf(dx[2]) < kStreamFast;
    if (fast) {
        // directly on the position words: add, one-period wrap (a word at
        // or above L 2^22 either crossed the top face or, for a negative
        // step, wrapped below zero), next cell from the shifted word
        uint32_t X[3] = {P.x, P.y, P.z};
        for (int d = 0; d < DIM; d++) {
            const int st = fx_rint22(dx[d]);
            const uint32_t Lw = (uint32_t)L[d] << kFracBits;
            uint32_t x = X[d] + (uint32_t)st;
            if (x >= Lw) x = st < 0 ? x + Lw : x - Lw;
            X[d] = x;
            const int a = (int)((x + (ksn[d] >> kCellBits)) >> kFracBits);
            idx[d] = a == L[d] ? 0 : a;
        }
        P.x = X[0];
        P.y = X[1];
        P.z = DIM == 3 ? X[2] : 0u;
        return;
    }
    int ci[3];
    uint32_t f[3];
    pos_unpack(P, ci, f);
    for (int d = 0; d < DIM; d++) {
        fx_stream(f[d], ci[d], dx[d]);
        ci[d] = ((ci[d] % L[d]) + L[d]) % L[d];
        idx[d] = fx_shift_axis_pbc(ci[d], f[d], ksn[d], L[d]);
    }
    if (DIM == 2) {
        ci[2] = 0;
        f[2] = 0u;
    }
    P = pos_pack(ci, f);
}

// Current-step cell indices of a record in a fully periodic box.
template <int DIM>
__device__ __forceinline__ void fx_cur_idx_periodic(const uint4 &P, const int L[3],
                                                    const uint32_t ks[3], int idx[3]) {
    const uint32_t X[3] = {P.x, P.y, P.z};
    idx[2] = 0;
    for (int d = 0; d < DIM; d++) {
        const int a = (int)((X[d] + (ks[d] >> kCellBits)) >> kFracBits);
        idx[d] = a == L[d] ? 0 : a;
    }
}

// Fixed-point representation of a coordinate (host and device).
__host__ __device__ __forceinline__ void fx_from_double(double q, int &ci, uint32_t &f) {
    double fl = floor(q);
    double fr = (q - fl) * 4194304.0;  // 2^22
    long long r = (long long)(fr + 0.5);
    ci = (int)fl;
    if (r >= (1LL << kFracBits)) {
        ci += 1;
        r = 0;
    }
    f = (uint32_t)r << kCellBits;
}


// Reordering of the state into counting-sort order, as a gather: k_perm scatters only the 4-byte source
// index of each destination slot, then k_gather_mix reads each destination's
// record from its source and writes the new order with coalesced stores
// (16-byte scattered writes would each touch a 32-byte sector).
static __global__ void __launch_bounds__(256) k_perm(int n, const int *key, const int *rank,
                                                     const int *start, int *perm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        perm[start[key[i]] + rank[i]] = i;
}
static __global__ void __launch_bounds__(256) k_gather_mix(MixState a, MixState b, int n,
                                                           const int *perm) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int i = __ldg(perm + j);
        b.P[j] = a.P[i];
        b.W[j] = a.W[i];
        if (a.sp) b.sp[j] = a.sp[i];
        if (a.U) b.U[j] = a.U[i];
    }
}

// Device-side conversion of an upload in the caller's FP64 layout (3 doubles
// per vector, original particle order) to the packed representation (the
// download's gather is k_mix_gather_aos in mpcd_xfer.cuh).  A non-finite
// value, a position outside the grid or a species id out of range counts in
// *err and leaves that particle unwritten.  Without U, a nematic state starts
// every orientation at (1, 0).
static __global__ void __launch_bounds__(256) k_mix_from_f64(MixState s,
                                                             const __grid_constant__ DevCfg c,
                                                             int n, const double *Q,
                                                             const double *V, const double *U,
                                                             const int *spid, int *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int ci[3] = {0, 0, 0};
        uint32_t f[3] = {0u, 0u, 0u};
        bool ok = true;
        for (int d = 0; d < c.dim; d++) {
            const double q = Q[3 * (size_t)i + d], v = V[3 * (size_t)i + d];
            if (!isfinite(q) || !isfinite(v)) {
                ok = false;
                break;
            }
            fx_from_double(q, ci[d], f[d]);
            if (ci[d] < 0 || ci[d] > c.L[d]) ok = false;
        }
        const int sp = spid ? spid[i] : 0;
        if (sp < 0 || sp >= c.n_species) ok = false;
        if (!ok) {
            atomicAdd(err, 1);
            continue;
        }
        s.P[i] = pos_pack(ci, f);
        s.W[i] = make_float4((float)V[3 * (size_t)i], (float)V[3 * (size_t)i + 1],
                             c.dim == 3 ? (float)V[3 * (size_t)i + 2] : 0.f, __int_as_float(i));
        if (s.sp) s.sp[i] = sp;
        if (s.U)
            s.U[i] = U ? make_float2((float)U[3 * (size_t)i], (float)U[3 * (size_t)i + 1])
                       : make_float2(1.f, 0.f);
    }
}
}  // namespace mpcd
