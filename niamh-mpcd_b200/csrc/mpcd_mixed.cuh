// mpcd_mixed.cuh -- the mixed-precision form of the solvent timestep.
//
// Particle state, 32 bytes per particle in two float4 records:
//   P = {ox, oy, oz, cell}   position = integer cell (10 bits per axis,
//                            packed) + FP32 offset in [0,1) within it
//   W = {vx, vy, vz, pid}    FP32 velocity + original particle index
// Positions never lose precision with box size, and the periodic wrap is an
// exact integer wrap (the reference shifts by L(1-2e-8) instead, bc.c:769).
// Shifted coordinates are formed exactly in FP64 (int + float + 32-bit
// shift fit in 53 bits), so cell keys follow the reference's gridShift/bin
// rules (mpc.c:728-736, 958-968) exactly.  Cell sums, the MPC-AT+a inertia
// tensor and its inverse are FP64; the SRD rotation and streaming are FP32.
#pragma once

#include "mpcd_device.cuh"
#include "mpcd_fp64.cuh"

namespace mpcd {

struct MixState {
    float4 *P;
    float4 *W;
    int *sp;  // species (nullptr for one species)
};

constexpr int kCellBits = 10;
constexpr int kCellMask = (1 << kCellBits) - 1;

__host__ __device__ __forceinline__ int pack_cell(int a, int b, int z) {
    return a | (b << kCellBits) | (z << (2 * kCellBits));
}
__host__ __device__ __forceinline__ void unpack_cell(int p, int &a, int &b, int &z) {
    a = p & kCellMask;
    b = (p >> kCellBits) & kCellMask;
    z = (p >> (2 * kCellBits)) & kCellMask;
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
    s.P = s.W = nullptr;
    s.sp = nullptr;
}

static inline int mix_alloc(MixState &s, size_t n, const DevCfg &c) {
    if (cudaMalloc((void **)&s.P, n * sizeof(float4)) != cudaSuccess) return MPCD_ERR_NOMEM;
    if (cudaMalloc((void **)&s.W, n * sizeof(float4)) != cudaSuccess) return MPCD_ERR_NOMEM;
    if (c.n_species > 1 && cudaMalloc((void **)&s.sp, n * sizeof(int)) != cudaSuccess)
        return MPCD_ERR_NOMEM;
    return MPCD_OK;
}

// Shifted-grid cell index of one axis from (cell ci, offset o) and the grid
// shift s, following gridShift_all + bin (mpc.c:728-736, 958-968): with
// Q = ci + o and Q' = Q + s, Q' is wrapped by -L when L < Q' <= L + s, the
// cell is trunc(Q'), and index L maps to 0 on periodic axes.  Only t = o + s
// is formed in FP64 (exact in every case that can change the outcome); 'rel'
// returns Q' relative to the origin of the returned cell.
__device__ __forceinline__ int mix_shift_axis(int ci, float o, double s, int L, int pbc,
                                              double &rel, int &esc) {
    const double t = (double)o + s;
    int a;
    if (ci <= L - 2) {
        const bool cy = t >= 1.0;
        a = ci + (cy ? 1 : 0);
        rel = cy ? t - 1.0 : t;
    } else if (ci == L - 1) {
        if (t > 1.0) {  // Q' > L: wrapped into cell 0
            a = 0;
            rel = t - 1.0;
        } else if (t == 1.0) {  // Q' == L exactly: not wrapped
            a = L;
            rel = 0.0;
        } else {
            a = L - 1;
            rel = t;
        }
    } else {  // ci == L: possible on non-periodic axes only
        if (o == 0.0f && s > 0.0) {
            a = 0;
            rel = t;
        } else if (t >= 1.0) {
            a = L + 1;
            rel = t - 1.0;
        } else {
            a = L;
            rel = t;
        }
    }
    if (pbc && a == L) a = 0;
    if (a < 0 || a > L) {
        esc = 1;
        a = a < 0 ? 0 : L;
    }
    return a;
}

__global__ void __launch_bounds__(256) k_scatter_mix(MixState a, MixState b, int n,
                                                     const int *key, const int *rank,
                                                     const int *start) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int dst = start[key[i]] + rank[i];
        b.P[dst] = a.P[i];
        b.W[dst] = a.W[i];
        if (a.sp) b.sp[dst] = a.sp[i];
    }
}

// Position of particle record p on the shifted grid relative to the origin
// of its shifted cell (exact in FP64).
template <int DIM>
__device__ __forceinline__ void mix_rel(const DevCfg &c, const float4 &p, const double *s,
                                        const int *cellc, double *r) {
    int ca, cb, cz;
    unpack_cell(__float_as_int(p.w), ca, cb, cz);
    int e = 0;
    mix_shift_axis(ca, p.x, s[0], c.L[0], c.pbc[0], r[0], e);
    mix_shift_axis(cb, p.y, s[1], c.L[1], c.pbc[1], r[1], e);
    r[2] = 0.0;
    if (DIM == 3) mix_shift_axis(cz, p.z, s[2], c.L[2], c.pbc[2], r[2], e);
}

// Stream an offset by dt*v in FP32 and carry whole cells into the index.
__device__ __forceinline__ void carry(float &o, int &ci) {
    float f = floorf(o);
    if (f != 0.0f) {
        o -= f;
        ci += (int)f;
        if (o >= 1.0f) {  // rounding at the top edge
            o = 0.0f;
            ci += 1;
        }
    }
}

// Host-side conversion to and from the packed representation.
static inline int mix_upload(MixState &s, const DevCfg &c, int n, const double *Q,
                             const double *V, const int *spid, cudaStream_t stream) {
    std::vector<float4> P((size_t)n), W((size_t)n);
    for (int i = 0; i < n; i++) {
        int ci[3] = {0, 0, 0};
        float o[3] = {0.f, 0.f, 0.f};
        for (int d = 0; d < c.dim; d++) {
            double q = Q[3 * (size_t)i + d];
            double f = std::floor(q);
            ci[d] = (int)f;
            o[d] = (float)(q - f);
            if (o[d] >= 1.0f) {
                o[d] = 0.0f;
                ci[d] += 1;
            }
            if (ci[d] < 0 || ci[d] > c.L[d]) return MPCD_ERR_ARG;
        }
        P[i] = make_float4(o[0], o[1], o[2], __int_as_float_host(pack_cell(ci[0], ci[1], ci[2])));
        W[i] = make_float4((float)V[3 * (size_t)i], (float)V[3 * (size_t)i + 1],
                           c.dim == 3 ? (float)V[3 * (size_t)i + 2] : 0.f,
                           __int_as_float_host(i));
    }
    if (cudaMemcpyAsync(s.P, P.data(), (size_t)n * sizeof(float4), cudaMemcpyHostToDevice,
                        stream) != cudaSuccess)
        return MPCD_ERR_CUDA;
    if (cudaMemcpyAsync(s.W, W.data(), (size_t)n * sizeof(float4), cudaMemcpyHostToDevice,
                        stream) != cudaSuccess)
        return MPCD_ERR_CUDA;
    if (s.sp) {
        std::vector<int> sp((size_t)n);
        for (int i = 0; i < n; i++) sp[i] = spid ? spid[i] : 0;
        if (cudaMemcpyAsync(s.sp, sp.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice,
                            stream) != cudaSuccess)
            return MPCD_ERR_CUDA;
        if (cudaStreamSynchronize(stream) != cudaSuccess) return MPCD_ERR_CUDA;
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) return MPCD_ERR_CUDA;
    return MPCD_OK;
}

static inline int mix_download(const MixState &s, const DevCfg &c, int n, double *Q,
                               double *V) {
    std::vector<float4> P((size_t)n), W((size_t)n);
    if (cudaMemcpy(P.data(), s.P, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return MPCD_ERR_CUDA;
    if (cudaMemcpy(W.data(), s.W, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return MPCD_ERR_CUDA;
    for (int i = 0; i < n; i++) {
        int pid = __float_as_int_host(W[i].w);
        if (pid < 0 || pid >= n) return MPCD_ERR_STATE;
        int ci[3];
        unpack_cell(__float_as_int_host(P[i].w), ci[0], ci[1], ci[2]);
        float o[3] = {P[i].x, P[i].y, P[i].z};
        float v[3] = {W[i].x, W[i].y, W[i].z};
        for (int d = 0; d < 3; d++) {
            if (Q) Q[3 * (size_t)pid + d] = d < c.dim ? (double)ci[d] + (double)o[d] : 0.0;
            if (V) V[3 * (size_t)pid + d] = d < c.dim ? (double)v[d] : 0.0;
        }
    }
    return MPCD_OK;
}

}  // namespace mpcd
