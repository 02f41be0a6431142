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

// Shifted-grid coordinate of one axis, exactly as gridShift_all + bin.
__device__ __forceinline__ int mix_shift_axis(int cidx, float o, double s, int L, int pbc,
                                              double &qs, int &esc) {
    double q = (double)cidx + (double)o;
    q = shift_fwd(q, s, L);
    qs = q;
    return bin_axis(q, L, pbc, 1, esc);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_bin_mix(const __grid_constant__ DevCfg c,
                                                 MixState st, int n, int *key, int *rank,
                                                 int *count, uint32_t step,
                                                 unsigned long long *status) {
    double s[3] = {0, 0, 0};
    if (c.galinv) mpcd_rng_shift(c.seed, c.replica, step, DIM, s);
    const float gx = (float)(c.dt * c.grav[0]), gy = (float)(c.dt * c.grav[1]),
                gz = (float)(c.dt * c.grav[2]);
    int esc_local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p = st.P[i];
        int ca, cb, cz;
        unpack_cell(__float_as_int(p.w), ca, cb, cz);
        int esc = 0;
        double qs;
        int a = mix_shift_axis(ca, p.x, s[0], c.L[0], c.pbc[0], qs, esc);
        int b = mix_shift_axis(cb, p.y, s[1], c.L[1], c.pbc[1], qs, esc);
        int z = 0;
        if (DIM == 3) z = mix_shift_axis(cz, p.z, s[2], c.L[2], c.pbc[2], qs, esc);
        esc_local += esc;
        int k = cell_lin(c, a, b, z);
        key[i] = k;
        rank[i] = atomicAdd(&count[k], 1);
        if (c.grav_flag) {
            float4 w = st.W[i];
            w.x += gx;
            w.y += gy;
            if (DIM == 3) w.z += gz;
            st.W[i] = w;
        }
    }
    if (esc_local) atomicAdd(&status[ST_ESCAPED], (unsigned long long)esc_local);
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
    double qs;
    mix_shift_axis(ca, p.x, s[0], c.L[0], c.pbc[0], qs, e);
    r[0] = qs - (double)cellc[0];
    mix_shift_axis(cb, p.y, s[1], c.L[1], c.pbc[1], qs, e);
    r[1] = qs - (double)cellc[1];
    r[2] = 0.0;
    if (DIM == 3) {
        mix_shift_axis(cz, p.z, s[2], c.L[2], c.pbc[2], qs, e);
        r[2] = qs - (double)cellc[2];
    }
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

template <int DIM>
__global__ void __launch_bounds__(256) k_cell_mix(const __grid_constant__ DevCfg c,
                                                  MixState st, const int *start,
                                                  uint32_t step, double *acc,
                                                  unsigned long long *status) {
    __shared__ double s_acc[ACC_WORDS];
    if (threadIdx.x < ACC_WORDS) s_acc[threadIdx.x] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    double s[3] = {0, 0, 0};
    if (c.galinv) mpcd_rng_shift(c.seed, c.replica, step, DIM, s);
    double ke = 0.0;
    int bounce = 0;
    if (cell < c.ncells) {
        const int b0 = start[cell], e0 = start[cell + 1], pop = e0 - b0;
        int cc[3];
        cell_coords(c, cell, cc[0], cc[1], cc[2]);
        const bool need_cm = (c.op == MPCD_COLL_RAT);
        double M = 0.0, pv[3] = {0, 0, 0}, pq[3] = {0, 0, 0};
        for (int j = b0 + lane; j < e0; j += 32) {
            int sp = st.sp ? st.sp[j] : 0;
            double m = c.mass[sp];
            float4 w = st.W[j];
            M += m;
            pv[0] += (double)w.x * m;
            pv[1] += (double)w.y * m;
            if (DIM == 3) pv[2] += (double)w.z * m;
            if (need_cm) {
                double r[3];
                mix_rel<DIM>(c, st.P[j], s, cc, r);
                for (int d = 0; d < DIM; d++) pq[d] += r[d] * m;
            }
        }
        M = warp_sum(M);
        double u[3] = {0, 0, 0}, cm[3] = {0, 0, 0};
        for (int d = 0; d < DIM; d++) {
            u[d] = warp_sum(pv[d]);
            if (need_cm) cm[d] = warp_sum(pq[d]);
            if (M > 0.0) {
                u[d] /= M;
                if (need_cm) cm[d] /= M;
            }
        }
        if (c.any_phantom && pop > 0 && pop < c.gndnst) {
            if (cell_cut_by_phantom<DIM>(c, cc[0], cc[1], cc[2], s)) {
                double invN = 1.0 / (c.gndnst - (double)pop);
                double sig = sqrt(c.kbt / invN);
                for (int d = 0; d < DIM; d++) {
                    float g = mpcd_rng_normal(c.seed, c.replica, step, MPCD_STREAM_GHOST,
                                              (uint32_t)cell, (uint32_t)d);
                    u[d] += sig * (double)g;
                    u[d] /= c.gndnst;
                }
            }
        }
        if (lane == 0)
            for (int d = 0; d < DIM; d++) atomicAdd(&s_acc[ACC_VCM + d], u[d]);
        if (pop > 1) {
            if (c.op == MPCD_COLL_ARBAXIS) {
                double L[3] = {0, 0, 1};
                float R[9];
                if (DIM == 3) mpcd_rng_axis3(c.seed, c.replica, step, (uint32_t)cell, L);
                srd_matrix<DIM, float>(c, L, R);
                const float ux = (float)u[0], uy = (float)u[1], uz = (float)u[2];
                for (int j = b0 + lane; j < e0; j += 32) {
                    float4 w = st.W[j];
                    float wx = w.x - ux, wy = w.y - uy, wz = DIM == 3 ? w.z - uz : 0.f;
                    if (DIM == 3) {
                        w.x = ux + (R[0] * wx + R[1] * wy + R[2] * wz);
                        w.y = uy + (R[3] * wx + R[4] * wy + R[5] * wz);
                        w.z = uz + (R[6] * wx + R[7] * wy + R[8] * wz);
                    } else {
                        w.x = ux + (R[0] * wx + R[1] * wy);
                        w.y = uy + (R[3] * wx + R[4] * wy);
                    }
                    st.W[j] = w;
                }
            } else {
                double rs[3] = {0, 0, 0};
                for (int j = b0 + lane; j < e0; j += 32) {
                    int sp = st.sp ? st.sp[j] : 0;
                    double rv[3];
                    thermal<DIM>(c, step, (uint32_t)__float_as_int(st.W[j].w), sp, rv);
                    for (int d = 0; d < DIM; d++) rs[d] += c.mass[sp] * rv[d];
                }
                for (int d = 0; d < DIM; d++) rs[d] = warp_sum(rs[d]) / M;
                double Wv[3] = {0, 0, 0};
                if (c.op == MPCD_COLL_RAT) {
                    double I6[6] = {0, 0, 0, 0, 0, 0}, Lm[3] = {0, 0, 0};
                    for (int j = b0 + lane; j < e0; j += 32) {
                        int sp = st.sp ? st.sp[j] : 0;
                        double m = c.mass[sp];
                        float4 w = st.W[j];
                        double r[3], rv[3], dv[3] = {0, 0, 0}, am[3];
                        mix_rel<DIM>(c, st.P[j], s, cc, r);
                        thermal<DIM>(c, step, (uint32_t)__float_as_int(w.w), sp, rv);
                        double vv[3] = {(double)w.x, (double)w.y, DIM == 3 ? (double)w.z : 0.0};
                        for (int d = 0; d < 3; d++) r[d] = d < DIM ? r[d] - cm[d] : 0.0;
                        for (int d = 0; d < DIM; d++) dv[d] = m * (vv[d] - rv[d]);
                        I6[0] += m * (r[1] * r[1] + r[2] * r[2]);
                        I6[1] += m * (r[0] * r[0] + r[2] * r[2]);
                        I6[2] += m * (r[0] * r[0] + r[1] * r[1]);
                        I6[3] += m * r[0] * r[1];
                        I6[4] += m * r[0] * r[2];
                        I6[5] += m * r[1] * r[2];
                        cross3(r, dv, am);
                        for (int d = 0; d < 3; d++) Lm[d] += am[d];
                    }
                    for (int k = 0; k < 6; k++) I6[k] = warp_sum(I6[k]);
                    for (int d = 0; d < 3; d++) Lm[d] = warp_sum(Lm[d]);
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
                    for (int x = 0; x < 3; x++)
                        for (int y = 0; y < 3; y++) Wv[x] += II[x * 3 + y] * Lm[y];
                }
                for (int j = b0 + lane; j < e0; j += 32) {
                    int sp = st.sp ? st.sp[j] : 0;
                    float4 w = st.W[j];
                    double rv[3];
                    thermal<DIM>(c, step, (uint32_t)__float_as_int(w.w), sp, rv);
                    double damp = c.damp[sp];
                    double nv[3];
                    if (c.op == MPCD_COLL_MPCAT) {
                        for (int d = 0; d < DIM; d++)
                            nv[d] = u[d] + rv[d] - rs[d] - damp * u[d] / (double)pop;
                    } else {
                        double r[3], ang[3];
                        mix_rel<DIM>(c, st.P[j], s, cc, r);
                        for (int d = 0; d < 3; d++) r[d] = d < DIM ? r[d] - cm[d] : 0.0;
                        cross3(Wv, r, ang);
                        for (int d = 0; d < DIM; d++)
                            nv[d] = u[d] + rv[d] - rs[d] - damp * u[d] + ang[d];
                    }
                    w.x = (float)nv[0];
                    w.y = (float)nv[1];
                    if (DIM == 3) w.z = (float)nv[2];
                    st.W[j] = w;
                }
            }
        }
        // ---- TEMP, stream (FP32), walls (FP64), exact periodic wrap ----
        const float dtf = (float)c.dt;
        for (int j = b0 + lane; j < e0; j += 32) {
            int sp = st.sp ? st.sp[j] : 0;
            float4 p = st.P[j];
            float4 w = st.W[j];
            double t = (double)w.x * (double)w.x + (double)w.y * (double)w.y;
            if (DIM == 3) t += (double)w.z * (double)w.z;
            ke += c.mass[sp] * t;
            int ci[3];
            unpack_cell(__float_as_int(p.w), ci[0], ci[1], ci[2]);
            float o[3] = {p.x, p.y, p.z};
            float vv[3] = {w.x, w.y, w.z};
            for (int d = 0; d < DIM; d++) {
                o[d] = fmaf(dtf, vv[d], o[d]);
                carry(o[d], ci[d]);
            }
            if (c.n_solid > 0) {
                double q[3] = {0, 0, 0}, v[3] = {0, 0, 0};
                for (int d = 0; d < DIM; d++) {
                    q[d] = (double)ci[d] + (double)o[d];
                    v[d] = (double)vv[d];
                }
                bool inside = false;
                for (int wi = 0; wi < c.n_walls; wi++) {
                    const DevWall &wl = c.walls[wi];
                    if (!wl.periodic && wall_W(wl, q, wl.Q, DIM) < 0.0) inside = true;
                }
                if (inside) {
                    bounce += wall_collisions<DIM>(c, q, v, sp, true);
                    for (int d = 0; d < DIM; d++) {
                        double f = floor(q[d]);
                        ci[d] = (int)f;
                        o[d] = (float)(q[d] - f);
                        if (o[d] >= 1.0f) {
                            o[d] = 0.0f;
                            ci[d] += 1;
                        }
                        vv[d] = (float)v[d];
                    }
                }
            }
            for (int d = 0; d < DIM; d++) {
                if (c.pbc[d]) {
                    if (ci[d] < 0 || ci[d] >= c.L[d]) ci[d] = ((ci[d] % c.L[d]) + c.L[d]) % c.L[d];
                } else {
                    if (ci[d] < 0) ci[d] = 0;  // escaped; counted by the next bin
                    if (ci[d] > c.L[d]) ci[d] = c.L[d];
                }
            }
            p.x = o[0];
            p.y = o[1];
            p.z = DIM == 3 ? o[2] : 0.0f;
            p.w = __int_as_float(pack_cell(ci[0], ci[1], DIM == 3 ? ci[2] : 0));
            w.x = vv[0];
            w.y = vv[1];
            if (DIM == 3) w.z = vv[2];
            st.P[j] = p;
            st.W[j] = w;
        }
    }
    ke = warp_sum(ke);
    if (lane == 0) atomicAdd(&s_acc[ACC_KE], ke);
    if (bounce) atomicAdd(&status[ST_BOUNCE], (unsigned long long)bounce);
    __syncthreads();
    if (threadIdx.x < ACC_WORDS) atomicAdd(&acc[threadIdx.x], s_acc[threadIdx.x]);
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

static inline int mix_step(MixState *mx, int &cur, const DevCfg &c, int n, uint32_t step,
                           int *key, int *rank, int *count, int *start, int *part, int nscan,
                           double *acc, unsigned long long *status, cudaStream_t stream,
                           int sm_count, int *launches) {
    MixState a = mx[cur], b = mx[1 - cur];
    int gb = (n + 255) / 256;
    if (gb > sm_count * 8) gb = sm_count * 8;
    if (gb < 1) gb = 1;
    int gc = (int)(((long long)c.ncells * 32 + 255) / 256);
    if (c.dim == 3)
        k_bin_mix<3><<<gb, 256, 0, stream>>>(c, a, n, key, rank, count, step, status);
    else
        k_bin_mix<2><<<gb, 256, 0, stream>>>(c, a, n, key, rank, count, step, status);
    k_scan_partial<<<nscan, 256, 0, stream>>>(count, c.ncells, part);
    k_scan_apply<<<nscan, 256, 0, stream>>>(count, c.ncells, part, start, acc);
    k_scatter_mix<<<gb, 256, 0, stream>>>(a, b, n, key, rank, start);
    if (c.dim == 3)
        k_cell_mix<3><<<gc, 256, 0, stream>>>(c, b, start, step, acc, status);
    else
        k_cell_mix<2><<<gc, 256, 0, stream>>>(c, b, start, step, acc, status);
    if (cudaGetLastError() != cudaSuccess) return MPCD_ERR_CUDA;
    cur = 1 - cur;
    *launches = 5;
    return MPCD_OK;
}

}  // namespace mpcd
