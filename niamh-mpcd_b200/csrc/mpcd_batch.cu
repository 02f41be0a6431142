// mpcd_batch.cu -- an ensemble of independent periodic 3D SRD boxes of
// different sizes, stepped together (mixed precision, resident kernel
// family).  Every kernel of a step runs once for the whole ensemble, driven
// by a per-box table; the step number lives in device memory, so one step is
// a fixed sequence of launches that is captured once in a CUDA graph and
// replayed.
//
// Layout: box b owns a run of particle slots starting at a multiple of the
// particle pass's chunk (padding slots carry pid -1 and are never moved by
// the physics) and a run of cells starting at a multiple of the cell pass's
// block, holding its (L+1)^3 cells, one extra "padding cell" that the
// counting sort sends padding slots to, and alignment.  A block of either
// pass therefore belongs to exactly one box, found in a per-block table.
//
// Box b uses the generator key (seed_b, replica b), so its trajectory is
// identical, bit for bit, to that of a single-box handle created with the
// same seed and replica (the resident family's sums are exact and
// order-independent).
// The ensemble's boxes are small (sides 8 to 32 in the ensemble benchmark):
// a 1024-slot table per block, so that four blocks fit on an SM.
#define MPCD_RES_SLOTS 1024
#define MPCD_RES_MINB 4
#define MPCD_RES_NS res_s1024_b4

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "mpcd_gpu.h"
#include "mpcd_device.cuh"
#include "mpcd_fp64.cuh"
#include "mpcd_mixed.cuh"
#include "mpcd_tile.cuh"
#include "mpcd_split.cuh"
#include "mpcd_resident.cuh"

using namespace mpcd;

int mpcd_build_devcfg(const mpcd_config *cfg, DevCfg *dc);

namespace {

constexpr int kCellsPerBlock = 256 * kResCellsPer;

struct BatchBox {
    int L[3];
    int cell0;   // first cell (global index)
    int ncells;  // (L+1)^3
    int part0;   // first particle slot (multiple of kResChunk)
    int npart;   // particles
    int nslots;  // slots including padding (multiple of kResChunk)
    int res_shift[3], res_mask[3];
    uint64_t seed;
    uint32_t replica;
    int key0;  // first sort key: the box's cells in brick order, then its padding key
    int g0;    // first of the box's particles in the caller's (box-major) order
    int pad_;
};

struct BatchStep {
    uint32_t ks[3], ksn[3];
    uint32_t step;
    uint32_t pad_;
};

// Grid shifts of the current and the next step for every box, from the
// device step counter (mpcd_rng_shift: s = 32-bit uniform * 2^-32).
__global__ void k_bat_shift(const BatchBox *box, int nb, BatchStep *st, const uint32_t *counter,
                            int galinv) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t step = *counter;
    BatchStep o;
    o.step = step;
    o.pad_ = 0u;
    for (int d = 0; d < 3; d++) o.ks[d] = o.ksn[d] = 0u;
    if (galinv) {
        const mpcd_u4 r = mpcd_block(box[b].seed, box[b].replica, step, MPCD_STREAM_SHIFT, 0u, 0u);
        const mpcd_u4 q =
            mpcd_block(box[b].seed, box[b].replica, step + 1u, MPCD_STREAM_SHIFT, 0u, 0u);
        // position words carry 22 fraction bits (mpcd_mixed.cuh)
        o.ks[0] = r.x & kShiftMask;
        o.ks[1] = r.y & kShiftMask;
        o.ks[2] = r.z & kShiftMask;
        o.ksn[0] = q.x & kShiftMask;
        o.ksn[1] = q.y & kShiftMask;
        o.ksn[2] = q.z & kShiftMask;
    }
    st[b] = o;
}

__global__ void k_bat_advance(uint32_t *counter) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *counter += 1u;
}

// Conversion of the caller's FP64 positions and velocities (3 doubles per
// particle, boxes one after another) into the slot layout, on the device:
// slot s of box b holds the box's particle s - part0 (or is padding: pid
// -1).  A position outside its box counts in *err.
__global__ void __launch_bounds__(256) k_bat_from_f64(const BatchBox *box, const int *chunk_box,
                                                      MixState a, int nslots, const double *Q,
                                                      const double *V, int *err) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
         s += gridDim.x * blockDim.x) {
        const BatchBox &bx = box[chunk_box[s / kResChunk]];
        const int j = s - bx.part0;
        if (j >= bx.npart) {
            a.P[s] = make_uint4(0u, 0u, 0u, 0u);
            a.W[s] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
            continue;
        }
        const size_t gi = (size_t)bx.g0 + (size_t)j;
        int ci[3];
        uint32_t f[3];
        bool ok = true;
        for (int d = 0; d < 3; d++) {
            const double q = Q[3 * gi + d];
            if (!(q >= 0.0 && q < (double)bx.L[d]) || !isfinite(V[3 * gi + d])) ok = false;
            fx_from_double(ok ? q : 0.0, ci[d], f[d]);
            if (ci[d] >= bx.L[d]) ci[d] -= bx.L[d];
        }
        if (!ok) atomicAdd(err, 1);
        a.P[s] = pos_pack(ci, f);
        a.W[s] = make_float4((float)V[3 * gi], (float)V[3 * gi + 1], (float)V[3 * gi + 2],
                             __int_as_float((int)gi));
    }
}

// The inverse: each real slot's particle to its place in the caller's order.
__global__ void __launch_bounds__(256) k_bat_to_f64(MixState a, int nslots, int n, double *Q,
                                                    double *V, int *err) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
         s += gridDim.x * blockDim.x) {
        const float4 w = a.W[s];
        const int pid = __float_as_int(w.w);
        if (pid < 0) continue;
        if (pid >= n) {
            atomicAdd(err, 1);
            continue;
        }
        int ci[3];
        uint32_t f[3];
        pos_unpack(a.P[s], ci, f);
        const float v[3] = {w.x, w.y, w.z};
        for (int d = 0; d < 3; d++) {
            Q[3 * (size_t)pid + d] = (double)ci[d] + (double)f[d] * kFxInv;
            V[3 * (size_t)pid + d] = (double)v[d];
        }
    }
}

// Sort key of every slot on the current grid and its rank, for the
// locality re-sort: the cell in the brick order of the single-box resident
// family (res_brick_key) after the box's first key; padding slots take the
// box's last key.
__global__ void __launch_bounds__(256) k_bat_key(const BatchBox *box, const int *chunk_box,
                                                 const BatchStep *st, MixState a, int nslots,
                                                 int *key, int *rank, int *count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nslots;
         i += gridDim.x * blockDim.x) {
        const int b = chunk_box[i / kResChunk];
        const BatchBox &bx = box[b];
        const int N1[3] = {bx.L[0] + 1, bx.L[1] + 1, bx.L[2] + 1};
        int k;
        if (i - bx.part0 < bx.npart) {
            int idx[3];
            fx_cur_idx_periodic<3>(a.P[i], bx.L, st[b].ks, idx);
            k = bx.key0 + res_brick_key(N1, idx);
        } else {
            k = bx.key0 + res_brick_keys(N1);
        }
        key[i] = k;
        rank[i] = atomicAdd(&count[k], 1);
    }
}

// Cell pass of the ensemble: as k_res_cells, one box per block.
__global__ void __launch_bounds__(256) k_bat_cells(const __grid_constant__ DevCfg c,
                                                   const BatchBox *box, const int *cblk_box,
                                                   const BatchStep *st, ResPlanes sums,
                                                   ResRec *crec, double *acc, double *acc_next,
                                                   int nb) {
    __shared__ float4 srec[2 * kCellsPerBlock];
    __shared__ double wsum[8][3];
    const int b = cblk_box[blockIdx.x];
    const BatchBox &bx = box[b];
    const uint32_t step = st[b].step;
    const int c0 = blockIdx.x * kCellsPerBlock;
    double av[3] = {0, 0, 0};
    if (blockIdx.x == 0)
        for (int j = threadIdx.x; j < nb * ACC_WORDS; j += blockDim.x) acc_next[j] = 0.0;
    ResSum s[kResCellsPer];
#pragma unroll
    for (int q = 0; q < kResCellsPer; q++) s[q] = sums.load(c0 + q * 256 + threadIdx.x);
#pragma unroll
    for (int q = 0; q < kResCellsPer; q++) {
        const int cell = c0 + q * 256 + threadIdx.x;
        const int local = cell - bx.cell0;
        sums.clear(cell);
        const int pop = local < bx.ncells ? (int)s[q].n : 0;
        // the record of k_res_cells (one species): u in FP32, the FP32 axis
        float u[3] = {0.f, 0.f, 0.f};
        if (pop > 0) {
            const float ip = __frcp_rn((float)pop);
            for (int d = 0; d < 3; d++) u[d] = (float)((double)s[q].p[d] * kSumFxInv) * ip;
        }
        for (int d = 0; d < 3; d++) av[d] += (double)u[d];
        float Lx[3] = {0.f, 0.f, 1.f};
        if (pop > 1) res_axis3(bx.seed, bx.replica, step, (uint32_t)local, Lx);
        float4 *my = srec + 2 * (q * 256 + threadIdx.x);
        my[0] = make_float4(u[0], u[1], u[2], __int_as_float(pop));
        my[1] = make_float4(Lx[0], Lx[1], Lx[2], 0.f);
    }
    __syncthreads();
    float4 *dst = (float4 *)(crec + c0);
    for (int j = threadIdx.x; j < 2 * kCellsPerBlock; j += 256) dst[j] = srec[j];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int d = 0; d < 3; d++) {
        const double t = warp_sum_d(av[d]);
        if (lane == 0) wsum[wid][d] = t;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += wsum[w][threadIdx.x];
        atomicAdd(&acc[b * ACC_WORDS + ACC_VCM + threadIdx.x], t);
    }
}

// Particle pass of the ensemble: as k_res_parts (one species, periodic),
// one box per block.
template <int MODE>
__global__ void __launch_bounds__(kResThreads, MPCD_RES_MINB) k_bat_parts(
    const __grid_constant__ DevCfg c, const BatchBox *box, const int *chunk_box,
    const BatchStep *st, MixState a, const ResRec *__restrict__ crec, ResPlanes sums,
    double *acc, unsigned long long *status) {
    extern __shared__ __align__(16) unsigned char res_smem[];
    __shared__ double red[8];
    const int tid = threadIdx.x;
    const int b = chunk_box[blockIdx.x];
    const BatchBox &bx = box[b];
    const BatchStep sp = st[b];
    int L[3], mask[3], shift[3];
    for (int d = 0; d < 3; d++) {
        L[d] = bx.L[d];
        mask[d] = bx.res_mask[d];
        shift[d] = bx.res_shift[d];
    }
    const int N1y = L[1] + 1, N1z = L[2] + 1;
    ResTable t;
    t.bind(res_smem, 3);
    {
        uint4 *w = (uint4 *)res_smem;
        const int nkey = kResSlots / 4, nall = res_table_init_bytes(3) / 16;
        for (int j = tid; j < nall; j += kResThreads)
            w[j] = j < nkey ? make_uint4(~0u, ~0u, ~0u, ~0u) : make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    float ke = 0.f;
    int bad = 0;
    const float dtf = (float)c.dt;
    const float cosf_a = (float)c.cosA, sinf_a = (float)c.sinA;
    const int base = blockIdx.x * kResChunk;
    const int end = bx.part0 + bx.npart;
    // the same software pipeline as k_res_parts: next particle loaded at the
    // top of an iteration, its record requested halfway through; the cell a
    // particle was added to at the end of the previous step is in P.w
    // (clamped to its box as a guard)
    const int clast = bx.cell0 + (L[0] + 1) * N1y * N1z - 1;
    auto cur_cell = [&](const MixRec &q) { return (int)min(q.P.w, (unsigned)clast); };
    MixRec nx;
    float4 na = make_float4(0.f, 0.f, 0.f, 0.f), nb = na;
    if (base + tid < end) {
        nx.P = a.P[base + tid];
        nx.W = a.W[base + tid];
        if (MODE == RES_STEP) res_load(crec + cur_cell(nx), na, nb);
    }
#pragma unroll 1
    for (int it = 0; it < MPCD_RES_PPT; it++) {
        const int i = base + it * kResThreads + tid;
        if (i >= end) break;
        MixRec r = nx;
        const float4 ca = na, cb = nb;
        const bool more = it + 1 < MPCD_RES_PPT && i + kResThreads < end;
        if (more) {
            nx.P = a.P[i + kResThreads];
            nx.W = a.W[i + kResThreads];
        }
        int kidx[3];
        if (MODE == RES_STEP) {
            res_apply<3>(r.W, ca, cb, cosf_a, sinf_a);
            ke += r.W.x * r.W.x + r.W.y * r.W.y + r.W.z * r.W.z;
            fx_finish_periodic<3>(r.P, r.W, dtf, L, sp.ksn, kidx);
        } else {
            fx_cur_idx_periodic<3>(r.P, L, sp.ks, kidx);
        }
        const int k = bx.cell0 + (kidx[0] * N1y + kidx[1]) * N1z + kidx[2];
        // the cell of the next step (RES_STEP) or of this one (RES_SUM),
        // read back by cur_cell
        r.P.w = (unsigned)k;
        a.P[i] = r.P;
        if (MODE == RES_STEP) {
            a.W[i] = r.W;
            if (more) res_load(crec + cur_cell(nx), na, nb);
        }
        const float vs[3] = {r.W.x, r.W.y, r.W.z};
        res_add<3>(t, mask, shift, sums, nullptr, k, kidx, vs, 1.0, false, bad);
    }
    __syncthreads();
    res_flush<3>(t, sums, nullptr, false);
    if (MODE == RES_STEP) {
        const double tk = block_sum256(c.mass[0] * (double)ke, red);
        if (tid == 0) atomicAdd(&acc[b * ACC_WORDS + ACC_KE], tk);
    }
    if (bad) atomicAdd(&status[ST_NONFINITE], (unsigned long long)bad);
}

}  // namespace

struct mpcd_batch {
    mpcd_config cfg;
    DevCfg dc;
    int nb = 0;
    std::vector<BatchBox> hbox;
    std::vector<int> hchunk_box, hcblk_box;
    int nslots = 0, ncells = 0, nchunks = 0, ncblk = 0, n = 0, nscan = 0;
    int nkeys = 0;  // sort keys of all boxes (brick order, one padding key each)
    BatchBox *box = nullptr;
    BatchStep *st = nullptr;
    int *chunk_box = nullptr, *cblk_box = nullptr;
    uint32_t *counter = nullptr;
    MixState mx[2] = {};
    int cur = 0;
    int *key = nullptr, *rank = nullptr, *perm = nullptr, *count = nullptr, *start = nullptr,
        *part = nullptr;
    ResSum *rsum = nullptr;
    ResRec *crec = nullptr;
    double *acc = nullptr;  // 2 x nb x ACC_WORDS, by step parity
    unsigned long long *status = nullptr;
    cudaStream_t stream = nullptr;      // where the steps run
    cudaStream_t cap_stream = nullptr;  // private stream the step graphs are captured on
    bool own_stream = true;
    // one captured step per (with re-sort, step parity, current state buffer)
    cudaGraphExec_t graph[2][2][2] = {};
    uint32_t next_step = 0;  // host mirror of the device step counter
    int sort_interval = 20, sort_age = -1;
    bool sums_ready = false;
    void *xfer = nullptr;  // device staging of uploads and downloads
    size_t xfer_bytes = 0;
    int sm_count = 0;
};

namespace {

#define BCK(call)                                                                   \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            fprintf(stderr, "mpcd batch: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return MPCD_ERR_CUDA;                                                   \
        }                                                                           \
    } while (0)

int grid_for(const mpcd_batch *b, int n) {
    int g = (n + 255) / 256;
    const int cap = b->sm_count * 8;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

// Release the device arrays and graphs (the stream stays).
void batch_free(mpcd_batch *b) {
    for (auto &x : b->graph)
        for (auto &y : x)
            for (auto &g : y) {
                if (g) cudaGraphExecDestroy(g);
                g = nullptr;
            }
    for (int k = 0; k < 2; k++) mix_free(b->mx[k]);
    void **ptrs[] = {(void **)&b->box,  (void **)&b->st,    (void **)&b->chunk_box,
                     (void **)&b->cblk_box, (void **)&b->counter, (void **)&b->key,
                     (void **)&b->rank, (void **)&b->perm,  (void **)&b->count,
                     (void **)&b->start, (void **)&b->part, (void **)&b->rsum,
                     (void **)&b->crec, (void **)&b->acc,   (void **)&b->status};
    for (void **p : ptrs) {
        cudaFree(*p);
        *p = nullptr;
    }
    cudaFree(b->xfer);
    b->xfer = nullptr;
    b->xfer_bytes = 0;
}

// Staging buffer of at least 'bytes' (grown, never shrunk).
int batch_xfer_reserve(mpcd_batch *b, size_t bytes) {
    if (bytes <= b->xfer_bytes) return MPCD_OK;
    cudaStreamSynchronize(b->stream);
    cudaFree(b->xfer);
    b->xfer = nullptr;
    b->xfer_bytes = 0;
    if (cudaMalloc(&b->xfer, bytes) != cudaSuccess) return MPCD_ERR_NOMEM;
    b->xfer_bytes = bytes;
    return MPCD_OK;
}

}  // namespace


extern "C" int mpcd_batch_create(const mpcd_config *base, int nboxes, const int *L,
                                 const uint64_t *seeds, mpcd_batch **out) {
    if (!base || !L || !out || nboxes < 1) return MPCD_ERR_ARG;
    *out = nullptr;
    if (base->dim != 3 || base->coll_op != MPCD_COLL_ARBAXIS || base->lc ||
        base->n_species != 1 || base->precision != MPCD_PREC_MIXED)
        return MPCD_ERR_UNSUPPORTED;
    for (int g = 0; g < 3; g++)
        if (base->grav[g] != 0.0) return MPCD_ERR_UNSUPPORTED;
    mpcd_batch *b = new mpcd_batch();
    b->cfg = *base;
    b->nb = nboxes;
    cudaGetDevice(&b->sm_count);
    {
        int dev = b->sm_count;
        cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, dev);
    }
    // geometry of the first box sets dc; per-box geometry lives in the table
    mpcd_config c0 = *base;
    for (int d = 0; d < 3; d++) c0.L[d] = L[d];
    c0.n_walls = 0;
    int r = mpcd_build_devcfg(&c0, &b->dc);
    if (r != MPCD_OK) {
        delete b;
        return r;
    }
    int cell0 = 0, key0 = 0;
    for (int k = 0; k < nboxes; k++) {
        BatchBox bx;
        memset(&bx, 0, sizeof(bx));
        for (int d = 0; d < 3; d++) {
            bx.L[d] = L[3 * k + d];
            if (bx.L[d] < 1 || bx.L[d] > 1023) {
                delete b;
                return MPCD_ERR_ARG;
            }
        }
        mpcd_config ck = c0;
        for (int d = 0; d < 3; d++) ck.L[d] = bx.L[d];
        DevCfg dk;
        if (mpcd_build_devcfg(&ck, &dk) != MPCD_OK) {
            delete b;
            return MPCD_ERR_ARG;
        }
        res_slot_bits(3, bx.L, bx.res_shift, bx.res_mask);
        bx.ncells = (bx.L[0] + 1) * (bx.L[1] + 1) * (bx.L[2] + 1);
        bx.cell0 = cell0;
        bx.key0 = key0;
        key0 += res_brick_keys(dk.N1) + 1;
        const int span = (bx.ncells + 1 + kCellsPerBlock - 1) / kCellsPerBlock;
        for (int j = 0; j < span; j++) b->hcblk_box.push_back(k);
        cell0 += span * kCellsPerBlock;
        bx.seed = seeds ? seeds[k] : base->seed;
        bx.replica = (uint32_t)k;
        b->hbox.push_back(bx);
    }
    b->ncells = cell0;
    b->nkeys = key0;
    b->ncblk = (int)b->hcblk_box.size();
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return MPCD_ERR_CUDA;
    }
    *out = b;
    return MPCD_OK;
}

extern "C" int mpcd_batch_destroy(mpcd_batch *b) {
    if (!b) return MPCD_ERR_ARG;
    cudaStreamSynchronize(b->stream);
    batch_free(b);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    delete b;
    return MPCD_OK;
}

// Upload the particles of all boxes: npart[b] particles per box, Q and V the
// concatenation of the boxes' arrays (3 doubles per particle, box order).
// step0 numbers the first step.
extern "C" int mpcd_batch_upload(mpcd_batch *b, const int *npart, const double *Q,
                                 const double *V, uint32_t step0) {
    if (!b || !npart || !Q || !V) return MPCD_ERR_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    // layout
    int slot0 = 0, n = 0;
    b->hchunk_box.clear();
    for (int k = 0; k < b->nb; k++) {
        if (npart[k] < 0) return MPCD_ERR_ARG;
        BatchBox &bx = b->hbox[k];
        bx.part0 = slot0;
        bx.npart = npart[k];
        bx.nslots = (npart[k] + kResChunk - 1) / kResChunk * kResChunk;
        for (int j = 0; j < bx.nslots / kResChunk; j++) b->hchunk_box.push_back(k);
        slot0 += bx.nslots;
        n += npart[k];
    }
    b->nslots = slot0;
    b->n = n;
    b->nchunks = (int)b->hchunk_box.size();
    b->nscan = (b->nkeys + kScanTile - 1) / kScanTile;
    {
        int g0 = 0;
        for (int k = 0; k < b->nb; k++) {
            b->hbox[k].g0 = g0;
            g0 += b->hbox[k].npart;
        }
    }
    // (re)allocate
    batch_free(b);
    const size_t S = (size_t)slot0 > 0 ? (size_t)slot0 : 1, C = (size_t)b->ncells;
    DevCfg dmix = b->dc;
    dmix.n_species = 1;
    dmix.lc = 0;
    for (int k = 0; k < 2; k++)
        if (mix_alloc(b->mx[k], S, dmix) != MPCD_OK) return MPCD_ERR_NOMEM;
#define BALLOC(p, bytes) \
    if (cudaMalloc((void **)&(p), (bytes)) != cudaSuccess) return MPCD_ERR_NOMEM
    BALLOC(b->box, sizeof(BatchBox) * b->nb);
    BALLOC(b->st, sizeof(BatchStep) * b->nb);
    BALLOC(b->chunk_box, sizeof(int) * (b->nchunks > 0 ? b->nchunks : 1));
    BALLOC(b->cblk_box, sizeof(int) * b->ncblk);
    BALLOC(b->counter, sizeof(uint32_t));
    BALLOC(b->key, sizeof(int) * S);
    BALLOC(b->rank, sizeof(int) * S);
    BALLOC(b->perm, sizeof(int) * S);
    BALLOC(b->count, sizeof(int) * (size_t)b->nkeys);
    BALLOC(b->start, sizeof(int) * ((size_t)b->nkeys + 1));
    BALLOC(b->part, sizeof(int) * b->nscan);
    BALLOC(b->rsum, sizeof(ResSum) * 2 * C);
    BALLOC(b->crec, sizeof(ResRec) * C);
    BALLOC(b->acc, sizeof(double) * 2 * b->nb * ACC_WORDS);
    BALLOC(b->status, sizeof(unsigned long long) * ST_WORDS);
#undef BALLOC
    BCK(cudaMemcpyAsync(b->box, b->hbox.data(), sizeof(BatchBox) * b->nb,
                        cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->chunk_box, b->hchunk_box.data(), sizeof(int) * b->nchunks,
                        cudaMemcpyHostToDevice, b->stream));
    {
        // the caller's arrays through the staging buffer, converted on the
        // device into the slot layout
        const int r = batch_xfer_reserve(b, (size_t)n * 48 + 16);
        if (r != MPCD_OK) return r;
        double *dq = (double *)b->xfer, *dv = dq + 3 * (size_t)n;
        int *derr = (int *)(dv + 3 * (size_t)n);
        if (n > 0) {
            BCK(cudaMemcpyAsync(dq, Q, (size_t)n * 24, cudaMemcpyHostToDevice, b->stream));
            BCK(cudaMemcpyAsync(dv, V, (size_t)n * 24, cudaMemcpyHostToDevice, b->stream));
        }
        BCK(cudaMemsetAsync(derr, 0, sizeof(int), b->stream));
        k_bat_from_f64<<<grid_for(b, slot0), 256, 0, b->stream>>>(b->box, b->chunk_box, b->mx[0],
                                                                  slot0, dq, dv, derr);
        int herr = 0;
        BCK(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        BCK(cudaStreamSynchronize(b->stream));
        if (herr) {
            b->nslots = 0;  // a rejected upload leaves nothing to step
            b->n = 0;
            return MPCD_ERR_ARG;
        }
    }
    BCK(cudaMemcpyAsync(b->cblk_box, b->hcblk_box.data(), sizeof(int) * b->ncblk,
                        cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->counter, &step0, sizeof(uint32_t), cudaMemcpyHostToDevice,
                        b->stream));
    BCK(cudaMemsetAsync(b->count, 0, sizeof(int) * (size_t)b->nkeys, b->stream));
    BCK(cudaMemsetAsync(b->rsum, 0, sizeof(ResSum) * 2 * C, b->stream));
    BCK(cudaMemsetAsync(b->acc, 0, sizeof(double) * 2 * b->nb * ACC_WORDS, b->stream));
    BCK(cudaMemsetAsync(b->status, 0, sizeof(unsigned long long) * ST_WORDS, b->stream));
    b->cur = 0;
    b->next_step = step0;
    b->sort_age = -1;
    b->sums_ready = false;
    BCK(cudaStreamSynchronize(b->stream));
    return MPCD_OK;
}

// Capture one step of the ensemble: the grid shifts, optionally the
// locality re-sort, the cell pass, the particle pass and the step counter.
static int record_step(mpcd_batch *b, bool sorted, int parity, int state_cur,
                       cudaGraphExec_t *out) {
    const size_t nc = (size_t)b->ncells;
    const ResPlanes sum_cur{(long long *)(b->rsum + (size_t)parity * nc), (int)nc};
    const ResPlanes sum_nxt{(long long *)(b->rsum + (size_t)(1 - parity) * nc), (int)nc};
    double *acc_cur = b->acc + (size_t)parity * b->nb * ACC_WORDS;
    double *acc_nxt = b->acc + (size_t)(1 - parity) * b->nb * ACC_WORDS;
    const int pbytes = res_table_bytes(3);
    int cur = state_cur;
    BCK(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    k_bat_shift<<<(b->nb + 127) / 128, 128, 0, b->cap_stream>>>(b->box, b->nb, b->st, b->counter,
                                                             b->dc.galinv);
    if (sorted) {
        k_bat_key<<<grid_for(b, b->nslots), 256, 0, b->cap_stream>>>(
            b->box, b->chunk_box, b->st, b->mx[cur], b->nslots, b->key, b->rank, b->count);
        k_scan_partial<<<b->nscan, 256, 0, b->cap_stream>>>(b->count, b->nkeys, b->part);
        k_scan_apply<<<b->nscan, 256, 0, b->cap_stream>>>(b->count, b->nkeys, b->part, b->start,
                                                      nullptr, nullptr);
        k_perm<<<grid_for(b, b->nslots), 256, 0, b->cap_stream>>>(b->nslots, b->key, b->rank,
                                                               b->start, b->perm);
        k_gather_mix<<<grid_for(b, b->nslots), 256, 0, b->cap_stream>>>(b->mx[cur],
                                                                      b->mx[1 - cur],
                                                                      b->nslots, b->perm);
        cur = 1 - cur;
    }
    k_bat_cells<<<b->ncblk, 256, 0, b->cap_stream>>>(b->dc, b->box, b->cblk_box, b->st, sum_cur,
                                                 b->crec, acc_cur, acc_nxt, b->nb);
    k_bat_parts<RES_STEP><<<b->nchunks, kResThreads, pbytes, b->cap_stream>>>(
        b->dc, b->box, b->chunk_box, b->st, b->mx[cur], b->crec, sum_nxt, acc_cur, b->status);
    k_bat_advance<<<1, 32, 0, b->cap_stream>>>(b->counter);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(b->cap_stream, &g);
    if (ec != cudaSuccess) {
        fprintf(stderr, "mpcd batch: capture failed: %s\n", cudaGetErrorString(ec));
        return MPCD_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return ei == cudaSuccess ? MPCD_OK : MPCD_ERR_CUDA;
}

// nsteps steps of every box; each step is one replay of a captured graph
// (the first step after an upload also forms the initial cell sums).
extern "C" int mpcd_batch_step(mpcd_batch *b, int nsteps) {
    if (!b || nsteps < 0) return MPCD_ERR_ARG;
    if (b->nslots == 0) return MPCD_ERR_STATE;
    const int pbytes = res_table_bytes(3);
    BCK(cudaFuncSetAttribute(k_bat_parts<RES_SUM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             pbytes));
    BCK(cudaFuncSetAttribute(k_bat_parts<RES_STEP>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, pbytes));
    for (int k = 0; k < nsteps; k++) {
        const uint32_t step = b->next_step;
        const int parity = (int)(step & 1u);
        if (!b->sums_ready) {
            k_bat_shift<<<(b->nb + 127) / 128, 128, 0, b->stream>>>(b->box, b->nb, b->st,
                                                                     b->counter, b->dc.galinv);
            BCK(cudaMemsetAsync(b->rsum, 0, sizeof(ResSum) * 2 * b->ncells, b->stream));
            BCK(cudaMemsetAsync(b->acc, 0, sizeof(double) * 2 * b->nb * ACC_WORDS, b->stream));
            k_bat_parts<RES_SUM><<<b->nchunks, kResThreads, pbytes, b->stream>>>(
                b->dc, b->box, b->chunk_box, b->st, b->mx[b->cur], b->crec,
                ResPlanes{(long long *)(b->rsum + (size_t)parity * b->ncells), b->ncells},
                b->acc, b->status);
            BCK(cudaGetLastError());
            b->sums_ready = true;
        }
        const int sorted = (b->sort_age < 0 || b->sort_age >= b->sort_interval) ? 1 : 0;
        cudaGraphExec_t &g = b->graph[sorted][parity][b->cur];
        if (!g) {
            const int r = record_step(b, sorted != 0, parity, b->cur, &g);
            if (r != MPCD_OK) return r;
        }
        BCK(cudaGraphLaunch(g, b->stream));
        if (sorted) {
            b->cur = 1 - b->cur;
            b->sort_age = 0;
        }
        b->sort_age++;
        b->next_step = step + 1u;
    }
    return MPCD_OK;
}

extern "C" int mpcd_batch_set_sort_interval(mpcd_batch *b, int steps) {
    if (!b || steps < 1) return MPCD_ERR_ARG;
    b->sort_interval = steps;
    return MPCD_OK;
}

// Particles of all boxes back, in the upload's order (concatenated boxes).
extern "C" int mpcd_batch_download(mpcd_batch *b, double *Q, double *V) {
    if (!b || !Q || !V) return MPCD_ERR_ARG;
    const size_t n = (size_t)b->n;
    const int r = batch_xfer_reserve(b, n * 48 + 16);
    if (r != MPCD_OK) return r;
    double *dq = (double *)b->xfer, *dv = dq + 3 * n;
    int *derr = (int *)(dv + 3 * n);
    BCK(cudaMemsetAsync(derr, 0, sizeof(int), b->stream));
    k_bat_to_f64<<<grid_for(b, b->nslots), 256, 0, b->stream>>>(b->mx[b->cur], b->nslots, b->n,
                                                                dq, dv, derr);
    int herr = 0;
    BCK(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    if (n > 0) {
        BCK(cudaMemcpyAsync(Q, dq, n * 24, cudaMemcpyDeviceToHost, b->stream));
        BCK(cudaMemcpyAsync(V, dv, n * 24, cudaMemcpyDeviceToHost, b->stream));
    }
    BCK(cudaStreamSynchronize(b->stream));
    return herr ? MPCD_ERR_STATE : MPCD_OK;
}

// Per-box global measures of the last step: kbt[b] = TEMP, avv[3b..3b+2] =
// avVel (therm.c:209-235, 362-367) of box b.
extern "C" int mpcd_batch_globals(mpcd_batch *b, double *kbt, double *avv) {
    if (!b) return MPCD_ERR_ARG;
    if (!b->sums_ready) return MPCD_ERR_STATE;
    const uint32_t last = b->next_step - 1u;
    std::vector<double> a((size_t)b->nb * ACC_WORDS);
    BCK(cudaStreamSynchronize(b->stream));
    BCK(cudaMemcpy(a.data(), b->acc + (size_t)(last & 1u) * b->nb * ACC_WORDS,
                   sizeof(double) * a.size(), cudaMemcpyDeviceToHost));
    for (int k = 0; k < b->nb; k++) {
        const BatchBox &bx = b->hbox[k];
        const double vol = (double)bx.L[0] * bx.L[1] * bx.L[2];
        if (kbt) kbt[k] = bx.npart > 0 ? a[(size_t)k * ACC_WORDS + ACC_KE] / (3.0 * bx.npart) : 0.0;
        if (avv)
            for (int d = 0; d < 3; d++) avv[3 * k + d] = a[(size_t)k * ACC_WORDS + ACC_VCM + d] / vol;
    }
    return MPCD_OK;
}

// Total particles, slots (with padding) and cells (with padding) of the
// ensemble, for sizing host buffers and reporting.
extern "C" int mpcd_batch_info(mpcd_batch *b, int *n, int *slots, int *cells) {
    if (!b) return MPCD_ERR_ARG;
    if (n) *n = b->n;
    if (slots) *slots = b->nslots;
    if (cells) *cells = b->ncells;
    return MPCD_OK;
}

// Run the steps on the caller's CUDA stream from now on (the graphs are
// captured on a private stream and launched on this one; any stream works,
// the legacy default stream included).
extern "C" int mpcd_batch_set_stream(mpcd_batch *b, void *stream) {
    if (!b) return MPCD_ERR_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    for (auto &x : b->graph)
        for (auto &y : x)
            for (auto &g : y) {
                if (g) cudaGraphExecDestroy(g);
                g = nullptr;
            }
    if (b->own_stream) cudaStreamDestroy(b->stream);
    b->stream = (cudaStream_t)stream;
    b->own_stream = false;
    return MPCD_OK;
}
