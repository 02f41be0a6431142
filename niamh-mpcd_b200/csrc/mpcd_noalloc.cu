// mpcd_noalloc.cu -- one SRD solvent timestep that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they want to
// step the fluid: a host program whose allocator already owns every byte of
// the GPU and hands out none at run time; code running while a CUDA stream
// is being captured into a graph, where cudaMalloc is not allowed; or a
// plugin inside another framework that must not create allocations of its
// own behind that framework's memory manager.  mpcd_srd_step_noalloc serves
// them: the caller passes its own device arrays of positions and velocities,
// and all scratch the step needs (the counting-sort buffers, cell counts and
// offsets, per-cell records, accumulators) lives in one file-scope device
// array of fixed size, g_scratch below.  The array exists on every GPU that
// loads this part of the library and stays there until the process exits.
//
// Shared state: every call, on every stream, uses the same g_scratch of its
// device, and the array keeps what the last call left in it.  Each call
// clears what must start at zero itself; two calls whose GPU work overlaps
// (different streams, or host threads) race on the array and corrupt each
// other's results, so a caller must serialise them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "mpcd_gpu.h"
#include "mpcd_device.cuh"
#include "mpcd_fp64.cuh"
#include "mpcd_mixed.cuh"
#include "mpcd_tile.cuh"
#include "mpcd_split.cuh"

using namespace mpcd;

int mpcd_build_devcfg(const mpcd_config *cfg, DevCfg *dc);

namespace {

// Capacity of the scratch array, in particles and cells (cells count the
// (L+1)^D grid).  At these maxima the array holds 11.6 MiB.
constexpr int kMaxParticles = MPCD_NOALLOC_MAX_PARTICLES;
constexpr int kMaxCells = MPCD_NOALLOC_MAX_CELLS;
constexpr int kMaxScan = (kMaxCells + kScanTile - 1) / kScanTile;

// byte layout of the scratch array
constexpr size_t kAlign = 256;
constexpr size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kPartF64 = up((size_t)kMaxParticles * sizeof(double));
constexpr size_t kPartI32 = up((size_t)kMaxParticles * sizeof(int));
constexpr size_t kCellI32 = up((size_t)(kMaxCells + 1) * sizeof(int));
constexpr size_t kOffBufA = 0;                               // 6 doubles + pid
constexpr size_t kOffBufB = kOffBufA + 6 * kPartF64 + kPartI32;  // same
constexpr size_t kOffKey = kOffBufB + 6 * kPartF64 + kPartI32;
constexpr size_t kOffRank = kOffKey + kPartI32;
constexpr size_t kOffCount = kOffRank + kPartI32;
constexpr size_t kOffFill = kOffCount + kCellI32;
constexpr size_t kOffStartA = kOffFill + kCellI32;
constexpr size_t kOffStartB = kOffStartA + kCellI32;
constexpr size_t kOffPart = kOffStartB + kCellI32;
constexpr size_t kOffCrec = kOffPart + up((size_t)kMaxScan * sizeof(int));
constexpr size_t kOffAcc = kOffCrec + up((size_t)kMaxCells * sizeof(SrdCell<F64T<3>>::Rec));
constexpr size_t kOffStatus = kOffAcc + up(ACC_WORDS * sizeof(double));
constexpr size_t kScratchBytes = kOffStatus + up(ST_WORDS * sizeof(unsigned long long));

}  // namespace

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

namespace {

// Device address of g_scratch, looked up once per CUDA context (the
// host-side symbol is only a stand-in, not a device address).  The cache is
// keyed by the context's unique id, so a device reset (which destroys the
// primary context; the module can then load at another address) makes the
// next call look the address up again.
struct ScratchSlot {
    unsigned long long ctx_id;
    unsigned char *ptr;
};
constexpr int kMaxContexts = 64;
ScratchSlot g_slots[kMaxContexts];
int g_nslots = 0;
std::mutex g_slots_mu;

// Unique id of the current CUDA context, through the driver's
// cuCtxGetCurrent and cuCtxGetId, fetched from the runtime so that the
// library does not link the driver library itself.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
int current_context_id(unsigned long long *id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)p;
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)p;
    });
    if (!get_current || !get_id) return MPCD_ERR_CUDA;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS)
        return MPCD_ERR_CUDA;
    return MPCD_OK;
}

int scratch_address(unsigned char **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MPCD_ERR_CUDA;
    // make the device's primary context current (it allocates nothing)
    if (cudaSetDevice(dev) != cudaSuccess) return MPCD_ERR_CUDA;
    unsigned long long id = 0;
    if (current_context_id(&id) != MPCD_OK) return MPCD_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_slots_mu);
    for (int i = 0; i < g_nslots; i++)
        if (g_slots[i].ctx_id == id) {
            *out = g_slots[i].ptr;
            return MPCD_OK;
        }
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return MPCD_ERR_CUDA;
    // a full table drops its oldest entry (a process that has reset its
    // devices more than kMaxContexts times)
    if (g_nslots == kMaxContexts) {
        for (int i = 1; i < kMaxContexts; i++) g_slots[i - 1] = g_slots[i];
        g_nslots--;
    }
    g_slots[g_nslots++] = ScratchSlot{id, (unsigned char *)p};
    *out = (unsigned char *)p;
    return MPCD_OK;
}

// AoS caller arrays -> structure-of-arrays buffer (pid = caller index)
template <int DIM>
__global__ void __launch_bounds__(256) k_na_load(const double *Q, const double *V, int n,
                                                 Fp64State a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int d = 0; d < DIM; d++) {
            a.q[d][i] = Q[3 * (size_t)i + d];
            a.v[d][i] = V[3 * (size_t)i + d];
        }
        a.pid[i] = i;
    }
}

// sorted buffer -> caller arrays, back in the caller's order
template <int DIM>
__global__ void __launch_bounds__(256) k_na_store(Fp64State b, int n, double *Q, double *V) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t p = (size_t)b.pid[i];
        for (int d = 0; d < DIM; d++) {
            Q[3 * p + d] = b.q[d][i];
            V[3 * p + d] = b.v[d][i];
        }
    }
}

// The step's global measures (KBTNOW, AVNOW) into the caller's globals,
// and its error counters added to the caller's counters (either may be
// null).
__global__ void k_na_finish(const double *acc, const unsigned long long *status, int n,
                            int dim, double vol, double *out, unsigned long long *counters) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        if (out) {
            out[0] = n > 0 ? acc[ACC_KE] / (double)(n * dim) : 0.0;
            for (int d = 0; d < 3; d++) out[1 + d] = d < dim ? acc[ACC_VCM + d] / vol : 0.0;
        }
        if (counters) {
            counters[0] += status[ST_ESCAPED];
            counters[1] += status[ST_BOUNCE];
            counters[2] += status[ST_NONFINITE];
        }
    }
}

template <int DIM>
int noalloc_step(const DevCfg &c, int n, double *Q, double *V, uint32_t step, double *globals,
                 unsigned long long *counters, cudaStream_t s, unsigned char *base) {
    Fp64State A, B;
    memset(&A, 0, sizeof(A));
    memset(&B, 0, sizeof(B));
    for (int d = 0; d < 3; d++) {
        A.q[d] = (double *)(base + kOffBufA + (size_t)d * kPartF64);
        A.v[d] = (double *)(base + kOffBufA + (size_t)(3 + d) * kPartF64);
        B.q[d] = (double *)(base + kOffBufB + (size_t)d * kPartF64);
        B.v[d] = (double *)(base + kOffBufB + (size_t)(3 + d) * kPartF64);
    }
    A.pid = (int *)(base + kOffBufA + 6 * kPartF64);
    B.pid = (int *)(base + kOffBufB + 6 * kPartF64);
    int *key = (int *)(base + kOffKey);
    int *rank = (int *)(base + kOffRank);
    int *count = (int *)(base + kOffCount);
    int *fill = (int *)(base + kOffFill);
    int *startA = (int *)(base + kOffStartA);
    int *startB = (int *)(base + kOffStartB);
    int *part = (int *)(base + kOffPart);
    auto *crec = (typename SrdCell<F64T<DIM>>::Rec *)(base + kOffCrec);
    double *acc = (double *)(base + kOffAcc);
    unsigned long long *status = (unsigned long long *)(base + kOffStatus);
    const int nc = c.ncells, nscan = (nc + kScanTile - 1) / kScanTile;
    // what the step needs at zero: counts, fill cursors, accumulators
    if (cudaMemsetAsync(count, 0, (size_t)nc * sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(fill, 0, (size_t)nc * sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(acc, 0, ACC_WORDS * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(status, 0, ST_WORDS * sizeof(unsigned long long), s) != cudaSuccess)
        return MPCD_ERR_CUDA;
    StepArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.step = step;
    if (c.galinv) {
        mpcd_rng_shift(c.seed, c.replica, step, DIM, sa.s);
        mpcd_rng_shift(c.seed, c.replica, step + 1u, DIM, sa.sn);
    }
    for (int d = 0; d < 3; d++) {
        sa.ks[d] = (uint32_t)(sa.s[d] * 4294967296.0);
        sa.ksn[d] = (uint32_t)(sa.sn[d] * 4294967296.0);
    }
    const int gp = (n + 255) / 256;
    // caller order -> sorted by cell of this step's shifted grid
    k_na_load<DIM><<<gp, 256, 0, s>>>(Q, V, n, A);
    k_key_f64<DIM><<<gp, 256, 0, s>>>(c, A, n, key, rank, count, sa, status);
    k_scan_partial<<<nscan, 256, 0, s>>>(count, nc, part);
    k_scan_apply<<<nscan, 256, 0, s>>>(count, nc, part, startA, nullptr, nullptr);
    k_scatter_f64v<DIM><<<gp, 256, 0, s>>>(A, B, n, key, rank, startA);
    // the step: cell records, next-cell histogram, scan, final write-out
    TileBufs tb;
    memset(&tb, 0, sizeof(tb));
    tb.start = startA;
    tb.start_next = startB;
    tb.count_next = count;
    tb.fill = fill;
    tb.key = key;
    tb.rank = rank;
    tb.acc = acc;
    tb.status = status;
    k_srd_cells<DIM, F64T<DIM>><<<(nc + 255) / 256, 256, 0, s>>>(c, B, startA, crec, sa, acc);
    k_srd_parts<DIM, F64T<DIM>, MODE_COUNT><<<gp, 256, 0, s>>>(c, B, A, n, crec, tb, sa);
    k_scan_partial<<<nscan, 256, 0, s>>>(count, nc, part);
    k_scan_apply<<<nscan, 256, 0, s>>>(count, nc, part, startB, fill, nullptr);
    k_srd_parts<DIM, F64T<DIM>, MODE_FINAL><<<gp, 256, 0, s>>>(c, B, A, n, crec, tb, sa);
    k_na_store<DIM><<<gp, 256, 0, s>>>(A, n, Q, V);
    if (globals || counters)
        k_na_finish<<<1, 32, 0, s>>>(acc, status, n, DIM, c.vol, globals, counters);
    return cudaGetLastError() == cudaSuccess ? MPCD_OK : MPCD_ERR_CUDA;
}

}  // namespace

extern "C" int mpcd_srd_step_noalloc(const mpcd_config *cfg, int n, double *Q, double *V,
                                     uint32_t step, double *globals,
                                     unsigned long long *counters, void *stream) {
    if (!cfg || n < 0 || (n > 0 && (!Q || !V))) return MPCD_ERR_ARG;
    DevCfg c;
    int r = mpcd_build_devcfg(cfg, &c);
    if (r != MPCD_OK) return r;
    // the SRD operator, FP64 state, one species (the caller passes no
    // species ids), no phantom walls, no nematic order
    if (c.op != MPCD_COLL_ARBAXIS || c.any_phantom || c.lc || c.n_species != 1 ||
        cfg->precision != MPCD_PREC_FP64)
        return MPCD_ERR_UNSUPPORTED;
    if (n > kMaxParticles || c.ncells > kMaxCells) return MPCD_ERR_SIZE;
    if (!(cfg->gndnst > 0.0)) c.gndnst = 0.0;  // phantom-free: GnDNST unused
    unsigned char *base = nullptr;
    r = scratch_address(&base);
    if (r != MPCD_OK) return r;
    if (n == 0) return MPCD_OK;
    cudaStream_t s = (cudaStream_t)stream;
    return c.dim == 3 ? noalloc_step<3>(c, n, Q, V, step, globals, counters, s, base)
                      : noalloc_step<2>(c, n, Q, V, step, globals, counters, s, base);
}
