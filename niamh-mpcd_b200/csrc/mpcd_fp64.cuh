// mpcd_fp64.cuh -- state of the plain-FP64 form and the counting-sort scan.
//
// FP64 state: structure-of-arrays doubles (q[3], v[3]) holding the
// reference's unshifted positions, plus the particle's original index (pid:
// keys every per-particle draw and the download order) and its species.
//
//   k_scan_partial / k_scan_apply: exclusive scan of the per-cell counts
//   into the cell start offsets of the sorted order.
#pragma once

#include <cuda/atomic>

#include "mpcd_device.cuh"

namespace mpcd {

struct Fp64State {
    double *q[3];
    double *v[3];
    int *pid;
    int *sp;      // species (nullptr when there is one species)
    double *u[2]; // nematic orientation (2D; nullptr when isotropic)
};

constexpr int kScanTile = 2048;  // cells per scan block (256 threads x 8)

// Block-wide exclusive scan of one int per thread (256 threads).
__device__ __forceinline__ int block_excl_scan256(int x, int &total) {
    __shared__ int warp_tot[8];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    int wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        int t = warp_tot[w];
        if (w < wid) wpre += t;
        tot += t;
    }
    __syncthreads();
    total = tot;
    return wpre + incl - x;
}

// Sum of each tile of counts.
static __global__ void __launch_bounds__(256) k_scan_partial(const int *count, int ncells,
                                                      int *part) {
    int base = blockIdx.x * kScanTile;
    int local = 0;
    for (int j = threadIdx.x; j < kScanTile; j += 256) {
        int idx = base + j;
        if (idx < ncells) local += count[idx];
    }
    int tot;
    block_excl_scan256(local, tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// Exclusive scan of the counts into start[0..ncells]; zeroes the counts
// (and the fill cursors, if given) for reuse, and the accumulators of the
// step that will use these starts.
static __global__ void __launch_bounds__(256) k_scan_apply(int *count, int ncells,
                                                    const int *part, int *start,
                                                    int *fill, double *acc) {
    // offset of this block: sum of the partial sums of the blocks before it,
    // loaded and reduced by all threads
    int mine = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += 256) mine += part[b];
    int s_off;
    block_excl_scan256(mine, s_off);
    if (acc && blockIdx.x == 0 && threadIdx.x < ACC_WORDS) acc[threadIdx.x] = 0.0;
    int base = blockIdx.x * kScanTile + threadIdx.x * 8;
    int v[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        int idx = base + j;
        v[j] = idx < ncells ? count[idx] : 0;
        sum += v[j];
    }
    int tot;
    int pre = block_excl_scan256(sum, tot) + s_off;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        int idx = base + j;
        if (idx < ncells) {
            start[idx] = pre;
            count[idx] = 0;
            if (fill) fill[idx] = 0;
        }
        pre += v[j];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 255) start[ncells] = pre;
}

// Single-pass exclusive scan of the counts (decoupled look-back).  Each block
// takes the next tile from a 64-bit ticket counter that is never reset: the
// ticket gives the tile (ticket mod tiles) and the launch's epoch (ticket div
// tiles), so the kernel needs no host-side state and replays unchanged inside
// a CUDA graph.  Tickets are handed out in the order blocks start, so every
// tile's predecessors are already running.  A tile publishes its sum, walks
// back over its predecessors' published words adding sums until it meets a
// published inclusive prefix, publishes its own inclusive prefix and writes
// its starts.  Word layout: bits 62-63 flag (1 sum, 2 prefix), 32-61 epoch,
// 0-31 value.  Every wait is bounded: after kScanSpin polls the block records
// the timeout in status[status_word] and carries on (the starts are then
// wrong and the step is reported failed).
constexpr unsigned long long kScanFlagA = 1ull << 62, kScanFlagP = 2ull << 62;
constexpr int kScanSpin = 1 << 22;

static __global__ void __launch_bounds__(256) k_scan_lookback(
    int *count, int ncells, int *start, int *fill, double *acc, unsigned long long *tstat,
    unsigned long long *ticket, unsigned long long *status, int status_word) {
    __shared__ int s_tile, s_off;
    __shared__ unsigned long long s_ep;
    const unsigned ntiles = gridDim.x;
    if (threadIdx.x == 0) {
        const unsigned long long t = atomicAdd(ticket, 1ull);
        s_tile = (int)(t % ntiles);
        s_ep = ((t / ntiles) & 0x3FFFFFFFull) << 32;
    }
    __syncthreads();
    const int tile = s_tile;
    const int base = tile * kScanTile + threadIdx.x * 8;
    int v[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int idx = base + j;
        v[j] = idx < ncells ? count[idx] : 0;
        sum += v[j];
    }
    int agg;
    int pre = block_excl_scan256(sum, agg);
    if (threadIdx.x == 0) {
        const unsigned long long ep = s_ep;
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> me(tstat[tile]);
        int prefix = 0;
        if (tile == 0) {
            me.store(kScanFlagP | ep | (unsigned)agg, cuda::memory_order_release);
        } else {
            me.store(kScanFlagA | ep | (unsigned)agg, cuda::memory_order_release);
            bool timed_out = false;
            for (int t = tile - 1; t >= 0; t--) {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> w(tstat[t]);
                unsigned long long x = w.load(cuda::memory_order_acquire);
                int spins = 0;
                while ((x & 0x3FFFFFFF00000000ull) != ep || (x >> 62) == 0) {
                    if (++spins > kScanSpin) {
                        timed_out = true;
                        break;
                    }
                    __nanosleep(32);
                    x = w.load(cuda::memory_order_acquire);
                }
                if (timed_out) break;
                prefix += (int)(unsigned)(x & 0xFFFFFFFFull);
                if ((x >> 62) == 2) break;
            }
            if (timed_out) atomicAdd(&status[status_word], 1ull);
            me.store(kScanFlagP | ep | (unsigned)(prefix + agg), cuda::memory_order_release);
        }
        s_off = prefix;
        if (acc && tile == 0)
            for (int k = 0; k < ACC_WORDS; k++) acc[k] = 0.0;
        if (tile == (int)ntiles - 1) start[ncells] = prefix + agg;
    }
    __syncthreads();
    pre += s_off;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int idx = base + j;
        if (idx < ncells) {
            start[idx] = pre;
            count[idx] = 0;
            if (fill) fill[idx] = 0;
        }
        pre += v[j];
    }
}

}  // namespace mpcd
