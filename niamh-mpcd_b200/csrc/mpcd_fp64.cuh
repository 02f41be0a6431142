// mpcd_fp64.cuh -- state of the plain-FP64 form and the counting-sort scan.
//
// FP64 state: structure-of-arrays doubles (q[3], v[3]) holding the
// reference's unshifted positions, plus the particle's original index (pid:
// keys every per-particle draw and the download order) and its species.
//
//   k_scan_partial / k_scan_apply: exclusive scan of the per-cell counts
//   into the cell start offsets of the sorted order.
#pragma once

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

}  // namespace mpcd
