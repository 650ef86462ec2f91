// Exclusive scan of int32 arrays on the device, shared by the sources that compact or rank (each
// includes its own copy: everything here has internal linkage).
#pragma once
#include "common.cuh"
#include <algorithm>

namespace {

// Exclusive scan of int32 in place: tiles of 4096 (1024 threads x 4) scanned in shared memory,
// tile sums scanned recursively, added back.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int64_t kScanTile = (int64_t)kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) k_scan_tile(int32_t* __restrict__ data, int64_t n,
                                                            int32_t* __restrict__ sums) {
    __shared__ int32_t s_warp[kScanThreads / 32];
    const int64_t base = blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    int32_t t = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? data[base + k] : 0;
        t += v[k];
    }
    // warp inclusive scan of the thread totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t inc = t;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;  // inclusive per warp
    }
    __syncthreads();
    int32_t run = (warp ? s_warp[warp - 1] : 0) + inc - t;  // exclusive start of this thread
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) data[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = run;
}

__global__ void k_scan_add(int32_t* __restrict__ data, int64_t n, const int32_t* __restrict__ offsets) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) data[i] += offsets[i / kScanTile];
}

// Scratch int32 words the scan of n elements needs: the tile sums of every recursion level, down to
// the level of one tile, plus one.
int64_t scan_scratch_words(int64_t n) {
    int64_t words = 1, tiles;
    do {
        tiles = (std::max<int64_t>(n, 1) + kScanTile - 1) / kScanTile;
        words += tiles;
        n = tiles;
    } while (tiles > 1);
    return words;
}

// Exclusive scan of data[0, n); the total is written to *total (device).
int scan_exclusive(int32_t* data, int64_t n, int32_t* total, int32_t* scratch, int64_t scratch_words,
                   cudaStream_t st) {
    if (n <= 0) {
        FB_CUDA(cudaMemsetAsync(total, 0, sizeof(int32_t), st));
        return FB_OK;
    }
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (scratch_words < tiles + 1) return FB_INVALID;
    int32_t* sums = scratch;
    k_scan_tile<<<(unsigned)tiles, kScanThreads, 0, st>>>(data, n, sums);
    FB_LAUNCH();
    if (tiles == 1) {
        FB_CUDA(cudaMemcpyAsync(total, sums, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
        return FB_OK;
    }
    if (int rc = scan_exclusive(sums, tiles, total, scratch + tiles, scratch_words - tiles, st)) return rc;
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(data, n, sums);
    FB_LAUNCH();
    return FB_OK;
}

}  // namespace
