// Shared helpers for the field engine's CUDA sources (sm_100a only).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

// Status codes of every C-ABI entry point.  0/1/2 follow the reference's native contract
// (src/field_engine/edt_native_v1/edt.cu:18-19: 0 success, 1 invalid input, 2 runtime failure);
// the CSG entry points add the reference's codes 3-5 (csg_batch_native_v1/execute.cpp).
enum {
    FB_OK = 0,
    FB_INVALID = 1,
    FB_RUNTIME = 2,
    FB_TIMEOUT = 6,   // a bounded device-side wait gave up; the context stays usable
    FB_NOALLOC_LIMIT = 7,  // the grid exceeds the fixed scratch of an allocation-free entry point
    FB_CAPACITY = 8,  // an output arena was too small for the result (what fitted is written)
};

#define FB_CUDA(call)                                    \
    do {                                                 \
        if ((call) != cudaSuccess) return FB_RUNTIME;    \
    } while (0)

#define FB_LAUNCH()                                      \
    do {                                                 \
        if (cudaGetLastError() != cudaSuccess) return FB_RUNTIME; \
    } while (0)

static inline int fb_div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Superblock edge in voxels, the middle level of the culling hierarchy (coarse regions are two
// superblocks wide, blocks below): 32, or 16 for grids of at most 128 voxels per axis -- there a
// 32-voxel superblock spans a quarter of the grid and culls little of a dense recipe.
__host__ __device__ inline int fb_super_edge(int64_t nx, int64_t ny, int64_t nz) {
    const int64_t m = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
    return m <= 128 ? 16 : 32;
}

// Number of SMs of the current device (148 on B200), cached per process.
int fb_sm_count();
