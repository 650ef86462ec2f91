// Block classification of a dense float32 SDF by its 8 corner samples -- the reference's rule
// (k_classify_dense, src/field_engine/faltkarna_v1_mesh_to_sdf.py:602-632; meshsdf_classify_cpu,
// mesh_sdf_native_v1/field.cpp:229-252): corners at the block's origin and origin + B per axis,
// clamped to the grid; kind 0 when the corner signs differ or min |v| <= margin, else -1 / +1 by
// sign.  Shared by the full-grid classification and the adaptive tree's per-node codes, so both
// decide every block the same way.
#pragma once
#include <cstdint>

// kind (-1 / 0 / +1) of the side-B block whose origin is voxel (x0, y0, z0); *mn = min |corner|.
__device__ __forceinline__ int dense_block_kind(const float* __restrict__ dense, int64_t nx, int64_t ny, int64_t nz,
                                                int B, int64_t x0, int64_t y0, int64_t z0, float margin, float* mn) {
    float m = 1.0e30f;
    bool pos = false, neg = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int64_t cx = min(x0 + (c & 1) * B, nx - 1);
        const int64_t cy = min(y0 + ((c >> 1) & 1) * B, ny - 1);
        const int64_t cz = min(z0 + ((c >> 2) & 1) * B, nz - 1);
        const float v = dense[(cx * ny + cy) * nz + cz];
        m = fminf(m, fabsf(v));
        if (v >= 0.0f) pos = true; else neg = true;
    }
    *mn = m;
    return (pos && neg) ? 0 : ((m <= margin) ? 0 : (neg ? -1 : 1));
}
