// Test infrastructure only: drives the reference's own CUDA EDT kernels on device buffers, so that
// they can be checked and timed beside field_b200 at sizes above the 2^20-voxel cap of the
// reference's host entry points.  The kernels come unmodified from the reference source named by
// REF_EDT_SOURCE (compiled in by oracle/Makefile); only the launch sequence lives here, and it
// follows the reference's host code step for step:
//   single polarity (REF_EDT_SOURCE = src/field_engine/edt_native_linear_v1/edt.cu):
//     init int32 = mask ? sentinel : 0 (edt.cu:44-45, done on the host there, by ref_init here),
//     then axis_envelope over x, y, z (edt.cu:49-53);
//   paired (REF_EDT_PAIRED, REF_EDT_SOURCE = src/field_engine/edt_persistent_pair_v1/edt.cu):
//     initialise, axis_envelope over x, y, z for both polarities, signed_output (edt.cu:66-73).
// Both kernels index with int: size * 2 must stay below 2^31 (512^3 does).
#ifndef REF_EDT_SOURCE
#error "REF_EDT_SOURCE must name the reference's edt.cu"
#endif
#include REF_EDT_SOURCE

#include <utility>

namespace {

int sentinel_of(int nx, int ny, int nz) { return (nx - 1) * (nx - 1) + (ny - 1) * (ny - 1) + (nz - 1) * (nz - 1) + 1; }

bool shape_ok(int nx, int ny, int nz) {
    return nx >= 1 && ny >= 1 && nz >= 1 && nx <= 512 && ny <= 512 && nz <= 512;
}

}  // namespace

#ifndef REF_EDT_PAIRED

__global__ void ref_init(const uint8_t* mask, int* out, int size, int sentinel) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < size) out[i] = mask[i] ? sentinel : 0;
}

// Squared distance of every voxel to the nearest zero voxel (the reference's edt_squared_large),
// on device buffers: d_mask (size bytes), a and b (size int32 each).  The result ends in *result
// (a or b).  Returns 0, or 1 for a bad shape, 2 for a launch failure.
extern "C" int ref_edt_linear_device(const uint8_t* d_mask, int nx, int ny, int nz, int* a, int* b, int** result,
                                     void* stream) {
    if (!d_mask || !a || !b || !result || !shape_ok(nx, ny, nz)) return 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int size = nx * ny * nz;
    ref_init<<<(size + 255) / 256, 256, 0, s>>>(d_mask, a, size, sentinel_of(nx, ny, nz));
    if (cudaGetLastError() != cudaSuccess) return 2;
    const int lengths[] = {nx, ny, nz}, strides[] = {ny * nz, nz, 1};
    for (int axis = 0; axis < 3; ++axis) {
        axis_envelope<<<(size / lengths[axis] + 127) / 128, 128, 0, s>>>(a, b, size, strides[axis], lengths[axis]);
        if (cudaGetLastError() != cudaSuccess) return 2;
        std::swap(a, b);
    }
    *result = a;
    return 0;
}

#else

// Signed distance and the squared pair (polarity 0: to the nonzero voxels) as the reference's
// edt_pair_query computes them, on device buffers: d_mask (size bytes), a and b (2 * size int32
// each), distance (size float32).  The squared pair ends in *result (a or b).
extern "C" int ref_edt_pair_device(const uint8_t* d_mask, int nx, int ny, int nz, double pitch, int* a, int* b,
                                   float* distance, int** result, void* stream) {
    if (!d_mask || !a || !b || !distance || !result || !shape_ok(nx, ny, nz)) return 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int size = nx * ny * nz;
    initialise<<<(size + 255) / 256, 256, 0, s>>>(d_mask, a, size, sentinel_of(nx, ny, nz));
    if (cudaGetLastError() != cudaSuccess) return 2;
    const int lengths[] = {nx, ny, nz}, strides[] = {ny * nz, nz, 1};
    for (int axis = 0; axis < 3; ++axis) {
        axis_envelope<<<(2 * size / lengths[axis] + 127) / 128, 128, 0, s>>>(a, b, size, strides[axis], lengths[axis]);
        if (cudaGetLastError() != cudaSuccess) return 2;
        std::swap(a, b);
    }
    signed_output<<<(size + 255) / 256, 256, 0, s>>>(a, distance, size, pitch);
    if (cudaGetLastError() != cudaSuccess) return 2;
    *result = a;
    return 0;
}

#endif
