// Process-wide helpers of the field engine library.
#include "common.cuh"

int fb_sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0)
            sms = n;
        else
            sms = 148;
    }
    return sms;
}

extern "C" {

// ABI version of this library; bumped when an exported signature changes.
int fb_abi_version() { return 1; }

// Compute capability of the current device times ten (100 on B200), or -1 without a device.
int fb_device_arch() {
    int dev = 0, major = 0, minor = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess) return -1;
    return major * 10 + minor;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// float32 FMA throughput probe: the denominator of the float32-pipe roofline (the driver's
// measured peaks cover HBM and bf16 tensor throughput only).  8 independent FMA chains per
// thread, `iters` steps each; 16 flops per thread per step.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fp32_peak(float* out, int iters, float seed) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float b = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
            a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
        }
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

extern "C" {

// Enqueue the probe; returns the flop count it performs (or -1).  `d_out` needs gridDim floats.
int64_t fb_fp32_peak_launch(float* d_out, int blocks, int iters, void* stream) {
    if (!d_out || blocks < 1 || iters < 1) return -1;
    k_fp32_peak<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_out, iters, 1.0f);
    if (cudaGetLastError() != cudaSuccess) return -1;
    return (int64_t)blocks * 256 * (int64_t)iters * 8 * 8 * 2;
}

int fb_sm_count_c() { return fb_sm_count(); }

}  // extern "C"

extern "C" {

// Stream-ordered copy between raw addresses, device or host (unified addressing picks the
// direction), e.g. out of a build's scratch; synchronises the stream.
int fb_copy_device(void* dst, const void* src, int64_t bytes, void* stream) {
    if (!dst || !src || bytes < 0) return 1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st) != cudaSuccess) return 2;
    return cudaStreamSynchronize(st) == cudaSuccess ? 0 : 2;
}

}  // extern "C"
