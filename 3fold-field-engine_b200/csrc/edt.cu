// Exact integer squared Euclidean distance transform and the paired signed distance, sm_100a.
//
// Algorithm (a from-scratch design, not the reference's one-thread-per-line envelope):
//   1. k_edt_bits  : the uint8 mask becomes one 32-bit word per 32 z-samples of every (x, y) line
//                    (1 B read + 1/8 B written per voxel); the same pass validates the mask
//                    (values 0/1, both classes present) with warp-aggregated counters.
//   2. k_edt_zy    : one CTA per (32-wide z chunk, x plane, polarity).  For every y line it finds
//                    the nearest site along z from the line's bit words (clz/ffs over the chunk's
//                    own word, a ballot over the other words), stages dz^2 for the chunk in shared
//                    memory, then runs the y pass there: g(y,z) = min_y' dz(y',z)^2 + (y-y')^2 by a
//                    window search that stops once t^2 >= best.  Writes int32 g (4 B/voxel).
//   3. k_edt_x     : one CTA per (z chunk, y row, polarity): stages the nx x 32 column block of g
//                    in shared memory with coalesced 128 B rows, runs the same window search along
//                    x and writes the final int32 (4 B/voxel) -- or, in the paired form, both
//                    polarities at once plus the correctly rounded signed float32 distance.
// Global traffic per voxel and polarity: 1 (mask) + 4 + 4 (g round trip) + 4 (output) + 1/4 (bit
// words, mostly L2) bytes -- the 13 B/voxel algorithmic figure.
//
// Exactness: every pass computes the exact min-plus of its input, so the result equals the
// reference's separable definition bit for bit (sentinel sum((n-1)^2)+1 where no site reaches,
// src/field_engine/field_edt_integer_v1.py:14-26, edt_native_large_v1/edt.cu:33-61).
#include "common.cuh"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <new>

namespace {

constexpr int kMaxAxis = 512;            // shared-memory staging holds 512 x 32 int32 per polarity
constexpr int kThreads = 512;

struct Counters {
    unsigned long long ones;     // mask bytes equal to 1
    unsigned long long invalid;  // mask bytes greater than 1
};

__global__ void __launch_bounds__(256) k_edt_bits(const uint8_t* __restrict__ mask, uint32_t* __restrict__ bits,
                                                  int64_t lines, int nz, int W, Counters* counters) {
    unsigned long long ones = 0, invalid = 0;
    const int64_t total = lines * W;
    const bool vec = (nz & 15) == 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t line = i / W;
        const int w = (int)(i - line * W);
        const int z0 = 32 * w;
        const int n = min(32, nz - z0);
        const uint8_t* src = mask + line * nz + z0;
        uint32_t word = 0;
        if (vec) {
            // 16-byte aligned: line*nz and z0 are multiples of 16.
            for (int h = 0; h < n; h += 16) {
                uint4 v = *reinterpret_cast<const uint4*>(src + h);
                uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        uint32_t byte = (q[j] >> (8 * b)) & 0xffu;
                        word |= (uint32_t)(byte != 0) << (h + 4 * j + b);
                        ones += byte == 1;
                        invalid += byte > 1;
                    }
                }
            }
        } else {
            for (int b = 0; b < n; ++b) {
                uint32_t byte = src[b];
                word |= (uint32_t)(byte != 0) << b;
                ones += byte == 1;
                invalid += byte > 1;
            }
        }
        bits[i] = word;
    }
    if (counters) {
        for (int o = 16; o > 0; o >>= 1) {
            ones += __shfl_xor_sync(0xffffffffu, ones, o);
            invalid += __shfl_xor_sync(0xffffffffu, invalid, o);
        }
        if ((threadIdx.x & 31) == 0) {
            if (ones) atomicAdd(&counters->ones, ones);
            if (invalid) atomicAdd(&counters->invalid, invalid);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Exact 1-D min-plus along a staged column, out(q) = min_s col(s) + (q - s)^2.
//
// The smallest minimiser s*(q) is non-decreasing in q (for q1 < q2 a smaller minimiser of q2
// would contradict the minimality of s*(q1); the squares' cross terms decide it).  So:
//   step A: every kSample-th target q gets (value, smallest minimiser) by a window search that
//           stops once t^2 exceeds the best value (no farther source can tie or win);
//   step B: every other target scans only [s*(q_a), s*(q_b)] between its two sampled neighbours,
//           all targets of an interval sharing each loaded source.
// Both steps are exact; the cost is ~window/kSample + interval width per target instead of
// ~2*window per target.
// ------------------------------------------------------------------------------------------
constexpr int kSample = 8;

// (value, smallest minimiser) at q; col is this lane's column (stride 32 in shared memory).
__device__ __forceinline__ int32_t window_argmin(const int32_t* col, int q, int len, int& arg) {
    int32_t best = col[q * 32];
    int bi = q;
    for (int t = 1; t < len; ++t) {
        const int32_t tt = t * t;
        if (tt > best) break;
        const int lo = q - t, hi = q + t;
        if (lo < 0 && hi >= len) break;
        if (hi < len) {  // a larger index wins only when strictly better
            const int32_t v = col[hi * 32] + tt;
            if (v < best) { best = v; bi = hi; }
        }
        if (lo >= 0) {   // a smaller index wins ties
            const int32_t v = col[lo * 32] + tt;
            if (v <= best) { best = v; bi = lo; }
        }
    }
    arg = bi;
    return best;
}

// One column pass over a shared-memory block col[len][32]; lanes are columns, warps split the
// targets.  `sidx` is shared scratch of ceil(len / kSample) * 32 int16.  `store(q, v)` receives
// every result.  Contains a __syncthreads(): every thread of the CTA must call it.
template <typename Store>
__device__ __forceinline__ void column_pass(const int32_t* col, int16_t* sidx, int len, Store store) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int nsamp = (len + kSample - 1) / kSample;
    for (int m = warp; m < nsamp; m += nwarps) {
        int arg;
        const int32_t v = window_argmin(col + lane, m * kSample, len, arg);
        sidx[m * 32 + lane] = (int16_t)arg;
        store(m * kSample, v);
    }
    __syncthreads();
    for (int m = warp; m < nsamp; m += nwarps) {
        const int q0 = m * kSample;
        const int nt = min(kSample - 1, len - 1 - q0);  // targets q0+1 .. q0+nt
        if (nt <= 0) continue;
        const int lo = sidx[m * 32 + lane];
        const int hi = m + 1 < nsamp ? sidx[(m + 1) * 32 + lane] : len - 1;
        int32_t best[kSample - 1];
#pragma unroll
        for (int i = 0; i < kSample - 1; ++i) best[i] = 0x7fffffff;
        for (int s = lo; s <= hi; ++s) {
            const int32_t f = col[s * 32 + lane];
            const int d = q0 + 1 - s;
#pragma unroll
            for (int i = 0; i < kSample - 1; ++i) best[i] = min(best[i], f + (d + i) * (d + i));
        }
#pragma unroll
        for (int i = 0; i < kSample - 1; ++i)
            if (i < nt) store(q0 + 1 + i, best[i]);
    }
}

// z pass (from bit words) + y pass.  grid = (W, nx, polarities); dynamic smem = ny * 32 * 4 bytes.
// Polarity p measures to set bits when (p ^ invert) == 0, to clear bits otherwise.
__global__ void __launch_bounds__(kThreads) k_edt_zy(const uint32_t* __restrict__ bits, int32_t* __restrict__ g,
                                                     int nx, int ny, int nz, int W, int invert, int32_t sentinel) {
    extern __shared__ int32_t col[];  // [ny][32]
    const int w = blockIdx.x, x = blockIdx.y, pol = blockIdx.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const bool flip = (pol ^ invert) != 0;
    const int tail = nz & 31;
    const uint32_t last_valid = tail ? ((1u << tail) - 1u) : 0xffffffffu;
    const int z = 32 * w + lane;
    for (int y = warp; y < ny; y += nwarps) {
        uint32_t word = 0;
        if (lane < W) {
            word = bits[((int64_t)x * ny + y) * W + lane];
            if (flip) word = ~word;
            if (lane == W - 1) word &= last_valid;
        }
        const uint32_t nonzero = __ballot_sync(0xffffffffu, word != 0);
        const uint32_t own = __shfl_sync(0xffffffffu, word, w);
        const uint32_t below = nonzero & ((1u << w) - 1u);
        const uint32_t above = nonzero & ~((2u << w) - 1u);
        const int pw = below ? 31 - __clz(below) : 0;
        const int nw = above ? __ffs(above) - 1 : 0;
        const uint32_t prev_word = __shfl_sync(0xffffffffu, word, pw);
        const uint32_t next_word = __shfl_sync(0xffffffffu, word, nw);
        int32_t value = sentinel;
        if (nonzero) {
            const uint32_t low = own & (0xffffffffu >> (31 - lane));
            const uint32_t high = own & (0xffffffffu << lane);
            int prev = -(1 << 20), next = 1 << 20;
            if (low) prev = 32 * w + 31 - __clz(low);
            else if (below) prev = 32 * pw + 31 - __clz(prev_word);
            if (high) next = 32 * w + __ffs(high) - 1;
            else if (above) next = 32 * nw + __ffs(next_word) - 1;
            const int d = min(z - prev, next - z);
            value = d * d;
        }
        col[y * 32 + lane] = value;
    }
    __syncthreads();
    int32_t* out = g + (int64_t)pol * nx * ny * nz;
    int16_t* sidx = reinterpret_cast<int16_t*>(col + ny * 32);
    const bool live = z < nz;
    column_pass(col, sidx, ny, [&](int y, int32_t v) {
        if (live) out[((int64_t)x * ny + y) * nz + z] = v;
    });
}

// Correctly rounded signed distance of one voxel from its two squared distances, the reference's
// definition (src/field_engine/edt_persistent_pair_v1/edt.cu:36-42).
__device__ __forceinline__ float signed_from_pair(int32_t sq_out, int32_t sq_in, double pitch, float half) {
    const float outside = __double2float_rn(__dmul_rn(__dsqrt_rn((double)sq_out), pitch));
    const float inside = __double2float_rn(__dmul_rn(__dsqrt_rn((double)sq_in), pitch));
    const float delta = __fsub_rn(outside, inside);
    const float sign = delta > 0.f ? 1.f : (delta < 0.f ? -1.f : 0.f);
    return __fsub_rn(delta, __fmul_rn(sign, half));
}

// x pass.  grid = (W, ny, npol_launch); dynamic smem = npol_stage * nx * 32 * 4 bytes.
// paired == 0: one polarity per CTA (blockIdx.z), writes int32 squared distances to out.
// paired == 1: both polarities in one CTA; writes the signed float32 distance and, if squared is
//              non-null, both squared arrays (polarity-major).
__global__ void __launch_bounds__(kThreads) k_edt_x(const int32_t* __restrict__ g, int32_t* __restrict__ out,
                                                    float* __restrict__ signed_out, int nx, int ny, int nz,
                                                    int paired, double pitch, float half) {
    // shared: col[npol][nx][32], then (paired) res0[nx][32], then sidx
    extern __shared__ int32_t col[];
    const int w = blockIdx.x, y = blockIdx.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int z = 32 * w + lane;
    const bool live = z < nz;
    const int64_t size = (int64_t)nx * ny * nz;
    const int npol = paired ? 2 : 1;
    const int pol0 = paired ? 0 : blockIdx.z;
    for (int p = 0; p < npol; ++p) {
        const int32_t* src = g + (int64_t)(pol0 + p) * size;
        for (int x = warp; x < nx; x += nwarps)
            col[(p * nx + x) * 32 + lane] = live ? src[((int64_t)x * ny + y) * nz + z] : 0;
    }
    int32_t* res0 = col + npol * nx * 32;
    int16_t* sidx = reinterpret_cast<int16_t*>(res0 + (paired ? nx * 32 : 0));
    __syncthreads();
    if (!paired) {
        int32_t* dst = out + (int64_t)pol0 * size;
        column_pass(col, sidx, nx, [&](int x, int32_t v) {
            if (live) dst[((int64_t)x * ny + y) * nz + z] = v;
        });
        return;
    }
    column_pass(col, sidx, nx, [&](int x, int32_t v) {
        res0[x * 32 + lane] = v;
        if (live && out) out[((int64_t)x * ny + y) * nz + z] = v;
    });
    __syncthreads();
    column_pass(col + nx * 32, sidx, nx, [&](int x, int32_t v) {
        if (!live) return;
        const int64_t i = ((int64_t)x * ny + y) * nz + z;
        signed_out[i] = signed_from_pair(res0[x * 32 + lane], v, pitch, half);
        if (out) out[size + i] = v;
    });
}

bool shape_ok(int nx, int ny, int nz) {
    return nx >= 1 && ny >= 1 && nz >= 1 && nx <= kMaxAxis && ny <= kMaxAxis && nz <= kMaxAxis;
}

int32_t sentinel_of(int nx, int ny, int nz) {
    return (nx - 1) * (nx - 1) + (ny - 1) * (ny - 1) + (nz - 1) * (nz - 1) + 1;
}

int words_of(int nz) { return (nz + 31) / 32; }

// Scratch layout: [Counters (256 B)] [bit words] [g for up to two polarities].
int64_t scratch_bytes(int nx, int ny, int nz, int npol) {
    const int64_t size = (int64_t)nx * ny * nz;
    const int64_t bits = ((int64_t)nx * ny * words_of(nz) * 4 + 255) / 256 * 256;
    return 256 + bits + (int64_t)npol * size * 4;
}

int sidx_bytes(int len) { return (len + kSample - 1) / kSample * 32 * 2; }

int configure_once() {
    static int done = 0;
    if (done) return FB_OK;
    FB_CUDA(cudaFuncSetAttribute(k_edt_zy, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kMaxAxis * 32 * 4 + sidx_bytes(kMaxAxis)));
    FB_CUDA(cudaFuncSetAttribute(k_edt_x, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 3 * kMaxAxis * 32 * 4 + sidx_bytes(kMaxAxis)));
    done = 1;
    return FB_OK;
}

// Enqueue the whole transform on `stream`.  paired == 0: sites are the nonzero mask bytes when
// sites_nonzero, else the zero bytes; writes int32 to out_sq.  paired == 1: both polarities
// (polarity 0 to the nonzero voxels), signed float32 to out_signed, optional squared pair to out_sq.
int enqueue(const uint8_t* d_mask, int nx, int ny, int nz, int paired, int sites_nonzero, double pitch,
            int32_t* out_sq, float* out_signed, void* scratch, int64_t scratch_len, cudaStream_t stream,
            bool count) {
    if (int rc = configure_once()) return rc;
    const int npol = paired ? 2 : 1;
    if (scratch_len < scratch_bytes(nx, ny, nz, npol)) return FB_INVALID;
    const int W = words_of(nz);
    const int64_t lines = (int64_t)nx * ny;
    const int64_t size = lines * nz;
    char* base = static_cast<char*>(scratch);
    Counters* counters = reinterpret_cast<Counters*>(base);
    uint32_t* bits = reinterpret_cast<uint32_t*>(base + 256);
    int32_t* g = reinterpret_cast<int32_t*>(base + 256 + ((lines * W * 4 + 255) / 256 * 256));
    if (count) FB_CUDA(cudaMemsetAsync(counters, 0, sizeof(Counters), stream));
    const int sms = fb_sm_count();
    const int64_t words = lines * W;
    int grid0 = (int)std::min<int64_t>((words + 255) / 256, (int64_t)sms * 8);
    k_edt_bits<<<grid0, 256, 0, stream>>>(d_mask, bits, lines, nz, W, count ? counters : nullptr);
    FB_LAUNCH();
    const int32_t sentinel = sentinel_of(nx, ny, nz);
    // Single polarity measuring to zero bytes = the set bits flipped.
    const int invert = paired ? 0 : (sites_nonzero ? 0 : 1);
    k_edt_zy<<<dim3(W, nx, npol), kThreads, ny * 32 * 4 + sidx_bytes(ny), stream>>>(bits, g, nx, ny, nz, W, invert,
                                                                                     sentinel);
    FB_LAUNCH();
    const float half = (float)(0.5 * pitch);
    if (paired) {
        k_edt_x<<<dim3(W, ny, 1), kThreads, 3 * nx * 32 * 4 + sidx_bytes(nx), stream>>>(g, out_sq, out_signed, nx, ny,
                                                                                         nz, 1, pitch, half);
    } else {
        k_edt_x<<<dim3(W, ny, 1), kThreads, nx * 32 * 4 + sidx_bytes(nx), stream>>>(g, out_sq, nullptr, nx, ny, nz, 0,
                                                                                     pitch, half);
    }
    FB_LAUNCH();
    (void)size;
    return FB_OK;
}

// Mask validity from the counters of k_edt_bits: 0 ok, 1 invalid (a byte > 1, or one class only).
int read_validity(const void* scratch, int64_t size, cudaStream_t stream) {
    Counters c;
    FB_CUDA(cudaMemcpyAsync(&c, scratch, sizeof(c), cudaMemcpyDeviceToHost, stream));
    FB_CUDA(cudaStreamSynchronize(stream));
    if (c.invalid) return FB_INVALID;
    if (c.ones == 0 || (int64_t)c.ones == size) return FB_INVALID;
    return FB_OK;
}

struct Pair {
    int nx, ny, nz;
    int64_t size;
    uint8_t* mask = nullptr;
    void* scratch = nullptr;
    int64_t scratch_len = 0;
    float* distance = nullptr;
    int32_t* squared = nullptr;
    cudaStream_t stream = nullptr;
    bool failed = false;
};

}  // namespace

// ---------------------------------------------------------------------------------------------
// Allocation-free EDT for callers that cannot allocate device memory.
//
// Some hosts own every byte of device memory themselves (an engine embedding this library behind
// its own pool allocator, a real-time loop that must never hit the implicit synchronisation of
// cudaMalloc/cudaFree, a plugin whose host forbids allocation calls); they can pass input and
// output buffers but not scratch.  For them the squared EDT below keeps its scratch (bit words
// and the int32 intermediate) in a fixed array compiled into this library.
//
// Limit: at most kNoAllocVoxels = 2^20 voxels and 512 per axis -- the reference's own EDT
// contract (src/field_engine/edt_native_large_v1/edt.cu:34-37).  Every GPU that loads this
// library holds the array (kNoAllocScratchBytes, about 5.1 MiB) until the process exits.
// ---------------------------------------------------------------------------------------------
constexpr int64_t kNoAllocVoxels = int64_t(1) << 20;
// bit words: nx*ny*ceil(nz/32) <= voxels/32 + nx*ny <= 2^15 + 512*512; plus 256 B of counters and
// one int32 intermediate per voxel
constexpr int64_t kNoAllocBitBytes = ((kNoAllocVoxels / 32 + 512 * 512) * 4 + 255) / 256 * 256;
constexpr int64_t kNoAllocScratchBytes = 256 + kNoAllocBitBytes + kNoAllocVoxels * 4;
static __device__ __align__(256) unsigned char g_edt_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_lock;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the array on the current device, looked up once per device.  The name
// g_edt_noalloc_scratch in host code is a host-side stand-in, not a device address, so kernels
// get this pointer instead.
int noalloc_scratch(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return FB_RUNTIME;
    std::lock_guard<std::mutex> guard(g_noalloc_lock);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_edt_noalloc_scratch) != cudaSuccess || !p) return FB_RUNTIME;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return FB_OK;
}

}  // namespace

extern "C" {

// Squared EDT exactly as fb_edt_squared_device, with no allocation and no caller scratch: the
// scratch is the library's fixed device array.  Inputs and outputs are the caller's device
// buffers.  Status 0 ok, 1 invalid arguments, 2 CUDA failure, 7 grid larger than the fixed
// scratch (more than 2^20 voxels) -- rejected before anything is enqueued.
// The first call on each device looks the array up (cudaGetSymbolAddress) with that device
// current; make that first call before any stream capture.  The array is shared by every call
// and keeps the last call's contents (nothing in it needs to start at zero: every word a call
// reads it writes first), so calls whose work overlaps on the GPU -- on different streams, or
// from different threads -- race on it and must be serialised by the caller.
int fb_edt_squared_device_noalloc(const uint8_t* d_mask, int nx, int ny, int nz, int sites_nonzero,
                                  int32_t* d_out, void* stream) noexcept {
    if (!d_mask || !d_out || !shape_ok(nx, ny, nz)) return FB_INVALID;
    if ((int64_t)nx * ny * nz > kNoAllocVoxels) return FB_NOALLOC_LIMIT;
    const int64_t need = scratch_bytes(nx, ny, nz, 1);
    if (need > kNoAllocScratchBytes) return FB_NOALLOC_LIMIT;
    void* scratch = nullptr;
    if (int rc = noalloc_scratch(&scratch)) return rc;
    return enqueue(d_mask, nx, ny, nz, 0, sites_nonzero, 1.0, d_out, nullptr, scratch, kNoAllocScratchBytes,
                   static_cast<cudaStream_t>(stream), false);
}

// Size in bytes of the fixed scratch array and the largest voxel count it serves.
int64_t fb_edt_noalloc_capacity(int64_t* max_voxels) noexcept {
    if (max_voxels) *max_voxels = kNoAllocVoxels;
    return kNoAllocScratchBytes;
}

}  // extern "C"

extern "C" {

// ---------------------------------------------------------------------------------------------
// Device-pointer forms (stream-ordered; nothing is allocated).
// ---------------------------------------------------------------------------------------------

int64_t fb_edt_scratch_bytes(int nx, int ny, int nz, int paired) {
    if (!shape_ok(nx, ny, nz)) return -1;
    return scratch_bytes(nx, ny, nz, paired ? 2 : 1);
}

int fb_edt_squared_device(const uint8_t* d_mask, int nx, int ny, int nz, int sites_nonzero, int32_t* d_out,
                          void* d_scratch, int64_t scratch_len, void* stream) noexcept {
    if (!d_mask || !d_out || !d_scratch || !shape_ok(nx, ny, nz)) return FB_INVALID;
    return enqueue(d_mask, nx, ny, nz, 0, sites_nonzero, 1.0, d_out, nullptr, d_scratch, scratch_len,
                   static_cast<cudaStream_t>(stream), false);
}

int fb_edt_pair_device(const uint8_t* d_mask, int nx, int ny, int nz, double pitch, float* d_signed,
                       int32_t* d_squared, void* d_scratch, int64_t scratch_len, void* stream) noexcept {
    if (!d_mask || !d_signed || !d_scratch || !shape_ok(nx, ny, nz)) return FB_INVALID;
    if (!std::isfinite(pitch) || pitch < 1e-12 || pitch > 1e12) return FB_INVALID;
    return enqueue(d_mask, nx, ny, nz, 1, 1, pitch, d_squared, d_signed, d_scratch, scratch_len,
                   static_cast<cudaStream_t>(stream), false);
}

// Mask check on the device: status 1 when a byte is > 1 or only one class is present.
int fb_edt_validate_device(const uint8_t* d_mask, int nx, int ny, int nz, void* d_scratch, int64_t scratch_len,
                           void* stream) noexcept {
    if (!d_mask || !d_scratch || !shape_ok(nx, ny, nz) || scratch_len < scratch_bytes(nx, ny, nz, 1))
        return FB_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int W = words_of(nz);
    const int64_t lines = (int64_t)nx * ny;
    char* base = static_cast<char*>(d_scratch);
    FB_CUDA(cudaMemsetAsync(base, 0, sizeof(Counters), s));
    int grid0 = (int)std::min<int64_t>((lines * W + 255) / 256, (int64_t)fb_sm_count() * 8);
    k_edt_bits<<<grid0, 256, 0, s>>>(d_mask, reinterpret_cast<uint32_t*>(base + 256), lines, nz, W,
                                     reinterpret_cast<Counters*>(base));
    FB_LAUNCH();
    return read_validity(base, lines * nz, s);
}

// ---------------------------------------------------------------------------------------------
// Host-pointer forms with the reference's names, arguments and status codes.
// ---------------------------------------------------------------------------------------------

static int squared_host(const uint8_t* mask, int nx, int ny, int nz, int32_t* output) {
    const int64_t size = (int64_t)nx * ny * nz;
    uint8_t* d_mask = nullptr;
    int32_t* d_out = nullptr;
    void* scratch = nullptr;
    const int64_t sb = scratch_bytes(nx, ny, nz, 1);
    int status = FB_RUNTIME;
    cudaStream_t s = nullptr;
    do {
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) break;
        if (cudaMallocAsync(&d_mask, size, s) != cudaSuccess) break;
        if (cudaMallocAsync(&d_out, size * 4, s) != cudaSuccess) break;
        if (cudaMallocAsync(&scratch, sb, s) != cudaSuccess) break;
        if (cudaMemcpyAsync(d_mask, mask, size, cudaMemcpyHostToDevice, s) != cudaSuccess) break;
        int rc = enqueue(d_mask, nx, ny, nz, 0, 0, 1.0, d_out, nullptr, scratch, sb, s, true);
        if (rc) { status = rc; break; }
        rc = read_validity(scratch, size, s);
        if (rc) { status = rc; break; }
        if (cudaMemcpyAsync(output, d_out, size * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) break;
        if (cudaStreamSynchronize(s) != cudaSuccess) break;
        status = FB_OK;
    } while (0);
    if (d_mask) cudaFreeAsync(d_mask, s);
    if (d_out) cudaFreeAsync(d_out, s);
    if (scratch) cudaFreeAsync(scratch, s);
    if (s) {
        if (cudaStreamSynchronize(s) != cudaSuccess) status = FB_RUNTIME;
        cudaStreamDestroy(s);
    }
    return status;
}

// Replaces src/field_engine/edt_native_large_v1/edt.cu:33 (edt_squared_large).  Same arguments
// and statuses; the axis limit stays 512 and the voxel cap is lifted from 2^20 to 512^3.
int edt_squared_large(const uint8_t* mask, int nx, int ny, int nz, int32_t* output) noexcept {
    if (!mask || !output || !shape_ok(nx, ny, nz)) return FB_INVALID;
    return squared_host(mask, nx, ny, nz, output);
}

// Replaces src/field_engine/edt_native_v1/edt.cu:20 (edt_squared): <= 128 per axis, <= 262144
// voxels, exactly the reference's bound.
int edt_squared(const uint8_t* mask, int nx, int ny, int nz, int32_t* output) noexcept {
    if (!mask || !output || nx < 1 || ny < 1 || nz < 1 || nx > 128 || ny > 128 || nz > 128) return FB_INVALID;
    if ((int64_t)nx * ny * nz > 262144) return FB_INVALID;
    return squared_host(mask, nx, ny, nz, output);
}

// Replaces src/field_engine/edt_persistent_pair_v1/edt.cu:48 (edt_pair_create).  Persistent
// device buffers and a private stream; the voxel cap is lifted from 2^20 to 512^3.
void* edt_pair_create(int nx, int ny, int nz) noexcept {
    if (!shape_ok(nx, ny, nz)) return nullptr;
    Pair* p = new (std::nothrow) Pair;
    if (!p) return nullptr;
    p->nx = nx;
    p->ny = ny;
    p->nz = nz;
    p->size = (int64_t)nx * ny * nz;
    p->scratch_len = scratch_bytes(nx, ny, nz, 2);
    bool ok = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&p->mask, p->size) == cudaSuccess &&
              cudaMalloc(&p->scratch, p->scratch_len) == cudaSuccess &&
              cudaMalloc(&p->distance, p->size * 4) == cudaSuccess &&
              cudaMalloc(&p->squared, p->size * 8) == cudaSuccess;
    if (!ok) {
        if (p->mask) cudaFree(p->mask);
        if (p->scratch) cudaFree(p->scratch);
        if (p->distance) cudaFree(p->distance);
        if (p->squared) cudaFree(p->squared);
        if (p->stream) cudaStreamDestroy(p->stream);
        delete p;
        return nullptr;
    }
    return p;
}

// Replaces src/field_engine/edt_persistent_pair_v1/edt.cu:59 (edt_pair_query).  Status 1 for
// invalid input (nothing written), 2 for a runtime failure, after which the handle stays failed.
int edt_pair_query(void* pointer, const uint8_t* mask, double pitch, float* output, int32_t* squared) noexcept {
    Pair* p = static_cast<Pair*>(pointer);
    if (!p || !mask || !output || !std::isfinite(pitch) || pitch < 1e-12 || pitch > 1e12) return FB_INVALID;
    if (p->failed) return FB_RUNTIME;
#define PAIR_CHECK(x)            \
    if ((x) != cudaSuccess) {    \
        p->failed = true;        \
        return FB_RUNTIME;       \
    }
    PAIR_CHECK(cudaMemcpyAsync(p->mask, mask, p->size, cudaMemcpyHostToDevice, p->stream));
    int rc = enqueue(p->mask, p->nx, p->ny, p->nz, 1, 1, pitch, p->squared, p->distance, p->scratch, p->scratch_len,
                     p->stream, true);
    if (rc) {
        p->failed = rc != FB_INVALID;
        return rc;
    }
    rc = read_validity(p->scratch, p->size, p->stream);
    if (rc == FB_INVALID) return FB_INVALID;
    if (rc) {
        p->failed = true;
        return rc;
    }
    PAIR_CHECK(cudaMemcpyAsync(output, p->distance, p->size * 4, cudaMemcpyDeviceToHost, p->stream));
    if (squared) PAIR_CHECK(cudaMemcpyAsync(squared, p->squared, p->size * 8, cudaMemcpyDeviceToHost, p->stream));
    PAIR_CHECK(cudaStreamSynchronize(p->stream));
#undef PAIR_CHECK
    return FB_OK;
}

// Replaces src/field_engine/edt_persistent_pair_v1/edt.cu:45 (edt_pair_destroy).
void edt_pair_destroy(void* pointer) noexcept {
    Pair* p = static_cast<Pair*>(pointer);
    if (!p) return;
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->mask) cudaFree(p->mask);
    if (p->scratch) cudaFree(p->scratch);
    if (p->distance) cudaFree(p->distance);
    if (p->squared) cudaFree(p->squared);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

}  // extern "C"
