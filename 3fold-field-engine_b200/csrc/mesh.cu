// Mesh -> signed distance field stage on the GPU: the reference's ray-parity winding rule and the
// paired exact EDT (src/field_engine/mesh_sdf_native_v1/field.cpp:19-226, the native form of
// faltkarna_v1_mesh_to_sdf's raypar_vindning path).
//
//   1. k_mesh_tri_count / k_mesh_tri_fill : for every triangle (a warp each, lanes over the
//      columns), the vertical rays of the (x, y) columns inside its bounding box that it crosses,
//      each hit's z and the triangle's xy orientation; count, scan, fill.  Float64 with the reference's operation order and no
//      contraction (every product and sum an explicit _rn operation), so each hit is the same bits.
//   2. k_mesh_col_count / scan / k_mesh_col_scatter : hits grouped by column (the winding sum does
//      not depend on their order within a column); the global z range by order-preserving atomics.
//   3. k_mesh_winding : a voxel is solid when the oriented hits above it (by the reference's
//      normalised key comparison) do not cancel; the voxels where winding and ray parity disagree
//      are counted.
//   4. the paired exact squared EDT of the solid mask (fb_edt_pair_device; k_long_z and
//      k_long_envelope when an axis exceeds the banded EDT's 512), then k_mesh_finish:
//      sd = float32(sqrt(sq_out) pitch) - float32(sqrt(sq_in) pitch) with the optional half-pitch
//      correction, and the surface layer (solid voxels on the boundary or next to a non-solid one).
//
// Bit-exact against the reference for the solid mask, the surface layer and the statistics.  The
// reference forms each distance from its nearest feature's offsets, sqrt((dx p)^2 + (dy p)^2 +
// (dz p)^2); here from the exact squared distance, sqrt(n) p -- the same number up to float64
// rounding, so the float32 distances agree except in the rare voxel whose value lies within a few
// float64 ulps of a float32 rounding boundary (then by one float32 ulp).
#include "common.cuh"
#include "scan.cuh"
#include <cmath>
#include <limits>

extern "C" int fb_edt_pair_device(const uint8_t* d_mask, int nx, int ny, int nz, double pitch, float* d_signed,
                                  int32_t* d_squared, void* d_scratch, int64_t scratch_len, void* stream) noexcept;
extern "C" int64_t fb_edt_scratch_bytes(int nx, int ny, int nz, int paired);

namespace {

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }

struct Grid {
    double ox, oy, oz, pitch, jx, jy;
    int64_t nx, ny, nz;
};

// Column range and orientation of triangle t (field.cpp:44-67); false when it casts no hit.
struct Tri {
    double ax, ay, az, bx, by, bz, cx, cy, cz, a2, sg;
    int64_t i0, i1, j0, j1;
    int8_t tk;
    bool local;
};

__device__ bool setup_tri(const double* __restrict__ V, const int64_t* __restrict__ T, int64_t t, const Grid& g,
                          Tri& r) {
    const double* A = V + 3 * T[3 * t];
    const double* B = V + 3 * T[3 * t + 1];
    const double* C = V + 3 * T[3 * t + 2];
    const double e1x = ds(B[0], A[0]), e1y = ds(B[1], A[1]), e2x = ds(C[0], A[0]), e2y = ds(C[1], A[1]);
    r.a2 = ds(dm(e1x, e2y), dm(e1y, e2x));
    const double skala = fmax(fmax(fabs(e1x), fabs(e1y)), fmax(fabs(e2x), fabs(e2y)));
    if (!(fabs(r.a2) > dm(dm(1e-12, skala), skala))) return false;
    const double xmin = fmin(fmin(A[0], B[0]), C[0]), xmax = fmax(fmax(A[0], B[0]), C[0]);
    const double ymin = fmin(fmin(A[1], B[1]), C[1]), ymax = fmax(fmax(A[1], B[1]), C[1]);
    int64_t i0 = (int64_t)ceil(ds(dd(ds(ds(xmin, g.jx), g.ox), g.pitch), 0.0));
    int64_t i1 = (int64_t)floor(ds(dd(ds(ds(xmax, g.jx), g.ox), g.pitch), 0.0));
    int64_t j0 = (int64_t)ceil(ds(dd(ds(ds(ymin, g.jy), g.oy), g.pitch), 0.0));
    int64_t j1 = (int64_t)floor(ds(dd(ds(ds(ymax, g.jy), g.oy), g.pitch), 0.0));
    i0 = min(max(i0, (int64_t)0), g.nx);
    i1 = min(max(i1, (int64_t)-1), g.nx - 1);
    j0 = min(max(j0, (int64_t)0), g.ny);
    j1 = min(max(j1, (int64_t)-1), g.ny - 1);
    if (i1 < i0 || j1 < j0) return false;
    r.i0 = i0; r.i1 = i1; r.j0 = j0; r.j1 = j1;
    r.sg = r.a2 > 0 ? 1.0 : (r.a2 < 0 ? -1.0 : 0.0);
    r.tk = (int8_t)(r.a2 > 0 ? 1 : (r.a2 < 0 ? -1 : 0));
    r.ax = A[0]; r.ay = A[1]; r.az = A[2];
    r.bx = B[0]; r.by = B[1]; r.bz = B[2];
    r.cx = C[0]; r.cy = C[1]; r.cz = C[2];
    const double e3 = fmax(fmax(fabs(ds(r.bx, r.ax)), fabs(ds(r.by, r.ay))), fabs(ds(r.bz, r.az)));
    const double e4 = fmax(fmax(fabs(ds(r.cx, r.ax)), fabs(ds(r.cy, r.ay))), fabs(ds(r.cz, r.az)));
    r.local = fabs(r.az) > dm(1024.0, fmax(e3, e4));
    return true;
}

// The hit of column (ii, jj), or false (field.cpp:68-80).
__device__ __forceinline__ bool column_hit(const Tri& r, const Grid& g, int64_t ii, int64_t jj, double& z) {
    const double px = da(da(g.ox, dm(da((double)ii, 0.0), g.pitch)), g.jx);
    const double py = da(da(g.oy, dm(da((double)jj, 0.0), g.pitch)), g.jy);
    const double l0 = ds(dm(ds(r.bx, px), ds(r.cy, py)), dm(ds(r.by, py), ds(r.cx, px)));
    if (!(dm(l0, r.sg) >= 0)) return false;
    const double l1 = ds(dm(ds(r.cx, px), ds(r.ay, py)), dm(ds(r.cy, py), ds(r.ax, px)));
    if (!(dm(l1, r.sg) >= 0)) return false;
    const double l2 = ds(dm(ds(r.ax, px), ds(r.by, py)), dm(ds(r.ay, py), ds(r.bx, px)));
    if (!(dm(l2, r.sg) >= 0)) return false;
    if (r.local) z = da(r.az, dd(da(dm(l1, ds(r.bz, r.az)), dm(l2, ds(r.cz, r.az))), r.a2));
    else z = dd(da(da(dm(l0, r.az), dm(l1, r.bz)), dm(l2, r.cz)), r.a2);
    return true;
}

// A warp per triangle: lanes take its bounding-box columns 32 at a time (large triangles would
// otherwise run thousands of column tests in one thread).  count[t] = hits of triangle t;
// misc[0] += its column pairs, misc[5] += its hits (64-bit totals).
__global__ void k_mesh_tri_count(const double* __restrict__ V, const int64_t* __restrict__ T, int64_t nt, Grid g,
                                 int32_t* __restrict__ count, unsigned long long* __restrict__ misc) {
    const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nt) return;  // uniform across the warp
    Tri r;
    if (!setup_tri(V, T, t, g, r)) {  // uniform: every lane computes the same setup
        if (lane == 0) count[t] = 0;
        return;
    }
    const int64_t w = r.j1 - r.j0 + 1, ncols = (r.i1 - r.i0 + 1) * w;
    int c = 0;
    for (int64_t q = lane; q < ncols; q += 32) {
        double z;
        c += column_hit(r, g, r.i0 + q / w, r.j0 + q % w, z);
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) {
        count[t] = c;
        atomicAdd(&misc[0], (unsigned long long)ncols);
        if (c) atomicAdd(&misc[5], (unsigned long long)c);
    }
}

// Order-preserving map of a float64 onto uint64 (for atomic min / max).
__device__ __forceinline__ unsigned long long order_key(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_key(unsigned long long k) {
    return __longlong_as_double((long long)((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k));
}

// A warp per triangle, as k_mesh_tri_count; the hits of one 32-column step are placed by a ballot
// prefix (their order within the triangle's range does not matter: they are regrouped by column).
__global__ void k_mesh_tri_fill(const double* __restrict__ V, const int64_t* __restrict__ T, int64_t nt, Grid g,
                                const int32_t* __restrict__ offset, int64_t* __restrict__ hcol,
                                double* __restrict__ hz, int8_t* __restrict__ hs, unsigned long long* __restrict__ zkey) {
    const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nt) return;  // uniform across the warp
    Tri r;
    if (!setup_tri(V, T, t, g, r)) return;  // uniform
    const int64_t w = r.j1 - r.j0 + 1, ncols = (r.i1 - r.i0 + 1) * w;
    int64_t at = offset[t];
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t q0 = 0; q0 < ncols; q0 += 32) {
        const int64_t q = q0 + lane;
        double z = 0.0;
        const int64_t ii = r.i0 + q / w, jj = r.j0 + q % w;
        const bool hit = q < ncols && column_hit(r, g, ii, jj, z);
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const int64_t k = at + __popc(mask & ((1u << lane) - 1u));
            hcol[k] = ii * g.ny + jj;
            hz[k] = z;
            hs[k] = r.tk;
            lo = fmin(lo, z);
            hi = fmax(hi, z);
        }
        at += __popc(mask);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0 && lo <= hi) {
        atomicMin(&zkey[0], order_key(lo));
        atomicMax(&zkey[1], order_key(hi));
    }
}

__global__ void k_mesh_col_count(const int64_t* __restrict__ hcol, int64_t nh, int32_t* __restrict__ cnt) {
    const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (h < nh) atomicAdd(&cnt[hcol[h]], 1);
}

__global__ void k_mesh_col_scatter(const int64_t* __restrict__ hcol, const double* __restrict__ hz,
                                   const int8_t* __restrict__ hs, int64_t nh, int32_t* __restrict__ cursor,
                                   double* __restrict__ cz, int8_t* __restrict__ cs) {
    const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (h >= nh) return;
    const int32_t k = atomicAdd(&cursor[hcol[h]], 1);
    cz[k] = hz[h];
    cs[k] = hs[h];
}

// One voxel per thread (field.cpp:100-123): w = sum of the orientations of the hits whose key lies
// above the voxel's key; solid = (w != 0); differs from ray parity when (count & 1) != solid.
__global__ void k_mesh_winding(const int32_t* __restrict__ start, const double* __restrict__ cz,
                               const int8_t* __restrict__ cs, Grid g, const unsigned long long* __restrict__ zkey,
                               uint8_t* __restrict__ solid, unsigned long long* __restrict__ counters) {
    const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t N = g.nx * g.ny * g.nz;
    unsigned diff = 0, nsolid = 0;
    if (v < N) {
        const int64_t c = v / g.nz, k = v - c * g.nz;
        const int32_t h0 = start[c], h1 = start[c + 1];
        uint8_t s = 0;
        if (h1 > h0) {
            const double zmin = from_key(zkey[0]), zmax = from_key(zkey[1]);
            const double span = fmax(ds(zmax, zmin), 1e-12);
            const double fc = (double)c;
            const double zc = da(g.oz, dm(da((double)k, 0.0), g.pitch));
            const double vv = da(0.25, dd(dm(0.5, ds(zc, zmin)), span));
            const double kc = da(fc, fmin(fmax(vv, 0.0), 0.999));
            const double base = da(fc, 0.25);
            int w = 0, np = 0;
            for (int32_t h = h0; h < h1; ++h) {
                const double key = da(base, dd(dm(0.5, ds(cz[h], zmin)), span));
                if (key > kc) {
                    w += cs[h];
                    ++np;
                }
            }
            s = (uint8_t)(w != 0);
            diff = (unsigned)((np & 1) != s);
        }
        solid[v] = s;
        nsolid = s;
    }
    for (int o = 16; o > 0; o >>= 1) {
        diff += __shfl_xor_sync(0xffffffffu, diff, o);
        nsolid += __shfl_xor_sync(0xffffffffu, nsolid, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (diff) atomicAdd(&counters[0], (unsigned long long)diff);
        if (nsolid) atomicAdd(&counters[1], (unsigned long long)nsolid);
    }
}

// ---- exact EDT for windows with an axis over 512 voxels (field.cpp:127-195) ----
// The banded pair EDT serves axes up to 512; longer windows (the reference accepts any grid below
// 2^31 cells) take these three separable passes, one class at a time, entirely in global memory:
//   z: a warp per (i, j) column, |offset| to the nearest feature along z (ballot scans), -1 if none;
//   y, x: a thread per line, the lower envelope of the parabolas (x - s)^2 + G(s) over the line's
//     sites with a finite G (sites without a feature are skipped, as the reference skips BIG), with
//     integer separation points (Meijster et al. 2000), so every squared distance is exact in int64.
// Adjacent threads take adjacent lines, whose elements lie next to each other in memory (lines
// along y differ in k, lines along x in (j, k)), so each step of the envelope reads coalesced.

// A warp per column: gz[v] = distance along z to the nearest voxel with (mask != 0) == feat, or -1.
__global__ void k_long_z(const uint8_t* __restrict__ mask, int64_t ncol, int64_t nz, int feat,
                         int32_t* __restrict__ gz) {
    const int64_t col = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (col >= ncol) return;  // uniform across the warp
    const uint8_t* m = mask + col * nz;
    int32_t* o = gz + col * nz;
    int64_t last = -1;
    for (int64_t k0 = 0; k0 < nz; k0 += 32) {
        const int64_t k = k0 + lane;
        const unsigned b = __ballot_sync(0xffffffffu, k < nz && ((m[k] != 0) == (feat != 0)));
        const unsigned upto = b & ((2u << lane) - 1u);  // features at or below this lane
        const int64_t at = upto ? k0 + 31 - __clz(upto) : last;
        if (k < nz) o[k] = at >= 0 ? (int32_t)(k - at) : -1;
        if (b) last = k0 + 31 - __clz(b);
    }
    int64_t next = -1;
    for (int64_t k0 = (nz - 1) / 32 * 32; k0 >= 0; k0 -= 32) {
        const int64_t k = k0 + lane;
        const unsigned b = __ballot_sync(0xffffffffu, k < nz && ((m[k] != 0) == (feat != 0)));
        const unsigned from = b & ~((1u << lane) - 1u);  // features at or above this lane
        const int64_t at = from ? k0 + __ffs(from) - 1 : next;
        if (k < nz && at >= 0) {
            const int32_t dn = (int32_t)(at - k), cur = o[k];
            if (cur < 0 || dn < cur) o[k] = dn;
        }
        if (b) next = k0 + __ffs(b) - 1;
    }
}

__device__ __forceinline__ int64_t floor_div(int64_t a, int64_t b) {  // b > 0
    return a >= 0 ? a / b : -((-a + b - 1) / b);
}

// A thread per line of n elements, stride `stride` (= the number of lines in one slab of the
// lines' outer index): line l starts at (l / stride) n stride + l % stride.  Input: int32 offsets
// (kFromZ, G = d^2) or int64 squared distances; -1 marks a site without a feature.  Output: int64
// squared distances, or (kToFloat) float32(sqrt(d2) pitch), the finish step's formula; -1 where the
// line has no site.  site/start: the envelope's stack, entry q of line l at q lines + l.
template <bool kFromZ, bool kToFloat>
__global__ void k_long_envelope(const void* __restrict__ in, int64_t lines, int64_t n, int64_t stride, double pitch,
                                void* __restrict__ out, int32_t* __restrict__ site, int32_t* __restrict__ start) {
    const int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (l >= lines) return;
    const int64_t base = l / stride * n * stride + l % stride;
    auto G = [&](int64_t u) -> int64_t {
        if (kFromZ) {
            const int64_t d = static_cast<const int32_t*>(in)[base + u * stride];
            return d < 0 ? -1 : d * d;
        }
        return static_cast<const int64_t*>(in)[base + u * stride];
    };
    int64_t q = -1;
    for (int64_t u = 0; u < n; ++u) {
        const int64_t gu = G(u);
        if (gu < 0) continue;
        while (q >= 0) {  // drop the sites that u beats at the first position they own
            const int64_t s = site[q * lines + l], t = start[q * lines + l];
            if ((t - s) * (t - s) + G(s) > (t - u) * (t - u) + gu) --q;
            else break;
        }
        if (q < 0) {
            q = 0;
            site[l] = (int32_t)u;
            start[l] = 0;
        } else {
            const int64_t s = site[q * lines + l];
            const int64_t w = 1 + floor_div(u * u - s * s + gu - G(s), 2 * (u - s));
            if (w < n) {
                ++q;
                site[q * lines + l] = (int32_t)u;
                start[q * lines + l] = (int32_t)w;
            }
        }
    }
    for (int64_t u = n - 1; u >= 0; --u) {
        int64_t d2 = -1;
        if (q >= 0) {
            const int64_t s = site[q * lines + l];
            d2 = (u - s) * (u - s) + G(s);
            if (u == start[q * lines + l]) --q;
        }
        if (kToFloat)
            static_cast<float*>(out)[base + u * stride] =
                d2 < 0 ? -1.0f : __double2float_rn(__dmul_rn(__dsqrt_rn((double)d2), pitch));
        else
            static_cast<int64_t*>(out)[base + u * stride] = d2;
    }
}

// sd and the surface layer (field.cpp:197-214).  sq: the pair [to solid | to non-solid] of squared
// distances; else dist: the pair of distances; else (both nullptr) one class is empty: that class's
// distance is then -1 (the reference's value for lines with no feature) and the other's 0 (every
// voxel is its own feature).
__global__ void k_mesh_finish(const uint8_t* __restrict__ solid, const int32_t* __restrict__ sq,
                              const float* __restrict__ dist, Grid g, int empty_class, int ytkorr,
                              float* __restrict__ sd, uint8_t* __restrict__ yta) {
    const int64_t lin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t N = g.nx * g.ny * g.nz;
    if (lin >= N) return;
    float d[2];
    for (int cls = 0; cls < 2; ++cls) {
        if (sq) d[cls] = __double2float_rn(__dmul_rn(__dsqrt_rn((double)sq[cls * N + lin]), g.pitch));
        else if (dist) d[cls] = dist[cls * N + lin];
        else d[cls] = cls == empty_class ? -1.0f : 0.0f;
    }
    float v = __fsub_rn(d[0], d[1]);
    if (ytkorr) {
        const float half = __double2float_rn(0.5 * g.pitch);
        const float sgn = v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f);
        v = __fsub_rn(v, __fmul_rn(sgn, half));
    }
    sd[lin] = v;
    const uint8_t s = solid[lin];
    uint8_t y = 0;
    if (s) {
        const int64_t k = lin % g.nz, j = (lin / g.nz) % g.ny, i = lin / (g.nz * g.ny);
        const int64_t pl = g.ny * g.nz;
        if (i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1 || k == 0 || k == g.nz - 1) y = 1;
        else if (!solid[lin - pl] || !solid[lin + pl] || !solid[lin - g.nz] || !solid[lin + g.nz] || !solid[lin - 1] ||
                 !solid[lin + 1])
            y = 1;
    }
    yta[lin] = y;
}

// One device allocation carved into 256-byte aligned parts (a call makes two: one sized before the
// ray hits are counted, one for the hits), so a call meets cudaMalloc / cudaFree twice, not per array.
struct Slab {
    char* base = nullptr;
    size_t size = 0;
    ~Slab() {
        if (base) cudaFree(base);
    }
    template <typename T>
    size_t reserve(int64_t n) {
        const size_t at = size;
        size += (std::max<int64_t>(n, 1) * sizeof(T) + 255) / 256 * 256;
        return at;
    }
    int allocate() { return cudaMalloc(&base, std::max<size_t>(size, 256)) == cudaSuccess ? FB_OK : FB_RUNTIME; }
    template <typename T>
    T* at(size_t offset) const {
        return reinterpret_cast<T*>(base + offset);
    }
};

}  // namespace

extern "C" {

// Replaces meshsdf_field_cpu, src/field_engine/mesh_sdf_native_v1/field.cpp:19-226, with the same
// arguments, outputs and status codes (1 contract, 2 face index outside [0, nv), 3 more than
// 2^31 - 2 hits), computed on the current GPU; nthreads is accepted and ignored, tstage[0..4] are
// the stage times in seconds (hits, grouping, winding, EDT, finish).  Host pointers.
int meshsdf_field_cpu(const double* V, int64_t nv, const int64_t* T, int64_t nt, double ox, double oy, double oz,
                      double pitch, double jx, double jy, int64_t nx, int64_t ny, int64_t nz, int ytkorr,
                      int nthreads, uint8_t* solid, float* sd, uint8_t* yta, int64_t* stats, double* tstage) noexcept {
    (void)nthreads;
    const int64_t CELLS_MAX = (int64_t)std::numeric_limits<int32_t>::max() - 1;
    if (!V || !T || !solid || !sd || !yta || !stats || !tstage) return 1;
    if (nv < 1 || nt < 1 || nt > CELLS_MAX || nv > std::numeric_limits<int64_t>::max() / 3) return 1;
    if (nx < 1 || ny < 1 || nz < 1 || nx > CELLS_MAX / ny || nx * ny > CELLS_MAX / nz) return 1;
    if (!(std::isfinite(pitch) && pitch > 0) || !std::isfinite(ox) || !std::isfinite(oy) || !std::isfinite(oz) ||
        !std::isfinite(jx) || !std::isfinite(jy))
        return 1;
    for (int64_t t = 0; t < 3 * nt; ++t)
        if (T[t] < 0 || T[t] >= nv) return 2;
    // axes over 512 voxels take the long-axis EDT passes instead of the banded pair EDT
    const bool long_axes = nx > 512 || ny > 512 || nz > 512;
    const Grid g{ox, oy, oz, pitch, jx, jy, nx, ny, nz};
    const int64_t ncol = nx * ny, N = ncol * nz;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return FB_RUNTIME;
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{st};
    cudaEvent_t ev[6];
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) return FB_RUNTIME;
    struct EventGuard {
        cudaEvent_t* e;
        ~EventGuard() {
            for (int i = 0; i < 6; ++i) cudaEventDestroy(e[i]);
        }
    } eguard{ev};
    const int64_t sb = long_axes ? 0 : fb_edt_scratch_bytes((int)nx, (int)ny, (int)nz, 1);
    if (sb < 0) return 1;
    const int64_t nl = long_axes ? N : 0;  // the long-axis passes' arrays
    const int64_t words_t = scan_scratch_words(nt), words_c = scan_scratch_words(ncol + 1);
    Slab A;
    const size_t oV = A.reserve<double>(3 * nv), oT = A.reserve<int64_t>(3 * nt), oCount = A.reserve<int32_t>(nt + 1),
                 oMisc = A.reserve<unsigned long long>(8), oScan = A.reserve<int32_t>(std::max(words_t, words_c)),
                 oStart = A.reserve<int32_t>(ncol + 1), oCursor = A.reserve<int32_t>(ncol + 1),
                 oSolid = A.reserve<uint8_t>(N), oYta = A.reserve<uint8_t>(N), oSd = A.reserve<float>(N),
                 oSq = A.reserve<int32_t>(long_axes ? 0 : 2 * N), oEdt = A.reserve<uint8_t>(sb),
                 oGz = A.reserve<int32_t>(nl), oF2 = A.reserve<int64_t>(nl), oSite = A.reserve<int32_t>(nl),
                 oFrom = A.reserve<int32_t>(nl), oDist = A.reserve<float>(2 * nl);
    if (A.allocate()) return FB_RUNTIME;
    double* const dV = A.at<double>(oV);
    int64_t* const dT = A.at<int64_t>(oT);
    int32_t* const tri_count = A.at<int32_t>(oCount);
    int32_t* const scan_scratch = A.at<int32_t>(oScan);
    int32_t* const start = A.at<int32_t>(oStart);
    int32_t* const cursor = A.at<int32_t>(oCursor);
    int32_t* const sq = A.at<int32_t>(oSq);
    unsigned long long* const misc = A.at<unsigned long long>(oMisc);  // npairs, zmin key, zmax key, ndiff, nsolid, nh
    uint8_t* const dsolid = A.at<uint8_t>(oSolid);
    uint8_t* const dyta = A.at<uint8_t>(oYta);
    uint8_t* const edt_scratch = A.at<uint8_t>(oEdt);
    float* const dsd = A.at<float>(oSd);
    FB_CUDA(cudaMemcpyAsync(dV, V, 3 * nv * sizeof(double), cudaMemcpyHostToDevice, st));
    FB_CUDA(cudaMemcpyAsync(dT, T, 3 * nt * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    const unsigned long long init[8] = {0, ~0ull, 0, 0, 0, 0, 0, 0};
    FB_CUDA(cudaMemcpyAsync(misc, init, sizeof(init), cudaMemcpyHostToDevice, st));
    FB_CUDA(cudaEventRecord(ev[0], st));
    // 1. hits per triangle, scanned to offsets
    const unsigned tb = (unsigned)((nt + 7) / 8);  // a warp per triangle, 8 per block
    k_mesh_tri_count<<<tb, 256, 0, st>>>(dV, dT, nt, g, tri_count, misc);
    FB_LAUNCH();
    // offsets of each triangle's hits; the int32 total lands in the spare last word (the 64-bit
    // total in misc[5] is the one checked)
    if (int rc = scan_exclusive(tri_count, nt, tri_count + nt, scan_scratch, words_t, st)) return rc;
    unsigned long long nh64 = 0;
    FB_CUDA(cudaMemcpyAsync(&nh64, misc + 5, sizeof(nh64), cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    // hit offsets are int32 (the scan above): beyond that the reference refuses too, before any output
    if (nh64 > (unsigned long long)CELLS_MAX) return 3;
    const int64_t nh = (int64_t)nh64;
    Slab B;
    const size_t oHcol = B.reserve<int64_t>(nh), oHz = B.reserve<double>(nh), oCz = B.reserve<double>(nh),
                 oHs = B.reserve<int8_t>(nh), oCs = B.reserve<int8_t>(nh);
    if (B.allocate()) return FB_RUNTIME;
    int64_t* const hcol = B.at<int64_t>(oHcol);
    double* const hz = B.at<double>(oHz);
    double* const cz = B.at<double>(oCz);
    int8_t* const hs = B.at<int8_t>(oHs);
    int8_t* const cs = B.at<int8_t>(oCs);
    k_mesh_tri_fill<<<tb, 256, 0, st>>>(dV, dT, nt, g, tri_count, hcol, hz, hs, misc + 1);
    FB_LAUNCH();
    FB_CUDA(cudaEventRecord(ev[1], st));
    // 2. hits grouped by column
    FB_CUDA(cudaMemsetAsync(start, 0, (ncol + 1) * sizeof(int32_t), st));
    const unsigned hb = (unsigned)((nh + 255) / 256);
    if (nh > 0) {
        k_mesh_col_count<<<hb, 256, 0, st>>>(hcol, nh, start);
        FB_LAUNCH();
    }
    // exclusive scan over ncol + 1 entries: start[ncol] becomes nh
    if (int rc = scan_exclusive(start, ncol + 1, cursor + ncol, scan_scratch, words_c, st))
        return rc;
    FB_CUDA(cudaMemcpyAsync(cursor, start, (ncol + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    if (nh > 0) {
        k_mesh_col_scatter<<<hb, 256, 0, st>>>(hcol, hz, hs, nh, cursor, cz, cs);
        FB_LAUNCH();
    }
    FB_CUDA(cudaEventRecord(ev[2], st));
    // 3. winding
    k_mesh_winding<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(start, cz, cs, g, misc + 1, dsolid,
                                                                   misc + 3);
    FB_LAUNCH();
    unsigned long long host_misc[8];
    FB_CUDA(cudaMemcpyAsync(host_misc, misc, sizeof(host_misc), cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    FB_CUDA(cudaEventRecord(ev[3], st));
    const int64_t nsolid = (int64_t)host_misc[4];
    // 4. paired EDT when both classes are present
    int empty = -1;
    if (nsolid == 0) empty = 0;       // no solid voxel: no feature for the distance to the solid
    else if (nsolid == N) empty = 1;  // no empty voxel
    float* const dist = A.at<float>(oDist);
    if (empty < 0 && long_axes) {
        int32_t* const gz = A.at<int32_t>(oGz);
        int64_t* const f2 = A.at<int64_t>(oF2);
        int32_t* const site = A.at<int32_t>(oSite);
        int32_t* const from = A.at<int32_t>(oFrom);
        for (int cls = 0; cls < 2; ++cls) {  // features: the solid voxels, then the others
            k_long_z<<<(unsigned)((ncol + 7) / 8), 256, 0, st>>>(dsolid, ncol, nz, cls == 0, gz);
            FB_LAUNCH();
            k_long_envelope<true, false><<<(unsigned)((nx * nz + 255) / 256), 256, 0, st>>>(gz, nx * nz, ny, nz, pitch,
                                                                                         f2, site, from);
            FB_LAUNCH();
            k_long_envelope<false, true><<<(unsigned)((ny * nz + 255) / 256), 256, 0, st>>>(
                f2, ny * nz, nx, ny * nz, pitch, dist + cls * N, site, from);
            FB_LAUNCH();
        }
    } else if (empty < 0) {
        if (int rc = fb_edt_pair_device(dsolid, (int)nx, (int)ny, (int)nz, pitch, dsd, sq, edt_scratch, sb, st))
            return rc == FB_INVALID ? 1 : FB_RUNTIME;
    }
    FB_CUDA(cudaEventRecord(ev[4], st));
    // 5. sd and the surface layer
    k_mesh_finish<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(dsolid, empty < 0 && !long_axes ? sq : nullptr,
                                                                  empty < 0 && long_axes ? dist : nullptr, g, empty,
                                                                  ytkorr ? 1 : 0, dsd, dyta);
    FB_LAUNCH();
    FB_CUDA(cudaEventRecord(ev[5], st));
    FB_CUDA(cudaMemcpyAsync(solid, dsolid, N, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaMemcpyAsync(sd, dsd, N * sizeof(float), cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaMemcpyAsync(yta, dyta, N, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    stats[0] = (int64_t)host_misc[0];
    stats[1] = nh;
    stats[2] = (int64_t)host_misc[3];
    stats[3] = nsolid;
    for (int i = 0; i < 5; ++i) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        tstage[i] = ms * 1e-3;
    }
    return 0;
}

}  // extern "C"
