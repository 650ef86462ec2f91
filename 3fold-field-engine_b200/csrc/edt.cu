// Exact integer squared Euclidean distance transform and the paired signed distance, sm_100a.
//
// Algorithm (a from-scratch design, not the reference's one-thread-per-line envelope):
//   1. k_edt_bits  : the uint8 mask becomes one 32-bit word per 32 z-samples of every (x, y) line
//                    (1 B read + 1/8 B written per voxel, four bytes per SWAR step); the validating
//                    form also checks the mask (values 0/1, both classes present) with
//                    warp-aggregated counters.
//   2. k_edt_zy    : one CTA per (32-wide z chunk, x plane, polarity), lanes = z columns.  For every
//                    y line it finds the nearest site along z from the line's bit words (clz/ffs over
//                    the chunk's own word, a ballot over the other words) into shared memory, then
//                    runs the y pass g(y,z) = min_y' dz(y',z)^2 + (y-y')^2 as an exact lower
//                    envelope (below), banded over the CTA's warps.  Writes int32 g (4 B/voxel).
//   3. k_edt_x     : one CTA per (z chunk, y row, polarity): stages the nx x 32 column block of g in
//                    shared memory with cp.async (coalesced 128 B rows, every load in flight at
//                    once), runs the same envelope along x in place and writes the final int32
//                    (4 B/voxel); the paired form runs both polarities, then k_edt_signed turns the
//                    two squared distances into the correctly rounded signed float32.
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

constexpr int kMaxAxis = 512;            // hull entries pack a site index < 2^11 and c < 2^21; smem holds 512 x 32

struct Counters {
    unsigned long long ones;     // mask bytes equal to 1
    unsigned long long invalid;  // mask bytes greater than 1
};

// Nonzero flags of the four bytes of q as bits 0..3 (byte i -> bit i).  The byte-wise OR folds
// every bit of a byte onto its bit 0; the multiply then gathers the four bit-0s: byte i's bit lands
// at bit 24 + i of the product and no partial products overlap, so nothing carries.
__device__ __forceinline__ uint32_t nonzero4(uint32_t q) {
    uint32_t t = q | (q >> 4);
    t |= t >> 2;
    t |= t >> 1;
    t &= 0x01010101u;
    return (t * 0x01020408u) >> 24;
}

// kCount: also count the mask bytes equal to 1 and flag bytes greater than 1.
template <bool kCount>
__global__ void __launch_bounds__(256) k_edt_bits(const uint8_t* __restrict__ mask, uint32_t* __restrict__ bits,
                                                  int64_t lines, int nz, int W, Counters* counters) {
    unsigned long long ones = 0;
    uint32_t bad = 0;
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
            // 16-byte aligned: line*nz and z0 are multiples of 16; n is 16 or 32.
            for (int h = 0; h < n; h += 16) {
                const uint4 v = *reinterpret_cast<const uint4*>(src + h);
                const uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    word |= nonzero4(q[j]) << (h + 4 * j);
                    if (kCount) {
                        ones += __popc(q[j] & 0x01010101u);
                        bad |= q[j] & 0xfefefefeu;
                    }
                }
            }
        } else {
            for (int b = 0; b < n; ++b) {
                const uint32_t byte = src[b];
                word |= (uint32_t)(byte != 0) << b;
                if (kCount) {
                    ones += byte & 1u;
                    bad |= byte & 0xfeu;
                }
            }
        }
        bits[i] = word;
    }
    if (kCount) {
        // a byte > 1 makes the mask invalid whatever `ones` says, so `ones` may count its low bit
        unsigned long long invalid = bad != 0;
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

void launch_bits(int grid, cudaStream_t stream, const uint8_t* mask, uint32_t* bits, int64_t lines, int nz, int W,
                 Counters* counters) {
    if (counters) k_edt_bits<true><<<grid, 256, 0, stream>>>(mask, bits, lines, nz, W, counters);
    else k_edt_bits<false><<<grid, 256, 0, stream>>>(mask, bits, lines, nz, W, nullptr);
}

// ------------------------------------------------------------------------------------------
// Exact 1-D min-plus along a column, out(q) = min_s f(s) + (q - s)^2, by lower envelopes.
//
// Site s contributes the parabola P_s(q) = c_s - 2 q s + q^2 with c_s = f(s) + s^2, so out(q) is the
// lower envelope of lines c_s - 2 q s plus q^2: the sites that matter are the vertices of the lower
// convex hull of the points (s, c_s), and site b between a and u is never strictly lowest exactly
// when (c_b - c_a)(u - b) >= (c_u - c_b)(b - a) -- an integer test, no division (the reference's
// envelope intersects parabolas with floor division instead, edt_persistent_pair_v1/edt.cu:12-29).
// Sites with no finite value (the sentinel) never win against a finite one and are left out.
//
// A CTA owns 32 adjacent columns (lanes) over the whole axis, staged in shared memory as rows of
// 32 words (row r holds f(r) of the 32 columns: 128 B, conflict-free per lane); its kBandWarps
// warps split the axis into bands:
//   1. stage : f of the band's rows lands in the band's own rows of the array (cp.async from global
//              memory in the x pass; computed from the bit words in the zy pass);
//   2. build : each warp runs the hull stack over its band's rows, one stack per lane, in place --
//              stack entry k overwrites row r0 + k, never beyond the row being read;
//   3. merge : pairwise joins of band groups in log2(kBandWarps) rounds -- the bridge between two
//              x-separated lower hulls trims a suffix of the left one and a prefix of the right one --
//              leaving each band a contiguous surviving range [lo, hi];
//   4. output: each warp finds the hull vertex covering its first target (band scan + binary search)
//              and walks the hull forward over its targets, one compare per step.
// Values are exact integers: c < 2^21 and |products| < 2^31 for axes up to 512.
// ------------------------------------------------------------------------------------------
constexpr int kBandWarps = 8;
constexpr int kBandThreads = 32 * kBandWarps;
constexpr int kNever = 1 << 30;  // c of a successor that never wins (every real c is < 2^21)

__device__ __forceinline__ uint32_t pack_site(int v, int c) { return ((uint32_t)v << 21) | (uint32_t)c; }
__device__ __forceinline__ int site_v(uint32_t e) { return (int)(e >> 21); }
__device__ __forceinline__ int site_c(uint32_t e) { return (int)(e & 0x1fffffu); }

// Middle site b of a < b < u is never strictly below both neighbours' parabolas.
__device__ __forceinline__ bool hidden(uint32_t a, uint32_t b, uint32_t u) {
    const int va = site_v(a), vb = site_v(b), vu = site_v(u);
    const int ca = site_c(a), cb = site_c(b), cu = site_c(u);
    return (cb - ca) * (vu - vb) >= (cu - cb) * (vb - va);
}

// P_next(q) <= P_cur(q) for sites cur < next: the hull walk moves on.
__device__ __forceinline__ bool next_wins(uint32_t cur, uint32_t nxt, int q) {
    return site_c(nxt) - site_c(cur) <= 2 * q * (site_v(nxt) - site_v(cur));
}

// Shared layout of a band pass over an axis of length n: hull[n][32] entries, then per band and
// lane the entry count and the surviving range.
struct BandSmem {
    uint32_t* hull;
    int* cnt;
    int* lo;
    int* hi;
};

__device__ __forceinline__ BandSmem band_smem(void* base, int n) {
    BandSmem b;
    b.hull = static_cast<uint32_t*>(base);
    b.cnt = reinterpret_cast<int*>(b.hull + n * 32);
    b.lo = b.cnt + kBandWarps * 32;
    b.hi = b.lo + kBandWarps * 32;
    return b;
}

__host__ __device__ __forceinline__ int band_rows(int n) { return (n + kBandWarps - 1) / kBandWarps; }

int band_smem_bytes(int n) { return n * 32 * 4 + 3 * kBandWarps * 32 * 4; }

// Hull stack of one lane over rows r0, r0 + 1, ... whose f values sit in the lane's column of
// the staged rows; entries overwrite the rows from r0 on (entry k at row r0 + k).  Registers hold
// the top entry (v1, c1) and its edge from the entry below (dv, dc), so the convexity test is one
// multiply-compare and a pop needs one shared-memory load.
struct InPlaceHull {
    uint32_t* base;  // &hull[r0 * 32 + lane]
    int r0;
    int top;             // index of the top entry, -1 when empty
    int v1, c1, dv, dc;  // top entry; top minus the entry below (valid when top >= 1)

    __device__ __forceinline__ InPlaceHull(uint32_t* hull, int r0_, int lane)
        : base(hull + r0_ * 32 + lane), r0(r0_), top(-1), v1(0), c1(0), dv(1), dc(0) {}

    // rows [ra, rb) in increasing order; f >= sentinel is no site
    __device__ __forceinline__ void rows(int ra, int rb, int32_t sentinel) {
#pragma unroll 4
        for (int v = ra; v < rb; ++v) {
            const int f = (int)base[(v - r0) * 32];
            if (f >= sentinel) continue;
            const int c = f + v * v;
            int ev = v - v1, ec = c - c1;
            // the top is hidden between the entry below it and the new site
            while (top >= 1 && dc * ev >= ec * dv) {
                --top;
                v1 -= dv;
                c1 -= dc;
                if (top >= 1) {
                    const uint32_t e = base[(top - 1) * 32];
                    dv = v1 - site_v(e);
                    dc = c1 - site_c(e);
                }
                ev = v - v1;
                ec = c - c1;
            }
            ++top;
            base[top * 32] = pack_site(v, c);
            v1 = v;
            c1 = c;
            dv = ev;
            dc = ec;
        }
    }
};

__device__ __forceinline__ bool band_live(const BandSmem& sm, int b, int lane) {
    return sm.hi[b * 32 + lane] >= sm.lo[b * 32 + lane];
}

// Phase 3: pairwise joins of band groups in log2(kBandWarps) rounds (warp j joins group j of the
// round), each the bridge between two x-separated lower hulls: trim the left group's suffix and the
// right group's prefix until the junction is convex.  Every band ends with a surviving range [lo, hi]
// (empty when hi < lo); the ranges in band order are the column's lower hull.  Contains
// __syncthreads(): every thread of the CTA calls it.
__device__ void hull_merge(const BandSmem& sm, int n) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rows = band_rows(n);
    sm.lo[warp * 32 + lane] = 0;
    sm.hi[warp * 32 + lane] = sm.cnt[warp * 32 + lane] - 1;
    for (int half = 1; half < kBandWarps; half *= 2) {
        __syncthreads();
        const int a = warp * 2 * half, m = a + half, e = min(kBandWarps, a + 2 * half);
        if (m < kBandWarps) {
            int L = m - 1;
            while (L >= a && !band_live(sm, L, lane)) --L;
            int R = m;
            while (R < e && !band_live(sm, R, lane)) ++R;
            if (L >= a && R < e) {
                // every step removes one entry: the loop ends within n steps
                for (int step = 0; step <= n; ++step) {
                    const int hiL = sm.hi[L * 32 + lane], loR = sm.lo[R * 32 + lane];
                    const uint32_t e1 = sm.hull[(L * rows + hiL) * 32 + lane];
                    const uint32_t r0 = sm.hull[(R * rows + loR) * 32 + lane];
                    int pb = L, pi = hiL - 1;
                    if (pi < sm.lo[L * 32 + lane]) {
                        pb = L - 1;
                        while (pb >= a && !band_live(sm, pb, lane)) --pb;
                        pi = pb >= a ? sm.hi[pb * 32 + lane] : -1;
                    }
                    if (pb >= a && hidden(sm.hull[(pb * rows + pi) * 32 + lane], e1, r0)) {
                        sm.hi[L * 32 + lane] = hiL - 1;
                        if (hiL - 1 < sm.lo[L * 32 + lane]) L = pb;
                        continue;
                    }
                    int sb = R, si = loR + 1;
                    if (si > sm.hi[R * 32 + lane]) {
                        sb = R + 1;
                        while (sb < e && !band_live(sm, sb, lane)) ++sb;
                        si = sb < e ? sm.lo[sb * 32 + lane] : -1;
                    }
                    if (sb < e && hidden(e1, r0, sm.hull[(sb * rows + si) * 32 + lane])) {
                        sm.lo[R * 32 + lane] = loR + 1;
                        if (loR + 1 > sm.hi[R * 32 + lane]) R = sb;
                        continue;
                    }
                    break;
                }
            }
        }
    }
    __syncthreads();
}

// Phase 4 for targets [q0, q1) of one warp: store(value) for q = q0, q0 + 1, ... in order; lanes
// whose column has no site store `sentinel`.
template <typename Store>
__device__ __forceinline__ void hull_output(const BandSmem& sm, int n, int q0, int q1, int32_t sentinel, Store store) {
    const int lane = threadIdx.x & 31;
    const int rows = band_rows(n);
    if (q0 >= q1) return;
    int b = 0;
    while (b < kBandWarps && !band_live(sm, b, lane)) ++b;
    if (b == kBandWarps) {
        for (int q = q0; q < q1; ++q) store(sentinel);
        return;
    }
    // band holding the vertex that covers q0: the first band whose last surviving entry is not
    // beaten at q0 by the next surviving band's first one
    for (;;) {
        int nb = b + 1;
        while (nb < kBandWarps && !band_live(sm, nb, lane)) ++nb;
        if (nb == kBandWarps) break;
        if (!next_wins(sm.hull[(b * rows + sm.hi[b * 32 + lane]) * 32 + lane],
                       sm.hull[(nb * rows + sm.lo[nb * 32 + lane]) * 32 + lane], q0))
            break;
        b = nb;
    }
    // binary search inside band b: the first index whose successor does not win at q0
    int lo = sm.lo[b * 32 + lane], hi = sm.hi[b * 32 + lane];
    {
        const uint32_t* band = sm.hull + b * rows * 32 + lane;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (next_wins(band[mid * 32], band[(mid + 1) * 32], q0)) lo = mid + 1;
            else hi = mid;
        }
    }
    // walk: p points at the successor of the current vertex (vc, cc), dn = its v - vc and cn its
    // c - cc; pend is the last surviving entry of p's band.  Past the last vertex the successor
    // never wins (dn = 0, cn = kNever).
    const uint32_t* p = sm.hull + (b * rows + lo) * 32 + lane;
    const uint32_t* pend = sm.hull + (b * rows + sm.hi[b * 32 + lane]) * 32 + lane;
    const uint32_t e = *p;
    int vc = site_v(e), cc = site_c(e);
    int dn = 0, cn = kNever;
    auto fetch = [&]() {
        if (p < pend) {
            p += 32;
        } else {
            int k = b + 1;
            while (k < kBandWarps && !band_live(sm, k, lane)) ++k;
            if (k == kBandWarps) {
                dn = 0;
                cn = kNever;
                return;
            }
            b = k;
            p = sm.hull + (k * rows + sm.lo[k * 32 + lane]) * 32 + lane;
            pend = sm.hull + (k * rows + sm.hi[k * 32 + lane]) * 32 + lane;
        }
        const uint32_t x = *p;
        dn = site_v(x) - vc;
        cn = site_c(x) - cc;
    };
    fetch();
#pragma unroll 4
    for (int q = q0; q < q1; ++q) {
        const int q2 = 2 * q;
        while (cn <= q2 * dn) {
            vc += dn;
            cc += cn;
            fetch();
        }
        store(cc + q * (q - 2 * vc));
    }
}

__device__ __forceinline__ void cp_async4(uint32_t* smem_dst, const int32_t* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// z pass (nearest set bit along z from the bit words) + y pass.  grid = (W, nx, polarities),
// block = kBandThreads, dynamic smem = band_smem_bytes(ny).  Polarity p measures to set bits when
// (p ^ invert) == 0, to clear bits otherwise.
__global__ void __launch_bounds__(kBandThreads) k_edt_zy(const uint32_t* __restrict__ bits, int32_t* __restrict__ g,
                                                         int nx, int ny, int nz, int W, int invert, int32_t sentinel) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BandSmem sm = band_smem(smem_raw, ny);
    const int w = blockIdx.x, x = blockIdx.y, pol = blockIdx.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool flip = (pol ^ invert) != 0;
    const int tail = nz & 31;
    const uint32_t last_valid = tail ? ((1u << tail) - 1u) : 0xffffffffu;
    const int z = 32 * w + lane;
    const int rows = band_rows(ny);
    const int y0 = warp * rows, y1 = min(ny, y0 + rows);
    // 1. f(y) = squared distance to the nearest site along z, for each row of the band, into the
    //    band's rows (sentinel where the row has no site)
    uint32_t* const mine = sm.hull + y0 * 32 + lane;
    const uint32_t* line = bits + ((int64_t)x * ny + y0) * W + lane;  // row y0's words, one per lane < W
    const bool loads = lane < W;
    const uint32_t below_mask = (1u << w) - 1u, above_mask = ~((2u << w) - 1u);
    const uint32_t low_mask = 0xffffffffu >> (31 - lane), high_mask = 0xffffffffu << lane;
    constexpr int kAhead = 8;  // rows of bit words in flight
    uint32_t ring[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; ++k) ring[k] = (loads && y0 + k < y1) ? line[k * W] : 0u;
    for (int yb = y0; yb < y1; yb += kAhead) {
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
            const int y = yb + k;
            uint32_t word = ring[k];
            ring[k] = (loads && y + kAhead < y1) ? line[(y + kAhead - y0) * W] : 0u;
            if (y >= y1) break;
            if (loads) {
                if (flip) word = ~word;
                if (lane == W - 1) word &= last_valid;
            }
            const uint32_t nonzero = __ballot_sync(0xffffffffu, word != 0);
            int f = sentinel;
            if (nonzero) {  // uniform across the warp
                const uint32_t own = __shfl_sync(0xffffffffu, word, w);
                const uint32_t below = nonzero & below_mask;
                const uint32_t above = nonzero & above_mask;
                const int pw = below ? 31 - __clz(below) : 0;
                const int nw = above ? __ffs(above) - 1 : 0;
                const uint32_t prev_word = __shfl_sync(0xffffffffu, word, pw);
                const uint32_t next_word = __shfl_sync(0xffffffffu, word, nw);
                const uint32_t low = own & low_mask;
                const uint32_t high = own & high_mask;
                int prev = -(1 << 20), next = 1 << 20;
                if (low) prev = 32 * w + 31 - __clz(low);
                else if (below) prev = 32 * pw + 31 - __clz(prev_word);
                if (high) next = 32 * w + __ffs(high) - 1;
                else if (above) next = 32 * nw + __ffs(next_word) - 1;
                const int d = min(z - prev, next - z);
                f = d * d;
            }
            mine[(y - y0) * 32] = (uint32_t)f;
        }
    }
    // 2. hull stack over the band, in place
    InPlaceHull st(sm.hull, y0, lane);
    st.rows(y0, y1, sentinel);
    sm.cnt[warp * 32 + lane] = st.top + 1;
    hull_merge(sm, ny);
    if (z >= nz) return;
    int32_t* out = g + (int64_t)pol * nx * ny * nz + ((int64_t)x * ny + y0) * nz + z;
    hull_output(sm, ny, y0, y1, sentinel, [&](int32_t v) {
        *out = v;
        out += nz;
    });
}

// x pass.  grid = (W, ny, polarities), block = kBandThreads, dynamic smem = band_smem_bytes(nx).
// Reads g (polarity-major, `size` voxels each) and writes out with the same layout; out may be g
// itself (each CTA reads its whole column block before it writes any of it).
__global__ void __launch_bounds__(kBandThreads) k_edt_x(const int32_t* g, int32_t* out, int nx, int ny, int nz,
                                                        int32_t sentinel) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BandSmem sm = band_smem(smem_raw, nx);
    const int w = blockIdx.x, y = blockIdx.y, pol = blockIdx.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int z = 32 * w + lane;
    const bool live = z < nz;
    const int64_t size = (int64_t)nx * ny * nz;
    const int64_t col = (int64_t)pol * size + (int64_t)y * nz + z;
    const int64_t stride = (int64_t)ny * nz;
    const int rows = band_rows(nx);
    const int x0 = warp * rows, x1 = min(nx, x0 + rows);
    // 1. stage the band's column values into its rows, in four commit groups so that the hull
    //    starts on the first quarter while the rest is in flight
    constexpr int kGroups = 4;
    const int chunk = (rows + kGroups - 1) / kGroups;
    uint32_t* const mine = sm.hull + x0 * 32 + lane;
    InPlaceHull st(sm.hull, x0, lane);
    if (live) {
        const int32_t* src = g + col + (int64_t)x0 * stride;
#pragma unroll
        for (int j = 0; j < kGroups; ++j) {
            const int ka = j * chunk, kb = min(x1 - x0, ka + chunk);
            for (int k = ka; k < kb; ++k) cp_async4(mine + k * 32, src + (int64_t)k * stride);
            cp_async_commit();
        }
        // 2. hull stack over the band, in place, one commit group at a time
        cp_async_wait<kGroups - 1>();
        st.rows(x0, min(x1, x0 + chunk), sentinel);
        cp_async_wait<kGroups - 2>();
        st.rows(min(x1, x0 + chunk), min(x1, x0 + 2 * chunk), sentinel);
        cp_async_wait<kGroups - 3>();
        st.rows(min(x1, x0 + 2 * chunk), min(x1, x0 + 3 * chunk), sentinel);
        cp_async_wait<0>();
        st.rows(min(x1, x0 + 3 * chunk), x1, sentinel);
    }
    sm.cnt[warp * 32 + lane] = st.top + 1;
    hull_merge(sm, nx);
    if (!live) return;
    int32_t* dst = out + col + (int64_t)x0 * stride;
    hull_output(sm, nx, x0, x1, sentinel, [&](int32_t v) {
        *dst = v;
        dst += stride;
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

// Signed float32 distance of every voxel from the two polarities' squared distances (sq[0]: to the
// nonzero voxels, sq[1]: to the zero voxels).
__global__ void __launch_bounds__(256) k_edt_signed(const int32_t* __restrict__ sq, float* __restrict__ out,
                                                    int64_t size, double pitch, float half) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < size; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = signed_from_pair(sq[i], sq[size + i], pitch, half);
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

// The column passes use more than 48 KB of dynamic shared memory at 512 rows, an opt-in that is a
// per-device function attribute: set once for every device that runs a transform (under a lock,
// since serving threads enqueue transforms concurrently).
constexpr int kMaxDevices = 64;
std::mutex g_configure_lock;
bool g_configured[kMaxDevices] = {};

int configure_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FB_RUNTIME;
    std::lock_guard<std::mutex> guard(g_configure_lock);
    if (g_configured[dev]) return FB_OK;
    FB_CUDA(cudaFuncSetAttribute(k_edt_zy, cudaFuncAttributeMaxDynamicSharedMemorySize, band_smem_bytes(kMaxAxis)));
    FB_CUDA(cudaFuncSetAttribute(k_edt_x, cudaFuncAttributeMaxDynamicSharedMemorySize, band_smem_bytes(kMaxAxis)));
    g_configured[dev] = true;
    return FB_OK;
}

// Enqueue the whole transform on `stream`.  paired == 0: sites are the nonzero mask bytes when
// sites_nonzero, else the zero bytes; writes int32 to out_sq.  paired == 1: both polarities
// (polarity 0 to the nonzero voxels), signed float32 to out_signed, optional squared pair to out_sq.
int enqueue(const uint8_t* d_mask, int nx, int ny, int nz, int paired, int sites_nonzero, double pitch,
            int32_t* out_sq, float* out_signed, void* scratch, int64_t scratch_len, cudaStream_t stream,
            bool count) {
    if (int rc = configure_device()) return rc;
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
    launch_bits(grid0, stream, d_mask, bits, lines, nz, W, count ? counters : nullptr);
    FB_LAUNCH();
    const int32_t sentinel = sentinel_of(nx, ny, nz);
    // Single polarity measuring to zero bytes = the set bits flipped.
    const int invert = paired ? 0 : (sites_nonzero ? 0 : 1);
    k_edt_zy<<<dim3(W, nx, npol), kBandThreads, band_smem_bytes(ny), stream>>>(bits, g, nx, ny, nz, W, invert, sentinel);
    FB_LAUNCH();
    if (paired) {
        // both polarities' x passes into the squared output (or in place), then the signed values
        int32_t* sq = out_sq ? out_sq : g;
        k_edt_x<<<dim3(W, ny, 2), kBandThreads, band_smem_bytes(nx), stream>>>(g, sq, nx, ny, nz, sentinel);
        FB_LAUNCH();
        const int grid = (int)std::min<int64_t>((size + 255) / 256, (int64_t)sms * 16);
        k_edt_signed<<<grid, 256, 0, stream>>>(sq, out_signed, size, pitch, (float)(0.5 * pitch));
    } else {
        k_edt_x<<<dim3(W, ny, 1), kBandThreads, band_smem_bytes(nx), stream>>>(g, out_sq, nx, ny, nz, sentinel);
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
struct NoAllocEntry {
    void* context;  // the driver context the address belongs to
    void* ptr;
};
NoAllocEntry g_noalloc[kNoAllocMaxDevices] = {};

// The current driver context (CUcontext), through the runtime's driver entry point so the library
// does not link libcuda itself; nullptr when it cannot be had.
void* current_context() {
    using GetCurrent = int (*)(void**);
    static GetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<GetCurrent>(f);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

// Device address of the array on the current device, looked up once per device and context.  The
// name g_edt_noalloc_scratch in host code is a host-side stand-in, not a device address, so kernels
// get this pointer instead.  A context torn down and created again (cudaDeviceReset) maps the array
// at a new address: the lookup is keyed on the context and repeated for a new one.
int noalloc_scratch(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return FB_RUNTIME;
    void* ctx = current_context();  // nullptr before the runtime has made a context current
    std::lock_guard<std::mutex> guard(g_noalloc_lock);
    NoAllocEntry& e = g_noalloc[dev];
    if (!e.ptr || !ctx || e.context != ctx) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_edt_noalloc_scratch) != cudaSuccess || !p) return FB_RUNTIME;
        e.ptr = p;
        e.context = ctx ? ctx : current_context();
    }
    *out = e.ptr;
    return FB_OK;
}

}  // namespace

extern "C" {

// Squared EDT exactly as fb_edt_squared_device, with no allocation and no caller scratch: the
// scratch is the library's fixed device array.  Inputs and outputs are the caller's device
// buffers.  Status 0 ok, 1 invalid arguments (a null pointer, an axis below 1), 2 CUDA failure,
// 7 grid beyond the fixed scratch (an axis above 512 or more than 2^20 voxels) -- both rejected
// before anything is enqueued.
// The first call on each device looks the array up (cudaGetSymbolAddress) with that device
// current; make that first call before any stream capture.  The array is shared by every call
// and keeps the last call's contents (nothing in it needs to start at zero: every word a call
// reads it writes first), so calls whose work overlaps on the GPU -- on different streams, or
// from different threads -- race on it and must be serialised by the caller.
int fb_edt_squared_device_noalloc(const uint8_t* d_mask, int nx, int ny, int nz, int sites_nonzero,
                                  int32_t* d_out, void* stream) noexcept {
    if (!d_mask || !d_out || nx < 1 || ny < 1 || nz < 1) return FB_INVALID;
    if (!shape_ok(nx, ny, nz) || (int64_t)nx * ny * nz > kNoAllocVoxels) return FB_NOALLOC_LIMIT;
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
    launch_bits(grid0, s, d_mask, reinterpret_cast<uint32_t*>(base + 256), lines, nz, W,
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
