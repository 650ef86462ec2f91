// Consumers of the EDT: the clearance field in millimetres, the clearance-valid mask, and the free
// space of an occupancy grid as a resistor network (node map, edge lists with conductances from the
// clearance, and the assembled CSR Laplacian).
//
// References (paths relative to the reference project root):
//   src/field_engine/opt/laplaceflode_v1.py:69-97   bygg_gitterlaplacian (node map, per-axis edges,
//                                                   conductance max(0.5 (E_a + E_b) / pitch, 0.1)^p,
//                                                   COO -> CSR with duplicates summed)
//   src/field_engine/opt/laplaceflode_v1.py:313-314 edt_mm = distance_transform_edt(~occ) * pitch
//   src/field_engine/opt/f33_1_topologi_v1.py:205-218 valid = free & (edt_mm >= min_r + margin)
//
// Orders fixed by the reference's arrays, reproduced exactly:
//   * node ids: free voxels in C order (np.arange over fri's True cells);
//   * edges: axis 0, then 1, then 2; inside an axis the edge of voxel p to p + stride in increasing
//     p (C order over the sliced arrays is increasing linear index of the lower voxel);
//   * CSR: columns ascending inside a row, i.e. p - sx, p - sy, p - 1, p, p + 1, p + sy, p + sx;
//     the diagonal is the left-to-right sum of the row's conductances in the order the COO lists
//     them (the node as the lower end of its axis 0, 1, 2 edges, then as the upper end of its
//     axis 0, 1, 2 edges), which is the order scipy's duplicate summation adds them in; a free node
//     without free neighbours has an empty row.
//
// Work split: tiles of 2048 consecutive voxels, 256 threads, 8 rounds of 256 consecutive voxels.
//   k_lat_count  per tile: free voxels, edges per axis, CSR entries;
//   (exclusive scans of the tile counts: nodes, the three edge axes as one array, entries)
//   k_lat_nodes  node map and CSR row starts (block scans of the round's flags);
//   k_lat_emit   edges (u, v, conductance) and CSR entries, reading the node map of the neighbours.
// Every pass reads the 1-byte occupancy; the emit pass the float64 clearance and the node map.
#include "common.cuh"
#include "scan.cuh"

namespace {

constexpr int kLatThreads = 256;
constexpr int kLatRounds = 8;
constexpr int kLatTile = kLatThreads * kLatRounds;
constexpr double kConductanceFloor = 0.1;  // laplaceflode_v1.py KONDUKTANS_GOLV

// Division of 32-bit unsigned integers by an invariant divisor d >= 1 through a multiply
// (Granlund and Montgomery, "Division by invariant integers using multiplication", PLDI 1994):
// s = ceil(log2 d), m = floor(2^32 (2^s - d) / d) + 1, n / d = (mulhi(n, m) + n) >> s for every
// 32-bit n (the sum taken in 64 bits).
struct FastDiv {
    uint32_t d, m;
    int s;
    static FastDiv of(uint32_t d) {
        FastDiv f;
        f.d = d;
        f.s = 0;
        while (f.s < 32 && (uint64_t(1) << f.s) < d) ++f.s;
        f.m = (uint32_t)(((uint64_t(1) << 32) * ((uint64_t(1) << f.s) - d)) / d + 1);
        return f;
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        return (uint32_t)(((uint64_t)__umulhi(n, m) + n) >> s);
    }
};

struct LatGrid {
    int nx, ny, nz;
    int64_t sx, sy, n;  // strides of axes 0 and 1 (axis 2 is contiguous), voxel count
    FastDiv div_sx, div_nz;
};

// Occupancy flags of voxel p: free, free forward neighbours along axes 0/1/2 (the edges p owns as
// their lower end), and the CSR row length (free neighbours + the diagonal when there is one).
struct VoxelFlags {
    uint32_t free, e0, e1, e2, b0, b1, b2, row;
};

__device__ __forceinline__ VoxelFlags voxel_flags(const uint8_t* __restrict__ occ, const LatGrid& g, int64_t p) {
    VoxelFlags f{};
    if (p >= g.n) return f;
    // cell counts stay below 2^31 (the entry points' limit): 32-bit index arithmetic; the seven
    // occupancy bytes are loaded independently of each other
    const uint32_t q = (uint32_t)p, sx = (uint32_t)g.sx, nz = (uint32_t)g.nz;
    const uint32_t x = g.div_sx.div(q), yz = q - x * sx, y = g.div_nz.div(yz), z = yz - y * nz;
    const bool self = occ[q] != 0;
    const bool fx = x + 1 < (uint32_t)g.nx && !occ[q + sx], bx = x > 0 && !occ[q - sx];
    const bool fy = y + 1 < (uint32_t)g.ny && !occ[q + nz], by = y > 0 && !occ[q - nz];
    const bool fz = z + 1 < nz && !occ[q + 1], bz = z > 0 && !occ[q - 1];
    if (self) return f;
    f.free = 1;
    f.e0 = fx;
    f.e1 = fy;
    f.e2 = fz;
    f.b0 = bx;
    f.b1 = by;
    f.b2 = bz;
    const uint32_t deg = f.e0 + f.e1 + f.e2 + f.b0 + f.b1 + f.b2;
    f.row = deg ? deg + 1 : 0;
    return f;
}

// Exclusive scan over the CTA's threads (thread order) of a word of four 16-bit counters; no
// counter's CTA total exceeds 16 bits.  `total` receives the CTA sums.  Every thread calls it.
__device__ __forceinline__ uint64_t block_scan4(uint64_t v, uint64_t* s_warp, uint64_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint64_t base = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kLatThreads / 32; ++w) {
        const uint64_t s = s_warp[w];
        if (w < warp) base += s;
        tot += s;
    }
    __syncthreads();
    total = tot;
    return base + inc - v;
}

__device__ __forceinline__ uint32_t field16(uint64_t w, int k) { return (uint32_t)(w >> (16 * k)) & 0xffffu; }

// Per tile: free voxels -> nodes[t], edges of axis a -> edges[a * tiles + t], CSR entries -> entries[t].
__global__ void __launch_bounds__(kLatThreads) k_lat_count(const uint8_t* __restrict__ occ, LatGrid g, int tiles,
                                                           int32_t* __restrict__ nodes, int32_t* __restrict__ edges,
                                                           int32_t* __restrict__ entries) {
    __shared__ uint64_t s_warp[kLatThreads / 32];
    __shared__ uint32_t s_rows[kLatThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kLatTile;
    uint64_t acc = 0;
    uint32_t rows = 0;
#pragma unroll 2
    for (int r = 0; r < kLatRounds; ++r) {
        const VoxelFlags f = voxel_flags(occ, g, base + r * kLatThreads + threadIdx.x);
        acc += (uint64_t)f.free | ((uint64_t)f.e0 << 16) | ((uint64_t)f.e1 << 32) | ((uint64_t)f.e2 << 48);
        rows += f.row;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, o);
        rows += __shfl_down_sync(0xffffffffu, rows, o);
    }
    if (lane == 0) {
        s_warp[warp] = acc;
        s_rows[warp] = rows;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t a = 0;
        uint32_t rr = 0;
        for (int w = 0; w < kLatThreads / 32; ++w) {
            a += s_warp[w];
            rr += s_rows[w];
        }
        nodes[blockIdx.x] = (int32_t)field16(a, 0);
        edges[blockIdx.x] = (int32_t)field16(a, 1);
        edges[tiles + blockIdx.x] = (int32_t)field16(a, 2);
        edges[2 * tiles + blockIdx.x] = (int32_t)field16(a, 3);
        entries[blockIdx.x] = (int32_t)rr;
    }
}

// Node map (-1 on occupied voxels) and CSR row starts; the thread of the last voxel also closes the
// row pointer array with the entry total.  Row starts beyond the caller's capacity are not written.
__global__ void __launch_bounds__(kLatThreads) k_lat_nodes(const uint8_t* __restrict__ occ, LatGrid g,
                                                           const int32_t* __restrict__ node_base,
                                                           const int32_t* __restrict__ entry_base,
                                                           const int32_t* __restrict__ totals,
                                                           int32_t* __restrict__ node_map,
                                                           int32_t* __restrict__ indptr, int64_t indptr_cap) {
    __shared__ uint64_t s_warp[kLatThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kLatTile;
    int32_t node = node_base[blockIdx.x], entry = entry_base[blockIdx.x];
    for (int r = 0; r < kLatRounds; ++r) {
        const int64_t p = base + r * kLatThreads + threadIdx.x;
        const VoxelFlags f = voxel_flags(occ, g, p);
        uint64_t tot;
        const uint64_t pre = block_scan4((uint64_t)f.free | ((uint64_t)f.row << 16), s_warp, tot);
        if (p < g.n) {
            const int32_t id = node + (int32_t)field16(pre, 0);
            node_map[p] = f.free ? id : -1;
            if (f.free && id < indptr_cap) indptr[id] = entry + (int32_t)field16(pre, 1);
            if (p == g.n - 1 && totals[0] < indptr_cap) indptr[totals[0]] = totals[2];
        }
        node += (int32_t)field16(tot, 0);
        entry += (int32_t)field16(tot, 1);
    }
}

// Conductance of the edge between cells a < b from their clearances, max(0.5 (E_a + E_b) / pitch,
// 0.1)^p, in the reference's operation order (NaN propagates through the max as in np.maximum).
// The reference's exponent 1.5 is m * sqrt(m) (correctly rounded root, one rounding of the product:
// within 2 ulp of libm's pow, as CUDA's pow is), 0 and 1 are exact; other exponents call pow.
__device__ __forceinline__ double conductance(double ea, double eb, double pitch, double p_kond) {
    const double c = __ddiv_rn(__dmul_rn(0.5, __dadd_rn(ea, eb)), pitch);
    const double m = (c != c) ? c : (c > kConductanceFloor ? c : kConductanceFloor);
    if (p_kond == 1.5) return __dmul_rn(m, __dsqrt_rn(m));
    if (p_kond == 1.0) return m;
    if (p_kond == 0.0) return 1.0;
    return pow(m, p_kond);
}

// Edges (u, v, conductance; axis-major, lower voxel ascending) and the CSR entries of every free
// voxel's row.  Each round's outputs are placed in shared memory at their block-scan offsets and
// then written out as contiguous runs, so every store instruction writes whole sectors.  Neighbour
// ids along the contiguous axis follow from the cell's own (free cells are numbered in C order).
constexpr int kLatRowMax = 7;

__global__ void __launch_bounds__(kLatThreads, 4) k_lat_emit(const uint8_t* __restrict__ occ,
                                                             const double* __restrict__ edt_mm, LatGrid g,
                                                             double pitch, double p_kond, int tiles,
                                                             const int32_t* __restrict__ edge_base,
                                                             const int32_t* __restrict__ entry_base,
                                                             const int32_t* __restrict__ node_map,
                                                             int32_t* __restrict__ u, int32_t* __restrict__ v,
                                                             double* __restrict__ kond, int64_t edge_cap,
                                                             int32_t* __restrict__ indices, double* __restrict__ data,
                                                             int64_t entry_cap) {
    __shared__ uint64_t s_warp[kLatThreads / 32];
    __shared__ double s_val[kLatThreads * kLatRowMax];
    __shared__ int32_t s_idx[kLatThreads * kLatRowMax];
    __shared__ double s_ek[3][kLatThreads];
    __shared__ int32_t s_eu[3][kLatThreads];
    __shared__ int32_t s_ev[3][kLatThreads];
    const int64_t base = (int64_t)blockIdx.x * kLatTile;
    int32_t eb[3] = {edge_base[blockIdx.x], edge_base[tiles + blockIdx.x], edge_base[2 * tiles + blockIdx.x]};
    int32_t cb = entry_base[blockIdx.x];
    for (int r = 0; r < kLatRounds; ++r) {
        const int64_t p = base + r * kLatThreads + threadIdx.x;
        const VoxelFlags f = voxel_flags(occ, g, p);
        // every load of the cell's row is issued before the round's block scan, so its latency
        // overlaps the scan's barriers
        double ec = 0.0, exp_ = 0.0, eyp = 0.0, ezp = 0.0, exm = 0.0, eym = 0.0, ezm = 0.0;
        int32_t id = 0, nxp = 0, nyp = 0, nxm = 0, nym = 0;
        if (f.free) {
            ec = edt_mm[p];
            id = node_map[p];
            if (f.e0) { exp_ = edt_mm[p + g.sx]; nxp = node_map[p + g.sx]; }
            if (f.e1) { eyp = edt_mm[p + g.sy]; nyp = node_map[p + g.sy]; }
            if (f.e2) ezp = edt_mm[p + 1];
            if (f.b0) { exm = edt_mm[p - g.sx]; nxm = node_map[p - g.sx]; }
            if (f.b1) { eym = edt_mm[p - g.sy]; nym = node_map[p - g.sy]; }
            if (f.b2) ezm = edt_mm[p - 1];
        }
        uint64_t tot;
        const uint64_t pre = block_scan4((uint64_t)f.e0 | ((uint64_t)f.e1 << 16) | ((uint64_t)f.e2 << 32) |
                                             ((uint64_t)f.row << 48),
                                         s_warp, tot);
        if (f.free) {
            // conductances: forward edges (the cell is the lower end), then backward ones
            const double kf0 = f.e0 ? conductance(ec, exp_, pitch, p_kond) : 0.0;
            const double kf1 = f.e1 ? conductance(ec, eyp, pitch, p_kond) : 0.0;
            const double kf2 = f.e2 ? conductance(ec, ezp, pitch, p_kond) : 0.0;
            const double kb0 = f.b0 ? conductance(exm, ec, pitch, p_kond) : 0.0;
            const double kb1 = f.b1 ? conductance(eym, ec, pitch, p_kond) : 0.0;
            const double kb2 = f.b2 ? conductance(ezm, ec, pitch, p_kond) : 0.0;
            if (f.e0) {
                const int k = (int)field16(pre, 0);
                s_eu[0][k] = id;
                s_ev[0][k] = nxp;
                s_ek[0][k] = kf0;
            }
            if (f.e1) {
                const int k = (int)field16(pre, 1);
                s_eu[1][k] = id;
                s_ev[1][k] = nyp;
                s_ek[1][k] = kf1;
            }
            if (f.e2) {
                const int k = (int)field16(pre, 2);
                s_eu[2][k] = id;
                s_ev[2][k] = id + 1;
                s_ek[2][k] = kf2;
            }
            if (f.row) {
                // diagonal in the COO's order: lower-end edges of axes 0, 1, 2, then upper-end ones
                // (an absent edge adds 0.0, which leaves the sum's bits unchanged: every term is
                // positive or NaN)
                const double diag = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(kf0, kf1), kf2), kb0), kb1), kb2);
                int k = (int)field16(pre, 3);
                if (f.b0) { s_idx[k] = nxm; s_val[k++] = -kb0; }
                if (f.b1) { s_idx[k] = nym; s_val[k++] = -kb1; }
                if (f.b2) { s_idx[k] = id - 1; s_val[k++] = -kb2; }
                s_idx[k] = id;
                s_val[k++] = diag;
                if (f.e2) { s_idx[k] = id + 1; s_val[k++] = -kf2; }
                if (f.e1) { s_idx[k] = nyp; s_val[k++] = -kf1; }
                if (f.e0) { s_idx[k] = nxp; s_val[k] = -kf0; }
            }
        }
        __syncthreads();
        const int ne0 = (int)field16(tot, 0), ne1 = (int)field16(tot, 1), ne2 = (int)field16(tot, 2);
        const int nrow = (int)field16(tot, 3);
        // outputs beyond the caller's capacities are not written
        for (int i = threadIdx.x; i < nrow; i += kLatThreads) {
            if ((int64_t)cb + i >= entry_cap) break;
            indices[cb + i] = s_idx[i];
            data[cb + i] = s_val[i];
        }
        for (int a = 0; a < 3; ++a) {
            const int ne = a == 0 ? ne0 : (a == 1 ? ne1 : ne2);
            for (int i = threadIdx.x; i < ne; i += kLatThreads) {
                if ((int64_t)eb[a] + i >= edge_cap) break;
                u[eb[a] + i] = s_eu[a][i];
                v[eb[a] + i] = s_ev[a][i];
                kond[eb[a] + i] = s_ek[a][i];
            }
        }
        __syncthreads();
        eb[0] += ne0;
        eb[1] += ne1;
        eb[2] += ne2;
        cb += nrow;
    }
}

// Clearance in millimetres from the squared voxel distance: float64(sqrt(sq)) * pitch, the value of
// scipy's distance_transform_edt (float64 root of the exact integer sum of squares) times the pitch.
__global__ void k_edt_mm(const int32_t* __restrict__ sq, int64_t n, double pitch, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __dmul_rn(__dsqrt_rn((double)sq[i]), pitch);
}

// valid = free & (edt_mm >= threshold), threshold = min_r + margin formed by the caller in float64.
__global__ void k_clearance_mask(const uint8_t* __restrict__ occ, const double* __restrict__ edt_mm, int64_t n,
                                 double threshold, uint8_t* __restrict__ valid) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        valid[i] = (!occ[i] && edt_mm[i] >= threshold) ? 1 : 0;
}

// Voxel limit: node ids, edge indices and CSR offsets are int32, and a row holds at most 7 entries.
constexpr int64_t kLatMaxVoxels = (int64_t)INT32_MAX / 7;

bool lat_shape(int nx, int ny, int nz, LatGrid& g) {
    if (nx < 1 || ny < 1 || nz < 1) return false;
    const int64_t n = (int64_t)nx * ny * nz;
    if (n > kLatMaxVoxels) return false;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.sy = nz;
    g.sx = (int64_t)ny * nz;
    g.n = n;
    g.div_sx = FastDiv::of((uint32_t)g.sx);
    g.div_nz = FastDiv::of((uint32_t)nz);
    return true;
}

// Scratch: per-tile counts (nodes, 3 x edges, entries), three totals, the scans' own words.
struct LatScratch {
    int32_t *nodes, *edges, *entries, *totals, *scan;
    int64_t scan_words;
};

int64_t lat_scratch_words(int64_t tiles) { return 5 * tiles + 3 + scan_scratch_words(3 * tiles); }

LatScratch lat_scratch(void* base, int64_t tiles) {
    LatScratch s;
    s.nodes = static_cast<int32_t*>(base);
    s.edges = s.nodes + tiles;
    s.entries = s.edges + 3 * tiles;
    s.totals = s.entries + tiles;
    s.scan = s.totals + 3;
    s.scan_words = scan_scratch_words(3 * tiles);
    return s;
}

int grid_blocks(int64_t n) {
    const int64_t cap = (int64_t)fb_sm_count() * 8;
    const int64_t want = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min(cap, want));
}

}  // namespace

extern "C" {

int64_t fb_lattice_scratch_bytes(int nx, int ny, int nz) {
    LatGrid g;
    if (!lat_shape(nx, ny, nz, g)) return -1;
    const int64_t tiles = (g.n + kLatTile - 1) / kLatTile;
    return 4 * lat_scratch_words(tiles);
}

int fb_lattice_count_device(const uint8_t* d_occ, int nx, int ny, int nz, int32_t* d_totals, void* d_scratch,
                            int64_t scratch_len, void* stream) noexcept {
    LatGrid g;
    if (!d_occ || !d_totals || !d_scratch || !lat_shape(nx, ny, nz, g)) return FB_INVALID;
    const int64_t tiles = (g.n + kLatTile - 1) / kLatTile;
    if (scratch_len < 4 * lat_scratch_words(tiles)) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const LatScratch s = lat_scratch(d_scratch, tiles);
    k_lat_count<<<(unsigned)tiles, kLatThreads, 0, st>>>(d_occ, g, (int)tiles, s.nodes, s.edges, s.entries);
    FB_LAUNCH();
    if (int rc = scan_exclusive(s.nodes, tiles, s.totals + 0, s.scan, s.scan_words, st)) return rc;
    if (int rc = scan_exclusive(s.edges, 3 * tiles, s.totals + 1, s.scan, s.scan_words, st)) return rc;
    if (int rc = scan_exclusive(s.entries, tiles, s.totals + 2, s.scan, s.scan_words, st)) return rc;
    FB_CUDA(cudaMemcpyAsync(d_totals, s.totals, 3 * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    return FB_OK;
}

int fb_lattice_emit_device(const uint8_t* d_occ, const double* d_edt_mm, int nx, int ny, int nz, double pitch,
                           double p_kond, int32_t* d_node_map, int32_t* d_u, int32_t* d_v, double* d_kond,
                           int64_t edge_cap, int32_t* d_indptr, int64_t indptr_cap, int32_t* d_indices,
                           double* d_data, int64_t entry_cap, const void* d_scratch, int64_t scratch_len,
                           void* stream) noexcept {
    LatGrid g;
    if (!d_occ || !d_edt_mm || !d_node_map || !d_scratch || !lat_shape(nx, ny, nz, g)) return FB_INVALID;
    if (edge_cap < 0 || indptr_cap < 1 || entry_cap < 0 || !d_indptr) return FB_INVALID;
    if (edge_cap > 0 && (!d_u || !d_v || !d_kond)) return FB_INVALID;
    if (entry_cap > 0 && (!d_indices || !d_data)) return FB_INVALID;
    const int64_t tiles = (g.n + kLatTile - 1) / kLatTile;
    if (scratch_len < 4 * lat_scratch_words(tiles)) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const LatScratch s = lat_scratch(const_cast<void*>(d_scratch), tiles);
    k_lat_nodes<<<(unsigned)tiles, kLatThreads, 0, st>>>(d_occ, g, s.nodes, s.entries, s.totals, d_node_map,
                                                           d_indptr, indptr_cap);
    FB_LAUNCH();
    k_lat_emit<<<(unsigned)tiles, kLatThreads, 0, st>>>(d_occ, d_edt_mm, g, pitch, p_kond, (int)tiles, s.edges,
                                                          s.entries, d_node_map, d_u, d_v, d_kond, edge_cap, d_indices,
                                                          d_data, entry_cap);
    FB_LAUNCH();
    return FB_OK;
}

int fb_edt_mm_device(const int32_t* d_sq, int64_t n, double pitch, double* d_out, void* stream) noexcept {
    if (!d_sq || !d_out || n < 0) return FB_INVALID;
    if (n == 0) return FB_OK;
    k_edt_mm<<<grid_blocks(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_sq, n, pitch, d_out);
    FB_LAUNCH();
    return FB_OK;
}

int fb_clearance_mask_device(const uint8_t* d_occ, const double* d_edt_mm, int64_t n, double threshold,
                             uint8_t* d_valid, void* stream) noexcept {
    if (!d_occ || !d_edt_mm || !d_valid || n < 0) return FB_INVALID;
    if (n == 0) return FB_OK;
    k_clearance_mask<<<grid_blocks(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_occ, d_edt_mm, n, threshold,
                                                                                      d_valid);
    FB_LAUNCH();
    return FB_OK;
}

}  // extern "C"
