// Packed adaptive fields on sm_100a: lossless packing with the reference's split decisions, exact
// unpacking, ordered CSG over sampled fields, and point queries on packed fields.
//
// Packing (src/field_engine/adaptive_pack_native_v1/pack.cpp:18-69, adaptive_sample_blocks_v1.py:19-58):
//   the candidate tree is expanded level by level.  For every candidate region one launch of
//   k_pack_flags computes, per axis, whether all samples are bitwise equal to the sample with that
//   coordinate at the region's low edge (chunks of 8192 samples per CTA, atomicAnd into the
//   region's three flags).  The host then applies the reference's rules -- leaf when the reduced
//   size is <= 64 or the region holds <= threshold samples, otherwise split the varying axis with
//   the largest extent at extent/2 -- keeps a split only if 52 + cost(left) + cost(right) is below
//   the leaf cost (bottom-up), flattens depth-first (left before right) and k_pack_payload copies
//   each leaf's reduced samples bit for bit.
// Unpacking + CSG (src/field_engine/csg_batch_native_v1/execute.cpp:10-53, csg_tile_native_v1/
//   gather.cpp:11-49): every used operand is expanded to a dense device array (a coverage count
//   detects overlaps and gaps, code 4), then k_csg_program evaluates the ordered program per
//   voxel with the NumPy tie rule (the second operand wins on equality) and float64 offsets.
// Queries (adaptive_sample_blocks_v1.py:103-151): tree descent per index, then the eight-sample
//   trilinear interpolation of scipy.ndimage.map_coordinates(order=1, mode='nearest').
#include "common.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#pragma pack(push, 1)
struct PackNode {  // 52-byte record of the reference (pack.cpp:7-10)
    int32_t lo[3], shape[3], stored[3], children[2];
    int64_t offset;
};
#pragma pack(pop)
static_assert(sizeof(PackNode) == 52, "packed node layout");

struct CsgInsn {  // 24-byte record of the reference (execute.cpp:8-9)
    int32_t op, left, right, pad;
    double offset;
};
static_assert(sizeof(CsgInsn) == 24, "CSG instruction layout");

namespace {

constexpr int kChunk = 8192;

struct Region {
    int lo[3], shape[3];
};

// ------------------------------------------------------------------------------------------ pack
// flags[r] bit a = 1 while every sample equals the one at coordinate 0 along axis a.
__global__ void __launch_bounds__(256) k_pack_flags(const uint32_t* __restrict__ data, int64_t s0, int64_t s1,
                                                    const Region* __restrict__ regions,
                                                    const int64_t* __restrict__ chunk_start, int nregions,
                                                    unsigned* __restrict__ flags) {
    // chunk_start[r] = first global chunk of region r (exclusive prefix); find r by binary search
    const int64_t chunk = blockIdx.x;
    int lo = 0, hi = nregions - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (chunk_start[mid] <= chunk) lo = mid; else hi = mid - 1;
    }
    const int r = lo;
    const Region R = regions[r];
    const int64_t count = (int64_t)R.shape[0] * R.shape[1] * R.shape[2];
    const int64_t first = (chunk - chunk_start[r]) * kChunk;
    const int64_t last = min(first + kChunk, count);
    unsigned ok = 7u;
    const int64_t syz = (int64_t)R.shape[1] * R.shape[2];
    for (int64_t e = first + threadIdx.x; e < last; e += blockDim.x) {
        const int x = (int)(e / syz), y = (int)((e / R.shape[2]) % R.shape[1]), z = (int)(e % R.shape[2]);
        const int64_t X = R.lo[0] + x, Y = R.lo[1] + y, Z = R.lo[2] + z;
        const uint32_t v = data[X * s0 + Y * s1 + Z];
        if (v != data[(int64_t)R.lo[0] * s0 + Y * s1 + Z]) ok &= ~1u;
        if (v != data[X * s0 + (int64_t)R.lo[1] * s1 + Z]) ok &= ~2u;
        if (v != data[X * s0 + Y * s1 + R.lo[2]]) ok &= ~4u;
    }
    ok = __reduce_and_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31) == 0 && ok != 7u) atomicAnd(&flags[r], ok);
}

// Non-finite check of the dense input (the reference rejects NaN / Inf bit patterns).
__global__ void k_pack_finite(const uint32_t* __restrict__ data, int64_t n, int* bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if ((data[i] & 0x7f800000u) == 0x7f800000u) { *bad = 1; return; }
}

struct LeafCopy {
    int lo[3], stored[3];
    int64_t offset;
};

// payload[offset + i] = the i-th sample of the leaf's reduced box (C order, bit copy).
__global__ void __launch_bounds__(256) k_pack_payload(const uint32_t* __restrict__ data, int64_t s0, int64_t s1,
                                                      const LeafCopy* __restrict__ leaves, int nleaves,
                                                      int64_t total, uint32_t* __restrict__ payload) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nleaves - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (leaves[mid].offset <= i) lo = mid; else hi = mid - 1;
        }
        const LeafCopy L = leaves[lo];
        const int64_t k = i - L.offset;
        const int z = (int)(k % L.stored[2]), y = (int)((k / L.stored[2]) % L.stored[1]);
        const int x = (int)(k / ((int64_t)L.stored[2] * L.stored[1]));
        payload[i] = data[(int64_t)(L.lo[0] + x) * s0 + (int64_t)(L.lo[1] + y) * s1 + (L.lo[2] + z)];
    }
}

struct Packed {
    std::vector<PackNode> nodes;
    std::vector<uint32_t> payload;   // host copy (filled by adaptive_copy / on demand)
    uint32_t* d_payload = nullptr;   // device copy
    int64_t n_payload = 0;
    bool host_ready = false;
};

struct Cand {
    Region r;
    int stored[3];
    int64_t cost;
    int left = -1, right = -1;  // candidate children
    bool split = false;          // kept split after the bottom-up pass
};

int pack_device(const uint32_t* d_data, const int32_t* shape, int threshold, cudaStream_t st, Packed& out) {
    const int64_t s1 = shape[2], s0 = (int64_t)shape[1] * shape[2];
    std::vector<Cand> cands;
    Cand root;
    for (int a = 0; a < 3; ++a) {
        root.r.lo[a] = 0;
        root.r.shape[a] = shape[a];
    }
    cands.push_back(root);
    std::vector<int> level = {0};
    Region* d_regions = nullptr;
    int64_t* d_chunks = nullptr;
    unsigned* d_flags = nullptr;
    size_t cap = 0;
    int status = FB_OK;
    while (!level.empty() && status == FB_OK) {
        const int n = (int)level.size();
        std::vector<Region> regions(n);
        std::vector<int64_t> chunks(n);
        int64_t total_chunks = 0;
        for (int i = 0; i < n; ++i) {
            regions[i] = cands[level[i]].r;
            const int64_t count = (int64_t)regions[i].shape[0] * regions[i].shape[1] * regions[i].shape[2];
            chunks[i] = total_chunks;
            total_chunks += (count + kChunk - 1) / kChunk;
        }
        if ((size_t)n > cap) {
            if (d_regions) cudaFreeAsync(d_regions, st);
            if (d_chunks) cudaFreeAsync(d_chunks, st);
            if (d_flags) cudaFreeAsync(d_flags, st);
            cap = std::max<size_t>(n, 2 * cap);
            if (cudaMallocAsync(&d_regions, cap * sizeof(Region), st) != cudaSuccess ||
                cudaMallocAsync(&d_chunks, cap * sizeof(int64_t), st) != cudaSuccess ||
                cudaMallocAsync(&d_flags, cap * sizeof(unsigned), st) != cudaSuccess) {
                status = FB_RUNTIME;
                break;
            }
        }
        std::vector<unsigned> flags(n, 7u);
        if (cudaMemcpyAsync(d_regions, regions.data(), n * sizeof(Region), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(d_chunks, chunks.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(d_flags, flags.data(), n * sizeof(unsigned), cudaMemcpyHostToDevice, st) != cudaSuccess) {
            status = FB_RUNTIME;
            break;
        }
        k_pack_flags<<<(unsigned)total_chunks, 256, 0, st>>>(d_data, s0, s1, d_regions, d_chunks, n, d_flags);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(flags.data(), d_flags, n * sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            status = FB_RUNTIME;
            break;
        }
        std::vector<int> next;
        for (int i = 0; i < n; ++i) {
            Cand& c = cands[level[i]];
            int64_t count = 1, reduced = 1;
            for (int a = 0; a < 3; ++a) {
                c.stored[a] = (flags[i] >> a) & 1u ? 1 : c.r.shape[a];
                count *= c.r.shape[a];
                reduced *= c.stored[a];
            }
            c.cost = (int64_t)sizeof(PackNode) + 4 * reduced;
            if (reduced <= 64 || count <= threshold) continue;
            int axis = -1;
            for (int a = 0; a < 3; ++a)
                if (c.stored[a] > 1 && (axis < 0 || c.r.shape[a] > c.r.shape[axis])) axis = a;
            if (axis < 0) continue;
            Cand L, R;
            L.r = c.r;
            R.r = c.r;
            L.r.shape[axis] = c.r.shape[axis] / 2;
            R.r.shape[axis] = c.r.shape[axis] - L.r.shape[axis];
            R.r.lo[axis] += L.r.shape[axis];
            const int li = (int)cands.size();
            cands.push_back(L);
            cands.push_back(R);
            cands[level[i]].left = li;  // `c` may be invalidated by push_back
            cands[level[i]].right = li + 1;
            next.push_back(li);
            next.push_back(li + 1);
        }
        level.swap(next);
    }
    if (d_regions) cudaFreeAsync(d_regions, st);
    if (d_chunks) cudaFreeAsync(d_chunks, st);
    if (d_flags) cudaFreeAsync(d_flags, st);
    if (status) return status;
    // bottom-up: children were appended after their parent, so a reverse sweep sees them first
    for (int i = (int)cands.size() - 1; i >= 0; --i) {
        Cand& c = cands[i];
        if (c.left < 0) continue;
        const int64_t split = (int64_t)sizeof(PackNode) + cands[c.left].cost + cands[c.right].cost;
        if (split < c.cost) {
            c.cost = split;
            c.split = true;
        }
    }
    // flatten depth-first, left before right
    out.nodes.clear();
    std::vector<LeafCopy> leaves;
    int64_t offset = 0;
    std::vector<std::pair<int, int>> stack;  // (candidate, node slot to fill)
    struct Frame { int cand; int slot; int state; };
    std::vector<Frame> frames;
    frames.push_back({0, -1, 0});
    // iterative pre-order with post-fix of the children indices
    std::vector<int> slot_of(cands.size(), -1);
    std::vector<int> order;
    {
        std::vector<int> todo = {0};
        while (!todo.empty()) {
            const int ci = todo.back();
            todo.pop_back();
            slot_of[ci] = (int)order.size();
            order.push_back(ci);
            const Cand& c = cands[ci];
            if (c.split) {
                todo.push_back(c.right);
                todo.push_back(c.left);
            }
        }
    }
    out.nodes.resize(order.size());
    for (size_t k = 0; k < order.size(); ++k) {
        const Cand& c = cands[order[k]];
        PackNode node;
        std::memset(&node, 0, sizeof(node));
        for (int a = 0; a < 3; ++a) {
            node.lo[a] = c.r.lo[a];
            node.shape[a] = c.r.shape[a];
        }
        if (c.split) {
            node.offset = -1;
            node.children[0] = slot_of[c.left];
            node.children[1] = slot_of[c.right];
        } else {
            node.offset = offset;
            node.children[0] = node.children[1] = -1;
            LeafCopy lc;
            for (int a = 0; a < 3; ++a) {
                node.stored[a] = c.stored[a];
                lc.lo[a] = c.r.lo[a];
                lc.stored[a] = c.stored[a];
            }
            lc.offset = offset;
            leaves.push_back(lc);
            offset += (int64_t)c.stored[0] * c.stored[1] * c.stored[2];
        }
        out.nodes[k] = node;
    }
    out.n_payload = offset;
    LeafCopy* d_leaves = nullptr;
    if (cudaMallocAsync(&out.d_payload, std::max<int64_t>(offset, 1) * 4, st) != cudaSuccess ||
        cudaMallocAsync(&d_leaves, std::max<size_t>(leaves.size(), 1) * sizeof(LeafCopy), st) != cudaSuccess ||
        cudaMemcpyAsync(d_leaves, leaves.data(), leaves.size() * sizeof(LeafCopy), cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
        status = FB_RUNTIME;
    if (!status) {
        const int grid = (int)std::min<int64_t>((offset + 255) / 256, (int64_t)fb_sm_count() * 16);
        k_pack_payload<<<std::max(grid, 1), 256, 0, st>>>(d_data, s0, s1, d_leaves, (int)leaves.size(), offset,
                                                         out.d_payload);
        if (cudaGetLastError() != cudaSuccess) status = FB_RUNTIME;
    }
    if (d_leaves) cudaFreeAsync(d_leaves, st);
    if (!status && cudaStreamSynchronize(st) != cudaSuccess) status = FB_RUNTIME;
    return status;
}

bool pack_args_ok(const int32_t* shape, int threshold) {
    if (!shape || threshold < 8 || threshold > 4096) return false;
    int64_t total = 1;
    for (int a = 0; a < 3; ++a) {
        if (shape[a] < 1 || shape[a] > 4096) return false;
        total *= shape[a];
    }
    return total <= 16777216;
}

// ------------------------------------------------------------------------------------------ unpack
// Operand sanity exactly as the reference's gather (gather.cpp:11-30): its argument bounds and every
// leaf's box and payload range.  Any failure of the gather is status 3 of csg_execute
// (execute.cpp:28), and these checks fail on the first tile, before any output is written.
int check_nodes(const PackNode* nodes, const void* payload, int64_t count, int64_t samples, const int32_t* shape) {
    if (!nodes || !payload || count < 1 || count > 33554432 || samples < 1 || samples > 16777216) return 3;
    for (int64_t n = 0; n < count; ++n) {
        const PackNode& node = nodes[n];
        if (node.children[0] >= 0) continue;
        int64_t size = 1;
        for (int a = 0; a < 3; ++a) {
            if (node.lo[a] < 0 || node.shape[a] < 1 || node.shape[a] > 4096 || node.lo[a] > 4096 - node.shape[a] ||
                (node.stored[a] != 1 && node.stored[a] != node.shape[a]))
                return 3;
            size *= node.stored[a];
        }
        if (node.offset < 0 || size > samples || node.offset > samples - size) return 3;
        (void)shape;
    }
    return 0;
}

// Dense expansion of the leaves: one thread per sample of each leaf's full (unreduced) box, the
// parts inside the grid only; `cover` counts the writes per voxel (overlap / gap detection).
__global__ void __launch_bounds__(256) k_unpack(const PackNode* __restrict__ nodes, const int64_t* __restrict__ leaf_ids,
                                                const int64_t* __restrict__ leaf_start, int nleaves, int64_t total,
                                                const uint32_t* __restrict__ payload, int sx, int sy, int sz,
                                                uint32_t* __restrict__ dense, unsigned* __restrict__ cover) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nleaves - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (leaf_start[mid] <= i) lo = mid; else hi = mid - 1;
        }
        const PackNode N = nodes[leaf_ids[lo]];
        const int64_t k = i - leaf_start[lo];
        const int z = (int)(k % N.shape[2]), y = (int)((k / N.shape[2]) % N.shape[1]);
        const int x = (int)(k / ((int64_t)N.shape[2] * N.shape[1]));
        const int X = N.lo[0] + x, Y = N.lo[1] + y, Z = N.lo[2] + z;
        if (X >= sx || Y >= sy || Z >= sz) continue;
        const int64_t src = N.offset + ((int64_t)(N.stored[0] == 1 ? 0 : x) * N.stored[1] + (N.stored[1] == 1 ? 0 : y)) *
                                           N.stored[2] + (N.stored[2] == 1 ? 0 : z);
        const int64_t dst = ((int64_t)X * sy + Y) * sz + Z;
        dense[dst] = payload[src];
        atomicAdd(&cover[dst], 1u);
    }
}

// The reference's csg_execute walks the grid in tiles of 16 x 32 x 16 voxels (x outermost) and stops
// at the first tile where a gather or a result fails, after writing every earlier tile.  A failure
// is recorded as the key 2 * tile + (0 gather, 1 non-finite result); the smallest key over all
// voxels is the reference's stopping point and status (a gather failure precedes the instructions
// of its own tile).
__device__ __forceinline__ unsigned long long csg_tile_of(int64_t v, int sy, int sz) {
    const int64_t x = v / ((int64_t)sy * sz), y = (v / sz) % sy, z = v % sz;
    const int64_t nty = (sy + 31) / 32, ntz = (sz + 15) / 16;
    return (unsigned long long)(((x / 16) * nty + y / 32) * ntz + z / 16);
}

// Voxels covered by no leaf or by several (the gather's gap / overlap) fail their tile's gather.
__global__ void k_cover_check(const unsigned* __restrict__ cover, int64_t n, int sy, int sz,
                              unsigned long long* __restrict__ fail) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (cover[i] != 1u) atomicMin(fail, 2ull * csg_tile_of(i, sy, sz));
}

// ------------------------------------------------------------------------------------------ CSG
// Per-voxel program.  Operands are input fields (read from their dense arrays, operand -1 - f) or
// intermediate slots (operand >= 0); a slot is reused after its value's last use (host allocation),
// so a left-deep chain needs two slots whatever its length.  Programs with up to kLocalSlots live
// intermediates keep them in a per-thread array; larger ones in a global array [slot][voxel]
// (coalesced across the warp), so every program the reference accepts (256 inputs, 1024
// instructions) runs.
struct CsgStep {
    int32_t op, a, b, dst;  // op 0 union, 1 difference, 2 offset
    double offset;
};
constexpr int kLocalSlots = 32;

template <bool kGlobal>
__device__ __forceinline__ float csg_read(const float* const* __restrict__ inputs, const float* slot,
                                          const float* __restrict__ gslots, int64_t n, int64_t v, int operand) {
    if (operand < 0) return inputs[-1 - operand][v];
    return kGlobal ? gslots[operand * n + v] : slot[operand];
}

template <bool kGlobal>
__global__ void __launch_bounds__(256) k_csg_program(const float* const* __restrict__ inputs,
                                                     const CsgStep* __restrict__ prog, int n_prog, int result,
                                                     int64_t n, int sy, int sz, float* __restrict__ out,
                                                     float* __restrict__ gslots, unsigned long long* __restrict__ fail) {
    extern __shared__ CsgStep s_prog[];
    for (int i = threadIdx.x; i < n_prog; i += blockDim.x) s_prog[i] = prog[i];
    __syncthreads();
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        float slot[kGlobal ? 1 : kLocalSlots];
        bool finite = true;
        float r = 0.f;
        for (int i = 0; i < n_prog; ++i) {
            const CsgStep I = s_prog[i];
            const float a = csg_read<kGlobal>(inputs, slot, gslots, n, v, I.a);
            if (I.op == 2) {
                r = __double2float_rn(__dsub_rn((double)a, I.offset));
            } else {
                const float b0 = csg_read<kGlobal>(inputs, slot, gslots, n, v, I.b);
                const float b = I.op == 0 ? b0 : -b0;
                // NumPy's minimum / maximum keep the second operand on equality, signed zeros included
                r = I.op == 0 ? (a < b ? a : b) : (a > b ? a : b);
            }
            finite &= isfinite(r);
            if (kGlobal) gslots[I.dst * n + v] = r;
            else slot[I.dst] = r;
        }
        if (!finite) atomicMin(fail, 2ull * csg_tile_of(v, sy, sz) + 1ull);
        out[v] = kGlobal ? gslots[result * n + v] : slot[result];
    }
}

// ------------------------------------------------------------------------------------------ query
// Sample bits at integer indices by descending the packed tree (adaptive_sample_blocks_v1.py:103-128).
__device__ __forceinline__ float tree_sample(const PackNode* __restrict__ nodes, const float* __restrict__ payload,
                                             int x, int y, int z) {
    int id = 0;
    for (int depth = 0; depth < 64; ++depth) {
        const PackNode N = nodes[id];
        if (N.children[0] < 0) {
            const int lx = N.stored[0] == 1 ? 0 : x - N.lo[0];
            const int ly = N.stored[1] == 1 ? 0 : y - N.lo[1];
            const int lz = N.stored[2] == 1 ? 0 : z - N.lo[2];
            return payload[N.offset + ((int64_t)lx * N.stored[1] + ly) * N.stored[2] + lz];
        }
        const PackNode L = nodes[N.children[0]];
        const bool in_left = x >= L.lo[0] && x < L.lo[0] + L.shape[0] && y >= L.lo[1] && y < L.lo[1] + L.shape[1] &&
                             z >= L.lo[2] && z < L.lo[2] + L.shape[2];
        id = in_left ? N.children[0] : N.children[1];
    }
    return __int_as_float(0x7fc00000);
}

__global__ void k_samples_at(const PackNode* __restrict__ nodes, const float* __restrict__ payload,
                             const int64_t* __restrict__ idx, int64_t n, float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = tree_sample(nodes, payload, (int)idx[3 * i], (int)idx[3 * i + 1], (int)idx[3 * i + 2]);
}

// Trilinear value at float64 points: coordinates (p - origin) / pitch clipped to [0, n-1], the eight
// samples of the cell (indices clamped to n-1), weights (1-f, f) per axis accumulated in float64 in
// the order scipy.ndimage.map_coordinates(order=1) uses (value x w0 x w1 x w2, C order over the
// 2x2x2 corners), rounded once to float32.
__global__ void k_query(const PackNode* __restrict__ nodes, const float* __restrict__ payload, int sx, int sy, int sz,
                        double ox, double oy, double oz, double pitch, const double* __restrict__ pts, int64_t n,
                        float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double c[3] = {__ddiv_rn(__dsub_rn(pts[3 * i], ox), pitch), __ddiv_rn(__dsub_rn(pts[3 * i + 1], oy), pitch),
                       __ddiv_rn(__dsub_rn(pts[3 * i + 2], oz), pitch)};
        const int n3[3] = {sx, sy, sz};
        int lo[3];
        double f[3];
        for (int a = 0; a < 3; ++a) {
            c[a] = fmin(fmax(c[a], 0.0), (double)(n3[a] - 1));
            const double fl = floor(c[a]);
            lo[a] = (int)fl;
            f[a] = __dsub_rn(c[a], fl);
        }
        double t = 0.0;
        for (int h = 0; h < 8; ++h) {
            const int a = (h >> 2) & 1, b = (h >> 1) & 1, d = h & 1;
            const int X = min(lo[0] + a, sx - 1), Y = min(lo[1] + b, sy - 1), Z = min(lo[2] + d, sz - 1);
            double coeff = (double)tree_sample(nodes, payload, X, Y, Z);
            coeff = __dmul_rn(coeff, 1.0);
            coeff = __dmul_rn(coeff, a ? f[0] : __dsub_rn(1.0, f[0]));
            coeff = __dmul_rn(coeff, b ? f[1] : __dsub_rn(1.0, f[1]));
            coeff = __dmul_rn(coeff, d ? f[2] : __dsub_rn(1.0, f[2]));
            t = __dadd_rn(t, coeff);
        }
        out[i] = __double2float_rn(t);
    }
}

// ------------------------------------------------------------------------------------------ host
// One operand's leaves unpacked into its dense array; voxels its leaves cover other than once fail
// their tile (a field without leaves leaves every voxel uncovered).
int upload_unpack(const PackNode* nodes, int64_t count, const void* payload, int64_t samples, const int32_t* shape,
                  uint32_t* d_dense, unsigned* d_cover, unsigned long long* d_fail, cudaStream_t st) {
    std::vector<int64_t> ids, starts;
    int64_t total = 0;
    for (int64_t k = 0; k < count; ++k) {
        if (nodes[k].children[0] >= 0) continue;
        ids.push_back(k);
        starts.push_back(total);
        total += (int64_t)nodes[k].shape[0] * nodes[k].shape[1] * nodes[k].shape[2];
    }
    const int64_t vox = (int64_t)shape[0] * shape[1] * shape[2];
    PackNode* d_nodes = nullptr;
    int64_t *d_ids = nullptr, *d_starts = nullptr;
    uint32_t* d_payload = nullptr;
    int status = FB_OK;
    if (cudaMemsetAsync(d_cover, 0, vox * 4, st) != cudaSuccess) return FB_RUNTIME;
    if (!ids.empty()) {
        if (cudaMallocAsync(&d_nodes, count * sizeof(PackNode), st) != cudaSuccess ||
            cudaMallocAsync(&d_ids, ids.size() * 8, st) != cudaSuccess ||
            cudaMallocAsync(&d_starts, ids.size() * 8, st) != cudaSuccess ||
            cudaMallocAsync(&d_payload, samples * 4, st) != cudaSuccess ||
            cudaMemcpyAsync(d_nodes, nodes, count * sizeof(PackNode), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(d_ids, ids.data(), ids.size() * 8, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(d_starts, starts.data(), ids.size() * 8, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(d_payload, payload, samples * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
            status = FB_RUNTIME;
        if (!status) {
            const int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)fb_sm_count() * 16);
            k_unpack<<<std::max(grid, 1), 256, 0, st>>>(d_nodes, d_ids, d_starts, (int)ids.size(), total, d_payload,
                                                       shape[0], shape[1], shape[2], d_dense, d_cover);
            if (cudaGetLastError() != cudaSuccess) status = FB_RUNTIME;
        }
    }
    if (!status) {
        k_cover_check<<<(int)std::min<int64_t>((vox + 255) / 256, (int64_t)fb_sm_count() * 16), 256, 0, st>>>(
            d_cover, vox, shape[1], shape[2], d_fail);
        if (cudaGetLastError() != cudaSuccess) status = FB_RUNTIME;
    }
    if (d_nodes) cudaFreeAsync(d_nodes, st);
    if (d_ids) cudaFreeAsync(d_ids, st);
    if (d_starts) cudaFreeAsync(d_starts, st);
    if (d_payload) cudaFreeAsync(d_payload, st);
    return status;
}

// Copy the tiles before `stop` (in the reference's tile order) of a dense result into `output`, row
// by row as the reference writes them (execute.cpp:44-49).
void copy_tiles_before(const float* dense, const int32_t* shape, uint64_t stop, float* output) {
    const int sx = shape[0], sy = shape[1], sz = shape[2];
    uint64_t tile = 0;
    for (int x = 0; x < sx; x += 16)
        for (int y = 0; y < sy; y += 32)
            for (int z = 0; z < sz; z += 16, ++tile) {
                if (tile >= stop) return;
                const int hx = std::min(x + 16, sx), hy = std::min(y + 32, sy), len = std::min(z + 16, sz) - z;
                for (int a = x; a < hx; ++a)
                    for (int b = y; b < hy; ++b) {
                        const int64_t index = ((int64_t)a * sy + b) * sz + z;
                        std::memcpy(output + index, dense + index, len * sizeof(float));
                    }
            }
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------------------------------ packing ABI
// Replaces adaptive_pack, src/field_engine/adaptive_pack_native_v1/pack.cpp:57-69: same arguments
// (host float32 samples, int32 shape[3], threshold 8..4096), same NULL on invalid input.
void* adaptive_pack(const void* data, const int32_t* shape, int threshold) noexcept {
    if (!data || !pack_args_ok(shape, threshold)) return nullptr;
    const int64_t total = (int64_t)shape[0] * shape[1] * shape[2];
    const uint32_t* bits = static_cast<const uint32_t*>(data);
    for (int64_t i = 0; i < total; ++i)
        if ((bits[i] & 0x7f800000u) == 0x7f800000u) return nullptr;
    cudaStream_t st = nullptr;
    uint32_t* d = nullptr;
    Packed* p = new (std::nothrow) Packed;
    if (!p) return nullptr;
    int status = FB_RUNTIME;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
        cudaMallocAsync(&d, total * 4, st) == cudaSuccess &&
        cudaMemcpyAsync(d, data, total * 4, cudaMemcpyHostToDevice, st) == cudaSuccess)
        status = pack_device(d, shape, threshold, st, *p);
    if (d) cudaFreeAsync(d, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (status) {
        if (p->d_payload) cudaFree(p->d_payload);
        delete p;
        return nullptr;
    }
    return p;
}

// Device-input form: `d_data` holds the float32 samples on the device; synchronises `stream`.
// Returns NULL on invalid input (non-finite samples included) or failure.
void* fb_pack_device(const float* d_data, const int32_t* shape, int threshold, void* stream) noexcept {
    if (!d_data || !pack_args_ok(shape, threshold)) return nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t total = (int64_t)shape[0] * shape[1] * shape[2];
    int* d_bad = nullptr;
    int bad = 0;
    if (cudaMallocAsync(&d_bad, 4, st) != cudaSuccess || cudaMemsetAsync(d_bad, 0, 4, st) != cudaSuccess)
        return nullptr;
    k_pack_finite<<<(int)std::min<int64_t>((total + 255) / 256, (int64_t)fb_sm_count() * 8), 256, 0, st>>>(
        reinterpret_cast<const uint32_t*>(d_data), total, d_bad);
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
                    cudaStreamSynchronize(st) == cudaSuccess;
    cudaFreeAsync(d_bad, st);
    if (!ok || bad) return nullptr;
    Packed* p = new (std::nothrow) Packed;
    if (!p) return nullptr;
    if (pack_device(reinterpret_cast<const uint32_t*>(d_data), shape, threshold, st, *p)) {
        if (p->d_payload) cudaFree(p->d_payload);
        delete p;
        return nullptr;
    }
    return p;
}

// Replace adaptive_nodes / adaptive_samples / adaptive_copy / adaptive_free, pack.cpp:70-79.
int64_t adaptive_nodes(const void* pointer) noexcept {
    return pointer ? (int64_t) static_cast<const Packed*>(pointer)->nodes.size() : 0;
}

int64_t adaptive_samples(const void* pointer) noexcept {
    return pointer ? static_cast<const Packed*>(pointer)->n_payload : 0;
}

int adaptive_copy(const void* pointer, void* nodes, int64_t count, void* payload, int64_t samples) noexcept {
    const Packed* p = static_cast<const Packed*>(pointer);
    if (!p || !nodes || !payload) return 1;
    if (count != (int64_t)p->nodes.size() || samples != p->n_payload) return 1;
    std::memcpy(nodes, p->nodes.data(), p->nodes.size() * sizeof(PackNode));
    if (samples && cudaMemcpy(payload, p->d_payload, samples * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    return 0;
}

void adaptive_free(void* pointer) noexcept {
    Packed* p = static_cast<Packed*>(pointer);
    if (!p) return;
    if (p->d_payload) cudaFree(p->d_payload);
    delete p;
}

// Device pointer of a packed payload (valid until adaptive_free).
const float* fb_pack_payload_device(const void* pointer) noexcept {
    return pointer ? reinterpret_cast<const float*>(static_cast<const Packed*>(pointer)->d_payload) : nullptr;
}

// ------------------------------------------------------------------------------------------ CSG ABI
// Replaces csg_execute, src/field_engine/csg_batch_native_v1/execute.cpp:10-53: same arguments (host
// pointers to each operand's 52-byte nodes and float32 payload), same statuses 1-5: 1 arguments, 2
// program, 3 any operand gather failure (bounds, malformed leaf, gap, overlap), 4 a non-finite
// result, 5 a runtime failure.  On 3 / 4 the output holds the tiles the reference would have
// written before stopping (its 16 x 32 x 16 tile order), and nothing beyond them.
int csg_execute(const void* const* nodes, const int64_t* counts, const void* const* payload, const int64_t* lengths,
                int32_t fields, const int32_t* shape, const CsgInsn* program, int32_t instructions,
                float* output) noexcept {
    try {
        if (!nodes || !counts || !payload || !lengths || !shape || !program || !output || fields < 1 || fields > 256 ||
            instructions < 1 || instructions > 1024)
            return 1;
        int64_t total = 1;
        for (int a = 0; a < 3; ++a) {
            if (shape[a] < 1 || shape[a] > 4096) return 1;
            total *= shape[a];
        }
        if (total > 16777216) return 1;
        std::vector<int> last(fields + instructions, -1);
        for (int n = 0; n < instructions; ++n) {
            const CsgInsn& p = program[n];
            if (p.op < 0 || p.op > 2 || p.left < 0 || p.left >= fields + n) return 2;
            last[p.left] = n;
            if (p.op == 2) {
                if (!std::isfinite(p.offset)) return 2;
            } else {
                if (p.right < 0 || p.right >= fields + n) return 2;
                last[p.right] = n;
            }
        }
        last.back() = instructions;
        // only the operands the program reads are gathered, as in the reference
        for (int f = 0; f < fields; ++f)
            if (last[f] >= 0) {
                const int rc = check_nodes(static_cast<const PackNode*>(nodes[f]), payload[f], counts[f], lengths[f],
                                           shape);
                if (rc) return rc;
            }
        // operands: inputs by index (-1 - f), intermediates in slots freed after their last use
        std::vector<CsgStep> prog;
        std::vector<int> operand(fields + instructions, 0);
        std::vector<int> used_inputs, input_of(fields, -1);
        for (int f = 0; f < fields; ++f)
            if (last[f] >= 0) {
                input_of[f] = (int)used_inputs.size();
                used_inputs.push_back(f);
                operand[f] = -1 - input_of[f];
            }
        std::vector<int> free_slots;
        int next_slot = 0;
        auto alloc = [&]() -> int {
            if (!free_slots.empty()) {
                const int s = free_slots.back();
                free_slots.pop_back();
                return s;
            }
            return next_slot++;
        };
        auto release = [&](int id) {
            if (id >= fields) free_slots.push_back(operand[id]);
        };
        for (int n = 0; n < instructions; ++n) {
            const CsgInsn& p = program[n];
            CsgStep s;
            s.op = p.op;
            s.a = operand[p.left];
            s.b = p.op == 2 ? 0 : operand[p.right];
            s.offset = p.op == 2 ? p.offset : 0.0;
            // operands whose last use is this instruction give their slot back before the result takes one
            if (last[p.left] == n) release(p.left);
            if (p.op != 2 && p.right != p.left && last[p.right] == n) release(p.right);
            s.dst = alloc();
            operand[fields + n] = s.dst;
            prog.push_back(s);
            if (last[fields + n] < 0) free_slots.push_back(s.dst);  // computed (and checked), never read
        }
        const int result_slot = operand[fields + instructions - 1];
        const bool global_slots = next_slot > kLocalSlots;
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return 5;
        const int nin = (int)used_inputs.size();
        std::vector<float*> d_fields(nin, nullptr);
        unsigned* d_cover = nullptr;
        unsigned long long* d_fail = nullptr;
        float** d_ptrs = nullptr;
        CsgStep* d_prog = nullptr;
        float* d_out = nullptr;
        float* d_slots = nullptr;
        int status = 0;
        if (cudaMallocAsync(&d_cover, total * 4, st) != cudaSuccess || cudaMallocAsync(&d_fail, 8, st) != cudaSuccess ||
            cudaMemsetAsync(d_fail, 0xff, 8, st) != cudaSuccess)
            status = 5;
        for (int i = 0; i < nin && !status; ++i) {
            const int f = used_inputs[i];
            if (cudaMallocAsync(&d_fields[i], total * 4, st) != cudaSuccess) { status = 5; break; }
            if (upload_unpack(static_cast<const PackNode*>(nodes[f]), counts[f], payload[f], lengths[f], shape,
                              reinterpret_cast<uint32_t*>(d_fields[i]), d_cover, d_fail, st))
                status = 5;
        }
        if (!status &&
            (cudaMallocAsync(&d_ptrs, nin * sizeof(float*), st) != cudaSuccess ||
             cudaMallocAsync(&d_prog, prog.size() * sizeof(CsgStep), st) != cudaSuccess ||
             cudaMallocAsync(&d_out, total * 4, st) != cudaSuccess ||
             (global_slots && cudaMallocAsync(&d_slots, (int64_t)next_slot * total * 4, st) != cudaSuccess) ||
             cudaMemcpyAsync(d_ptrs, d_fields.data(), nin * sizeof(float*), cudaMemcpyHostToDevice, st) != cudaSuccess ||
             cudaMemcpyAsync(d_prog, prog.data(), prog.size() * sizeof(CsgStep), cudaMemcpyHostToDevice, st) !=
                 cudaSuccess))
            status = 5;
        unsigned long long fail = ~0ull;
        if (!status) {
            const size_t smem = prog.size() * sizeof(CsgStep);  // <= 1024 x 24 B
            const int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)fb_sm_count() * 8);
            if (global_slots)
                k_csg_program<true><<<grid, 256, smem, st>>>(d_ptrs, d_prog, (int)prog.size(), result_slot, total,
                                                             shape[1], shape[2], d_out, d_slots, d_fail);
            else
                k_csg_program<false><<<grid, 256, smem, st>>>(d_ptrs, d_prog, (int)prog.size(), result_slot, total,
                                                              shape[1], shape[2], d_out, nullptr, d_fail);
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(&fail, d_fail, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                status = 5;
        }
        if (!status) {
            if (fail == ~0ull) {
                if (cudaMemcpyAsync(output, d_out, total * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess)
                    status = 5;
            } else {
                // the reference's stopping point: the tiles before it are written, then 3 or 4
                const uint64_t stop = fail >> 1;
                if (stop > 0) {
                    std::vector<float> dense(total);
                    if (cudaMemcpyAsync(dense.data(), d_out, total * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                        cudaStreamSynchronize(st) != cudaSuccess)
                        status = 5;
                    else
                        copy_tiles_before(dense.data(), shape, stop, output);
                }
                if (!status) status = (fail & 1ull) ? 4 : 3;
            }
        }
        for (float* d : d_fields)
            if (d) cudaFreeAsync(d, st);
        if (d_cover) cudaFreeAsync(d_cover, st);
        if (d_fail) cudaFreeAsync(d_fail, st);
        if (d_ptrs) cudaFreeAsync(d_ptrs, st);
        if (d_prog) cudaFreeAsync(d_prog, st);
        if (d_out) cudaFreeAsync(d_out, st);
        if (d_slots) cudaFreeAsync(d_slots, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        return status;
    } catch (...) {
        return 5;
    }
}

// ------------------------------------------------------------------------------------------ query ABI
// Exact samples at int64 index triples (host pointers), the reference's samples_at
// (src/field_engine/adaptive_sample_blocks_v1.py:103-128).  Indices are validated by the caller.
int fb_packed_samples_at(const void* nodes, int64_t count, const float* payload, int64_t samples,
                         const int64_t* indices, int64_t n, float* out) noexcept {
    if (!nodes || !payload || !indices || !out || count < 1 || samples < 1 || n < 0) return 1;
    if (n == 0) return 0;
    cudaStream_t st = nullptr;
    PackNode* d_nodes = nullptr;
    float *d_payload = nullptr, *d_out = nullptr;
    int64_t* d_idx = nullptr;
    int status = 2;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
        cudaMallocAsync(&d_nodes, count * sizeof(PackNode), st) == cudaSuccess &&
        cudaMallocAsync(&d_payload, samples * 4, st) == cudaSuccess &&
        cudaMallocAsync(&d_idx, n * 24, st) == cudaSuccess && cudaMallocAsync(&d_out, n * 4, st) == cudaSuccess &&
        cudaMemcpyAsync(d_nodes, nodes, count * sizeof(PackNode), cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(d_payload, payload, samples * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(d_idx, indices, n * 24, cudaMemcpyHostToDevice, st) == cudaSuccess) {
        k_samples_at<<<(int)std::min<int64_t>((n + 255) / 256, (int64_t)fb_sm_count() * 8), 256, 0, st>>>(
            d_nodes, d_payload, d_idx, n, d_out);
        if (cudaGetLastError() == cudaSuccess &&
            cudaMemcpyAsync(out, d_out, n * 4, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
            cudaStreamSynchronize(st) == cudaSuccess)
            status = 0;
    }
    if (d_nodes) cudaFreeAsync(d_nodes, st);
    if (d_payload) cudaFreeAsync(d_payload, st);
    if (d_idx) cudaFreeAsync(d_idx, st);
    if (d_out) cudaFreeAsync(d_out, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    return status;
}

// Trilinear point query on a packed field with device-resident nodes / payload / points / output
// (the reference's AdaptiveSampleBlocks.query, adaptive_sample_blocks_v1.py:130-151).
int fb_packed_query_device(const void* d_nodes, const float* d_payload, const int32_t* shape, const double* origin,
                           double pitch, const double* d_points, int64_t n, float* d_out, void* stream) noexcept {
    if (!d_nodes || !d_payload || !shape || !origin || !d_points || !d_out || n < 0 || !(pitch > 0)) return 1;
    if (n == 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_query<<<(int)std::min<int64_t>((n + 127) / 128, (int64_t)fb_sm_count() * 16), 128, 0, st>>>(
        static_cast<const PackNode*>(d_nodes), d_payload, shape[0], shape[1], shape[2], origin[0], origin[1], origin[2],
        pitch, d_points, n, d_out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // extern "C"
