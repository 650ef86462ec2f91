// Packed adaptive block tree of a dense SDF on the GPU (the reference's AdaptiveBlocks format,
// src/field_engine/field_adaptive_blocks_v1.py): 2-bit node codes, breadth-first, four per byte;
// rank checkpoints every 64 bytes for the branch (2) and value (3) codes; float32 values of the
// value leaves in node order.
//
// Build, level by level (sides 8, 4, 2, 1; field_adaptive_blocks_v1.py:113-147):
//   k_tree_codes  : code of every node of the level from the dense classification rule of its
//                   block (dense_block_kind, evaluated for the level's nodes only -- not for every
//                   block of the grid at that side): outside the grid 0, kind > 0 -> 0, kind < 0
//                   -> 1, kind 0 -> 3 at side 1 else 2; and the flag the level's exclusive scan
//                   ranks (2 at sides > 1, 3 at 1);
//   k_tree_expand : each branch of rank b writes its 8 children at 8b + (4i + 2j + k) of the next
//                   level -- the breadth-first order in which the children of the b-th branch of
//                   the whole tree start at root_count + 8b;
//   k_tree_values : each value leaf of rank r copies dense[x, y, z] to values[r].
// Then k_tree_pack packs the concatenated codes and k_tree_group_counts + the scan give the rank
// checkpoints.  k_tree_sample walks the tree for grid indices the way AdaptiveBlocks.sample does
// (field_adaptive_blocks_v1.py:35-82), counting codes 16 nodes per 32-bit word with popc.
#include "common.cuh"
#include "dense.cuh"
#include "scan.cuh"
#include <algorithm>

namespace {

// ------------------------------------------------------------------------------------ build
struct Level {
    const int32_t* coords;  // [n][3] node corners, or nullptr for the root level (C order over the root grid)
    int64_t rx, ry, rz;     // root grid (root level only)
};

__device__ __forceinline__ void node_corner(const Level& L, int64_t i, int64_t& x, int64_t& y, int64_t& z) {
    if (L.coords) {
        x = L.coords[3 * i];
        y = L.coords[3 * i + 1];
        z = L.coords[3 * i + 2];
    } else {
        z = (i % L.rz) * 8;
        y = ((i / L.rz) % L.ry) * 8;
        x = (i / (L.rz * L.ry)) * 8;
    }
}

__global__ void k_tree_codes(const float* __restrict__ dense, int side, float margin, int64_t nx, int64_t ny,
                             int64_t nz, Level L, int64_t n, uint8_t* __restrict__ codes, int32_t* __restrict__ flag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t x, y, z;
    node_corner(L, i, x, y, z);
    int code = 0;
    if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) {
        float mn;
        const int k = dense_block_kind(dense, nx, ny, nz, side, x, y, z, margin, &mn);
        code = k > 0 ? 0 : (k < 0 ? 1 : (side == 1 ? 3 : 2));
    }
    codes[i] = (uint8_t)code;
    flag[i] = side == 1 ? (code == 3) : (code == 2);
}

__global__ void k_tree_expand(const uint8_t* __restrict__ codes, const int32_t* __restrict__ rank, Level L, int64_t n,
                              int side, int32_t* __restrict__ child) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n || codes[i] != 2) return;
    int64_t x, y, z;
    node_corner(L, i, x, y, z);
    const int half = side / 2;
    int32_t* out = child + (int64_t)rank[i] * 24;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        out[3 * c] = (int32_t)(x + ((c >> 2) & 1) * half);
        out[3 * c + 1] = (int32_t)(y + ((c >> 1) & 1) * half);
        out[3 * c + 2] = (int32_t)(z + (c & 1) * half);
    }
}

__global__ void k_tree_values(const float* __restrict__ dense, int64_t ny, int64_t nz, const uint8_t* __restrict__ codes,
                              const int32_t* __restrict__ rank, const int32_t* __restrict__ coords, int64_t n,
                              float* __restrict__ values) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n || codes[i] != 3) return;
    const int64_t x = coords[3 * i], y = coords[3 * i + 1], z = coords[3 * i + 2];
    values[rank[i]] = dense[(x * ny + y) * nz + z];
}

// Four 2-bit codes per byte (node i at bits 2 (i % 4)); the bytes past the last node are zero.
__global__ void k_tree_pack(const uint8_t* __restrict__ codes, int64_t node_count, uint8_t* __restrict__ packed,
                            int64_t nbytes_padded) {
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nbytes_padded) return;
    uint32_t v = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int64_t i = 4 * b + s;
        if (i < node_count) v |= (uint32_t)(codes[i] & 3) << (2 * s);
    }
    packed[b] = (uint8_t)v;
}

// Fields of a 32-bit word (16 two-bit codes) equal to `code`, as a mask of their low bits.
__device__ __forceinline__ uint32_t code_hits(uint32_t w, int code) {
    const uint32_t t = w ^ (0x55555555u * (uint32_t)code);
    return ~(t | (t >> 1)) & 0x55555555u;
}

// counts[c][g] = nodes of code 2 + c in the 64 bytes (16 words) of group g, for the full groups.
__global__ void k_tree_group_counts(const uint32_t* __restrict__ words, int64_t groups, int32_t* __restrict__ branch,
                                    int32_t* __restrict__ value) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= groups) return;
    int nb = 0, nv = 0;
#pragma unroll 4
    for (int j = 0; j < 16; ++j) {
        const uint32_t w = words[g * 16 + j];
        nb += __popc(code_hits(w, 2));
        nv += __popc(code_hits(w, 3));
    }
    branch[g] = nb;
    value[g] = nv;
}

// Nodes of `code` before `node`: the checkpoint of its 256-node group plus the words in between.
__device__ __forceinline__ int64_t rank_before(const uint32_t* __restrict__ words, const int32_t* __restrict__ prefix,
                                               int64_t node, int code) {
    const int64_t g = node >> 8;
    int64_t r = prefix[g];
    const int64_t wend = node >> 4;
    for (int64_t j = g * 16; j < wend; ++j) r += __popc(code_hits(words[j], code));
    const int rem = (int)(node & 15);
    if (rem) r += __popc(code_hits(words[wend], code) & ((1u << (2 * rem)) - 1u));
    return r;
}

// counts[j] of code 2 / code 3 in word j (16 nodes), for the per-word rank table of the sampler.
__global__ void k_tree_word_counts(const uint32_t* __restrict__ words, int64_t nwords, int32_t* __restrict__ branch,
                                   int32_t* __restrict__ value) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nwords) return;
    const uint32_t w = words[j];
    branch[j] = __popc(code_hits(w, 2));
    value[j] = __popc(code_hits(w, 3));
}

// Nodes of `code` before `node` from the per-word table (its exclusive prefix over words).
__device__ __forceinline__ int64_t rank_word(const uint32_t* __restrict__ words, const int32_t* __restrict__ table,
                                             int64_t node, int code) {
    const int64_t w = node >> 4;
    const int rem = (int)(node & 15);
    int64_t r = table[w];
    if (rem) r += __popc(code_hits(words[w], code) & ((1u << (2 * rem)) - 1u));
    return r;
}

// Status bits of a sample launch.
enum { kBadIndex = 1, kBadDepth = 2, kBadNode = 4 };

__global__ void k_tree_sample(const uint32_t* __restrict__ words, int64_t node_count, const int32_t* __restrict__ bprefix,
                              const int32_t* __restrict__ vprefix, const int32_t* __restrict__ bword,
                              const int32_t* __restrict__ vword, const float* __restrict__ values, int64_t n_values,
                              int64_t root_count, int64_t r1, int64_t r2, int64_t nx, int64_t ny, int64_t nz,
                              double pitch, const int64_t* __restrict__ ijk, int64_t n, float* __restrict__ out,
                              int* __restrict__ status) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int64_t i = ijk[3 * q], j = ijk[3 * q + 1], k = ijk[3 * q + 2];
    if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) {
        out[q] = __int_as_float(0x7fc00000);
        atomicOr(status, kBadIndex);
        return;
    }
    int64_t node = ((i >> 3) * r1 + (j >> 3)) * r2 + (k >> 3);
    int64_t size = 8;
    for (int depth = 0; depth < 4; ++depth) {
        if (node < 0 || node >= node_count) break;
        const int code = (int)((words[node >> 4] >> (2 * (node & 15))) & 3u);
        if (code < 2) {
            // (sign * sqrt(3)) * size * pitch in float64, rounded once to float32 (the reference's
            // np.where(kind == 0, 1., -1.) * np.sqrt(3.) * size * pitch stored into float32)
            const double s = code == 0 ? 1.7320508075688772 : -1.7320508075688772;
            out[q] = __double2float_rn(__dmul_rn(__dmul_rn(s, (double)size), pitch));
            return;
        }
        if (code == 3) {
            const int64_t r = vword ? rank_word(words, vword, node, 3) : rank_before(words, vprefix, node, 3);
            if (r < 0 || r >= n_values) break;
            out[q] = values[r];
            return;
        }
        const int64_t half = size >> 1;
        if (half < 1) {
            out[q] = __int_as_float(0x7fc00000);
            atomicOr(status, kBadDepth);
            return;
        }
        const int child = (int)(4 * ((i / half) & 1) + 2 * ((j / half) & 1) + ((k / half) & 1));
        node = root_count + 8 * (bword ? rank_word(words, bword, node, 2) : rank_before(words, bprefix, node, 2)) + child;
        size = half;
    }
    out[q] = __int_as_float(0x7fc00000);
    atomicOr(status, kBadNode);
}

}  // namespace

extern "C" {

// Scratch bytes of fb_tree_codes_device for a level of n nodes (its exclusive scan).
int64_t fb_tree_scan_bytes(int64_t n) noexcept {
    if (n < 0) return -1;
    return scan_scratch_words(n) * 4;
}

// One level of the tree: codes[n] and rank[n] (exclusive count of the level's ranked code: 2 at
// sides 8/4/2, 3 at side 1) with the level total in *d_total.  Each node is classified from the
// dense field by the block rule with this side's margin (float32 of sqrt(3) * side * pitch);
// d_coords: the level's node corners [n][3], or nullptr for the root level (C order over
// rx x ry x rz root blocks of side 8).
int fb_tree_codes_device(const float* d_dense, int64_t nx, int64_t ny, int64_t nz, int32_t side, float margin,
                         const int32_t* d_coords, int64_t rx, int64_t ry, int64_t rz, int64_t n, uint8_t* d_codes,
                         int32_t* d_rank, int32_t* d_total, void* d_scratch, int64_t scratch_len,
                         void* stream) noexcept {
    if (!d_dense || !d_codes || !d_rank || !d_total || n < 0 || (side != 8 && side != 4 && side != 2 && side != 1))
        return FB_INVALID;
    if (nx < 1 || ny < 1 || nz < 1 || n >= (int64_t(1) << 31)) return FB_INVALID;
    if (!d_coords && (side != 8 || rx < 1 || ry < 1 || rz < 1 || rx * ry * rz != n)) return FB_INVALID;
    if (n > 0 && (!d_scratch || scratch_len < fb_tree_scan_bytes(n))) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Level L{d_coords, rx, ry, rz};
    if (n > 0) {
        k_tree_codes<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_dense, side, margin, nx, ny, nz, L, n, d_codes,
                                                                 d_rank);
        FB_LAUNCH();
    }
    return scan_exclusive(d_rank, n, d_total, static_cast<int32_t*>(d_scratch), scratch_len / 4, st);
}

// The next level's node corners: 8 per branch of this level (side > 1), at 8 * rank + child.
int fb_tree_expand_device(const uint8_t* d_codes, const int32_t* d_rank, const int32_t* d_coords, int64_t rx,
                          int64_t ry, int64_t rz, int64_t n, int32_t side, int32_t* d_child, void* stream) noexcept {
    if (!d_codes || !d_rank || !d_child || n < 0 || (side != 8 && side != 4 && side != 2)) return FB_INVALID;
    if (!d_coords && (side != 8 || rx * ry * rz != n)) return FB_INVALID;
    if (n == 0) return FB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Level L{d_coords, rx, ry, rz};
    k_tree_expand<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_codes, d_rank, L, n, side, d_child);
    FB_LAUNCH();
    return FB_OK;
}

// values[rank] = dense[corner] for the value leaves of the side-1 level.
int fb_tree_values_device(const float* d_dense, int64_t nx, int64_t ny, int64_t nz, const uint8_t* d_codes,
                          const int32_t* d_rank, const int32_t* d_coords, int64_t n, float* d_values,
                          void* stream) noexcept {
    if (!d_dense || !d_codes || !d_rank || !d_coords || !d_values || n < 0 || nx < 1 || ny < 1 || nz < 1)
        return FB_INVALID;
    if (n == 0) return FB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_tree_values<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_dense, ny, nz, d_codes, d_rank, d_coords, n, d_values);
    FB_LAUNCH();
    return FB_OK;
}

// Scratch bytes of fb_tree_pack_device for node_count nodes.
int64_t fb_tree_pack_scratch_bytes(int64_t node_count) noexcept {
    if (node_count < 0) return -1;
    const int64_t groups = (node_count + 255) / 256 + 1;
    return (scan_scratch_words(groups) + 1) * 4;  // the scans' scratch, then one word for their totals
}

// packed[ceil(node_count / 4)] (allocated to a multiple of 4 bytes, the tail zeroed here) and the
// checkpoints branch_prefix / value_prefix[floor(len(packed) / 64) + 1] (nodes of code 2 / 3 in the
// bytes before 64 g).  d_codes: every node's code in tree order.
int fb_tree_pack_device(const uint8_t* d_codes, int64_t node_count, uint8_t* d_packed, int32_t* d_branch_prefix,
                        int32_t* d_value_prefix, void* d_scratch, int64_t scratch_len, void* stream) noexcept {
    if (!d_codes || !d_packed || !d_branch_prefix || !d_value_prefix || node_count < 1 ||
        node_count >= (int64_t(1) << 31))
        return FB_INVALID;
    if (!d_scratch || scratch_len < fb_tree_pack_scratch_bytes(node_count)) return FB_INVALID;
    if (reinterpret_cast<uintptr_t>(d_packed) & 3) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nbytes = (node_count + 3) / 4;
    const int64_t padded = (nbytes + 3) / 4 * 4;
    k_tree_pack<<<(unsigned)((padded + 255) / 256), 256, 0, st>>>(d_codes, node_count, d_packed, padded);
    FB_LAUNCH();
    const int64_t full = nbytes / 64;  // checkpoints at 0, 64, ..., 64 * full
    if (full > 0) {
        k_tree_group_counts<<<(unsigned)((full + 255) / 256), 256, 0, st>>>(reinterpret_cast<const uint32_t*>(d_packed),
                                                                           full, d_branch_prefix, d_value_prefix);
        FB_LAUNCH();
    }
    // exclusive scans of the group counts over full + 1 entries (the last entry's count is a
    // placeholder zero, so the scan's last element is the total of the full groups)
    FB_CUDA(cudaMemsetAsync(d_branch_prefix + full, 0, sizeof(int32_t), st));
    FB_CUDA(cudaMemsetAsync(d_value_prefix + full, 0, sizeof(int32_t), st));
    int32_t* scratch = static_cast<int32_t*>(d_scratch);
    const int64_t words = scratch_len / 4;
    // the total goes to the scratch's last word (unused by the scan of full + 1 elements)
    if (int rc = scan_exclusive(d_branch_prefix, full + 1, scratch + words - 1, scratch, words - 1, st)) return rc;
    if (int rc = scan_exclusive(d_value_prefix, full + 1, scratch + words - 1, scratch, words - 1, st)) return rc;
    return FB_OK;
}

// Scratch bytes of fb_tree_rank_words_device for node_count nodes.
int64_t fb_tree_rank_words_scratch_bytes(int64_t node_count) noexcept {
    if (node_count < 0) return -1;
    return (scan_scratch_words((node_count + 15) / 16 + 1) + 1) * 4;  // the scans' scratch, then their totals word
}

// The sampler's per-word rank tables (not part of the stored format): d_branch_words /
// d_value_words[w] = nodes of code 2 / 3 before word w (16 nodes per word), ceil(node_count / 16)
// + 1 entries each.
int fb_tree_rank_words_device(const uint8_t* d_packed, int64_t node_count, int32_t* d_branch_words,
                              int32_t* d_value_words, void* d_scratch, int64_t scratch_len, void* stream) noexcept {
    if (!d_packed || !d_branch_words || !d_value_words || !d_scratch || node_count < 1 ||
        node_count >= (int64_t(1) << 31) || (reinterpret_cast<uintptr_t>(d_packed) & 3))
        return FB_INVALID;
    if (scratch_len < fb_tree_rank_words_scratch_bytes(node_count)) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nwords = (node_count + 15) / 16;
    k_tree_word_counts<<<(unsigned)((nwords + 255) / 256), 256, 0, st>>>(reinterpret_cast<const uint32_t*>(d_packed),
                                                                        nwords, d_branch_words, d_value_words);
    FB_LAUNCH();
    FB_CUDA(cudaMemsetAsync(d_branch_words + nwords, 0, sizeof(int32_t), st));
    FB_CUDA(cudaMemsetAsync(d_value_words + nwords, 0, sizeof(int32_t), st));
    int32_t* scratch = static_cast<int32_t*>(d_scratch);
    const int64_t words = scratch_len / 4;
    if (int rc = scan_exclusive(d_branch_words, nwords + 1, scratch + words - 1, scratch, words - 1, st)) return rc;
    if (int rc = scan_exclusive(d_value_words, nwords + 1, scratch + words - 1, scratch, words - 1, st)) return rc;
    return FB_OK;
}

// Values at grid indices ijk[n][3] (int64) of a packed tree; out[n] float32.  d_packed must be
// 4-byte aligned with its bytes up to a multiple of 4 readable (fb_tree_pack_device writes them).
// d_branch_words / d_value_words: the per-word rank tables of fb_tree_rank_words_device, or NULL
// to rank from the 64-byte checkpoints alone.  *d_status (device, OR-ed): 1 an index outside the
// grid, 2 a branch below side 1, 4 a node or value rank outside the arrays; those outputs are NaN.
int fb_tree_sample_device(const uint8_t* d_packed, int64_t node_count, const int32_t* d_branch_prefix,
                          const int32_t* d_value_prefix, const int32_t* d_branch_words, const int32_t* d_value_words,
                          const float* d_values, int64_t n_values, int64_t root_count,
                          int64_t r0, int64_t r1, int64_t r2, int64_t nx, int64_t ny, int64_t nz, double pitch,
                          const int64_t* d_ijk, int64_t n, float* d_out, int32_t* d_status, void* stream) noexcept {
    if (!d_packed || !d_branch_prefix || !d_value_prefix || !d_ijk || !d_out || !d_status || n < 0 || node_count < 1 ||
        root_count != r0 * r1 * r2 || root_count < 1 || root_count > node_count)
        return FB_INVALID;
    if (reinterpret_cast<uintptr_t>(d_packed) & 3) return FB_INVALID;
    if (n_values > 0 && !d_values) return FB_INVALID;
    if (n == 0) return FB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if ((d_branch_words == nullptr) != (d_value_words == nullptr)) return FB_INVALID;
    k_tree_sample<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(reinterpret_cast<const uint32_t*>(d_packed), node_count,
                                                               d_branch_prefix, d_value_prefix, d_branch_words,
                                                               d_value_words, d_values, n_values,
                                                               root_count, r1, r2, nx, ny, nz, pitch, d_ijk, n, d_out,
                                                               d_status);
    FB_LAUNCH();
    return FB_OK;
}

}  // extern "C"
