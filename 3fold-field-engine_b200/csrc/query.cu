// SDF value and gradient point queries on sm_100a.
//
// Recipes (src/field_engine/ikarus_v1/eval_warp.py:478-488 eval_batch, :718-733 gradient_batch):
//   k_eval_points evaluates the compiled program at float32 points (thread per point).  With a
//   built field's culling lists (the lists a classification left in its scratch) each point inside
//   the grid walks only its block's list where the classification kept one, else its superblock's
//   -- exact for every point of that region, by the same strict-domination argument as the build --
//   instead of the whole chain.
//   k_gradient_points: central differences with step h along each axis, the six offset points
//   formed in float64 and rounded to float32 as the reference does.
// Per-block pitch fields (src/field_engine/faltkarna_v1_multires.py:84-104, :384-459):
//   k_multires_tiles fills each active brick's (B*2^l + 1)^3 lattice at pitch h/2^l;
//   k_multires_value answers avstand (trilinear at the brick's own pitch, +-margin outside active
//   bricks) and k_multires_gradient the brick-clamped central difference.
#include "common.cuh"
#include "prims.cuh"
#include <algorithm>
#include <cmath>

namespace {

// Program value at a float32 world point.  chain_mode 1: `list` (entries chain index << 2 | mode)
// over the chain; chain_mode 0: the postfix program with a float32 stack.
__device__ float eval_point(const PrimF* __restrict__ primf, const FbInsn* __restrict__ chain, int n_chain,
                            int chain_mode, const uint32_t* __restrict__ list, int len, float x, float y, float z) {
    if (chain_mode) {
        float acc = 0.f;
        for (int i = 0; i < len; ++i) {
            const uint32_t e = list ? list[i] : (uint32_t)i << 2;
            const FbInsn I = chain[e >> 2];
            const uint32_t mode = e & 3u;
            const int op = mode == 1u ? CH_SET : (mode == 2u ? CH_SETNEG : I.op);
            const float v = op == CH_OFFSET ? 0.f : primf_world(primf[I.arg], x, y, z);
            acc = chain_apply(op, acc, v, (float)I.k);
        }
        return acc;
    }
    float st[32];
    int sp = 0;
    for (int i = 0; i < n_chain; ++i) {
        const FbInsn I = chain[i];
        if (I.op == OP_PUSH) {
            if (sp < 32) st[sp++] = primf_world(primf[I.arg], x, y, z);
        } else if (I.op == OP_OFFSET) {
            if (sp > 0) st[sp - 1] -= (float)I.k;
        } else if (sp > 1) {
            const float b = st[--sp];
            const int op = I.op == OP_UNION ? CH_UNION : (I.op == OP_INTERSECT ? CH_INTERSECT : CH_SUBTRACT);
            st[sp - 1] = combine_f(op, st[sp - 1], b, (float)I.k);
        }
    }
    return sp == 1 ? st[0] : __int_as_float(0x7fc00000);
}

struct Accel {  // a built field's culling lists (nullptr pool: walk the whole chain)
    const uint32_t* pool;
    const int64_t* sb_off;
    const int32_t* sb_len;
    // per-block lists (nullable): used where kind == 0, or for every block when blk_all
    const int32_t* kind;
    const int32_t* blk_off;
    const int32_t* blk_len;
    const uint32_t* blk_pool;
    int64_t blk_cap;
    int blk_all;
    double x0, y0, z0, pitch;
    int nx, ny, nz, B, S, nsy, nsz, nbx, nby, nbz;
};

// The list a point at (x, y, z) walks and its key: block b (0 <= b < nblocks) where the
// classification kept the block's list, nblocks + superblock for other points inside the grid,
// nblocks + nsuper (nullptr list) for the whole chain.
__device__ __forceinline__ int64_t accel_list(const Accel& A, int n_chain, float x, float y, float z,
                                              const uint32_t*& list, int& len) {
    const int64_t nblocks = (int64_t)A.nbx * A.nby * A.nbz;
    const int64_t nsuper = (int64_t)((A.nbx + A.S - 1) / A.S) * A.nsy * A.nsz;
    if (A.pool) {
        // the voxel cell containing the point, inside the grid's block range
        const double fx = ((double)x - A.x0) / A.pitch, fy = ((double)y - A.y0) / A.pitch,
                     fz = ((double)z - A.z0) / A.pitch;
        const double ex = (double)A.nbx * A.B, ey = (double)A.nby * A.B, ez = (double)A.nbz * A.B;
        if (fx >= 0 && fy >= 0 && fz >= 0 && fx <= ex && fy <= ey && fz <= ez) {
            const int bi = min((int)(fx / A.B), A.nbx - 1), bj = min((int)(fy / A.B), A.nby - 1),
                      bk = min((int)(fz / A.B), A.nbz - 1);
            if (A.blk_len) {  // the block's own list: culled for a region holding the whole block
                const int64_t b = ((int64_t)bi * A.nby + bj) * A.nbz + bk;
                if (A.blk_all || A.kind[b] == 0) {
                    const int n = A.blk_len[b];
                    const int64_t off = n >= 0 ? (int64_t)A.blk_off[b] : -1;
                    if (n >= 0 && off >= 0 && off + n <= A.blk_cap) {
                        list = A.blk_pool + off;
                        len = n;
                        return b;
                    }
                }
            }
            const int64_t s = ((int64_t)(bi / A.S) * A.nsy + bj / A.S) * A.nsz + bk / A.S;
            list = A.pool + A.sb_off[s];
            len = A.sb_len[s];
            return nblocks + s;
        }
    }
    list = nullptr;
    len = n_chain;
    return nblocks + nsuper;
}

__device__ __forceinline__ float eval_accel(const PrimF* primf, const FbInsn* chain, int n_chain, int chain_mode,
                                            const Accel& A, float x, float y, float z) {
    if (chain_mode) {
        const uint32_t* list;
        int len;
        accel_list(A, n_chain, x, y, z, list, len);
        return eval_point(primf, chain, n_chain, 1, list, len, x, y, z);
    }
    return eval_point(primf, chain, n_chain, chain_mode, nullptr, n_chain, x, y, z);
}

__global__ void k_eval_points(const PrimF* __restrict__ primf, const FbInsn* __restrict__ chain, int n_chain,
                              int chain_mode, Accel A, const float* __restrict__ pts, int64_t n,
                              float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = eval_accel(primf, chain, n_chain, chain_mode, A, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
}

// Central difference with step h: (f(p + h e_a) - f(p - h e_a)) / (2h) in float32, the offset
// points formed in float64 and rounded to float32 (eval_warp.py:718-733).  `value` (nullable)
// also receives f(p).
__global__ void k_gradient_points(const PrimF* __restrict__ primf, const FbInsn* __restrict__ chain, int n_chain,
                                  int chain_mode, Accel A, const float* __restrict__ pts, int64_t n, double h,
                                  float* __restrict__ grad, float* __restrict__ value) {
    const float inv = (float)(2.0 * h);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
        for (int a = 0; a < 3; ++a) {
            float q[2][3];
            for (int s = 0; s < 2; ++s)
                for (int c = 0; c < 3; ++c) q[s][c] = (float)(c == a ? p[c] + (s ? -h : h) : p[c]);
            const float vp = eval_accel(primf, chain, n_chain, chain_mode, A, q[0][0], q[0][1], q[0][2]);
            const float vm = eval_accel(primf, chain, n_chain, chain_mode, A, q[1][0], q[1][1], q[1][2]);
            grad[3 * i + a] = (vp - vm) / inv;
        }
        if (value) value[i] = eval_accel(primf, chain, n_chain, chain_mode, A, (float)p[0], (float)p[1], (float)p[2]);
    }
}

// ------------------------------------------------------------------------------------ binned queries
// Evaluation points sorted by the list they walk, so that the lanes of a warp share one list
// (broadcast loads, one primitive kind at a time) instead of each lane walking its own.  Point e of
// a query with `nvar` variants is point e / nvar at variant e % nvar: 0 the point itself, 1 + 2a + s
// the offset along axis a (s = 0: +h, 1: -h), formed in float64 and rounded to float32 exactly as
// k_gradient_points forms them, and every value is computed by the same eval_point -- so the
// results are bit-identical to the unsorted kernels.
__device__ __forceinline__ void variant_point(const float* __restrict__ pts, int64_t e, int nvar, double h, float& x,
                                              float& y, float& z) {
    const int64_t i = e / nvar;
    const int v = (int)(e - i * nvar);
    const double p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    float q[3];
    for (int c = 0; c < 3; ++c) q[c] = (float)p[c];
    if (v > 0) {
        const int a = (v - 1) >> 1, s = (v - 1) & 1;
        q[a] = (float)(p[a] + (s ? -h : h));
    }
    x = q[0];
    y = q[1];
    z = q[2];
}

__global__ void k_query_keys(Accel A, int n_chain, const float* __restrict__ pts, int64_t ne, int nvar, double h,
                             int32_t* __restrict__ keys, int32_t* __restrict__ count) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        variant_point(pts, e, nvar, h, x, y, z);
        const uint32_t* list;
        int len;
        const int32_t key = (int32_t)accel_list(A, n_chain, x, y, z, list, len);
        keys[e] = key;
        atomicAdd(&count[key], 1);
    }
}

// Exclusive scan of count[0, n) in place: tiles of kScanTile per CTA, then the tile sums, then the
// tile offsets added back.
constexpr int kScanThreads = 1024, kScanItems = 4, kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int32_t block_exclusive_scan(int32_t v, int32_t* warp_sums, int32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int32_t w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    total = warp_sums[(blockDim.x >> 5) - 1];
    const int32_t before = warp > 0 ? warp_sums[warp - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(int32_t* __restrict__ data, int64_t n,
                                                             int32_t* __restrict__ tile_sums) {
    __shared__ int32_t warp_sums[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? data[base + k] : 0;
        sum += v[k];
    }
    int32_t total;
    int32_t run = block_exclusive_scan(sum, warp_sums, total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) data[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One CTA scans the tile sums (at most kScanTile of them) in place.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int32_t* __restrict__ tile_sums, int ntiles) {
    __shared__ int32_t warp_sums[32];
    const int base = threadIdx.x * kScanItems;
    int32_t v[kScanItems], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < ntiles ? tile_sums[base + k] : 0;
        sum += v[k];
    }
    int32_t total;
    int32_t run = block_exclusive_scan(sum, warp_sums, total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < ntiles) tile_sums[base + k] = run;
        run += v[k];
    }
}

__global__ void k_scan_add(int32_t* __restrict__ data, int64_t n, const int32_t* __restrict__ tile_sums) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        data[i] += tile_sums[i / kScanTile];
}

// cursor[key] starts at the key's first sorted position and ends past its last.
__global__ void k_query_scatter(const int32_t* __restrict__ keys, int64_t ne, int32_t* __restrict__ cursor,
                                int32_t* __restrict__ order) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x)
        order[atomicAdd(&cursor[keys[e]], 1)] = (int32_t)e;
}

__global__ void k_query_eval_sorted(const PrimF* __restrict__ primf, const FbInsn* __restrict__ chain, int n_chain,
                                    Accel A, const float* __restrict__ pts, int64_t ne, int nvar, double h,
                                    const int32_t* __restrict__ order, float* __restrict__ vals) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ne; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = order[t];
        float x, y, z;
        variant_point(pts, e, nvar, h, x, y, z);
        const uint32_t* list;
        int len;
        accel_list(A, n_chain, x, y, z, list, len);
        vals[e] = eval_point(primf, chain, n_chain, 1, list, len, x, y, z);
    }
}

// value = variant 0, gradient component a = (v(1 + 2a) - v(2 + 2a)) / (2h), k_gradient_points' arithmetic.
__global__ void k_query_combine(const float* __restrict__ vals, int64_t n, double h, float* __restrict__ grad,
                                float* __restrict__ value) {
    const float inv = (float)(2.0 * h);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float* v = vals + 7 * i;
        for (int a = 0; a < 3; ++a) grad[3 * i + a] = (v[1 + 2 * a] - v[2 + 2 * a]) / inv;
        if (value) value[i] = v[0];
    }
}

struct BinnedPlan {
    int64_t ne, nbins, ntiles;
    int64_t keys, order, vals, count, tiles, total;
};

BinnedPlan binned_plan(int64_t n, int nvar, int64_t nbins) {
    BinnedPlan p{};
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    p.ne = n * nvar;
    p.nbins = nbins;
    p.ntiles = (nbins + kScanTile - 1) / kScanTile;
    int64_t at = 0;
    p.keys = at; at += al(p.ne * 4);
    p.order = at; at += al(p.ne * 4);
    p.vals = at; at += al(p.ne * 4);
    p.count = at; at += al(nbins * 4);
    p.tiles = at; at += al(p.ntiles * 4);
    p.total = at;
    return p;
}

int64_t accel_bins(const int32_t* dims) {
    const int B = dims[3];
    if (B < 1) return -1;
    const int64_t nbx = (dims[0] + B - 1) / B, nby = (dims[1] + B - 1) / B, nbz = (dims[2] + B - 1) / B;
    const int64_t S = std::max(1, fb_super_edge(dims[0], dims[1], dims[2]) / B);
    const int64_t ns = ((nbx + S - 1) / S) * ((nby + S - 1) / S) * ((nbz + S - 1) / S);
    return nbx * nby * nbz + ns + 1;
}

constexpr int64_t kMaxBins = int64_t(kScanTile) * kScanTile;  // one tile-sum CTA covers them
constexpr int64_t kMaxBinnedPoints = int64_t(1) << 31;          // sorted positions are int32

// ------------------------------------------------------------------------------------ multires
struct Multi {
    double lx, ly, lz;   // world origin of the brick lattice
    double h;            // coarse pitch
    int B, bx, by, bz;   // brick edge in coarse voxels, brick grid
    double margin;       // +-margin answers outside active bricks (float64, as the reference)
};

// Samples of brick b at level l: (B*2^l + 1)^3 float32 at pitch h/2^l from the brick origin.
// Warp per active brick.  The brick's culled list (its classification block's, whose culling
// region is the brick's closed box) is localised to the brick origin once in shared memory, the
// lattice is evaluated in block-local float32, and values inside the guard band are recomputed in
// float64 -- the leaf kernel's scheme.
constexpr int kTileWarps = 4, kTileCap = 48;

__global__ void __launch_bounds__(32 * kTileWarps) k_multires_tiles(
    const PrimF* __restrict__ primf, const FbInsn* __restrict__ chain, int n_chain, int chain_mode,
    const FbPrim* __restrict__ prims, Multi M, const int32_t* __restrict__ bricks, const int8_t* __restrict__ levels,
    const int64_t* __restrict__ offsets, int64_t nbricks, const int32_t* __restrict__ blk_off,
    const int32_t* __restrict__ blk_len, const uint32_t* __restrict__ blk_pool, float guard, float* __restrict__ pool) {
    __shared__ LocalPrim s_prim[kTileWarps][kTileCap];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    LocalPrim* sp = s_prim[warp];
    for (int64_t k = gwarp; k < nbricks; k += nwarps) {
        const int64_t b = bricks[k];
        const int l = levels[k];
        const int bk = (int)(b % M.bz), bj = (int)((b / M.bz) % M.by), bi = (int)(b / ((int64_t)M.bz * M.by));
        const int m = (M.B << l) + 1;
        const double pitch = M.h / (double)(1 << l);
        const float fpitch = (float)pitch;
        // every float64 operation rounded once, as NumPy does (no contraction)
        const double ox = rn_add(M.lx, rn_mul((double)(bi * M.B), M.h)), oy = rn_add(M.ly, rn_mul((double)(bj * M.B), M.h)),
                     oz = rn_add(M.lz, rn_mul((double)(bk * M.B), M.h));
        const bool listed = blk_len && blk_len[b] >= 0;
        const uint32_t* list = listed ? blk_pool + blk_off[b] : nullptr;
        const int len = listed ? blk_len[b] : n_chain;
        const bool staged = chain_mode && listed && len <= kTileCap;
        if (staged) {
            for (int i = lane; i < len; i += 32) {
                const uint32_t e = list[i];
                const FbInsn I = chain[e >> 2];
                const uint32_t mode = e & 3u;
                const int op = mode == 1u ? CH_SET : (mode == 2u ? CH_SETNEG : I.op);
                if (op == CH_OFFSET) {
                    sp[i].op = op;
                    sp[i].k = (float)I.k;
                } else {
                    localise(prims[I.arg], primf[I.arg], ox, oy, oz, op, (float)I.k, sp[i]);
                }
            }
        }
        __syncwarp();
        float* out = pool + offsets[k];
        const int64_t total = (int64_t)m * m * m;
        for (int64_t v = lane; v < total; v += 32) {
            const int iz = (int)(v % m), iy = (int)((v / m) % m), ix = (int)(v / ((int64_t)m * m));
            const double x = rn_add(ox, rn_mul((double)ix, pitch)), y = rn_add(oy, rn_mul((double)iy, pitch)),
                         z = rn_add(oz, rn_mul((double)iz, pitch));
            float val;
            if (!chain_mode) {
                val = (float)program_eval_d(prims, chain, n_chain, x, y, z);
            } else {
                if (staged) {
                    const float dx = ix * fpitch, dy = iy * fpitch, dz = iz * fpitch;
                    float acc = 0.f;
                    for (int i = 0; i < len; ++i) {
                        const LocalPrim& P = sp[i];
                        acc = P.op == CH_OFFSET ? acc - P.k : chain_apply(P.op, acc, local_eval(P, dx, dy, dz), P.k);
                    }
                    val = acc;
                } else {
                    val = eval_point(primf, chain, n_chain, 1, list, len, (float)x, (float)y, (float)z);
                }
                if (!(fabsf(val) >= guard) || !staged) {  // float64 inside the guard band (and when unstaged)
                    double acc = 0.0;
                    for (int i = 0; i < len; ++i) {
                        const uint32_t e = list ? list[i] : (uint32_t)i << 2;
                        const FbInsn I = chain[e >> 2];
                        const uint32_t mode = e & 3u;
                        const int op = mode == 1u ? CH_SET : (mode == 2u ? CH_SETNEG : I.op);
                        const double pv = op == CH_OFFSET ? 0.0 : prim_world_d(prims[I.arg], x, y, z);
                        acc = chain_apply_d(op, acc, pv, I.k);
                    }
                    val = (float)acc;
                }
            }
            out[v] = val;
        }
        __syncwarp();
    }
}

// Brick of a world point, preferring an active brick when the point lies exactly on a face
// (faltkarna_v1_multires.py:384-402).  Returns false when the point is outside the lattice.
__device__ bool brick_of(const Multi& M, const int8_t* __restrict__ kind, double px, double py, double pz, int b[3]) {
    const double L = rn_mul((double)M.B, M.h);
    const double rel[3] = {rn_div(rn_sub(px, M.lx), L), rn_div(rn_sub(py, M.ly), L), rn_div(rn_sub(pz, M.lz), L)};
    const int shp[3] = {M.bx, M.by, M.bz};
    bool outside = false;
    for (int a = 0; a < 3; ++a) {
        const double f = floor(rel[a]);
        long long v = (long long)f;
        outside |= v < 0 || v >= shp[a];
        b[a] = (int)min(max(v, 0ll), (long long)shp[a] - 1);
    }
    auto kind_at = [&](int x, int y, int z) { return kind[((int64_t)x * M.by + y) * M.bz + z]; };
    bool inactive = kind_at(b[0], b[1], b[2]) != 0;
    for (int a = 0; a < 3; ++a) {
        const bool on_plane = rel[a] == floor(rel[a]) && b[a] > 0 && inactive && !outside;
        if (!on_plane) continue;
        int c[3] = {b[0], b[1], b[2]};
        c[a] -= 1;
        if (kind_at(c[0], c[1], c[2]) == 0) b[a] -= 1;
        inactive = kind_at(b[0], b[1], b[2]) != 0;
    }
    return !outside;
}

// scipy.ndimage.map_coordinates(tile, coords, order=1, mode='nearest') at one point of a cubic
// (m x m x m) float32 tile: each coordinate clamped into [0, m-1], weights (1-t, t) per axis,
// sum over the eight corners in C order of value x w0 x w1 x w2 in float64.
__device__ double tile_trilinear(const float* __restrict__ t, int m, double cx, double cy, double cz) {
    const double c[3] = {fmin(fmax(cx, 0.0), (double)(m - 1)), fmin(fmax(cy, 0.0), (double)(m - 1)),
                         fmin(fmax(cz, 0.0), (double)(m - 1))};
    int s[3];
    double f[3];
    for (int a = 0; a < 3; ++a) {
        const double fl = floor(c[a]);
        s[a] = (int)fl;
        f[a] = __dsub_rn(c[a], fl);
    }
    double acc = 0.0;
    for (int h = 0; h < 8; ++h) {
        const int a = (h >> 2) & 1, b = (h >> 1) & 1, d = h & 1;
        const int X = min(s[0] + a, m - 1), Y = min(s[1] + b, m - 1), Z = min(s[2] + d, m - 1);
        double coeff = (double)t[((int64_t)X * m + Y) * m + Z];
        coeff = __dmul_rn(coeff, a ? f[0] : __dsub_rn(1.0, f[0]));
        coeff = __dmul_rn(coeff, b ? f[1] : __dsub_rn(1.0, f[1]));
        coeff = __dmul_rn(coeff, d ? f[2] : __dsub_rn(1.0, f[2]));
        acc = __dadd_rn(acc, coeff);
    }
    return acc;
}

__device__ double multires_value(const Multi& M, const int8_t* __restrict__ kind, const int8_t* __restrict__ level,
                                 const int64_t* __restrict__ tile_off, const float* __restrict__ pool, double px,
                                 double py, double pz) {
    int b[3];
    const bool inside = brick_of(M, kind, px, py, pz, b);
    const int64_t lin = ((int64_t)b[0] * M.by + b[1]) * M.bz + b[2];
    const int kd = kind[lin];
    if (!inside) return M.margin;
    if (kd != 0) return kd < 0 ? -M.margin : M.margin;
    const int l = level[lin];
    const double pitch = rn_div(M.h, (double)(1 << l));
    const double L = rn_mul((double)M.B, M.h);
    const double ox = rn_add(M.lx, rn_mul((double)b[0], L)), oy = rn_add(M.ly, rn_mul((double)b[1], L)),
                 oz = rn_add(M.lz, rn_mul((double)b[2], L));
    const int m = (M.B << l) + 1;
    // map_coordinates returns the tile's dtype: one float32 rounding
    return (double)__double2float_rn(
        tile_trilinear(pool + tile_off[lin], m, rn_div(rn_sub(px, ox), pitch), rn_div(rn_sub(py, oy), pitch),
                       rn_div(rn_sub(pz, oz), pitch)));
}

__global__ void k_multires_value(Multi M, const int8_t* __restrict__ kind, const int8_t* __restrict__ level,
                                 const int64_t* __restrict__ tile_off, const float* __restrict__ pool,
                                 const double* __restrict__ pts, int64_t n, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = multires_value(M, kind, level, tile_off, pool, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
}

// Central difference at the point's brick pitch, both probes clamped into the brick
// (faltkarna_v1_multires.py:437-459).
__global__ void k_multires_gradient(Multi M, const int8_t* __restrict__ kind, const int8_t* __restrict__ level,
                                    const int64_t* __restrict__ tile_off, const float* __restrict__ pool,
                                    const double* __restrict__ pts, int64_t n, double* __restrict__ out) {
    const double L = rn_mul((double)M.B, M.h);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
        int b[3];
        brick_of(M, kind, p[0], p[1], p[2], b);
        const int lv = level[((int64_t)b[0] * M.by + b[1]) * M.bz + b[2]];
        const double h = rn_div(M.h, (double)(1 << max(lv, 0)));
        const double o[3] = {rn_add(M.lx, rn_mul((double)b[0], L)), rn_add(M.ly, rn_mul((double)b[1], L)),
                             rn_add(M.lz, rn_mul((double)b[2], L))};
        for (int a = 0; a < 3; ++a) {
            double pa[3] = {p[0], p[1], p[2]}, pb[3] = {p[0], p[1], p[2]};
            pa[a] = fmin(rn_add(p[a], rn_mul(0.5, h)), rn_add(o[a], L));
            pb[a] = fmax(rn_sub(p[a], rn_mul(0.5, h)), o[a]);
            for (int c = 0; c < 3; ++c)
                if (c != a) {
                    pa[c] = fmin(p[c], rn_add(o[c], L));
                    pb[c] = fmax(p[c], o[c]);
                }
            const double step = rn_sub(pa[a], pb[a]);
            const double va = multires_value(M, kind, level, tile_off, pool, pa[0], pa[1], pa[2]);
            const double vb = multires_value(M, kind, level, tile_off, pool, pb[0], pb[1], pb[2]);
            out[3 * i + a] = rn_div(rn_sub(va, vb), fmax(step, 1e-12));
        }
    }
}

// Overlap band (faltkarna_v1_multires.py:211-251): every face of a fine brick whose neighbour is an
// active brick of a coarser level takes the trilinear sample of the neighbour's lattice at the face's
// own sample points.  One CTA per brick of the launch's level, its six faces in the reference's order
// (axis 0..2, side -1 then +1; a later face overwrites the edges it shares with an earlier one).  The
// reference walks the bricks in ascending id and overwrites lattices in place, so a neighbour of level
// >= 1 is read as overwritten when its id is smaller than this brick's and as built otherwise: the
// host launches level 1, 2, 3 in turn and passes `orig`, a copy of the pool taken before the band.
__global__ void __launch_bounds__(256) k_multires_band(Multi M, const int8_t* __restrict__ kind,
                                                       const int8_t* __restrict__ level,
                                                       const int64_t* __restrict__ tile_off, float* __restrict__ pool,
                                                       const float* __restrict__ orig,
                                                       const int32_t* __restrict__ bricks, int n_bricks, int lvl,
                                                       int* __restrict__ faces) {
    const int idx = blockIdx.x;
    if (idx >= n_bricks) return;
    const int lin = bricks[idx];
    const int b[3] = {lin / (M.by * M.bz), (lin / M.bz) % M.by, lin % M.bz};
    const double L = rn_mul((double)M.B, M.h);
    const double lo[3] = {M.lx, M.ly, M.lz};
    const int shp[3] = {M.bx, M.by, M.bz};
    const int n_l = M.B << lvl, m = n_l + 1;
    const double h_f = rn_div(M.h, (double)(1 << lvl));
    double bo[3];
    for (int a = 0; a < 3; ++a) bo[a] = rn_add(lo[a], rn_mul((double)b[a], L));
    float* tile = pool + tile_off[lin];
    for (int ax = 0; ax < 3; ++ax) {
        for (int sida = -1; sida <= 1; sida += 2) {
            int nb[3] = {b[0], b[1], b[2]};
            nb[ax] += sida;
            if (nb[ax] < 0 || nb[ax] >= shp[ax]) continue;
            const int64_t nlin = ((int64_t)nb[0] * M.by + nb[1]) * M.bz + nb[2];
            if (kind[nlin] != 0) continue;
            const int lvl_n = level[nlin];
            if (lvl_n < 0 || lvl_n >= lvl) continue;
            const float* src = (lvl_n >= 1 && nlin < lin ? pool : orig) + tile_off[nlin];
            const int m_n = (M.B << lvl_n) + 1;
            const double h_n = rn_div(M.h, (double)(1 << lvl_n));
            double no[3];
            for (int a = 0; a < 3; ++a) no[a] = rn_add(lo[a], rn_mul((double)nb[a], L));
            const int u = ax == 0 ? 1 : 0, w = ax == 2 ? 1 : 2;  // the face's free axes, ascending
            const int fixed = sida < 0 ? 0 : n_l;
            for (int k = threadIdx.x; k < m * m; k += blockDim.x) {
                int g[3];
                g[ax] = fixed;
                g[u] = k / m;
                g[w] = k % m;
                double c[3];
                for (int a = 0; a < 3; ++a) {
                    const double pt = rn_add(rn_mul((double)g[a], h_f), bo[a]);
                    c[a] = rn_div(rn_sub(pt, no[a]), h_n);
                }
                tile[((int64_t)g[0] * m + g[1]) * m + g[2]] = (float)tile_trilinear(src, m_n, c[0], c[1], c[2]);
            }
            if (threadIdx.x == 0) atomicAdd(faces, 1);
            __syncthreads();
        }
    }
}

Multi make_multi(const double* lo, double h, int B, const int32_t* bshape, double margin) {
    Multi M;
    M.lx = lo[0];
    M.ly = lo[1];
    M.lz = lo[2];
    M.h = h;
    M.B = B;
    M.bx = bshape[0];
    M.by = bshape[1];
    M.bz = bshape[2];
    M.margin = margin;
    return M;
}

// Many (leaf A, leaf B) gridfield pairs in one launch (src/field_engine/ikarus_v1/eval_warp.py:521-564):
// thread per point, pair = pair_of_point[i], value max(sample(A), sample(B)) with the gridfield
// sampler.  params: 12 floats per leaf (the gridfield record layout: origin, pitch, iso, is_sdf, nx,
// ny, nz, -, table address halves).  An index outside its table reads NaN.
__global__ void k_grid_pairs(const float* __restrict__ params, int n_leaves, const float* __restrict__ pts,
                             const int32_t* __restrict__ pair, int64_t n, const int32_t* __restrict__ la,
                             const int32_t* __restrict__ lb, int n_pairs, float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int pid = pair[i];
        float v = __int_as_float(0x7fc00000);
        if (pid >= 0 && pid < n_pairs) {
            const int a = la[pid], b = lb[pid];
            if (a >= 0 && a < n_leaves && b >= 0 && b < n_leaves) {
                const float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
                v = fmaxf(grid_sample_f(params + 12 * a, x, y, z), grid_sample_f(params + 12 * b, x, y, z));
            }
        }
        out[i] = v;
    }
}

}  // namespace

extern "C" {

// Overlap band of a per-block-pitch field (k_multires_band): d_orig is caller scratch the size of
// the pool (its state before the band); d_bricks lists the active bricks of level >= 1 sorted by
// level (n_of_level[l] of level l = 1..3 after n_of_level[0] = 0); d_faces (one int) counts the faces
// written.  Stream-ordered.
int fb_multires_band_device(const double* lo, double h, int32_t B, const int32_t* bshape, const int8_t* d_kind,
                            const int8_t* d_level, const int64_t* d_tile_off, float* d_pool, int64_t pool_len,
                            float* d_orig, const int32_t* d_bricks, const int32_t* n_of_level, int32_t* d_faces,
                            void* stream) noexcept {
    if (!lo || !bshape || !d_kind || !d_level || !d_tile_off || !d_pool || !d_orig || !n_of_level || !d_faces ||
        B < 1 || !(h > 0) || pool_len < 0)
        return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Multi M = make_multi(lo, h, B, bshape, 0.0);
    FB_CUDA(cudaMemsetAsync(d_faces, 0, sizeof(int32_t), st));
    FB_CUDA(cudaMemcpyAsync(d_orig, d_pool, pool_len * 4, cudaMemcpyDeviceToDevice, st));
    int at = 0;
    for (int l = 1; l <= 3; ++l) {
        const int n = n_of_level[l];
        if (n < 0) return FB_INVALID;
        if (n > 0) {
            if (!d_bricks) return FB_INVALID;
            k_multires_band<<<n, 256, 0, st>>>(M, d_kind, d_level, d_tile_off, d_pool, d_orig, d_bricks + at, n, l,
                                               d_faces);
            FB_LAUNCH();
        }
        at += n;
    }
    return FB_OK;
}

// The multi-pair gridfield sweep (k_grid_pairs); all pointers on the device, stream-ordered.
int fb_grid_pairs_device(const float* d_params, int32_t n_leaves, const float* d_pts, const int32_t* d_pair,
                         int64_t n, const int32_t* d_leaf_a, const int32_t* d_leaf_b, int32_t n_pairs, float* d_out,
                         void* stream) noexcept {
    if (n < 0 || n_leaves < 1 || n_pairs < 1 || !d_params ||
        (n > 0 && (!d_pts || !d_pair || !d_leaf_a || !d_leaf_b || !d_out)))
        return FB_INVALID;
    if (n == 0) return FB_OK;
    k_grid_pairs<<<(int)std::min<int64_t>((n + 255) / 256, (int64_t)fb_sm_count() * 16), 256, 0,
                   static_cast<cudaStream_t>(stream)>>>(d_params, n_leaves, d_pts, d_pair, n, d_leaf_a, d_leaf_b,
                                                        n_pairs, d_out);
    FB_LAUNCH();
    return FB_OK;
}


// Values (and gradients) of a compiled recipe at float32 points, device pointers.  d_primf is the
// float32 primitive mirror a field build prepared (fb_query_prepare fills one).  accel_* (all
// nullable) are a built field's superblock lists and grid; without them every point walks the
// whole chain / program.
int fb_query_prepare(const FbPrim* d_prims, int32_t n_prims, void* d_primf, void* stream) noexcept;

// Scratch bytes of the sorted query path for n points (with_grad: value + gradient, 7 evaluations
// per point) on an accelerated grid of dims (nx, ny, nz, B); -1 when that grid takes the unsorted path.
int64_t fb_query_scratch_bytes(const int32_t* accel_dims, int64_t n, int32_t with_grad) noexcept {
    if (!accel_dims || n < 0) return -1;
    const int64_t nbins = accel_bins(accel_dims);
    const int nvar = with_grad ? 7 : 1;
    if (nbins <= 0 || nbins > kMaxBins || n * nvar >= kMaxBinnedPoints) return -1;
    return binned_plan(n, nvar, nbins).total;
}

int fb_query_points_device(const void* d_primf, const FbInsn* d_chain, int32_t n_chain, int32_t mode,
                           const void* accel_pool, const int64_t* accel_off, const int32_t* accel_len,
                           const double* accel_grid /* x0,y0,z0,pitch */, const int32_t* accel_dims /* nx,ny,nz,B */,
                           const int32_t* d_kind, const int32_t* blk_off, const int32_t* blk_len,
                           const uint32_t* blk_pool, int64_t blk_cap, int32_t blk_all, const float* d_points, int64_t n,
                           double h, float* d_value, float* d_grad, void* d_scratch, int64_t scratch_len,
                           void* stream) noexcept {
    if (!d_primf || !d_chain || n_chain < 1 || !d_points || n < 0 || (!d_value && !d_grad)) return FB_INVALID;
    if (n == 0) return FB_OK;
    Accel A{};
    if (accel_pool && accel_off && accel_len && accel_grid && accel_dims && mode == 1) {
        A.pool = static_cast<const uint32_t*>(accel_pool);
        A.sb_off = accel_off;
        A.sb_len = accel_len;
        A.x0 = accel_grid[0]; A.y0 = accel_grid[1]; A.z0 = accel_grid[2]; A.pitch = accel_grid[3];
        A.nx = accel_dims[0]; A.ny = accel_dims[1]; A.nz = accel_dims[2]; A.B = accel_dims[3];
        A.nbx = (A.nx + A.B - 1) / A.B; A.nby = (A.ny + A.B - 1) / A.B; A.nbz = (A.nz + A.B - 1) / A.B;
        A.S = std::max(1, fb_super_edge(A.nx, A.ny, A.nz) / A.B);
        A.nsy = (A.nby + A.S - 1) / A.S;
        A.nsz = (A.nbz + A.S - 1) / A.S;
        if (blk_off && blk_len && blk_pool && blk_cap > 0 && (blk_all || d_kind)) {
            A.kind = d_kind;
            A.blk_off = blk_off;
            A.blk_len = blk_len;
            A.blk_pool = blk_pool;
            A.blk_cap = blk_cap;
            A.blk_all = blk_all ? 1 : 0;
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)fb_sm_count() * 16);
    const PrimF* primf = static_cast<const PrimF*>(d_primf);
    const int nvar = d_grad ? 7 : 1;
    const int64_t nbins = A.pool ? accel_bins(accel_dims) : -1;
    if (d_scratch && A.pool && nbins > 0 && nbins <= kMaxBins && n * nvar < kMaxBinnedPoints) {
        const BinnedPlan P = binned_plan(n, nvar, nbins);
        if (scratch_len < P.total) return FB_INVALID;
        char* b = static_cast<char*>(d_scratch);
        int32_t* keys = reinterpret_cast<int32_t*>(b + P.keys);
        int32_t* order = reinterpret_cast<int32_t*>(b + P.order);
        float* vals = d_grad ? reinterpret_cast<float*>(b + P.vals) : d_value;
        int32_t* count = reinterpret_cast<int32_t*>(b + P.count);
        int32_t* tiles = reinterpret_cast<int32_t*>(b + P.tiles);
        const int ge = (int)std::min<int64_t>((P.ne + 255) / 256, (int64_t)fb_sm_count() * 16);
        FB_CUDA(cudaMemsetAsync(count, 0, nbins * 4, st));
        k_query_keys<<<ge, 256, 0, st>>>(A, n_chain, d_points, P.ne, nvar, h, keys, count);
        FB_LAUNCH();
        k_scan_tiles<<<(unsigned)P.ntiles, kScanThreads, 0, st>>>(count, nbins, tiles);
        FB_LAUNCH();
        k_scan_sums<<<1, kScanThreads, 0, st>>>(tiles, (int)P.ntiles);
        FB_LAUNCH();
        k_scan_add<<<(int)std::min<int64_t>((nbins + 255) / 256, (int64_t)fb_sm_count() * 16), 256, 0, st>>>(
            count, nbins, tiles);
        FB_LAUNCH();
        k_query_scatter<<<ge, 256, 0, st>>>(keys, P.ne, count, order);
        FB_LAUNCH();
        k_query_eval_sorted<<<ge, 256, 0, st>>>(primf, d_chain, n_chain, A, d_points, P.ne, nvar, h, order, vals);
        FB_LAUNCH();
        if (d_grad) {
            k_query_combine<<<grid, 128, 0, st>>>(vals, n, h, d_grad, d_value);
            FB_LAUNCH();
        }
        return FB_OK;
    }
    if (d_grad) {
        k_gradient_points<<<grid, 128, 0, st>>>(primf, d_chain, n_chain, mode, A, d_points, n, h, d_grad, d_value);
    } else {
        k_eval_points<<<grid, 128, 0, st>>>(primf, d_chain, n_chain, mode, A, d_points, n, d_value);
    }
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_RUNTIME;
}

// Fill the (B*2^l+1)^3 lattices of the listed active bricks (device pointers).  levels[k] in 0..3,
// offsets[k] = start of brick k's lattice in d_pool.  blk_* (nullable) are the per-block culled
// lists of a classification of the same recipe on the brick grid.
int fb_multires_tiles_device(const void* d_primf, const FbInsn* d_chain, int32_t n_chain, int32_t mode,
                             const FbPrim* d_prims, const double* lo, double h, int32_t B, const int32_t* bshape,
                             const int32_t* d_bricks, const int8_t* d_levels, const int64_t* d_offsets,
                             int64_t nbricks, const int32_t* d_blk_off, const int32_t* d_blk_len,
                             const uint32_t* d_blk_pool, float guard, float* d_pool, void* stream) noexcept {
    if (!d_primf || !d_chain || !d_prims || !lo || !bshape || !d_pool || nbricks < 0 || B < 1 || !(h > 0))
        return FB_INVALID;
    if (nbricks == 0) return FB_OK;
    const Multi M = make_multi(lo, h, B, bshape, 0.0);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_multires_tiles<<<fb_sm_count() * 8, 32 * kTileWarps, 0, st>>>(static_cast<const PrimF*>(d_primf), d_chain, n_chain, mode,
                                                       d_prims, M, d_bricks, d_levels, d_offsets, nbricks, d_blk_off,
                                                       d_blk_len, d_blk_pool, guard, d_pool);
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_RUNTIME;
}

// avstand / gradient of a per-block-pitch field at float64 points (device pointers); d_grad
// (nullable) gets (n, 3) when requested, d_value (nullable) the values.
int fb_multires_query_device(const double* lo, double h, int32_t B, const int32_t* bshape, double margin,
                             const int8_t* d_kind, const int8_t* d_level, const int64_t* d_tile_off,
                             const float* d_pool, const double* d_points, int64_t n, double* d_value,
                             double* d_grad, void* stream) noexcept {
    if (!lo || !bshape || !d_kind || !d_level || !d_tile_off || !d_pool || !d_points || n < 0 || B < 1 || !(h > 0))
        return FB_INVALID;
    if (n == 0) return FB_OK;
    const Multi M = make_multi(lo, h, B, bshape, margin);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)fb_sm_count() * 16);
    if (d_value) k_multires_value<<<grid, 128, 0, st>>>(M, d_kind, d_level, d_tile_off, d_pool, d_points, n, d_value);
    if (d_grad) k_multires_gradient<<<grid, 128, 0, st>>>(M, d_kind, d_level, d_tile_off, d_pool, d_points, n, d_grad);
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_RUNTIME;
}

}  // extern "C"
