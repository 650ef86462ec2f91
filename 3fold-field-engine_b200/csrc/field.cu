// Block-sparse field build on sm_100a: block classification, stream compaction and fused
// leaf-tile evaluation with min/max CSG, for analytic recipes and for dense sampled fields.
//
// Analytic pipeline (all stream-ordered, no host round trip between kernels):
//   k_prepare_prims  float32 mirror of the primitive table + per-primitive Lipschitz bound.
//   k_cull           warp per region: walks the parent region's CSG chain list and keeps only the
//                    elements that can influence the region (Lipschitz interval arithmetic, exact
//                    for min/max: a skipped element is strictly dominated everywhere in the
//                    region, and an element that strictly dominates resets the list).  Two levels:
//                    coarse regions (two superblocks wide) from the full chain, superblocks (32
//                    voxels, 16 on grids of at most 128 per axis) from those.
//   k_classify_blocks  thread per block: culls the superblock list to the block, evaluates the 8
//                    corners in float32 in block-local coordinates, decides kind -1/0/+1 by the
//                    reference rule, re-evaluating in float64 when a corner value lies within the
//                    guard band of 0 or of the margin; the active blocks keep their lists.
//   k_compact        single-pass decoupled look-back scan: ascending active block ids + count.
//   k_leaf<B>        warp per active block: block-level culling, float64 -> float32 localisation of
//                    each surviving primitive, float32 evaluation of all B^3 voxels, float64 recheck
//                    inside the guard band, vectorised 128-bit tile stores.
// Reference semantics: src/field_engine/faltkarna_v1.py:51-82 (grid and layout), :129-164
// (classification rule), :167-190 (tile order), :277 (ascending compaction); dense input
// src/field_engine/faltkarna_v1_mesh_to_sdf.py:602-657.
#include "common.cuh"
#include "dense.cuh"
#include "prims.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

// Grid geometry of one build, fb_geom in include/field_b200.h.
struct FbGeom {
    double x0, y0, z0, pitch;
    int32_t nx, ny, nz, block;
    float margin, guard;
    int32_t reserved[2];
};
static_assert(sizeof(FbGeom) == 64, "fb_geom layout");

// One recipe of a batch, as fb_batch_item in include/field_b200.h.
struct FbBatchItem {
    const FbGeom* geom;
    const FbPrim* d_prims;
    const FbInsn* d_chain;
    int32_t n_prims, n_chain;
    int32_t* d_kind;
    float* d_cma;
    int32_t* d_active;
    int32_t* d_count;
    void* d_scratch;
    int64_t scratch_len;
    int32_t* d_slot;  // nullable: with d_mask, the recipe takes part in fb_batch_occupancy_device
    uint8_t* d_mask;
};
static_assert(sizeof(FbBatchItem) == 96, "fb_batch_item layout");

namespace {

constexpr float kBig = 1.0e6f;  // background of interior (-) and exterior (+) blocks, faltkarna_v1.py:46
constexpr int kCapCoarse = 1024;           // least list capacity of a coarse region
constexpr int kCapSuper = 256;             // least list capacity of a superblock
constexpr int64_t kCapBudget = 8 << 20;    // list entries per level beyond which capacities stop growing
constexpr int kCapBlock = 48;              // leaf staging chunk and the leaf pass's own culled-list capacity
constexpr int kCoarseDiv = 2;     // superblocks per coarse-region edge
constexpr int kTile = 2048;       // compaction tile (256 threads x 8)
constexpr int kLeafWarps = 4;     // warps per CTA in k_leaf


struct Geo {
    double x0, y0, z0, pitch;
    float fx0, fy0, fz0, fpitch;
    int nx, ny, nz, B;
    int nbx, nby, nbz;
    int64_t nblocks;
    int S, nsx, nsy, nsz;
    int64_t nsuper;
    int ncx, ncy, ncz;
    int64_t ncoarse;
    float margin, guard, eps;
    int special;  // fb_geom.reserved[0] bits 0-1: sampled-grid leaves, or tori of a large ring radius
};

Geo make_geo(const FbGeom& g) {
    Geo o{};
    o.x0 = g.x0; o.y0 = g.y0; o.z0 = g.z0; o.pitch = g.pitch;
    o.fx0 = (float)g.x0; o.fy0 = (float)g.y0; o.fz0 = (float)g.z0; o.fpitch = (float)g.pitch;
    o.nx = g.nx; o.ny = g.ny; o.nz = g.nz; o.B = g.block;
    o.nbx = (g.nx + g.block - 1) / g.block;
    o.nby = (g.ny + g.block - 1) / g.block;
    o.nbz = (g.nz + g.block - 1) / g.block;
    o.nblocks = (int64_t)o.nbx * o.nby * o.nbz;
    o.S = std::max(1, fb_super_edge(g.nx, g.ny, g.nz) / g.block);
    o.nsx = (o.nbx + o.S - 1) / o.S;
    o.nsy = (o.nby + o.S - 1) / o.S;
    o.nsz = (o.nbz + o.S - 1) / o.S;
    o.nsuper = (int64_t)o.nsx * o.nsy * o.nsz;
    o.ncx = (o.nsx + kCoarseDiv - 1) / kCoarseDiv;
    o.ncy = (o.nsy + kCoarseDiv - 1) / kCoarseDiv;
    o.ncz = (o.nsz + kCoarseDiv - 1) / kCoarseDiv;
    o.ncoarse = (int64_t)o.ncx * o.ncy * o.ncz;
    o.margin = g.margin;
    o.guard = g.guard;
    o.eps = 4.0f * g.guard;
    o.special = (g.reserved[0] & 3) != 0;
    return o;
}

bool geom_ok(const FbGeom& g) {
    if (!(g.pitch > 0) || !std::isfinite(g.pitch) || !std::isfinite(g.x0) || !std::isfinite(g.y0) ||
        !std::isfinite(g.z0))
        return false;
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || g.nx > 16384 || g.ny > 16384 || g.nz > 16384) return false;
    if (g.block != 4 && g.block != 8 && g.block != 16) return false;
    if (!(g.margin >= 0) || !(g.guard >= 0)) return false;
    return true;
}

// ------------------------------------------------------------------------------------ scratch
struct Plan {
    int64_t primf, pool, off, len, status, misc, total;
    int64_t blk_off, blk_len, blk_pool, blk_cap;  // per-block culled lists of active blocks
    int64_t pool_full, pool_coarse, pool_super;  // element offsets inside pool
    int64_t ntiles;
    int cap_coarse, cap_super;  // list capacities per coarse region / superblock
};

// List capacity of a level: grows while the level's lists stay within kCapBudget entries, never
// beyond the chain length (a list is a subsequence of the chain, so that capacity never overflows).
int level_cap(int64_t nregions, int base, int n_chain) {
    const int64_t grown = std::max<int64_t>(base, kCapBudget / std::max<int64_t>(nregions, 1));
    return (int)std::min<int64_t>(grown, std::max(n_chain, 1));
}

int64_t align256(int64_t x) { return (x + 255) / 256 * 256; }

Plan make_plan(const Geo& G, int n_prims, int n_chain) {
    Plan p{};
    int64_t at = 0;
    p.primf = at; at += align256((int64_t)std::max(n_prims, 1) * sizeof(PrimF));
    p.cap_coarse = level_cap(G.ncoarse, kCapCoarse, n_chain);
    p.cap_super = level_cap(G.nsuper, kCapSuper, n_chain);
    p.pool_full = 0;
    p.pool_coarse = n_chain;
    p.pool_super = p.pool_coarse + G.ncoarse * p.cap_coarse;
    const int64_t pool_elems = p.pool_super + G.nsuper * p.cap_super;
    p.pool = at; at += align256(pool_elems * 4);
    p.off = at; at += align256((G.ncoarse + G.nsuper) * 8);
    p.len = at; at += align256((G.ncoarse + G.nsuper) * 4);
    p.ntiles = (G.nblocks + kTile - 1) / kTile;
    p.status = at; at += align256(p.ntiles * 8);
    p.misc = at; at += 256;  // [0] ticket, [1] error flag, [2] block-list pool cursor
    p.blk_off = at; at += align256(G.nblocks * 4);
    p.blk_len = at; at += align256(G.nblocks * 4);
    p.blk_cap = std::max<int64_t>(G.nblocks * 12, 4096);  // active blocks' lists (<= kCapBlock each)
    p.blk_pool = at; at += align256(p.blk_cap * 4);
    p.total = at;
    return p;
}

// Compaction needs only the status words and the misc block.
int64_t compact_scratch(int64_t nblocks) { return align256((nblocks + kTile - 1) / kTile * 8) + 256; }

// ------------------------------------------------------------------------------------ prepare
__device__ void prepare_prim(const FbPrim* __restrict__ prims, int i, PrimF* __restrict__ out) {
    const FbPrim P = prims[i];
    PrimF F;
    F.type = P.type;
    F.s = (float)P.s;
    F.off = (float)P.off;
    F.ball = F.ball_k = F.pad = 0.f;
    bool ident = true;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) ident &= P.A[r * 4 + c] == (r == c ? 1.0 : 0.0);
    F.ident = ident ? 1 : 0;
    for (int j = 0; j < 12; ++j) F.A[j] = (float)P.A[j];
    // Lipschitz bound of x -> f(A x + t): sqrt of the Gershgorin bound on A^T A.
    double G[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += P.A[k * 4 + r] * P.A[k * 4 + c];
            G[r][c] = s;
        }
    double row = 0;
    for (int r = 0; r < 3; ++r) row = fmax(row, fabs(G[r][0]) + fabs(G[r][1]) + fabs(G[r][2]));
    double canon = 1.0;
    for (int j = 0; j < 12; ++j) F.p[j] = 0.f;
    const double* p = P.p;
    switch (P.type) {
    case P_CONE:
        canon = 2.0 + fabs(p[1] - p[0]) / p[2];
        F.p[0] = (float)p[0]; F.p[1] = (float)p[1]; F.p[2] = (float)p[2]; F.p[3] = (float)(1.0 / p[2]);
        break;
    case P_FRUSTUM: {
        const double z1 = p[0], hx0 = p[1], hy0 = p[2], hx1 = p[3], hy1 = p[4], cx1 = p[5], cy1 = p[6];
        const double kx = (hx1 - hx0) / z1, ky = (hy1 - hy0) / z1, kcx = cx1 / z1, kcy = cy1 / z1;
        const double a[4] = {-(kx + kcx), -(kx - kcx), -(ky + kcy), -(ky - kcy)};
        F.p[0] = (float)z1; F.p[1] = (float)hx0; F.p[2] = (float)hy0;
        for (int j = 0; j < 4; ++j) {
            F.p[3 + j] = (float)a[j];
            F.p[7 + j] = (float)(1.0 / sqrt(1.0 + a[j] * a[j]));
        }
        break;
    }
    case P_CAPSULE: {
        const double bb = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        for (int j = 0; j < 4; ++j) F.p[j] = (float)p[j];
        F.p[4] = bb > 0 ? (float)(1.0 / bb) : 0.f;
        F.p[5] = 0.f;  // segment parameter range [0, 1] in the canonical frame
        F.p[6] = 1.f;
        break;
    }
    case P_GRID:
    case P_REVOLVE:
    case P_POCKET: {
        // no Lipschitz bound (a table's jump to 1e6 outside its grid, the arch's vertical tangents):
        // an unbounded interval, so these elements are never culled and never cull another
        canon = 1.0e30;
        for (int j = 0; j < 10; ++j) F.p[j] = (float)p[j];
        const unsigned long long t = (unsigned long long)__double_as_longlong(p[10]);  // table address
        F.p[10] = __uint_as_float((unsigned)(t & 0xffffffffull));
        F.p[11] = __uint_as_float((unsigned)(t >> 32));
        break;
    }
    default:
        for (int j = 0; j < 12; ++j) F.p[j] = (float)p[j];
    }
    F.lip = (float)(fabs(P.s) * sqrt(row) * canon * (1.0 + 1e-6));
    // Bounding ball, for kinds whose canonical value is the exact Euclidean distance, of the
    // canonical solid (centre cc, radius rc).  When the frame map is a similarity (A_lin^T A_lin =
    // a^2 I) and s > 0, value(x) = s a d_world(x) - off with d_world the exact distance to the world
    // solid, which lies in the ball of centre A_lin^-1 (cc - t), radius rc / a: so
    //   s a (|x - c| - r) - off <= value(x) <= s a (|x - c| + r) - off.
    // Stored in the spare slots p[8..11] (these kinds read p[0..4] only), flagged by ball = 1.
    double cc[3] = {0.0, 0.0, 0.0}, rc = -1.0;
    switch (P.type) {
    case P_SPHERE: rc = p[0]; break;
    case P_BOX: rc = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]); break;
    case P_CYLINDER: rc = sqrt(p[0] * p[0] + p[1] * p[1]); break;
    case P_CAPSULE: {
        const double len = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        for (int c = 0; c < 3; ++c) cc[c] = 0.5 * p[c];
        rc = 0.5 * len + p[3];
        break;
    }
    case P_TORUS: rc = p[0] + p[1]; break;
    default: break;
    }
    const double a2 = (G[0][0] + G[1][1] + G[2][2]) / 3.0;
    bool similar = rc >= 0.0 && a2 > 0.0 && P.s > 0.0;
    for (int r = 0; r < 3 && similar; ++r)
        for (int c = 0; c < 3; ++c) similar &= fabs(G[r][c] - (r == c ? a2 : 0.0)) <= 1e-9 * a2;
    if (similar) {
        const double a = sqrt(a2);
        double cw[3];
        for (int c = 0; c < 3; ++c) {  // A_lin^-1 = A_lin^T / a^2 for a similarity
            double v = 0.0;
            for (int r = 0; r < 3; ++r) v += P.A[r * 4 + c] * (cc[r] - P.A[r * 4 + 3]);
            cw[c] = v / a2;
        }
        const double rw = rc / a;
        const double mag = fmax(fabs(cw[0]), fmax(fabs(cw[1]), fabs(cw[2])));
        F.ball = 1.f;
        F.ball_k = (float)(P.s * a);
        for (int c = 0; c < 3; ++c) F.p[8 + c] = (float)cw[c];
        F.p[11] = (float)(rw * (1.0 + 1e-6) + 1e-6 * mag);  // covers rounding the centre to float32
    }
    out[i] = F;
}

__global__ void k_prepare_prims(const FbPrim* __restrict__ prims, int n, PrimF* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) prepare_prim(prims, i, out);
}

// sqrt_sum over n inputs (the self-test export fb_sqrt_sum_probe).
__global__ void k_sqrt_sum(const float* __restrict__ x, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = sqrt_sum(x[i]);
}

__global__ void k_full_list(uint32_t* __restrict__ list, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) list[i] = (uint32_t)i << 2;
}

// ------------------------------------------------------------------------------------ culling
// One interval step of the chain walk.  Returns 0 skip, 1 keep, 2 reset to "set", 3 reset to
// "set negated".  [alo, ahi] bounds the accumulator over the region.
__device__ __forceinline__ int interval_step(int op, float k, float plo, float phi, float& alo, float& ahi) {
    switch (op) {
    case CH_SET:
        alo = plo; ahi = phi;
        return 2;
    case CH_SETNEG:
        alo = -phi; ahi = -plo;
        return 3;
    case CH_UNION:
        if (plo > ahi + k) return 0;
        if (phi < alo - k) { alo = plo; ahi = phi; return 2; }
        alo = fminf(alo, plo) - 0.25f * k;
        ahi = fminf(ahi, phi);
        return 1;
    case CH_INTERSECT:
        if (phi < alo - k) return 0;
        if (plo > ahi + k) { alo = plo; ahi = phi; return 2; }
        alo = fmaxf(alo, plo);
        ahi = fmaxf(ahi, phi) + 0.25f * k;
        return 1;
    case CH_SUBTRACT:
        if (-plo < alo - k) return 0;
        if (-phi > ahi + k) { alo = -phi; ahi = -plo; return 3; }
        alo = fmaxf(alo, -phi);
        ahi = fmaxf(ahi, -plo) + 0.25f * k;
        return 1;
    default:  // offset
        alo -= k; ahi -= k;
        return 1;
    }
}

__device__ __forceinline__ int effective_op(uint32_t entry, int op) {
    const uint32_t mode = entry & 3u;
    return mode == 1u ? CH_SET : (mode == 2u ? CH_SETNEG : op);
}

// Interval of one chain element's primitive around (cx, cy, cz) with radius R.
__device__ __forceinline__ void element_interval(const PrimF& P, float cx, float cy, float cz, float R, float eps,
                                                 float& lo, float& hi) {
    const float v = primf_world(P, cx, cy, cz);
    const float r = fmaf(P.lip, R, eps + 1e-6f * fabsf(v));
    lo = v - r;
    hi = v + r;
}

// A hard (k == 0) union / intersection / subtraction: consecutive ones of the same kind form a
// run whose result is an order-free min or max of the accumulator and the run's elements.
__device__ __forceinline__ bool runnable(int op, float k) {
    return k == 0.f && (op == CH_UNION || op == CH_INTERSECT || op == CH_SUBTRACT);
}

struct Elem {
    uint32_t ent;
    int op;
    float k;
    float lo, hi;  // bounds of the value the combine sees (-p for a subtraction)
};

// The same enclosure from the primitive's bounding ball (PrimF.ball == 1): no evaluation of the
// primitive, a few loads -- looser by up to the ball's diameter.
__device__ __forceinline__ void element_interval_ball(const PrimF& P, float cx, float cy, float cz, float R, float eps,
                                                      float& lo, float& hi) {
    const float dx = cx - P.p[8], dy = cy - P.p[9], dz = cz - P.p[10];
    const float d = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
    const float k = P.ball_k, rw = P.p[11];
    const float m = eps + 1e-6f * (k * (d + R + rw) + fabsf(P.off));
    lo = fmaf(k, d - R - rw, -P.off) - m;
    hi = fmaf(k, d + R + rw, -P.off) + m;
}

__device__ __forceinline__ Elem load_elem(const uint32_t* __restrict__ in, int e, const FbInsn* __restrict__ chain,
                                          const PrimF* __restrict__ primf, float cx, float cy, float cz, float R,
                                          float eps, bool with_bounds, bool ball = false) {
    Elem E;
    E.ent = in ? in[e] : (uint32_t)e << 2;  // a null list is the whole chain in order
    const FbInsn I = chain[E.ent >> 2];
    E.op = effective_op(E.ent, I.op);
    E.k = (float)I.k;
    E.lo = E.hi = 0.f;
    if (with_bounds && E.op != CH_OFFSET) {
        float lo, hi;
        const PrimF& P = primf[I.arg];
        if (ball && P.ball != 0.f) element_interval_ball(P, cx, cy, cz, R, eps, lo, hi);
        else element_interval(P, cx, cy, cz, R, eps, lo, hi);
        if (E.op == CH_SUBTRACT || E.op == CH_SETNEG) { E.lo = -hi; E.hi = -lo; }
        else { E.lo = lo; E.hi = hi; }
    }
    return E;
}

// Run decision.  union: result = min(acc, run); an element whose lower bound exceeds
// H = min(acc_hi, min run hi) is never the minimum and is dropped; when min run hi < acc_lo the
// accumulator so far is dominated everywhere and dropped (the run restarts the list).
// intersection / subtraction: the mirror image with max.  All comparisons are strict, so every
// decision is exact for the float values the bounds enclose.
struct RunState {
    float bound;   // H (union) or L (max kinds)
    bool reset;
};

__device__ __forceinline__ RunState run_decide(int op, float agg, float alo, float ahi) {
    RunState r;
    if (op == CH_UNION) {
        r.reset = agg < alo;
        r.bound = r.reset ? agg : fminf(ahi, agg);
    } else {
        r.reset = agg > ahi;
        r.bound = r.reset ? agg : fmaxf(alo, agg);
    }
    return r;
}

__device__ __forceinline__ bool run_keep(int op, const Elem& E, float bound) {
    return op == CH_UNION ? !(E.lo > bound) : !(E.hi < bound);
}

// Warp-cooperative chain walk over `in` for the region centred at (cx, cy, cz) with radius R.
// Hard runs are decided with two warp-parallel passes (aggregate bound, then keep/drop with
// ballot compaction); other elements (offsets, smooth booleans, sets) step one at a time.
// Returns the kept count (may exceed cap: then the output is incomplete and must not be used).
// kBall: bound primitives by their bounding balls where they have one (the coarse level, where
// every region walks the whole chain).
template <bool kBall = false>
__device__ int warp_walk(const uint32_t* __restrict__ in, int n_in, const FbInsn* __restrict__ chain,
                         const PrimF* __restrict__ primf, float cx, float cy, float cz, float R, float eps,
                         uint32_t* __restrict__ out, int cap) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    float alo = 0.f, ahi = 0.f;
    int n = 0;
    int i = 0;
    while (i < n_in) {
        const Elem head = load_elem(in, i, chain, primf, cx, cy, cz, R, eps, false);
        if (!runnable(head.op, head.k)) {
            const Elem E = load_elem(in, i, chain, primf, cx, cy, cz, R, eps, true);
            float plo = E.lo, phi = E.hi;  // back to the primitive's own bounds
            if (E.op == CH_SUBTRACT || E.op == CH_SETNEG) { plo = -E.hi; phi = -E.lo; }
            const int act = interval_step(E.op, E.k, plo, phi, alo, ahi);
            if (act) {
                uint32_t rec = E.ent;
                if (act == 2) { n = 0; rec = (E.ent & ~3u) | 1u; }
                if (act == 3) { n = 0; rec = (E.ent & ~3u) | 2u; }
                if (n < cap && lane == 0) out[n] = rec;
                ++n;
            }
            ++i;
            continue;
        }
        const int op = head.op;
        // pass 1, 32 elements at a time: the run's end (the first element of another kind) and the
        // aggregate bound of the elements before it.  With ball bounds the same pass also writes the
        // candidates: elements not beaten by the bound so far (the minimum over everything up to and
        // including their chunk) -- a superset of those the final bound keeps.
        float agg = op == CH_UNION ? 3.0e38f : -3.0e38f;
        int j = n_in;
        const int n0 = n;
        for (int b = i; b < n_in; b += 32) {
            const int e = b + lane;
            bool same = false;
            Elem E;
            if (e < n_in) {
                E = load_elem(in, e, chain, primf, cx, cy, cz, R, eps, true, kBall);
                same = e == i || (E.op == op && runnable(E.op, E.k));
            }
            const unsigned stop = __ballot_sync(0xffffffffu, e < n_in && !same);
            const int end = stop ? b + __ffs(stop) - 1 : min(b + 32, n_in);
            if (e < end) agg = op == CH_UNION ? fminf(agg, E.hi) : fmaxf(agg, E.lo);
            if (kBall) {
                float run = agg;
                for (int o = 16; o > 0; o >>= 1) {
                    const float t = __shfl_xor_sync(0xffffffffu, run, o);
                    run = op == CH_UNION ? fminf(run, t) : fmaxf(run, t);
                }
                const bool keep = e < end && run_keep(op, E, run);
                const unsigned kept = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int pos = n + __popc(kept & below);
                    if (pos < cap) out[pos] = E.ent;
                }
                n += __popc(kept);
            }
            if (stop) {
                j = end;
                break;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float t = __shfl_xor_sync(0xffffffffu, agg, o);
            agg = op == CH_UNION ? fminf(agg, t) : fmaxf(agg, t);
        }
        RunState rs = run_decide(op, agg, alo, ahi);
        float klo = 3.0e38f, khi = -3.0e38f;
        if (kBall) {
            // pass 1 wrote the candidates (every other element of the run provably loses, so the run's
            // result is the candidates' result); the exact bounds of the candidates alone give the
            // run's decision, and the candidates are compacted in place with it
            const int nc = n - n0;  // candidates at out[n0, n)
            if (n > cap) {          // overflowed: the region falls back to its parent's list anyway
                i = j;
                continue;
            }
            float agg2 = op == CH_UNION ? 3.0e38f : -3.0e38f;
            for (int b = 0; b < nc; b += 32) {
                if (b + lane < nc) {
                    const Elem E = load_elem(out + n0, b + lane, chain, primf, cx, cy, cz, R, eps, true);
                    agg2 = op == CH_UNION ? fminf(agg2, E.hi) : fmaxf(agg2, E.lo);
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const float t = __shfl_xor_sync(0xffffffffu, agg2, o);
                agg2 = op == CH_UNION ? fminf(agg2, t) : fmaxf(agg2, t);
            }
            rs = run_decide(op, agg2, alo, ahi);
            n = rs.reset ? 0 : n0;  // compaction target: positions never above the ones being read
            bool first = rs.reset;
            for (int b = 0; b < nc; b += 32) {
                bool keep = false;
                Elem E;
                if (b + lane < nc) {
                    E = load_elem(out + n0, b + lane, chain, primf, cx, cy, cz, R, eps, true);
                    keep = run_keep(op, E, rs.bound);
                    if (keep) { klo = fminf(klo, E.lo); khi = fmaxf(khi, E.hi); }
                }
                const unsigned kept = __ballot_sync(0xffffffffu, keep);  // every read precedes the writes
                if (keep) {
                    const int pos = n + __popc(kept & below);
                    uint32_t rec = E.ent;
                    if (first && pos == 0) rec = (E.ent & ~3u) | (op == CH_SUBTRACT ? 2u : 1u);
                    out[pos] = rec;
                }
                if (kept) first = false;
                n += __popc(kept);
            }
        } else {
            if (rs.reset) n = 0;
            bool first = rs.reset;
            // pass 2: keep / drop, ballot compaction in chain order
            for (int b = i; b < j; b += 32) {
                const int e = b + lane;
                bool keep = false;
                Elem E;
                if (e < j) {
                    E = load_elem(in, e, chain, primf, cx, cy, cz, R, eps, true);
                    keep = run_keep(op, E, rs.bound);
                    if (keep) { klo = fminf(klo, E.lo); khi = fmaxf(khi, E.hi); }
                }
                const unsigned kept = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int pos = n + __popc(kept & below);
                    uint32_t rec = E.ent;
                    if (first && pos == 0) rec = (E.ent & ~3u) | (op == CH_SUBTRACT ? 2u : 1u);
                    if (pos < cap) out[pos] = rec;
                }
                if (kept) first = false;
                n += __popc(kept);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            klo = fminf(klo, __shfl_xor_sync(0xffffffffu, klo, o));
            khi = fmaxf(khi, __shfl_xor_sync(0xffffffffu, khi, o));
        }
        if (op == CH_UNION) {
            alo = rs.reset ? klo : fminf(alo, klo);
            ahi = rs.bound;
        } else {
            alo = rs.bound;
            ahi = rs.reset ? khi : fmaxf(ahi, khi);
        }
        i = j;
    }
    return n;
}

// The same walk by one thread (each block's own list in k_classify_blocks): the lanes of a warp
// walk the same superblock list together, so its loads are broadcasts.
__device__ int seq_walk(const uint32_t* __restrict__ in, int n_in, const FbInsn* __restrict__ chain,
                        const PrimF* __restrict__ primf, float cx, float cy, float cz, float R, float eps,
                        uint32_t* __restrict__ out, int cap) {
    float alo = 0.f, ahi = 0.f;
    int n = 0;
    int i = 0;
    while (i < n_in) {
        const Elem head = load_elem(in, i, chain, primf, cx, cy, cz, R, eps, false);
        if (!runnable(head.op, head.k)) {
            const Elem E = load_elem(in, i, chain, primf, cx, cy, cz, R, eps, true);
            float plo = E.lo, phi = E.hi;  // back to the primitive's own bounds
            if (E.op == CH_SUBTRACT || E.op == CH_SETNEG) { plo = -E.hi; phi = -E.lo; }
            const int act = interval_step(E.op, E.k, plo, phi, alo, ahi);
            if (act) {
                uint32_t rec = E.ent;
                if (act == 2) { n = 0; rec = (E.ent & ~3u) | 1u; }
                if (act == 3) { n = 0; rec = (E.ent & ~3u) | 2u; }
                if (n < cap) out[n] = rec;
                ++n;
            }
            ++i;
            continue;
        }
        const int op = head.op;
        // pass 1: the run's end and its aggregate bound in one traversal
        float agg = op == CH_UNION ? 3.0e38f : -3.0e38f;
        int j = i;
        while (j < n_in) {
            const Elem E = load_elem(in, j, chain, primf, cx, cy, cz, R, eps, true);
            if (j > i && !(E.op == op && runnable(E.op, E.k))) break;
            agg = op == CH_UNION ? fminf(agg, E.hi) : fmaxf(agg, E.lo);
            ++j;
        }
        const RunState rs = run_decide(op, agg, alo, ahi);
        if (rs.reset) n = 0;
        bool first = rs.reset;
        float klo = 3.0e38f, khi = -3.0e38f;
        for (int e = i; e < j; ++e) {
            const Elem E = load_elem(in, e, chain, primf, cx, cy, cz, R, eps, true);
            if (!run_keep(op, E, rs.bound)) continue;
            klo = fminf(klo, E.lo);
            khi = fmaxf(khi, E.hi);
            uint32_t rec = E.ent;
            if (first) rec = (E.ent & ~3u) | (op == CH_SUBTRACT ? 2u : 1u);
            first = false;
            if (n < cap) out[n] = rec;
            ++n;
        }
        if (op == CH_UNION) {
            alo = rs.reset ? klo : fminf(alo, klo);
            ahi = rs.bound;
        } else {
            alo = rs.bound;
            ahi = rs.reset ? khi : fmaxf(ahi, khi);
        }
        i = j;
    }
    return n;
}

// Level cull.  Regions of `edge` voxels on a (rnx, rny, rnz) grid; parent region = coords / div
// on a (pnx, pny, pnz) grid (parent_off == nullptr: the single full list [0, n_full)).
template <bool kBall>
__device__ void cull_region(const Geo& G, const FbInsn* __restrict__ chain, const PrimF* __restrict__ primf,
                            uint32_t* __restrict__ pool, const int64_t* __restrict__ parent_off,
                            const int32_t* __restrict__ parent_len, int n_full, int div, int pny, int pnz,
                            int64_t* __restrict__ off, int32_t* __restrict__ len, int64_t pool_base, int cap, int edge,
                            int rny, int rnz, int64_t r) {
    const int rz = (int)(r % rnz), ry = (int)((r / rnz) % rny), rx = (int)(r / ((int64_t)rnz * rny));
    int64_t poff = 0;
    int plen = n_full;
    if (parent_off) {
        const int64_t pr = ((int64_t)(rx / div) * pny + ry / div) * pnz + rz / div;
        poff = parent_off[pr];
        plen = parent_len[pr];
    }
    const float half = 0.5f * edge;
    const float cx = G.fx0 + (rx * edge + half) * G.fpitch;
    const float cy = G.fy0 + (ry * edge + half) * G.fpitch;
    const float cz = G.fz0 + (rz * edge + half) * G.fpitch;
    const float R = 1.7320509f * half * G.fpitch;
    uint32_t* dst = pool + pool_base + r * cap;
    const int n = warp_walk<kBall>(parent_off ? pool + poff : nullptr, plen, chain, primf, cx, cy, cz, R, G.eps, dst,
                                   cap);
    if ((threadIdx.x & 31) == 0) {
        if (n <= cap) {
            off[r] = pool_base + r * cap;
            len[r] = n;
        } else {  // overflow: the region keeps its parent's list (still exact, only slower)
            off[r] = poff;
            len[r] = plen;
        }
    }
}

template <bool kBall>
__global__ void k_cull(Geo G, const FbInsn* __restrict__ chain, const PrimF* __restrict__ primf,
                       uint32_t* __restrict__ pool, const int64_t* __restrict__ parent_off,
                       const int32_t* __restrict__ parent_len, int n_full, int div, int pny, int pnz,
                       int64_t* __restrict__ off, int32_t* __restrict__ len, int64_t pool_base, int cap, int edge,
                       int rnx, int rny, int rnz) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (r >= (int64_t)rnx * rny * rnz) return;
    cull_region<kBall>(G, chain, primf, pool, parent_off, parent_len, n_full, div, pny, pnz, off, len, pool_base, cap,
                       edge, rny, rnz, r);
}


// ------------------------------------------------------------------------------------ localisation
// ------------------------------------------------------------------------------------ classify
// float64 value of a block list at a world point (guard-band recheck).
__device__ __noinline__ double list_eval_d(const uint32_t* __restrict__ list, int n, const FbInsn* __restrict__ chain,
                              const FbPrim* __restrict__ prims, double x, double y, double z) {
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
        const uint32_t e = list[i];
        const FbInsn I = chain[e >> 2];
        const int op = effective_op(e, I.op);
        const double v = op == CH_OFFSET ? 0.0 : prim_world_d(prims[I.arg], x, y, z);
        acc = chain_apply_d(op, acc, v, I.k);
    }
    return acc;
}

// Threads of one superblock are consecutive (a warp never spans two superblocks in the chain
// mode), so the walk over the superblock's list runs in lockstep with broadcast loads.
__host__ __device__ __forceinline__ int threads_per_super(int S) {
    const int n = S * S * S;
    return n >= 32 ? (n + 31) / 32 * 32 : n;  // 1 or 8: several superblocks share a warp
}

// Kind and corner_min_abs of one block from its 8 corner values: float32 decisions unless a corner
// lies within the guard band of 0 or of the margin (or is NaN); then all 8 corners are re-evaluated
// in float64 by `corner_d(c)` and the decision is taken in float64, exactly as the oracle's.
template <typename CornerD>
__device__ __forceinline__ int decide_block(const Geo& G, const float* v, float& cma_out, CornerD corner_d) {
    bool use_d = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float a = fabsf(v[c]);
        use_d |= a < G.guard || fabsf(a - G.margin) < G.guard || !(a == a);
    }
    bool pos = false, neg = false;
    if (use_d) {
        double mn = 1.0e30;
        for (int c = 0; c < 8; ++c) {
            const double vd = corner_d(c);
            mn = fmin(mn, fabs(vd));
            if (vd >= 0.0) pos = true; else neg = true;
        }
        cma_out = (float)mn;
        return (pos && neg) ? 0 : (mn <= (double)G.margin ? 0 : (neg ? -1 : 1));
    }
    float mn = 1.0e30f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        mn = fminf(mn, fabsf(v[c]));
        if (v[c] >= 0.f) pos = true; else neg = true;
    }
    cma_out = mn;
    return (pos && neg) ? 0 : (mn <= G.margin ? 0 : (neg ? -1 : 1));
}

// World coordinate of grid vertex index i along one axis, in float64 (the oracle's sample point).
__device__ __forceinline__ double vertex_d(double origin, int64_t i, double pitch) {
    return rn_add(origin, rn_mul((double)i, pitch));
}

// Thread-per-block classification of a chain recipe: thread t of the superblock-major order --
// threads of one superblock are consecutive, so a warp never spans two superblocks and walks in
// lockstep with broadcast loads -- evaluates its block's 8 corners in float32 in block-local
// coordinates.  The block culls the superblock list itself (seq_walk, kCapBlock entries) and an
// active block keeps that list for the leaf pass and point queries: the warp's lists are
// placed with one atomicAdd on `cursor` (blk_len -1 where a list overflowed or the pool is full;
// the leaf pass then culls the block itself).  Every lane of a warp reaches the placement, so
// threads outside the grid only skip the evaluation.
template <int VG, bool kEdge = true>
__device__ __forceinline__ uint32_t eval_group(const LocalPrim& P, float dx, float dy, const float* dz, float* v);
template <int VG>
__device__ __forceinline__ void combine_group(int op, float k, float* acc, const float* v);

__device__ void classify_block(const Geo& G, const FbPrim* __restrict__ prims, const PrimF* __restrict__ primf,
                               const FbInsn* __restrict__ chain, const uint32_t* __restrict__ pool,
                               const int64_t* __restrict__ sb_off, const int32_t* __restrict__ sb_len,
                               int32_t* __restrict__ kind, float* __restrict__ cma, int32_t* __restrict__ blk_off,
                               int32_t* __restrict__ blk_len, uint32_t* __restrict__ blk_pool, int64_t blk_cap,
                               int* __restrict__ cursor, int64_t t) {
    const int S = G.S;
    const int T = threads_per_super(S);
    const int64_t s_id = t / T;
    const int local = (int)(t % T);
    const int sz = (int)(s_id % G.nsz), sy = (int)((s_id / G.nsz) % G.nsy), sx = (int)(s_id / ((int64_t)G.nsz * G.nsy));
    const int bi = sx * S + local / (S * S), bj = sy * S + (local / S) % S, bk = sz * S + local % S;
    const bool valid = s_id < G.nsuper && local < S * S * S && bi < G.nbx && bj < G.nby && bk < G.nbz;
    const int64_t b = ((int64_t)bi * G.nby + bj) * G.nbz + bk;
    const int B = G.B;
    uint32_t blist[kCapBlock];
    int nblist = -1;
    int kd = 1;
    if (valid) {
        const uint32_t* list;
        int len;
        const uint32_t* plist = pool + sb_off[s_id];
        const int plen = sb_len[s_id];
        const float half = 0.5f * B;
        const int n = seq_walk(plist, plen, chain, primf, G.fx0 + (bi * B + half) * G.fpitch,
                               G.fy0 + (bj * B + half) * G.fpitch, G.fz0 + (bk * B + half) * G.fpitch,
                               1.7320509f * half * G.fpitch, G.eps, blist, kCapBlock);
        nblist = n;
        list = n <= kCapBlock ? blist : plist;
        len = n <= kCapBlock ? n : plen;
        const double ox = G.x0 + (double)(bi * B) * G.pitch;
        const double oy = G.y0 + (double)(bj * B) * G.pitch;
        const double oz = G.z0 + (double)(bk * B) * G.pitch;
        const float side = (float)B * G.fpitch;
        float v[8];
        bool edge = false;  // a corner sampled a grid table at its boundary: decide in float64
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = 0.f;
        for (int i = 0; i < len; ++i) {
            const uint32_t e = list[i];
            const FbInsn I = chain[e >> 2];
            const int op = effective_op(e, I.op);
            const float k = (float)I.k;
            if (op == CH_OFFSET) {
#pragma unroll
                for (int c = 0; c < 8; ++c) v[c] -= k;
                continue;
            }
            LocalPrim P;
            // canonical forms (no extent): the corner decisions have the float64 guard band
            localise(prims[I.arg], primf[I.arg], ox, oy, oz, op, k, P);
            // the corners as 4 (x, y) columns of 2 along z: one inlined evaluation body (the kind
            // switch outside, the points inside) walked over the columns, the corner values rotated
            // through registers -- 8 unrolled kind switches would not fit the instruction cache
            const float dz2[2] = {0.f, side};
            for (int col = 0; col < 4; ++col) {
                float pv[2], acc2[2] = {v[0], v[4]};
                edge |= eval_group<2>(P, (col & 1) ? side : 0.f, (col & 2) ? side : 0.f, dz2, pv) != 0;
                combine_group<2>(op, k, acc2, pv);
                const float t0 = acc2[0], t4 = acc2[1];
                v[0] = v[1]; v[1] = v[2]; v[2] = v[3]; v[3] = t0;
                v[4] = v[5]; v[5] = v[6]; v[6] = v[7]; v[7] = t4;
            }
        }
        if (edge) v[0] = __int_as_float(0x7fc00000);  // NaN: decide_block takes the float64 path
        float m;
        kd = decide_block(G, v, m, [&](int c) {
            return list_eval_d(list, len, chain, prims, vertex_d(G.x0, (int64_t)bi * B + (c & 1) * B, G.pitch),
                               vertex_d(G.y0, (int64_t)bj * B + ((c >> 1) & 1) * B, G.pitch),
                               vertex_d(G.z0, (int64_t)bk * B + ((c >> 2) & 1) * B, G.pitch));
        });
        kind[b] = kd;
        cma[b] = m;
    }
    {
        // the warp's active blocks' lists: an inclusive scan of their lengths, one atomicAdd
        const int lane = threadIdx.x & 31;
        const bool keep = valid && kd == 0 && nblist >= 0 && nblist <= kCapBlock;
        const int need = keep ? nblist : 0;
        int incl = need;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int base = 0;
        if (lane == 31 && total > 0) base = atomicAdd(cursor, total);
        base = __shfl_sync(0xffffffffu, base, 31);
        if (valid && kd == 0) {
            const int64_t slot = (int64_t)base + incl - need;
            int len_b = -1;
            if (keep && slot + need <= blk_cap) {
                for (int i = 0; i < need; ++i) blk_pool[slot + i] = blist[i];
                blk_off[b] = (int32_t)slot;
                len_b = need;
            }
            blk_len[b] = len_b;  // -1: the leaf pass culls the block itself
        }
    }
}

// 6 CTAs per SM (80 registers): measured against 8 and 10 (64 / 48 registers, more spills) and 4.
__global__ void __launch_bounds__(128, 6) k_classify_blocks(Geo G, const FbPrim* __restrict__ prims,
                                                             const PrimF* __restrict__ primf,
                                                             const FbInsn* __restrict__ chain,
                                                             const uint32_t* __restrict__ pool,
                                                             const int64_t* __restrict__ sb_off,
                                                             const int32_t* __restrict__ sb_len,
                                                             int32_t* __restrict__ kind, float* __restrict__ cma,
                                                             int32_t* __restrict__ blk_off, int32_t* __restrict__ blk_len,
                                                             uint32_t* __restrict__ blk_pool, int64_t blk_cap,
                                                             int* __restrict__ cursor) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    classify_block(G, prims, primf, chain, pool, sb_off, sb_len, kind, cma, blk_off, blk_len, blk_pool, blk_cap, cursor,
                   t);
}

// General postfix programs: every corner of every block in float64, no culling.
__global__ void __launch_bounds__(128) k_classify_program(Geo G, const FbPrim* __restrict__ prims,
                                                          const FbInsn* __restrict__ prog, int n_prog,
                                                          int32_t* __restrict__ kind, float* __restrict__ cma) {
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= G.nblocks) return;
    const int bk = (int)(b % G.nbz), bj = (int)((b / G.nbz) % G.nby), bi = (int)(b / ((int64_t)G.nbz * G.nby));
    const int B = G.B;
    double mn = 1.0e30;
    bool pos = false, neg = false;
    for (int c = 0; c < 8; ++c) {
        const double vd = program_eval_d(prims, prog, n_prog, vertex_d(G.x0, (int64_t)bi * B + (c & 1) * B, G.pitch),
                                         vertex_d(G.y0, (int64_t)bj * B + ((c >> 1) & 1) * B, G.pitch),
                                         vertex_d(G.z0, (int64_t)bk * B + ((c >> 2) & 1) * B, G.pitch));
        mn = fmin(mn, fabs(vd));
        if (vd >= 0.0) pos = true; else neg = true;
    }
    kind[b] = (pos && neg) ? 0 : (mn <= (double)G.margin ? 0 : (neg ? -1 : 1));
    cma[b] = (float)mn;
}

// ------------------------------------------------------------------------------------ compaction
// Single-pass scan with decoupled look-back over tiles of kTile block kinds.  Tiles are claimed in
// order from a ticket counter, so every predecessor is already running when a tile waits on it;
// each wait is bounded and a timeout raises the error flag instead of hanging.
__device__ __forceinline__ unsigned long long ld_status(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

constexpr long long kLookbackSpins = 1ll << 24;  // ~0.5 s of 32 ns sleeps before a wait gives up

// One tile of the scan.  `tile` is this CTA's tile of the kind array, taken in order from a ticket
// counter by the caller (so every predecessor tile is already running); `err` is raised when a wait
// gives up.  Every thread of the CTA calls it.
__device__ void compact_tile(const int32_t* __restrict__ kind, int64_t n, int32_t* __restrict__ active,
                             int32_t* __restrict__ count, unsigned long long* __restrict__ status, int64_t tile,
                             int64_t ntiles, int* __restrict__ err, long long spin_limit) {
    __shared__ int s_warp[8];
    __shared__ long long s_prefix;
    const int64_t base = tile * kTile + (int64_t)threadIdx.x * 8;
    unsigned flags = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t i = base + j;
        if (i < n && kind[i] == 0) flags |= 1u << j;
    }
    const int c = __popc(flags);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    int wbase = 0, total = 0;
    for (int w = 0; w < 8; ++w) {
        if (w < warp) wbase += s_warp[w];
        total += s_warp[w];
    }
    const int excl = wbase + incl - c;
    constexpr unsigned long long kAgg = 1ull << 62, kInc = 2ull << 62, kMask = (1ull << 62) - 1;
    if (threadIdx.x == 0) {
        long long prefix = 0;
        if (tile == 0) {
            atomicExch(&status[0], kInc | (unsigned long long)total);
        } else {
            atomicExch(&status[tile], kAgg | (unsigned long long)total);
            int64_t j = tile - 1;
            long long spins = 0;
            while (j >= 0) {
                const unsigned long long s = ld_status(&status[j]);
                const unsigned long long flag = s & ~kMask;
                if (flag == 0) {
                    if (++spins > spin_limit) {
                        atomicExch(err, 1);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                prefix += (long long)(s & kMask);
                if (flag == kInc) break;
                --j;
            }
            __threadfence();
            atomicExch(&status[tile], kInc | (unsigned long long)(prefix + total));
        }
        s_prefix = prefix;
        if (tile == ntiles - 1) count[0] = (int32_t)(prefix + total);
    }
    __syncthreads();
    const long long start = s_prefix + excl;
    int k = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if (flags & (1u << j)) active[start + k++] = (int32_t)(base + j);
}

__global__ void __launch_bounds__(256) k_compact(const int32_t* __restrict__ kind, int64_t n,
                                                 int32_t* __restrict__ active, int32_t* __restrict__ count,
                                                 unsigned long long* __restrict__ status, int* __restrict__ misc,
                                                 int64_t ntiles, long long spin_limit) {
    __shared__ int s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(&misc[0], 1);
    __syncthreads();
    compact_tile(kind, n, active, count, status, s_tile, ntiles, &misc[1], spin_limit);
}

// ------------------------------------------------------------------------------------ leaf eval

// Canonical primitive of a fixed type (the switch is taken once per primitive and group of
// voxels, not once per voxel, which keeps the evaluation loop small enough for the i-cache).
template <int T>
__device__ __forceinline__ float canon_t(const float* __restrict__ p, float x, float y, float z) {
    // z-dependent terms outermost: across a group of voxels along z the x/y parts are shared
    if (T == P_SPHERE) return sqrt_sum(fmaf(z, z, fmaf(x, x, y * y))) - p[0];
    if (T == P_BOX) {
        const float qx = fabsf(x) - p[0], qy = fabsf(y) - p[1], qz = fabsf(z) - p[2];
        const float ox = fmaxf(qx, 0.f), oy = fmaxf(qy, 0.f), oz = fmaxf(qz, 0.f);
        return sqrt_sum(fmaf(oz, oz, fmaf(ox, ox, oy * oy))) + fminf(fmaxf(qz, fmaxf(qx, qy)), 0.f);
    }
    if (T == P_CAPSULE) {
        const float h = fminf(fmaxf(fmaf(z, p[2], fmaf(x, p[0], y * p[1])) * p[4], p[5]), p[6]);
        const float dx = fmaf(-p[0], h, x), dy = fmaf(-p[1], h, y), dz = fmaf(-p[2], h, z);
        return sqrt_sum(fmaf(dz, dz, fmaf(dx, dx, dy * dy))) - p[3];
    }
    if (T == P_TORUS) {
        const float qx = sqrt_sum(fmaf(x, x, y * y)) - p[0];
        return sqrt_sum(fmaf(z, z, qx * qx)) - p[1];
    }
    return canon_f(T, p, x, y, z);
}

// Sphere in difference form: with q = L + e (e the voxel's offset in the sphere's frame),
// |q| - r = (|L|^2 - r^2 + e.(2L + e)) / (|q| + r).  The constant |L|^2 - r^2 is formed in float64 per
// block (LocalPrim.L[3]); the numerator then carries only small per-voxel terms, so the error stays
// near one rounding of the value instead of growing with the sphere's size (coordinates of up to
// ~50 pitches put the direct form near 1e-5 pitch).
template <int VG>
__device__ __forceinline__ void eval_group_sphere(const LocalPrim& P, float dx, float dy, const float* dz, float* v) {
    const float L0 = P.L[0], L1 = P.L[1], L2 = P.L[2], K = P.L[3], r = P.p[0];
    float ebx, eby, ebz, cx, cy, cz;  // e = eb + c * dz
    if (P.ident) {
        ebx = dx; eby = dy; ebz = 0.f; cx = 0.f; cy = 0.f; cz = 1.f;
    } else {
        ebx = fmaf(P.A[0], dx, P.A[1] * dy);
        eby = fmaf(P.A[3], dx, P.A[4] * dy);
        ebz = fmaf(P.A[6], dx, P.A[7] * dy);
        cx = P.A[2]; cy = P.A[5]; cz = P.A[8];
    }
#pragma unroll
    for (int k = 0; k < VG; ++k) {
        const float ex = fmaf(cx, dz[k], ebx), ey = fmaf(cy, dz[k], eby), ez = fmaf(cz, dz[k], ebz);
        const float x = L0 + ex, y = L1 + ey, z = L2 + ez;
        const float num = fmaf(ez, fmaf(2.f, L2, ez), fmaf(ey, fmaf(2.f, L1, ey), fmaf(ex, fmaf(2.f, L0, ex), K)));
        const float den = sqrt_sum(fmaf(z, z, fmaf(x, x, y * y))) + r;
        v[k] = fmaf(P.s, __fdiv_rn(num, den), -P.off);
    }
}

// VG voxels along z of one lane: values of primitive P at block offsets (dx, dy, dz0 + k*pz).
template <int VG, int T>
__device__ __forceinline__ void eval_group_t(const LocalPrim& P, float dx, float dy, const float* dz, float* v) {
    if (T == P_SPHERE && P.diff) {
        eval_group_sphere<VG>(P, dx, dy, dz, v);
        return;
    }
    const float* p = P.p;
    if (P.ident) {
        const float x = P.L[0] + dx, y = P.L[1] + dy;
#pragma unroll
        for (int k = 0; k < VG; ++k) v[k] = fmaf(P.s, canon_t<T>(p, x, y, P.L[2] + dz[k]), -P.off);
    } else {
        const float bx = fmaf(P.A[0], dx, fmaf(P.A[1], dy, P.L[0]));
        const float by = fmaf(P.A[3], dx, fmaf(P.A[4], dy, P.L[1]));
        const float bz = fmaf(P.A[6], dx, fmaf(P.A[7], dy, P.L[2]));
#pragma unroll
        for (int k = 0; k < VG; ++k)
            v[k] = fmaf(P.s, canon_t<T>(p, fmaf(P.A[2], dz[k], bx), fmaf(P.A[5], dz[k], by), fmaf(P.A[8], dz[k], bz)),
                        -P.off);
    }
}

// The kinds the milling recipes rarely use, out of line and one voxel per call (scalar arguments
// stay in registers): the hot loop keeps only the four common kinds inlined, small enough to stay in
// the instruction cache.  A sampled grid's voxel next to its table's boundary
// (grid_edge_f) returns NaN: the caller marks it for the float64 recheck -- one call site, so the
// hot loop keeps a single call on its rare path.
__device__ __noinline__ float eval_one_rare(const LocalPrim& P, float dx, float dy, float dz) {
    float x, y, z;
    if (P.ident) {
        x = P.L[0] + dx; y = P.L[1] + dy; z = P.L[2] + dz;
    } else {
        x = fmaf(P.A[2], dz, fmaf(P.A[0], dx, fmaf(P.A[1], dy, P.L[0])));
        y = fmaf(P.A[5], dz, fmaf(P.A[3], dx, fmaf(P.A[4], dy, P.L[1])));
        z = fmaf(P.A[8], dz, fmaf(P.A[6], dx, fmaf(P.A[7], dy, P.L[2])));
    }
    if (P.type == P_GRID && grid_edge_f(P.p, x, y, z)) return __int_as_float(0x7fc00000);
    return fmaf(P.s, canon_f(P.type, P.p, x, y, z), -P.off);
}

// A torus in its ring frame (localise): u = x - R and w = y of the rotated frame, rho - R =
// u + w^2 / (rho + R + u); the quotient is a correction of a few pitches, so the fast division's two
// ulps of it stay far below the float32 rounding of the coordinates themselves.  Out of line, and
// only in the leaf kernels built for recipes with such tori: in the common kernel's loop the extra
// path cost the leaf pass 10-20 % even where it never ran.
template <int VG>
struct Vals {
    float v[VG];
};

template <int VG>
__device__ __noinline__ Vals<VG> eval_group_torus_ring(const LocalPrim& P, float dx, float dy, const float* dz) {
    Vals<VG> out;
    const float L0 = P.L[0], L2 = P.L[2], R = P.p[0], r = P.p[1];
    const float ebx = fmaf(P.A[0], dx, P.A[1] * dy), eby = fmaf(P.A[3], dx, P.A[4] * dy),
                ebz = fmaf(P.A[6], dx, P.A[7] * dy);
#pragma unroll
    for (int k = 0; k < VG; ++k) {
        const float u = L0 + fmaf(P.A[2], dz[k], ebx), w = fmaf(P.A[5], dz[k], eby), z = L2 + fmaf(P.A[8], dz[k], ebz);
        const float t = R + u;  // x of the rotated frame: <= 0 only past the axis (a block across it)
        const float rho = sqrt_sum(fmaf(t, t, w * w));
        const float qx = t > 0.f ? u + __fdividef(w * w, rho + t) : rho - R;
        out.v[k] = fmaf(P.s, sqrt_sum(fmaf(z, z, qx * qx)) - r, -P.off);
    }
    return out;
}

// Returns bit k set where voxel k sampled a grid table next to its boundary (eval_one_rare's NaN):
// its value and the decisions on it are then taken in float64.  kEdge = false: recipes with neither
// sampled-grid leaves nor ring-frame tori (fb_geom.reserved[0] bits 0-1), whose leaf loop then
// carries neither the marks nor the ring path.
template <int VG, bool kEdge>
__device__ __forceinline__ uint32_t eval_group(const LocalPrim& P, float dx, float dy, const float* dz, float* v) {
    uint32_t edge = 0;
    switch (P.type) {
    case P_SPHERE: eval_group_t<VG, P_SPHERE>(P, dx, dy, dz, v); break;
    case P_BOX: eval_group_t<VG, P_BOX>(P, dx, dy, dz, v); break;
    case P_CAPSULE: eval_group_t<VG, P_CAPSULE>(P, dx, dy, dz, v); break;
    case P_TORUS:
        if (kEdge && P.diff) {
            const Vals<VG> r = eval_group_torus_ring<VG>(P, dx, dy, dz);
#pragma unroll
            for (int k = 0; k < VG; ++k) v[k] = r.v[k];
        } else {
            eval_group_t<VG, P_TORUS>(P, dx, dy, dz, v);
        }
        break;
    default:
#pragma unroll
        for (int k = 0; k < VG; ++k) {
            v[k] = eval_one_rare(P, dx, dy, dz[k]);
            if (kEdge) edge |= (uint32_t)!(v[k] == v[k]) << k;
        }
    }
    return edge;
}

// acc = op(acc, v) for the VG voxels; the operator switch is taken once.
template <int VG>
__device__ __forceinline__ void combine_group(int op, float k, float* acc, const float* v) {
    if (k > 0.f) {
#pragma unroll
        for (int j = 0; j < VG; ++j) acc[j] = chain_apply(op, acc[j], v[j], k);
        return;
    }
    switch (op) {
    case CH_SET:
#pragma unroll
        for (int j = 0; j < VG; ++j) acc[j] = v[j];
        break;
    case CH_SETNEG:
#pragma unroll
        for (int j = 0; j < VG; ++j) acc[j] = -v[j];
        break;
    case CH_UNION:
#pragma unroll
        for (int j = 0; j < VG; ++j) acc[j] = sel_min(acc[j], v[j]);
        break;
    case CH_INTERSECT:
#pragma unroll
        for (int j = 0; j < VG; ++j) acc[j] = sel_max(acc[j], v[j]);
        break;
    default:  // subtraction
#pragma unroll
        for (int j = 0; j < VG; ++j) acc[j] = sel_max(acc[j], -v[j]);
    }
}

__device__ __noinline__ double guard_value(const uint32_t* __restrict__ list, int len, const FbInsn* __restrict__ chain,
                                           const FbPrim* __restrict__ prims, const Geo& G, int64_t ix, int64_t iy,
                                           int64_t iz) {
    return list_eval_d(list, len, chain, prims, rn_add(G.x0, rn_mul((double)ix, G.pitch)),
                       rn_add(G.y0, rn_mul((double)iy, G.pitch)), rn_add(G.z0, rn_mul((double)iz, G.pitch)));
}

// float32 operations of one localised primitive evaluation (affine + canonical formula + scale),
// counting an FMA as two; the executed-work basis of the float32-pipe roofline.
__device__ __forceinline__ unsigned prim_flops(int type, int ident) {
    const unsigned affine = ident ? 3u : 18u;
    unsigned f;
    switch (type) {
    case P_SPHERE: f = 7; break;      // 2 fma + mul + sqrt + sub
    case P_BOX: f = 19; break;
    case P_CYLINDER: f = 15; break;
    case P_CONE: f = 22; break;
    case P_HALFSPACE: f = 5; break;
    case P_FRUSTUM: f = 30; break;
    case P_CAPSULE: f = 22; break;
    case P_TORUS: f = 12; break;
    case P_GRID: f = 40; break;
    case P_REVOLVE: f = 32; break;
    case P_BAR: f = 9; break;
    case P_POCKET: f = 24; break;
    case P_XBORE: f = 9; break;
    default: f = 5;
    }
    return affine + f + 2;
}

// One lane's group of VG consecutive voxels: vector stores, coalesced across the warp.
template <int VG>
__device__ __forceinline__ void store_group(float* out, int group, const float* acc) {
    if (VG == 8) {
        float4* o = reinterpret_cast<float4*>(out) + 2 * group;
        o[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
        o[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
    } else if (VG == 4) {
        reinterpret_cast<float4*>(out)[group] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    } else {
        reinterpret_cast<float2*>(out)[group] = make_float2(acc[0], acc[1]);
    }
}

template <int VG>
__device__ __forceinline__ void load_group(const float* out, int group, float* acc) {
    if (VG == 8) {
        const float4* o = reinterpret_cast<const float4*>(out) + 2 * group;
        const float4 a = o[0], b = o[1];
        acc[0] = a.x; acc[1] = a.y; acc[2] = a.z; acc[3] = a.w;
        acc[4] = b.x; acc[5] = b.y; acc[6] = b.z; acc[7] = b.w;
    } else if (VG == 4) {
        const float4 a = reinterpret_cast<const float4*>(out)[group];
        acc[0] = a.x; acc[1] = a.y; acc[2] = a.z; acc[3] = a.w;
    } else {
        const float2 a = reinterpret_cast<const float2*>(out)[group];
        acc[0] = a.x; acc[1] = a.y;
    }
}


// ------------------------------------------------------------------------------------ 8^3 tiles
// An 8^3 block's tile, primitive by primitive over all 512 voxels: lane l owns voxels
// (2g + l/16, (l/2) % 8, 4 (l % 2) + k) for g, k in 0..3 -- the voxels, and the float operations in
// their order, of the grouped loop below -- and keeps their running values in shared memory (one
// float4 per group), so a staged primitive is read and dispatched once per 16 voxels rather than
// once per 4, while the kind bodies stay one group long (a loop over the 4 groups, small enough for
// the instruction cache).  The per-voxel arithmetic of the common kinds runs on float32 pairs
// (FFMA2 / FADD2 / FMUL2 on sm_100: two voxels per instruction, each element rounded as its scalar
// form), so the tiles equal the grouped loop's bit for bit.  Hard combines have the subtraction's
// sign folded into the primitive's scale at staging and take one min or max per voxel; a set starts
// from NaN, which min replaces.  Smooth combines, the rarely used kinds and the common kinds in a
// general frame go voxel by voxel through the out-of-line evaluation.
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 abs2(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float2 max2(float2 a, float b) { return make_float2(fmaxf(a.x, b), fmaxf(a.y, b)); }

// num / den for den > 0 (a sum with a positive radius): one Newton step from the approximate
// reciprocal y, q = q0 + y (num - q0 den) with q0 = num y and the residual formed exactly by one FMA
// (Markstein's correction, as for sqrt_sum).  Branch-free; tests/test_prims_gpu.py compares it with
// the IEEE quotient.
__device__ __forceinline__ float2 quotient2(float2 num, float2 den) {
    float2 y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(den.x));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(den.y));
    const float2 q0 = mul2(num, y);
    return fma2(fma2(neg2(q0), den, num), y, q0);
}

// sqrt_sum of both elements.
__device__ __forceinline__ float2 sqrt_sum2(float2 x) {
    float2 y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(fmaxf(x.x, 1e-30f)));
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(fmaxf(x.y, 1e-30f)));
    const float2 s = mul2(x, y);
    return fma2(mul2(dup2(0.5f), y), fma2(neg2(s), s, x), s);
}

// One voxel of any staged primitive, as the grouped evaluation computes it (out of line: smooth
// combines, the rarely used kinds and general frames).  NaN marks a sampled grid's voxel at its
// table's boundary.
__device__ __noinline__ float eval_one_any(const LocalPrim& P, float dx, float dy, float dz) {
    if (P.type == P_SPHERE && P.diff) {
        const float ex = fmaf(P.A[2], dz, fmaf(P.A[0], dx, P.A[1] * dy));
        const float ey = fmaf(P.A[5], dz, fmaf(P.A[3], dx, P.A[4] * dy));
        const float ez = fmaf(P.A[8], dz, fmaf(P.A[6], dx, P.A[7] * dy));
        const float x = P.L[0] + ex, y = P.L[1] + ey, z = P.L[2] + ez;
        const float num =
            fmaf(ez, fmaf(2.f, P.L[2], ez), fmaf(ey, fmaf(2.f, P.L[1], ey), fmaf(ex, fmaf(2.f, P.L[0], ex), P.L[3])));
        const float den = sqrt_sum(fmaf(z, z, fmaf(x, x, y * y))) + P.p[0];
        return fmaf(P.s, __fdiv_rn(num, den), -P.off);
    }
    if (P.type == P_TORUS && P.diff) {
        const float dzs[1] = {dz};
        return eval_group_torus_ring<1>(P, dx, dy, dzs).v[0];
    }
    float x, y, z;
    if (P.ident) {
        x = P.L[0] + dx; y = P.L[1] + dy; z = P.L[2] + dz;
    } else {
        x = fmaf(P.A[2], dz, fmaf(P.A[0], dx, fmaf(P.A[1], dy, P.L[0])));
        y = fmaf(P.A[5], dz, fmaf(P.A[3], dx, fmaf(P.A[4], dy, P.L[1])));
        z = fmaf(P.A[8], dz, fmaf(P.A[6], dx, fmaf(P.A[7], dy, P.L[2])));
    }
    float c;
    switch (P.type) {
    case P_SPHERE: c = canon_t<P_SPHERE>(P.p, x, y, z); break;
    case P_BOX: c = canon_t<P_BOX>(P.p, x, y, z); break;
    case P_CAPSULE: c = canon_t<P_CAPSULE>(P.p, x, y, z); break;
    case P_TORUS: c = canon_t<P_TORUS>(P.p, x, y, z); break;
    default:
        if (P.type == P_GRID && grid_edge_f(P.p, x, y, z)) return __int_as_float(0x7fc00000);
        c = canon_f(P.type, P.p, x, y, z);
    }
    return fmaf(P.s, c, -P.off);
}

// One voxel's combine as the grouped loop applies it (smooth and hard, sign not folded).
__device__ __forceinline__ float combine1(int op, float k, float acc, float v) {
    if (k > 0.f) return chain_apply(op, acc, v, k);
    switch (op) {
    case CH_SET: return v;
    case CH_SETNEG: return -v;
    case CH_UNION: return sel_min(acc, v);
    case CH_INTERSECT: return sel_max(acc, v);
    default: return sel_max(acc, -v);
    }
}

// Lane geometry of a tile: group g's x offset is (2g + hi) * fpitch, then dy and the z offset pairs.
struct Lane16 {
    int hi;
    float fpitch, dy;
    float2 dz[2];
    __device__ __forceinline__ float dx(int g) const { return (2 * g + hi) * fpitch; }
};

// Running values of a lane's group g (acc: the lane's slot of group 0; groups 32 float4 apart) and
// the hard combine of a group's 4 values into them.  mode 2 (set) replaces them.
struct Group4 {
    float2 a0, a1;
    __device__ __forceinline__ Group4(const float4* acc, int g, int mode) {
        const float4 v = mode == 2 ? make_float4(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000),
                                                 __int_as_float(0x7fc00000), __int_as_float(0x7fc00000))
                                   : acc[g * 32];
        a0 = make_float2(v.x, v.y);
        a1 = make_float2(v.z, v.w);
    }
    __device__ __forceinline__ void combine(bool mx, float2 v0, float2 v1) {
        a0.x = mx ? fmaxf(a0.x, v0.x) : fminf(a0.x, v0.x);
        a0.y = mx ? fmaxf(a0.y, v0.y) : fminf(a0.y, v0.y);
        a1.x = mx ? fmaxf(a1.x, v1.x) : fminf(a1.x, v1.x);
        a1.y = mx ? fmaxf(a1.y, v1.y) : fminf(a1.y, v1.y);
    }
    __device__ __forceinline__ void store(float4* acc, int g) const { acc[g * 32] = make_float4(a0.x, a0.y, a1.x, a1.y); }
};

// Sphere in the difference form (any frame: the identity frame gives the grouped loop's values).
__device__ __forceinline__ void tile16_sphere_diff(const LocalPrim& P, const Lane16& Q, int mode, float4* acc) {
    const float2 L0 = dup2(P.L[0]), L1 = dup2(P.L[1]), L2 = dup2(P.L[2]), K = dup2(P.L[3]), r = dup2(P.p[0]);
    const float2 s = dup2(P.s), noff = dup2(-P.off), two = dup2(2.f);
    const float2 c2 = dup2(P.A[2]), c5 = dup2(P.A[5]), c8 = dup2(P.A[8]);
    const float a0 = P.A[0], a3 = P.A[3], a6 = P.A[6];
    const float a1 = P.A[1] * Q.dy, a4 = P.A[4] * Q.dy, a7 = P.A[7] * Q.dy;
    const bool mx = mode == 1;
#pragma unroll 2
    for (int g = 0; g < 4; ++g) {
        const float dx = Q.dx(g);
        const float2 ebx = dup2(fmaf(a0, dx, a1)), eby = dup2(fmaf(a3, dx, a4)), ebz = dup2(fmaf(a6, dx, a7));
        float2 v[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float2 ex = fma2(c2, Q.dz[j], ebx), ey = fma2(c5, Q.dz[j], eby), ez = fma2(c8, Q.dz[j], ebz);
            const float2 x = add2(L0, ex), y = add2(L1, ey), z = add2(L2, ez);
            const float2 num = fma2(ez, fma2(two, L2, ez), fma2(ey, fma2(two, L1, ey), fma2(ex, fma2(two, L0, ex), K)));
            const float2 den = add2(sqrt_sum2(fma2(z, z, fma2(x, x, mul2(y, y)))), r);
            v[j] = fma2(s, quotient2(num, den), noff);
        }
        Group4 a(acc, g, mode);
        a.combine(mx, v[0], v[1]);
        a.store(acc, g);
    }
}

// Sphere, direct form, identity frame.
__device__ __forceinline__ void tile16_sphere(const LocalPrim& P, const Lane16& Q, int mode, float4* acc) {
    const float L0 = P.L[0], y = P.L[1] + Q.dy, yy = y * y;
    const float2 z0 = add2(dup2(P.L[2]), Q.dz[0]), z1 = add2(dup2(P.L[2]), Q.dz[1]);
    const float2 s = dup2(P.s), noff = dup2(-P.off), nr = dup2(-P.p[0]);
    const bool mx = mode == 1;
#pragma unroll 2
    for (int g = 0; g < 4; ++g) {
        const float x = L0 + Q.dx(g);
        const float2 xy = dup2(fmaf(x, x, yy));
        const float2 v0 = fma2(s, add2(sqrt_sum2(fma2(z0, z0, xy)), nr), noff);
        const float2 v1 = fma2(s, add2(sqrt_sum2(fma2(z1, z1, xy)), nr), noff);
        Group4 a(acc, g, mode);
        a.combine(mx, v0, v1);
        a.store(acc, g);
    }
}

// Box, identity frame.
__device__ __forceinline__ void tile16_box(const LocalPrim& P, const Lane16& Q, int mode, float4* acc) {
    const float L0 = P.L[0], p0 = P.p[0];
    const float y = P.L[1] + Q.dy, qy = fabsf(y) - P.p[1], oy = fmaxf(qy, 0.f), oyy = oy * oy;
    const float2 qz0 = add2(abs2(add2(dup2(P.L[2]), Q.dz[0])), dup2(-P.p[2]));
    const float2 qz1 = add2(abs2(add2(dup2(P.L[2]), Q.dz[1])), dup2(-P.p[2]));
    const float2 oz0 = max2(qz0, 0.f), oz1 = max2(qz1, 0.f);
    const float2 s = dup2(P.s), noff = dup2(-P.off);
    const bool mx = mode == 1;
#pragma unroll 2
    for (int g = 0; g < 4; ++g) {
        const float qx = fabsf(L0 + Q.dx(g)) - p0, ox = fmaxf(qx, 0.f);
        const float2 oxy = dup2(fmaf(ox, ox, oyy));
        const float mxy = fmaxf(qx, qy);
        const float2 in0 = make_float2(fminf(fmaxf(qz0.x, mxy), 0.f), fminf(fmaxf(qz0.y, mxy), 0.f));
        const float2 in1 = make_float2(fminf(fmaxf(qz1.x, mxy), 0.f), fminf(fmaxf(qz1.y, mxy), 0.f));
        const float2 v0 = fma2(s, add2(sqrt_sum2(fma2(oz0, oz0, oxy)), in0), noff);
        const float2 v1 = fma2(s, add2(sqrt_sum2(fma2(oz1, oz1, oxy)), in1), noff);
        Group4 a(acc, g, mode);
        a.combine(mx, v0, v1);
        a.store(acc, g);
    }
}

// Capsule, identity frame.
__device__ __forceinline__ void tile16_capsule(const LocalPrim& P, const Lane16& Q, int mode, float4* acc) {
    const float* p = P.p;
    const float L0 = P.L[0], p0 = p[0], p5 = p[5], p6 = p[6];
    const float y = P.L[1] + Q.dy, yp1 = y * p[1];
    const float2 z[2] = {add2(dup2(P.L[2]), Q.dz[0]), add2(dup2(P.L[2]), Q.dz[1])};
    const float2 s = dup2(P.s), noff = dup2(-P.off), nr = dup2(-p[3]), p2 = dup2(p[2]), p4 = dup2(p[4]);
    const float2 np0 = dup2(-p0), np1 = dup2(-p[1]), np2 = dup2(-p[2]), y2 = dup2(y);
    const bool mx = mode == 1;
#pragma unroll 2
    for (int g = 0; g < 4; ++g) {
        const float x = L0 + Q.dx(g);
        const float2 xy = dup2(fmaf(x, p0, yp1)), x2 = dup2(x);
        float2 v[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float2 t = mul2(fma2(z[j], p2, xy), p4);
            const float2 h = make_float2(fminf(fmaxf(t.x, p5), p6), fminf(fmaxf(t.y, p5), p6));
            const float2 ex = fma2(np0, h, x2), ey = fma2(np1, h, y2), ez = fma2(np2, h, z[j]);
            v[j] = fma2(s, add2(sqrt_sum2(fma2(ez, ez, fma2(ex, ex, mul2(ey, ey)))), nr), noff);
        }
        Group4 a(acc, g, mode);
        a.combine(mx, v[0], v[1]);
        a.store(acc, g);
    }
}

// Torus, any frame (the identity frame gives the grouped loop's values).
__device__ __forceinline__ void tile16_torus(const LocalPrim& P, const Lane16& Q, int mode, float4* acc) {
    const float t0 = fmaf(P.A[1], Q.dy, P.L[0]), t1 = fmaf(P.A[4], Q.dy, P.L[1]), t2 = fmaf(P.A[7], Q.dy, P.L[2]);
    const float a0 = P.A[0], a3 = P.A[3], a6 = P.A[6];
    const float2 c2 = dup2(P.A[2]), c5 = dup2(P.A[5]), c8 = dup2(P.A[8]);
    const float2 s = dup2(P.s), noff = dup2(-P.off), nR = dup2(-P.p[0]), nr = dup2(-P.p[1]);
    const bool mx = mode == 1;
#pragma unroll 2
    for (int g = 0; g < 4; ++g) {
        const float dx = Q.dx(g);
        const float2 bx = dup2(fmaf(a0, dx, t0)), by = dup2(fmaf(a3, dx, t1)), bz = dup2(fmaf(a6, dx, t2));
        float2 v[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float2 x = fma2(c2, Q.dz[j], bx), y = fma2(c5, Q.dz[j], by), z = fma2(c8, Q.dz[j], bz);
            const float2 qx = add2(sqrt_sum2(fma2(x, x, mul2(y, y))), nR);
            v[j] = fma2(s, add2(sqrt_sum2(fma2(z, z, mul2(qx, qx))), nr), noff);
        }
        Group4 a(acc, g, mode);
        a.combine(mx, v[0], v[1]);
        a.store(acc, g);
    }
}

// A torus in its ring frame (leaf kernels built for recipes with such tori), on pairs: the
// operations of eval_group_torus_ring in their order, the fast division per element.
__device__ __forceinline__ void tile16_torus_ring(const LocalPrim& P, const Lane16& Q, int mode, float4* acc) {
    const float2 L0 = dup2(P.L[0]), L2 = dup2(P.L[2]), R = dup2(P.p[0]), nR = dup2(-P.p[0]), nr = dup2(-P.p[1]);
    const float2 s = dup2(P.s), noff = dup2(-P.off);
    const float2 c2 = dup2(P.A[2]), c5 = dup2(P.A[5]), c8 = dup2(P.A[8]);
    const float a0 = P.A[0], a3 = P.A[3], a6 = P.A[6];
    const float a1 = P.A[1] * Q.dy, a4 = P.A[4] * Q.dy, a7 = P.A[7] * Q.dy;
    const bool mx = mode == 1;
#pragma unroll 2
    for (int g = 0; g < 4; ++g) {
        const float dx = Q.dx(g);
        const float2 ebx = dup2(fmaf(a0, dx, a1)), eby = dup2(fmaf(a3, dx, a4)), ebz = dup2(fmaf(a6, dx, a7));
        float2 v[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float2 u = add2(L0, fma2(c2, Q.dz[j], ebx)), w = fma2(c5, Q.dz[j], eby);
            const float2 z = add2(L2, fma2(c8, Q.dz[j], ebz));
            const float2 t = add2(R, u), ww = mul2(w, w);
            const float2 rho = sqrt_sum2(fma2(t, t, ww));
            const float2 den = add2(rho, t), far = add2(rho, nR);
            const float2 qx = make_float2(t.x > 0.f ? u.x + __fdividef(ww.x, den.x) : far.x,
                                          t.y > 0.f ? u.y + __fdividef(ww.y, den.y) : far.y);
            v[j] = fma2(s, add2(sqrt_sum2(fma2(z, z, mul2(qx, qx))), nr), noff);
        }
        Group4 a(acc, g, mode);
        a.combine(mx, v[0], v[1]);
        a.store(acc, g);
    }
}

// Any other staged element (mode 3): an offset, a smooth combine, a rarely used kind or a common
// kind in a general frame, voxel by voxel.  Returns the voxels that sampled a grid table at its
// boundary (bit 4g + k).
__device__ __forceinline__ uint32_t tile16_other(const LocalPrim& P, const Lane16& Q, float4* acc) {
    const int op = P.op;
    const float k = P.k;
    uint32_t edge = 0;
#pragma unroll 2
    for (int g = 0; g < 4; ++g) {
        float4 a = acc[g * 32];
        if (op == CH_OFFSET) {
            a.x -= k; a.y -= k; a.z -= k; a.w -= k;
        } else {
            const float dx = Q.dx(g);
            const float v0 = eval_one_any(P, dx, Q.dy, Q.dz[0].x), v1 = eval_one_any(P, dx, Q.dy, Q.dz[0].y);
            const float v2 = eval_one_any(P, dx, Q.dy, Q.dz[1].x), v3 = eval_one_any(P, dx, Q.dy, Q.dz[1].y);
            edge |= ((uint32_t)!(v0 == v0) | (uint32_t)!(v1 == v1) << 1 | (uint32_t)!(v2 == v2) << 2 |
                     (uint32_t)!(v3 == v3) << 3) << (4 * g);
            a.x = combine1(op, k, a.x, v0);
            a.y = combine1(op, k, a.y, v1);
            a.z = combine1(op, k, a.z, v2);
            a.w = combine1(op, k, a.w, v3);
        }
        acc[g * 32] = a;
    }
    return edge;
}

// The tile of one 8^3 block from its culled list (leaf_block's list and frame), with the running
// values in this warp's `acc` (4 groups x 32 lanes float4, shared memory); returns the lane's
// guard-band bits (bit 4g + k: voxel k of group g), as the grouped loop's deferred recheck reads
// them.  Every lane of the warp calls it with the same block.
template <bool kEdge>
__device__ __forceinline__ uint32_t tile16(const Geo& G, const FbPrim* __restrict__ prims,
                                           const PrimF* __restrict__ primf, const FbInsn* __restrict__ chain,
                                           const uint32_t* list, int len, double ox, double oy, double oz,
                                           float* __restrict__ out, LocalPrim* sp, float4* acc_warp) {
    const int lane = threadIdx.x & 31;
    Lane16 Q;
    Q.hi = lane >> 4;
    Q.fpitch = G.fpitch;
    Q.dy = ((lane >> 1) & 7) * G.fpitch;
    const int lk0 = 4 * (lane & 1);
    Q.dz[0] = make_float2(lk0 * G.fpitch, (lk0 + 1) * G.fpitch);
    Q.dz[1] = make_float2((lk0 + 2) * G.fpitch, (lk0 + 3) * G.fpitch);
    float4* acc = acc_warp + lane;
#pragma unroll
    for (int g = 0; g < 4; ++g) acc[g * 32] = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t edge = 0;  // kEdge: bit 4g + k marks a voxel that sampled a grid table at its boundary
    for (int c0 = 0; c0 < len; c0 += kCapBlock) {
        const int clen = min(kCapBlock, len - c0);
        __syncwarp();
        for (int i = lane; i < clen; i += 32) {
            const uint32_t e = list[c0 + i];
            const FbInsn I = chain[e >> 2];
            const int op = effective_op(e, I.op);
            LocalPrim& S = sp[i];
            if (op == CH_OFFSET) {
                S.op = op;
                S.k = (float)I.k;
                S.mode = 3;
                continue;
            }
            localise(prims[I.arg], primf[I.arg], ox, oy, oz, op, (float)I.k, S, 8 * G.fpitch, kEdge);
            const int t = S.type;
            const bool fast = t == P_TORUS || (t == P_SPHERE && S.diff) ||
                              (S.ident && (t == P_SPHERE || t == P_BOX || t == P_CAPSULE));
            int mode = 3;
            if (fast && !(S.k > 0.f)) {
                mode = (op == CH_SET || op == CH_SETNEG) ? 2 : (op == CH_INTERSECT || op == CH_SUBTRACT) ? 1 : 0;
                if (op == CH_SUBTRACT || op == CH_SETNEG) {
                    S.s = -S.s;
                    S.off = -S.off;
                }
            }
            S.mode = mode;
        }
        __syncwarp();
        for (int i = 0; i < clen; ++i) {
            const LocalPrim& P = sp[i];
            const int mode = P.mode;
            if (mode == 3) {
                const uint32_t e = tile16_other(P, Q, acc);
                if (kEdge) edge |= e;
                continue;
            }
            switch (P.type) {
            case P_SPHERE:
                if (P.diff) tile16_sphere_diff(P, Q, mode, acc);
                else tile16_sphere(P, Q, mode, acc);
                break;
            case P_BOX: tile16_box(P, Q, mode, acc); break;
            case P_CAPSULE: tile16_capsule(P, Q, mode, acc); break;
            default:  // P_TORUS: the staging gives modes 0-2 to the kinds above only
                if (kEdge && P.diff) tile16_torus_ring(P, Q, mode, acc);
                else tile16_torus(P, Q, mode, acc);
            }
        }
    }
    uint32_t near = 0;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        float4 a = acc[g * 32];
        if (kEdge) {  // sampled a grid table at its boundary: decided in float64
            const float nan = __int_as_float(0x7fc00000);
            if ((edge >> (4 * g)) & 1u) a.x = nan;
            if ((edge >> (4 * g + 1)) & 1u) a.y = nan;
            if ((edge >> (4 * g + 2)) & 1u) a.z = nan;
            if ((edge >> (4 * g + 3)) & 1u) a.w = nan;
        }
        near |= ((uint32_t)!(fabsf(a.x) >= G.guard) | (uint32_t)!(fabsf(a.y) >= G.guard) << 1 |
                 (uint32_t)!(fabsf(a.z) >= G.guard) << 2 | (uint32_t)!(fabsf(a.w) >= G.guard) << 3) << (4 * g);
        reinterpret_cast<float4*>(out)[g * 32 + lane] = a;
    }
    return near;
}

// quotient2 over n pairs (the self-test export fb_quotient_probe).
__global__ void k_quotient(const float* __restrict__ num, const float* __restrict__ den, float* __restrict__ out,
                           int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = quotient2(make_float2(num[i], 0.f), make_float2(den[i], 1.f)).x;
}

// Leaf tiles of a chain recipe: warp per active block.  Each lane owns groups of VG consecutive
// voxels along z (VG = 4, or 2 for 4^3 blocks) and stores each group with one vector store.
// One active block's tile: the block's culled list (as the classification left it, else culled
// here from the superblock list into `sl`), localised kCapBlock primitives at a time into `sp`, each
// lane evaluating groups of VG consecutive voxels along z (VG = 4, or 2 for 4^3 blocks) and storing
// each group with one vector store.  Every lane of the warp calls it with the same block.  kEdge:
// the recipe has sampled-grid leaves, whose voxels at a table's boundary are marked for the float64
// recheck (the marks cost registers in the hot loop, so recipes without such leaves leave them out).
// The float64 recheck of a lane's guard-band voxels (bit g * VG + k: voxel k of its group g).
template <int B, int VG>
__device__ __noinline__ void recheck_near(uint32_t near, int lane, float* out, const uint32_t* list, int len,
                                          const FbInsn* __restrict__ chain, const FbPrim* __restrict__ prims,
                                          const Geo& G, int bi, int bj, int bk) {
    while (near) {
        const int bit = __ffs(near) - 1;
        near &= near - 1;
        const int v = ((bit / VG) * 32 + lane) * VG + bit % VG;
        const int li = v / (B * B), lj = (v / B) % B, lk = v % B;
        out[v] = (float)guard_value(list, len, chain, prims, G, (int64_t)bi * B + li, (int64_t)bj * B + lj,
                                    (int64_t)bk * B + lk);
    }
}

template <int B, bool kEdge>
__device__ void leaf_block(const Geo& G, const FbPrim* __restrict__ prims, const PrimF* __restrict__ primf,
                           const FbInsn* __restrict__ chain, const uint32_t* __restrict__ pool,
                           const int64_t* __restrict__ sb_off, const int32_t* __restrict__ sb_len, int64_t blk,
                           float* __restrict__ out, unsigned long long* __restrict__ work,
                           const int32_t* __restrict__ kind, const int32_t* __restrict__ blk_off,
                           const int32_t* __restrict__ blk_len, const uint32_t* __restrict__ blk_pool, int64_t blk_cap,
                           LocalPrim* sp, uint32_t* sl, float4* acc) {
    constexpr int kVox = B * B * B;
    constexpr int VG = B == 4 ? 2 : 4;
    constexpr int kGroups = kVox / (32 * VG);
    constexpr bool kDeferGuard = kGroups * VG <= 32;  // the lane's voxels fit one bit mask (B <= 8)
    const int lane = threadIdx.x & 31;
    if (blk < 0 || blk >= G.nblocks) {  // an id outside the grid (a corrupted list) reads as exterior
        for (int v = lane; v < kVox; v += 32) out[v] = kBig;
        return;
    }
    int bi, bj, bk;
    if (G.nblocks <= 0xffffffffll) {  // 32-bit division (grids below 2^32 blocks)
        const uint32_t b32 = (uint32_t)blk, q = b32 / (uint32_t)G.nbz;
        bk = (int)(b32 - q * (uint32_t)G.nbz);
        bj = (int)(q % (uint32_t)G.nby);
        bi = (int)(q / (uint32_t)G.nby);
    } else {
        bk = (int)(blk % G.nbz);
        bj = (int)((blk / G.nbz) % G.nby);
        bi = (int)(blk / ((int64_t)G.nbz * G.nby));
    }
    const double ox = G.x0 + (double)(bi * B) * G.pitch;
    const double oy = G.y0 + (double)(bj * B) * G.pitch;
    const double oz = G.z0 + (double)(bk * B) * G.pitch;
    // the block's culled list, as the classification left it; cull again if it is not there
    const uint32_t* list;
    int len;
    bool fits = true;
    int stored = kind[blk] == 0 ? blk_len[blk] : -1;
    const int64_t soff = stored >= 0 ? (int64_t)blk_off[blk] : 0;
    if (stored < 0 || soff < 0 || soff + stored > blk_cap) stored = -1;
    if (stored >= 0) {
        list = blk_pool + soff;
        len = stored;
    } else {
        const int64_t s = ((int64_t)(bi / G.S) * G.nsy + bj / G.S) * G.nsz + bk / G.S;
        const uint32_t* plist = pool + sb_off[s];
        const int plen = sb_len[s];
        const float half = 0.5f * B;
        const float cx = G.fx0 + (bi * B + half) * G.fpitch;
        const float cy = G.fy0 + (bj * B + half) * G.fpitch;
        const float cz = G.fz0 + (bk * B + half) * G.fpitch;
        const float R = 1.7320509f * half * G.fpitch;
        __syncwarp();
        const int nk = warp_walk(plist, plen, chain, primf, cx, cy, cz, R, G.eps, sl, kCapBlock);
        __syncwarp();
        fits = nk <= kCapBlock;
        list = fits ? sl : plist;
        len = fits ? nk : plen;
    }
    if (work) {  // executed primitive evaluations and their float32 operation count
        unsigned long long evals = 0, flops = 0;
        for (int i = lane; i < len; i += 32) {
            const FbInsn I = chain[list[i] >> 2];
            const int op = effective_op(list[i], I.op);
            if (op == CH_OFFSET) { flops += 1; continue; }
            evals += 1;
            flops += prim_flops(primf[I.arg].type, primf[I.arg].ident) + (I.k > 0 ? 8 : 1);
        }
        for (int o = 16; o > 0; o >>= 1) {
            evals += __shfl_xor_sync(0xffffffffu, evals, o);
            flops += __shfl_xor_sync(0xffffffffu, flops, o);
        }
        if (lane == 0) {
            atomicAdd(&work[0], evals * kVox);
            atomicAdd(&work[1], flops * kVox);
        }
    }
    (void)fits;
    // the list in chunks of kCapBlock localised primitives; between chunks each lane keeps its
    // partial fold in its own part of the tile (the same float operations in the same order)
    uint32_t near = 0;  // bit g * VG + k: voxel k of this lane's group g lies in the guard band
    if constexpr (B == 8) {
        near = tile16<kEdge>(G, prims, primf, chain, list, len, ox, oy, oz, out, sp, acc);
    } else {
        for (int c0 = 0; c0 == 0 || c0 < len; c0 += kCapBlock) {  // one pass even for an empty list
            const int clen = max(0, min(kCapBlock, len - c0));
            const bool first = c0 == 0, last = c0 + clen >= len;
            __syncwarp();
            for (int i = lane; i < clen; i += 32) {
                const uint32_t e = list[c0 + i];
                const FbInsn I = chain[e >> 2];
                const int op = effective_op(e, I.op);
                if (op == CH_OFFSET) {
                    sp[i].op = op;
                    sp[i].k = (float)I.k;
                } else {
                    localise(prims[I.arg], primf[I.arg], ox, oy, oz, op, (float)I.k, sp[i], B * G.fpitch, kEdge);
                }
            }
            __syncwarp();
            for (int g = 0; g < kGroups; ++g) {
                const int v0 = (g * 32 + lane) * VG;
                const int li = v0 / (B * B), lj = (v0 / B) % B, lk0 = v0 % B;
                const float dx = li * G.fpitch, dy = lj * G.fpitch;
                float dz[VG], acc[VG], v[VG];
                uint32_t edge = 0;
    #pragma unroll
                for (int k = 0; k < VG; ++k) dz[k] = (lk0 + k) * G.fpitch;
                if (first) {
    #pragma unroll
                    for (int k = 0; k < VG; ++k) acc[k] = 0.f;
                } else {
                    load_group<VG>(out, g * 32 + lane, acc);
                    if (kEdge) {
    #pragma unroll
                        for (int k = 0; k < VG; ++k) edge |= (uint32_t)!(acc[k] == acc[k]) << k;  // an earlier chunk's mark
                    }
                }
                for (int i = 0; i < clen; ++i) {
                    const LocalPrim& P = sp[i];
                    const int op = P.op;
                    if (op == CH_OFFSET) {
    #pragma unroll
                        for (int k = 0; k < VG; ++k) acc[k] -= P.k;
                        continue;
                    }
                    edge |= eval_group<VG, kEdge>(P, dx, dy, dz, v);
                    combine_group<VG>(op, P.k, acc, v);
                }
                if (kEdge && edge) {  // sampled a grid table at its boundary: carried to the last chunk as NaN
    #pragma unroll
                    for (int k = 0; k < VG; ++k)
                        if ((edge >> k) & 1u) acc[k] = __int_as_float(0x7fc00000);
                }
                if (last) {
                    if (kDeferGuard) {
    #pragma unroll
                        for (int k = 0; k < VG; ++k) near |= (uint32_t)!(fabsf(acc[k]) >= G.guard) << (g * VG + k);
                    } else {
    #pragma unroll
                        for (int k = 0; k < VG; ++k)
                            if (!(fabsf(acc[k]) >= G.guard))
                                acc[k] = (float)guard_value(list, len, chain, prims, G, (int64_t)bi * B + li,
                                                            (int64_t)bj * B + lj, (int64_t)bk * B + lk0 + k);
                    }
                }
                store_group<VG>(out, g * 32 + lane, acc);
            }
        }
    }
    // guard band: a float64 recheck of the few voxels near zero, so the sign never disagrees with
    // the float64 value -- after the tile is stored, in one out-of-line call only where a lane has
    // such voxels (the call inside the kernel's own loop cost the leaf pass 8 % in registers)
    if (near) recheck_near<B, VG>(near, lane, out, list, len, chain, prims, G, bi, bj, bk);
}

// Leaf tiles of a chain recipe: a warp per active block (leaf_block).
template <int B, bool kEdge>
__global__ void __launch_bounds__(32 * kLeafWarps, 6) k_leaf(Geo G, const FbPrim* __restrict__ prims,
                                                             const PrimF* __restrict__ primf,
                                                             const FbInsn* __restrict__ chain,
                                                             const uint32_t* __restrict__ pool,
                                                             const int64_t* __restrict__ sb_off,
                                                             const int32_t* __restrict__ sb_len,
                                                             const int32_t* __restrict__ active,
                                                             const int32_t* __restrict__ count, int64_t capacity,
                                                             float* __restrict__ tiles,
                                                             unsigned long long* __restrict__ work,
                                                             const int32_t* __restrict__ kind,
                                                             const int32_t* __restrict__ blk_off,
                                                             const int32_t* __restrict__ blk_len,
                                                             const uint32_t* __restrict__ blk_pool, int64_t blk_cap) {
    __shared__ LocalPrim s_prim[kLeafWarps][kCapBlock];
    __shared__ uint32_t s_list[kLeafWarps][kCapBlock];
    __shared__ float4 s_acc[kLeafWarps][B == 8 ? 128 : 1];  // 8^3 tiles: running values, 4 groups x 32 lanes
    const int warp = threadIdx.x >> 5;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n_active = min((int64_t)count[0], capacity);
    for (int64_t a = gwarp; a < n_active; a += nwarps)
        leaf_block<B, kEdge>(G, prims, primf, chain, pool, sb_off, sb_len, active[a], tiles + a * (B * B * B), work,
                             kind, blk_off, blk_len, blk_pool, blk_cap, s_prim[warp], s_list[warp], s_acc[warp]);
}

// Leaf tiles of a general postfix program: float64 per voxel, no culling.
template <int B>
__global__ void __launch_bounds__(128) k_leaf_program(Geo G, const FbPrim* __restrict__ prims,
                                                      const FbInsn* __restrict__ prog, int n_prog,
                                                      const int32_t* __restrict__ active,
                                                      const int32_t* __restrict__ count, int64_t capacity,
                                                      float* __restrict__ tiles) {
    constexpr int kVox = B * B * B;
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n_active = min((int64_t)count[0], capacity);
    for (int64_t a = gwarp; a < n_active; a += nwarps) {
        const int64_t blk = active[a];
        float* out = tiles + a * kVox;
        if (blk < 0 || blk >= G.nblocks) {
            for (int v = lane; v < kVox; v += 32) out[v] = kBig;
            continue;
        }
        const int bk = (int)(blk % G.nbz), bj = (int)((blk / G.nbz) % G.nby), bi = (int)(blk / ((int64_t)G.nbz * G.nby));
        for (int v = lane; v < kVox; v += 32) {
            const int li = v / (B * B), lj = (v / B) % B, lk = v % B;
            const double x = rn_add(G.x0, rn_mul((double)(bi * B + li), G.pitch));
            const double y = rn_add(G.y0, rn_mul((double)(bj * B + lj), G.pitch));
            const double z = rn_add(G.z0, rn_mul((double)(bk * B + lk), G.pitch));
            out[v] = (float)program_eval_d(prims, prog, n_prog, x, y, z);
        }
    }
}

// ------------------------------------------------------------------------------------ dense input
__global__ void k_classify_dense(const float* __restrict__ dense, int64_t nx, int64_t ny, int64_t nz, int B,
                                 int nby, int nbz, int64_t nblocks, float margin, int32_t* __restrict__ kind,
                                 float* __restrict__ cma) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nblocks) return;
    const int64_t bk = t % nbz, bj = (t / nbz) % nby, bi = t / ((int64_t)nbz * nby);
    float mn;
    const int k = dense_block_kind(dense, nx, ny, nz, B, bi * B, bj * B, bk * B, margin, &mn);
    if (cma) cma[t] = mn;
    kind[t] = k;
}

// Warp per active block; each lane copies voxels with the index clamped to n-1.
__global__ void k_tiles_dense(const float* __restrict__ dense, int64_t nx, int64_t ny, int64_t nz, int B, int nby,
                              int nbz, const int32_t* __restrict__ active, const int32_t* __restrict__ count,
                              int64_t capacity, float* __restrict__ tiles) {
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n_active = min((int64_t)count[0], capacity);
    const int b3 = B * B * B;
    for (int64_t a = gwarp; a < n_active; a += nwarps) {
        const int64_t lin = active[a];
        const int64_t bk = lin % nbz, bi = lin / ((int64_t)nbz * nby), bj = (lin / nbz) % nby;
        for (int v = lane; v < b3; v += 32) {
            const int li = v / (B * B), lj = (v / B) % B, lk = v % B;
            const int64_t vx = min(bi * B + li, nx - 1), vy = min(bj * B + lj, ny - 1), vz = min(bk * B + lk, nz - 1);
            tiles[a * b3 + v] = dense[(vx * ny + vy) * nz + vz];
        }
    }
}

// ------------------------------------------------------------------------------------ reconstruction
__global__ void k_slot_map(const int32_t* __restrict__ active, int64_t n_active, int32_t* __restrict__ slot) {
    const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a < n_active) slot[active[a]] = (int32_t)a;
}

// Dense (nx, ny, nz) field: tile values for active blocks, -BIG / +BIG elsewhere
// (src/field_engine/faltkarna_v1.py:302-350, cropped to the grid).
__global__ void k_reconstruct(const int32_t* __restrict__ kind, const int32_t* __restrict__ slot,
                              const float* __restrict__ tiles, int64_t nx, int64_t ny, int64_t nz, int B, int nby,
                              int nbz, float big, float* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nx * ny * nz) return;
    const int64_t z = i % nz, y = (i / nz) % ny, x = i / (nz * ny);
    const int64_t blk = ((x / B) * nby + y / B) * nbz + z / B;
    const int32_t s = slot[blk];
    float v;
    if (s >= 0) v = tiles[(int64_t)s * B * B * B + ((x % B) * B + (y % B)) * B + (z % B)];
    else v = kind[blk] < 0 ? -big : big;
    out[i] = v;
}

// Slot map of the first count[0] active blocks (device-side count: no host round trip).
__global__ void k_slot_map_dev(const int32_t* __restrict__ active, const int32_t* __restrict__ count,
                               int64_t capacity, int32_t* __restrict__ slot) {
    const int64_t n = min((int64_t)count[0], capacity);
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < n; a += (int64_t)gridDim.x * blockDim.x)
        slot[active[a]] = (int32_t)a;
}

// Occupancy (1 where the field is negative) of every voxel: tile values in active blocks, the
// block kind elsewhere.  One thread per 16 consecutive z voxels of an (x, y) row: the row's block
// runs are read as float4 from the tiles (a tile row of B floats is contiguous along z) and the 16
// bytes leave in one 128-bit store when rows are 16-byte aligned (nz % 16 == 0).
// Item t of the occupancy pass (one row of 16 z voxels).
template <int B>
__device__ __forceinline__ void occupancy_item(const int32_t* __restrict__ kind, const int32_t* __restrict__ slot,
                                               const float* __restrict__ tiles, int nx, int ny, int nz, int nby,
                                               int nbz, uint8_t* __restrict__ mask, int64_t t) {
    constexpr int kB3 = B * B * B;
    const int chunks = (nz + 15) >> 4;
    const bool vec = (nz & 15) == 0;
    const int64_t row = t / chunks;
    const int c = (int)(t - row * chunks);
    const int x = (int)(row / ny), y = (int)(row - (int64_t)x * ny);
    const int z0 = c << 4;
    const int64_t blk_row = ((int64_t)(x / B) * nby + y / B) * nbz;
    const int lxy = ((x % B) * B + (y % B)) * B;
    uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int seg = 0; seg < 16; seg += (B < 16 ? B : 16)) {
        const int z = z0 + seg;
        if (z >= nz) continue;  // (not break: the loop stays fully unrolled, w[] in registers)
        const int64_t blk = blk_row + z / B;
        const int32_t s = slot[blk];
        constexpr int kRun = B < 16 ? B : 16;
        if (s >= 0) {
            const float4* src = reinterpret_cast<const float4*>(tiles + (int64_t)s * kB3 + lxy + (z % B));
#pragma unroll
            for (int q = 0; q < kRun / 4; ++q) {
                const float4 v = src[q];
                const int k = seg + 4 * q;  // byte index within the 16
                const uint32_t bits = (uint32_t)(v.x < 0.f) | ((uint32_t)(v.y < 0.f) << 8) |
                                      ((uint32_t)(v.z < 0.f) << 16) | ((uint32_t)(v.w < 0.f) << 24);
                w[k >> 2] = bits;
            }
        } else {
            const uint32_t fill = kind[blk] < 0 ? 0x01010101u : 0u;
#pragma unroll
            for (int q = 0; q < kRun / 4; ++q) w[(seg >> 2) + q] = fill;
        }
    }
    uint8_t* dst = mask + row * nz + z0;
    if (vec) {
        *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
        const int n = min(16, nz - z0);
        for (int k = 0; k < n; ++k) {
            const uint32_t wk = k < 8 ? (k < 4 ? w[0] : w[1]) : (k < 12 ? w[2] : w[3]);
            dst[k] = (uint8_t)(wk >> (8 * (k & 3)));
        }
    }
}

template <int B>
__global__ void __launch_bounds__(256) k_occupancy(const int32_t* __restrict__ kind, const int32_t* __restrict__ slot,
                                                   const float* __restrict__ tiles, int nx, int ny, int nz, int nby,
                                                   int nbz, uint8_t* __restrict__ mask) {
    const int64_t total = (int64_t)nx * ny * ((nz + 15) >> 4);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x)
        occupancy_item<B>(kind, slot, tiles, nx, ny, nz, nby, nbz, mask, t);
}

// Sum of trunc(v * scale) over negative values, in int64 (determinism-safe checksum,
// src/field_engine/faltkarna_v1.py:250-255).
__global__ void k_checksum_i64(const float* __restrict__ v, int64_t n, double scale, unsigned long long* out) {
    long long acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = v[i];
        if (x < 0.0f) acc += (long long)((double)x * scale);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, (unsigned long long)acc);
}

// Exact sum of int32 values into one int64 word: per-thread partial sums, a warp reduction, one
// 64-bit atomic per warp (wraps modulo 2^64 like the signed sum).
__global__ void __launch_bounds__(256) k_sum_i32(const int32_t* __restrict__ v, int64_t n, unsigned long long* out) {
    long long acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += v[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, (unsigned long long)acc);
}

// ------------------------------------------------------------------------------------ host side
struct Scratch {
    int32_t* blk_off;
    int32_t* blk_len;
    uint32_t* blk_pool;
    PrimF* primf;
    uint32_t* pool;
    int64_t* off;
    int32_t* len;
    unsigned long long* status;
    int* misc;
};

Scratch carve(void* base, const Plan& p, const Geo& G) {
    char* b = static_cast<char*>(base);
    Scratch s;
    s.primf = reinterpret_cast<PrimF*>(b + p.primf);
    s.pool = reinterpret_cast<uint32_t*>(b + p.pool);
    s.off = reinterpret_cast<int64_t*>(b + p.off);
    s.len = reinterpret_cast<int32_t*>(b + p.len);
    s.status = reinterpret_cast<unsigned long long*>(b + p.status);
    s.misc = reinterpret_cast<int*>(b + p.misc);
    s.blk_off = reinterpret_cast<int32_t*>(b + p.blk_off);
    s.blk_len = reinterpret_cast<int32_t*>(b + p.blk_len);
    s.blk_pool = reinterpret_cast<uint32_t*>(b + p.blk_pool);
    (void)G;
    return s;
}

int launch_compact(const int32_t* kind, int64_t nblocks, int32_t* active, int32_t* count, unsigned long long* status,
                   int* misc, cudaStream_t st) {
    const int64_t ntiles = (nblocks + kTile - 1) / kTile;
    FB_CUDA(cudaMemsetAsync(status, 0, ntiles * 8, st));
    FB_CUDA(cudaMemsetAsync(misc, 0, 256, st));
    k_compact<<<(unsigned)ntiles, 256, 0, st>>>(kind, nblocks, active, count, status, misc, ntiles, kLookbackSpins);
    FB_LAUNCH();
    return FB_OK;
}

int classify_impl(const FbGeom& g, const FbPrim* prims, int n_prims, const FbInsn* chain, int n_chain, int mode,
                  int32_t* kind, float* cma, int32_t* active, int32_t* count, void* scratch, int64_t scratch_len,
                  cudaStream_t st) {
    if (!geom_ok(g) || !prims || !chain || n_prims < 1 || n_chain < 1 || !kind || !cma || !active || !count ||
        !scratch)
        return FB_INVALID;
    const Geo G = make_geo(g);
    const Plan P = make_plan(G, n_prims, n_chain);
    if (scratch_len < P.total) return FB_INVALID;
    Scratch S = carve(scratch, P, G);
    k_prepare_prims<<<fb_div_up(n_prims, 128), 128, 0, st>>>(prims, n_prims, S.primf);
    FB_LAUNCH();
    if (mode == 1) {
        k_full_list<<<fb_div_up(n_chain, 256), 256, 0, st>>>(S.pool + P.pool_full, n_chain);
        FB_LAUNCH();
        // coarse regions from the full chain
        k_cull<true><<<fb_div_up(G.ncoarse * 32, 128), 128, 0, st>>>(G, chain, S.primf, S.pool, nullptr, nullptr, n_chain, 1,
                                                               1, 1, S.off, S.len, P.pool_coarse, P.cap_coarse,
                                                               G.S * G.B * kCoarseDiv, G.ncx, G.ncy, G.ncz);
        FB_LAUNCH();
        // superblocks from their coarse region
        k_cull<false><<<fb_div_up(G.nsuper * 32, 128), 128, 0, st>>>(G, chain, S.primf, S.pool, S.off, S.len, 0, kCoarseDiv,
                                                              G.ncy, G.ncz, S.off + G.ncoarse, S.len + G.ncoarse,
                                                              P.pool_super, P.cap_super, G.S * G.B, G.nsx, G.nsy, G.nsz);
        FB_LAUNCH();
        FB_CUDA(cudaMemsetAsync(S.misc, 0, 256, st));
        // a thread per block: its own cull of the superblock list, kept for the active blocks
        k_classify_blocks<<<fb_div_up(G.nsuper * threads_per_super(G.S), 128), 128, 0, st>>>(
            G, prims, S.primf, chain, S.pool, S.off + G.ncoarse, S.len + G.ncoarse, kind, cma, S.blk_off, S.blk_len,
            S.blk_pool, P.blk_cap, S.misc + 2);
    } else {
        k_classify_program<<<fb_div_up(G.nblocks, 128), 128, 0, st>>>(G, prims, chain, n_chain, kind, cma);
    }
    FB_LAUNCH();
    if (int rc = launch_compact(kind, G.nblocks, active, count, S.status, S.misc, st)) return rc;
    return FB_OK;
}

int leaf_impl(const FbGeom& g, const FbPrim* prims, int n_prims, const FbInsn* chain, int n_chain, int mode,
              const int32_t* kind, const int32_t* active, const int32_t* count, float* tiles, int64_t capacity,
              void* scratch, int64_t scratch_len, cudaStream_t st, unsigned long long* work = nullptr) {
    if (!geom_ok(g) || !prims || !chain || n_prims < 1 || n_chain < 1 || !kind || !active || !count || !tiles ||
        !scratch || capacity < 0)
        return FB_INVALID;
    const Geo G = make_geo(g);
    const Plan P = make_plan(G, n_prims, n_chain);
    if (scratch_len < P.total) return FB_INVALID;
    Scratch S = carve(scratch, P, G);
    const int grid = fb_sm_count() * 16;
    const int64_t* sb_off = S.off + G.ncoarse;
    const int32_t* sb_len = S.len + G.ncoarse;
    if (mode != 1) {
        switch (G.B) {
        case 4: k_leaf_program<4><<<grid, 128, 0, st>>>(G, prims, chain, n_chain, active, count, capacity, tiles); break;
        case 8: k_leaf_program<8><<<grid, 128, 0, st>>>(G, prims, chain, n_chain, active, count, capacity, tiles); break;
        default: k_leaf_program<16><<<grid, 128, 0, st>>>(G, prims, chain, n_chain, active, count, capacity, tiles);
        }
    } else {
#define FB_LEAF(BB, EDGE)                                                                                   \
    k_leaf<BB, EDGE><<<grid, 32 * kLeafWarps, 0, st>>>(G, prims, S.primf, chain, S.pool, sb_off, sb_len, active, \
                                                       count, capacity, tiles, work, kind, S.blk_off, S.blk_len,  \
                                                       S.blk_pool, P.blk_cap)
        const bool edge = G.special != 0;
        switch (G.B) {
        case 4: if (edge) FB_LEAF(4, true); else FB_LEAF(4, false); break;
        case 8: if (edge) FB_LEAF(8, true); else FB_LEAF(8, false); break;
        default: if (edge) FB_LEAF(16, true); else FB_LEAF(16, false);
        }
#undef FB_LEAF
    }
    FB_LAUNCH();
    return FB_OK;
}

// ------------------------------------------------------------------------------------ batched builds
// Many chain recipes built together: every phase is one launch over a work-list spanning all the
// recipes (their coarse regions, superblocks, blocks, compaction tiles, active blocks), so small
// recipes fill the GPU beside large ones and a batch costs about fifteen launches instead of ~9
// per recipe.  Work-list g of a phase maps to (recipe, item) through the phase's group: the recipes
// taking part (rec[j]) and the exclusive prefix of their item counts (pre[j]); a warp or thread
// finds j by binary search.  Static groups (everything fixed by the geometry) are built on the
// host once per batch; the active-block groups are built on the device after the compaction
// (k_batch_offsets), which also places every recipe's tiles in the caller's arena in recipe order.
// Each recipe keeps its own culling scratch and outputs (the FieldBuilder layout); the batch adds
// one device table of descriptors, the groups, and the compaction state of all recipes.
struct RecDesc {
    Geo G;
    const FbPrim* prims;
    PrimF* primf;
    const FbInsn* chain;
    int32_t n_prims, n_chain;
    uint32_t* pool;
    int64_t* off;  // coarse regions then superblocks
    int32_t* len;
    int64_t pool_coarse, pool_super;
    int32_t cap_coarse, cap_super;
    int32_t* kind;
    float* cma;
    int32_t* active;
    int32_t* count;
    int32_t* blk_off;
    int32_t* blk_len;
    uint32_t* blk_pool;
    int64_t blk_cap;
    unsigned long long* status;  // this recipe's compaction status words (batch state)
    int64_t ntiles;
    int32_t* slot;  // occupancy: block -> tile slot (n_blocks), nullable
    uint8_t* mask;  // occupancy mask (nx, ny, nz), nullable
};

struct Group {  // device arrays of one phase's work-list
    const int32_t* rec;
    const int64_t* pre;  // m + 1 entries
    int32_t m;
};

// j with pre[j] <= g < pre[j + 1] (g < pre[m]).
__device__ __forceinline__ int group_find(const Group& W, int64_t g) {
    int lo = 0, hi = W.m - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (W.pre[mid] <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_b_prepare(const RecDesc* __restrict__ D, Group W, int64_t total) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int j = group_find(W, g);
    const RecDesc& R = D[W.rec[j]];
    prepare_prim(R.prims, (int)(g - W.pre[j]), R.primf);
}

__global__ void k_b_full_list(const RecDesc* __restrict__ D, Group W, int64_t total) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int j = group_find(W, g);
    const int64_t i = g - W.pre[j];
    D[W.rec[j]].pool[i] = (uint32_t)i << 2;
}

// kLevel 0: coarse regions from the full chain (bounding-ball bounds); 1: superblocks from their
// coarse region.
template <int kLevel>
__global__ void __launch_bounds__(128) k_b_cull(const RecDesc* __restrict__ D, Group W, int64_t total) {
    const int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (g >= total) return;
    const int j = group_find(W, g);
    const RecDesc& R = D[W.rec[j]];
    const Geo& G = R.G;
    const int64_t r = g - W.pre[j];
    if (kLevel == 0)
        cull_region<true>(G, R.chain, R.primf, R.pool, nullptr, nullptr, R.n_chain, 1, 1, 1, R.off, R.len,
                          R.pool_coarse, R.cap_coarse, G.S * G.B * kCoarseDiv, G.ncy, G.ncz, r);
    else
        cull_region<false>(G, R.chain, R.primf, R.pool, R.off, R.len, 0, kCoarseDiv, G.ncy, G.ncz, R.off + G.ncoarse,
                           R.len + G.ncoarse, R.pool_super, R.cap_super, G.S * G.B, G.nsy, G.nsz, r);
}


// Each recipe's thread range is a multiple of 32 (nsuper x threads_per_super), so a warp never
// spans two recipes.
__global__ void __launch_bounds__(128, 6) k_b_classify_blocks(const RecDesc* __restrict__ D, Group W, int64_t total,
                                                               int* __restrict__ cursors) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int j = group_find(W, g);
    const RecDesc& R = D[W.rec[j]];
    classify_block(R.G, R.prims, R.primf, R.chain, R.pool, R.off + R.G.ncoarse, R.len + R.G.ncoarse, R.kind,
                          R.cma, R.blk_off, R.blk_len, R.blk_pool, R.blk_cap, &cursors[W.rec[j]], g - W.pre[j]);
}


// Compaction of every recipe: tiles are taken from one ticket counter in the group's order, so a
// recipe's predecessor tiles always hold smaller tickets (already running when a tile waits).
__global__ void __launch_bounds__(256) k_b_compact(const RecDesc* __restrict__ D, Group W, int* __restrict__ misc,
                                                   long long spin_limit) {
    __shared__ int s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(&misc[0], 1);
    __syncthreads();
    const int j = group_find(W, s_tile);
    const RecDesc& R = D[W.rec[j]];
    compact_tile(R.kind, R.G.nblocks, R.active, R.count, R.status, s_tile - W.pre[j], R.ntiles, &misc[1], spin_limit);
}

// After the compaction: each recipe's tile offset in the arena (recipe order, floats), the tiles it
// gets (count, clipped to the room left; the overflow flag misc[2] raised when clipped), and the
// prefixes of the active-block groups leaf[0..5] (B = 4, 8, 16; then the same for recipes with
// sampled-grid leaves) and occ (recipes with a mask).  One thread: a batch holds a few hundred to a
// few thousand recipes.
constexpr int kLeafGroups = 6;
struct LeafGroups {
    Group g[kLeafGroups];
    int64_t* pre[kLeafGroups];
};

__global__ void k_batch_offsets(const RecDesc* __restrict__ D, int n, int64_t capacity,
                                int64_t* __restrict__ tile_off, int32_t* __restrict__ leaf_count, LeafGroups L,
                                Group occ, int64_t* __restrict__ occ_pre, int* __restrict__ misc) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int64_t at = 0;
    for (int r = 0; r < n; ++r) {
        const int64_t b3 = (int64_t)D[r].G.B * D[r].G.B * D[r].G.B;
        const int64_t c = min((int64_t)D[r].count[0], D[r].G.nblocks);
        const int64_t room = max((int64_t)0, (capacity - at) / b3);
        const int64_t take = min(c, room);
        if (take < c) misc[2] = 1;
        tile_off[r] = at;
        leaf_count[r] = (int32_t)take;
        at += take * b3;
    }
    int64_t t = 0;
    for (int q = 0; q < kLeafGroups; ++q) {
        t = 0;
        for (int j = 0; j < L.g[q].m; ++j) {
            L.pre[q][j] = t;
            t += leaf_count[L.g[q].rec[j]];
        }
        L.pre[q][L.g[q].m] = t;
    }
    t = 0;
    for (int j = 0; j < occ.m; ++j) {
        occ_pre[j] = t;
        t += leaf_count[occ.rec[j]];
    }
    occ_pre[occ.m] = t;
}

// Occupancy of every recipe that carries a mask: slot map (-1, then the slot of each tiled block),
// then one thread per 16 z voxels (occupancy_item).
__global__ void k_b_fill_slot(const RecDesc* __restrict__ D, Group W, int64_t total) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int j = group_find(W, g);
    D[W.rec[j]].slot[g - W.pre[j]] = -1;
}

__global__ void k_b_slot_map(const RecDesc* __restrict__ D, Group W) {
    const int64_t total = W.pre[W.m];
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        const int j = group_find(W, g);
        const RecDesc& R = D[W.rec[j]];
        const int64_t a = g - W.pre[j];
        R.slot[R.active[a]] = (int32_t)a;
    }
}

template <int B>
__global__ void __launch_bounds__(256) k_b_occupancy(const RecDesc* __restrict__ D, Group W, int64_t total,
                                                     const float* __restrict__ tiles,
                                                     const int64_t* __restrict__ tile_off) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int j = group_find(W, g);
    const int r = W.rec[j];
    const RecDesc& R = D[r];
    const Geo& G = R.G;
    occupancy_item<B>(R.kind, R.slot, tiles + tile_off[r], G.nx, G.ny, G.nz, G.nby, G.nbz, R.mask, g - W.pre[j]);
}

// 5 CTAs per SM (96 registers; the 8^3 form's spill stores 108 -> 16 bytes): the batch's leaf phase
// 16.55 -> 15.59 ms, where the single-recipe k_leaf keeps 6 (at 5 its 1024^3 pass went 1.50 -> 1.57 ms).
template <int B, bool kEdge>
__global__ void __launch_bounds__(32 * kLeafWarps, 5) k_b_leaf(const RecDesc* __restrict__ D, Group W,
                                                               float* __restrict__ tiles,
                                                               const int64_t* __restrict__ tile_off,
                                                               unsigned long long* __restrict__ work) {
    __shared__ LocalPrim s_prim[kLeafWarps][kCapBlock];
    __shared__ uint32_t s_list[kLeafWarps][kCapBlock];
    __shared__ float4 s_acc[kLeafWarps][B == 8 ? 128 : 1];  // 8^3 tiles: running values, 4 groups x 32 lanes
    const int warp = threadIdx.x >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t total = W.pre[W.m];
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < total; g += nwarps) {
        const int j = group_find(W, g);
        const int r = W.rec[j];
        const RecDesc& R = D[r];
        const int64_t a = g - W.pre[j];
        leaf_block<B, kEdge>(R.G, R.prims, R.primf, R.chain, R.pool, R.off + R.G.ncoarse, R.len + R.G.ncoarse, R.active[a],
                      tiles + tile_off[r] + a * (B * B * B), work, R.kind, R.blk_off, R.blk_len, R.blk_pool,
                      R.blk_cap, s_prim[warp], s_list[warp], s_acc[warp]);
    }
}

// Host plan of a batch: the descriptors, the groups and the batch state in one device allocation
// made at creation; building enqueues the phases on a stream and allocates nothing.
struct BatchHost {
    int n = 0;
    std::vector<RecDesc> desc;
    char* dev = nullptr;  // device allocation
    int64_t dev_bytes = 0;
    RecDesc* d_desc = nullptr;
    // static groups and their totals
    Group prims{}, chain{}, coarse{}, super_{}, cclass{}, tiles{};
    int64_t n_prims = 0, n_chain = 0, n_coarse = 0, n_super = 0, n_cclass = 0, n_tiles = 0;
    // dynamic groups (prefixes written by k_batch_offsets)
    Group leaf[kLeafGroups]{}, occ{};
    int64_t* leaf_pre[kLeafGroups] = {};
    int64_t* occ_pre = nullptr;
    // occupancy groups (recipes carrying a mask): their blocks, and their rows of 16 z voxels per B
    Group occ_blocks{}, occ_rows[3]{};
    int64_t n_occ_blocks = 0, n_occ_rows[3] = {0, 0, 0};
    unsigned long long* status = nullptr;
    int* misc = nullptr;     // [0] ticket, [1] wait error, [2] tile overflow
    int* cursors = nullptr;  // per recipe
    int64_t* tile_off = nullptr;
    int32_t* leaf_count = nullptr;
    int64_t state_bytes = 0;  // status + misc + cursors, cleared per build
};

int b_index(int B) { return B == 4 ? 0 : (B == 8 ? 1 : 2); }

}  // namespace

extern "C" {

// A batch of chain recipes built together (see the batched-builds section above).  Validates every
// item as fb_field_build_device would (chain form only), builds the descriptors and work-lists, and
// makes the batch's one device allocation; synchronises `stream`.  NULL on invalid input or
// failure.  The items' device buffers must outlive the batch.
void* fb_batch_create(const FbBatchItem* items, int32_t n, void* stream) noexcept {
    if (!items || n < 1) return nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BatchHost* H = new (std::nothrow) BatchHost;
    if (!H) return nullptr;
    try {
        H->n = n;
        H->desc.resize(n);
        std::vector<int64_t> tile_pre(n + 1, 0);
        for (int r = 0; r < n; ++r) {
            const FbBatchItem& it = items[r];
            if (!it.geom || !geom_ok(*it.geom) || !it.d_prims || !it.d_chain || it.n_prims < 1 || it.n_chain < 1 ||
                !it.d_kind || !it.d_cma || !it.d_active || !it.d_count || !it.d_scratch) {
                delete H;
                return nullptr;
            }
            const Geo G = make_geo(*it.geom);
            const Plan P = make_plan(G, it.n_prims, it.n_chain);
            if (it.scratch_len < P.total) {
                delete H;
                return nullptr;
            }
            const Scratch S = carve(it.d_scratch, P, G);
            RecDesc& d = H->desc[r];
            std::memset(&d, 0, sizeof(d));
            d.G = G;
            d.prims = it.d_prims;
            d.primf = S.primf;
            d.chain = it.d_chain;
            d.n_prims = it.n_prims;
            d.n_chain = it.n_chain;
            d.pool = S.pool;
            d.off = S.off;
            d.len = S.len;
            d.pool_coarse = P.pool_coarse;
            d.pool_super = P.pool_super;
            d.cap_coarse = P.cap_coarse;
            d.cap_super = P.cap_super;
            d.kind = it.d_kind;
            d.cma = it.d_cma;
            d.active = it.d_active;
            d.count = it.d_count;
            d.blk_off = S.blk_off;
            d.blk_len = S.blk_len;
            d.blk_pool = S.blk_pool;
            d.blk_cap = P.blk_cap;
            d.ntiles = (G.nblocks + kTile - 1) / kTile;
            d.slot = it.d_slot;
            d.mask = it.d_mask;
            if ((d.slot == nullptr) != (d.mask == nullptr) || (d.mask && (reinterpret_cast<uintptr_t>(d.mask) & 15))) {
                delete H;
                return nullptr;
            }
            tile_pre[r + 1] = tile_pre[r] + d.ntiles;
        }
        // host images of the groups: recipe ids and item prefixes
        struct HostGroup {
            std::vector<int32_t> rec;
            std::vector<int64_t> pre{0};
            void add(int r, int64_t items) {
                rec.push_back(r);
                pre.push_back(pre.back() + items);
            }
        };
        HostGroup g_prims, g_chain, g_coarse, g_super, g_cclass, g_tiles, g_leaf[kLeafGroups], g_occ, g_occ_blocks,
            g_occ_rows[3];
        for (int r = 0; r < n; ++r) {
            const RecDesc& d = H->desc[r];
            const Geo& G = d.G;
            g_prims.add(r, d.n_prims);
            g_chain.add(r, d.n_chain);
            g_coarse.add(r, G.ncoarse);
            g_super.add(r, G.nsuper);
            // classification threads rounded up to whole warps: a warp never spans two recipes
            const int64_t cls_threads = (G.nsuper * threads_per_super(G.S) + 31) / 32 * 32;
            g_cclass.add(r, cls_threads);
            g_tiles.add(r, d.ntiles);
            g_leaf[b_index(G.B) + (G.special ? 3 : 0)].add(r, 0);
            if (d.mask) {
                g_occ.add(r, 0);
                g_occ_blocks.add(r, G.nblocks);
                g_occ_rows[b_index(G.B)].add(r, (int64_t)G.nx * G.ny * ((G.nz + 15) / 16));
            }
        }
        // one device allocation: descriptors, groups, dynamic prefixes, cleared state, outputs
        int64_t at = 0;
        auto place = [&](int64_t bytes) {
            const int64_t o = at;
            at += align256(std::max<int64_t>(bytes, 1));
            return o;
        };
        const int64_t o_desc = place((int64_t)n * sizeof(RecDesc));
        struct Placed {
            int64_t rec, pre;
        };
        auto place_group = [&](const HostGroup& hg) {
            Placed q;
            q.rec = place((int64_t)hg.rec.size() * 4);
            q.pre = place((int64_t)hg.pre.size() * 8);
            return q;
        };
        // group slots: 0-3 prims, chain, coarse, super; 4 classification; 5 tiles; 6-11 leaves (B = 4,
        // 8, 16, then with sampled-grid leaves); 12 occupancy recipes; 13 their blocks; 14-16 their rows
        HostGroup* statics[] = {&g_prims, &g_chain, &g_coarse, &g_super, &g_cclass, &g_tiles, &g_leaf[0], &g_leaf[1],
                                &g_leaf[2], &g_leaf[3], &g_leaf[4], &g_leaf[5], &g_occ, &g_occ_blocks,
                                &g_occ_rows[0], &g_occ_rows[1], &g_occ_rows[2]};
        constexpr int kGroups = 17;
        Placed placed[kGroups];
        for (int q = 0; q < kGroups; ++q) placed[q] = place_group(*statics[q]);
        const int64_t o_state = at;
        const int64_t o_status = place(tile_pre[n] * 8);
        const int64_t o_misc = place(256);
        const int64_t o_cursors = place((int64_t)n * 4);
        H->state_bytes = at - o_state;
        const int64_t o_tile_off = place((int64_t)n * 8);
        const int64_t o_leaf_count = place((int64_t)n * 4);
        H->dev_bytes = at;
        if (cudaMalloc(&H->dev, H->dev_bytes) != cudaSuccess) {
            H->dev = nullptr;
            delete H;
            return nullptr;
        }
        char* D = H->dev;
        H->d_desc = reinterpret_cast<RecDesc*>(D + o_desc);
        H->status = reinterpret_cast<unsigned long long*>(D + o_status);
        H->misc = reinterpret_cast<int*>(D + o_misc);
        H->cursors = reinterpret_cast<int*>(D + o_cursors);
        H->tile_off = reinterpret_cast<int64_t*>(D + o_tile_off);
        H->leaf_count = reinterpret_cast<int32_t*>(D + o_leaf_count);
        for (int r = 0; r < n; ++r) H->desc[r].status = H->status + tile_pre[r];
        // host image of the static part, copied in one transfer
        std::vector<char> image(o_state, 0);
        std::memcpy(image.data() + o_desc, H->desc.data(), (size_t)n * sizeof(RecDesc));
        Group* dst[] = {&H->prims, &H->chain, &H->coarse, &H->super_, &H->cclass, &H->tiles, &H->leaf[0], &H->leaf[1],
                        &H->leaf[2], &H->leaf[3], &H->leaf[4], &H->leaf[5], &H->occ, &H->occ_blocks,
                        &H->occ_rows[0], &H->occ_rows[1], &H->occ_rows[2]};
        for (int q = 0; q < kGroups; ++q) {
            const HostGroup& hg = *statics[q];
            std::memcpy(image.data() + placed[q].rec, hg.rec.data(), hg.rec.size() * 4);
            std::memcpy(image.data() + placed[q].pre, hg.pre.data(), hg.pre.size() * 8);
            dst[q]->rec = reinterpret_cast<const int32_t*>(D + placed[q].rec);
            dst[q]->pre = reinterpret_cast<const int64_t*>(D + placed[q].pre);
            dst[q]->m = (int32_t)hg.rec.size();
        }
        for (int q = 0; q < kLeafGroups; ++q) H->leaf_pre[q] = reinterpret_cast<int64_t*>(D + placed[6 + q].pre);
        H->occ_pre = reinterpret_cast<int64_t*>(D + placed[12].pre);
        H->n_occ_blocks = g_occ_blocks.pre.back();
        for (int q = 0; q < 3; ++q) H->n_occ_rows[q] = g_occ_rows[q].pre.back();
        H->n_prims = g_prims.pre.back();
        H->n_chain = g_chain.pre.back();
        H->n_coarse = g_coarse.pre.back();
        H->n_super = g_super.pre.back();
        H->n_cclass = g_cclass.pre.back();
        H->n_tiles = g_tiles.pre.back();
        if (cudaMemcpyAsync(D, image.data(), o_state, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaFree(H->dev);
            delete H;
            return nullptr;
        }
        return H;
    } catch (...) {
        if (H->dev) cudaFree(H->dev);
        delete H;
        return nullptr;
    }
}

// Build every recipe of the batch, stream-ordered, with no host synchronisation and no allocation:
// culling, classification, compaction, per-block lists, then the leaf tiles of every recipe into
// d_tiles (capacity floats), recipe r's tiles at tile offset fb_batch_outputs' tile_off[r] (floats),
// its first leaf_count[r] active blocks (all of them unless the arena ran out; fb_batch_status then
// reports 8).  Each recipe's kind / cma / active / count land in its own buffers.  ctas_per_sm
// (1..64; 0 for the default 16) sizes the grids of the active-block passes, whose work is known
// only on the device.
int fb_batch_build_timed_device(void* batch, float* d_tiles, int64_t capacity, int32_t ctas_per_sm,
                                void* const* events, uint64_t* d_work, void* stream) noexcept;

int fb_batch_build_device(void* batch, float* d_tiles, int64_t capacity, int32_t ctas_per_sm, void* stream) noexcept {
    return fb_batch_build_timed_device(batch, d_tiles, capacity, ctas_per_sm, nullptr, nullptr, stream);
}

// The same build with instrumentation: events (nullable; six cudaEvent_t) are recorded on the stream
// at the start and after the culling levels, the classification (with the active blocks' own
// lists), the compaction (with the tile placement), an empty phase kept for the six-event layout,
// and the leaf tiles; d_work (nullable; two uint64) accumulates the
// leaf pass's executed primitive evaluations and float32 operations.
int fb_batch_build_timed_device(void* batch, float* d_tiles, int64_t capacity, int32_t ctas_per_sm,
                                void* const* events, uint64_t* d_work, void* stream) noexcept {
    BatchHost* H = static_cast<BatchHost*>(batch);
    if (!H || !d_tiles || capacity < 0 || ctas_per_sm > 64) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto mark = [&](int k) -> int {
        if (events && events[k]) FB_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(events[k]), st));
        return FB_OK;
    };
    unsigned long long* work = reinterpret_cast<unsigned long long*>(d_work);
    const RecDesc* D = H->d_desc;
    const int sms = fb_sm_count();
    const int dyn = sms * (ctas_per_sm > 0 ? ctas_per_sm : 16);  // CTAs of the active-block passes
    if (int rc = mark(0)) return rc;
    FB_CUDA(cudaMemsetAsync(H->status, 0, H->state_bytes, st));
    k_b_prepare<<<fb_div_up(H->n_prims, 128), 128, 0, st>>>(D, H->prims, H->n_prims);
    FB_LAUNCH();
    k_b_full_list<<<fb_div_up(H->n_chain, 256), 256, 0, st>>>(D, H->chain, H->n_chain);
    FB_LAUNCH();
    k_b_cull<0><<<fb_div_up(H->n_coarse * 32, 128), 128, 0, st>>>(D, H->coarse, H->n_coarse);
    FB_LAUNCH();
    k_b_cull<1><<<fb_div_up(H->n_super * 32, 128), 128, 0, st>>>(D, H->super_, H->n_super);
    FB_LAUNCH();
    if (int rc = mark(1)) return rc;
    if (H->n_cclass) {
        k_b_classify_blocks<<<fb_div_up(H->n_cclass, 128), 128, 0, st>>>(D, H->cclass, H->n_cclass, H->cursors);
        FB_LAUNCH();
    }
    if (int rc = mark(2)) return rc;
    k_b_compact<<<(unsigned)H->n_tiles, 256, 0, st>>>(D, H->tiles, H->misc, kLookbackSpins);
    FB_LAUNCH();
    LeafGroups LG;
    for (int q = 0; q < kLeafGroups; ++q) {
        LG.g[q] = H->leaf[q];
        LG.pre[q] = H->leaf_pre[q];
    }
    k_batch_offsets<<<1, 32, 0, st>>>(D, H->n, capacity, H->tile_off, H->leaf_count, LG, H->occ, H->occ_pre, H->misc);
    FB_LAUNCH();
    if (int rc = mark(3)) return rc;
    if (int rc = mark(4)) return rc;
    for (int q = 0; q < kLeafGroups; ++q) {
        if (!H->leaf[q].m) continue;
        const Group& W = H->leaf[q];
        switch (q) {
        case 0: k_b_leaf<4, false><<<dyn, 32 * kLeafWarps, 0, st>>>(D, W, d_tiles, H->tile_off, work); break;
        case 1: k_b_leaf<8, false><<<dyn, 32 * kLeafWarps, 0, st>>>(D, W, d_tiles, H->tile_off, work); break;
        case 2: k_b_leaf<16, false><<<dyn, 32 * kLeafWarps, 0, st>>>(D, W, d_tiles, H->tile_off, work); break;
        case 3: k_b_leaf<4, true><<<dyn, 32 * kLeafWarps, 0, st>>>(D, W, d_tiles, H->tile_off, work); break;
        case 4: k_b_leaf<8, true><<<dyn, 32 * kLeafWarps, 0, st>>>(D, W, d_tiles, H->tile_off, work); break;
        default: k_b_leaf<16, true><<<dyn, 32 * kLeafWarps, 0, st>>>(D, W, d_tiles, H->tile_off, work);
        }
        FB_LAUNCH();
    }
    return mark(5);
}

// Device arrays of a batch's outputs: tile_off[n] (int64, floats into the arena) and
// leaf_count[n] (int32, tiles written per recipe); valid after a build on the build's stream.
int fb_batch_outputs(void* batch, const int64_t** tile_off, const int32_t** leaf_count) noexcept {
    BatchHost* H = static_cast<BatchHost*>(batch);
    if (!H) return FB_INVALID;
    if (tile_off) *tile_off = H->tile_off;
    if (leaf_count) *leaf_count = H->leaf_count;
    return FB_OK;
}

// Occupancy masks (uint8, 1 where the field is negative) of the recipes whose items carry d_slot /
// d_mask, from the last build's tiles in d_tiles; stream-ordered after that build, no host
// synchronisation (5 launches at most).
int fb_batch_occupancy_device(void* batch, const float* d_tiles, void* stream) noexcept {
    BatchHost* H = static_cast<BatchHost*>(batch);
    if (!H || !d_tiles || (reinterpret_cast<uintptr_t>(d_tiles) & 15)) return FB_INVALID;
    if (!H->occ.m) return FB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const RecDesc* D = H->d_desc;
    k_b_fill_slot<<<fb_div_up(H->n_occ_blocks, 256), 256, 0, st>>>(D, H->occ_blocks, H->n_occ_blocks);
    FB_LAUNCH();
    k_b_slot_map<<<fb_sm_count() * 8, 256, 0, st>>>(D, H->occ);
    FB_LAUNCH();
    for (int q = 0; q < 3; ++q) {
        const int64_t n = H->n_occ_rows[q];
        if (!n) continue;
        const int grid = fb_div_up(n, 256);
        if (q == 0) k_b_occupancy<4><<<grid, 256, 0, st>>>(D, H->occ_rows[0], n, d_tiles, H->tile_off);
        else if (q == 1) k_b_occupancy<8><<<grid, 256, 0, st>>>(D, H->occ_rows[1], n, d_tiles, H->tile_off);
        else k_b_occupancy<16><<<grid, 256, 0, st>>>(D, H->occ_rows[2], n, d_tiles, H->tile_off);
        FB_LAUNCH();
    }
    return FB_OK;
}

// Launches one build enqueues (the batch's own kernels and its one memset).
int32_t fb_batch_launches(void* batch) noexcept {
    BatchHost* H = static_cast<BatchHost*>(batch);
    if (!H) return -1;
    int n = 1 + 4 + 2;  // memset; prepare, full list, two cull levels; compaction, offsets
    if (H->n_cclass) n += 1;
    for (int q = 0; q < kLeafGroups; ++q) n += H->leaf[q].m ? 1 : 0;
    return n;
}

// Status of the last build (synchronises): 0, 6 when a compaction wait gave up, 8 when the tile
// arena was too small (recipes beyond it got fewer tiles than active blocks).
int fb_batch_status(void* batch, void* stream) noexcept {
    BatchHost* H = static_cast<BatchHost*>(batch);
    if (!H) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int flags[3] = {0, 0, 0};
    FB_CUDA(cudaMemcpyAsync(flags, H->misc, 12, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    if (flags[1]) return FB_TIMEOUT;
    if (flags[2]) return FB_CAPACITY;
    return FB_OK;
}

void fb_batch_destroy(void* batch) noexcept {
    BatchHost* H = static_cast<BatchHost*>(batch);
    if (!H) return;
    if (H->dev) cudaFree(H->dev);  // waits for the device's outstanding work first
    delete H;
}

}  // extern "C"

namespace {

}  // namespace

extern "C" {

// Scratch bytes of one analytic build (classify + leaf) for this geometry and program size.
int64_t fb_field_scratch_bytes(const FbGeom* g, int32_t n_prims, int32_t n_chain) {
    if (!g || !geom_ok(*g) || n_prims < 1 || n_chain < 1) return -1;
    const Geo G = make_geo(*g);
    return make_plan(G, n_prims, n_chain).total;
}

// Classification + compaction of an analytic recipe.  mode 1: `chain` is the left-deep chain
// (CH_* ops, culled); mode 0: `chain` is a general postfix program (OP_* ops, float64, no culling).
// Writes kind[n_blocks], corner_min_abs[n_blocks], active[<= n_blocks] ascending and count[0].
int fb_field_classify_device(const FbGeom* g, const FbPrim* d_prims, int32_t n_prims, const FbInsn* d_chain,
                             int32_t n_chain, int32_t mode, int32_t* d_kind, float* d_cma, int32_t* d_active,
                             int32_t* d_count, void* d_scratch, int64_t scratch_len, void* stream) noexcept {
    if (!g) return FB_INVALID;
    return classify_impl(*g, d_prims, n_prims, d_chain, n_chain, mode, d_kind, d_cma, d_active, d_count, d_scratch,
                         scratch_len, static_cast<cudaStream_t>(stream));
}

// Leaf tiles of the first min(count, capacity) active blocks, tile order (li, lj, lk).  Uses the
// culling lists left in `d_scratch` by fb_field_classify_device for the same recipe and geometry.
int fb_field_leaf_device(const FbGeom* g, const FbPrim* d_prims, int32_t n_prims, const FbInsn* d_chain,
                         int32_t n_chain, int32_t mode, const int32_t* d_kind, const int32_t* d_active,
                         const int32_t* d_count, float* d_tiles, int64_t capacity, void* d_scratch, int64_t scratch_len,
                         void* stream) noexcept {
    if (!g) return FB_INVALID;
    return leaf_impl(*g, d_prims, n_prims, d_chain, n_chain, mode, d_kind, d_active, d_count, d_tiles, capacity, d_scratch,
                     scratch_len, static_cast<cudaStream_t>(stream));
}

// fb_field_leaf_device plus a count of the executed work: d_work[0] += primitive evaluations,
// d_work[1] += float32 operations (two uint64 counters, accumulated).
int fb_field_leaf_work_device(const FbGeom* g, const FbPrim* d_prims, int32_t n_prims, const FbInsn* d_chain,
                              int32_t n_chain, int32_t mode, const int32_t* d_kind, const int32_t* d_active,
                              const int32_t* d_count, float* d_tiles, int64_t capacity, void* d_scratch,
                              int64_t scratch_len, uint64_t* d_work, void* stream) noexcept {
    if (!g || !d_work) return FB_INVALID;
    return leaf_impl(*g, d_prims, n_prims, d_chain, n_chain, mode, d_kind, d_active, d_count, d_tiles, capacity, d_scratch,
                     scratch_len, static_cast<cudaStream_t>(stream), reinterpret_cast<unsigned long long*>(d_work));
}

// Whole analytic build in one stream-ordered call (classify, compact, leaf tiles); tiles beyond
// `capacity` active blocks are not written (count still reports the full number).
int fb_field_build_device(const FbGeom* g, const FbPrim* d_prims, int32_t n_prims, const FbInsn* d_chain,
                          int32_t n_chain, int32_t mode, int32_t* d_kind, float* d_cma, int32_t* d_active,
                          int32_t* d_count, float* d_tiles, int64_t capacity, void* d_scratch, int64_t scratch_len,
                          void* stream) noexcept {
    if (!g) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = classify_impl(*g, d_prims, n_prims, d_chain, n_chain, mode, d_kind, d_cma, d_active, d_count, d_scratch,
                           scratch_len, st);
    if (rc) return rc;
    return leaf_impl(*g, d_prims, n_prims, d_chain, n_chain, mode, d_kind, d_active, d_count, d_tiles, capacity,
                     d_scratch, scratch_len, st);
}

// Scratch bytes of a dense classification (compaction state only).
int64_t fb_dense_scratch_bytes(int64_t nx, int64_t ny, int64_t nz, int32_t block) {
    if (nx < 1 || ny < 1 || nz < 1 || block < 1 || block > 1024) return -1;
    const int64_t nb = ((nx + block - 1) / block) * ((ny + block - 1) / block) * ((nz + block - 1) / block);
    return align256(nb / kTile * 8 + 8) + 256 + 256;
}

// Dense-input classification, compaction and tile gather: the reference's k_classify_dense /
// k_eval_tile_dense and meshsdf_classify_cpu / meshsdf_tiles_cpu
// (src/field_engine/mesh_sdf_native_v1/field.cpp:229-273) on the device.  d_cma may be null.
int fb_dense_classify_device(const float* d_dense, int64_t nx, int64_t ny, int64_t nz, int32_t block, float margin,
                             int32_t* d_kind, float* d_cma, int32_t* d_active, int32_t* d_count, float* d_tiles,
                             int64_t capacity, void* d_scratch, int64_t scratch_len, void* stream) noexcept {
    if (!d_dense || !d_kind || !d_active || !d_count || nx < 1 || ny < 1 || nz < 1 || block < 1 || block > 1024 ||
        !d_scratch || capacity < 0 || (capacity > 0 && !d_tiles))
        return FB_INVALID;
    if (scratch_len < fb_dense_scratch_bytes(nx, ny, nz, block)) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nby = (int)((ny + block - 1) / block), nbz = (int)((nz + block - 1) / block);
    const int64_t nblocks = ((nx + block - 1) / block) * nby * nbz;
    k_classify_dense<<<fb_div_up(nblocks, 256), 256, 0, st>>>(d_dense, nx, ny, nz, block, nby, nbz, nblocks, margin,
                                                              d_kind, d_cma);
    FB_LAUNCH();
    char* b = static_cast<char*>(d_scratch);
    const int64_t ntiles = (nblocks + kTile - 1) / kTile;
    unsigned long long* status = reinterpret_cast<unsigned long long*>(b);
    int* misc = reinterpret_cast<int*>(b + align256(ntiles * 8));
    if (int rc = launch_compact(d_kind, nblocks, d_active, d_count, status, misc, st)) return rc;
    if (capacity > 0) {
        k_tiles_dense<<<fb_sm_count() * 8, 256, 0, st>>>(d_dense, nx, ny, nz, block, nby, nbz, d_active, d_count,
                                                          capacity, d_tiles);
        FB_LAUNCH();
    }
    return FB_OK;
}

// Dense reconstruction of a sparse field; d_slot is caller scratch of n_blocks int32.
int fb_field_reconstruct_device(const int32_t* d_kind, const int32_t* d_active, int64_t n_active, const float* d_tiles,
                                int64_t nx, int64_t ny, int64_t nz, int32_t block, float big, int32_t* d_slot,
                                float* d_out, void* stream) noexcept {
    if (!d_kind || !d_slot || !d_out || nx < 1 || ny < 1 || nz < 1 || block < 1 || n_active < 0 ||
        (n_active > 0 && (!d_active || !d_tiles)))
        return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nby = (int)((ny + block - 1) / block), nbz = (int)((nz + block - 1) / block);
    const int64_t nblocks = ((nx + block - 1) / block) * nby * nbz;
    FB_CUDA(cudaMemsetAsync(d_slot, 0xff, nblocks * 4, st));
    if (n_active > 0) {
        k_slot_map<<<fb_div_up(n_active, 256), 256, 0, st>>>(d_active, n_active, d_slot);
        FB_LAUNCH();
    }
    k_reconstruct<<<fb_div_up(nx * ny * nz, 256), 256, 0, st>>>(d_kind, d_slot, d_tiles, nx, ny, nz, block, nby, nbz,
                                                                big, d_out);
    FB_LAUNCH();
    return FB_OK;
}

// float32 primitive mirror (128-byte records) for the point-query kernels.
int fb_query_prepare(const FbPrim* d_prims, int32_t n_prims, void* d_primf, void* stream) noexcept {
    if (!d_prims || !d_primf || n_prims < 1) return FB_INVALID;
    k_prepare_prims<<<fb_div_up(n_prims, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        d_prims, n_prims, static_cast<PrimF*>(d_primf));
    FB_LAUNCH();
    return FB_OK;
}

// Device addresses of a classification's culling lists inside its scratch (for accelerated point
// queries): superblock pool base, offsets and lengths; per-block offsets, lengths and pool, the
// pool's capacity, and whether every block has a list (else only blocks of kind 0).
int fb_field_accel(const FbGeom* g, int32_t n_prims, int32_t n_chain, const void* d_scratch, const void** pool,
                   const int64_t** sb_off, const int32_t** sb_len, const int32_t** blk_off, const int32_t** blk_len,
                   const uint32_t** blk_pool, int64_t* blk_cap, int32_t* blk_all) noexcept {
    if (!g || !geom_ok(*g) || !d_scratch || n_prims < 1 || n_chain < 1) return FB_INVALID;
    const Geo G = make_geo(*g);
    const Plan P = make_plan(G, n_prims, n_chain);
    const char* b = static_cast<const char*>(d_scratch);
    if (pool) *pool = b + P.pool;
    if (sb_off) *sb_off = reinterpret_cast<const int64_t*>(b + P.off) + G.ncoarse;
    if (sb_len) *sb_len = reinterpret_cast<const int32_t*>(b + P.len) + G.ncoarse;
    if (blk_off) *blk_off = reinterpret_cast<const int32_t*>(b + P.blk_off);
    if (blk_len) *blk_len = reinterpret_cast<const int32_t*>(b + P.blk_len);
    if (blk_pool) *blk_pool = reinterpret_cast<const uint32_t*>(b + P.blk_pool);
    if (blk_cap) *blk_cap = P.blk_cap;
    if (blk_all) *blk_all = 0;  // lists are kept for blocks of kind 0 only
    return FB_OK;
}

// Occupancy mask (uint8, 1 = solid) of a built field, from device-resident kind / active / count /
// tiles; stream-ordered, no host synchronisation.  d_slot: caller scratch of n_blocks int32.
int fb_field_occupancy_device(const int32_t* d_kind, const int32_t* d_active, const int32_t* d_count,
                              const float* d_tiles, int64_t capacity, int64_t nx, int64_t ny, int64_t nz,
                              int32_t block, int32_t* d_slot, uint8_t* d_mask, void* stream) noexcept {
    if (!d_kind || !d_active || !d_count || !d_tiles || !d_slot || !d_mask || nx < 1 || ny < 1 || nz < 1 ||
        (block != 4 && block != 8 && block != 16) || capacity < 0 || nx > INT32_MAX || ny > INT32_MAX ||
        nz > INT32_MAX || (reinterpret_cast<uintptr_t>(d_tiles) & 15) || (reinterpret_cast<uintptr_t>(d_mask) & 15))
        return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nby = (int)((ny + block - 1) / block), nbz = (int)((nz + block - 1) / block);
    const int64_t nblocks = ((nx + block - 1) / block) * nby * nbz;
    FB_CUDA(cudaMemsetAsync(d_slot, 0xff, nblocks * 4, st));
    k_slot_map_dev<<<fb_sm_count() * 4, 256, 0, st>>>(d_active, d_count, capacity, d_slot);
    FB_LAUNCH();
    const int64_t items = nx * ny * ((nz + 15) / 16);
    const int grid = (int)std::min<int64_t>((items + 255) / 256, (int64_t)fb_sm_count() * 16);
    switch (block) {
        case 4: k_occupancy<4><<<grid, 256, 0, st>>>(d_kind, d_slot, d_tiles, (int)nx, (int)ny, (int)nz, nby, nbz, d_mask); break;
        case 8: k_occupancy<8><<<grid, 256, 0, st>>>(d_kind, d_slot, d_tiles, (int)nx, (int)ny, (int)nz, nby, nbz, d_mask); break;
        default: k_occupancy<16><<<grid, 256, 0, st>>>(d_kind, d_slot, d_tiles, (int)nx, (int)ny, (int)nz, nby, nbz, d_mask); break;
    }
    FB_LAUNCH();
    return FB_OK;
}

// int64 fixed-point checksum of the negative values (accumulates into d_out[0]).
int fb_checksum_i64_device(const float* d_values, int64_t n, double scale, int64_t* d_out, void* stream) noexcept {
    if (!d_values || !d_out || n < 0) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n == 0) return FB_OK;
    k_checksum_i64<<<std::min<int64_t>(fb_div_up(n, 256), fb_sm_count() * 8), 256, 0, st>>>(
        d_values, n, scale, reinterpret_cast<unsigned long long*>(d_out));
    FB_LAUNCH();
    return FB_OK;
}

// Sum of n int32 values into d_out[0] (set to zero first, on the stream).
int fb_sum_i32_device(const int32_t* d_values, int64_t n, int64_t* d_out, void* stream) noexcept {
    if (!d_out || n < 0 || (n > 0 && !d_values)) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    FB_CUDA(cudaMemsetAsync(d_out, 0, sizeof(int64_t), st));
    if (n == 0) return FB_OK;
    k_sum_i32<<<std::min<int64_t>(fb_div_up(n, 256), fb_sm_count() * 8), 256, 0, st>>>(
        d_values, n, reinterpret_cast<unsigned long long*>(d_out));
    FB_LAUNCH();
    return FB_OK;
}

// Test of the compaction's bounded wait: the tile ticket starts at 1, so no CTA takes tile 0 and its
// status word is never published; tile 1's look-back waits on it, gives up after `spin_limit`
// sleeps, raises the error flag and publishes its own status, so every later wait ends.  Returns
// FB_TIMEOUT (6) when the flag was raised, as the product path reports it.  d_scratch: the
// compaction state of fb_dense_scratch_bytes(n, 1, 1, 1).  Needs n > 2048 (two tiles or more); the
// active ids written are not meaningful.
int fb_compact_timeout_probe(const int32_t* d_kind, int64_t n, int32_t* d_active, int32_t* d_count, void* d_scratch,
                             int64_t scratch_len, int64_t spin_limit, void* stream) noexcept {
    const int64_t ntiles = (n + kTile - 1) / kTile;
    if (!d_kind || !d_active || !d_count || !d_scratch || ntiles < 2 || spin_limit < 1 ||
        scratch_len < fb_dense_scratch_bytes(n, 1, 1, 1))
        return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* b = static_cast<char*>(d_scratch);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(b);
    int* misc = reinterpret_cast<int*>(b + align256(ntiles * 8));
    const int one = 1;
    FB_CUDA(cudaMemsetAsync(status, 0, ntiles * 8, st));
    FB_CUDA(cudaMemsetAsync(misc, 0, 256, st));
    FB_CUDA(cudaMemcpyAsync(misc, &one, sizeof(int), cudaMemcpyHostToDevice, st));  // ticket starts at tile 1
    k_compact<<<(unsigned)(ntiles - 1), 256, 0, st>>>(d_kind, n, d_active, d_count, status, misc, ntiles, spin_limit);
    FB_LAUNCH();
    int flags[2] = {0, 0};
    FB_CUDA(cudaMemcpyAsync(flags, misc, 8, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    return flags[1] ? FB_TIMEOUT : FB_OK;
}

// The grouped evaluations' square root (sqrt_sum) over n device floats, stream-ordered.
int fb_sqrt_sum_probe(const float* d_x, float* d_out, int64_t n, void* stream) noexcept {
    if (!d_x || !d_out || n < 0) return FB_INVALID;
    if (n == 0) return FB_OK;
    const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_sqrt_sum<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_x, d_out, n);
    FB_LAUNCH();
    return FB_OK;
}

// The 8^3 tiles' quotient (quotient2) of n device float pairs, stream-ordered.
int fb_quotient_probe(const float* d_num, const float* d_den, float* d_out, int64_t n, void* stream) noexcept {
    if (!d_num || !d_den || !d_out || n < 0) return FB_INVALID;
    if (n == 0) return FB_OK;
    const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_quotient<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_num, d_den, d_out, n);
    FB_LAUNCH();
    return FB_OK;
}

// Error flag of the last compaction (1 when a bounded wait gave up), read from the scratch.
int fb_field_compact_error(const FbGeom* g, int32_t n_prims, int32_t n_chain, const void* d_scratch, void* stream) {
    if (!g || !geom_ok(*g) || !d_scratch) return FB_INVALID;
    const Geo G = make_geo(*g);
    const Plan P = make_plan(G, n_prims, n_chain);
    int flags[2] = {0, 0};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    FB_CUDA(cudaMemcpyAsync(flags, static_cast<const char*>(d_scratch) + P.misc, 8, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    return flags[1] ? FB_TIMEOUT : FB_OK;
}

}  // extern "C"
