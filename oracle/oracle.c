/*
 * CPU oracle for the block-sparse SDF field path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file restates the reference algorithms in plain C so that the tests, the smoke check and
 * the CPU-baseline leg of the benchmark can check the CUDA library against them.  It is never
 * linked into the product library and nothing in the product imports it.
 *
 * Built with -O2 -fopenmp -ffp-contract=off (see oracle/Makefile): every floating-point
 * operation below is rounded exactly once in the written order, so that the float64 results are
 * reproducible and the float32 ones follow NumPy's elementwise rounding.
 *
 * Every function cites the reference file:line it restates (paths relative to the reference
 * project root).  Parity pins live in tests/golden/ (fixtures made from the reference's own
 * captures and compiled code by tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_INVALID 1
#define OR_RUNTIME 2

/* ------------------------------------------------------------------------------------------------
 * Exact integer squared EDT
 * ---------------------------------------------------------------------------------------------- */

/* Sentinel for "no site": sum over axes of (n-1)^2, plus one.
 * src/field_engine/field_edt_integer_v1.py:17 and edt_native_large_v1/edt.cu:42. */
static int32_t or_sentinel(int nx, int ny, int nz) {
    return (nx - 1) * (nx - 1) + (ny - 1) * (ny - 1) + (nz - 1) * (nz - 1) + 1;
}

/* First integer position at which the parabola rooted at q is strictly below the one rooted at v,
 * with floor division that rounds toward minus infinity for negative numerators.
 * src/field_engine/edt_native_linear_v1/edt.cu:8-12 (exact integer floor). */
static int or_separation(int q, int v, int fq, int fv) {
    int num = fq + q * q - fv - v * v;
    int den = 2 * (q - v);
    int fl = num >= 0 ? num / den : -((-num + den - 1) / den);
    return fl + 1;
}

/* One 1-D lower-envelope pass along a strided line (Felzenszwalb & Huttenlocher, integer form).
 * src/field_engine/edt_native_linear_v1/edt.cu:13-29. */
static void or_envelope_line(const int32_t *src, int32_t *dst, int64_t base, int64_t stride, int len,
                             int *site, int *start) {
    int k = 0;
    site[0] = 0;
    start[0] = -2147483647;
    start[1] = 2147483647;
    for (int q = 1; q < len; ++q) {
        int fq = src[base + (int64_t)q * stride];
        int s = or_separation(q, site[k], fq, src[base + (int64_t)site[k] * stride]);
        while (s <= start[k]) {
            --k;
            s = or_separation(q, site[k], fq, src[base + (int64_t)site[k] * stride]);
        }
        ++k;
        site[k] = q;
        start[k] = s;
        start[k + 1] = 2147483647;
    }
    k = 0;
    for (int q = 0; q < len; ++q) {
        while (start[k + 1] <= q) ++k;
        int d = q - site[k];
        dst[base + (int64_t)q * stride] = src[base + (int64_t)site[k] * stride] + d * d;
    }
}

/* Squared distance of every voxel to the nearest zero of `binary` (C order, z fastest).
 * Axis order 0,1,2 with strides ny*nz, nz, 1.  src/field_engine/field_edt_integer_v1.py:14-26
 * (min-plus definition), src/field_engine/edt_native_large_v1/edt.cu:33-61 (host contract).
 * Returns 1 for invalid input (a null pointer, an axis outside 1..4096). */
int or_edt_squared(const uint8_t *binary, int nx, int ny, int nz, int32_t *out) {
    if (!binary || !out || nx < 1 || ny < 1 || nz < 1 || nx > 4096 || ny > 4096 || nz > 4096)
        return OR_INVALID;
    int64_t size = (int64_t)nx * ny * nz;
    int32_t sentinel = or_sentinel(nx, ny, nz);
    int32_t *tmp = (int32_t *)malloc((size_t)size * sizeof(int32_t));
    if (!tmp) return OR_RUNTIME;
    for (int64_t i = 0; i < size; ++i) out[i] = binary[i] ? sentinel : 0;
    int lengths[3] = {nx, ny, nz};
    int64_t strides[3] = {(int64_t)ny * nz, nz, 1};
    int32_t *a = out, *b = tmp;
    for (int axis = 0; axis < 3; ++axis) {
        int len = lengths[axis];
        int64_t stride = strides[axis];
        int64_t lines = size / len;
#pragma omp parallel
        {
            int *site = (int *)malloc(sizeof(int) * (len + 1));
            int *start = (int *)malloc(sizeof(int) * (len + 2));
#pragma omp for schedule(static)
            for (int64_t line = 0; line < lines; ++line) {
                int64_t base = (line / stride) * len * stride + line % stride;
                or_envelope_line(a, b, base, stride, len, site, start);
            }
            free(site);
            free(start);
        }
        int32_t *t = a; a = b; b = t;
    }
    if (a != out) memcpy(out, a, (size_t)size * sizeof(int32_t));
    free(tmp);
    return OR_OK;
}

/* Direct min-plus per voxel: O(n) per voxel and axis.  Used by the tests to pin the envelope
 * restatement on small grids.  src/field_engine/field_edt_integer_v1.py:19-25. */
int or_edt_squared_brute(const uint8_t *binary, int nx, int ny, int nz, int32_t *out) {
    if (!binary || !out || nx < 1 || ny < 1 || nz < 1) return OR_INVALID;
    int64_t size = (int64_t)nx * ny * nz;
    int32_t sentinel = or_sentinel(nx, ny, nz);
    int32_t *tmp = (int32_t *)malloc((size_t)size * sizeof(int32_t));
    if (!tmp) return OR_RUNTIME;
    for (int64_t i = 0; i < size; ++i) out[i] = binary[i] ? sentinel : 0;
    int lengths[3] = {nx, ny, nz};
    int64_t strides[3] = {(int64_t)ny * nz, nz, 1};
    int32_t *a = out, *b = tmp;
    for (int axis = 0; axis < 3; ++axis) {
        int len = lengths[axis];
        int64_t stride = strides[axis];
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < size; ++v) {
            int pos = (int)((v / stride) % len);
            int64_t base = v - (int64_t)pos * stride;
            int32_t best = INT32_MAX;
            for (int s = 0; s < len; ++s) {
                int32_t c = a[base + (int64_t)s * stride] + (s - pos) * (s - pos);
                if (c < best) best = c;
            }
            b[v] = best;
        }
        int32_t *t = a; a = b; b = t;
    }
    if (a != out) memcpy(out, a, (size_t)size * sizeof(int32_t));
    free(tmp);
    return OR_OK;
}

/* Signed distance from the two squared transforms: outside = f32(sqrt(f64(sq_out)) * pitch),
 * inside likewise, d = outside - inside in f32, then d - sign(d) * f32(0.5 * pitch).
 * src/field_engine/edt_persistent_pair_v1/edt.cu:36-42 and field_edt_integer_v1.py:40-43.
 * `mask` is the solid; polarity 0 measures to the nearest solid voxel, polarity 1 to the nearest
 * empty one (edt.cu:32-35).  `pair` (nullable) receives both squared arrays, polarity-major. */
int or_edt_signed(const uint8_t *mask, int nx, int ny, int nz, double pitch, float *out,
                  int32_t *pair) {
    if (!mask || !out || nx < 1 || ny < 1 || nz < 1) return OR_INVALID;
    if (!isfinite(pitch) || pitch < 1e-12 || pitch > 1e12) return OR_INVALID;
    int64_t size = (int64_t)nx * ny * nz;
    int32_t *sq = (int32_t *)malloc((size_t)size * 2 * sizeof(int32_t));
    uint8_t *inv = (uint8_t *)malloc((size_t)size);
    if (!sq || !inv) {
        free(sq);
        free(inv);
        return OR_RUNTIME;
    }
    for (int64_t i = 0; i < size; ++i) inv[i] = mask[i] ? 0 : 1;
    int rc = or_edt_squared(inv, nx, ny, nz, sq);               /* sites = solid voxels */
    if (rc == OR_OK) rc = or_edt_squared(mask, nx, ny, nz, sq + size); /* sites = empty voxels */
    if (rc == OR_OK) {
        float half = (float)(0.5 * pitch);
        for (int64_t i = 0; i < size; ++i) {
            float o = (float)(sqrt((double)sq[i]) * pitch);
            float n = (float)(sqrt((double)sq[size + i]) * pitch);
            float d = o - n;
            float sg = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
            float corr = sg * half;
            out[i] = d - corr;
        }
        if (pair) memcpy(pair, sq, (size_t)size * 2 * sizeof(int32_t));
    }
    free(sq);
    free(inv);
    return rc;
}

/* ------------------------------------------------------------------------------------------------
 * Dense-input block classification and tile gather
 * ---------------------------------------------------------------------------------------------- */

/* Eight corners per block at voxel offsets {0, B} clamped to n-1; a corner value v counts as
 * positive when v >= 0; kind = 0 if both signs occur or min|v| <= margin, else -1 (all negative) or
 * +1.  src/field_engine/faltkarna_v1_mesh_to_sdf.py:602-632 (k_classify_dense) and
 * src/field_engine/mesh_sdf_native_v1/field.cpp:229-252.  `cma` (nullable) gets min|v|. */
int or_classify_dense(const float *dense, int64_t nx, int64_t ny, int64_t nz, int64_t block, float margin,
                      int32_t *kind, float *cma) {
    if (!dense || !kind || nx < 1 || ny < 1 || nz < 1 || block < 1 || block > 1024) return OR_INVALID;
    int64_t nbx = (nx + block - 1) / block, nby = (ny + block - 1) / block, nbz = (nz + block - 1) / block;
    int64_t nb = nbx * nby * nbz;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < nb; ++t) {
        int64_t bk = t % nbz, bj = (t / nbz) % nby, bi = t / (nbz * nby);
        float mn = 1.0e30f;
        int pos = 0, neg = 0;
        for (int c = 0; c < 8; ++c) {
            int64_t cx = bi * block + (c & 1) * block;
            int64_t cy = bj * block + ((c >> 1) & 1) * block;
            int64_t cz = bk * block + ((c >> 2) & 1) * block;
            if (cx > nx - 1) cx = nx - 1;
            if (cy > ny - 1) cy = ny - 1;
            if (cz > nz - 1) cz = nz - 1;
            float v = dense[(cx * ny + cy) * nz + cz];
            float a = fabsf(v);
            if (a < mn) mn = a;
            if (v >= 0.0f) pos = 1; else neg = 1;
        }
        if (cma) cma[t] = mn;
        kind[t] = (pos && neg) ? 0 : ((mn <= margin) ? 0 : (neg ? -1 : 1));
    }
    return OR_OK;
}

/* Tile gather of the active blocks, C order (li, lj, lk), voxel index clamped to n-1.
 * src/field_engine/faltkarna_v1_mesh_to_sdf.py:635-657, mesh_sdf_native_v1/field.cpp:254-273. */
int or_tiles_dense(const float *dense, int64_t nx, int64_t ny, int64_t nz, int64_t block,
                   const int32_t *active, int64_t nact, float *out) {
    if (!dense || nx < 1 || ny < 1 || nz < 1 || block < 1 || nact < 0 || (nact > 0 && (!active || !out)))
        return OR_INVALID;
    int64_t nby = (ny + block - 1) / block, nbz = (nz + block - 1) / block, b3 = block * block * block;
    int64_t nb = ((nx + block - 1) / block) * nby * nbz;
    for (int64_t a = 0; a < nact; ++a)
        if (active[a] < 0 || active[a] >= nb) return OR_RUNTIME;
#pragma omp parallel for schedule(static)
    for (int64_t a = 0; a < nact; ++a) {
        int64_t lin = active[a];
        int64_t bk = lin % nbz, bi = lin / (nbz * nby), bj = (lin / nbz) % nby;
        float *o = out + a * b3;
        for (int64_t li = 0; li < block; ++li)
            for (int64_t lj = 0; lj < block; ++lj)
                for (int64_t lk = 0; lk < block; ++lk) {
                    int64_t vx = bi * block + li, vy = bj * block + lj, vz = bk * block + lk;
                    if (vx > nx - 1) vx = nx - 1;
                    if (vy > ny - 1) vy = ny - 1;
                    if (vz > nz - 1) vz = nz - 1;
                    *o++ = dense[(vx * ny + vy) * nz + vz];
                }
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------------------------------
 * Ordered CSG over sampled fields on one grid (dense operands)
 * ---------------------------------------------------------------------------------------------- */

typedef struct {
    int32_t op, left, right, pad;
    double offset;
} or_csg_insn;

/* Instruction n produces value id fields+n; union = (a < b ? a : b), difference = (a > -b ? a : -b)
 * (on equality NumPy keeps the second operand, signed zeros included), offset = f32(f64(a) - d).
 * A non-finite result is status 4.  src/field_engine/csg_batch_native_v1/execute.cpp:10-53 and
 * src/field_engine/field_csg_batch_v1.py:18-79 (validation 19-58). */
int or_csg_execute(const float *const *fields, int32_t nfields, const int32_t *shape, const or_csg_insn *prog,
                   int32_t ninsn, float *out) {
    if (!fields || !shape || !prog || !out || nfields < 1 || nfields > 256 || ninsn < 1 || ninsn > 1024)
        return 1;
    int64_t total = 1;
    for (int a = 0; a < 3; ++a) {
        if (shape[a] < 1 || shape[a] > 4096) return 1;
        total *= shape[a];
    }
    if (total > 16777216) return 1;
    for (int n = 0; n < ninsn; ++n) {
        const or_csg_insn *p = &prog[n];
        if (p->op < 0 || p->op > 2 || p->left < 0 || p->left >= nfields + n) return 2;
        if (p->op == 2) {
            if (!isfinite(p->offset)) return 2;
        } else if (p->right < 0 || p->right >= nfields + n) {
            return 2;
        }
    }
    int bad = 0;
    float *vals = (float *)malloc(sizeof(float) * (size_t)(nfields + ninsn));
    if (!vals) return 5;
    for (int64_t i = 0; i < total && !bad; ++i) {
        for (int f = 0; f < nfields; ++f) vals[f] = fields[f][i];
        for (int n = 0; n < ninsn; ++n) {
            const or_csg_insn *p = &prog[n];
            float a = vals[p->left], r;
            if (p->op == 2) {
                r = (float)((double)a - p->offset);
            } else {
                float b = p->op == 0 ? vals[p->right] : -vals[p->right];
                r = p->op == 0 ? (a < b ? a : b) : (a > b ? a : b);
            }
            if (!isfinite(r)) {
                bad = 1;
                break;
            }
            vals[nfields + n] = r;
        }
        out[i] = vals[nfields + ninsn - 1];
    }
    free(vals);
    return bad ? 4 : 0;
}

/* ------------------------------------------------------------------------------------------------
 * Lossless adaptive packing (split decisions, node order, payload order)
 * ---------------------------------------------------------------------------------------------- */

#pragma pack(push, 1)
typedef struct {
    int32_t lo[3], shape[3], stored[3], children[2];
    int64_t offset;
} or_node;
#pragma pack(pop)

typedef struct or_tree {
    int lo[3], shape[3], stored[3];
    int64_t cost;
    struct or_tree *left, *right;
} or_tree;

typedef struct {
    const uint32_t *bits;
    int64_t s0, s1;
    int threshold;
} or_packer;

static uint32_t or_at(const or_packer *p, int x, int y, int z) { return p->bits[x * p->s0 + y * p->s1 + z]; }

static void or_tree_free(or_tree *t) {
    if (!t) return;
    or_tree_free(t->left);
    or_tree_free(t->right);
    free(t);
}

/* Collapse each axis along which the samples are bitwise invariant; a leaf if the reduced size is
 * <= 64 or the region holds <= threshold samples; else split the varying axis with the largest
 * extent at extent/2 and keep the split only if 52 + cost(left) + cost(right) < cost(leaf).
 * src/field_engine/adaptive_pack_native_v1/pack.cpp:18-42, adaptive_sample_blocks_v1.py:19-43. */
static or_tree *or_build(const or_packer *p, const int *lo, const int *shape) {
    or_tree *t = (or_tree *)calloc(1, sizeof(or_tree));
    if (!t) return NULL;
    int64_t count = 1, reduced = 1;
    for (int a = 0; a < 3; ++a) {
        t->lo[a] = lo[a];
        t->shape[a] = shape[a];
        count *= shape[a];
    }
    for (int axis = 0; axis < 3; ++axis) {
        int same = 1;
        for (int x = 0; x < shape[0] && same; ++x)
            for (int y = 0; y < shape[1] && same; ++y)
                for (int z = 0; z < shape[2] && same; ++z) {
                    int q[3] = {x, y, z};
                    q[axis] = 0;
                    same = or_at(p, lo[0] + x, lo[1] + y, lo[2] + z) ==
                           or_at(p, lo[0] + q[0], lo[1] + q[1], lo[2] + q[2]);
                }
        t->stored[axis] = same ? 1 : shape[axis];
        reduced *= t->stored[axis];
    }
    t->cost = 52 + 4 * reduced;
    if (reduced <= 64 || count <= p->threshold) return t;
    int axis = -1;
    for (int a = 0; a < 3; ++a)
        if (t->stored[a] > 1 && (axis < 0 || shape[a] > shape[axis])) axis = a;
    if (axis < 0) return t;
    int ls[3], rs[3], rl[3];
    for (int a = 0; a < 3; ++a) {
        ls[a] = rs[a] = shape[a];
        rl[a] = lo[a];
    }
    ls[axis] = shape[axis] / 2;
    rs[axis] -= ls[axis];
    rl[axis] += ls[axis];
    or_tree *l = or_build(p, lo, ls), *r = or_build(p, rl, rs);
    if (l && r && 52 + l->cost + r->cost < t->cost) {
        t->cost = 52 + l->cost + r->cost;
        t->left = l;
        t->right = r;
    } else {
        or_tree_free(l);
        or_tree_free(r);
    }
    return t;
}

typedef struct {
    or_node *nodes;
    int64_t n_nodes, cap_nodes;
    uint32_t *payload;
    int64_t n_payload, cap_payload;
} or_packed;

static int or_push_node(or_packed *o) {
    if (o->n_nodes == o->cap_nodes) {
        int64_t c = o->cap_nodes ? 2 * o->cap_nodes : 64;
        or_node *n = (or_node *)realloc(o->nodes, (size_t)c * sizeof(or_node));
        if (!n) return -1;
        o->nodes = n;
        o->cap_nodes = c;
    }
    memset(&o->nodes[o->n_nodes], 0, sizeof(or_node));
    return (int)(o->n_nodes++);
}

/* Depth-first, left before right; leaves append their reduced samples to the payload.
 * src/field_engine/adaptive_pack_native_v1/pack.cpp:43-55, adaptive_sample_blocks_v1.py:46-58. */
static int or_flatten(const or_packer *p, const or_tree *t, or_packed *o) {
    int idx = or_push_node(o);
    if (idx < 0) return -1;
    or_node node;
    memset(&node, 0, sizeof(node));
    for (int a = 0; a < 3; ++a) {
        node.lo[a] = t->lo[a];
        node.shape[a] = t->shape[a];
    }
    if (t->left) {
        node.offset = -1;
        int l = or_flatten(p, t->left, o);
        int r = or_flatten(p, t->right, o);
        if (l < 0 || r < 0) return -1;
        node.children[0] = l;
        node.children[1] = r;
    } else {
        node.offset = o->n_payload;
        node.children[0] = node.children[1] = -1;
        int64_t need = (int64_t)t->stored[0] * t->stored[1] * t->stored[2];
        if (o->n_payload + need > o->cap_payload) {
            int64_t c = o->cap_payload ? o->cap_payload : 1024;
            while (c < o->n_payload + need) c *= 2;
            uint32_t *np = (uint32_t *)realloc(o->payload, (size_t)c * 4);
            if (!np) return -1;
            o->payload = np;
            o->cap_payload = c;
        }
        for (int a = 0; a < 3; ++a) node.stored[a] = t->stored[a];
        for (int x = 0; x < t->stored[0]; ++x)
            for (int y = 0; y < t->stored[1]; ++y)
                for (int z = 0; z < t->stored[2]; ++z)
                    o->payload[o->n_payload++] = or_at(p, t->lo[0] + x, t->lo[1] + y, t->lo[2] + z);
    }
    o->nodes[idx] = node;
    return idx;
}

/* Same contract as the reference packer: 8 <= threshold <= 4096, axes 1..4096, <= 2^24 samples,
 * non-finite payload rejected.  Returns NULL on failure.  pack.cpp:57-69. */
void *or_pack(const float *data, const int32_t *shape, int threshold) {
    if (!data || !shape || threshold < 8 || threshold > 4096) return NULL;
    int64_t total = 1;
    for (int a = 0; a < 3; ++a) {
        if (shape[a] < 1 || shape[a] > 4096) return NULL;
        total *= shape[a];
    }
    if (total > 16777216) return NULL;
    const uint32_t *bits = (const uint32_t *)data;
    for (int64_t i = 0; i < total; ++i)
        if ((bits[i] & 0x7f800000u) == 0x7f800000u) return NULL;
    or_packer p = {bits, (int64_t)shape[1] * shape[2], shape[2], threshold};
    int lo[3] = {0, 0, 0};
    int sh[3] = {shape[0], shape[1], shape[2]};
    or_tree *root = or_build(&p, lo, sh);
    if (!root) return NULL;
    or_packed *o = (or_packed *)calloc(1, sizeof(or_packed));
    if (!o || or_flatten(&p, root, o) < 0) {
        or_tree_free(root);
        if (o) {
            free(o->nodes);
            free(o->payload);
            free(o);
        }
        return NULL;
    }
    or_tree_free(root);
    return o;
}

int64_t or_pack_nodes(const void *h) { return h ? ((const or_packed *)h)->n_nodes : 0; }
int64_t or_pack_samples(const void *h) { return h ? ((const or_packed *)h)->n_payload : 0; }
int or_pack_copy(const void *h, void *nodes, int64_t count, void *payload, int64_t samples) {
    const or_packed *o = (const or_packed *)h;
    if (!o || !nodes || !payload || count != o->n_nodes || samples != o->n_payload) return 1;
    memcpy(nodes, o->nodes, (size_t)count * sizeof(or_node));
    memcpy(payload, o->payload, (size_t)samples * 4);
    return 0;
}
void or_pack_free(void *h) {
    or_packed *o = (or_packed *)h;
    if (!o) return;
    free(o->nodes);
    free(o->payload);
    free(o);
}

/* ------------------------------------------------------------------------------------------------
 * Analytic primitives and CSG programs in float64
 * ---------------------------------------------------------------------------------------------- */

/* Primitive record: value = s * f(A x + t) - off, with f the canonical primitive centred on its
 * own origin.  Layout shared with the host compiler (field_b200.expr). */
typedef struct {
    int32_t type, flags;
    double p[12];
    double A[12]; /* rows of the 3x4 world->local map: A[0..3], A[4..7], A[8..11] */
    double s, off;
} or_prim;

typedef struct {
    int32_t op, arg;
    double k;
} or_insn;

enum { OP_PUSH = 0, OP_UNION = 1, OP_INTERSECT = 2, OP_SUBTRACT = 3, OP_OFFSET = 4 };
enum { P_SPHERE = 0, P_BOX, P_CYLINDER, P_CONE, P_HALFSPACE, P_FRUSTUM, P_CAPSULE, P_TORUS, P_CYL_INF,
       P_GRID, P_REVOLVE, P_BAR, P_POCKET, P_XBORE };

static double or_max(double a, double b) { return a > b ? a : b; }
static double or_min(double a, double b) { return a < b ? a : b; }
static double or_clamp01(double t) { return or_min(or_max(t, 0.0), 1.0); }

/* Canonical primitive SDFs.  Sphere, box, cylinder, cone, halfspace and rect_frustum restate
 * src/field_engine/ikarus_v1/expr.py:268-340 (and faltkarna_v1.py:91-99 for the box); capsule and
 * torus have no counterpart in the reference and follow the textbook closed forms (segment
 * distance minus radius; distance to the major circle minus the minor radius). */
/* Table-backed leaves keep the address of their float32 table in p[10] (raw bits). */
static const float *or_table(const double *p) {
    uint64_t bits;
    memcpy(&bits, &p[10], sizeof(bits));
    return (const float *)(uintptr_t)bits;
}

static double or_lerp(double a, double b, double t) { return a * (1.0 - t) + b * t; }

/* Gridfield leaf: src/field_engine/ikarus_v1/eval_warp.py:94-147 -- 1e6 outside the grid, else the
 * trilinear sample (lerps in x, then y, then z); occupancy tables read (iso - v) * pitch.
 * p = {ox, oy, oz, pitch, iso, is_sdf, nx, ny, nz, -, table}. */
static double or_grid(const double *p, double x, double y, double z) {
    const int nx = (int)p[6], ny = (int)p[7], nz = (int)p[8];
    const double pitch = p[3];
    const double fx = (x - p[0]) / pitch, fy = (y - p[1]) / pitch, fz = (z - p[2]) / pitch;
    if (!(fx >= 0.0 && fy >= 0.0 && fz >= 0.0 && fx <= nx - 1 && fy <= ny - 1 && fz <= nz - 1)) return 1.0e6;
    const int ix = (int)floor(fx), iy = (int)floor(fy), iz = (int)floor(fz);
    const int ix1 = ix + 1 < nx ? ix + 1 : nx - 1, iy1 = iy + 1 < ny ? iy + 1 : ny - 1, iz1 = iz + 1 < nz ? iz + 1 : nz - 1;
    const double tx = fx - ix, ty = fy - iy, tz = fz - iz;
    const float *g = or_table(p);
#define AT(i, j, k) ((double)g[((int64_t)(i) * ny + (j)) * nz + (k)])
    const double c00 = or_lerp(AT(ix, iy, iz), AT(ix1, iy, iz), tx), c10 = or_lerp(AT(ix, iy1, iz), AT(ix1, iy1, iz), tx);
    const double c01 = or_lerp(AT(ix, iy, iz1), AT(ix1, iy, iz1), tx), c11 = or_lerp(AT(ix, iy1, iz1), AT(ix1, iy1, iz1), tx);
#undef AT
    const double val = or_lerp(or_lerp(c00, c10, ty), or_lerp(c01, c11, ty), tz);
    return p[5] != 0.0 ? val : (p[4] - val) * pitch;
}

/* Revolved (r, z) table: src/field_engine/tillverkningsfalt_v1_kernel.py:265-277 -- r the distance
 * from the z axis, cell indices truncated then clamped to the table, weights clamped to [0, 1].
 * p = {r0, z0, pitch, nr, nz, -, ..., table}. */
static double or_revolve(const double *p, double x, double y, double z) {
    const int nr = (int)p[3], nz = (int)p[4];
    const double r = sqrt(x * x + y * y);
    const double fr = (r - p[0]) / p[2], fz = (z - p[1]) / p[2];
    const double cr = fr < -1e9 ? -1e9 : (fr > 1e9 ? 1e9 : fr), cz = fz < -1e9 ? -1e9 : (fz > 1e9 ? 1e9 : fz);
    int ir = (int)cr, iz = (int)cz;
    ir = ir < 0 ? 0 : (ir > nr - 2 ? nr - 2 : ir);
    iz = iz < 0 ? 0 : (iz > nz - 2 ? nz - 2 : iz);
    const double tr = or_clamp01(fr - ir), tz = or_clamp01(fz - iz);
    const float *g = or_table(p);
    const double v00 = g[(int64_t)ir * nz + iz], v01 = g[(int64_t)ir * nz + iz + 1];
    const double v10 = g[(int64_t)(ir + 1) * nz + iz], v11 = g[(int64_t)(ir + 1) * nz + iz + 1];
    return v00 * (1.0 - tr) * (1.0 - tz) + v01 * (1.0 - tr) * tz + v10 * tr * (1.0 - tz) + v11 * tr * tz;
}

static double or_prim_local(const or_prim *P, double x, double y, double z) {
    const double *p = P->p;
    switch (P->type) {
    case P_SPHERE:
        return sqrt(x * x + y * y + z * z) - p[0];
    case P_BOX: {
        double qx = fabs(x) - p[0], qy = fabs(y) - p[1], qz = fabs(z) - p[2];
        double ox = or_max(qx, 0.0), oy = or_max(qy, 0.0), oz = or_max(qz, 0.0);
        double outside = sqrt(ox * ox + oy * oy + oz * oz);
        double inside = or_min(or_max(qx, or_max(qy, qz)), 0.0);
        return outside + inside;
    }
    case P_CYLINDER: {
        double rad = sqrt(x * x + y * y);
        double qx = rad - p[0], qy = fabs(z) - p[1];
        double ox = or_max(qx, 0.0), oy = or_max(qy, 0.0);
        return sqrt(ox * ox + oy * oy) + or_min(or_max(qx, qy), 0.0);
    }
    case P_CONE: {
        double rad = sqrt(x * x + y * y), h = p[2];
        double t = or_clamp01((z + h / 2.0) / h);
        double r_at = p[0] + (p[1] - p[0]) * t;
        double qy = fabs(z) - h / 2.0, qx = rad - r_at;
        double ox = or_max(qx, 0.0), oy = or_max(qy, 0.0);
        return sqrt(ox * ox + oy * oy) + or_min(or_max(qx, qy), 0.0);
    }
    case P_HALFSPACE:
        return x * p[0] + y * p[1] + z * p[2];
    case P_FRUSTUM: {
        /* centred on (cx0, cy0, z0): p = {z1, hx0, hy0, hx1, hy1, cx1, cy1} with z0 = cx0 = cy0 = 0 */
        double z1 = p[0], hx0 = p[1], hy0 = p[2], hx1 = p[3], hy1 = p[4], cx1 = p[5], cy1 = p[6];
        double kx = (hx1 - hx0) / z1, ky = (hy1 - hy0) / z1, kcx = cx1 / z1, kcy = cy1 / z1;
        double d_zlo = -z, d_zhi = z - z1;
        double a1 = -(kx + kcx), n1 = sqrt(1.0 + a1 * a1);
        double a2 = -(kx - kcx), n2 = sqrt(1.0 + a2 * a2);
        double a3 = -(ky + kcy), n3 = sqrt(1.0 + a3 * a3);
        double a4 = -(ky - kcy), n4 = sqrt(1.0 + a4 * a4);
        double d_xhi = (x + a1 * z - hx0) / n1;
        double d_xlo = (-x + a2 * z - hx0) / n2;
        double d_yhi = (y + a3 * z - hy0) / n3;
        double d_ylo = (-y + a4 * z - hy0) / n4;
        return or_max(or_max(or_max(d_zlo, d_zhi), or_max(d_xhi, d_xlo)), or_max(d_yhi, d_ylo));
    }
    case P_CAPSULE: {
        double bx = p[0], by = p[1], bz = p[2];
        double bb = bx * bx + by * by + bz * bz;
        double h = bb > 0.0 ? or_clamp01((x * bx + y * by + z * bz) / bb) : 0.0;
        double dx = x - bx * h, dy = y - by * h, dz = z - bz * h;
        return sqrt(dx * dx + dy * dy + dz * dz) - p[3];
    }
    case P_TORUS: {
        double qx = sqrt(x * x + y * y) - p[0];
        return sqrt(qx * qx + z * z) - p[1];
    }
    case P_CYL_INF: /* unbounded z cylinder, src/field_engine/faltkarna_v1.py:102-104 */
        return sqrt(x * x + y * y) - p[0];
    case P_GRID:
        return or_grid(p, x, y, z);
    case P_REVOLVE:
        return or_revolve(p, x, y, z);
    case P_BAR: /* round bar (the blank), src/field_engine/tillverkningsfalt_v1_kernel.py:262-263 */
        return or_max(sqrt(x * x + y * y) - p[0], or_max(p[1] - z, z - p[2]));
    case P_POCKET: { /* rounded-box pocket under an arched roof, tillverkningsfalt_v1_kernel.py:281-291 */
        double qx = fabs(x) - (p[0] - p[2]), qy = fabs(y) - (p[1] - p[2]);
        double ox = or_max(qx, 0.0), oy = or_max(qy, 0.0);
        double dxy = sqrt(ox * ox + oy * oy) + or_min(or_max(qx, qy), 0.0) - p[2];
        double roof = p[4] + sqrt(or_max(p[3] * p[3] - x * x, 0.0));
        return or_max(dxy, z - roof);
    }
    case P_XBORE: { /* cross bore along x clipped to |x| <= half, tillverkningsfalt_v1_kernel.py:294-297 */
        double dz = z - p[1];
        return or_max(sqrt(y * y + dz * dz) - p[0], fabs(x) - p[2]);
    }
    default:
        return NAN;
    }
}

double or_prim_eval(const or_prim *P, double x, double y, double z) {
    const double *A = P->A;
    double lx = A[0] * x + A[1] * y + A[2] * z + A[3];
    double ly = A[4] * x + A[5] * y + A[6] * z + A[7];
    double lz = A[8] * x + A[9] * y + A[10] * z + A[11];
    return P->s * or_prim_local(P, lx, ly, lz) - P->off;
}

/* Hard and polynomial-smooth booleans: union = min, intersect = max, subtract = max(a, -b);
 * smooth forms subtract/add h*h*k/4 with h = max(k - |a -+ b|, 0)/k.
 * src/field_engine/ikarus_v1/expr.py:364-384. */
static double or_combine(int op, double a, double b, double k) {
    if (op == OP_UNION) {
        if (k <= 0.0) return or_min(a, b);
        double h = or_max(k - fabs(a - b), 0.0) / k;
        return or_min(a, b) - h * h * k * 0.25;
    }
    if (op == OP_INTERSECT) {
        if (k <= 0.0) return or_max(a, b);
        double h = or_max(k - fabs(a - b), 0.0) / k;
        return or_max(a, b) + h * h * k * 0.25;
    }
    if (k <= 0.0) return or_max(a, -b);
    double h = or_max(k - fabs(a + b), 0.0) / k;
    return or_max(a, -b) + h * h * k * 0.25;
}

#define OR_STACK 64

/* Postfix program evaluation at one point; returns NAN on a malformed program. */
double or_program_eval(const or_prim *prims, int32_t nprim, const or_insn *prog, int32_t ninsn, double x,
                       double y, double z) {
    double st[OR_STACK];
    int sp = 0;
    for (int i = 0; i < ninsn; ++i) {
        const or_insn *I = &prog[i];
        if (I->op == OP_PUSH) {
            if (sp >= OR_STACK || I->arg < 0 || I->arg >= nprim) return NAN;
            st[sp++] = or_prim_eval(&prims[I->arg], x, y, z);
        } else if (I->op == OP_OFFSET) {
            if (sp < 1) return NAN;
            st[sp - 1] = st[sp - 1] - I->k;
        } else {
            if (sp < 2) return NAN;
            double b = st[--sp];
            st[sp - 1] = or_combine(I->op, st[sp - 1], b, I->k);
        }
    }
    return sp == 1 ? st[0] : NAN;
}

int or_eval_points(const or_prim *prims, int32_t nprim, const or_insn *prog, int32_t ninsn, const double *pts,
                   int64_t n, double *out) {
    if (!prims || !prog || !pts || !out || n < 0) return OR_INVALID;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        out[i] = or_program_eval(prims, nprim, prog, ninsn, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    return OR_OK;
}

/* Analytic classification in float64.  Block (bi, bj, bk) has corners at voxel indices
 * (bi*B + cB, ...) for c in {0, 1}, at world position x0 + index * pitch; positive iff v >= 0;
 * kind = 0 when both signs occur or min|v| <= margin (the float32 margin widened to float64),
 * else -1 / +1.  src/field_engine/faltkarna_v1.py:129-164 (k_classify_testfalt) with the field
 * replaced by the program; block id lin = (bi*n_by + bj)*n_bz + bk (faltkarna_v1.py:77-82). */
int or_classify_program(const or_prim *prims, int32_t nprim, const or_insn *prog, int32_t ninsn, double x0,
                        double y0, double z0, double pitch, int nx, int ny, int nz, int block, float margin,
                        int32_t *kind, double *cma) {
    if (!prims || !prog || !kind || nx < 1 || ny < 1 || nz < 1 || block < 1) return OR_INVALID;
    int64_t nbx = (nx + block - 1) / block, nby = (ny + block - 1) / block, nbz = (nz + block - 1) / block;
    int64_t nb = nbx * nby * nbz;
    double m = (double)margin;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < nb; ++t) {
        int64_t bk = t % nbz, bj = (t / nbz) % nby, bi = t / (nbz * nby);
        double mn = 1.0e30;
        int pos = 0, neg = 0;
        for (int c = 0; c < 8; ++c) {
            int64_t ix = bi * block + (c & 1) * block;
            int64_t iy = bj * block + ((c >> 1) & 1) * block;
            int64_t iz = bk * block + ((c >> 2) & 1) * block;
            double v = or_program_eval(prims, nprim, prog, ninsn, x0 + (double)ix * pitch,
                                       y0 + (double)iy * pitch, z0 + (double)iz * pitch);
            double a = fabs(v);
            if (a < mn) mn = a;
            if (v >= 0.0) pos = 1; else neg = 1;
        }
        if (cma) cma[t] = mn;
        kind[t] = (pos && neg) ? 0 : ((mn <= m) ? 0 : (neg ? -1 : 1));
    }
    return OR_OK;
}

/* The same classification for a list of block ids only (a bounded sample for CPU timing). */
int or_classify_blocks(const or_prim *prims, int32_t nprim, const or_insn *prog, int32_t ninsn, double x0,
                       double y0, double z0, double pitch, int nx, int ny, int nz, int block, float margin,
                       const int64_t *blocks, int64_t n, int32_t *kind, double *cma) {
    if (!prims || !prog || !blocks || !kind || nx < 1 || ny < 1 || nz < 1 || block < 1 || n < 0) return OR_INVALID;
    int64_t nby = (ny + block - 1) / block, nbz = (nz + block - 1) / block;
    double m = (double)margin;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t s = 0; s < n; ++s) {
        int64_t t = blocks[s];
        int64_t bk = t % nbz, bj = (t / nbz) % nby, bi = t / (nbz * nby);
        double mn = 1.0e30;
        int pos = 0, neg = 0;
        for (int c = 0; c < 8; ++c) {
            int64_t ix = bi * block + (c & 1) * block;
            int64_t iy = bj * block + ((c >> 1) & 1) * block;
            int64_t iz = bk * block + ((c >> 2) & 1) * block;
            double v = or_program_eval(prims, nprim, prog, ninsn, x0 + (double)ix * pitch,
                                       y0 + (double)iy * pitch, z0 + (double)iz * pitch);
            double a = fabs(v);
            if (a < mn) mn = a;
            if (v >= 0.0) pos = 1; else neg = 1;
        }
        if (cma) cma[s] = mn;
        kind[s] = (pos && neg) ? 0 : ((mn <= m) ? 0 : (neg ? -1 : 1));
    }
    return OR_OK;
}

/* Float64 values of the leaf voxels of the given active blocks, tile order (li, lj, lk), voxel
 * (bi*B + li, ...) at x0 + index * pitch.  src/field_engine/faltkarna_v1.py:167-190. */
int or_tiles_program(const or_prim *prims, int32_t nprim, const or_insn *prog, int32_t ninsn, double x0,
                     double y0, double z0, double pitch, int nx, int ny, int nz, int block, const int32_t *active,
                     int64_t nact, double *out) {
    if (!prims || !prog || nx < 1 || ny < 1 || nz < 1 || block < 1 || nact < 0 || (nact && (!active || !out)))
        return OR_INVALID;
    int64_t nby = (ny + block - 1) / block, nbz = (nz + block - 1) / block, b3 = (int64_t)block * block * block;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t a = 0; a < nact; ++a) {
        int64_t lin = active[a];
        int64_t bk = lin % nbz, bi = lin / (nbz * nby), bj = (lin / nbz) % nby;
        double *o = out + a * b3;
        for (int li = 0; li < block; ++li)
            for (int lj = 0; lj < block; ++lj)
                for (int lk = 0; lk < block; ++lk)
                    *o++ = or_program_eval(prims, nprim, prog, ninsn, x0 + (double)(bi * block + li) * pitch,
                                           y0 + (double)(bj * block + lj) * pitch,
                                           z0 + (double)(bk * block + lk) * pitch);
    }
    return OR_OK;
}

int or_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
