// Primitive records and their evaluation on the device: float32 (bulk, block-localised) and
// float64 (guard-band recheck, general programs).
//
// A primitive's world value is  s * f(A x + t) - off  with f the canonical primitive centred on
// its own origin (the host compiler folds transforms, scales, axis projections and leaf offsets
// into A, t, s, off).  Canonical formulas: sphere, box, cylinder, cone, halfspace and rect_frustum
// follow src/field_engine/ikarus_v1/expr.py:268-340 (box also faltkarna_v1.py:91-99), the
// unbounded z cylinder faltkarna_v1.py:102-104; capsule and torus are the textbook closed forms.
// Table-backed kinds read a float32 table whose address the host writes into the record (p[10] of
// the float64 record as raw bits; p[10] / p[11] of the float32 mirror as its two 32-bit halves):
// the gridfield leaf's trilinear sample (src/field_engine/ikarus_v1/eval_warp.py:94-147) and the
// revolved (r, z) table of the machining scene (tillverkningsfalt_v1_kernel.py:265-277); that scene's
// round bar, arched rounded-box pocket and x-clipped cross bore follow its :262-300.
#pragma once
#include <cstdint>

enum : int32_t {
    P_SPHERE = 0, P_BOX, P_CYLINDER, P_CONE, P_HALFSPACE, P_FRUSTUM, P_CAPSULE, P_TORUS, P_CYL_INF,
    // table-backed and machining-scene kinds (never culled where no Lipschitz bound holds)
    P_GRID, P_REVOLVE, P_BAR, P_POCKET, P_XBORE
};
enum : int32_t { OP_PUSH = 0, OP_UNION, OP_INTERSECT, OP_SUBTRACT, OP_OFFSET };
enum : int32_t { CH_SET = 0, CH_SETNEG, CH_UNION, CH_INTERSECT, CH_SUBTRACT, CH_OFFSET };

// Host-compiled record (216 bytes, float64), the C-ABI layout of fb_prim in include/field_b200.h.
struct FbPrim {
    int32_t type, flags;
    double p[12];
    double A[12];  // rows of the 3x4 world -> canonical map
    double s, off;
};
static_assert(sizeof(FbPrim) == 216, "fb_prim layout");

// One program / chain instruction (16 bytes), fb_insn in include/field_b200.h.
struct FbInsn {
    int32_t op, arg;
    double k;
};
static_assert(sizeof(FbInsn) == 16, "fb_insn layout");

// float32 mirror used for interval culling in world coordinates (128 bytes).
struct __align__(16) PrimF {
    int32_t type, ident;
    float s, off, lip;
    float ball, ball_k, pad;  // bounding ball present (1) and its value scale; centre, radius in p[8..11]
    float A[12];
    float p[12];
};

// Block-localised float32 record: q = L + A_lin * d, d the offset from the block origin; L[3] holds
// a kind's per-block float64 constant rounded once (the sphere's |L|^2 - r^2); diff selects the
// sphere's difference form for this block.
struct __align__(16) LocalPrim {
    int32_t type, op, ident, diff;
    float k, s, off;
    int32_t mode;  // 8^3 leaf tiles: 0 min, 1 max, 2 set (hard combines, sign folded into s/off), 3 other
    float L[4];
    float A[12];   // A_lin rows (9 used)
    float p[12];
};

// ------------------------------------------------------------------------------------ float32
__device__ __forceinline__ float sel_min(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float sel_max(float a, float b) { return a > b ? a : b; }

// Square root of a sum of squares (x >= 0 or NaN) for the grouped float32 evaluations: one Newton
// step on s^2 = x from the hardware's approximate reciprocal square root y, s = x*y, with the
// residual x - s^2 formed exactly by one FMA (Markstein's correction, "IA-64 and Elementary
// Functions", 2000): s + (y/2)(x - s^2).  Branch-free; correctly rounded on every input of [1, 4)
// (tests/test_prims_gpu.py compares it with sqrtf across binades), so the tiles equal those of
// sqrtf.  Inputs below 1e-30 (subnormal squares of offsets under 1e-15) give their root to within
// 1e-15; x = 0 gives 0 and NaN stays NaN.
__device__ __forceinline__ float sqrt_sum(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(fmaxf(x, 1e-30f)));
    const float s = x * y;
    return fmaf(0.5f * y, fmaf(-s, s, x), s);
}

// float32 lerp with the product form a*(1-t) + b*t, each operation rounded once.
__device__ __forceinline__ float lerp_f(float a, float b, float t) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.f, t)), __fmul_rn(b, t));
}

__device__ __forceinline__ const float* table_of(const float* __restrict__ p) {
    return reinterpret_cast<const float*>((uint64_t)__float_as_uint(p[10]) | ((uint64_t)__float_as_uint(p[11]) << 32));
}

// Gridfield leaf, p = {ox, oy, oz, pitch, iso, is_sdf, nx, ny, nz, -, table}: 1e6 outside the grid
// (NaN coordinates included), else the trilinear sample; occupancy tables read (iso - v) * pitch.
static __device__ __noinline__ float grid_sample_f(const float* __restrict__ p, float x, float y, float z) {
    const int nx = (int)p[6], ny = (int)p[7], nz = (int)p[8];
    const float pitch = p[3];
    const float fx = __fdiv_rn(__fsub_rn(x, p[0]), pitch);
    const float fy = __fdiv_rn(__fsub_rn(y, p[1]), pitch);
    const float fz = __fdiv_rn(__fsub_rn(z, p[2]), pitch);
    if (!(fx >= 0.f && fy >= 0.f && fz >= 0.f && fx <= (float)(nx - 1) && fy <= (float)(ny - 1) &&
          fz <= (float)(nz - 1)))
        return 1.0e6f;
    const int ix = (int)floorf(fx), iy = (int)floorf(fy), iz = (int)floorf(fz);
    const int ix1 = min(ix + 1, nx - 1), iy1 = min(iy + 1, ny - 1), iz1 = min(iz + 1, nz - 1);
    const float tx = __fsub_rn(fx, (float)ix), ty = __fsub_rn(fy, (float)iy), tz = __fsub_rn(fz, (float)iz);
    const float* g = table_of(p);
    auto at = [&](int i, int j, int k) { return g[((int64_t)i * ny + j) * nz + k]; };
    const float c00 = lerp_f(at(ix, iy, iz), at(ix1, iy, iz), tx), c10 = lerp_f(at(ix, iy1, iz), at(ix1, iy1, iz), tx);
    const float c01 = lerp_f(at(ix, iy, iz1), at(ix1, iy, iz1), tx), c11 = lerp_f(at(ix, iy1, iz1), at(ix1, iy1, iz1), tx);
    const float val = lerp_f(lerp_f(c00, c10, ty), lerp_f(c01, c11, ty), tz);
    return p[5] != 0.f ? val : __fmul_rn(__fsub_rn(p[4], val), pitch);
}

// True where (x, y, z) lies within a thousandth of a cell of a sampled grid's boundary: there the
// value jumps between the table and the outside constant, and a float32 inside test may decide
// otherwise than the float64 one (the coordinate itself carries float32 rounding), so the caller
// takes that sample's decisions in float64.
static __device__ __noinline__ bool grid_edge_f(const float* __restrict__ p, float x, float y, float z) {
    const float n[3] = {p[6] - 1.f, p[7] - 1.f, p[8] - 1.f};
    const float f[3] = {(x - p[0]) / p[3], (y - p[1]) / p[3], (z - p[2]) / p[3]};
    constexpr float tol = 1e-3f;
    bool within = true, edge = false;
    for (int a = 0; a < 3; ++a) {
        within &= f[a] >= -tol && f[a] <= n[a] + tol;
        edge |= fabsf(f[a]) < tol || fabsf(f[a] - n[a]) < tol;
    }
    return within && edge;
}

// Revolved (r, z) table, p = {r0, z0, pitch, nr, nz, -, ..., table}: bilinear at (r, z), r the
// distance from the z axis, cell indices truncated and clamped to the table, weights clamped to [0, 1].
static __device__ __noinline__ float revolve_sample_f(const float* __restrict__ p, float x, float y, float z) {
    const int nr = (int)p[3], nz = (int)p[4];
    const float r = sqrtf(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)));
    const float fr = __fdiv_rn(__fsub_rn(r, p[0]), p[2]), fz = __fdiv_rn(__fsub_rn(z, p[1]), p[2]);
    const float cr = fminf(fmaxf(fr, -1.0e9f), 1.0e9f), cz = fminf(fmaxf(fz, -1.0e9f), 1.0e9f);  // int range
    const int ir = min(max((int)cr, 0), nr - 2), iz = min(max((int)cz, 0), nz - 2);
    const float tr = fminf(fmaxf(__fsub_rn(fr, (float)ir), 0.f), 1.f), tz = fminf(fmaxf(__fsub_rn(fz, (float)iz), 0.f), 1.f);
    const float* g = table_of(p);
    const float v00 = g[(int64_t)ir * nz + iz], v01 = g[(int64_t)ir * nz + iz + 1];
    const float v10 = g[(int64_t)(ir + 1) * nz + iz], v11 = g[(int64_t)(ir + 1) * nz + iz + 1];
    const float ur = __fsub_rn(1.f, tr), uz = __fsub_rn(1.f, tz);
    float v = __fmul_rn(__fmul_rn(v00, ur), uz);
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(v01, ur), tz));
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(v10, tr), uz));
    return __fadd_rn(v, __fmul_rn(__fmul_rn(v11, tr), tz));
}

__device__ __forceinline__ float canon_f(int type, const float* __restrict__ p, float x, float y, float z) {
    switch (type) {
    case P_SPHERE:
        return sqrtf(fmaf(x, x, fmaf(y, y, z * z))) - p[0];
    case P_BOX: {
        const float qx = fabsf(x) - p[0], qy = fabsf(y) - p[1], qz = fabsf(z) - p[2];
        const float ox = fmaxf(qx, 0.f), oy = fmaxf(qy, 0.f), oz = fmaxf(qz, 0.f);
        return sqrtf(fmaf(ox, ox, fmaf(oy, oy, oz * oz))) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.f);
    }
    case P_CYLINDER: {
        const float qx = sqrtf(fmaf(x, x, y * y)) - p[0], qy = fabsf(z) - p[1];
        const float ox = fmaxf(qx, 0.f), oy = fmaxf(qy, 0.f);
        return sqrtf(fmaf(ox, ox, oy * oy)) + fminf(fmaxf(qx, qy), 0.f);
    }
    case P_CONE: {  // p = {r1, r2, h, 1/h}
        const float t = fminf(fmaxf((z + 0.5f * p[2]) * p[3], 0.f), 1.f);
        const float qx = sqrtf(fmaf(x, x, y * y)) - fmaf(p[1] - p[0], t, p[0]);
        const float qy = fabsf(z) - 0.5f * p[2];
        const float ox = fmaxf(qx, 0.f), oy = fmaxf(qy, 0.f);
        return sqrtf(fmaf(ox, ox, oy * oy)) + fminf(fmaxf(qx, qy), 0.f);
    }
    case P_HALFSPACE:
        return fmaf(x, p[0], fmaf(y, p[1], z * p[2]));
    case P_FRUSTUM: {  // p = {z1, hx0, hy0, a1, a2, a3, a4, 1/n1, 1/n2, 1/n3, 1/n4}
        float d = fmaxf(-z, z - p[0]);
        d = fmaxf(d, (fmaf(p[3], z, x) - p[1]) * p[7]);
        d = fmaxf(d, (fmaf(p[4], z, -x) - p[1]) * p[8]);
        d = fmaxf(d, (fmaf(p[5], z, y) - p[2]) * p[9]);
        d = fmaxf(d, (fmaf(p[6], z, -y) - p[2]) * p[10]);
        return d;
    }
    case P_CAPSULE: {  // p = {bx, by, bz, r, 1/|b|^2 (0 if degenerate), h_lo, h_hi}
        // segment h*b for h in [h_lo, h_hi]: [0, 1] in the canonical frame, shifted when the frame
        // is re-anchored on the segment (block-local records)
        const float h = fminf(fmaxf(fmaf(x, p[0], fmaf(y, p[1], z * p[2])) * p[4], p[5]), p[6]);
        const float dx = fmaf(-p[0], h, x), dy = fmaf(-p[1], h, y), dz = fmaf(-p[2], h, z);
        return sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz))) - p[3];
    }
    case P_TORUS: {
        const float qx = sqrtf(fmaf(x, x, y * y)) - p[0];
        return sqrtf(fmaf(qx, qx, z * z)) - p[1];
    }
    case P_CYL_INF:
        return sqrtf(fmaf(x, x, y * y)) - p[0];
    case P_GRID:
        return grid_sample_f(p, x, y, z);
    case P_REVOLVE:
        return revolve_sample_f(p, x, y, z);
    case P_BAR: {  // p = {R, z_lo, z_hi}: max(r - R, max(z_lo - z, z - z_hi))
        const float r = sqrtf(fmaf(x, x, y * y));
        return fmaxf(r - p[0], fmaxf(p[1] - z, z - p[2]));
    }
    case P_POCKET: {  // p = {half_x, half_y, edge_r, arch_r, arch_cz}
        const float qx = fabsf(x) - (p[0] - p[2]), qy = fabsf(y) - (p[1] - p[2]);
        const float ox = fmaxf(qx, 0.f), oy = fmaxf(qy, 0.f);
        const float dxy = sqrtf(fmaf(ox, ox, oy * oy)) + fminf(fmaxf(qx, qy), 0.f) - p[2];
        const float roof = p[4] + sqrtf(fmaxf(fmaf(-x, x, p[3] * p[3]), 0.f));
        return fmaxf(dxy, z - roof);
    }
    case P_XBORE: {  // p = {radius, axis_z, half_length}
        const float dz = z - p[1];
        return fmaxf(sqrtf(fmaf(y, y, dz * dz)) - p[0], fabsf(x) - p[2]);
    }
    default:
        return __int_as_float(0x7fc00000);
    }
}

// World-coordinate float32 value (culling intervals only).
__device__ __forceinline__ float primf_world(const PrimF& P, float x, float y, float z) {
    const float lx = fmaf(P.A[0], x, fmaf(P.A[1], y, fmaf(P.A[2], z, P.A[3])));
    const float ly = fmaf(P.A[4], x, fmaf(P.A[5], y, fmaf(P.A[6], z, P.A[7])));
    const float lz = fmaf(P.A[8], x, fmaf(P.A[9], y, fmaf(P.A[10], z, P.A[11])));
    return fmaf(P.s, canon_f(P.type, P.p, lx, ly, lz), -P.off);
}

// Block-localised float32 value at offset (dx, dy, dz) from the block origin.
__device__ __forceinline__ float local_eval(const LocalPrim& P, float dx, float dy, float dz) {
    float x, y, z;
    if (P.ident) {
        x = P.L[0] + dx;
        y = P.L[1] + dy;
        z = P.L[2] + dz;
    } else {
        x = fmaf(P.A[0], dx, fmaf(P.A[1], dy, fmaf(P.A[2], dz, P.L[0])));
        y = fmaf(P.A[3], dx, fmaf(P.A[4], dy, fmaf(P.A[5], dz, P.L[1])));
        z = fmaf(P.A[6], dx, fmaf(P.A[7], dy, fmaf(P.A[8], dz, P.L[2])));
    }
    return fmaf(P.s, canon_f(P.type, P.p, x, y, z), -P.off);
}

// Hard / polynomial-smooth booleans in float32; on equality the second operand wins, as in NumPy.
__device__ __forceinline__ float combine_f(int op, float a, float b, float k) {
    if (op == CH_UNION) {
        const float m = sel_min(a, b);
        if (k <= 0.f) return m;
        const float h = fmaxf(k - fabsf(a - b), 0.f) / k;
        return m - h * h * k * 0.25f;
    }
    if (op == CH_INTERSECT) {
        const float m = sel_max(a, b);
        if (k <= 0.f) return m;
        const float h = fmaxf(k - fabsf(a - b), 0.f) / k;
        return m + h * h * k * 0.25f;
    }
    const float m = sel_max(a, -b);
    if (k <= 0.f) return m;
    const float h = fmaxf(k - fabsf(a + b), 0.f) / k;
    return m + h * h * k * 0.25f;
}

// Apply one chain element (effective op) with primitive value v to the accumulator.
__device__ __forceinline__ float chain_apply(int op, float acc, float v, float k) {
    switch (op) {
    case CH_SET: return v;
    case CH_SETNEG: return -v;
    case CH_OFFSET: return acc - k;
    default: return combine_f(op, acc, v, k);
    }
}

// Block-local float32 record of one primitive: L = A * origin + t in float64, rounded once.
// A capsule's frame is re-anchored at the projection h0 * b of the block origin onto its segment
// (float64, before rounding): its local coordinates then stay near the block's own size instead of
// growing with the distance along the segment (a milling sweep is up to ~1.7 length units long, where
// one float32 ulp is ~1e-7), and the segment becomes [-h0, 1 - h0] * b.  The clamp bound that can be
// active inside the block is the one near zero, which float32 holds to a relative 6e-8.
//
// A sphere takes the difference form (|L|^2 - r^2 + e.(2L + e)) / (|q| + r) when its radius exceeds
// twice the block's extent in its frame, else the direct |q| - r.  A torus whose ring radius R
// does takes the ring frame: rotated about its axis so the block origin lies on +x, x measured from
// the ring (u = x - R, w = y), where rho - R = u + w^2 / (rho + R + u) -- u carries the rounding of a
// short offset instead of a coordinate of size R, and the quotient is a correction of a few
// pitches.  extent 0 (callers that evaluate through local_eval) keeps the canonical forms, and the
// ring frame needs `ring` (leaf kernels built with its path).  Their float32 errors: about
// u (|d| + 6 |e|) for the difference form (d = |L| - r, independent of r) and u (|L| + 2 |q|) ~ 3 u r for
// the direct one (u = 2^-24): large spheres against small blocks favour the first, small spheres
// against large blocks the second.  extent: the largest offset the block's evaluation uses.
__device__ __forceinline__ void localise(const FbPrim& D, const PrimF& F, double ox, double oy, double oz, int op,
                                         float k, LocalPrim& out, float extent = 0.f, bool ring = false) {
    out.type = F.type;
    out.op = op;
    out.ident = F.ident;
    out.k = k;
    out.s = F.s;
    out.off = F.off;
    const double* A = D.A;
    double lx = fma(A[0], ox, fma(A[1], oy, fma(A[2], oz, A[3])));
    double ly = fma(A[4], ox, fma(A[5], oy, fma(A[6], oz, A[7])));
    double lz = fma(A[8], ox, fma(A[9], oy, fma(A[10], oz, A[11])));
#pragma unroll
    for (int j = 0; j < 12; ++j) out.p[j] = F.p[j];
    if (F.type == P_CAPSULE) {
        const double bx = D.p[0], by = D.p[1], bz = D.p[2];
        // any anchor on the segment serves (the bounds below are formed from the same h0), so the
        // float32 1/|b|^2 of the mirror stands in for a float64 division
        const double inv = (double)F.p[4];
        const double h0 = inv > 0.0 ? fmin(fmax(fma(lx, bx, fma(ly, by, lz * bz)) * inv, 0.0), 1.0) : 0.0;
        lx = fma(-bx, h0, lx);
        ly = fma(-by, h0, ly);
        lz = fma(-bz, h0, lz);
        out.p[5] = (float)(-h0);
        out.p[6] = (float)(1.0 - h0);
    }
    out.L[0] = (float)lx;
    out.L[1] = (float)ly;
    out.L[2] = (float)lz;
    // sphere: |L|^2 - r^2 in float64, the constant term of the difference form of |q| - r
    out.L[3] = F.type == P_SPHERE ? (float)(fma(lx, lx, fma(ly, ly, lz * lz)) - D.p[0] * D.p[0]) : 0.f;
    out.diff = 0;
    if (F.type == P_SPHERE || (ring && F.type == P_TORUS)) {
        // the extent in the primitive's frame: the linear part's root-mean-square stretch (the
        // Frobenius norm over sqrt 3; exact for a rotation or permutation times a uniform scale)
        const double a2 = (A[0] * A[0] + A[1] * A[1] + A[2] * A[2] + A[4] * A[4] + A[5] * A[5] + A[6] * A[6] +
                           A[8] * A[8] + A[9] * A[9] + A[10] * A[10]) / 3.0;
        // extent 0: the caller evaluates through local_eval (canonical forms only).  A torus's direct
        // form is within 1e-5 pitch below four extents of ring radius (its tube's norm then bounds the
        // error of either form), and its ring frame runs out of line
        const double k = F.type == P_TORUS ? 4.0 : 2.0;
        out.diff = extent > 0.f && D.p[0] > k * (double)extent * (F.ident ? 1.0 : sqrt(a2)) ? 1 : 0;
    }
    out.A[0] = F.A[0]; out.A[1] = F.A[1]; out.A[2] = F.A[2];
    out.A[3] = F.A[4]; out.A[4] = F.A[5]; out.A[5] = F.A[6];
    out.A[6] = F.A[8]; out.A[7] = F.A[9]; out.A[8] = F.A[10];
    if (ring && F.type == P_TORUS && out.diff) {
        // ring frame: rotate about the torus axis so the block origin lies on +x, and measure x from
        // the ring (the torus is symmetric under the rotation); only the offsets go through the
        // rotation, whose float32 rounding then scales them by ~1 + 2^-24 at most
        const double n2 = fma(lx, lx, ly * ly);
        const double inv = n2 > 0.0 ? rsqrt(n2) : 0.0;  // any rotation serves: only n must be accurate
        const double n = n2 * inv;
        const double cs = n2 > 0.0 ? lx * inv : 1.0, sn = n2 > 0.0 ? ly * inv : 0.0;
        out.L[0] = (float)(n - D.p[0]);
        out.L[1] = 0.f;
        out.L[3] = 0.f;
        for (int j = 0; j < 3; ++j) {
            const double r0 = A[j], r1 = A[4 + j];
            out.A[j] = (float)fma(cs, r0, sn * r1);
            out.A[3 + j] = (float)fma(-sn, r0, cs * r1);
        }
        out.ident = 0;
    }
}

// ------------------------------------------------------------------------------------ float64
// Every operation rounds once, in the written order (no contraction), so the values equal the
// CPU float64 evaluation of the same program bit for bit.
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double rn_max(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double rn_min(double a, double b) { return a < b ? a : b; }

static __device__ __forceinline__ const float* table_of_d(const double* __restrict__ p) {
    return reinterpret_cast<const float*>(__double_as_longlong(p[10]));
}

static __device__ __forceinline__ double lerp_d(double a, double b, double t) {
    return rn_add(rn_mul(a, rn_sub(1.0, t)), rn_mul(b, t));
}

// The same samples in float64 (the table's float32 values promoted).
static __device__ double grid_sample_d(const double* __restrict__ p, double x, double y, double z) {
    const int nx = (int)p[6], ny = (int)p[7], nz = (int)p[8];
    const double pitch = p[3];
    const double fx = rn_div(rn_sub(x, p[0]), pitch), fy = rn_div(rn_sub(y, p[1]), pitch),
                 fz = rn_div(rn_sub(z, p[2]), pitch);
    if (!(fx >= 0.0 && fy >= 0.0 && fz >= 0.0 && fx <= (double)(nx - 1) && fy <= (double)(ny - 1) &&
          fz <= (double)(nz - 1)))
        return 1.0e6;
    const int ix = (int)floor(fx), iy = (int)floor(fy), iz = (int)floor(fz);
    const int ix1 = min(ix + 1, nx - 1), iy1 = min(iy + 1, ny - 1), iz1 = min(iz + 1, nz - 1);
    const double tx = rn_sub(fx, (double)ix), ty = rn_sub(fy, (double)iy), tz = rn_sub(fz, (double)iz);
    const float* g = table_of_d(p);
    auto at = [&](int i, int j, int k) { return (double)g[((int64_t)i * ny + j) * nz + k]; };
    const double c00 = lerp_d(at(ix, iy, iz), at(ix1, iy, iz), tx), c10 = lerp_d(at(ix, iy1, iz), at(ix1, iy1, iz), tx);
    const double c01 = lerp_d(at(ix, iy, iz1), at(ix1, iy, iz1), tx), c11 = lerp_d(at(ix, iy1, iz1), at(ix1, iy1, iz1), tx);
    const double val = lerp_d(lerp_d(c00, c10, ty), lerp_d(c01, c11, ty), tz);
    return p[5] != 0.0 ? val : rn_mul(rn_sub(p[4], val), pitch);
}

static __device__ double revolve_sample_d(const double* __restrict__ p, double x, double y, double z) {
    const int nr = (int)p[3], nz = (int)p[4];
    const double r = __dsqrt_rn(rn_add(rn_mul(x, x), rn_mul(y, y)));
    const double fr = rn_div(rn_sub(r, p[0]), p[2]), fz = rn_div(rn_sub(z, p[1]), p[2]);
    const double cr = fmin(fmax(fr, -1.0e9), 1.0e9), cz = fmin(fmax(fz, -1.0e9), 1.0e9);
    const int ir = min(max((int)cr, 0), nr - 2), iz = min(max((int)cz, 0), nz - 2);
    const double tr = fmin(fmax(rn_sub(fr, (double)ir), 0.0), 1.0), tz = fmin(fmax(rn_sub(fz, (double)iz), 0.0), 1.0);
    const float* g = table_of_d(p);
    const double v00 = g[(int64_t)ir * nz + iz], v01 = g[(int64_t)ir * nz + iz + 1];
    const double v10 = g[(int64_t)(ir + 1) * nz + iz], v11 = g[(int64_t)(ir + 1) * nz + iz + 1];
    const double ur = rn_sub(1.0, tr), uz = rn_sub(1.0, tz);
    double v = rn_mul(rn_mul(v00, ur), uz);
    v = rn_add(v, rn_mul(rn_mul(v01, ur), tz));
    v = rn_add(v, rn_mul(rn_mul(v10, tr), uz));
    return rn_add(v, rn_mul(rn_mul(v11, tr), tz));
}

static __device__ __noinline__ double canon_d(int type, const double* __restrict__ p, double x, double y, double z) {
    switch (type) {
    case P_SPHERE:
        return rn_sub(__dsqrt_rn(rn_add(rn_add(rn_mul(x, x), rn_mul(y, y)), rn_mul(z, z))), p[0]);
    case P_BOX: {
        const double qx = rn_sub(fabs(x), p[0]), qy = rn_sub(fabs(y), p[1]), qz = rn_sub(fabs(z), p[2]);
        const double ox = rn_max(qx, 0.0), oy = rn_max(qy, 0.0), oz = rn_max(qz, 0.0);
        const double out = __dsqrt_rn(rn_add(rn_add(rn_mul(ox, ox), rn_mul(oy, oy)), rn_mul(oz, oz)));
        return rn_add(out, rn_min(rn_max(qx, rn_max(qy, qz)), 0.0));
    }
    case P_CYLINDER: {
        const double rad = __dsqrt_rn(rn_add(rn_mul(x, x), rn_mul(y, y)));
        const double qx = rn_sub(rad, p[0]), qy = rn_sub(fabs(z), p[1]);
        const double ox = rn_max(qx, 0.0), oy = rn_max(qy, 0.0);
        return rn_add(__dsqrt_rn(rn_add(rn_mul(ox, ox), rn_mul(oy, oy))), rn_min(rn_max(qx, qy), 0.0));
    }
    case P_CONE: {
        const double rad = __dsqrt_rn(rn_add(rn_mul(x, x), rn_mul(y, y))), h = p[2];
        const double t = rn_min(rn_max(rn_div(rn_add(z, rn_div(h, 2.0)), h), 0.0), 1.0);
        const double r_at = rn_add(p[0], rn_mul(rn_sub(p[1], p[0]), t));
        const double qy = rn_sub(fabs(z), rn_div(h, 2.0)), qx = rn_sub(rad, r_at);
        const double ox = rn_max(qx, 0.0), oy = rn_max(qy, 0.0);
        return rn_add(__dsqrt_rn(rn_add(rn_mul(ox, ox), rn_mul(oy, oy))), rn_min(rn_max(qx, qy), 0.0));
    }
    case P_HALFSPACE:
        return rn_add(rn_add(rn_mul(x, p[0]), rn_mul(y, p[1])), rn_mul(z, p[2]));
    case P_FRUSTUM: {
        const double z1 = p[0], hx0 = p[1], hy0 = p[2], hx1 = p[3], hy1 = p[4], cx1 = p[5], cy1 = p[6];
        const double kx = rn_div(rn_sub(hx1, hx0), z1), ky = rn_div(rn_sub(hy1, hy0), z1);
        const double kcx = rn_div(cx1, z1), kcy = rn_div(cy1, z1);
        const double d_zlo = -z, d_zhi = rn_sub(z, z1);
        const double a1 = -rn_add(kx, kcx), n1 = __dsqrt_rn(rn_add(1.0, rn_mul(a1, a1)));
        const double a2 = -rn_sub(kx, kcx), n2 = __dsqrt_rn(rn_add(1.0, rn_mul(a2, a2)));
        const double a3 = -rn_add(ky, kcy), n3 = __dsqrt_rn(rn_add(1.0, rn_mul(a3, a3)));
        const double a4 = -rn_sub(ky, kcy), n4 = __dsqrt_rn(rn_add(1.0, rn_mul(a4, a4)));
        const double d_xhi = rn_div(rn_sub(rn_add(x, rn_mul(a1, z)), hx0), n1);
        const double d_xlo = rn_div(rn_sub(rn_add(-x, rn_mul(a2, z)), hx0), n2);
        const double d_yhi = rn_div(rn_sub(rn_add(y, rn_mul(a3, z)), hy0), n3);
        const double d_ylo = rn_div(rn_sub(rn_add(-y, rn_mul(a4, z)), hy0), n4);
        return rn_max(rn_max(rn_max(d_zlo, d_zhi), rn_max(d_xhi, d_xlo)), rn_max(d_yhi, d_ylo));
    }
    case P_CAPSULE: {
        const double bx = p[0], by = p[1], bz = p[2];
        const double bb = rn_add(rn_add(rn_mul(bx, bx), rn_mul(by, by)), rn_mul(bz, bz));
        const double h = bb > 0.0 ? rn_min(rn_max(rn_div(rn_add(rn_add(rn_mul(x, bx), rn_mul(y, by)), rn_mul(z, bz)), bb), 0.0), 1.0)
                                  : 0.0;
        const double dx = rn_sub(x, rn_mul(bx, h)), dy = rn_sub(y, rn_mul(by, h)), dz = rn_sub(z, rn_mul(bz, h));
        return rn_sub(__dsqrt_rn(rn_add(rn_add(rn_mul(dx, dx), rn_mul(dy, dy)), rn_mul(dz, dz))), p[3]);
    }
    case P_TORUS: {
        const double qx = rn_sub(__dsqrt_rn(rn_add(rn_mul(x, x), rn_mul(y, y))), p[0]);
        return rn_sub(__dsqrt_rn(rn_add(rn_mul(qx, qx), rn_mul(z, z))), p[1]);
    }
    case P_CYL_INF:
        return rn_sub(__dsqrt_rn(rn_add(rn_mul(x, x), rn_mul(y, y))), p[0]);
    case P_GRID:
        return grid_sample_d(p, x, y, z);
    case P_REVOLVE:
        return revolve_sample_d(p, x, y, z);
    case P_BAR: {
        const double r = __dsqrt_rn(rn_add(rn_mul(x, x), rn_mul(y, y)));
        return rn_max(rn_sub(r, p[0]), rn_max(rn_sub(p[1], z), rn_sub(z, p[2])));
    }
    case P_POCKET: {
        const double qx = rn_sub(fabs(x), rn_sub(p[0], p[2])), qy = rn_sub(fabs(y), rn_sub(p[1], p[2]));
        const double ox = rn_max(qx, 0.0), oy = rn_max(qy, 0.0);
        const double dxy = rn_sub(rn_add(__dsqrt_rn(rn_add(rn_mul(ox, ox), rn_mul(oy, oy))), rn_min(rn_max(qx, qy), 0.0)), p[2]);
        const double roof = rn_add(p[4], __dsqrt_rn(rn_max(rn_sub(rn_mul(p[3], p[3]), rn_mul(x, x)), 0.0)));
        return rn_max(dxy, rn_sub(z, roof));
    }
    case P_XBORE: {
        const double dz = rn_sub(z, p[1]);
        return rn_max(rn_sub(__dsqrt_rn(rn_add(rn_mul(y, y), rn_mul(dz, dz))), p[0]), rn_sub(fabs(x), p[2]));
    }
    default:
        return __longlong_as_double(0x7ff8000000000000ll);
    }
}

__device__ __forceinline__ double prim_world_d(const FbPrim& P, double x, double y, double z) {
    const double* A = P.A;
    const double lx = rn_add(rn_add(rn_add(rn_mul(A[0], x), rn_mul(A[1], y)), rn_mul(A[2], z)), A[3]);
    const double ly = rn_add(rn_add(rn_add(rn_mul(A[4], x), rn_mul(A[5], y)), rn_mul(A[6], z)), A[7]);
    const double lz = rn_add(rn_add(rn_add(rn_mul(A[8], x), rn_mul(A[9], y)), rn_mul(A[10], z)), A[11]);
    return rn_sub(rn_mul(P.s, canon_d(P.type, P.p, lx, ly, lz)), P.off);
}

__device__ __forceinline__ double combine_d(int op, double a, double b, double k) {
    if (op == OP_UNION) {
        if (k <= 0.0) return rn_min(a, b);
        const double h = rn_div(rn_max(rn_sub(k, fabs(rn_sub(a, b))), 0.0), k);
        return rn_sub(rn_min(a, b), rn_mul(rn_mul(rn_mul(h, h), k), 0.25));
    }
    if (op == OP_INTERSECT) {
        if (k <= 0.0) return rn_max(a, b);
        const double h = rn_div(rn_max(rn_sub(k, fabs(rn_sub(a, b))), 0.0), k);
        return rn_add(rn_max(a, b), rn_mul(rn_mul(rn_mul(h, h), k), 0.25));
    }
    if (k <= 0.0) return rn_max(a, -b);
    const double h = rn_div(rn_max(rn_sub(k, fabs(rn_add(a, b))), 0.0), k);
    return rn_add(rn_max(a, -b), rn_mul(rn_mul(rn_mul(h, h), k), 0.25));
}

__device__ __forceinline__ double chain_apply_d(int op, double acc, double v, double k) {
    switch (op) {
    case CH_SET: return v;
    case CH_SETNEG: return -v;
    case CH_OFFSET: return rn_sub(acc, k);
    case CH_UNION: return combine_d(OP_UNION, acc, v, k);
    case CH_INTERSECT: return combine_d(OP_INTERSECT, acc, v, k);
    default: return combine_d(OP_SUBTRACT, acc, v, k);
    }
}

// General postfix program in float64 at one world point (stack depth <= 32).
static __device__ double program_eval_d(const FbPrim* __restrict__ prims, const FbInsn* __restrict__ prog, int n,
                                 double x, double y, double z) {
    double st[32];
    int sp = 0;
    for (int i = 0; i < n; ++i) {
        const FbInsn I = prog[i];
        if (I.op == OP_PUSH) {
            if (sp < 32) st[sp++] = prim_world_d(prims[I.arg], x, y, z);
        } else if (I.op == OP_OFFSET) {
            if (sp > 0) st[sp - 1] = rn_sub(st[sp - 1], I.k);
        } else if (sp > 1) {
            const double b = st[--sp];
            st[sp - 1] = combine_d(I.op, st[sp - 1], b, I.k);
        }
    }
    return sp == 1 ? st[0] : __longlong_as_double(0x7ff8000000000000ll);
}
