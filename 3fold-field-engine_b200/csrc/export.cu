// Export step: the zero (or `level`) isosurface of a resident sparse field as a triangle mesh,
// straight from the leaf tiles -- the mesh that marching cubes gives on the dense reconstruction
// (tiles in active blocks, -BIG / +BIG elsewhere; src/field_engine/faltkarna_v1.py:302-350 followed
// by skimage.measure.marching_cubes, and faltvolym_v1.py:83-104 for the enclosed volume).
//
// Vertices: one per grid edge whose ends lie on opposite sides (inside = value < level, the
// classifier's convention that 0 counts as outside), at the linear interpolation
// t = g0 / (g0 - g1), g = value - level, in float64, stored as float32 world coordinates
// origin + pitch (index + t).  Each edge is owned by the active block of its lower end, else by the
// active block of its upper end; a block numbers its edges in slot order (inner edges
// ((lx B + ly) B + lz) 3 + axis, then the edges that enter it across its low faces), so vertex ids
// run block by block in ascending block id.  A bit word per 32 slots and the word's exclusive
// prefix turn an edge into its vertex id with one popcount.
//
// Faces: per cube, the crossing edges are joined on each of its six faces into segments that keep
// the inside on their left as seen from outside the cube; a face with four crossings is resolved by
// the asymptotic decider (the sign of the bilinear saddle value, evaluated from the face's own four
// values, so both cubes that share the face agree and the surface has no cracks).  The segments
// close into loops; a loop is fanned from its first vertex, in loop order from its lowest-numbered
// edge, that lies on no cube face the loop crosses twice (else from the lowest edge: possible only
// where the field changes sign several times across one cube, and then the fan can lay a flat
// zero-volume triangle into such a face), triangles wound so that their normals point to the
// outside (increasing value).  A cube is owned by the active block of its lowest
// corner, else by the first active block among its corners; triangles run block by block, cubes in
// lexicographic order inside a block's range, loops by lowest edge.  Cubes whose interior is
// ambiguous (two loops that the trilinear interior would join by a tunnel) keep the two loops.
#include "common.cuh"
#include "scan.cuh"
#include <algorithm>
#include <climits>

namespace {

constexpr int kMcThreads = 256;
constexpr int kMcMaxBlock = 32;

struct McField {
    const int32_t* kind;
    const int32_t* slot;
    const float* tiles;
    int64_t nx, ny, nz;
    int B, nby, nbz;
    double ox, oy, oz, pitch, level;
    float big;
};

__host__ __device__ inline int64_t mc_slots(int B) { return 3LL * B * B * B + 3LL * B * B; }
__host__ __device__ inline int64_t mc_words(int B) { return (mc_slots(B) + 31) / 32; }

// Corner c of a cube: bit 0 = +x, bit 1 = +y, bit 2 = +z.  Edge e = axis * 4 + w runs along
// `axis` from the corner whose other two bits are w (lower axis in bit 0).
__device__ __forceinline__ int edge_corner0(int e) {
    const int a = e >> 2, w = e & 3;
    if (a == 0) return ((w & 1) << 1) | ((w >> 1) << 2);
    if (a == 1) return (w & 1) | ((w >> 1) << 2);
    return (w & 1) | ((w >> 1) << 1);
}
__device__ __forceinline__ int edge_of(int ca, int cb) {  // corners that differ in one bit
    const int d = __ffs(ca ^ cb) - 1, c = ca & cb;
    int w;
    if (d == 0) w = ((c >> 1) & 1) | (((c >> 2) & 1) << 1);
    else if (d == 1) w = (c & 1) | (((c >> 2) & 1) << 1);
    else w = (c & 1) | (((c >> 1) & 1) << 1);
    return d * 4 + w;
}

// The loops of one cube: next[e] for every crossing edge e (cross bit e).  g: value - level at the
// eight corners, float64.
struct CubeLoops {
    unsigned cross;
    int8_t next[12];
};

__device__ CubeLoops cube_loops(const double g[8]) {
    CubeLoops L;
    unsigned in = 0;
    for (int c = 0; c < 8; ++c) in |= (unsigned)(g[c] < 0.0) << c;
    L.cross = 0;
    for (int e = 0; e < 12; ++e) L.next[e] = -1;
    if (in == 0 || in == 255) return L;
    for (int e = 0; e < 12; ++e) {
        const int c0 = edge_corner0(e), c1 = c0 | (1 << (e >> 2));
        L.cross |= (unsigned)(((in >> c0) & 1) != ((in >> c1) & 1)) << e;
    }
    for (int f = 0; f < 6; ++f) {
        const int a = f >> 1, s = f & 1, u = (a + 1) % 3, v = (a + 2) % 3;
        // corners in counter-clockwise order as seen from outside the face
        int q[4];
        const int b = s << a;
        q[0] = b;
        q[2] = b | (1 << u) | (1 << v);
        q[1] = b | (1 << (s ? u : v));
        q[3] = b | (1 << (s ? v : u));
        int E[4], inq[4];
        for (int i = 0; i < 4; ++i) {
            E[i] = edge_of(q[i], q[(i + 1) & 3]);
            inq[i] = (in >> q[i]) & 1;
        }
        const int k = (inq[0] != inq[1]) + (inq[1] != inq[2]) + (inq[2] != inq[3]) + (inq[3] != inq[0]);
        if (k == 2) {
            int st = -1, en = -1;
            for (int i = 0; i < 4; ++i) {
                if (inq[i] && !inq[(i + 1) & 3]) st = E[i];
                if (!inq[i] && inq[(i + 1) & 3]) en = E[i];
            }
            L.next[st] = (int8_t)en;
        } else if (k == 4) {
            // asymptotic decider on the (u, v)-ordered values: the saddle value's sign
            const double g00 = g[b], g10 = g[b | (1 << u)], g11 = g[b | (1 << u) | (1 << v)], g01 = g[b | (1 << v)];
            const double num = __dsub_rn(__dmul_rn(g00, g11), __dmul_rn(g10, g01));
            const bool connected = (g00 < 0.0) ? (num > 0.0) : (num < 0.0);  // inside corners joined
            for (int i = 0; i < 4; ++i)
                if (inq[i]) L.next[E[i]] = (int8_t)(connected ? E[(i + 1) & 3] : E[(i + 3) & 3]);
        }
    }
    return L;
}

// Bit mask of the two cube faces (axis * 2 + side) that contain edge e.
__device__ __forceinline__ unsigned edge_faces(int e) {
    const int c0 = edge_corner0(e), a = e >> 2;
    unsigned m = 0;
    for (int b = 0; b < 3; ++b)
        if (b != a) m |= 1u << (b * 2 + ((c0 >> b) & 1));
    return m;
}

// Next edge of a loop; every crossing edge starts exactly one face segment (the two faces through
// an edge walk it in opposite directions), so next is a permutation of the crossing edges.  The
// checks only keep a broken table inside the cube's 12 edges.
__device__ __forceinline__ int loop_next(const CubeLoops& L, int e) {
    const int n = L.next[e];
    return n >= 0 && n < 12 ? n : -1;
}

// Triangles of a cube's loops: sum over loops of (length - 2).
__device__ __forceinline__ int cube_triangles(const CubeLoops& L) {
    int loops = 0;
    unsigned todo = L.cross;
    while (todo) {
        const int e0 = __ffs(todo) - 1;
        int e = e0;
        for (int i = 0; i < 12; ++i) {
            todo &= ~(1u << e);
            e = loop_next(L, e);
            if (e < 0 || e == e0) break;
        }
        if (e != e0) return 0;
        ++loops;
    }
    return __popc(L.cross) - 2 * loops;
}

// Value at global voxel (x, y, z) inside the grid: tile value, or -BIG / +BIG by the block's kind.
__device__ __forceinline__ float voxel_value(const McField& F, int64_t x, int64_t y, int64_t z) {
    const int B = F.B;
    const int64_t blk = ((x / B) * F.nby + y / B) * F.nbz + z / B;
    const int32_t s = F.slot[blk];
    if (s >= 0) return F.tiles[(int64_t)s * B * B * B + ((x % B) * B + (y % B)) * B + (z % B)];
    return F.kind[blk] < 0 ? -F.big : F.big;
}

// World position of the vertex on edge (p, axis), p the edge's lower end.
__device__ __forceinline__ void edge_vertex(const McField& F, int64_t px, int64_t py, int64_t pz, int a, double g0,
                                            double g1, float* out) {
    const double t = __ddiv_rn(g0, __dsub_rn(g0, g1));
    double p[3] = {(double)px, (double)py, (double)pz};
    p[a] = __dadd_rn(p[a], t);
    out[0] = (float)__dadd_rn(F.ox, __dmul_rn(F.pitch, p[0]));
    out[1] = (float)__dadd_rn(F.oy, __dmul_rn(F.pitch, p[1]));
    out[2] = (float)__dadd_rn(F.oz, __dmul_rn(F.pitch, p[2]));
}

// Vertex id of edge (p, axis): owner block, slot, popcount below the slot.  -1 if the edge has no
// vertex (never for the edges of a cube's loops).
__device__ int64_t vertex_id(const McField& F, int64_t px, int64_t py, int64_t pz, int a, const uint32_t* bits,
                             const int32_t* wpre, const int32_t* voff, int64_t W) {
    const int B = F.B;
    int64_t blk = ((px / B) * F.nby + py / B) * F.nbz + pz / B;
    int32_t s = F.slot[blk];
    int64_t sl;
    if (s >= 0) {
        sl = (((px % B) * B + (py % B)) * B + (pz % B)) * 3 + a;
    } else {
        int64_t q[3] = {px, py, pz};
        q[a] += 1;
        blk = ((q[0] / B) * F.nby + q[1] / B) * F.nbz + q[2] / B;
        s = F.slot[blk];
        if (s < 0) return -1;
        const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
        sl = 3LL * B * B * B + (int64_t)a * B * B + (q[u] % B) * B + (q[v] % B);
    }
    const uint32_t word = bits[s * W + (sl >> 5)];
    if (!((word >> (sl & 31)) & 1u)) return -1;
    return (int64_t)voff[s] + wpre[s * W + (sl >> 5)] + __popc(word & ((1u << (sl & 31)) - 1u));
}

// Block-wide exclusive scan of one int per thread (kMcThreads); returns the prefix, *total the sum.
__device__ __forceinline__ int block_scan(int v, int* s_warp, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kMcThreads / 32 ? s_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kMcThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const int before = (warp ? s_warp[warp - 1] : 0) + inc - v;
    *total = s_warp[kMcThreads / 32 - 1];
    __syncthreads();
    return before;
}

// One CTA per active block (grid-stride).  kEmit = false: edge bits, word prefixes, vertex and
// triangle counts.  kEmit = true: vertices, triangles and the block's volume term.
template <bool kEmit>
__global__ void __launch_bounds__(kMcThreads) k_mc(McField F, const int32_t* __restrict__ active, int64_t n_active,
                                                   uint32_t* __restrict__ bits, int32_t* __restrict__ wpre,
                                                   int32_t* __restrict__ vcount, int32_t* __restrict__ tcount,
                                                   float* __restrict__ verts, int64_t* __restrict__ vkey,
                                                   int32_t* __restrict__ faces, double* __restrict__ vol_part,
                                                   int32_t* __restrict__ err, unsigned long long* __restrict__ totals) {
    extern __shared__ float s_val[];  // (B + 2)^3 values of the block and its low/high shell
    __shared__ int s_nslot[27];
    __shared__ int s_warp[kMcThreads / 32];
    __shared__ double s_vol[kMcThreads / 32];
    const int B = F.B, R = B + 2;
    const int64_t W = mc_words(B), S = mc_slots(B);
    const int64_t nbx = (F.nx + B - 1) / B;
    for (int64_t sa = blockIdx.x; sa < n_active; sa += gridDim.x) {
        const int64_t id = active[sa];
        const int64_t bx = id / ((int64_t)F.nby * F.nbz), by = (id / F.nbz) % F.nby, bz = id % F.nbz;
        const int64_t x0 = bx * B, y0 = by * B, z0 = bz * B;
        if (threadIdx.x < 27) {
            const int64_t nx_ = bx + threadIdx.x / 9 - 1, ny_ = by + (threadIdx.x / 3) % 3 - 1, nz_ = bz + threadIdx.x % 3 - 1;
            int v = -2;  // outside the grid
            if (nx_ >= 0 && nx_ < nbx && ny_ >= 0 && ny_ < F.nby && nz_ >= 0 && nz_ < F.nbz)
                v = F.slot[(nx_ * F.nby + ny_) * F.nbz + nz_];
            s_nslot[threadIdx.x] = v;
        }
        for (int r = threadIdx.x; r < R * R * R; r += kMcThreads) {
            const int64_t x = x0 - 1 + r / (R * R), y = y0 - 1 + (r / R) % R, z = z0 - 1 + r % R;
            float v = 0.f;
            if (x >= 0 && x < F.nx && y >= 0 && y < F.ny && z >= 0 && z < F.nz) v = voxel_value(F, x, y, z);
            s_val[r] = v;
        }
        __syncthreads();
        auto val = [&](int64_t x, int64_t y, int64_t z) -> double {  // value - level, from the region
            return __dsub_rn((double)s_val[((x - x0 + 1) * R + (y - y0 + 1)) * R + (z - z0 + 1)], F.level);
        };
        // ---- edges ----
        int run = 0;  // vertices before this chunk (emit) / count (count pass)
        for (int64_t c0 = 0; c0 < S; c0 += kMcThreads) {
            const int64_t sl = c0 + threadIdx.x;
            bool hit = false;
            int64_t p[3] = {0, 0, 0};
            int a = 0;
            if (sl < S) {
                if (sl < 3LL * B * B * B) {
                    a = (int)(sl % 3);
                    const int64_t lin = sl / 3;
                    p[0] = x0 + lin / (B * B);
                    p[1] = y0 + (lin / B) % B;
                    p[2] = z0 + lin % B;
                } else {
                    const int64_t r = sl - 3LL * B * B * B;
                    a = (int)(r / (B * B));
                    const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
                    p[0] = x0;
                    p[1] = y0;
                    p[2] = z0;
                    p[u] += (r % (B * B)) / B;
                    p[v] += r % B;
                    p[a] -= 1;
                }
                const int64_t n[3] = {F.nx, F.ny, F.nz};
                bool ok = p[0] >= 0 && p[1] >= 0 && p[2] >= 0 && p[0] < n[0] && p[1] < n[1] && p[2] < n[2] &&
                          p[a] + 1 < n[a];
                if (ok && sl >= 3LL * B * B * B) {  // entering edge: ours only when its lower block is inactive
                    const int nb = a == 0 ? 4 : (a == 1 ? 10 : 12);  // the (-1) neighbour along a
                    ok = s_nslot[nb] < 0;
                }
                if (ok) {
                    int64_t q[3] = {p[0], p[1], p[2]};
                    q[a] += 1;
                    const double g0 = val(p[0], p[1], p[2]), g1 = val(q[0], q[1], q[2]);
                    hit = (g0 < 0.0) != (g1 < 0.0);
                    if (kEmit && hit) {
                        // vertex id: this block's offset + words before + bits below, from the count pass
                        const uint32_t word = bits[sa * W + (sl >> 5)];
                        const int64_t vid = (int64_t)vcount[sa] + wpre[sa * W + (sl >> 5)] +
                                            __popc(word & ((1u << (sl & 31)) - 1u));
                        edge_vertex(F, p[0], p[1], p[2], a, g0, g1, verts + 3 * vid);
                        if (vkey) vkey[vid] = ((p[0] * F.ny + p[1]) * F.nz + p[2]) * 3 + a;
                    }
                }
            }
            const unsigned ball = __ballot_sync(0xffffffffu, hit);
            if (!kEmit) {
                // word prefixes inside the block: a running count over the chunk's words
                const int wc = (threadIdx.x & 31) == 0 ? __popc(ball) : 0;
                int chunk_total;
                const int before = block_scan(wc, s_warp, &chunk_total);
                if ((threadIdx.x & 31) == 0 && sl < S) {
                    bits[sa * W + (sl >> 5)] = ball;
                    wpre[sa * W + (sl >> 5)] = run + before;
                }
                run += chunk_total;
            }
        }
        if (!kEmit && threadIdx.x == 0) {
            vcount[sa] = run;
            atomicAdd(&totals[0], (unsigned long long)run);
        }
        // ---- cubes: lowest corners x0 - 1 .. x0 + B - 1 per axis, lexicographic ----
        const int C = B + 1;
        const int64_t ncube = (int64_t)C * C * C;
        int tri_run = 0;
        double vol = 0.0;
        for (int64_t c0 = 0; c0 < ncube; c0 += kMcThreads) {
            const int64_t ci = c0 + threadIdx.x;
            int ntri = 0;
            CubeLoops L;
            L.cross = 0;
            int64_t m[3] = {0, 0, 0};
            if (ci < ncube) {
                m[0] = x0 - 1 + ci / (C * C);
                m[1] = y0 - 1 + (ci / C) % C;
                m[2] = z0 - 1 + ci % C;
                bool ok = m[0] >= 0 && m[1] >= 0 && m[2] >= 0 && m[0] + 1 < F.nx && m[1] + 1 < F.ny && m[2] + 1 < F.nz;
                if (ok && (m[0] < x0 || m[1] < y0 || m[2] < z0)) {
                    // a cube reaching into the low shell: ours if its first corner in an active block is here
                    int first = -1;
                    for (int c = 0; c < 8 && first < 0; ++c) {
                        const int o0 = m[0] + (c & 1) < x0 ? 0 : (m[0] + (c & 1) >= x0 + B ? 2 : 1);
                        const int o1 = m[1] + ((c >> 1) & 1) < y0 ? 0 : (m[1] + ((c >> 1) & 1) >= y0 + B ? 2 : 1);
                        const int o2 = m[2] + ((c >> 2) & 1) < z0 ? 0 : (m[2] + ((c >> 2) & 1) >= z0 + B ? 2 : 1);
                        const int nb = o0 * 9 + o1 * 3 + o2;
                        if (s_nslot[nb] >= 0) first = nb;
                    }
                    ok = first == 13;
                }
                if (ok) {
                    double g[8];
                    for (int c = 0; c < 8; ++c) g[c] = val(m[0] + (c & 1), m[1] + ((c >> 1) & 1), m[2] + ((c >> 2) & 1));
                    L = cube_loops(g);
                    ntri = cube_triangles(L);
                }
            }
            if (!kEmit) {
                tri_run += ntri;
                continue;
            }
            int chunk_total;
            const int before = block_scan(ntri, s_warp, &chunk_total);
            if (ntri) {
                int64_t at = (int64_t)tcount[sa] + tri_run + before;
                unsigned todo = L.cross;
                while (todo) {
                    const int e0 = __ffs(todo) - 1;
                    int64_t vid[12];
                    float pos[12][3];
                    int el[12];
                    int len = 0, e = e0;
                    do {  // a permutation cycle of at most 12 edges (cube_triangles counted it)
                        todo &= ~(1u << e);
                        el[len] = e;
                        const int cc = edge_corner0(e);
                        const int64_t px = m[0] + (cc & 1), py = m[1] + ((cc >> 1) & 1), pz = m[2] + ((cc >> 2) & 1);
                        const int ax = e >> 2;
                        vid[len] = vertex_id(F, px, py, pz, ax, bits, wpre, vcount, W);
                        int64_t q[3] = {px, py, pz};
                        q[ax] += 1;
                        edge_vertex(F, px, py, pz, ax, val(px, py, pz), val(q[0], q[1], q[2]), pos[len]);
                        ++len;
                        e = loop_next(L, e);
                    } while (e >= 0 && e != e0 && len < 12);
                    // fan centre: the first vertex on no face that the loop crosses twice (a fan
                    // from such a face would lay a flat triangle into it), else the lowest edge
                    unsigned seen = 0, twice = 0;
                    for (int i = 0; i < len; ++i) {
                        const unsigned f = edge_faces(el[i]) & edge_faces(el[i + 1 < len ? i + 1 : 0]);
                        twice |= seen & f;
                        seen |= f;
                    }
                    int c = 0;
                    while (c < len && (edge_faces(el[c]) & twice)) ++c;
                    if (c == len) c = 0;
                    for (int i = 1; i + 1 < len; ++i) {
                        const int j0 = c, j1 = (c + i + 1) % len, j2 = (c + i) % len;
                        const int64_t t3 = 3 * (at++);
                        if (vid[j0] < 0 || vid[j1] < 0 || vid[j2] < 0) atomicAdd(err, 1);
                        faces[t3] = (int32_t)vid[j0];
                        faces[t3 + 1] = (int32_t)vid[j1];
                        faces[t3 + 2] = (int32_t)vid[j2];
                        // signed volume term v0 . (v1 x v2) of the triangle as written
                        const double ax_ = pos[j0][0], ay = pos[j0][1], az = pos[j0][2];
                        const double bx_ = pos[j1][0], by_ = pos[j1][1], bz_ = pos[j1][2];
                        const double cx = pos[j2][0], cy = pos[j2][1], cz = pos[j2][2];
                        vol += ax_ * (by_ * cz - bz_ * cy) + ay * (bz_ * cx - bx_ * cz) + az * (bx_ * cy - by_ * cx);
                    }
                }
            }
            tri_run += chunk_total;
        }
        if (!kEmit) {
            // block triangle count: a reduction over the threads' sums
            int dummy;
            const int before = block_scan(tri_run, s_warp, &dummy);
            (void)before;
            if (threadIdx.x == 0) {
                tcount[sa] = dummy;
                atomicAdd(&totals[1], (unsigned long long)dummy);
            }
        } else {
            for (int o = 16; o > 0; o >>= 1) vol += __shfl_xor_sync(0xffffffffu, vol, o);
            if ((threadIdx.x & 31) == 0) s_vol[threadIdx.x >> 5] = vol;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int w = 0; w < kMcThreads / 32; ++w) t += s_vol[w];
                vol_part[sa] = t;
            }
        }
        __syncthreads();
    }
}

// Sum of the blocks' volume terms in block order (one CTA, fixed tree): deterministic.
__global__ void k_mc_volume(const double* __restrict__ part, int64_t n, double* __restrict__ out) {
    __shared__ double s[kMcThreads];
    double t = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += kMcThreads) t += part[i];
    s[threadIdx.x] = t;
    __syncthreads();
    for (int o = kMcThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = s[0] / 6.0;
}

__global__ void k_mc_slot_map(const int32_t* __restrict__ active, int64_t n_active, int32_t* __restrict__ slot) {
    const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a < n_active) slot[active[a]] = (int32_t)a;
}

int mc_field(McField& F, const int32_t* d_kind, const float* d_tiles, int64_t nx, int64_t ny, int64_t nz, int32_t block,
             double ox, double oy, double oz, double pitch, double level, float big, const int32_t* d_slot) {
    if (!d_kind || !d_slot || nx < 1 || ny < 1 || nz < 1 || block < 1 || block > kMcMaxBlock ||
        !(pitch > 0) || !(level == level) || level > 1e300 || level < -1e300)
        return FB_INVALID;
    F = McField{d_kind, d_slot, d_tiles, nx, ny, nz, block, (int)((ny + block - 1) / block),
                (int)((nz + block - 1) / block), ox, oy, oz, pitch, level, big};
    return FB_OK;
}

size_t mc_smem(int B) { return (size_t)(B + 2) * (B + 2) * (B + 2) * sizeof(float); }

template <bool kEmit>
int mc_launch(const McField& F, const int32_t* d_active, int64_t n_active, uint32_t* bits, int32_t* wpre,
              int32_t* vcount, int32_t* tcount, float* verts, int64_t* vkey, int32_t* faces, double* vol_part,
              int32_t* err, unsigned long long* totals, cudaStream_t st) {
    if (n_active == 0) return FB_OK;
    const size_t smem = mc_smem(F.B);
    if (smem > 48 * 1024) FB_CUDA(cudaFuncSetAttribute(k_mc<kEmit>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (int)std::min<int64_t>(n_active, (int64_t)fb_sm_count() * 8);
    k_mc<kEmit><<<grid, kMcThreads, smem, st>>>(F, d_active, n_active, bits, wpre, vcount, tcount, verts, vkey,
                                               faces, vol_part, err, totals);
    FB_LAUNCH();
    return FB_OK;
}

// ---- connected components of the exported mesh (faltvolym_v1.py:95-101 keeps the largest) ----
// Union-find over the vertices, a thread per triangle; a root is always linked under the smaller
// root, so parent[v] <= v, every chain ends, and a component's final root is its smallest vertex id
// whatever the order of the unions.  Reads go through volatile pointers (other threads link and
// halve paths meanwhile); path halving only writes ancestors into non-roots.
constexpr int kUnionTries = 1 << 16;

__device__ __forceinline__ int32_t cc_find(volatile int32_t* parent, int32_t x) {
    while (true) {  // strictly decreasing ids: at most x steps
        const int32_t p = parent[x];
        if (p == x) return x;
        const int32_t gp = parent[p];
        if (gp != p) parent[x] = gp;
        x = gp;
    }
}

__device__ __forceinline__ void cc_union(int32_t* parent, int32_t a, int32_t b, int32_t* err) {
    for (int it = 0; it < kUnionTries; ++it) {
        a = cc_find(parent, a);
        b = cc_find(parent, b);
        if (a == b) return;
        if (a < b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        const int32_t old = atomicCAS(parent + a, a, b);
        if (old == a) return;
        a = old;  // linked meanwhile: continue from its new parent
    }
    atomicAdd(err, 1);
}

__global__ void k_cc_init(int32_t* __restrict__ parent, double* __restrict__ vol, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) {
        parent[i] = (int32_t)i;
        vol[i] = 0.0;
    }
}

__global__ void k_cc_union(const int32_t* __restrict__ faces, int64_t nf, int32_t* parent, int32_t* err) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nf) return;
    cc_union(parent, faces[3 * t], faces[3 * t + 1], err);
    cc_union(parent, faces[3 * t], faces[3 * t + 2], err);
}

__global__ void k_cc_label(int32_t* parent, int64_t n, int32_t* __restrict__ count) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t r = cc_find(parent, (int32_t)i);
    if (r == (int32_t)i) atomicAdd(count, 1);
}

__global__ void k_cc_flatten(const int32_t* __restrict__ parent, int64_t n, int32_t* __restrict__ label) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t x = (int32_t)i;
    while (parent[x] != x) x = parent[x];  // stable parents: decreasing ids
    label[i] = x;
}

// Volume of each component, at its root: sum over its triangles of v0 . (v1 x v2) / 6.
__global__ void k_cc_volume(const int32_t* __restrict__ faces, int64_t nf, const float* __restrict__ verts,
                            const int32_t* __restrict__ label, double* __restrict__ vol) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nf) return;
    const float* a = verts + 3 * (int64_t)faces[3 * t];
    const float* b = verts + 3 * (int64_t)faces[3 * t + 1];
    const float* c = verts + 3 * (int64_t)faces[3 * t + 2];
    const double ax = a[0], ay = a[1], az = a[2], bx = b[0], by = b[1], bz = b[2], cx = c[0], cy = c[1], cz = c[2];
    const double term = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
    atomicAdd(vol + label[faces[3 * t]], term / 6.0);
}

}  // namespace

extern "C" {

// Connected components of a triangle mesh (faces: 3 int32 vertex ids each, < n_verts): d_label[v]
// = the smallest vertex id of v's component (n_verts int32), d_count[0] = number of components
// (isolated vertices count as components), d_comp_volume[r] = signed volume of the component with
// root r (n_verts float64; other entries 0; summed with atomics, so the last bits may depend on
// the order of the additions), d_err[0] = unions that gave up (0).  d_parent: n_verts int32 scratch.
int fb_mesh_components_device(const int32_t* d_faces, int64_t n_faces, const float* d_verts, int64_t n_verts,
                              int32_t* d_parent, int32_t* d_label, double* d_comp_volume, int32_t* d_count,
                              int32_t* d_err, void* stream) noexcept {
    if (n_faces < 0 || n_verts < 0 || n_verts > INT32_MAX || !d_count || !d_err ||
        (n_faces > 0 && (!d_faces || !d_verts)) || (n_verts > 0 && (!d_parent || !d_label || !d_comp_volume)))
        return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    FB_CUDA(cudaMemsetAsync(d_count, 0, 4, st));
    FB_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    if (n_verts == 0) return FB_OK;
    k_cc_init<<<fb_div_up(n_verts, 256), 256, 0, st>>>(d_parent, d_comp_volume, n_verts);
    FB_LAUNCH();
    if (n_faces > 0) {
        k_cc_union<<<fb_div_up(n_faces, 256), 256, 0, st>>>(d_faces, n_faces, d_parent, d_err);
        FB_LAUNCH();
    }
    k_cc_label<<<fb_div_up(n_verts, 256), 256, 0, st>>>(d_parent, n_verts, d_count);
    FB_LAUNCH();
    k_cc_flatten<<<fb_div_up(n_verts, 256), 256, 0, st>>>(d_parent, n_verts, d_label);
    FB_LAUNCH();
    if (n_faces > 0) {
        k_cc_volume<<<fb_div_up(n_faces, 256), 256, 0, st>>>(d_faces, n_faces, d_verts, d_label, d_comp_volume);
        FB_LAUNCH();
    }
    return FB_OK;
}

// Bit words per active block of the edge map (3 B^3 + 3 B^2 slots).
int64_t fb_mc_words(int32_t block) { return block >= 1 && block <= kMcMaxBlock ? mc_words(block) : -1; }

// Scratch int32 words the count pass's scans need for n_active blocks.
int64_t fb_mc_scan_words(int64_t n_active) { return n_active < 0 ? -1 : scan_scratch_words(n_active + 1) + 1; }

// Pass 1 of the export mesh (faltkarna_v1.py:302-350 + marching cubes): the slot map (d_slot,
// n_blocks int32), each active block's edge bits and word prefixes (d_bits, d_wpre: n_active x
// fb_mc_words), and in d_vcount / d_tcount (n_active + 1 int32 each) the exclusive offsets of the
// blocks' vertices and triangles, their totals in the last entry, and the same totals in 64 bits in
// d_totals[0..1] (the int32 offsets are valid while both stay below 2^31; the caller checks them).
// Stream-ordered; block <= 32.  Status 1 for invalid arguments.
int fb_mc_count_device(const int32_t* d_kind, const int32_t* d_active, int64_t n_active, const float* d_tiles,
                       int64_t nx, int64_t ny, int64_t nz, int32_t block, double ox, double oy, double oz,
                       double pitch, double level, float big, int32_t* d_slot, uint32_t* d_bits, int32_t* d_wpre,
                       int32_t* d_vcount, int32_t* d_tcount, int64_t* d_totals, int32_t* d_scan,
                       int64_t scan_words, void* stream) noexcept {
    McField F;
    if (int rc = mc_field(F, d_kind, d_tiles, nx, ny, nz, block, ox, oy, oz, pitch, level, big, d_slot)) return rc;
    if (n_active < 0 || !d_vcount || !d_tcount || !d_scan || !d_totals ||
        (n_active > 0 && (!d_active || !d_tiles || !d_bits || !d_wpre)))
        return FB_INVALID;
    if (scan_words < scan_scratch_words(n_active + 1) + 1) return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nblocks = ((nx + block - 1) / block) * F.nby * F.nbz;
    FB_CUDA(cudaMemsetAsync(d_slot, 0xff, nblocks * 4, st));
    if (n_active > 0) {
        k_mc_slot_map<<<fb_div_up(n_active, 256), 256, 0, st>>>(d_active, n_active, d_slot);
        FB_LAUNCH();
    }
    FB_CUDA(cudaMemsetAsync(d_vcount + n_active, 0, 4, st));
    FB_CUDA(cudaMemsetAsync(d_tcount + n_active, 0, 4, st));
    FB_CUDA(cudaMemsetAsync(d_totals, 0, 16, st));
    if (int rc = mc_launch<false>(F, d_active, n_active, d_bits, d_wpre, d_vcount, d_tcount, nullptr, nullptr,
                                  nullptr, nullptr, nullptr, reinterpret_cast<unsigned long long*>(d_totals), st))
        return rc;
    if (int rc = scan_exclusive(d_vcount, n_active + 1, d_scan, d_scan + 1, scan_words - 1, st)) return rc;
    if (int rc = scan_exclusive(d_tcount, n_active + 1, d_scan, d_scan + 1, scan_words - 1, st)) return rc;
    return FB_OK;
}

// Pass 2: vertices (float32 x, y, z world coordinates, d_vcount[n_active] of them; d_vkey, if not
// null, the vertex's edge as (linear index of its lower end) * 3 + axis), triangles
// (int32 vertex ids, d_tcount[n_active] of them, outward normals) and the enclosed volume
// sum(v0 . (v1 x v2)) / 6 in float64 (d_volume[0]; d_vol_part: n_active float64 scratch), summed in a
// fixed order.  The arguments of pass 1 unchanged.  d_err[0] counts triangle corners without a
// vertex (0 unless the field changed in between).
int fb_mc_emit_device(const int32_t* d_kind, const int32_t* d_active, int64_t n_active, const float* d_tiles,
                      int64_t nx, int64_t ny, int64_t nz, int32_t block, double ox, double oy, double oz, double pitch,
                      double level, float big, const int32_t* d_slot, const uint32_t* d_bits, const int32_t* d_wpre,
                      const int32_t* d_vcount, const int32_t* d_tcount, float* d_verts, int64_t* d_vkey,
                      int32_t* d_faces, double* d_vol_part, double* d_volume, int32_t* d_err, void* stream) noexcept {
    McField F;
    if (int rc = mc_field(F, d_kind, d_tiles, nx, ny, nz, block, ox, oy, oz, pitch, level, big, d_slot)) return rc;
    if (n_active < 0 || !d_vcount || !d_tcount || !d_volume || !d_err ||
        (n_active > 0 && (!d_active || !d_tiles || !d_bits || !d_wpre || !d_vol_part)))
        return FB_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    FB_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    if (int rc = mc_launch<true>(F, d_active, n_active, const_cast<uint32_t*>(d_bits), const_cast<int32_t*>(d_wpre),
                                 const_cast<int32_t*>(d_vcount), const_cast<int32_t*>(d_tcount), d_verts, d_vkey,
                                 d_faces, d_vol_part, d_err, nullptr, st))
        return rc;
    k_mc_volume<<<1, kMcThreads, 0, st>>>(d_vol_part, n_active, d_volume);
    FB_LAUNCH();
    return FB_OK;
}

}  // extern "C"
