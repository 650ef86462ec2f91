/*
 * field_b200.h -- C ABI of libfield_b200.so, the B200-native (sm_100a) block-sparse SDF field path.
 *
 * Conventions (the reference's native contract, src/field_engine/edt_native_v1/edt.cu:18-19 and
 * src/field_engine/csg_batch_native_v1/execute.cpp):
 *   - every entry point is extern "C" and noexcept; integer status: 0 ok, 1 invalid input,
 *     2 runtime / CUDA failure, 3-5 the CSG codes of execute.cpp/gather.cpp, 6 a bounded device
 *     wait gave up (the context stays usable), 7 a grid beyond an allocation-free entry point's
 *     fixed scratch, 8 an output arena too small for the result (what fitted is written);
 *   - arguments are validated before any output is written;
 *   - handles are created and destroyed explicitly; a handle that failed stays failed;
 *   - *_device entry points take device pointers and a cudaStream_t (as void*), enqueue their
 *     kernels on that stream and return without synchronising; they allocate nothing -- the
 *     caller passes scratch sized by the matching *_scratch_bytes function;
 *   - entry points without the _device suffix take host pointers and are synchronous, with the
 *     reference's names and arguments.
 * Paths in citations are relative to the reference project root.
 */
#ifndef FIELD_B200_H
#define FIELD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------ records */

/* Grid of one build: vertex-centred samples at x0 + i*pitch, blocks of block^3 voxels (4, 8 or 16),
 * margin = float32(sqrt(3)*block*pitch), guard = float64-recheck band.
 * Mirrors GridMeta, src/field_engine/faltkarna_v1.py:50-64. */
typedef struct fb_geom {
    double x0, y0, z0, pitch;
    int32_t nx, ny, nz, block;
    float margin, guard;
    int32_t reserved[2]; /* [0] bit 0: the recipe has sampled-grid leaves (type 9), whose voxels at a
                          * table's boundary the leaf and classification passes decide in float64;
                          * other bits and [1]: 0 */
} fb_geom; /* 64 bytes */

/* One primitive: value = s * f(A x + t) - off, f canonical (type 0 sphere, 1 box, 2 cylinder, 3 cone,
 * 4 halfspace, 5 rect_frustum, 6 capsule, 7 torus, 8 unbounded z cylinder).
 * Primitive set of src/field_engine/ikarus_v1/expr.py:93-210 plus capsule/torus. */
typedef struct fb_prim {
    int32_t type, flags;
    double p[12];
    double A[12]; /* rows of the 3x4 world -> canonical map */
    double s, off;
} fb_prim; /* 216 bytes */

/* Program instruction.  Chain form (mode 1): op 0 set, 1 set-negated, 2 union, 3 intersect,
 * 4 subtract, 5 offset; arg = primitive (or -1), k = smooth radius or offset.  Postfix form
 * (mode 0): op 0 push primitive arg, 1 union, 2 intersect, 3 subtract, 4 offset by k.
 * Semantics of src/field_engine/ikarus_v1/expr.py:364-384. */
typedef struct fb_insn {
    int32_t op, arg;
    double k;
} fb_insn; /* 16 bytes */

/* ------------------------------------------------------------------------------------------ runtime */

int fb_abi_version(void);     /* no reference counterpart: ABI version of this library */
int fb_device_arch(void);     /* no reference counterpart: compute capability x10 of the current device */
int fb_sm_count_c(void);      /* no reference counterpart: SM count of the current device */
/* No reference counterpart: float32 FMA throughput probe (roofline denominator); returns its flops. */
int64_t fb_fp32_peak_launch(float* d_out, int blocks, int iters, void* stream);
/* No reference counterpart: stream-ordered copy between raw device or host addresses (synchronises). */
int fb_copy_device(void* dst, const void* src, int64_t bytes, void* stream);

/* ------------------------------------------------------------------------------------------ EDT */

/* Replaces edt_squared, src/field_engine/edt_native_v1/edt.cu:20 (<= 128 per axis, <= 262144 voxels).
 * Squared distance of every voxel to the nearest zero byte of `mask` (host pointers). */
int edt_squared(const uint8_t* mask, int nx, int ny, int nz, int32_t* output);

/* Replaces edt_squared_large, src/field_engine/edt_native_large_v1/edt.cu:33 (<= 512 per axis; the
 * reference's 2^20-voxel cap is lifted to 512^3). */
int edt_squared_large(const uint8_t* mask, int nx, int ny, int nz, int32_t* output);

/* Replace edt_pair_create / edt_pair_query / edt_pair_destroy,
 * src/field_engine/edt_persistent_pair_v1/edt.cu:45-79 (persistent device buffers; signed float32
 * distance, negative inside `mask`, and optionally both squared transforms, polarity-major). */
void* edt_pair_create(int nx, int ny, int nz);
int edt_pair_query(void* handle, const uint8_t* mask, double pitch, float* output, int32_t* squared);
void edt_pair_destroy(void* handle);

/* Device forms of the same transforms (src/field_engine/edt_persistent_pair_v1/edt.cu:12-42).
 * fb_edt_squared_device: sites are the nonzero bytes when sites_nonzero, else the zero bytes.
 * fb_edt_pair_device: polarity 0 to the nonzero voxels; d_squared (nullable) gets both.
 * fb_edt_validate_device: status 1 when a byte is > 1 or only one class is present (synchronises). */
int64_t fb_edt_scratch_bytes(int nx, int ny, int nz, int paired);
int fb_edt_squared_device(const uint8_t* d_mask, int nx, int ny, int nz, int sites_nonzero, int32_t* d_out,
                          void* d_scratch, int64_t scratch_len, void* stream);
int fb_edt_pair_device(const uint8_t* d_mask, int nx, int ny, int nz, double pitch, float* d_signed,
                       int32_t* d_squared, void* d_scratch, int64_t scratch_len, void* stream);
int fb_edt_validate_device(const uint8_t* d_mask, int nx, int ny, int nz, void* d_scratch, int64_t scratch_len,
                           void* stream);

/* No counterpart in the reference.  For callers that cannot allocate device memory (hosts that own
 * every device byte through their own allocator, loops that must never meet cudaMalloc's implicit
 * synchronisation): fb_edt_squared_device without caller scratch -- the scratch is a fixed
 * ~5.1 MiB device array inside this library, so grids are limited to 2^20 voxels and 512 per axis
 * (status 7 for an axis above 512 or more than 2^20 voxels; status 1 for a null pointer or an axis
 * below 1).  The first call on a device (and again after a device reset, which maps the array at a
 * new address) resolves the array's address and should come before any stream capture; calls that
 * overlap on the GPU share the array and race.
 * fb_edt_noalloc_capacity returns the array's size and writes the voxel limit. */
int fb_edt_squared_device_noalloc(const uint8_t* d_mask, int nx, int ny, int nz, int sites_nonzero,
                                  int32_t* d_out, void* stream);
int64_t fb_edt_noalloc_capacity(int64_t* max_voxels);

/* ------------------------------------------------------------------------------------------ field build */

/* Replace the Warp kernels behind klassificera_och_evaluera_testfalt, src/field_engine/faltkarna_v1.py:
 * k_classify_testfalt :129-164, host compaction np.where :277, k_eval_tile_testfalt :167-190 -- for any
 * compiled recipe.  mode 1: d_chain is the culled chain form; mode 0: a postfix program (float64).
 * Outputs: kind[n_blocks] (-1/0/+1), corner_min_abs[n_blocks], ascending active ids, count[0],
 * tiles[count][block^3] (C order li, lj, lk).  fb_field_leaf_device reuses the lists that
 * fb_field_classify_device left in d_scratch for the same recipe and grid. */
int64_t fb_field_scratch_bytes(const fb_geom* g, int32_t n_prims, int32_t n_chain);
int fb_field_classify_device(const fb_geom* g, const fb_prim* d_prims, int32_t n_prims, const fb_insn* d_chain,
                             int32_t n_chain, int32_t mode, int32_t* d_kind, float* d_cma, int32_t* d_active,
                             int32_t* d_count, void* d_scratch, int64_t scratch_len, void* stream);
int fb_field_leaf_device(const fb_geom* g, const fb_prim* d_prims, int32_t n_prims, const fb_insn* d_chain,
                         int32_t n_chain, int32_t mode, const int32_t* d_kind, const int32_t* d_active,
                         const int32_t* d_count, float* d_tiles, int64_t capacity, void* d_scratch,
                         int64_t scratch_len, void* stream);
int fb_field_leaf_work_device(const fb_geom* g, const fb_prim* d_prims, int32_t n_prims, const fb_insn* d_chain,
                              int32_t n_chain, int32_t mode, const int32_t* d_kind, const int32_t* d_active,
                              const int32_t* d_count, float* d_tiles, int64_t capacity, void* d_scratch,
                              int64_t scratch_len, uint64_t* d_work, void* stream);
int fb_field_build_device(const fb_geom* g, const fb_prim* d_prims, int32_t n_prims, const fb_insn* d_chain,
                          int32_t n_chain, int32_t mode, int32_t* d_kind, float* d_cma, int32_t* d_active,
                          int32_t* d_count, float* d_tiles, int64_t capacity, void* d_scratch,
                          int64_t scratch_len, void* stream);
/* Status 6 when the last compaction's bounded look-back wait gave up (synchronises). */
int fb_field_compact_error(const fb_geom* g, int32_t n_prims, int32_t n_chain, const void* d_scratch, void* stream);
/* Batched builds of many chain recipes, replacing the reference's recipe-by-recipe orchestration
 * (src/field_engine/faltkarna_v1_g7_fix.py:56-112: classify, host read of the kinds, compaction, tile
 * evaluation, per part).  Every phase is one launch over a device work-list spanning all recipes;
 * the active counts, each recipe's place in the tile arena and the active-block work-lists are
 * formed on the device, so a build has no host synchronisation and allocates nothing (CUDA-graph
 * capturable).  Each item carries the buffers of one fb_field_build_device call (chain form, mode 1);
 * they must outlive the batch.  fb_batch_create synchronises its stream and returns NULL on invalid
 * input.  fb_batch_build_device writes recipe r's tiles at d_tiles + tile_off[r] (floats, recipe
 * order), leaf_count[r] of its active blocks (all of them unless the arena of `capacity` floats ran
 * out: fb_batch_status then returns 8; 6 when a compaction wait gave up); ctas_per_sm (0 = 16) sizes
 * the active-block passes.  fb_batch_outputs gives the device arrays tile_off[n] (int64) and
 * leaf_count[n] (int32); fb_batch_launches the launches one build enqueues. */
typedef struct fb_batch_item {
    const fb_geom* geom;
    const fb_prim* d_prims;
    const fb_insn* d_chain;
    int32_t n_prims, n_chain;
    int32_t* d_kind;
    float* d_cma;
    int32_t* d_active;
    int32_t* d_count;
    void* d_scratch;
    int64_t scratch_len;
    int32_t* d_slot;  /* nullable; with d_mask (16-byte aligned, nx*ny*nz bytes) the recipe takes part */
    uint8_t* d_mask;  /* in fb_batch_occupancy_device; d_slot holds n_blocks int32 */
} fb_batch_item; /* 96 bytes */
void* fb_batch_create(const fb_batch_item* items, int32_t n, void* stream);
int fb_batch_build_device(void* batch, float* d_tiles, int64_t capacity, int32_t ctas_per_sm, void* stream);
/* No reference counterpart: the same build, recording events[0..5] (nullable cudaEvent_t) at its
 * start and after culling, classification (with the active blocks' lists), compaction, an empty
 * phase, and leaves, and adding the
 * leaf pass's executed primitive evaluations and float32 operations to d_work[0..1] (nullable). */
int fb_batch_build_timed_device(void* batch, float* d_tiles, int64_t capacity, int32_t ctas_per_sm,
                                void* const* events, uint64_t* d_work, void* stream);
int fb_batch_outputs(void* batch, const int64_t** tile_off, const int32_t** leaf_count);
/* Occupancy masks (1 where the field is negative) of the items that carry d_slot / d_mask, from the
 * last build's tiles; stream-ordered after it (the reference rasterises occupancy on the host). */
int fb_batch_occupancy_device(void* batch, const float* d_tiles, void* stream);
int32_t fb_batch_launches(void* batch);
int fb_batch_status(void* batch, void* stream);
void fb_batch_destroy(void* batch);

/* No counterpart in the reference (the reference compacts on the host).  Test of the bounded wait in
 * the compaction's look-back: runs the compaction kernel over n kinds with tile 0's status never
 * published and a wait limit of spin_limit sleeps; returns 6 when the wait gave up and raised the
 * error flag, as the product path reports it.  d_scratch: fb_dense_scratch_bytes(n, 1, 1, 1) bytes;
 * n > 2048.  The active ids it writes are not meaningful. */
int fb_compact_timeout_probe(const int32_t* d_kind, int64_t n, int32_t* d_active, int32_t* d_count,
                             void* d_scratch, int64_t scratch_len, int64_t spin_limit, void* stream);

/* No counterpart in the reference.  Self-test of the square root the float32 leaf and corner
 * evaluations use (a Newton step from the approximate reciprocal square root): d_out[i] = that root
 * of d_x[i] for n device floats, stream-ordered.  Inputs are sums of squares (>= 0, or NaN). */
int fb_sqrt_sum_probe(const float* d_x, float* d_out, int64_t n, void* stream);
/* No counterpart in the reference.  Self-test of the quotient the 8^3 leaf tiles use for the sphere's
 * difference form (a Newton step from the approximate reciprocal): d_out[i] = d_num[i] / d_den[i] for
 * n device floats, d_den[i] > 0, stream-ordered. */
int fb_quotient_probe(const float* d_num, const float* d_den, float* d_out, int64_t n, void* stream);

/* Replace meshsdf_classify_cpu / meshsdf_tiles_cpu, src/field_engine/mesh_sdf_native_v1/field.cpp:229,254,
 * and k_classify_dense / k_eval_tile_dense, src/field_engine/faltkarna_v1_mesh_to_sdf.py:602-657. */
int64_t fb_dense_scratch_bytes(int64_t nx, int64_t ny, int64_t nz, int32_t block);
int fb_dense_classify_device(const float* d_dense, int64_t nx, int64_t ny, int64_t nz, int32_t block, float margin,
                             int32_t* d_kind, float* d_cma, int32_t* d_active, int32_t* d_count, float* d_tiles,
                             int64_t capacity, void* d_scratch, int64_t scratch_len, void* stream);

/* Replaces rekonstruera_tat_gpu (k_fill_background + k_scatter_tiles), src/field_engine/faltkarna_v1.py:193-236,328-350;
 * output cropped to (nx, ny, nz).  d_slot: caller scratch of n_blocks int32. */
int fb_field_reconstruct_device(const int32_t* d_kind, const int32_t* d_active, int64_t n_active,
                                const float* d_tiles, int64_t nx, int64_t ny, int64_t nz, int32_t block, float big,
                                int32_t* d_slot, float* d_out, void* stream);

/* Replaces the solid reconstruction of src/field_engine/faltkarna_v1_mesh_to_sdf.py:695-713
 * (reconstruct_solid_from_sparse) on device-resident fields: uint8 mask, 1 where the field is
 * negative; reads the active count on the device (no synchronisation).  d_slot: n_blocks int32.
 * block is 4, 8 or 16; d_tiles and d_mask are 16-byte aligned (status 1 otherwise). */
int fb_field_occupancy_device(const int32_t* d_kind, const int32_t* d_active, const int32_t* d_count,
                              const float* d_tiles, int64_t capacity, int64_t nx, int64_t ny, int64_t nz,
                              int32_t block, int32_t* d_slot, uint8_t* d_mask, void* stream);

/* Replaces k_reduce_checksum_i64_safe, src/field_engine/faltkarna_v1.py:250-255 (accumulates into d_out[0]). */
int fb_checksum_i64_device(const float* d_values, int64_t n, double scale, int64_t* d_out, void* stream);
/* Exact sum of n int32 values into d_out[0] (zeroed first, stream-ordered); the served EDT
 * request's result summary.  No counterpart in the reference, which sums on the host. */
int fb_sum_i32_device(const int32_t* d_values, int64_t n, int64_t* d_out, void* stream);

/* Packed adaptive block tree (the reference's AdaptiveBlocks, src/field_engine/field_adaptive_blocks_v1.py):
 * build(), :113-147, one level at a time, each node classified from the dense field by the rule of
 * fb_dense_classify_device at its side, then packing and rank checkpoints; sample(), :53-82.
 * fb_tree_codes_device: codes of one level's n nodes and the exclusive rank of its ranked code
 * (2 at sides 8/4/2, 3 at side 1), the level total in *d_total; d_coords = NULL for the root level
 * (rx x ry x rz root blocks in C order).  fb_tree_expand_device: 8 child corners per branch at
 * 8 * rank + child.  fb_tree_values_device: dense samples of the side-1 value leaves by rank.
 * fb_tree_pack_device: 2-bit codes four per byte (d_packed 4-byte aligned, sized to a multiple of
 * 4 bytes) and the checkpoints every 64 bytes (floor(bytes / 64) + 1 entries each).
 * fb_tree_rank_words_device: the sampler's per-word rank tables (nodes of code 2 / 3 before each
 * 16-node word; not part of the stored format).  fb_tree_sample_device: values at int64 grid
 * indices [n][3], ranking from those tables when given (else from the checkpoints); *d_status OR-ed
 * with 1 (index outside the grid), 2 (branch below side 1), 4 (rank outside the arrays), those
 * outputs NaN. */
int64_t fb_tree_scan_bytes(int64_t n);
int fb_tree_codes_device(const float* d_dense, int64_t nx, int64_t ny, int64_t nz, int32_t side, float margin,
                         const int32_t* d_coords, int64_t rx, int64_t ry, int64_t rz, int64_t n, uint8_t* d_codes,
                         int32_t* d_rank, int32_t* d_total, void* d_scratch, int64_t scratch_len, void* stream);
int fb_tree_expand_device(const uint8_t* d_codes, const int32_t* d_rank, const int32_t* d_coords, int64_t rx,
                          int64_t ry, int64_t rz, int64_t n, int32_t side, int32_t* d_child, void* stream);
int fb_tree_values_device(const float* d_dense, int64_t nx, int64_t ny, int64_t nz, const uint8_t* d_codes,
                          const int32_t* d_rank, const int32_t* d_coords, int64_t n, float* d_values, void* stream);
int64_t fb_tree_pack_scratch_bytes(int64_t node_count);
int fb_tree_pack_device(const uint8_t* d_codes, int64_t node_count, uint8_t* d_packed, int32_t* d_branch_prefix,
                        int32_t* d_value_prefix, void* d_scratch, int64_t scratch_len, void* stream);
int64_t fb_tree_rank_words_scratch_bytes(int64_t node_count);
int fb_tree_rank_words_device(const uint8_t* d_packed, int64_t node_count, int32_t* d_branch_words,
                              int32_t* d_value_words, void* d_scratch, int64_t scratch_len, void* stream);
int fb_tree_sample_device(const uint8_t* d_packed, int64_t node_count, const int32_t* d_branch_prefix,
                          const int32_t* d_value_prefix, const int32_t* d_branch_words, const int32_t* d_value_words,
                          const float* d_values, int64_t n_values, int64_t root_count,
                          int64_t r0, int64_t r1, int64_t r2, int64_t nx, int64_t ny, int64_t nz, double pitch,
                          const int64_t* d_ijk, int64_t n, float* d_out, int32_t* d_status, void* stream);

/* ------------------------------------------------------------------------------------------ packed fields */

/* Replace adaptive_pack / adaptive_nodes / adaptive_samples / adaptive_copy / adaptive_free,
 * src/field_engine/adaptive_pack_native_v1/pack.cpp:57-79: host float32 samples, int32 shape[3],
 * threshold 8..4096; NULL on invalid input; 52-byte nodes and float32 payload with the reference's
 * split decisions and order.  fb_pack_device takes device samples (synchronises the stream);
 * fb_pack_payload_device returns the handle's device payload. */
void* adaptive_pack(const void* data, const int32_t* shape, int threshold);
void* fb_pack_device(const float* d_data, const int32_t* shape, int threshold, void* stream);
int64_t adaptive_nodes(const void* handle);
int64_t adaptive_samples(const void* handle);
int adaptive_copy(const void* handle, void* nodes, int64_t count, void* payload, int64_t samples);
void adaptive_free(void* handle);
const float* fb_pack_payload_device(const void* handle);

/* Replaces csg_execute, src/field_engine/csg_batch_native_v1/execute.cpp:10-53 (24-byte instructions
 * {op, left, right, pad, offset}; statuses 1-5; the output is written only on success). */
int csg_execute(const void* const* nodes, const int64_t* counts, const void* const* payload, const int64_t* lengths,
                int32_t fields, const int32_t* shape, const void* program, int32_t instructions, float* output);

/* Replace AdaptiveSampleBlocks.samples_at / query, src/field_engine/adaptive_sample_blocks_v1.py:182-230. */
int fb_packed_samples_at(const void* nodes, int64_t count, const float* payload, int64_t samples,
                         const int64_t* indices, int64_t n, float* out);
int fb_packed_query_device(const void* d_nodes, const float* d_payload, const int32_t* shape, const double* origin,
                           double pitch, const double* d_points, int64_t n, float* d_out, void* stream);

/* ------------------------------------------------------------------------------------------ point queries */

/* Replaces _lagg_overlappsband, src/field_engine/faltkarna_v1_multires.py:211-251: every fine brick's
 * faces that meet an active coarser brick take the trilinear sample (scipy map_coordinates order 1,
 * mode nearest) of that brick's lattice, in the reference's brick and face order.  d_orig: scratch of
 * pool_len floats; d_bricks: active bricks of level >= 1 sorted by level and id, n_of_level[1..3]
 * of each level (n_of_level[0] unused); d_faces: faces written.  Stream-ordered. */
int fb_multires_band_device(const double* lo, double h, int32_t B, const int32_t* bshape, const int8_t* d_kind,
                            const int8_t* d_level, const int64_t* d_tile_off, float* d_pool, int64_t pool_len,
                            float* d_orig, const int32_t* d_bricks, const int32_t* n_of_level, int32_t* d_faces,
                            void* stream);

/* Replaces eval_batch_multi_pair, src/field_engine/ikarus_v1/eval_warp.py:545-564: max(sample(A),
 * sample(B)) per point, A / B the gridfield leaves of the point's pair, every pair in one launch.
 * d_params: 12 float32 per leaf (origin xyz, pitch, iso, is_sdf, nx, ny, nz, unused, the table's
 * device address as two 32-bit halves); an out-of-range pair or leaf index reads NaN. */
int fb_grid_pairs_device(const float* d_params, int32_t n_leaves, const float* d_pts, const int32_t* d_pair,
                         int64_t n, const int32_t* d_leaf_a, const int32_t* d_leaf_b, int32_t n_pairs, float* d_out,
                         void* stream);

/* Replace eval_batch / gradient_batch, src/field_engine/ikarus_v1/eval_warp.py:478-488,718-733.
 * fb_query_prepare fills the 128-byte float32 primitive mirror; fb_field_accel exposes a
 * classification's culling lists inside its scratch (superblock and per-block) so that points
 * inside that grid walk only their block's list (where the classification kept one; blk_all = 1:
 * every block, else blocks of kind 0) or their superblock's list. */
int fb_query_prepare(const fb_prim* d_prims, int32_t n_prims, void* d_primf, void* stream);
int fb_field_accel(const fb_geom* g, int32_t n_prims, int32_t n_chain, const void* d_scratch, const void** pool,
                   const int64_t** sb_off, const int32_t** sb_len, const int32_t** blk_off, const int32_t** blk_len,
                   const uint32_t** blk_pool, int64_t* blk_cap, int32_t* blk_all);
int fb_query_points_device(const void* d_primf, const fb_insn* d_chain, int32_t n_chain, int32_t mode,
                           const void* accel_pool, const int64_t* accel_off, const int32_t* accel_len,
                           const double* accel_grid, const int32_t* accel_dims, const int32_t* d_kind,
                           const int32_t* blk_off, const int32_t* blk_len, const uint32_t* blk_pool, int64_t blk_cap,
                           int32_t blk_all, const float* d_points, int64_t n, double h, float* d_value, float* d_grad,
                           void* d_scratch, int64_t scratch_len, void* stream);
/* Scratch of the sorted query path (evaluation points sorted by the culled list they walk, so a
 * warp's lanes share one list); -1 when the grid takes the unsorted path.  No reference
 * counterpart: an execution strategy of fb_query_points_device, same results bit for bit. */
int64_t fb_query_scratch_bytes(const int32_t* accel_dims, int64_t n, int32_t with_grad);

/* Replace the per-block-pitch field's lattices and its avstand / gradient queries,
 * src/field_engine/faltkarna_v1_multires.py:84-104,384-459 (lattices built from a recipe). */
int fb_multires_tiles_device(const void* d_primf, const fb_insn* d_chain, int32_t n_chain, int32_t mode,
                             const fb_prim* d_prims, const double* lo, double h, int32_t B, const int32_t* bshape,
                             const int32_t* d_bricks, const int8_t* d_levels, const int64_t* d_offsets,
                             int64_t nbricks, const int32_t* d_blk_off, const int32_t* d_blk_len,
                             const uint32_t* d_blk_pool, float guard, float* d_pool, void* stream);
int fb_multires_query_device(const double* lo, double h, int32_t B, const int32_t* bshape, double margin,
                             const int8_t* d_kind, const int8_t* d_level, const int64_t* d_tile_off,
                             const float* d_pool, const double* d_points, int64_t n, double* d_value, double* d_grad,
                             void* stream);

/* Replaces meshsdf_field_cpu, src/field_engine/mesh_sdf_native_v1/field.cpp:19-226 (same arguments and
 * statuses: 1 contract, 2 face index outside [0, nv), 3 more than 2^31 - 2 ray hits); computed on the
 * current GPU, host pointers; window axes up to 512 (the EDT's contract); nthreads ignored; tstage[5]
 * = seconds of the hits, grouping, winding, EDT and finishing stages. */
int meshsdf_field_cpu(const double* V, int64_t nv, const int64_t* T, int64_t nt, double ox, double oy, double oz,
                      double pitch, double jx, double jy, int64_t nx, int64_t ny, int64_t nz, int ytkorr,
                      int nthreads, uint8_t* solid, float* sd, uint8_t* yta, int64_t* stats, double* tstage);

/* Export step: the isosurface of a resident sparse field straight from its tiles -- the mesh that
 * marching cubes gives on the dense reconstruction, replacing rekonstruera_tat(_gpu) followed by
 * skimage.measure.marching_cubes (src/field_engine/faltkarna_v1.py:302-350) and the enclosed
 * volume of faltvolym_v1.py:83-104.  Pass 1 (count) then pass 2 (emit) with the same arguments;
 * block <= 32.  d_bits / d_wpre: n_active x fb_mc_words(block) words; d_vcount / d_tcount:
 * n_active + 1 int32 (block offsets, totals last); d_totals: 2 int64 (vertex and triangle totals,
 * valid as int32 offsets below 2^31); d_scan: fb_mc_scan_words(n_active) int32. */
int64_t fb_mc_words(int32_t block);
int64_t fb_mc_scan_words(int64_t n_active);
int fb_mc_count_device(const int32_t* d_kind, const int32_t* d_active, int64_t n_active, const float* d_tiles,
                       int64_t nx, int64_t ny, int64_t nz, int32_t block, double ox, double oy, double oz,
                       double pitch, double level, float big, int32_t* d_slot, uint32_t* d_bits, int32_t* d_wpre,
                       int32_t* d_vcount, int32_t* d_tcount, int64_t* d_totals, int32_t* d_scan,
                       int64_t scan_words, void* stream);
/* d_verts: 3 float32 per vertex (world coordinates); d_vkey (optional): per vertex
 * (linear index of the edge's lower end) * 3 + axis; d_faces: 3 int32 per triangle, outward normals;
 * d_volume[0]: sum(v0 . (v1 x v2)) / 6 (d_vol_part: n_active float64 scratch); d_err[0]: triangle
 * corners without a vertex (0 unless the field changed between the passes). */
int fb_mc_emit_device(const int32_t* d_kind, const int32_t* d_active, int64_t n_active, const float* d_tiles,
                      int64_t nx, int64_t ny, int64_t nz, int32_t block, double ox, double oy, double oz, double pitch,
                      double level, float big, const int32_t* d_slot, const uint32_t* d_bits, const int32_t* d_wpre,
                      const int32_t* d_vcount, const int32_t* d_tcount, float* d_verts, int64_t* d_vkey,
                      int32_t* d_faces, double* d_vol_part, double* d_volume, int32_t* d_err, void* stream);

/* Connected components of a triangle mesh (the component split of faltvolym_v1.py:95-101):
 * d_label[v] = smallest vertex id of v's component, d_count[0] = components, d_comp_volume[root] =
 * the component's signed volume (atomically summed: last bits order-dependent), d_err[0] = unions
 * that gave up.  d_parent / d_label: n_verts int32, d_comp_volume: n_verts float64. */
int fb_mesh_components_device(const int32_t* d_faces, int64_t n_faces, const float* d_verts, int64_t n_verts,
                              int32_t* d_parent, int32_t* d_label, double* d_comp_volume, int32_t* d_count,
                              int32_t* d_err, void* stream);

/* ------------------------------------------------------------------------------------------ EDT consumers */

/* Clearance in millimetres, float64(sqrt(sq)) * pitch: replaces `distance_transform_edt(~occ) * pitch_mm`
 * of src/field_engine/opt/laplaceflode_v1.py:313-314 and opt/f33_1_topologi_v1.py:205-206, fed by
 * fb_edt_squared_device with sites_nonzero = 1 on the occupancy. */
int fb_edt_mm_device(const int32_t* d_sq, int64_t n, double pitch, double* d_out, void* stream);
/* d_valid[i] = !occ[i] && edt_mm[i] >= threshold (threshold = min_r + margin, formed by the caller in
 * float64): replaces `free & (edt_mm >= min_r_mm + margin_mm)`, opt/f33_1_topologi_v1.py:207-208. */
int fb_clearance_mask_device(const uint8_t* d_occ, const double* d_edt_mm, int64_t n, double threshold,
                             uint8_t* d_valid, void* stream);
/* The free space of an occupancy grid as a resistor network, replacing bygg_gitterlaplacian,
 * src/field_engine/opt/laplaceflode_v1.py:69-97.  Two calls on one stream with the same scratch:
 * fb_lattice_count_device writes d_totals = {nodes, edges, CSR entries} (int32, device); the caller
 * sizes the outputs from them and fb_lattice_emit_device writes the node map (nx*ny*nz int32, -1 on
 * occupied cells), the edges u, v, kond (axis 0, 1, 2; lower cell ascending; kond = max(0.5 (E_u +
 * E_v) / pitch, 0.1)^p_kond) and the CSR Laplacian (indptr[nodes + 1], indices and data[entries]:
 * columns ascending, -kond off the diagonal, the diagonal summed in scipy's COO order).  The
 * capacities are the lengths of the caller's u / v / kond (edges), indptr (nodes + 1) and indices /
 * data (entries) buffers: outputs beyond them are not written, and a null pointer is accepted only
 * where its capacity is 0.  At most (2^31 - 1) / 7 cells (status 1 beyond);
 * fb_lattice_scratch_bytes returns -1 for such shapes. */
int64_t fb_lattice_scratch_bytes(int nx, int ny, int nz);
int fb_lattice_count_device(const uint8_t* d_occ, int nx, int ny, int nz, int32_t* d_totals, void* d_scratch,
                            int64_t scratch_len, void* stream);
int fb_lattice_emit_device(const uint8_t* d_occ, const double* d_edt_mm, int nx, int ny, int nz, double pitch,
                           double p_kond, int32_t* d_node_map, int32_t* d_u, int32_t* d_v, double* d_kond,
                           int64_t edge_cap, int32_t* d_indptr, int64_t indptr_cap, int32_t* d_indices,
                           double* d_data, int64_t entry_cap, const void* d_scratch, int64_t scratch_len,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FIELD_B200_H */
