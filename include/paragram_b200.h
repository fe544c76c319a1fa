/*
 * paragram_b200.h -- C ABI of the B200 diagram builder (libparagram_b200.so).
 *
 * Drop-in boundary for the reference's pybind entry points
 *   laguerre::build_voronoi_ultra            (paragram/csrc/laguerre/laguerre.h:24-29,
 *                                             bound at paragram/csrc/ext.cpp:21-29)
 *   laguerre::build_laguerre_voronoi_ultra   (paragram/csrc/laguerre/laguerre.h:13-20,
 *                                             bound at paragram/csrc/ext.cpp:10-19)
 * which take CUDA tensors and return (adjacency, offsets, status). A C ABI
 * cannot return tensors whose size is data dependent, so one reference call
 * is split into plain-pointer steps:
 *
 *   pg_workspace_size(N, &bytes)          -> caller allocates `bytes` of device memory
 *   pg_build(..., offsets, status, &E)    -> fills offsets [N+1] and status [N],
 *                                            returns the adjacency length E
 *                                            (the reference's cudaMemcpy of the total,
 *                                            voronoi_ultra.cu:352-354)
 *   pg_emit_adjacency(..., adjacency)     -> caller allocates E int32, this fills it
 *
 * All pointers except `options` are device pointers. Every call is ordered on
 * `stream` (a cudaStream_t, NULL = legacy default stream); pg_build
 * synchronises the stream once to read E back, like the reference.
 * Outputs match the reference's Diagram: int32 CSR adjacency (rows sorted),
 * int32 offsets of shape (N+1,), int32 per-point status
 * (0 success, 1 plane_overflow, 2 vertex_overflow, 3 empty_cell,
 * 4 security_radius_not_reached, 5 inconsistent_boundary;
 * faster_convex_cell.cuh:99-108).
 *
 * Return codes: 0 on success, negative on error; pg_last_error() describes the
 * last error of the calling thread. PG_ERR_INVALID corresponds to the
 * reference's argument ASSERTs (std::runtime_error, voronoi_ultra.cu:20-24).
 */
#ifndef PARAGRAM_B200_H
#define PARAGRAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_OK 0
#define PG_ERR_INVALID (-1)   /* bad argument (reference: ASSERT -> std::runtime_error) */
#define PG_ERR_CUDA (-2)      /* CUDA runtime error (reference: cuda_check, cuda_helpers.h:79-102) */
#define PG_ERR_INTERNAL (-3)  /* internal capacity exceeded */

/* Options of one build. Mirrors the keyword arguments of the reference
 * (paragram/_api.py:65-123; defaults at paragram/csrc/ext.cpp:14-19). */
typedef struct pg_options
{
    int32_t knn;        /* reference: kNN(knn) warm start (voronoi_ultra.cu:205-227). Accepted for
                           compatibility: the best-first BVH traversal visits the seed's own leaf first,
                           which serves as the warm start. Results never depend on it. */
    int32_t leaf_size;  /* reference: BVH leaf threshold, -1 = default (voronoi_ultra.cu:175-177).
                           Here <= 0 selects 16; at most 32. Results do not depend on it. */
    int32_t debug;      /* reference: print phase timings (voronoi_ultra.cu:196-219). Bit 0 prints them,
                           bit 1 only records them for pg_last_profile. */
    int32_t num_chunks; /* reference: PARAGRAM_NUM_CHUNKS / PARAGRAM_MEM_FRAC chunk plan
                           (chunking.h:16-56). 0 = read the environment; > 0 = split the cell
                           pass into this many launches. Results do not depend on it. */
    int32_t blocks_per_sm; /* register budget of the cell kernel: resident blocks of 8 warps per SM
                              (2 or 3; 0 = default 2). No reference counterpart; chosen by the
                              autotuner. Results do not depend on it. */
    int32_t predicates;    /* 0 (default): FP32 side tests behind a rigorous error filter, undecided ones
                              re-evaluated in FP64 and exact expansions (exact results). 1: FP32 side
                              tests only, undecided ones taken by the sign of the FP32 value, as the
                              reference's FP32 clipping: no escalation, results may differ from the
                              exact diagram on near-degenerate inputs. */
    const void *model;     /* learned search radius: device pointer to a pg_model, or NULL for the
                              plain traversal. No reference counterpart. Results do not depend on it. */
    const float *radius_hint; /* device float32 [num_points] or NULL: a search radius per point (for
                              instance the radius_out of a previous build of slightly moved points).
                              Used like the model's prediction; ignored when model is set. Results
                              do not depend on it. */
    float *radius_out;     /* device float32 [num_points] or NULL: per point, the certified radius of its
                              final cell (max distance of a vertex from the point, power-adjusted;
                              0 for an empty cell). Training targets of the learned radius. */
    int32_t *work_out;     /* device int32 [4 * num_points] or NULL: per point, BVH nodes visited, leaves
                              visited, candidates tested and the peak length of the node queue. */
    float *features_out;   /* device float32 [16 * num_points] or NULL: per point, the 16 features of
                              the learned search radius (training inputs; pg_model below). */
    int32_t *order_out;    /* device int32 [num_points] or NULL: the points' curve order (sorted slot
                              -> point index) used by the BVH and by the features' windows. */
    float *geometry_out;   /* device float32 [4 * num_points], 16-byte aligned, or NULL: per point, the
                              centroid (x, y, z) and the volume of its cell (the geometry the reference
                              computes and discards, voronoi_ultra.cu:125-138). An empty cell gives
                              volume 0 and a NaN centroid; a plane_overflow cell NaN. */
    /* Vertex export (no reference counterpart; the reference keeps its vertices in per-thread
     * scratch and discards them, voronoi_ultra.cu:125-138). Added in version 200: a caller must
     * check pg_version() >= 200 before passing a pg_options with these fields, since an older
     * library reads the shorter struct. */
    int32_t vertex_cap;    /* vertices per cell that vertices_out / vertex_planes_out hold (0: none) */
    float *vertices_out;   /* device float32 [num_points * vertex_cap * 4], 16-byte aligned, or NULL: per
                              cell, its vertices relative to the cell's point (x, y, z) and w, a
                              rigorous bound on the distance from (x, y, z) to the exact vertex (the
                              error radius of the FP32 side tests) */
    int32_t *vertex_planes_out; /* device int32 [num_points * vertex_cap * 3] or NULL: the three planes
                              meeting at each vertex: the neighbour's point index for a bisector, or
                              -1 - code for a face of the box (code = 2 * axis + 1 on the high side) */
    int32_t *vertex_count_out; /* device int32 [num_points] or NULL: the number of vertices of each cell
                              (0 for an empty cell); vertices beyond vertex_cap are counted, not written */
} pg_options;

/* Learned search radius (no reference counterpart). A 16 -> 64 -> 64 -> 2 MLP
 * with BF16 weights: features of a point (its curve-order window, see
 * features_out) -> (log of its cell's certified radius relative to the
 * window's mean neighbour distance, neighbour count / 16), both normalised as
 * (t - target_mean) * target_scale. A build given a model predicts every
 * point's radius (times exp(radius_margin)) and caps its first traversal pass
 * with it; the cap is kept only when the final radius is within it, so the
 * diagram never depends on the model. Device memory, pg_mlp_model_bytes()
 * bytes, magic = PG_MODEL_MAGIC, w3 rows 2..7 zero. */
#define PG_MODEL_MAGIC 0x314D4750u /* "PGM1" */
typedef struct pg_model
{
    uint32_t magic;
    uint32_t num_features; /* 16 */
    uint32_t hidden;       /* 64 */
    uint32_t reserved;
    float feat_mean[16];   /* inputs are (x - feat_mean) * feat_scale, rounded to BF16 */
    float feat_scale[16];
    float target_mean[2];
    float target_scale[2];
    float radius_margin;   /* added to the predicted log radius */
    float route_degree;    /* > 0: a point whose predicted neighbour count is at least this skips the
                              first pass (64 vertex slots) and is built by the 128-slot tier directly;
                              0: off. The diagram does not depend on it. */
    float pad[2];
    float b1[64];
    float b2[64];
    float b3[8];           /* entries 2..7 unused */
    uint16_t w1[64 * 16];  /* BF16 bits, [out][in] */
    uint16_t w2[64 * 64];
    uint16_t w3[8 * 64];   /* rows 2..7 zero */
} pg_model;

/* Library version (major * 10000 + minor * 100 + patch). */
int pg_version(void);

/* Message of the last error returned on this thread ("" if none). */
const char *pg_last_error(void);

/* Device workspace needed for num_points points (any weights / options).
 * Replaces the reference's internal torch / cudaMalloc allocations
 * (voronoi_ultra.cu:186, 207, 230-232, 267-268, 319-324; pwr_bvh.cu:228-269). */
int pg_workspace_size(int64_t num_points, size_t *bytes);

/* Build the diagram. Replaces build_voronoi_ultra (weights == NULL) and
 * build_laguerre_voronoi_ultra (weights != NULL), laguerre.h:13-29.
 *   points      float32 [num_points * 3], xyz interleaved (contiguous (N, 3) tensor)
 *   weights     float32 [num_points] or NULL
 *   initial_guesses / initial_guesses_offsets
 *               int32 CSR of candidate neighbours per point (original ids), or both NULL
 *               (reference: voronoi_ultra.cu:69-85). Results do not depend on them.
 *   options     host pointer or NULL (defaults: knn 8, leaf_size -1, debug 0, num_chunks 0, blocks_per_sm 0,
 *               no model, no per-point diagnostics)
 *   workspace   device buffer of at least pg_workspace_size() bytes, 256-byte aligned;
 *               it must stay alive until pg_emit_adjacency returns
 *   offsets     int32 [num_points + 1]  (output)
 *   status      int32 [num_points]      (output)
 *   num_edges   host int64              (output) = offsets[num_points]
 */
int pg_build(int64_t num_points, const float *points, const float *weights, const int32_t *initial_guesses,
             const int32_t *initial_guesses_offsets, const pg_options *options, void *workspace,
             size_t workspace_bytes, int32_t *offsets, int32_t *status, int64_t *num_edges, void *stream);

/* Write the adjacency (int32 [num_edges]) of the last pg_build on this
 * workspace. Replaces populate_symmetric_adjacency (adjacency.cuh:120-159). */
int pg_emit_adjacency(int64_t num_points, const void *workspace, const int32_t *offsets, int32_t *adjacency,
                      void *stream);

/* Counters of the last pg_build on this workspace (synchronises the stream):
 * out[0] FP32 side tests, out[1] tests escalated to FP64, out[2] tests escalated
 * to exact expansions, out[3] deferrals to a larger tier (128 slots, then 256), out[4] BVH
 * nodes visited, out[5] leaves visited, out[6] clips that changed a cell,
 * out[7] candidates that reached the vertex test. No reference counterpart
 * (the reference only prints timings, voronoi_ultra.cu:196-219). */
int pg_stats(const void *workspace, int64_t num_points, uint64_t *out, int32_t count, void *stream);

/* ---- One diagram over several GPUs (no reference counterpart: the reference builds on one
 * device). Every rank holds all points (an all-gather of their shards), builds the LBVH and the
 * cells of its own range of sorted slots, and exchanges its rows:
 *   pg_build_range   the LBVH of all points and the cells of sorted slots [cell_begin, cell_end)
 *                    (the curve order of the LBVH: equal ranges are balanced and compact); status
 *                    [num_points] receives those cells' statuses. Synchronises the stream.
 *   pg_range_pack    the range's rows as one int32 pack: count, the cells' point indices [count],
 *                    statuses [count], row starts [count + 1], then the neighbour indices. With
 *                    pack == NULL only *words_needed is set (synchronises the stream).
 *   pg_range_unpack  another rank's pack (count = its cell_end - cell_begin) into this workspace.
 *   pg_range_finish  the symmetric CSR offsets of the assembled rows and the edge count
 *                    (synchronises); pg_emit_adjacency then fills the adjacency as after pg_build.
 * Every rank that unpacks all other ranks' packs holds the same Diagram as a single pg_build. */
int pg_build_range(int64_t num_points, const float *points, const float *weights, const pg_options *options,
                   void *workspace, size_t workspace_bytes, int64_t cell_begin, int64_t cell_end, int32_t *status,
                   void *stream);
int pg_range_pack(int64_t num_points, const void *workspace, const int32_t *status, int64_t cell_begin,
                  int64_t cell_end, int32_t *pack, int64_t pack_words, int64_t *words_needed, void *stream);
int pg_range_unpack(int64_t num_points, void *workspace, int32_t *status, const int32_t *pack, int64_t count,
                    int64_t pack_words, void *stream);
int pg_range_finish(int64_t num_points, void *workspace, int32_t *offsets, int64_t *num_edges, void *stream);

/* Where the BVH lives inside a workspace/* Where the BVH lives inside a workspace that pg_build (num_clouds = 1) or pg_build_batch
 * filled: out[k] = byte offset from the workspace's start of
 *   [0] the sorted points (float4 x, y, z, w per sorted slot, N of them),
 *   [1] sorted slot -> original point index (int32 [N]),
 *   [2] the traversal records, 4 float4 per internal node (node i at 64 i bytes):
 *       (c0.lo.x, c0.lo.y, c0.lo.z, c0.hi.x), (c0.hi.y, c0.hi.z, c1.lo.x, c1.lo.y),
 *       (c1.lo.z, c1.hi.x, c1.hi.y, c1.hi.z), (ref0, ref1 as int32 bits, maxw0, maxw1);
 *       a reference < 0 is a leaf: bit 31, count - 1 in bits 26..30, first sorted slot in
 *       bits 0..25; a reference >= 0 is another record,
 *   [3] the root reference of each cloud (int32 [num_clouds]),
 *   [4] each cloud's box (float32 [8 per cloud]: lo xyz, hi xyz, max weight, unused).
 * For inspection and tests (the layout depends on num_points and num_clouds only).
 * No reference counterpart (the reference's BVH is cuBQL's, pwr_bvh.cu:42-339). */
int pg_workspace_tree(int64_t num_points, int32_t num_clouds, int64_t *out, int32_t count);

/* The k nearest other points of every point (1 <= k <= 32): neighbours [num_points * k] receives,
 * per point in input order, the original indices of its k nearest points by unweighted FP32
 * Euclidean distance (ties by index; the point itself excluded, copies at its position included),
 * -1 where the cloud has fewer points. Builds the LBVH in workspace (pg_workspace_size bytes,
 * 256-byte aligned) and synchronises the stream. Replaces the reference's kNN query
 * (pwr_bvh.cu:159-215), which warm-starts its cells (voronoi_ultra.cu:205-227); here the cell pass
 * does not need it (its traversal starts at the point's own leaf), and a caller that wants the
 * reference's warm start passes the result to pg_build as initial guesses. */
int pg_knn(int64_t num_points, const float *points, int32_t k, void *workspace, size_t workspace_bytes,
           int32_t *neighbours, void *stream);

/* Profile of the last pg_build + pg_emit_adjacency on this thread:
 * out[0] kernel launches, out[1] LBVH ms, out[2] cell pass ms, out[3] deferred-cell
 * pass ms, out[4] CSR count + scan ms, out[5] deferred cells, out[6] cell-pass chunks,
 * out[7] deferred cells rebuilt with 256 slots, out[8] with 512 slots, out[9] cells a
 * learned model routed past the first pass (pg_model.route_degree).
 * The times are recorded only when options->debug != 0 (CUDA events on the stream).
 * No reference counterpart (the reference prints timings with debug=True,
 * voronoi_ultra.cu:196-219, 368-373). */
int pg_last_profile(double *out, int32_t count);

/* ---- Batches: many independent point clouds in one build --------------------
 * No single reference counterpart: the reference builds one cloud per call
 * (paragram/_api.py:65-123); a batch is equivalent to one call per cloud.
 * Cloud c owns points [cloud_offsets[c], cloud_offsets[c+1]) of the concatenated
 * arrays; every cloud gets its own box and its own diagram. Output: one CSR over
 * all points whose rows list GLOBAL point indices (a cloud's rows only list its
 * own points); offsets [total + 1], status [total].
 * With num_edges == NULL the call never synchronises: the total edge count stays
 * in offsets[total] on the device, the whole call can be captured in a CUDA graph,
 * and pg_batch_check reports errors afterwards. pg_emit_adjacency fills the
 * adjacency as for a single diagram. */
int pg_batch_workspace_size(int64_t total_points, int32_t num_clouds, size_t *bytes);
int pg_build_batch(int64_t total_points, int32_t num_clouds, const int32_t *cloud_offsets, const float *points,
                   const float *weights, const pg_options *options, void *workspace, size_t workspace_bytes,
                   int32_t *offsets, int32_t *status, int64_t *num_edges, void *stream);
int pg_batch_check(const void *workspace, int64_t total_points, int32_t num_clouds, void *stream);

/* Training and evaluation kernels of the learned search radius (no reference
 * counterpart). Parameters: a flat float32 vector of pg_mlp_num_params()
 * master weights in the order w1 [64][16], b1 [64], w2 [64][64], b2 [64],
 * w3 [2][64], b3 [2]; the model holds their BF16 / FP32 copies.
 *   pg_mlp_forward  out [n][2] = network(features [n][16])
 *   pg_mlp_grad     adds to grad [num_params] the gradient of
 *                   L = sum_s w_s |y_s - t'_s|^2 * inv_total_weight / 2 (t' = normalised targets [n][2],
 *                   w = sample_weights [n]) and adds L to *loss (device float); the caller zeroes both
 *   pg_mlp_adam     one Adam step of params (m, v: moments, step >= 1), then writes the model's weights
 *   pg_mlp_pack     writes the model's weights from params
 * All pointers are device pointers; calls are ordered on `stream`. */
int pg_mlp_num_params(void);
size_t pg_mlp_model_bytes(void);
int pg_mlp_forward(int64_t n, const float *features, const void *model, float *out, void *stream);
int pg_mlp_grad(int64_t n, const float *features, const float *targets, const float *sample_weights,
                float inv_total_weight, const void *model, float *grad, float *loss, void *stream);
int pg_mlp_adam(float *params, const float *grad, float *m, float *v, int64_t step, float lr, float beta1,
                float beta2, float eps, void *model, void *stream);
int pg_mlp_pack(const float *params, void *model, void *stream);

/* Facet areas of a built diagram, aligned with its adjacency (no reference counterpart: the
 * reference computes each cell's polytope and keeps only the neighbour ids, voronoi_ultra.cu:125-138).
 * Inputs are the vertex export of the build (pg_options.vertices_out, vertex_planes_out,
 * vertex_count_out with capacity vertex_cap <= 256), the build's points (float32 [N * 3]) and its
 * Diagram (offsets [N + 1], adjacency [E]). areas (float32 [E], output): for entry e of row u, the
 * area of the facet between u's cell and adjacency[e]'s; NaN when a cell's vertices exceeded
 * vertex_cap. All pointers are device pointers; ordered on stream. */
int pg_face_areas(int64_t num_points, int32_t vertex_cap, const float *vertices, const int32_t *vertex_planes,
                  const int32_t *vertex_count, const float *points, const int32_t *offsets, const int32_t *adjacency,
                  float *areas, void *stream);

/* CSR offsets from per-row degrees, allocating nothing. No counterpart in the
 * reference: it is for callers that cannot allocate device memory when they
 * call (a device-memory budget fixed at start-up, device memory owned by
 * another framework's allocator, or a path that cannot afford the implicit
 * synchronisation of cudaMalloc / cudaFree).
 *   degrees  int32 [num_rows], non-negative, sum < 2^31 (device)
 *   offsets  int32 [num_rows + 1] (device, output): exclusive prefix sum, offsets[num_rows] = total
 * Its scratch is a fixed device array inside the library (129 KB per GPU,
 * held until exit), so num_rows is limited to 2^26 - 1; larger sizes return
 * PG_ERR_INVALID. The first call on a device resolves the array's address
 * (cudaGetSymbolAddress) with that device current; make that first call before
 * any stream capture. All calls on a device share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. The resolved
 * address is kept per device ordinal for the life of the process: after a
 * cudaDeviceReset (or a new primary context) on that device it is stale, so a
 * caller that resets a device must not call this entry point afterwards. */
int pg_degrees_to_offsets_noalloc(int64_t num_rows, const int32_t *degrees, int32_t *offsets, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PARAGRAM_B200_H */
