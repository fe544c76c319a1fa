// pg_kernels.cuh -- host-side launchers shared between the translation units.
#pragma once

#include <string>

#include "pg_common.cuh"

struct pg_model; // include/paragram_b200.h

namespace pg
{

// kernel launches issued by the calling thread (reported by pg_last_profile)
extern thread_local long long g_launches;

// pg_scan.cu
size_t scan_tmp_elems(int64_t n);
void exclusive_scan(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *tmp, cudaStream_t st);

// pg_lbvh.cu
int sort_blocks(int64_t n);
void lbvh_build(const Workspace &ws, int64_t n, int num_clouds, const float *points, const float *weights,
                int leaf_size, cudaStream_t st);

// pg_cells.cu
struct CellLaunch
{
    int64_t n;
    int leaf_size;
    int num_clouds;           // independent point sets sharing the launch
    int window;               // warm-start half width (0: off)
    const int *guesses;       // initial guesses (original ids) or nullptr
    const int *guess_off;     // [N+1] offsets of the initial guesses
    int64_t cell_begin, cell_end; // sorted-slot range of this launch
    int weighted;
    int min_blocks; // register-budget variant of the cell kernel (2 or 3 blocks per SM)
    int64_t big_cap; // deferred-row slots
    float *radius_out; // per original id: certified radius of the final cell, or nullptr
    int *work_out;     // per original id: nodes, leaves, candidates, peak queue; or nullptr
    float *geometry_out; // per original id: centroid x, y, z and volume of the cell; or nullptr
    int vertex_cap;            // vertex export: slots per cell
    float *vertices_out;       // per original id x vertex_cap: vertex relative to the point, error bound
    int *vertex_planes_out;    // per original id x vertex_cap x 3: planes of the vertex (ids / -1 - box code)
    int *vertex_count_out;     // per original id: number of vertices
    int use_hint;      // the workspace holds a search radius per sorted slot
    int fp32_only;     // side tests in FP32 only (no escalation; not exact)
};
void cells_launch(const Workspace &ws, const CellLaunch &cl, int *status, int num_sms, cudaStream_t st);
void cells_big_launch(const Workspace &ws, const CellLaunch &cl, int *status, int64_t big_cap, cudaStream_t st);

// pg_mlp.cu
void features_launch(const Workspace &ws, int64_t n, int num_clouds, float *out, cudaStream_t st);
// The learned radius of every sorted slot into ws.hint; with the model's route_degree set, the
// slots predicted at or above it (at most route_cap) are listed for the 128-slot tier, their
// rows marked deferred and their hint negated (the first pass skips them).
void predict_launch(const Workspace &ws, int64_t n, int num_clouds, const ::pg_model *model, int *status,
                    int64_t route_cap, cudaStream_t st);
int set_last_error(int code, const std::string &msg);

// pg_csr.cu
void csr_count(const Workspace &ws, int64_t n, int32_t *offsets, cudaStream_t st);
void csr_fill(const Workspace &ws, int64_t n, const int32_t *offsets, int32_t *adjacency, cudaStream_t st);

} // namespace pg
