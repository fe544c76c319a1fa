// pg_api.cu -- C ABI (include/paragram_b200.h) and host orchestration.
//
// Reference orchestration: build_voronoi_ultra (voronoi_ultra.cu:143-376) and
// build_laguerre_voronoi_ultra (laguerre_ultra.cu:176-454):
// pack -> BVH + kNN -> chunked cell kernel -> gather -> symmetrise -> cumsum
// -> populate. Here: LBVH -> chunked cell launches -> deferred-cell pass ->
// CSR count + scan (offsets) -> [host reads E] -> CSR fill.
#include <atomic>
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/paragram_b200.h"
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

static thread_local std::string g_last_error;
thread_local long long g_launches = 0;
static thread_local double g_profile[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

static int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

int set_last_error(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

static size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

// Deferred-row slots: room for the cells that outgrow the first pass's 64 slots
// (65536 + n / 32) plus the cells a learned model routes to the 128-slot tier
// directly (at most route_cap, so that routing never exhausts the room of the
// cells that overflow).
static int64_t route_cap(int64_t n) { return std::min<int64_t>(n, 4096 + n / 128); }
static int64_t big_cap(int64_t n) { return std::min<int64_t>(n, 65536 + n / 32 + route_cap(n)); }

size_t workspace_layout(int64_t n, int num_clouds, char *base, Workspace *ws)
{
    size_t C = (size_t)std::max(num_clouds, 1);
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        char *p = base ? base + off : nullptr;
        off += align_up(bytes);
        return p;
    };
    size_t N = (size_t)std::max<int64_t>(n, 1);
    int blocks = sort_blocks((int64_t)N);
    size_t hist_elems = (size_t)256 * blocks + 1;
    size_t scan_elems = scan_tmp_elems((int64_t)std::max(hist_elems, N + 1));
    Workspace w;
    w.counters = (int *)take(16 * sizeof(int));
    w.stats = (unsigned long long *)take(kNumStats * sizeof(unsigned long long));
    w.keys0 = (unsigned long long *)take(8 * N);
    w.keys1 = (unsigned long long *)take(8 * N);
    w.vals0 = (uint32_t *)take(4 * N);
    w.vals1 = (uint32_t *)take(4 * N);
    w.hist = (uint32_t *)take(4 * hist_elems);
    w.scan_tmp = (uint32_t *)take(4 * scan_elems);
    w.pts = (float4 *)take(16 * N);
    w.oid = (int *)take(4 * N);
    w.rank = (int *)take(4 * N);
    w.left = (int *)take(4 * N);
    w.right = (int *)take(4 * N);
    w.first = (int *)take(4 * N);
    w.last = (int *)take(4 * N);
    w.parent_int = (int *)take(4 * N);
    w.parent_leaf = (int *)take(4 * N);
    w.flags = (int *)take(4 * N);
    w.nbox = (float4 *)take(32 * N);
    w.records = (float4 *)take(64 * N);
    w.rparent = (int *)take(4 * N);
    w.pleaf = (int *)take(4 * N);
    w.hint = (float *)take(4 * N);
    w.rows = (int *)take(4 * N * kRowWidth);
    w.deg = (int *)take(4 * N);
    w.big_list = (int *)take(4 * N);
    w.big_list2 = (int *)take(4 * (size_t)big_cap((int64_t)N));
    w.big_slot2 = (int *)take(4 * (size_t)big_cap((int64_t)N));
    w.big_rows = (int *)take(4 * (size_t)big_cap((int64_t)N) * kBigRowWidth);
    w.huge_slabs = take(huge_slab_bytes());
    w.cnt = (int *)take(4 * N);
    w.miss = (int *)take(4 * N);
    w.fill = (int *)take(4 * N);
    w.rmask = (unsigned long long *)take(16 * N);
    w.sizes = (uint32_t *)take(4 * (N + 1));
    // per-cloud segments last, so that every other offset is independent of the cloud count
    w.bounds = (int *)take(8 * C * sizeof(int));
    w.box = (float *)take(8 * C * sizeof(float));
    w.morton = (float *)take(4 * C * sizeof(float));
    w.cloud_off = (int *)take((C + 1) * sizeof(int));
    w.cloud_root = (int *)take(C * sizeof(int));
    w.bytes = off;
    if (ws)
        *ws = w;
    return off;
}

// Total memory of the current device, queried once per device.
static size_t device_total_memory()
{
    static std::atomic<size_t> total[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    {
        cudaGetLastError();
        return 0;
    }
    size_t t = total[dev].load();
    if (t == 0)
    {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
            t = prop.totalGlobalMem;
        cudaGetLastError();
        total[dev].store(t);
    }
    return t;
}

// Chunk plan of the cell pass. Mirrors plan_convex_cell_chunks (chunking.h:16-56):
// PARAGRAM_NUM_CHUNKS forces a count; otherwise the per-cell scratch is compared
// with PARAGRAM_MEM_FRAC (0.05 < f < 0.95, default 0.5) of the free device
// memory. The clipper keeps its per-cell polyhedron in shared memory, so its
// only per-cell global scratch is the directed row (kRowWidth ints). The free
// memory is queried only when the scratch exceeds that fraction of a quarter of
// the device's total memory (never below 2^26 points on a B200): the query
// takes the driver's lock, and a build that waited for it left the GPU idle
// between its launches.
static int plan_chunks(int64_t n, int requested)
{
    if (requested > 0)
        return requested;
    const char *force = std::getenv("PARAGRAM_NUM_CHUNKS");
    if (force && std::atoi(force) > 0)
        return std::atoi(force);
    double frac = 0.5;
    const char *fe = std::getenv("PARAGRAM_MEM_FRAC");
    if (fe)
    {
        double f = std::atof(fe);
        if (f > 0.05 && f < 0.95)
            frac = f;
    }
    size_t full = (size_t)n * kRowWidth * sizeof(int);
    const size_t total = device_total_memory();
    if (total > 0 && (double)full <= frac * (double)(total / 4))
        return 1;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
    {
        cudaGetLastError();
        return 1;
    }
    size_t budget = (size_t)(frac * (double)free_b);
    if (budget > 0 && full > budget)
        return (int)((full + budget - 1) / budget);
    return 1;
}

static int device_sms()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    return sms;
}


__global__ void k_single_cloud(int *off, int n)
{
    off[0] = 0;
    off[1] = n;
}

// search radius per sorted slot from the caller's per-point radii (negative and NaN radii:
// none; a negative hint is the model's routing mark)
__global__ void k_hint_gather(int64_t n, const int *oid, const float *radius, float *hint)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        hint[i] = fmaxf(radius[oid[i]], 0.0f);
}

// ---- One diagram over several GPUs: every rank builds the LBVH of all points and the cells of
// its own range of sorted slots, packs its rows, receives the others' packs and assembles the CSR.
// A pack (int32 words): count, the cells' original indices [count], statuses [count], row starts
// [count + 1] (exclusive scan of the degrees), then the rows' neighbour indices.

// The row of original point u: the fast-pass row, or (deferred cells) a deferred-row slot.
__device__ __forceinline__ const int *shard_row(const int *rows, const int *big_rows, const int *deg, int u, int &d)
{
    int dv = deg[u];
    if (dv & (int)kBigFlag)
    {
        d = dv & ~(int)kBigFlag;
        return big_rows + (size_t)rows[(size_t)u * kRowWidth] * kBigRowWidth;
    }
    d = dv;
    return rows + (size_t)u * kRowWidth;
}

__global__ void k_pack_degrees(int64_t begin, int64_t count, const int *oid, const int *deg, uint32_t *sizes)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count)
        sizes[t] = (uint32_t)(deg[oid[begin + t]] & ~(int)kBigFlag);
    else if (t == count)
        sizes[t] = 0u;
}

__global__ void k_pack_rows(int64_t begin, int64_t count, const int *oid, const int *rows, const int *big_rows,
                            const int *deg, const int *status, const uint32_t *start, int *out)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t > count)
        return;
    int *ids = out + 1, *sts = ids + count;
    int *st = sts + count, *nb = st + count + 1;
    st[t] = (int)start[t];
    if (t == count)
    {
        out[0] = (int)count;
        return;
    }
    int u = oid[begin + t], d = 0;
    const int *r = shard_row(rows, big_rows, deg, u, d);
    ids[t] = u;
    sts[t] = status[u];
    int *o = nb + start[t];
    for (int j = 0; j < d; ++j)
        o[j] = r[j];
}

// Rows of another rank's cells into this workspace: fast-pass rows where they fit, else a
// deferred-row slot after the ones in use. Flags: 4 = no deferred-row slot left, 5 = malformed pack.
__global__ void k_unpack_rows(int64_t n, int64_t count, int64_t words, const int *pack, int *rows, int *big_rows,
                              int *deg, int *status, int *counters, int64_t big_capacity)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count)
        return;
    const int *ids = pack + 1, *sts = ids + count, *st = sts + count, *nb = st + count + 1;
    const int64_t nb_words = words - (2 + 3 * count);
    int u = ids[t], s0 = st[t], s1 = st[t + 1];
    int d = s1 - s0;
    if (u < 0 || u >= n || s0 < 0 || d < 0 || d > kBigRowWidth || (int64_t)s1 > nb_words)
    {
        atomicExch(&counters[2], 5);
        return;
    }
    int *row;
    if (d <= kRowWidth)
    {
        row = rows + (size_t)u * kRowWidth;
        deg[u] = d;
    }
    else
    {
        int slot = atomicAdd(&counters[1], 1);
        if ((int64_t)slot >= big_capacity)
        {
            atomicExch(&counters[2], 4);
            return;
        }
        row = big_rows + (size_t)slot * kBigRowWidth;
        rows[(size_t)u * kRowWidth] = slot;
        deg[u] = d | (int)kBigFlag;
    }
    for (int j = 0; j < d; ++j)
        row[j] = nb[s0 + j];
    status[u] = sts[t];
}

static int check_counters(const int *host, int64_t n)
{
    if (host[2] == 1)
        return fail(PG_ERR_INTERNAL, "cell kernel consistency check failed (exact predicate capacity or "
                                     "polytope topology)");
    if (host[2] == 2)
        return fail(PG_ERR_INTERNAL, "a cloud's points do not form one BVH subtree");
    if (host[2] == 4)
        return fail(PG_ERR_INTERNAL, "received rows exceed the deferred-row capacity");
    if (host[2] == 5)
        return fail(PG_ERR_INVALID, "malformed row pack");
    if (host[1] > big_cap(n))
        return fail(PG_ERR_INTERNAL, "too many cells exceeded 64 vertices (" + std::to_string(host[1]) +
                                         " > capacity " + std::to_string(big_cap(n)) + ")");
    return PG_OK;
}

// One build of num_clouds independent diagrams over n points (cloud c owns points
// [cloud_offsets[c], cloud_offsets[c+1]) ). num_edges == NULL: no host synchronisation
// (the total stays in offsets[n] on the device; errors via pg_batch_check).
static int build_impl(int64_t n, int num_clouds, const int32_t *cloud_offsets, const float *points,
                      const float *weights, const int32_t *guesses, const int32_t *guess_off,
                      const pg_options *options, void *workspace, size_t workspace_bytes, int32_t *offsets,
                      int32_t *status, int64_t *num_edges, void *stream, int64_t range_begin = 0,
                      int64_t range_end = -1)
{
    // range_end >= 0: only the cells of sorted slots [range_begin, range_end), no CSR (a shard of a
    // diagram built on several GPUs; pg_build_range)
    const bool ranged = range_end >= 0;
    g_last_error.clear();
    cudaStream_t st = (cudaStream_t)stream;
    pg_options opt{};
    opt.knn = 8;
    opt.leaf_size = -1;
    if (options)
        opt = *options;
    const bool sync = num_edges != nullptr;
    if (n < 0 || n >= kMaxPoints)
        return fail(PG_ERR_INVALID, "num_points must be in [0, 2^26)");
    if (!offsets && !ranged)
        return fail(PG_ERR_INVALID, "offsets must not be NULL");
    if (ranged && (range_begin < 0 || range_begin > range_end || range_end > n))
        return fail(PG_ERR_INVALID, "the cell range must lie within [0, num_points]");
    if ((guesses == nullptr) != (guess_off == nullptr))
        return fail(PG_ERR_INVALID, "initial_guesses and initial_guesses_offsets must be provided together");
    if (n > 0 && (!points || !status || !workspace))
        return fail(PG_ERR_INVALID, "points, status and workspace must not be NULL");
    if (((uintptr_t)workspace & 255u) != 0)
        return fail(PG_ERR_INVALID, "workspace must be 256-byte aligned");
    if (opt.leaf_size > kMaxLeaf)
        return fail(PG_ERR_INVALID, "leaf_size must be at most 32");
    if (opt.predicates != 0 && opt.predicates != 1)
        return fail(PG_ERR_INVALID, "options.predicates must be 0 (filtered exact) or 1 (FP32 only)");
    if (((uintptr_t)opt.features_out & 15u) != 0 || ((uintptr_t)opt.model & 15u) != 0)
        return fail(PG_ERR_INVALID, "features_out and model must be 16-byte aligned");
    if (((uintptr_t)opt.work_out & 15u) != 0 || ((uintptr_t)opt.radius_out & 3u) != 0)
        return fail(PG_ERR_INVALID, "work_out must be 16-byte and radius_out 4-byte aligned");
    if (((uintptr_t)opt.geometry_out & 15u) != 0)
        return fail(PG_ERR_INVALID, "geometry_out must be 16-byte aligned");
    if (opt.vertex_cap < 0 || ((opt.vertices_out || opt.vertex_planes_out) && opt.vertex_cap == 0))
        return fail(PG_ERR_INVALID, "vertex_cap must be >= 0, and > 0 when vertices_out or vertex_planes_out is set");
    if (((uintptr_t)opt.vertices_out & 15u) != 0)
        return fail(PG_ERR_INVALID, "vertices_out must be 16-byte aligned");
    size_t need = workspace_layout(n, num_clouds, nullptr, nullptr);
    if (workspace_bytes < need)
        return fail(PG_ERR_INVALID, "workspace too small: need " + std::to_string(need) + " bytes");
    cudaGetLastError();
    if (n == 0)
    {
        if (offsets)
            cudaMemsetAsync(offsets, 0, sizeof(int32_t), st);
        if (!sync)
            return PG_OK;
        *num_edges = 0;
        cudaError_t e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? PG_OK : fail(PG_ERR_CUDA, cudaGetErrorString(e));
    }
    Workspace ws;
    workspace_layout(n, num_clouds, (char *)workspace, &ws);
    int leaf = opt.leaf_size > 0 ? opt.leaf_size : kDefaultLeaf;
    g_launches = 0;
    for (double &v : g_profile)
        v = 0.0;
    // debug bit 0: print phase timings (reference behaviour); bit 1: record them for pg_last_profile
    const bool timing = sync && opt.debug != 0;
    cudaEvent_t ev[5];
    if (timing)
        for (auto &e : ev)
            cudaEventCreate(&e);
    if (timing)
        cudaEventRecord(ev[0], st);
    cudaMemsetAsync(ws.counters, 0, 16 * sizeof(int), st);
    cudaMemsetAsync(ws.stats, 0, kNumStats * sizeof(unsigned long long), st);
    if (cloud_offsets)
        cudaMemcpyAsync(ws.cloud_off, cloud_offsets, sizeof(int) * (size_t)(num_clouds + 1), cudaMemcpyDeviceToDevice,
                        st);
    else
    {
        ++g_launches;
        k_single_cloud<<<1, 1, 0, st>>>(ws.cloud_off, (int)n);
    }
    lbvh_build(ws, n, num_clouds, points, weights, leaf, st);
    if (timing)
        cudaEventRecord(ev[1], st);
    CellLaunch cl;
    cl.n = n;
    cl.leaf_size = leaf;
    cl.num_clouds = num_clouds;
    // The reference warm-starts every cell with its kNN(knn) (voronoi_ultra.cu:205-227). The best-first
    // traversal here reaches the seed's own leaf first, which plays that role, so knn does not select
    // anything.
    cl.window = 0;
    cl.guesses = guesses;
    cl.guess_off = guess_off;
    cl.weighted = weights != nullptr;
    cl.min_blocks = opt.blocks_per_sm == 3 ? 3 : 2; // register budget of the cell kernel
    cl.big_cap = big_cap(n);
    cl.fp32_only = opt.predicates == 1;
    cl.radius_out = opt.radius_out;
    cl.work_out = opt.work_out;
    cl.geometry_out = opt.geometry_out;
    cl.vertex_cap = opt.vertex_cap;
    cl.vertices_out = opt.vertices_out;
    cl.vertex_planes_out = opt.vertex_planes_out;
    cl.vertex_count_out = opt.vertex_count_out;
    cl.use_hint = 0;
    if (opt.features_out != nullptr)
        features_launch(ws, n, num_clouds, opt.features_out, st);
    if (opt.order_out != nullptr)
        cudaMemcpyAsync(opt.order_out, ws.oid, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    if (opt.model != nullptr)
    {
        predict_launch(ws, n, num_clouds, (const pg_model *)opt.model, status, route_cap(n), st);
        cl.use_hint = 1;
    }
    else if (opt.radius_hint != nullptr)
    {
        ++g_launches;
        k_hint_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, ws.oid, opt.radius_hint, ws.hint);
        cl.use_hint = 1;
    }
    int chunks = sync ? plan_chunks(n, opt.num_chunks) : std::max(opt.num_chunks, 1);
    int sms = device_sms();
    const int64_t rb = ranged ? range_begin : 0, re = ranged ? range_end : n;
    int64_t per = (re - rb + chunks - 1) / chunks;
    for (int c = 0; c < chunks; ++c)
    {
        cl.cell_begin = rb + (int64_t)c * per;
        cl.cell_end = std::min<int64_t>(re, cl.cell_begin + per);
        if (cl.cell_begin >= cl.cell_end)
            break;
        cells_launch(ws, cl, status, sms, st);
    }
    if (timing)
        cudaEventRecord(ev[4], st);
    // Cells that outgrew 64 slots: a second launch over the deferred list. Rebuilt inside the first
    // launch, their large code evicted the first pass's from the instruction cache (surface data).
    cells_big_launch(ws, cl, status, big_cap(n), st);
    if (timing)
        cudaEventRecord(ev[2], st);
    if (!ranged)
        csr_count(ws, n, offsets, st);
    g_profile[0] = (double)g_launches;
    g_profile[6] = (double)chunks;
    if (!sync)
    {
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? PG_OK : fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    }
    int host[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t edges = 0;
    {
        uint32_t e32 = 0;
        if (!ranged)
            cudaMemcpyAsync(&e32, offsets + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(host, ws.counters, 8 * sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            return fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
        edges = e32;
    }
    if (timing)
    {
        cudaEventRecord(ev[3], st);
        cudaEventSynchronize(ev[3]);
        float t_bvh = 0, t_cells = 0, t_fast = 0, t_csr = 0;
        cudaEventElapsedTime(&t_bvh, ev[0], ev[1]);
        cudaEventElapsedTime(&t_cells, ev[1], ev[2]);
        cudaEventElapsedTime(&t_fast, ev[1], ev[4]);
        cudaEventElapsedTime(&t_csr, ev[2], ev[3]);
        g_profile[1] = t_bvh;
        g_profile[2] = t_fast;
        g_profile[3] = t_cells - t_fast;
        g_profile[4] = t_csr;
        if (opt.debug & 1)
        {
            std::printf("BVH Creation time: %f ms\n", t_bvh);
            std::printf("Cell construction time: %f ms (%d chunk(s), %d deferred cell(s))\n", t_cells, chunks,
                        host[1]);
            std::printf("CSR count time: %f ms\n", t_csr);
        }
        for (auto &e : ev)
            cudaEventDestroy(e);
    }
    g_profile[5] = (double)host[1];
    g_profile[7] = (double)host[5];                                 // rebuilt with 256 slots
    g_profile[8] = (double)std::min(host[4], kHugeSlabs);           // rebuilt with 512 slots
    g_profile[9] = (double)std::min<int64_t>(host[7], route_cap(n)); // routed past the first pass
    int rc = check_counters(host, n);
    if (rc != PG_OK)
        return rc;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    *num_edges = edges;
    return PG_OK;
}

} // namespace pg

extern "C" {

int pg_version(void) { return 200; }

const char *pg_last_error(void) { return pg::g_last_error.c_str(); }

int pg_workspace_size(int64_t num_points, size_t *bytes)
{
    if (!bytes)
        return pg::fail(PG_ERR_INVALID, "bytes must not be NULL");
    if (num_points < 0 || num_points >= pg::kMaxPoints)
        return pg::fail(PG_ERR_INVALID, "num_points must be in [0, 2^26)");
    *bytes = pg::workspace_layout(num_points, 1, nullptr, nullptr);
    return PG_OK;
}

int pg_build(int64_t n, const float *points, const float *weights, const int32_t *guesses, const int32_t *guess_off,
             const pg_options *options, void *workspace, size_t workspace_bytes, int32_t *offsets, int32_t *status,
             int64_t *num_edges, void *stream)
{
    if (!num_edges)
        return pg::fail(PG_ERR_INVALID, "num_edges must not be NULL");
    return pg::build_impl(n, 1, nullptr, points, weights, guesses, guess_off, options, workspace, workspace_bytes,
                          offsets, status, num_edges, stream);
}

int pg_workspace_tree(int64_t num_points, int32_t num_clouds, int64_t *out, int32_t count)
{
    if (!out || count < 0 || num_clouds < 1 || num_points < 0 || num_points >= pg::kMaxPoints)
        return pg::fail(PG_ERR_INVALID, "need out != NULL, count >= 0, num_clouds >= 1 and num_points in [0, 2^26)");
    // the layout from a stand-in base address; only differences from it are used
    char *base = reinterpret_cast<char *>((uintptr_t)1 << 40);
    pg::Workspace w;
    pg::workspace_layout(num_points, num_clouds, base, &w);
    const char *ptrs[5] = {(const char *)w.pts, (const char *)w.oid, (const char *)w.records,
                           (const char *)w.cloud_root, (const char *)w.box};
    for (int k = 0; k < count && k < 5; ++k)
        out[k] = (int64_t)(ptrs[k] - base);
    return pg::set_last_error(PG_OK, "");
}

int pg_batch_workspace_size(int64_t total_points, int32_t num_clouds, size_t *bytes)
{
    if (!bytes || num_clouds < 1 || total_points < 0 || total_points >= pg::kMaxPoints)
        return pg::fail(PG_ERR_INVALID, "need bytes != NULL, num_clouds >= 1 and total_points in [0, 2^26)");
    *bytes = pg::workspace_layout(total_points, num_clouds, nullptr, nullptr);
    return PG_OK;
}

int pg_build_batch(int64_t total_points, int32_t num_clouds, const int32_t *cloud_offsets, const float *points,
                   const float *weights, const pg_options *options, void *workspace, size_t workspace_bytes,
                   int32_t *offsets, int32_t *status, int64_t *num_edges, void *stream)
{
    if (num_clouds < 1 || !cloud_offsets)
        return pg::fail(PG_ERR_INVALID, "num_clouds must be >= 1 and cloud_offsets must not be NULL");
    return pg::build_impl(total_points, num_clouds, cloud_offsets, points, weights, nullptr, nullptr, options,
                          workspace, workspace_bytes, offsets, status, num_edges, stream);
}

int pg_batch_check(const void *workspace, int64_t total_points, int32_t num_clouds, void *stream)
{
    using namespace pg;
    if (!workspace || num_clouds < 1)
        return fail(PG_ERR_INVALID, "bad arguments");
    Workspace ws;
    workspace_layout(total_points, num_clouds, (char *)workspace, &ws);
    int host[4] = {0, 0, 0, 0};
    cudaStream_t st = (cudaStream_t)stream;
    cudaMemcpyAsync(host, ws.counters, 4 * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    return check_counters(host, total_points);
}

int pg_build_range(int64_t n, const float *points, const float *weights, const pg_options *options, void *workspace,
                   size_t workspace_bytes, int64_t cell_begin, int64_t cell_end, int32_t *status, void *stream)
{
    int64_t unused = 0;
    return pg::build_impl(n, 1, nullptr, points, weights, nullptr, nullptr, options, workspace, workspace_bytes,
                          nullptr, status, &unused, stream, cell_begin, cell_end);
}

int pg_range_pack(int64_t n, const void *workspace, const int32_t *status, int64_t cell_begin, int64_t cell_end,
                  int32_t *pack, int64_t pack_words, int64_t *words_needed, void *stream)
{
    using namespace pg;
    g_last_error.clear();
    if (n < 0 || n >= kMaxPoints || cell_begin < 0 || cell_begin > cell_end || cell_end > n)
        return fail(PG_ERR_INVALID, "need 0 <= cell_begin <= cell_end <= num_points < 2^26");
    if (!workspace || !status || !words_needed)
        return fail(PG_ERR_INVALID, "workspace, status and words_needed must not be NULL");
    Workspace ws;
    workspace_layout(n, 1, (char *)workspace, &ws);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t count = cell_end - cell_begin;
    const unsigned g = (unsigned)((count + 1 + 255) / 256);
    ++g_launches;
    k_pack_degrees<<<g, 256, 0, st>>>(cell_begin, count, ws.oid, ws.deg, ws.sizes);
    exclusive_scan(ws.sizes, ws.sizes, count + 1, ws.scan_tmp, st);
    uint32_t total = 0;
    cudaMemcpyAsync(&total, ws.sizes + count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    const int64_t need = 2 + 3 * count + (int64_t)total;
    *words_needed = need;
    if (!pack)
        return PG_OK;
    if (pack_words < need)
        return fail(PG_ERR_INVALID, "pack too small: need " + std::to_string(need) + " words");
    ++g_launches;
    k_pack_rows<<<g, 256, 0, st>>>(cell_begin, count, ws.oid, ws.rows, ws.big_rows, ws.deg, status, ws.sizes, pack);
    e = cudaGetLastError();
    return e == cudaSuccess ? PG_OK : fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
}

int pg_range_unpack(int64_t n, void *workspace, int32_t *status, const int32_t *pack, int64_t count,
                    int64_t pack_words, void *stream)
{
    using namespace pg;
    g_last_error.clear();
    if (n < 0 || n >= kMaxPoints || count < 0 || count > n)
        return fail(PG_ERR_INVALID, "need 0 <= count <= num_points < 2^26");
    if (!workspace || !status || !pack)
        return fail(PG_ERR_INVALID, "workspace, status and pack must not be NULL");
    if (pack_words < 2 + 3 * count)
        return fail(PG_ERR_INVALID, "pack shorter than its index");
    if (count == 0)
        return PG_OK;
    Workspace ws;
    workspace_layout(n, 1, (char *)workspace, &ws);
    cudaStream_t st = (cudaStream_t)stream;
    ++g_launches;
    k_unpack_rows<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(n, count, pack_words, pack, ws.rows, ws.big_rows,
                                                                   ws.deg, status, ws.counters, big_cap(n));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PG_OK : fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
}

int pg_range_finish(int64_t n, void *workspace, int32_t *offsets, int64_t *num_edges, void *stream)
{
    using namespace pg;
    g_last_error.clear();
    if (n < 0 || n >= kMaxPoints)
        return fail(PG_ERR_INVALID, "num_points must be in [0, 2^26)");
    if (!workspace || !offsets || !num_edges)
        return fail(PG_ERR_INVALID, "workspace, offsets and num_edges must not be NULL");
    Workspace ws;
    workspace_layout(n, 1, (char *)workspace, &ws);
    cudaStream_t st = (cudaStream_t)stream;
    csr_count(ws, n, offsets, st);
    int host[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t e32 = 0;
    cudaMemcpyAsync(&e32, offsets + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(host, ws.counters, 8 * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    int rc = check_counters(host, n);
    if (rc != PG_OK)
        return rc;
    *num_edges = e32;
    return PG_OK;
}

int pg_emit_adjacency(int64_t n, const void *workspace, const int32_t *offsets, int32_t *adjacency, void *stream)
{
    using namespace pg;
    g_last_error.clear();
    if (n < 0 || n >= kMaxPoints)
        return fail(PG_ERR_INVALID, "num_points must be in [0, 2^26)");
    if (n == 0)
        return PG_OK;
    if (!workspace || !offsets || !adjacency)
        return fail(PG_ERR_INVALID, "workspace, offsets and adjacency must not be NULL");
    Workspace ws;
    workspace_layout(n, 1, (char *)workspace, &ws); // the CSR segments do not depend on the cloud count
    long long before = g_launches;
    csr_fill(ws, n, offsets, adjacency, (cudaStream_t)stream);
    g_profile[0] += (double)(g_launches - before);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    return PG_OK;
}

int pg_last_profile(double *out, int32_t count)
{
    if (!out || count < 0)
        return pg::fail(PG_ERR_INVALID, "bad arguments");
    for (int i = 0; i < count && i < 10; ++i)
        out[i] = pg::g_profile[i];
    return PG_OK;
}

int pg_stats(const void *workspace, int64_t n, uint64_t *out, int32_t count, void *stream)
{
    using namespace pg;
    if (!workspace || !out || count < 0)
        return fail(PG_ERR_INVALID, "bad arguments");
    Workspace ws;
    workspace_layout(n, 1, (char *)workspace, &ws);
    unsigned long long tmp[kNumStats];
    cudaStream_t st = (cudaStream_t)stream;
    cudaMemcpyAsync(tmp, ws.stats, sizeof(tmp), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(PG_ERR_CUDA, cudaGetErrorString(e));
    for (int i = 0; i < count && i < kNumStats; ++i)
        out[i] = tmp[i];
    return PG_OK;
}

} // extern "C"
