// pg_knn.cu -- k nearest neighbours of every point on the build's LBVH.
//
// The reference queries cuBQL for each point's K + 1 nearest points and drops
// the point itself (pwr_bvh.cu:159-215); it warm-starts every cell with them
// (voronoi_ultra.cu:205-227). Here the query runs on the LBVH of pg_build
// (pg_lbvh.cu): one thread per sorted slot (neighbouring threads query
// neighbouring points, so their traversals share nodes in L1/L2), a
// depth-first descent into the nearer child first with a fixed stack, the k
// best kept sorted by (squared distance, original index). Distances are the
// unweighted Euclidean ones in FP32 (like the reference's, also for power
// diagrams), each product and sum rounded separately so that a CPU restatement
// in float32 reproduces them and their ties exactly. A point's copies at the
// same position are neighbours like any other point; only its own index is
// excluded. The cell pass does not use the result (its traversal starts at the
// point's own leaf); pg_knn exports it, and the Python layer can pass it to a
// build as initial guesses, which is the reference's warm start.
#include <algorithm>
#include <string>

#include "../../include/paragram_b200.h"
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

constexpr int kKnnMax = 32;   // largest k
constexpr int kKnnStack = 96; // pending subtrees; the descent pushes one per tree level

__global__ void k_knn_single_cloud(int *cloud_off, int n)
{
    cloud_off[0] = 0;
    cloud_off[1] = n;
}

__device__ __forceinline__ float sq_dist(float4 a, float4 b)
{
    float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Lower bound of the squared distance from q to the box (lo, hi), slightly rounded down.
__device__ __forceinline__ float box_sq_dist(float4 q, float lx, float ly, float lz, float hx, float hy, float hz)
{
    float dx = fmaxf(fmaxf(lx - q.x, q.x - hx), 0.0f);
    float dy = fmaxf(fmaxf(ly - q.y, q.y - hy), 0.0f);
    float dz = fmaxf(fmaxf(lz - q.z, q.z - hz), 0.0f);
    return (dx * dx + dy * dy + dz * dz) * (1.0f - 1e-5f);
}

__global__ void __launch_bounds__(128) k_knn(int64_t n, int k, const float4 *__restrict__ pts,
                                             const int *__restrict__ oid, const float4 *__restrict__ rec,
                                             const int *__restrict__ cloud_off, int num_clouds,
                                             const int *__restrict__ cloud_root, int *__restrict__ out, int *err)
{
    int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= n)
        return;
    const int i = (int)ii;
    const float4 q = pts[i];
    const int root = cloud_root[cloud_of(cloud_off, num_clouds, i)];
    float bd[kKnnMax];
    int bi[kKnnMax];
    int cnt = 0;
    int stk[kKnnStack];
    float skey[kKnnStack];
    int sp = 0;
    stk[sp] = root;
    skey[sp++] = 0.0f;
    while (sp > 0)
    {
        --sp;
        const int ref = stk[sp];
        const float key = skey[sp];
        const float worst = cnt < k ? INFINITY : bd[k - 1];
        if (key > worst)
            continue;
        if (ref < 0)
        {
            for (int j = leaf_first(ref), e = j + leaf_count(ref); j < e; ++j)
            {
                if (j == i)
                    continue;
                const float d = sq_dist(q, pts[j]);
                const int id = oid[j];
                if (cnt == k && (d > bd[k - 1] || (d == bd[k - 1] && id > bi[k - 1])))
                    continue;
                // insertion into the sorted list (the last entry drops out when it is full)
                int at = cnt < k ? cnt++ : k - 1;
                while (at > 0 && (bd[at - 1] > d || (bd[at - 1] == d && bi[at - 1] > id)))
                {
                    bd[at] = bd[at - 1];
                    bi[at] = bi[at - 1];
                    --at;
                }
                bd[at] = d;
                bi[at] = id;
            }
            continue;
        }
        const float4 *r = rec + 4 * (size_t)ref;
        const float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
        const float k0 = box_sq_dist(q, r0.x, r0.y, r0.z, r0.w, r1.x, r1.y);
        const float k1 = box_sq_dist(q, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w);
        const int c0 = __float_as_int(r3.x), c1 = __float_as_int(r3.y);
        if (sp + 2 > kKnnStack)
        {
            atomicExch(err, 3);
            break;
        }
        // the nearer child is popped first
        const bool near0 = k0 <= k1;
        stk[sp] = near0 ? c1 : c0;
        skey[sp++] = near0 ? k1 : k0;
        stk[sp] = near0 ? c0 : c1;
        skey[sp++] = near0 ? k0 : k1;
    }
    int *o = out + (size_t)oid[i] * k;
    for (int t = 0; t < k; ++t)
        o[t] = t < cnt ? bi[t] : -1;
}

} // namespace pg

extern "C" int pg_knn(int64_t num_points, const float *points, int32_t k, void *workspace, size_t workspace_bytes,
                      int32_t *neighbours, void *stream)
{
    using namespace pg;
    if (num_points < 0 || num_points >= kMaxPoints)
        return set_last_error(PG_ERR_INVALID, "num_points must be in [0, 2^26)");
    if (k < 1 || k > kKnnMax)
        return set_last_error(PG_ERR_INVALID, "k must be in [1, " + std::to_string(kKnnMax) + "]");
    if (num_points == 0)
        return set_last_error(PG_OK, "");
    if (!points || !workspace || !neighbours)
        return set_last_error(PG_ERR_INVALID, "points, workspace and neighbours must not be NULL");
    if (((uintptr_t)workspace & 255u) != 0)
        return set_last_error(PG_ERR_INVALID, "workspace must be 256-byte aligned");
    const size_t need = workspace_layout(num_points, 1, nullptr, nullptr);
    if (workspace_bytes < need)
        return set_last_error(PG_ERR_INVALID, "workspace too small: need " + std::to_string(need) + " bytes");
    cudaStream_t st = (cudaStream_t)stream;
    cudaGetLastError();
    Workspace ws;
    workspace_layout(num_points, 1, (char *)workspace, &ws);
    cudaMemsetAsync(ws.counters, 0, 16 * sizeof(int), st);
    ++g_launches;
    k_knn_single_cloud<<<1, 1, 0, st>>>(ws.cloud_off, (int)num_points);
    lbvh_build(ws, num_points, 1, points, nullptr, kDefaultLeaf, st);
    ++g_launches;
    k_knn<<<(unsigned)((num_points + 127) / 128), 128, 0, st>>>(num_points, k, ws.pts, ws.oid, ws.records,
                                                                ws.cloud_off, 1, ws.cloud_root, neighbours,
                                                                &ws.counters[2]);
    int flag = 0;
    cudaMemcpyAsync(&flag, &ws.counters[2], sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return set_last_error(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    if (flag == 2)
        return set_last_error(PG_ERR_INTERNAL, "the points do not form one BVH subtree");
    if (flag == 3)
        return set_last_error(PG_ERR_INTERNAL, "kNN descent exceeded its stack (BVH deeper than 96 levels)");
    return set_last_error(PG_OK, "");
}
