// pg_faces.cu -- area of every facet of a built diagram, aligned with its CSR adjacency.
//
// No reference counterpart: the reference's cell kernel computes each cell's
// polytope and keeps only the neighbour ids (voronoi_ultra.cu:125-138,
// laguerre_ultra.cu:155-172). The areas come from the vertices that pg_build
// exports (pg_options.vertices_out / vertex_planes_out / vertex_count_out):
// the facet of cell u on neighbour v is the convex polygon of u's vertices
// that lie on plane v. One warp per row: for each entry v it selects those
// vertices (a ballot over the cell's vertex slots), orders them by angle
// around their centroid in the facet's plane (whose normal is the direction
// from u's point to v's) and sums the fan of triangles from the centroid.
// An entry whose facet u's vertices do not carry (a reverse entry added by the
// symmetrisation, adjacency.cuh:78-159) takes the facet from v's cell.
#include <algorithm>
#include <string>

#include "../../include/paragram_b200.h"
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

constexpr int kFaceWarps = 4;
constexpr int kFaceMaxCap = 256; // vertex slots a cell may export

struct FaceScratch
{
    float2 p[kFaceMaxCap]; // selected vertices in the facet's plane basis, relative to their centroid
    float ang[kFaceMaxCap];
    float2 sorted[kFaceMaxCap];
};

// Area of the facet of cell c on plane q from c's exported vertices; -1 when fewer
// than three of them lie on q (c does not carry that facet), NaN when c's
// vertices were truncated.
__device__ float facet_area(int c, int q, int cap, const float4 *__restrict__ V, const int *__restrict__ P,
                            const int *__restrict__ cnt, const float *__restrict__ pts, FaceScratch &S, int lane)
{
    const unsigned full = 0xFFFFFFFFu;
    int k = cnt[c];
    if (k > cap)
        return __int_as_float(0x7fc00000);
    float nx = pts[3 * (size_t)q] - pts[3 * (size_t)c], ny = pts[3 * (size_t)q + 1] - pts[3 * (size_t)c + 1],
          nz = pts[3 * (size_t)q + 2] - pts[3 * (size_t)c + 2];
    float nn = sqrtf(nx * nx + ny * ny + nz * nz);
    if (!(nn > 0.0f))
        return -1.0f;
    nx /= nn;
    ny /= nn;
    nz /= nn;
    // select the vertices on plane q and their centroid
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    int m = 0;
    for (int base = 0; base < k; base += 32)
    {
        int j = base + lane;
        bool on = false;
        float4 x = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (j < k)
        {
            const int *pl = P + ((size_t)c * cap + j) * 3;
            on = pl[0] == q || pl[1] == q || pl[2] == q;
            if (on)
                x = V[(size_t)c * cap + j];
        }
        unsigned b = __ballot_sync(full, on);
        if (on)
        {
            int r = m + __popc(b & ((1u << lane) - 1u));
            S.sorted[r] = make_float2(x.x, x.y); // staging: x, y here, z below
            S.ang[r] = x.z;
        }
        cx += on ? x.x : 0.0f;
        cy += on ? x.y : 0.0f;
        cz += on ? x.z : 0.0f;
        m += __popc(b);
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        cx += __shfl_xor_sync(full, cx, o);
        cy += __shfl_xor_sync(full, cy, o);
        cz += __shfl_xor_sync(full, cz, o);
    }
    if (m < 3)
        return -1.0f;
    cx /= (float)m;
    cy /= (float)m;
    cz /= (float)m;
    __syncwarp();
    // a basis (e1, e2) of the facet's plane: e1 orthogonal to n from the coordinate axis least aligned with it
    float ax = fabsf(nx), ay = fabsf(ny), az = fabsf(nz);
    float tx = 0.0f, ty = 0.0f, tz = 0.0f;
    if (ax <= ay && ax <= az)
        tx = 1.0f;
    else if (ay <= az)
        ty = 1.0f;
    else
        tz = 1.0f;
    float d = tx * nx + ty * ny + tz * nz;
    float e1x = tx - d * nx, e1y = ty - d * ny, e1z = tz - d * nz;
    float e1n = rsqrtf(e1x * e1x + e1y * e1y + e1z * e1z);
    e1x *= e1n;
    e1y *= e1n;
    e1z *= e1n;
    float e2x = ny * e1z - nz * e1y, e2y = nz * e1x - nx * e1z, e2z = nx * e1y - ny * e1x;
    for (int r = lane; r < m; r += 32)
    {
        float2 xy = S.sorted[r];
        float px = xy.x - cx, py = xy.y - cy, pz = S.ang[r] - cz;
        float u = px * e1x + py * e1y + pz * e1z, v = px * e2x + py * e2y + pz * e2z;
        S.p[r] = make_float2(u, v);
    }
    __syncwarp();
    for (int r = lane; r < m; r += 32)
        S.ang[r] = atan2f(S.p[r].y, S.p[r].x);
    __syncwarp();
    // order by angle (ties by index): each item's rank is the number of items before it
    for (int r = lane; r < m; r += 32)
    {
        float a = S.ang[r];
        int rank = 0;
        for (int t = 0; t < m; ++t)
        {
            float b = S.ang[t];
            rank += (b < a) || (b == a && t < r);
        }
        S.sorted[rank] = S.p[r];
    }
    __syncwarp();
    float area = 0.0f;
    for (int r = lane; r < m; r += 32)
    {
        float2 a = S.sorted[r], b = S.sorted[r + 1 < m ? r + 1 : 0];
        area += 0.5f * (a.x * b.y - a.y * b.x);
    }
    for (int o = 16; o > 0; o >>= 1)
        area += __shfl_xor_sync(full, area, o);
    __syncwarp();
    return fabsf(area);
}

__global__ void __launch_bounds__(kFaceWarps * 32) k_face_areas(int64_t n, int cap, const float4 *__restrict__ V,
                                                                const int *__restrict__ P, const int *__restrict__ cnt,
                                                                const float *__restrict__ pts,
                                                                const int *__restrict__ off,
                                                                const int *__restrict__ adj, float *__restrict__ out)
{
    __shared__ FaceScratch scratch[kFaceWarps];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    FaceScratch &S = scratch[w];
    int64_t warps = (int64_t)gridDim.x * kFaceWarps;
    for (int64_t u = (int64_t)blockIdx.x * kFaceWarps + w; u < n; u += warps)
    {
        int e0 = off[u], e1 = off[u + 1];
        for (int e = e0; e < e1; ++e)
        {
            int v = adj[e];
            float a = facet_area((int)u, v, cap, V, P, cnt, pts, S, lane);
            if (a == -1.0f)
            {
                a = facet_area(v, (int)u, cap, V, P, cnt, pts, S, lane);
                if (a == -1.0f)
                    a = 0.0f;
            }
            if (lane == 0)
                out[e] = a;
        }
    }
}

} // namespace pg

extern "C" int pg_face_areas(int64_t num_points, int32_t vertex_cap, const float *vertices,
                             const int32_t *vertex_planes, const int32_t *vertex_count, const float *points,
                             const int32_t *offsets, const int32_t *adjacency, float *areas, void *stream)
{
    using namespace pg;
    if (num_points < 0 || num_points >= kMaxPoints)
        return set_last_error(PG_ERR_INVALID, "num_points must be in [0, 2^26)");
    if (vertex_cap < 1 || vertex_cap > kFaceMaxCap)
        return set_last_error(PG_ERR_INVALID, "vertex_cap must be in [1, " + std::to_string(kFaceMaxCap) + "]");
    if (num_points == 0)
        return set_last_error(PG_OK, "");
    if (!vertices || !vertex_planes || !vertex_count || !points || !offsets || !adjacency || !areas)
        return set_last_error(PG_ERR_INVALID, "pointers must not be NULL");
    if (((uintptr_t)vertices & 15u) != 0)
        return set_last_error(PG_ERR_INVALID, "vertices must be 16-byte aligned");
    cudaGetLastError();
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t need = (num_points + kFaceWarps - 1) / kFaceWarps;
    int64_t grid = std::min<int64_t>(need, (int64_t)sms * 16);
    ++g_launches;
    k_face_areas<<<(unsigned)grid, kFaceWarps * 32, 0, (cudaStream_t)stream>>>(
        num_points, vertex_cap, reinterpret_cast<const float4 *>(vertices), vertex_planes, vertex_count, points,
        offsets, adjacency, areas);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_last_error(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    return set_last_error(PG_OK, "");
}
