// pg_csr.cu -- directed rows -> symmetric CSR with sorted rows.
//
// Reference semantics (adjacency.cuh:78-159, count_symmetrized_adjacency_sizes
// and populate_symmetric_adjacency): the directed edge u->v is kept iff v's
// directed degree is > 0, and the reverse v->u is added when v does not list
// u. The reference places entries with atomics (row order nondeterministic);
// here kept entries keep the (sorted) directed order, added reverse entries
// are appended and the few rows that received one are re-sorted, so every
// row comes out sorted and the output is deterministic.
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

__device__ __forceinline__ const int *row_of(const int *rows, const int *big_rows, const int *deg, int u, int &d)
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

__device__ __forceinline__ bool row_has(const int *r, int d, int x)
{
    int lo = 0, hi = d;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        int v = r[mid];
        if (v == x)
            return true;
        if (v < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return false;
}

__global__ void k_csr_count(const int *__restrict__ rows, const int *__restrict__ big_rows,
                            const int *__restrict__ deg, int64_t n, int *__restrict__ cnt, int *__restrict__ miss)
{
    int64_t uu = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (uu >= n)
        return;
    int u = (int)uu, d;
    const int *r = row_of(rows, big_rows, deg, u, d);
    int kept = 0;
    for (int k = 0; k < d; ++k)
    {
        int v = r[k], dv;
        const int *rv = row_of(rows, big_rows, deg, v, dv);
        if (dv <= 0)
            continue;
        ++kept;
        if (!row_has(rv, dv, u))
            atomicAdd(&miss[v], 1);
    }
    cnt[u] = kept;
}

__global__ void k_csr_sizes(const int *__restrict__ cnt, const int *__restrict__ miss, int64_t n,
                            uint32_t *__restrict__ sizes)
{
    int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n)
        sizes[u] = (uint32_t)(cnt[u] + miss[u]);
}

__global__ void k_csr_fill(const int *__restrict__ rows, const int *__restrict__ big_rows, const int *__restrict__ deg,
                           int64_t n, const int *__restrict__ off, const int *__restrict__ cnt, int *__restrict__ fill,
                           int *__restrict__ adj)
{
    int64_t uu = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (uu >= n)
        return;
    int u = (int)uu, d;
    const int *r = row_of(rows, big_rows, deg, u, d);
    int pos = off[u];
    for (int k = 0; k < d; ++k)
    {
        int v = r[k], dv;
        const int *rv = row_of(rows, big_rows, deg, v, dv);
        if (dv <= 0)
            continue;
        adj[pos++] = v;
        if (!row_has(rv, dv, u))
            adj[off[v] + cnt[v] + atomicAdd(&fill[v], 1)] = u;
    }
}

__global__ void k_csr_sort(const int *__restrict__ miss, int64_t n, const int *__restrict__ off, int *__restrict__ adj)
{
    int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n || miss[u] == 0)
        return;
    int b = off[u], e = off[u + 1];
    for (int i = b + 1; i < e; ++i)
    {
        int x = adj[i], j = i - 1;
        while (j >= b && adj[j] > x)
        {
            adj[j + 1] = adj[j];
            --j;
        }
        adj[j + 1] = x;
    }
}

void csr_count(const Workspace &ws, int64_t n, int32_t *offsets, cudaStream_t st)
{
    unsigned g = (unsigned)((n + 255) / 256);
    cudaMemsetAsync(ws.miss, 0, sizeof(int) * (size_t)n, st);
    ++g_launches;
    k_csr_count<<<g, 256, 0, st>>>(ws.rows, ws.big_rows, ws.deg, n, ws.cnt, ws.miss);
    ++g_launches;
    k_csr_sizes<<<g, 256, 0, st>>>(ws.cnt, ws.miss, n, ws.sizes);
    exclusive_scan(ws.sizes, (uint32_t *)offsets, n, ws.scan_tmp, st);
}

void csr_fill(const Workspace &ws, int64_t n, const int32_t *offsets, int32_t *adjacency, cudaStream_t st)
{
    unsigned g = (unsigned)((n + 255) / 256);
    cudaMemsetAsync(ws.fill, 0, sizeof(int) * (size_t)n, st);
    ++g_launches;
    k_csr_fill<<<g, 256, 0, st>>>(ws.rows, ws.big_rows, ws.deg, n, offsets, ws.cnt, ws.fill, adjacency);
    ++g_launches;
    k_csr_sort<<<g, 256, 0, st>>>(ws.miss, n, offsets, adjacency);
}

} // namespace pg
