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

// Whether the sorted row r[0, d) lists x, for d <= kRowWidth: one pass of independent
// 16-byte loads over the row (a single round trip to L2, where a binary search would make
// four dependent ones). Rows start 16-byte aligned (kRowWidth = 36 ints, deferred rows
// kBigRowWidth) and the loads stay within the row's first kRowWidth slots.
__device__ __forceinline__ bool row_has_scan(const int *r, int d, int x)
{
    const int4 *r4 = reinterpret_cast<const int4 *>(r);
    bool hit = false;
#pragma unroll
    for (int k = 0; k < kRowWidth / 4; ++k)
    {
        if (4 * k >= d)
            break;
        int4 q = __ldg(r4 + k);
        hit = hit || (q.x == x && 4 * k < d) || (q.y == x && 4 * k + 1 < d) || (q.z == x && 4 * k + 2 < d) ||
              (q.w == x && 4 * k + 3 < d);
    }
    return hit;
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

// Rows are visited in curve order (thread t takes sorted slot t), so that a
// block's cells are spatial neighbours and the rows their searches read are
// shared through L2. Per row, two bit masks over its directed entries record
// what the fill needs: entry k is kept (its target has a nonempty row) and
// entry k's target does not list this row (a reverse entry to add). Rows of
// deferred cells (up to kBigRowWidth entries) do not fit the masks and are
// re-examined by the fill.
__global__ void k_csr_count(const int *__restrict__ rows, const int *__restrict__ big_rows,
                            const int *__restrict__ deg, const int *__restrict__ oid, int64_t n, int *__restrict__ cnt,
                            int *__restrict__ miss, unsigned long long *__restrict__ masks)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    int u = oid[t], d;
    const int *r = row_of(rows, big_rows, deg, u, d);
    int kept = 0;
    unsigned long long keep_bits = 0, miss_bits = 0;
    for (int k = 0; k < d; ++k)
    {
        int v = r[k], dv;
        const int *rv = row_of(rows, big_rows, deg, v, dv);
        if (dv <= 0)
            continue;
        ++kept;
        bool missing = !(dv <= kRowWidth ? row_has_scan(rv, dv, u) : row_has(rv, dv, u));
        if (missing)
            atomicAdd(&miss[v], 1);
        if (k < 64)
        {
            keep_bits |= 1ull << k;
            miss_bits |= (unsigned long long)missing << k;
        }
    }
    cnt[u] = kept;
    masks[2 * (size_t)u] = keep_bits;
    masks[2 * (size_t)u + 1] = miss_bits;
}

__global__ void k_csr_sizes(const int *__restrict__ cnt, const int *__restrict__ miss, int64_t n,
                            uint32_t *__restrict__ sizes)
{
    int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n)
        sizes[u] = (uint32_t)(cnt[u] + miss[u]);
}

// The fill reads no neighbour row (the count's masks decided every entry): rows are taken in
// their own order, so that reads of the rows and writes of the adjacency are contiguous.
__global__ void k_csr_fill(const int *__restrict__ rows, const int *__restrict__ big_rows, const int *__restrict__ deg,
                           int64_t n, const int *__restrict__ off, const int *__restrict__ cnt,
                           const unsigned long long *__restrict__ masks, int *__restrict__ fill,
                           int *__restrict__ adj)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    int u = (int)t, d;
    const int *r = row_of(rows, big_rows, deg, u, d);
    int pos = off[u];
    if (d <= 64)
    {
        // the count pass already decided every entry
        unsigned long long keep_bits = masks[2 * (size_t)u], miss_bits = masks[2 * (size_t)u + 1];
        for (int k = 0; k < d; ++k)
        {
            if (!((keep_bits >> k) & 1ull))
                continue;
            int v = r[k];
            adj[pos++] = v;
            if ((miss_bits >> k) & 1ull)
                adj[off[v] + cnt[v] + atomicAdd(&fill[v], 1)] = u;
        }
        return;
    }
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
    k_csr_count<<<g, 256, 0, st>>>(ws.rows, ws.big_rows, ws.deg, ws.oid, n, ws.cnt, ws.miss, ws.rmask);
    ++g_launches;
    k_csr_sizes<<<g, 256, 0, st>>>(ws.cnt, ws.miss, n, ws.sizes);
    exclusive_scan(ws.sizes, (uint32_t *)offsets, n, ws.scan_tmp, st);
}

void csr_fill(const Workspace &ws, int64_t n, const int32_t *offsets, int32_t *adjacency, cudaStream_t st)
{
    unsigned g = (unsigned)((n + 255) / 256);
    cudaMemsetAsync(ws.fill, 0, sizeof(int) * (size_t)n, st);
    ++g_launches;
    k_csr_fill<<<g, 256, 0, st>>>(ws.rows, ws.big_rows, ws.deg, n, offsets, ws.cnt, ws.rmask, ws.fill, adjacency);
    ++g_launches;
    k_csr_sort<<<g, 256, 0, st>>>(ws.miss, n, offsets, adjacency);
}

} // namespace pg
