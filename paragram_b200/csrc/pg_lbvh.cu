// pg_lbvh.cu -- linear BVH over the input points.
//
// Replaces the reference's third-party cuBQL builder (pwr_bvh.cu:217-339:
// degenerate point boxes -> cuBQL::gpuBuilder with makeLeafThreshold, then a
// max-weight copy and bottom-up propagation, pwr_bvh.cu:42-157). Here:
//   1. scene bounds (one reduction) -> the reference's initial box
//      (root AABB -1.0f/+1.0f, voronoi_ultra.cu:234-238, then -1e-5f/+1e-5f,
//      faster_convex_cell.cuh:206-221) and the Morton frame;
//   2. 63-bit Morton codes (21 bits per axis);
//   3. LSD radix sort of (code, index), 8 passes of 8 bits (hand written);
//   4. points gathered in curve order (x, y, z, w) so leaves are contiguous;
//   5. binary radix tree (T. Karras, "Maximizing Parallelism in the
//      Construction of BVHs, Octrees, and k-d Trees", HPG 2012);
//   6. bottom-up box + max-weight refit with arrival counters;
//   7. 64-byte traversal records for every internal node with more than
//      leaf_size points: both child boxes, child references (a child with at
//      most leaf_size points becomes a leaf: a contiguous range of sorted
//      points) and both child max weights.
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

constexpr int kSortThreads = 256;
constexpr int kSortSteps = 16;
constexpr int kSortTile = kSortThreads * kSortSteps;

int sort_blocks(int64_t n) { return (int)((n + kSortTile - 1) / kSortTile); }

__global__ void k_bounds_init(int *b, int num_clouds)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_clouds * 8)
        return;
    int k = t & 7;
    b[t] = float_to_ordered(k < 3 ? INFINITY : -INFINITY);
}

// Per-cloud bounds: warps reduce per distinct cloud (normally one) before the atomics.
__global__ void k_bounds(const float *__restrict__ p, const float *__restrict__ w, int64_t n,
                         const int *__restrict__ coff, int num_clouds, int *b)
{
    const unsigned full = 0xFFFFFFFFu;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x)
    {
        int64_t i = base + threadIdx.x;
        bool ok = i < n;
        int c = ok ? cloud_of(coff, num_clouds, (int)i) : -1;
        float v[7] = {0, 0, 0, 0, 0, 0, 0};
        if (ok)
        {
            v[0] = v[3] = p[i * 3 + 0];
            v[1] = v[4] = p[i * 3 + 1];
            v[2] = v[5] = p[i * 3 + 2];
            v[6] = w ? w[i] : 0.0f;
        }
        unsigned todo = __ballot_sync(full, ok);
        while (todo)
        {
            int leader = __ffs(todo) - 1;
            int cl = __shfl_sync(full, c, leader);
            bool mine = ok && c == cl;
            todo &= ~__ballot_sync(full, mine);
#pragma unroll
            for (int k = 0; k < 7; ++k)
            {
                int key = float_to_ordered(mine ? v[k] : (k < 3 ? INFINITY : -INFINITY));
                int r = k < 3 ? __reduce_min_sync(full, key) : __reduce_max_sync(full, key);
                if ((int)(threadIdx.x & 31) == leader)
                {
                    if (k < 3)
                        atomicMin(&b[cl * 8 + k], r);
                    else
                        atomicMax(&b[cl * 8 + k], r);
                }
            }
        }
    }
}

// Per cloud: the reference box in FP32 (same operations as the reference) and the Morton frame.
__global__ void k_box(const int *b, float *box, float *morton, int num_clouds)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= num_clouds)
        return;
    float mn[3], mx[3], ext = 0.0f;
    for (int k = 0; k < 3; ++k)
    {
        mn[k] = ordered_to_float(b[c * 8 + k]);
        mx[k] = ordered_to_float(b[c * 8 + 3 + k]);
        box[c * 8 + k] = __fsub_rn(__fsub_rn(mn[k], 1.0f), 1e-5f);
        box[c * 8 + 3 + k] = __fadd_rn(__fadd_rn(mx[k], 1.0f), 1e-5f);
        ext = fmaxf(ext, mx[k] - mn[k]);
        morton[c * 4 + k] = mn[k];
    }
    box[c * 8 + 6] = ordered_to_float(b[c * 8 + 6]); // max weight
    morton[c * 4 + 3] = ext;                          // extent; the scale depends on the bits per axis
}

__device__ __forceinline__ unsigned long long spread3(unsigned long long x)
{
    x &= 0x1FFFFFull;
    x = (x | x << 32) & 0x1F00000000FFFFull;
    x = (x | x << 16) & 0x1F0000FF0000FFull;
    x = (x | x << 8) & 0x100F00F00F00F00Full;
    x = (x | x << 4) & 0x10C30C30C30C30C3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__device__ __forceinline__ unsigned long long quant(float v, float o, float s, float top)
{
    float t = (v - o) * s;
    t = fminf(fmaxf(t, 0.0f), top);
    return (unsigned long long)t;
}

// key = cloud id in the top bits, then a Morton code with `bits` bits per axis in the cloud's frame
__global__ void k_morton(const float *__restrict__ p, int64_t n, const int *__restrict__ coff, int num_clouds,
                         int bits, const float *__restrict__ morton, unsigned long long *__restrict__ keys,
                         uint32_t *__restrict__ vals)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int c = cloud_of(coff, num_clouds, (int)i);
    float top = (float)((1u << bits) - 1u);
    float ext = morton[c * 4 + 3];
    float sc = ext > 0.0f ? top / ext : 0.0f;
    unsigned long long x = quant(p[i * 3 + 0], morton[c * 4 + 0], sc, top);
    unsigned long long y = quant(p[i * 3 + 1], morton[c * 4 + 1], sc, top);
    unsigned long long z = quant(p[i * 3 + 2], morton[c * 4 + 2], sc, top);
    keys[i] = ((unsigned long long)c << (3 * bits)) | (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
    vals[i] = (uint32_t)i;
}

// Root of every cloud's subtree: clouds are contiguous in curve order (their id is
// the key prefix), so each cloud with more than `leaf` points is one Karras subtree.
__global__ void k_cloud_roots(const int *__restrict__ coff, int num_clouds, int leaf, const int *__restrict__ first,
                              const int *__restrict__ last, const int *__restrict__ parent_int,
                              const int *__restrict__ parent_leaf, int *__restrict__ roots, int *err)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= num_clouds)
        return;
    int a = coff[c], b = coff[c + 1], nc = b - a;
    if (nc <= 0)
    {
        roots[c] = 0;
        return;
    }
    if (nc <= leaf)
    {
        roots[c] = leaf_ref(a, nc);
        return;
    }
    int node = parent_leaf[a];
    for (int it = 0; it < 200 && node >= 0; ++it)
    {
        if (first[node] == a && last[node] == b - 1)
        {
            roots[c] = node;
            return;
        }
        node = parent_int[node];
    }
    roots[c] = 0;
    atomicExch(err, 2);
}

// ---------------------------------------------------------------------------
// LSD radix sort, 8-bit digits. hist is digit-major: hist[d * blocks + b].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kSortThreads) k_hist(const unsigned long long *__restrict__ keys, int64_t n,
                                                      int shift, uint32_t *__restrict__ hist)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int s = 0; s < kSortSteps; ++s)
    {
        int64_t i = base + (int64_t)s * kSortThreads + threadIdx.x;
        if (i < n)
            atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_scatter(const unsigned long long *__restrict__ kin,
                                                         const uint32_t *__restrict__ vin, int64_t n, int shift,
                                                         const uint32_t *__restrict__ offs,
                                                         unsigned long long *__restrict__ kout,
                                                         uint32_t *__restrict__ vout)
{
    __shared__ uint32_t base[256];
    __shared__ uint32_t wc[kSortThreads / 32][256];
    int t = threadIdx.x, w = t >> 5, lane = t & 31;
    base[t] = offs[(size_t)t * gridDim.x + blockIdx.x];
#pragma unroll
    for (int k = 0; k < kSortThreads / 32; ++k)
        wc[k][t] = 0;
    __syncthreads();
    int64_t tile = (int64_t)blockIdx.x * kSortTile;
    const uint32_t lt = (1u << lane) - 1u;
    for (int s = 0; s < kSortSteps; ++s)
    {
        int64_t i = tile + (int64_t)s * kSortThreads + t;
        bool ok = i < n;
        unsigned long long key = ok ? kin[i] : 0ull;
        uint32_t val = ok ? vin[i] : 0u;
        uint32_t d = ok ? (uint32_t)((key >> shift) & 255u) : (256u + lane);
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        uint32_t r = __popc(peers & lt);
        if (ok && r == 0)
            wc[w][d] = __popc(peers);
        __syncthreads();
        if (ok)
        {
            uint32_t pre = 0;
            for (int k = 0; k < w; ++k)
                pre += wc[k][d];
            uint32_t pos = base[d] + pre + r;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        uint32_t tot = 0;
#pragma unroll
        for (int k = 0; k < kSortThreads / 32; ++k)
        {
            tot += wc[k][t];
            wc[k][t] = 0;
        }
        base[t] += tot;
        __syncthreads();
    }
}

__global__ void k_gather(const float *__restrict__ p, const float *__restrict__ w, int64_t n,
                         const uint32_t *__restrict__ vals, float4 *__restrict__ pts, int *__restrict__ oid,
                         int *__restrict__ rank)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    uint32_t v = vals[i];
    pts[i] = make_float4(p[(size_t)v * 3 + 0], p[(size_t)v * 3 + 1], p[(size_t)v * 3 + 2], w ? w[v] : 0.0f);
    oid[i] = (int)v;
    rank[v] = (int)i;
}

// ---------------------------------------------------------------------------
// Karras radix tree: internal node i in [0, n-2]; node 0 is the root.
// Children: >= 0 internal node, < 0 leaf point ~c.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int common_prefix(const unsigned long long *k, int64_t n, int i, int j)
{
    if (j < 0 || j >= n)
        return -1;
    unsigned long long a = k[i], b = k[j];
    if (a == b)
        return 64 + __clz((unsigned)(i ^ j));
    return __clzll(a ^ b);
}

__global__ void k_karras(const unsigned long long *__restrict__ k, int64_t n, int *__restrict__ left,
                         int *__restrict__ right, int *__restrict__ first, int *__restrict__ last,
                         int *__restrict__ parent_int, int *__restrict__ parent_leaf)
{
    int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= n - 1)
        return;
    int i = (int)ii;
    int d = (common_prefix(k, n, i, i + 1) - common_prefix(k, n, i, i - 1)) > 0 ? 1 : -1;
    int dmin = common_prefix(k, n, i, i - d);
    int lmax = 2;
    while (common_prefix(k, n, i, i + lmax * d) > dmin)
        lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (common_prefix(k, n, i, i + (l + t) * d) > dmin)
            l += t;
    int j = i + l * d;
    int dnode = common_prefix(k, n, i, j);
    int s = 0, t = l;
    do
    {
        t = (t + 1) >> 1;
        if (common_prefix(k, n, i, i + (s + t) * d) > dnode)
            s += t;
    } while (t > 1);
    int gamma = i + s * d + (d < 0 ? -1 : 0);
    int lo = min(i, j), hi = max(i, j);
    int lc, rc;
    if (lo == gamma)
    {
        lc = ~gamma;
        parent_leaf[gamma] = i;
    }
    else
    {
        lc = gamma;
        parent_int[gamma] = i;
    }
    if (hi == gamma + 1)
    {
        rc = ~(gamma + 1);
        parent_leaf[gamma + 1] = i;
    }
    else
    {
        rc = gamma + 1;
        parent_int[gamma + 1] = i;
    }
    left[i] = lc;
    right[i] = rc;
    first[i] = lo;
    last[i] = hi;
    if (i == 0)
        parent_int[0] = -1;
}

__device__ __forceinline__ void child_box(int c, const float4 *pts, const float4 *nbox, float4 &lo, float4 &hi)
{
    if (c < 0)
    {
        float4 p = pts[~c];
        lo = make_float4(p.x, p.y, p.z, p.w);
        hi = make_float4(p.x, p.y, p.z, __int_as_float(1));
    }
    else
    {
        lo = __ldcg(&nbox[2 * (size_t)c]);
        hi = __ldcg(&nbox[2 * (size_t)c + 1]);
    }
}

// Bottom-up refit: the second thread to reach a node merges its children.
__global__ void k_refit(const float4 *__restrict__ pts, int64_t n, const int *__restrict__ left,
                        const int *__restrict__ right, const int *__restrict__ parent_int,
                        const int *__restrict__ parent_leaf, int *flags, float4 *nbox)
{
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n)
        return;
    int node = parent_leaf[j];
    while (node >= 0)
    {
        __threadfence();
        if (atomicAdd(&flags[node], 1) == 0)
            return;
        __threadfence();
        float4 l0, l1, r0, r1;
        child_box(left[node], pts, nbox, l0, l1);
        child_box(right[node], pts, nbox, r0, r1);
        int cnt = __float_as_int(l1.w) + __float_as_int(r1.w);
        float4 lo = make_float4(fminf(l0.x, r0.x), fminf(l0.y, r0.y), fminf(l0.z, r0.z), fmaxf(l0.w, r0.w));
        float4 hi = make_float4(fmaxf(l1.x, r1.x), fmaxf(l1.y, r1.y), fmaxf(l1.z, r1.z), __int_as_float(cnt));
        __stcg(&nbox[2 * (size_t)node], lo);
        __stcg(&nbox[2 * (size_t)node + 1], hi);
        node = parent_int[node];
    }
}

// Traversal record of internal node i (only nodes with > leaf points are read):
//   r0 = (c0.lo.x, c0.lo.y, c0.lo.z, c0.hi.x)
//   r1 = (c0.hi.y, c0.hi.z, c1.lo.x, c1.lo.y)
//   r2 = (c1.lo.z, c1.hi.x, c1.hi.y, c1.hi.z)
//   r3 = (ref0, ref1, maxw0, maxw1)
__global__ void k_records(const float4 *__restrict__ pts, int64_t n, const int *__restrict__ left,
                          const int *__restrict__ right, const int *__restrict__ first, const float4 *__restrict__ nbox,
                          int leaf, float4 *__restrict__ rec, int *__restrict__ rparent, int *__restrict__ pleaf)
{
    int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= n - 1)
        return;
    int i = (int)ii;
    if (__float_as_int(nbox[2 * (size_t)i + 1].w) <= leaf)
        return;
    int cref[2];
    float4 clo[2], chi[2];
    int ch[2] = {left[i], right[i]};
    for (int c = 0; c < 2; ++c)
    {
        int x = ch[c];
        child_box(x, pts, nbox, clo[c], chi[c]);
        int cnt = __float_as_int(chi[c].w);
        if (x < 0)
            cref[c] = leaf_ref(~x, 1);
        else if (cnt <= leaf)
            cref[c] = leaf_ref(first[x], cnt);
        else
            cref[c] = x;
        // upward links for traversals that start at a point's own leaf
        if (cref[c] < 0)
            for (int p = leaf_first(cref[c]), e = p + leaf_count(cref[c]); p < e; ++p)
                pleaf[p] = (i << 1) | c;
        else
            rparent[x] = (i << 1) | c;
    }
    rec[4 * (size_t)i + 0] = make_float4(clo[0].x, clo[0].y, clo[0].z, chi[0].x);
    rec[4 * (size_t)i + 1] = make_float4(chi[0].y, chi[0].z, clo[1].x, clo[1].y);
    rec[4 * (size_t)i + 2] = make_float4(clo[1].z, chi[1].x, chi[1].y, chi[1].z);
    rec[4 * (size_t)i + 3] = make_float4(__int_as_float(cref[0]), __int_as_float(cref[1]), clo[0].w, clo[1].w);
}

void lbvh_build(const Workspace &ws, int64_t n, int num_clouds, const float *points, const float *weights,
                int leaf_size, cudaStream_t st)
{
    ++g_launches;
    k_bounds_init<<<(num_clouds * 8 + 255) / 256, 256, 0, st>>>(ws.bounds, num_clouds);
    int nb = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    if (nb < 1)
        nb = 1;
    ++g_launches;
    k_bounds<<<nb, 256, 0, st>>>(points, weights, n, ws.cloud_off, num_clouds, ws.bounds);
    ++g_launches;
    k_box<<<(num_clouds + 127) / 128, 128, 0, st>>>(ws.bounds, ws.box, ws.morton, num_clouds);
    int cbits = 0;
    while ((1 << cbits) < num_clouds)
        ++cbits;
    int bits = std::min(21, (63 - cbits) / 3);
    unsigned g = (unsigned)((n + 255) / 256);
    ++g_launches;
    k_morton<<<g, 256, 0, st>>>(points, n, ws.cloud_off, num_clouds, bits, ws.morton, ws.keys0, ws.vals0);
    int blocks = sort_blocks(n);
    unsigned long long *ka = ws.keys0, *kb = ws.keys1;
    uint32_t *va = ws.vals0, *vb = ws.vals1;
    for (int pass = 0; pass < 8; ++pass)
    {
        int shift = pass * 8;
        ++g_launches;
        k_hist<<<blocks, kSortThreads, 0, st>>>(ka, n, shift, ws.hist);
        exclusive_scan(ws.hist, ws.hist, (int64_t)256 * blocks, ws.scan_tmp, st);
        ++g_launches;
        k_scatter<<<blocks, kSortThreads, 0, st>>>(ka, va, n, shift, ws.hist, kb, vb);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    // after 8 passes the sorted data is back in keys0 / vals0
    ++g_launches;
    k_gather<<<g, 256, 0, st>>>(points, weights, n, va, ws.pts, ws.oid, ws.rank);
    if (n >= 2)
    {
        ++g_launches;
        k_karras<<<g, 256, 0, st>>>(ka, n, ws.left, ws.right, ws.first, ws.last, ws.parent_int, ws.parent_leaf);
        cudaMemsetAsync(ws.flags, 0, sizeof(int) * (size_t)n, st);
        ++g_launches;
        k_refit<<<g, 256, 0, st>>>(ws.pts, n, ws.left, ws.right, ws.parent_int, ws.parent_leaf, ws.flags, ws.nbox);
        ++g_launches;
        cudaMemsetAsync(ws.rparent, 0xFF, sizeof(int) * (size_t)n, st); // -1: no parent record
        k_records<<<g, 256, 0, st>>>(ws.pts, n, ws.left, ws.right, ws.first, ws.nbox, leaf_size, ws.records,
                                     ws.rparent, ws.pleaf);
    }
    ++g_launches;
    k_cloud_roots<<<(num_clouds + 127) / 128, 128, 0, st>>>(ws.cloud_off, num_clouds, leaf_size, ws.first, ws.last,
                                                            ws.parent_int, ws.parent_leaf, ws.cloud_root,
                                                            &ws.counters[2]);
}

} // namespace pg
