// pg_scan.cu -- exclusive prefix sum over uint32 (reduce / scan-of-sums /
// downsweep), used for radix-sort digit offsets and for the CSR offsets.
//
// The reference computes its CSR offsets with torch::cumsum over an int32
// tensor (voronoi_ultra.cu:347-350, laguerre_ultra.cu:425-428); this is the
// hand-written replacement. out[n] receives the total.
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v)
{
    int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o)
            v += t;
    }
    return v;
}

// exclusive scan of one value per thread over a 256-thread block
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = warp_inclusive(v);
    if (lane == 31)
        warp_sums[w] = inc;
    __syncthreads();
    if (w == 0)
    {
        uint32_t s = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
        s = warp_inclusive(s);
        if (lane < kScanThreads / 32)
            warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t off = w > 0 ? warp_sums[w - 1] : 0;
    *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return off + inc - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t *__restrict__ in, int64_t n,
                                                             uint32_t *__restrict__ sums)
{
    int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n)
            s += in[i];
    }
    uint32_t total;
    block_exclusive(s, &total);
    if (threadIdx.x == 0)
        sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(const uint32_t *in, int64_t n, uint32_t *out,
                                                           const uint32_t *__restrict__ offsets)
{
    __shared__ uint32_t tile[kScanTile + kScanTile / 32];
    int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        int j = k * kScanThreads + threadIdx.x;
        int64_t i = base + j;
        tile[j + (j >> 5)] = i < n ? in[i] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        int j = threadIdx.x * kScanItems + k;
        v[k] = tile[j + (j >> 5)];
        s += v[k];
    }
    uint32_t total;
    uint32_t pre = block_exclusive(s, &total);
    uint32_t boff = offsets ? offsets[blockIdx.x] : 0u;
    pre += boff;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        int j = threadIdx.x * kScanItems + k;
        tile[j + (j >> 5)] = pre;
        pre += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        int j = k * kScanThreads + threadIdx.x;
        int64_t i = base + j;
        if (i < n)
            out[i] = tile[j + (j >> 5)];
    }
    if (threadIdx.x == 0 && base + kScanTile >= n)
        out[n] = boff + total;
}

size_t scan_tmp_elems(int64_t n)
{
    size_t t = 0;
    while (n > kScanTile)
    {
        int64_t nb = (n + kScanTile - 1) / kScanTile;
        t += (size_t)nb + 1 + 64;
        n = nb;
    }
    return t + 64;
}

void exclusive_scan(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *tmp, cudaStream_t st)
{
    int64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 1)
    {
        ++g_launches;
        k_scan_down<<<1, kScanThreads, 0, st>>>(in, n, out, nullptr);
        return;
    }
    uint32_t *sums = tmp;
    uint32_t *rest = tmp + nb + 1 + 64;
    ++g_launches;
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, sums);
    exclusive_scan(sums, sums, nb, rest, st);
    ++g_launches;
    k_scan_down<<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, out, sums);
}

} // namespace pg
