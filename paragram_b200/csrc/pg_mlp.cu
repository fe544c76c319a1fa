// pg_mlp.cu -- learned search radius: features, a 16 -> 64 -> 64 -> 2 MLP on
// the tensor cores (BF16 operands, FP32 accumulation), its training kernels
// (forward + backward with weight gradients, Adam) and the fused prediction
// used by the cell pass.
//
// No reference counterpart: the reference warm-starts every cell with its
// kNN and shrinks the search radius (voronoi_ultra.cu:39-141). Here the model
// predicts, from cheap local features, the certified radius of a point's
// final cell; the cell pass uses it as a cap on its first traversal pass and
// keeps the result only if the final radius is within the cap (pg_cells.cu),
// so a wrong prediction costs time and never changes the diagram.
//
// Features of sorted slot i (its cloud [c0, c1), window = the slots
// i-16 .. i+16 of the cloud other than i, d = distances to the window points
// that differ from the point, d1 <= .. <= d8 the 8 smallest, padded with the
// largest when fewer, lref = mean log dk, dref = exp(lref)):
//   f0..f7   log dk - lref
//   f8       lref - log s_c,  s_c = (volume of the cloud's box / points)^(1/3)
//   f9       (w_i - mean window weight) / dref^2
//   f10..12  log(sorted extents of the window's box, >= 1e-6 dref) - lref
//   f13      |mean offset to the 8 nearest| / dref
//   f14      log(max(distance to the cloud's box faces, 1e-6 dref)) - lref
//   f15      (window points with d <= 2 dref) / 32
// A point without a distinct window point has all features 0 and no radius.
//
// Matrix products use mma.sync.m16n8k16 (BF16 in, FP32 accumulate): a warp
// owns 16 rows (points or training samples); the FP32 accumulator fragment of
// one layer is, after ReLU and BF16 rounding, exactly the A fragment of the
// next layer, so activations stay in registers in the forward pass. Weight
// gradients contract over the samples: a block stages 64 samples' activations
// and deltas transposed in shared memory and each warp owns a 16-row slice of
// every weight gradient across all chunks of the batch.
#include <atomic>
#include <cuda_bf16.h>

#include "../../include/paragram_b200.h"
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

constexpr int kF = 16;       // features
constexpr int kH = 64;       // hidden units
constexpr int kO = 2;        // outputs: log radius, neighbour count / 16
constexpr int kHalfWin = 16; // window half width
constexpr int kNParam = kH * kF + kH + kH * kH + kH + kO * kH + kO;
static_assert(kNParam == 5378, "flat parameter layout");
// offsets in the flat parameter vector: w1 [64][16], b1, w2 [64][64], b2, w3 [2][64], b3
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kO * kH;

// shared-memory row strides (BF16 elements): 16-byte padding keeps the fragment loads conflict free
constexpr int kS16 = kF + 8;  // rows of 16
constexpr int kS64 = kH + 8;  // rows of 64

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi); // .x = lo (low half), .y = hi
    return *reinterpret_cast<unsigned *>(&v);
}

__device__ __forceinline__ unsigned ld32(const __nv_bfloat16 *base, int row, int col, int stride)
{
    return *reinterpret_cast<const unsigned *>(base + row * stride + col);
}

__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------------------
// Features
// ---------------------------------------------------------------------------
struct CloudFrame
{
    float mn[3], mx[3];
    float ls; // log s_c
    int c0, c1;
};

__device__ __forceinline__ CloudFrame cloud_frame(const int *bounds, const int *cloud_off, int num_clouds, int i)
{
    CloudFrame f;
    int c = cloud_of(cloud_off, num_clouds, i);
    f.c0 = cloud_off[c];
    f.c1 = cloud_off[c + 1];
    float vol = 1.0f;
    for (int k = 0; k < 3; ++k)
    {
        f.mn[k] = ordered_to_float(bounds[c * 8 + k]);
        f.mx[k] = ordered_to_float(bounds[c * 8 + 3 + k]);
        vol *= fmaxf(f.mx[k] - f.mn[k], 1e-20f);
    }
    f.ls = logf(vol / (float)(f.c1 - f.c0)) * (1.0f / 3.0f);
    return f;
}

// Features of sorted slot i; returns false (features 0) without a distinct window point.
__device__ bool point_features(const float4 *__restrict__ pts, int i, const CloudFrame &cf, float (&f)[kF],
                               float &lref)
{
    float4 s = pts[i];
    float nd[8], ox[8], oy[8], oz[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        nd[k] = INFINITY;
        ox[k] = oy[k] = oz[k] = 0.0f;
    }
    int m = 0;
    float wsum = 0.0f;
    float bl[3] = {s.x, s.y, s.z}, bh[3] = {s.x, s.y, s.z};
    int lo = max(cf.c0, i - kHalfWin), hi = min(cf.c1 - 1, i + kHalfWin);
    float dall[2 * kHalfWin];
    int nall = 0;
    for (int j = lo; j <= hi; ++j)
    {
        if (j == i)
            continue;
        float4 q = pts[j];
        float dx = q.x - s.x, dy = q.y - s.y, dz = q.z - s.z;
        bl[0] = fminf(bl[0], q.x); bl[1] = fminf(bl[1], q.y); bl[2] = fminf(bl[2], q.z);
        bh[0] = fmaxf(bh[0], q.x); bh[1] = fmaxf(bh[1], q.y); bh[2] = fmaxf(bh[2], q.z);
        float d = sqrtf(dx * dx + dy * dy + dz * dz);
        if (!(d > 0.0f))
            continue;
        dall[nall++] = d;
        wsum += q.w;
        ++m;
        // insert into the 8 nearest (sorted ascending, stable)
        if (d < nd[7])
        {
            float cd = d, cx = dx, cy = dy, cz = dz;
#pragma unroll
            for (int k = 0; k < 8; ++k)
            {
                if (cd < nd[k])
                {
                    float t = nd[k]; nd[k] = cd; cd = t;
                    t = ox[k]; ox[k] = cx; cx = t;
                    t = oy[k]; oy[k] = cy; cy = t;
                    t = oz[k]; oz[k] = cz; cz = t;
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kF; ++k)
        f[k] = 0.0f;
    lref = 0.0f;
    if (m == 0)
        return false;
    int m8 = min(m, 8);
    float last = nd[m8 - 1];
    float logd[8], sum = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        logd[k] = logf(k < m8 ? nd[k] : last);
        sum += logd[k];
    }
    lref = sum * 0.125f;
    float dref = expf(lref);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        f[k] = logd[k] - lref;
    f[8] = lref - cf.ls;
    f[9] = (s.w - wsum / (float)m) / (dref * dref);
    float e[3];
    for (int k = 0; k < 3; ++k)
        e[k] = fmaxf(bh[k] - bl[k], 1e-6f * dref);
    // sort 3
    if (e[0] > e[1]) { float t = e[0]; e[0] = e[1]; e[1] = t; }
    if (e[1] > e[2]) { float t = e[1]; e[1] = e[2]; e[2] = t; }
    if (e[0] > e[1]) { float t = e[0]; e[0] = e[1]; e[1] = t; }
    f[10] = logf(e[0]) - lref;
    f[11] = logf(e[1]) - lref;
    f[12] = logf(e[2]) - lref;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        if (k < m8)
        {
            sx += ox[k];
            sy += oy[k];
            sz += oz[k];
        }
    f[13] = sqrtf(sx * sx + sy * sy + sz * sz) / ((float)m8 * dref);
    float face = fminf(fminf(fminf(s.x - cf.mn[0], cf.mx[0] - s.x), fminf(s.y - cf.mn[1], cf.mx[1] - s.y)),
                       fminf(s.z - cf.mn[2], cf.mx[2] - s.z));
    f[14] = logf(fmaxf(face, 1e-6f * dref)) - lref;
    int close = 0;
    for (int k = 0; k < nall; ++k)
        close += dall[k] <= 2.0f * dref;
    f[15] = (float)close * (1.0f / 32.0f);
    return true;
}

// Features per original index (training inputs).
__global__ void k_features(int64_t n, const float4 *__restrict__ pts, const int *__restrict__ oid,
                           const int *__restrict__ bounds, const int *__restrict__ cloud_off, int num_clouds,
                           float *__restrict__ out)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    CloudFrame cf = cloud_frame(bounds, cloud_off, num_clouds, (int)i);
    float f[kF], lref;
    point_features(pts, (int)i, cf, f, lref);
    float4 *o = reinterpret_cast<float4 *>(out + (size_t)oid[i] * kF);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        o[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
}

// ---------------------------------------------------------------------------
// The network
// ---------------------------------------------------------------------------
struct MlpSmem
{
    __nv_bfloat16 w1[kH * kS16];  // [out][in]
    __nv_bfloat16 w2[kH * kS64];  // [out][in]
    __nv_bfloat16 w3[8 * kS64];   // [out][in], rows 2..7 zero
    __nv_bfloat16 w2t[kH * kS64]; // [in][out]
    __nv_bfloat16 w3t[kH * kS16]; // [in][out], columns 2..15 zero
    float b1[kH], b2[kH], b3[8];
    float mean[kF], scale[kF];
    float tmean[kO], tscale[kO], margin, route;
};

__device__ void load_model(MlpSmem &S, const pg_model *M, bool transposed)
{
    const __nv_bfloat16 *w1 = reinterpret_cast<const __nv_bfloat16 *>(M->w1);
    const __nv_bfloat16 *w2 = reinterpret_cast<const __nv_bfloat16 *>(M->w2);
    const __nv_bfloat16 *w3 = reinterpret_cast<const __nv_bfloat16 *>(M->w3);
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    for (int t = threadIdx.x; t < kH * kF; t += blockDim.x)
        S.w1[(t / kF) * kS16 + t % kF] = w1[t];
    for (int t = threadIdx.x; t < kH * kH; t += blockDim.x)
    {
        int r = t / kH, c = t % kH;
        S.w2[r * kS64 + c] = w2[t];
        if (transposed)
            S.w2t[c * kS64 + r] = w2[t];
    }
    for (int t = threadIdx.x; t < 8 * kH; t += blockDim.x)
    {
        int r = t / kH, c = t % kH;
        __nv_bfloat16 v = r < kO ? w3[t] : zero;
        S.w3[r * kS64 + c] = v;
    }
    if (transposed)
        for (int t = threadIdx.x; t < kH * kS16; t += blockDim.x)
        {
            int r = t / kS16, c = t % kS16; // r = hidden unit, c = output
            S.w3t[t] = c < kO ? w3[c * kH + r] : zero;
        }
    for (int t = threadIdx.x; t < kH; t += blockDim.x)
    {
        S.b1[t] = M->b1[t];
        S.b2[t] = M->b2[t];
    }
    if (threadIdx.x < 8)
        S.b3[threadIdx.x] = threadIdx.x < kO ? M->b3[threadIdx.x] : 0.0f;
    if (threadIdx.x < kF)
    {
        S.mean[threadIdx.x] = M->feat_mean[threadIdx.x];
        S.scale[threadIdx.x] = M->feat_scale[threadIdx.x];
    }
    if (threadIdx.x < kO)
    {
        S.tmean[threadIdx.x] = M->target_mean[threadIdx.x];
        S.tscale[threadIdx.x] = M->target_scale[threadIdx.x];
    }
    if (threadIdx.x == 0)
        S.margin = M->radius_margin;
        S.route = M->route_degree;
}

// Forward pass of one 16-row tile. ax: A fragments of the normalized BF16
// features. Outputs: y (lanes with t == 0 hold rows g and g + 8, columns 0, 1
// in y[0..1] and y[2..3]); h1/h2: A fragments of the hidden activations
// (after ReLU, BF16) for 4 k-steps; pos1/pos2: bit (j * 4 + e) set when the
// pre-activation of accumulator element e of column tile j is > 0.
struct Fwd
{
    float y[4];
    unsigned h1[4][4], h2[4][4];
    unsigned pos1, pos2;
};

__device__ __forceinline__ void mlp_tile_forward(const MlpSmem &S, const unsigned (&ax)[4], int lane, Fwd &F)
{
    const int g = lane >> 2, t = lane & 3;
    float c[8][4];
    // layer 1: [16 x 16] x [16 x 64]
#pragma unroll
    for (int j = 0; j < 8; ++j)
    {
        float b0 = S.b1[8 * j + 2 * t], b1 = S.b1[8 * j + 2 * t + 1];
        c[j][0] = b0; c[j][1] = b1; c[j][2] = b0; c[j][3] = b1;
        mma16816(c[j], ax, ld32(S.w1, 8 * j + g, 2 * t, kS16), ld32(S.w1, 8 * j + g, 2 * t + 8, kS16));
    }
    F.pos1 = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (c[j][e] > 0.0f)
                F.pos1 |= 1u << (j * 4 + e);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
    {
        F.h1[kk][0] = pack_bf16(fmaxf(c[2 * kk][0], 0.0f), fmaxf(c[2 * kk][1], 0.0f));
        F.h1[kk][1] = pack_bf16(fmaxf(c[2 * kk][2], 0.0f), fmaxf(c[2 * kk][3], 0.0f));
        F.h1[kk][2] = pack_bf16(fmaxf(c[2 * kk + 1][0], 0.0f), fmaxf(c[2 * kk + 1][1], 0.0f));
        F.h1[kk][3] = pack_bf16(fmaxf(c[2 * kk + 1][2], 0.0f), fmaxf(c[2 * kk + 1][3], 0.0f));
    }
    // layer 2: [16 x 64] x [64 x 64]
#pragma unroll
    for (int j = 0; j < 8; ++j)
    {
        float b0 = S.b2[8 * j + 2 * t], b1 = S.b2[8 * j + 2 * t + 1];
        c[j][0] = b0; c[j][1] = b1; c[j][2] = b0; c[j][3] = b1;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            mma16816(c[j], F.h1[kk], ld32(S.w2, 8 * j + g, 16 * kk + 2 * t, kS64),
                     ld32(S.w2, 8 * j + g, 16 * kk + 2 * t + 8, kS64));
    }
    F.pos2 = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (c[j][e] > 0.0f)
                F.pos2 |= 1u << (j * 4 + e);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
    {
        F.h2[kk][0] = pack_bf16(fmaxf(c[2 * kk][0], 0.0f), fmaxf(c[2 * kk][1], 0.0f));
        F.h2[kk][1] = pack_bf16(fmaxf(c[2 * kk][2], 0.0f), fmaxf(c[2 * kk][3], 0.0f));
        F.h2[kk][2] = pack_bf16(fmaxf(c[2 * kk + 1][0], 0.0f), fmaxf(c[2 * kk + 1][1], 0.0f));
        F.h2[kk][3] = pack_bf16(fmaxf(c[2 * kk + 1][2], 0.0f), fmaxf(c[2 * kk + 1][3], 0.0f));
    }
    // layer 3: [16 x 64] x [64 x 8] (outputs 2..7 are padding)
    float b0 = S.b3[2 * t], b1 = S.b3[2 * t + 1];
    F.y[0] = b0; F.y[1] = b1; F.y[2] = b0; F.y[3] = b1;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
        mma16816(F.y, F.h2[kk], ld32(S.w3, g, 16 * kk + 2 * t, kS64), ld32(S.w3, g, 16 * kk + 2 * t + 8, kS64));
}

// A fragments of 16 normalized feature rows stored row-major (BF16) in shared memory.
__device__ __forceinline__ void feature_fragments(const __nv_bfloat16 *xr, int lane, unsigned (&ax)[4])
{
    const int g = lane >> 2, t = lane & 3;
    ax[0] = ld32(xr, g, 2 * t, kS16);
    ax[1] = ld32(xr, g + 8, 2 * t, kS16);
    ax[2] = ld32(xr, g, 2 * t + 8, kS16);
    ax[3] = ld32(xr, g + 8, 2 * t + 8, kS16);
}

__device__ __forceinline__ void store_normalized(const MlpSmem &S, const float (&f)[kF], __nv_bfloat16 *row)
{
#pragma unroll
    for (int k = 0; k < kF; ++k)
        row[k] = __float2bfloat16_rn((f[k] - S.mean[k]) * S.scale[k]);
}

// Where the prediction lists the cells it routes past the first pass.
struct Route
{
    int *counters;   // [1]: deferred cells, [7]: routing requests
    int *big_list;   // deferred sorted slots
    int *deg;        // directed degree by original index
    int *status;     // status by original index
    const int *oid;  // sorted slot -> original index
    int64_t cap;     // at most this many routed cells
};

// A routed cell: listed for the 128-slot tier with a placeholder row (an empty row whose
// plane_overflow status the deferred pass replaces), while the routing share lasts.
__device__ __forceinline__ bool route_cell(const Route &rt, int64_t i)
{
    if ((int64_t)atomicAdd(&rt.counters[7], 1) >= rt.cap)
        return false;
    int d = atomicAdd(&rt.counters[1], 1);
    rt.big_list[d] = (int)i;
    int o = rt.oid[i];
    rt.deg[o] = 0;
    rt.status[o] = kPlaneOverflow;
    return true;
}

// Search radius of each sorted slot from its features (the cell pass's cap).
// Block = 8 warps, a warp predicts 32 consecutive slots.
__global__ void __launch_bounds__(256) k_mlp_predict(int64_t n, const float4 *__restrict__ pts,
                                                     const int *__restrict__ bounds, const int *__restrict__ cloud_off,
                                                     int num_clouds, const pg_model *__restrict__ model,
                                                     float *__restrict__ hint, Route rt)
{
    __shared__ MlpSmem S;
    __shared__ __align__(16) __nv_bfloat16 xr[8][32 * kS16];
    __shared__ float lr[8][32];
    load_model(S, model, false);
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    for (int64_t base = ((int64_t)blockIdx.x * 8 + w) * 32; base < n; base += (int64_t)gridDim.x * 8 * 32)
    {
        int64_t i = base + lane;
        float f[kF], lref = 0.0f;
        bool ok = false;
        if (i < n)
        {
            CloudFrame cf = cloud_frame(bounds, cloud_off, num_clouds, (int)i);
            ok = point_features(pts, (int)i, cf, f, lref);
        }
        else
        {
#pragma unroll
            for (int k = 0; k < kF; ++k)
                f[k] = 0.0f;
        }
        store_normalized(S, f, &xr[w][lane * kS16]);
        lr[w][lane] = ok ? lref : NAN;
        __syncwarp();
#pragma unroll
        for (int tile = 0; tile < 2; ++tile)
        {
            unsigned ax[4];
            feature_fragments(&xr[w][tile * 16 * kS16], lane, ax);
            Fwd F;
            mlp_tile_forward(S, ax, lane, F);
            if (t == 0)
            {
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    int r = tile * 16 + g + 8 * h;
                    int64_t ir = base + r;
                    float lref_r = lr[w][r];
                    if (ir < n)
                    {
                        float ly = F.y[2 * h] / S.tscale[0] + S.tmean[0] + S.margin + lref_r;
                        float rad = expf(ly);
                        // a predicted neighbour count at or above route_degree: the cell is listed
                        // for the 128-slot tier and its radius negated (the first pass skips it)
                        float deg = (F.y[2 * h + 1] / S.tscale[1] + S.tmean[1]) * 16.0f;
                        bool ok_r = lref_r == lref_r && rad < 1e30f;
                        bool routed = ok_r && S.route > 0.0f && deg >= S.route && route_cell(rt, ir);
                        hint[ir] = ok_r ? (routed ? -rad : rad) : 0.0f;
                    }
                }
            }
        }
        __syncwarp();
    }
}

// Outputs [n][2] of the network on raw features [n][16] (evaluation).
__global__ void __launch_bounds__(256) k_mlp_forward(int64_t n, const float *__restrict__ x,
                                                     const pg_model *__restrict__ model, float *__restrict__ y)
{
    __shared__ MlpSmem S;
    __shared__ __align__(16) __nv_bfloat16 xr[8][16 * kS16];
    load_model(S, model, false);
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    for (int64_t base = ((int64_t)blockIdx.x * 8 + w) * 16; base < n; base += (int64_t)gridDim.x * 8 * 16)
    {
        if (lane < 16)
        {
            float f[kF];
            int64_t i = base + lane;
#pragma unroll
            for (int k = 0; k < kF; ++k)
                f[k] = i < n ? x[i * kF + k] : 0.0f;
            store_normalized(S, f, &xr[w][lane * kS16]);
        }
        __syncwarp();
        unsigned ax[4];
        feature_fragments(xr[w], lane, ax);
        Fwd F;
        mlp_tile_forward(S, ax, lane, F);
        if (t == 0)
            for (int h = 0; h < 2; ++h)
            {
                int64_t i = base + g + 8 * h;
                if (i < n)
                {
                    y[i * kO] = F.y[2 * h];
                    y[i * kO + 1] = F.y[2 * h + 1];
                }
            }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Training: loss and gradient of a batch
// ---------------------------------------------------------------------------
constexpr int kChunk = 64; // samples per block step (4 warps x 16)

struct GradSmem
{
    MlpSmem M;
    __nv_bfloat16 xr[kChunk * kS16]; // normalized features, row-major [sample][feature]
    __nv_bfloat16 xt[kF * (kChunk + 8)];   // [feature][sample]
    __nv_bfloat16 h1t[kH * (kChunk + 8)];  // [unit][sample]
    __nv_bfloat16 h2t[kH * (kChunk + 8)];
    __nv_bfloat16 d1t[kH * (kChunk + 8)];
    __nv_bfloat16 d2t[kH * (kChunk + 8)];
    __nv_bfloat16 dyt[16 * (kChunk + 8)];  // [output][sample], rows 2..15 zero
};
constexpr int kSC = kChunk + 8;
static_assert(sizeof(pg_model) == 11984, "pg_model layout");
static_assert(sizeof(GradSmem) <= 200 * 1024, "k_mlp_grad shared memory");

// Writes the 16 x 64 tile held as A fragments (4 k-steps) transposed into dst[unit][sample].
__device__ __forceinline__ void store_t64(__nv_bfloat16 *dst, const unsigned (&a)[4][4], int s0, int lane)
{
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
#pragma unroll
        for (int r = 0; r < 4; ++r)
        {
            int row = g + ((r & 1) ? 8 : 0);
            int col = 16 * kk + 2 * t + ((r & 2) ? 8 : 0);
            __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(&a[kk][r]);
            dst[col * kSC + s0 + row] = v.x;
            dst[(col + 1) * kSC + s0 + row] = v.y;
        }
}

__global__ void __launch_bounds__(128) k_mlp_grad(int64_t n, const float *__restrict__ x, const float *__restrict__ tgt,
                                                  const float *__restrict__ sw, float inv_total,
                                                  const pg_model *__restrict__ model, float *__restrict__ grad,
                                                  float *__restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
    load_model(S.M, model, true);
    for (int k = threadIdx.x; k < 16 * kSC; k += blockDim.x)
        S.dyt[k] = __float2bfloat16_rn(0.0f);
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    float aw2[8][4], aw1[2][4], aw3[2][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            aw2[j][e] = 0.0f;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            aw1[j][e] = aw3[j][e] = 0.0f;
    float ab1 = 0.0f, ab2 = 0.0f, ab3 = 0.0f, lsum = 0.0f;
    for (int64_t base = (int64_t)blockIdx.x * kChunk; base < n; base += (int64_t)gridDim.x * kChunk)
    {
        // 1. stage normalized features (row-major and transposed)
        for (int k = threadIdx.x; k < kChunk * kF; k += blockDim.x)
        {
            int s = k / kF, f = k % kF;
            int64_t i = base + s;
            float v = i < n ? x[i * kF + f] : 0.0f;
            __nv_bfloat16 b = __float2bfloat16_rn((v - S.M.mean[f]) * S.M.scale[f]);
            S.xr[s * kS16 + f] = b;
            S.xt[f * kSC + s] = b;
        }
        __syncthreads();
        // 2. forward and backward of this warp's 16 samples
        const int s0 = 16 * w;
        unsigned ax[4];
        feature_fragments(&S.xr[s0 * kS16], lane, ax);
        Fwd F;
        mlp_tile_forward(S.M, ax, lane, F);
        store_t64(S.h1t, F.h1, s0, lane);
        store_t64(S.h2t, F.h2, s0, lane);
        // dy = sw (y - t') / total, rows g and g + 8, outputs 0, 1 (lanes with t == 0)
        float dy[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (t == 0)
        {
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                int64_t i = base + s0 + g + 8 * h;
                if (i < n)
                {
                    float wgt = sw[i];
#pragma unroll
                    for (int o = 0; o < 2; ++o)
                    {
                        float tn = (tgt[i * kO + o] - S.M.tmean[o]) * S.M.tscale[o];
                        float r = F.y[2 * h + o] - tn;
                        lsum += wgt * r * r;
                        dy[2 * h + o] = wgt * r * inv_total;
                    }
                }
            }
        }
        unsigned ady[4] = {pack_bf16(dy[0], dy[1]), pack_bf16(dy[2], dy[3]), 0u, 0u};
        if (t == 0)
        {
            __nv_bfloat162 v0 = *reinterpret_cast<__nv_bfloat162 *>(&ady[0]);
            __nv_bfloat162 v1 = *reinterpret_cast<__nv_bfloat162 *>(&ady[1]);
            S.dyt[0 * kSC + s0 + g] = v0.x;
            S.dyt[1 * kSC + s0 + g] = v0.y;
            S.dyt[0 * kSC + s0 + g + 8] = v1.x;
            S.dyt[1 * kSC + s0 + g + 8] = v1.y;
        }
        // dh2 = (dy W3) * [a2 > 0]
        float c[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
            c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.0f;
            mma16816(c[j], ady, ld32(S.M.w3t, 8 * j + g, 2 * t, kS16), ld32(S.M.w3t, 8 * j + g, 2 * t + 8, kS16));
        }
        unsigned d2[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
        {
            float v[2][4];
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    v[hh][e] = ((F.pos2 >> ((2 * kk + hh) * 4 + e)) & 1u) ? c[2 * kk + hh][e] : 0.0f;
            d2[kk][0] = pack_bf16(v[0][0], v[0][1]);
            d2[kk][1] = pack_bf16(v[0][2], v[0][3]);
            d2[kk][2] = pack_bf16(v[1][0], v[1][1]);
            d2[kk][3] = pack_bf16(v[1][2], v[1][3]);
        }
        store_t64(S.d2t, d2, s0, lane);
        // dh1 = (dh2 W2) * [a1 > 0]
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
            c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.0f;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                mma16816(c[j], d2[kk], ld32(S.M.w2t, 8 * j + g, 16 * kk + 2 * t, kS64),
                         ld32(S.M.w2t, 8 * j + g, 16 * kk + 2 * t + 8, kS64));
        }
        unsigned d1[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
        {
            float v[2][4];
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    v[hh][e] = ((F.pos1 >> ((2 * kk + hh) * 4 + e)) & 1u) ? c[2 * kk + hh][e] : 0.0f;
            d1[kk][0] = pack_bf16(v[0][0], v[0][1]);
            d1[kk][1] = pack_bf16(v[0][2], v[0][3]);
            d1[kk][2] = pack_bf16(v[1][0], v[1][1]);
            d1[kk][3] = pack_bf16(v[1][2], v[1][3]);
        }
        store_t64(S.d1t, d1, s0, lane);
        __syncthreads();
        // 3. weight gradients over the chunk's 64 samples (K = samples)
        // dW2 [64 x 64] = d2t x h1t^T: warp w owns rows 16w..16w+15
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
        {
            unsigned a[4] = {ld32(S.d2t, 16 * w + g, 16 * ks + 2 * t, kSC), ld32(S.d2t, 16 * w + g + 8, 16 * ks + 2 * t, kSC),
                             ld32(S.d2t, 16 * w + g, 16 * ks + 2 * t + 8, kSC),
                             ld32(S.d2t, 16 * w + g + 8, 16 * ks + 2 * t + 8, kSC)};
#pragma unroll
            for (int j = 0; j < 8; ++j)
                mma16816(aw2[j], a, ld32(S.h1t, 8 * j + g, 16 * ks + 2 * t, kSC),
                         ld32(S.h1t, 8 * j + g, 16 * ks + 2 * t + 8, kSC));
            // dW1 [64 x 16] = d1t x xt^T
            unsigned a1[4] = {ld32(S.d1t, 16 * w + g, 16 * ks + 2 * t, kSC), ld32(S.d1t, 16 * w + g + 8, 16 * ks + 2 * t, kSC),
                              ld32(S.d1t, 16 * w + g, 16 * ks + 2 * t + 8, kSC),
                              ld32(S.d1t, 16 * w + g + 8, 16 * ks + 2 * t + 8, kSC)};
#pragma unroll
            for (int j = 0; j < 2; ++j)
                mma16816(aw1[j], a1, ld32(S.xt, 8 * j + g, 16 * ks + 2 * t, kSC),
                         ld32(S.xt, 8 * j + g, 16 * ks + 2 * t + 8, kSC));
            // dW3 [16 (2 used) x 64] = dyt x h2t^T: warp w owns columns 16w..16w+15
            unsigned a3[4] = {ld32(S.dyt, g, 16 * ks + 2 * t, kSC), ld32(S.dyt, g + 8, 16 * ks + 2 * t, kSC),
                              ld32(S.dyt, g, 16 * ks + 2 * t + 8, kSC), ld32(S.dyt, g + 8, 16 * ks + 2 * t + 8, kSC)};
#pragma unroll
            for (int j = 0; j < 2; ++j)
                mma16816(aw3[j], a3, ld32(S.h2t, 16 * w + 8 * j + g, 16 * ks + 2 * t, kSC),
                         ld32(S.h2t, 16 * w + 8 * j + g, 16 * ks + 2 * t + 8, kSC));
        }
        // bias gradients: row sums of the transposed deltas
        if (threadIdx.x < kH)
        {
            for (int s = 0; s < kChunk; ++s)
            {
                ab2 += __bfloat162float(S.d2t[threadIdx.x * kSC + s]);
                ab1 += __bfloat162float(S.d1t[threadIdx.x * kSC + s]);
            }
        }
        else if (threadIdx.x < kH + kO)
        {
            for (int s = 0; s < kChunk; ++s)
                ab3 += __bfloat162float(S.dyt[(threadIdx.x - kH) * kSC + s]);
        }
        __syncthreads();
    }
    // 4. add the block's partial sums to the batch gradient
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
        {
            int r = 16 * w + g + ((e & 2) ? 8 : 0), cc = 8 * j + 2 * t + (e & 1);
            atomicAdd(&grad[kOffW2 + r * kH + cc], aw2[j][e]);
        }
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
        {
            int r = 16 * w + g + ((e & 2) ? 8 : 0), cc = 8 * j + 2 * t + (e & 1);
            atomicAdd(&grad[kOffW1 + r * kF + cc], aw1[j][e]);
            int r3 = g + ((e & 2) ? 8 : 0), c3 = 16 * w + 8 * j + 2 * t + (e & 1);
            if (r3 < kO)
                atomicAdd(&grad[kOffW3 + r3 * kH + c3], aw3[j][e]);
        }
    if (threadIdx.x < kH)
    {
        atomicAdd(&grad[kOffB1 + threadIdx.x], ab1);
        atomicAdd(&grad[kOffB2 + threadIdx.x], ab2);
    }
    else if (threadIdx.x < kH + kO)
        atomicAdd(&grad[kOffB3 + threadIdx.x - kH], ab3);
    // loss: sum of the lanes' weighted squared errors / (2 total)
    for (int o = 16; o > 0; o >>= 1)
        lsum += __shfl_xor_sync(0xFFFFFFFFu, lsum, o);
    if (lane == 0)
        atomicAdd(loss, 0.5f * lsum * inv_total);
}

// One Adam step on the FP32 master weights; writes the BF16 weights and FP32
// biases of the model.
__global__ void k_mlp_adam(float *__restrict__ params, const float *__restrict__ grad, float *__restrict__ m,
                           float *__restrict__ v, float lr, float beta1, float beta2, float eps, float c1, float c2,
                           pg_model *__restrict__ model)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNParam)
        return;
    float gr = grad[p];
    float mm = beta1 * m[p] + (1.0f - beta1) * gr;
    float vv = beta2 * v[p] + (1.0f - beta2) * gr * gr;
    m[p] = mm;
    v[p] = vv;
    float val = params[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    params[p] = val;
    __nv_bfloat16 b = __float2bfloat16_rn(val);
    unsigned short bits = *reinterpret_cast<unsigned short *>(&b);
    if (p < kOffB1)
        model->w1[p - kOffW1] = bits;
    else if (p < kOffW2)
        model->b1[p - kOffB1] = val;
    else if (p < kOffB2)
        model->w2[p - kOffW2] = bits;
    else if (p < kOffW3)
        model->b2[p - kOffB2] = val;
    else if (p < kOffB3)
        model->w3[p - kOffW3] = bits;
    else
        model->b3[p - kOffB3] = val;
}

// Copies FP32 master weights into the model (BF16 weights, FP32 biases).
__global__ void k_mlp_pack(const float *__restrict__ params, pg_model *__restrict__ model)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNParam)
        return;
    float val = params[p];
    __nv_bfloat16 b = __float2bfloat16_rn(val);
    unsigned short bits = *reinterpret_cast<unsigned short *>(&b);
    if (p < kOffB1)
        model->w1[p - kOffW1] = bits;
    else if (p < kOffW2)
        model->b1[p - kOffB1] = val;
    else if (p < kOffB2)
        model->w2[p - kOffW2] = bits;
    else if (p < kOffW3)
        model->b2[p - kOffB2] = val;
    else if (p < kOffB3)
        model->w3[p - kOffW3] = bits;
    else
        model->b3[p - kOffB3] = val;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
void features_launch(const Workspace &ws, int64_t n, int num_clouds, float *out, cudaStream_t st)
{
    ++g_launches;
    k_features<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, ws.pts, ws.oid, ws.bounds, ws.cloud_off, num_clouds,
                                                             out);
}

void predict_launch(const Workspace &ws, int64_t n, int num_clouds, const pg_model *model, int *status,
                    int64_t route_cap, cudaStream_t st)
{
    int64_t warps = (n + 31) / 32;
    int64_t grid = std::min<int64_t>((warps + 7) / 8, 148 * 8);
    Route rt{ws.counters, ws.big_list, ws.deg, status, ws.oid, route_cap};
    ++g_launches;
    k_mlp_predict<<<(unsigned)std::max<int64_t>(grid, 1), 256, 0, st>>>(n, ws.pts, ws.bounds, ws.cloud_off,
                                                                        num_clouds, model, ws.hint, rt);
}

} // namespace pg

using namespace pg;

extern "C" {

int pg_mlp_num_params(void) { return kNParam; }

size_t pg_mlp_model_bytes(void) { return sizeof(pg_model); }

int pg_mlp_forward(int64_t n, const float *features, const void *model, float *out, void *stream)
{
    if (n < 0 || (n > 0 && (!features || !model || !out)))
        return set_last_error(PG_ERR_INVALID, "pg_mlp_forward: bad arguments");
    if (n == 0)
        return PG_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int64_t tiles = (n + 15) / 16;
    int64_t grid = std::min<int64_t>((tiles + 7) / 8, 148 * 8);
    k_mlp_forward<<<(unsigned)grid, 256, 0, st>>>(n, features, (const pg_model *)model, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PG_OK : set_last_error(PG_ERR_CUDA, cudaGetErrorString(e));
}

int pg_mlp_grad(int64_t n, const float *features, const float *targets, const float *sample_weights,
                float inv_total_weight, const void *model, float *grad, float *loss, void *stream)
{
    if (n < 0 || (n > 0 && (!features || !targets || !sample_weights || !model || !grad || !loss)))
        return set_last_error(PG_ERR_INVALID, "pg_mlp_grad: bad arguments");
    if (n == 0)
        return PG_OK;
    cudaStream_t st = (cudaStream_t)stream;
    size_t smem = sizeof(GradSmem);
    // the shared-memory opt-in is a per-device attribute of the kernel: set once per device
    static std::atomic<unsigned long long> attr{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr.load() & bit))
    {
        cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr.fetch_or(bit);
    }
    int64_t chunks = (n + kChunk - 1) / kChunk;
    int64_t grid = std::min<int64_t>(chunks, 148 * 4);
    k_mlp_grad<<<(unsigned)grid, 128, smem, st>>>(n, features, targets, sample_weights, inv_total_weight,
                                                  (const pg_model *)model, grad, loss);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PG_OK : set_last_error(PG_ERR_CUDA, cudaGetErrorString(e));
}

int pg_mlp_adam(float *params, const float *grad, float *m, float *v, int64_t step, float lr, float beta1,
                float beta2, float eps, void *model, void *stream)
{
    if (!params || !grad || !m || !v || !model || step < 1)
        return set_last_error(PG_ERR_INVALID, "pg_mlp_adam: bad arguments");
    float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_mlp_adam<<<(kNParam + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, lr, beta1, beta2, eps, c1,
                                                                        c2, (pg_model *)model);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PG_OK : set_last_error(PG_ERR_CUDA, cudaGetErrorString(e));
}

int pg_mlp_pack(const float *params, void *model, void *stream)
{
    if (!params || !model)
        return set_last_error(PG_ERR_INVALID, "pg_mlp_pack: bad arguments");
    k_mlp_pack<<<(kNParam + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, (pg_model *)model);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PG_OK : set_last_error(PG_ERR_CUDA, cudaGetErrorString(e));
}

} // extern "C"
