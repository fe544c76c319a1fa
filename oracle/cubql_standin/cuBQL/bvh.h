// Stand-in for the few names of NVIDIA/cuBQL that the reference's CUDA
// extension uses (pinned cuBQL version unknown: the reference's submodule
// paragram/external/cubql is empty). TEST INFRASTRUCTURE ONLY: it lets the
// unmodified reference kernels (paragram/csrc/laguerre/*.cu) be compiled into
// oracle/_ref/ and run as a parity and timing baseline. Nothing in the
// paragram_b200 product includes it.
//
// Names and layouts follow their uses in the reference:
//   vec_t<float, 3> (12-byte x, y, z; reinterpret-cast from an (N, 3) float
//     array, pwr_bvh.cu:247-252), box_t (lower, upper, pwr_bvh.cu:36-37),
//   BinaryBVH<float, 3> with node_t {bounds, admin{offset:48, count:16} |
//     offsetAndCountBits}, nodes / numNodes / primIDs / numPrims
//     (pwr_bvh.cu:56-75, voronoi_bvh.cuh:164-246): an inner node's children are
//     nodes[offset] and nodes[offset + 1]; a leaf lists primIDs[offset ..
//     offset + count); the root is nodes[0];
//   BuildConfig::makeLeafThreshold and gpuBuilder (pwr_bvh.cu:234-240).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#ifndef CUBQL_ALIGN
#define CUBQL_ALIGN(a) __align__(a)
#endif

namespace cuBQL
{

template <typename T, int D> struct vec_t;

template <typename T> struct vec_t<T, 3>
{
    T x, y, z;
};

template <typename T> __host__ __device__ inline vec_t<T, 3> operator-(vec_t<T, 3> a, T s)
{
    return vec_t<T, 3>{a.x - s, a.y - s, a.z - s};
}
template <typename T> __host__ __device__ inline vec_t<T, 3> operator+(vec_t<T, 3> a, T s)
{
    return vec_t<T, 3>{a.x + s, a.y + s, a.z + s};
}

template <typename T, int D> struct box_t
{
    vec_t<T, D> lower, upper;
};

template <typename T, int D> struct BinaryBVH
{
    using scalar_t = T;
    using vec_t = cuBQL::vec_t<T, D>;
    using box_t = cuBQL::box_t<T, D>;

    struct CUBQL_ALIGN(16) Node
    {
        enum
        {
            count_bits = 16,
            offset_bits = 64 - count_bits
        };
        box_t bounds;
        struct Admin
        {
            union
            {
                struct
                {
                    uint64_t offset : offset_bits;
                    uint64_t count : count_bits; // 0 for an inner node
                };
                uint64_t offsetAndCountBits;
            };
        };
        Admin admin;
    };
    using node_t = Node;

    node_t *nodes = 0;
    uint32_t numNodes = 0;
    uint32_t *primIDs = 0;
    uint32_t numPrims = 0;
};

struct BuildConfig
{
    // a node with at most this many primitives becomes a leaf
    int makeLeafThreshold = 1;
};

// Builds `bvh` over n boxes in device memory (nodes and primIDs are cudaMalloc'ed;
// the reference frees them with cudaFree). Defined in builder/cuda.h.
template <typename T, int D>
void gpuBuilder(BinaryBVH<T, D> &bvh, const box_t<T, D> *d_boxes, uint32_t n, BuildConfig config,
                cudaStream_t stream = 0);

} // namespace cuBQL
