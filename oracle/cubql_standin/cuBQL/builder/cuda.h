// Stand-in for cuBQL::gpuBuilder (TEST INFRASTRUCTURE ONLY; see cuBQL/bvh.h).
//
// A binary BVH over the boxes (points, as the reference passes them), built
// on the host and uploaded: top-down median split along the longest axis of
// the node's centroid bounds (ties by primitive index, so the tree is
// deterministic), a leaf as soon as a node holds at most makeLeafThreshold
// primitives. Children of a node are allocated as an adjacent pair. The
// reference's outputs depend on the tree only through the order in which its
// traversal meets candidates (which decides FP32 rounding near degeneracies and
// its capacity statuses), never on its correctness.
#pragma once

#include <algorithm>
#include <cstdio>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "../bvh.h"

namespace cuBQL
{

namespace standin
{
// The tree over n host boxes: nodes (root first, children as adjacent pairs) and
// the primitive permutation `prim` the leaves index into.
template <typename T, int D>
std::vector<typename BinaryBVH<T, D>::Node> build_host(const box_t<T, D> *boxes, uint32_t n, int threshold,
                                                       std::vector<uint32_t> &prim)
{
    static_assert(D == 3, "the stand-in builds 3-D trees only");
    using Node = typename BinaryBVH<T, D>::Node;
    prim.resize(n);
    std::iota(prim.begin(), prim.end(), 0u);
    std::vector<Node> nodes;
    if (n == 0)
        return nodes;
    std::vector<T> cen[3];
    for (int a = 0; a < 3; ++a)
        cen[a].resize(n);
    for (uint32_t i = 0; i < n; ++i)
    {
        cen[0][i] = (boxes[i].lower.x + boxes[i].upper.x) * T(0.5);
        cen[1][i] = (boxes[i].lower.y + boxes[i].upper.y) * T(0.5);
        cen[2][i] = (boxes[i].lower.z + boxes[i].upper.z) * T(0.5);
    }
    const uint32_t leaf = (uint32_t)std::min(std::max(threshold, 1), 65535);
    nodes.resize(1);
    nodes.reserve(2 * (size_t)n / leaf + 2);
    struct Task
    {
        uint32_t node, begin, end;
    };
    std::vector<Task> todo{{0u, 0u, n}};
    while (!todo.empty())
    {
        Task t = todo.back();
        todo.pop_back();
        box_t<T, D> b = boxes[prim[t.begin]];
        T clo[3] = {cen[0][prim[t.begin]], cen[1][prim[t.begin]], cen[2][prim[t.begin]]};
        T chi[3] = {clo[0], clo[1], clo[2]};
        for (uint32_t i = t.begin + 1; i < t.end; ++i)
        {
            const box_t<T, D> &q = boxes[prim[i]];
            b.lower.x = std::min(b.lower.x, q.lower.x);
            b.lower.y = std::min(b.lower.y, q.lower.y);
            b.lower.z = std::min(b.lower.z, q.lower.z);
            b.upper.x = std::max(b.upper.x, q.upper.x);
            b.upper.y = std::max(b.upper.y, q.upper.y);
            b.upper.z = std::max(b.upper.z, q.upper.z);
            for (int a = 0; a < 3; ++a)
            {
                clo[a] = std::min(clo[a], cen[a][prim[i]]);
                chi[a] = std::max(chi[a], cen[a][prim[i]]);
            }
        }
        const uint32_t cnt = t.end - t.begin;
        Node node{};
        node.bounds = b;
        if (cnt <= leaf)
        {
            node.admin.offset = t.begin;
            node.admin.count = cnt;
            nodes[t.node] = node;
            continue;
        }
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (chi[a] - clo[a] > chi[axis] - clo[axis])
                axis = a;
        const std::vector<T> &c = cen[axis];
        const uint32_t mid = t.begin + cnt / 2;
        std::nth_element(prim.begin() + t.begin, prim.begin() + mid, prim.begin() + t.end,
                         [&c](uint32_t x, uint32_t y) { return c[x] < c[y] || (c[x] == c[y] && x < y); });
        const uint32_t child = (uint32_t)nodes.size();
        node.admin.offset = child;
        node.admin.count = 0;
        nodes[t.node] = node;
        nodes.emplace_back();
        nodes.emplace_back();
        todo.push_back({child + 1, mid, t.end});
        todo.push_back({child, t.begin, mid});
    }
    return nodes;
}
} // namespace standin

template <typename T, int D>
void gpuBuilder(BinaryBVH<T, D> &bvh, const box_t<T, D> *d_boxes, uint32_t n, BuildConfig config,
                cudaStream_t stream)
{
    using Node = typename BinaryBVH<T, D>::Node;
    bvh.nodes = nullptr;
    bvh.primIDs = nullptr;
    bvh.numNodes = 0;
    bvh.numPrims = 0;
    if (n == 0)
        return;
    std::vector<box_t<T, D>> boxes(n);
    if (cudaStreamSynchronize(stream) != cudaSuccess ||
        cudaMemcpy(boxes.data(), d_boxes, sizeof(box_t<T, D>) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("cuBQL stand-in: reading the boxes failed");
    std::vector<uint32_t> prim;
    std::vector<Node> nodes = standin::build_host(boxes.data(), n, config.makeLeafThreshold, prim);
    bvh.numNodes = (uint32_t)nodes.size();
    bvh.numPrims = n;
    if (cudaMalloc(&bvh.nodes, sizeof(Node) * nodes.size()) != cudaSuccess ||
        cudaMalloc(&bvh.primIDs, sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMemcpy(bvh.nodes, nodes.data(), sizeof(Node) * nodes.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(bvh.primIDs, prim.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("cuBQL stand-in: uploading the tree failed");
}

} // namespace cuBQL
