// Stand-in for cuBQL::points::findKNN (TEST INFRASTRUCTURE ONLY; see
// cuBQL/bvh.h): the k nearest points of a query by a depth-first BVH
// traversal, nearer child first, pruning nodes whose box is not closer than the
// current k-th candidate. The caller's candidate array (primID -1, sqrDist
// +inf on entry, pwr_bvh.cu:186-191) is kept sorted by increasing squared
// distance; a candidate replaces the k-th only when strictly closer, so equal
// distances keep the one met first. Result::numFound counts the filled slots.
#pragma once

#include "../../bvh.h"
#include "../../math/conservativeDistances.h"

namespace cuBQL
{
namespace knn
{
struct Candidate
{
    int primID;
    float sqrDist;
};
struct Result
{
    int numFound;
    float sqrDistMax;
};
} // namespace knn

namespace points
{

template <typename T, int D>
__device__ knn::Result findKNN(knn::Candidate *cand, int k, BinaryBVH<T, D> bvh, const vec_t<T, D> *points,
                               vec_t<T, D> query, float maxDist)
{
    knn::Result res{0, 0.0f};
    if (k <= 0 || bvh.numNodes == 0)
        return res;
    const float cutoff = maxDist * maxDist;
    constexpr int kStack = 96; // a median-split tree over < 2^32 points is at most 33 levels deep
    uint32_t stack[kStack];
    int sp = 0;
    stack[sp++] = 0u;
    while (sp > 0)
    {
        uint32_t ni = stack[--sp];
        const auto &node = bvh.nodes[ni];
        float worst = fminf(cand[k - 1].sqrDist, cutoff);
        if (!(fSqrDistance_rd(query, node.bounds) < worst))
            continue;
        if (node.admin.count > 0)
        {
            uint32_t off = (uint32_t)node.admin.offset, cnt = (uint32_t)node.admin.count;
            for (uint32_t j = 0; j < cnt; ++j)
            {
                int id = (int)bvh.primIDs[off + j];
                vec_t<T, D> p = points[id];
                float dx = p.x - query.x, dy = p.y - query.y, dz = p.z - query.z;
                float d2 = dx * dx + dy * dy + dz * dz;
                if (!(d2 < fminf(cand[k - 1].sqrDist, cutoff)))
                    continue;
                int s = k - 1;
                while (s > 0 && cand[s - 1].sqrDist > d2)
                {
                    cand[s] = cand[s - 1];
                    --s;
                }
                cand[s].primID = id;
                cand[s].sqrDist = d2;
            }
            continue;
        }
        uint32_t c0 = (uint32_t)node.admin.offset, c1 = c0 + 1;
        float d0 = fSqrDistance_rd(query, bvh.nodes[c0].bounds), d1 = fSqrDistance_rd(query, bvh.nodes[c1].bounds);
        uint32_t nearer = d0 <= d1 ? c0 : c1, farther = d0 <= d1 ? c1 : c0;
        if (sp + 2 > kStack)
            continue; // cannot happen for the stand-in's trees; never write past the stack
        stack[sp++] = farther;
        stack[sp++] = nearer;
    }
    for (int s = 0; s < k; ++s)
        if (cand[s].primID >= 0)
        {
            ++res.numFound;
            res.sqrDistMax = cand[s].sqrDist;
        }
    return res;
}

} // namespace points
} // namespace cuBQL
