// Stand-in for cuBQL::fSqrDistance_rd (TEST INFRASTRUCTURE ONLY; see
// cuBQL/bvh.h): the squared distance of a point to a box, every operation
// rounded toward -infinity, so that it never exceeds the exact distance (its
// uses: voronoi_ultra.cu:92, laguerre_ultra.cu:100).
#pragma once

#include "../bvh.h"

namespace cuBQL
{

__device__ inline float fSqrDistance_rd(vec_t<float, 3> p, box_t<float, 3> b)
{
    float dx = fmaxf(fmaxf(__fsub_rd(b.lower.x, p.x), __fsub_rd(p.x, b.upper.x)), 0.0f);
    float dy = fmaxf(fmaxf(__fsub_rd(b.lower.y, p.y), __fsub_rd(p.y, b.upper.y)), 0.0f);
    float dz = fmaxf(fmaxf(__fsub_rd(b.lower.z, p.z), __fsub_rd(p.z, b.upper.z)), 0.0f);
    return __fadd_rd(__fadd_rd(__fmul_rd(dx, dx), __fmul_rd(dy, dy)), __fmul_rd(dz, dz));
}

} // namespace cuBQL
