// Invariant check of the cuBQL stand-in's BVH (test infrastructure): every
// primitive is listed by exactly one leaf, leaves hold 1..threshold
// primitives, children are inside the node array (never the root), and every
// node's box contains its children's boxes and its primitives' boxes.
// Prints one line per case and "bad=0" when all invariants hold.
#include "cuBQL/builder/cuda.h"

#include <cstdio>
#include <random>
#include <utility>

int main()
{
    std::mt19937 gen(1);
    std::uniform_real_distribution<float> u(0.0f, 1.0f);
    size_t total_bad = 0;
    for (int n : {1, 2, 3, 10, 11, 1000, 100000})
        for (int leaf : {0, 1, 10, 16})
            for (int flat : {0, 1})
            {
                std::vector<cuBQL::box_t<float, 3>> b(n);
                for (auto &x : b)
                {
                    float a = flat ? 0.5f : u(gen), c = u(gen), d = flat ? 0.25f : u(gen);
                    x.lower = {a, c, d};
                    x.upper = {a, c, d};
                }
                std::vector<uint32_t> prim;
                auto nodes = cuBQL::standin::build_host(b.data(), (uint32_t)n, leaf, prim);
                std::vector<int> seen(n, 0);
                size_t bad = 0, depth = 0;
                const uint64_t cap = (uint64_t)(leaf < 1 ? 1 : leaf);
                auto inside = [](const cuBQL::box_t<float, 3> &in, const cuBQL::box_t<float, 3> &out) {
                    return in.lower.x >= out.lower.x && in.lower.y >= out.lower.y && in.lower.z >= out.lower.z &&
                           in.upper.x <= out.upper.x && in.upper.y <= out.upper.y && in.upper.z <= out.upper.z;
                };
                std::vector<std::pair<uint64_t, size_t>> st{{0, 0}};
                while (!st.empty())
                {
                    auto [i, dep] = st.back();
                    st.pop_back();
                    depth = std::max(depth, dep);
                    const auto &nd = nodes[i];
                    if (nd.admin.count)
                    {
                        if (nd.admin.count > cap || nd.admin.offset + nd.admin.count > (uint64_t)n)
                        {
                            ++bad;
                            continue;
                        }
                        for (uint64_t j = 0; j < nd.admin.count; ++j)
                        {
                            uint32_t p = prim[nd.admin.offset + j];
                            seen[p]++;
                            if (!inside(b[p], nd.bounds))
                                ++bad;
                        }
                        continue;
                    }
                    for (uint64_t c = 0; c < 2; ++c)
                    {
                        uint64_t ci = nd.admin.offset + c;
                        if (ci == 0 || ci >= nodes.size() || !inside(nodes[ci].bounds, nd.bounds))
                        {
                            ++bad;
                            continue;
                        }
                        st.push_back({ci, dep + 1});
                    }
                }
                for (int i = 0; i < n; ++i)
                    bad += seen[i] != 1;
                std::printf("n=%d leaf=%d flat=%d nodes=%zu depth=%zu bad=%zu\n", n, leaf, flat, nodes.size(), depth,
                            bad);
                total_bad += bad;
            }
    std::printf("total bad=%zu\n", total_bad);
    return total_bad == 0 ? 0 : 1;
}
