// Host build of the product's exact side test (paragram_b200/csrc/pg_exact.cuh)
// for the CPU unit tests: the same source the CUDA kernels compile, checked
// against the oracle's independent big-integer evaluation.
#include "../../paragram_b200/csrc/pg_exact.cuh"

using namespace pg::exact;

static PlaneSrc make_src(const float *p4, int box, int oid)
{
    PlaneSrc s;
    s.x = p4[0];
    s.y = p4[1];
    s.z = p4[2];
    s.w = p4[3];
    s.box = box;
    s.oid = oid;
    return s;
}

// stage: 0 full cascade, 1 FP64 stage only (-1 undecided), 2 expansion stage only
extern "C" int pgx_side_test(const float *seed4, int seed_oid, const float *planes4, const int *box, const int *oid,
                             const float *cand4, int cand_oid, int stage)
{
    PlaneSrc vp[3];
    for (int i = 0; i < 3; ++i)
        vp[i] = make_src(planes4 + 4 * i, box[i], oid[i]);
    PlaneSrc cp = make_src(cand4, -1, cand_oid);
    if (stage == 1)
    {
        DRow dv[3], dc;
        for (int i = 0; i < 3; ++i)
            make_drow(vp[i], seed4[0], seed4[1], seed4[2], seed4[3], dv[i]);
        make_drow(cp, seed4[0], seed4[1], seed4[2], seed4[3], dc);
        return fp64_stage(dv, dc);
    }
    if (stage == 2)
        return expansion_stage(vp, cp, seed4[0], seed4[1], seed4[2], seed4[3], seed_oid);
    int used = 0;
    return side_test(vp, cp, seed4[0], seed4[1], seed4[2], seed4[3], seed_oid, &used);
}
