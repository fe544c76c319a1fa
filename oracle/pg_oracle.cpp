// pg_oracle.cpp -- CPU restatement of paragram's diagram construction.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity oracle: only tests/, the
// smoke check and bench.py's CPU-baseline leg load it. The product path
// (paragram_b200) never links or calls it.
//
// What it computes, per input point s (the "seed"):
//   the cell  { x in box : pow(x,s) <= pow(x,q) for every other point q },
//   pow(x,q) = |x-q|^2 - w_q, clipped to the reference's initial box
//   (root AABB of the points, -1.0f/+1.0f, then -1e-5f/+1e-5f, all in FP32:
//   voronoi_ultra.cu:234-238 / laguerre_ultra.cu:281-287 and
//   faster_convex_cell.cuh:206-221), and from it
//     * the directed row: ids of the points whose bisector plane carries a
//       facet of the cell (voronoi_ultra.cu:126-138 writes exactly the planes
//       referenced by surviving vertices),
//     * the status (faster_convex_cell.cuh:99-108 codes).
//   The directed rows are then symmetrised with the reference's rule
//   (adjacency.cuh:78-159): u->v is kept iff deg(v) > 0, and v->u is added
//   when missing. Rows are emitted sorted (the reference's row order is
//   atomic-order nondeterministic).
//
// Arithmetic. The reference clips in FP32 fast-math
// (faster_convex_cell.cuh:256-294, 411-512). Here every clipping decision is
// made EXACTLY: the vertex-vs-bisector side test is the sign of a 4x4
// determinant of plane rows (a, beta) with a = q - s and
// beta = |q - s|^2 - (w_q - w_s), divided by the sign of the 3x3 vertex
// determinant. A double-precision evaluation with a rigorous error bound
// decides almost every test; the rest are decided with arbitrary-precision
// integers (every FP32 input is an integer multiple of 2^-149). Exact ties
// are broken by Simulation of Simplicity (Edelsbrunner & Muecke, ACM TOG
// 1990) applied to the weights: w_j -> w_j + eps^(j), eps_i >> eps_j for
// i < j (original point index), which makes the result independent of the
// order in which candidates are clipped.
//
// Deliberate differences from the reference:
//   * the power "too far" test of faster_convex_cell.cuh:391-408 uses |t|,
//     which skips planes lying behind the seed; here such planes clip (the
//     cell becomes empty, as in the exact power diagram);
//   * capacity statuses are defined on the exact cell: vertex_overflow (2)
//     when the final cell has more than 64 vertices (MAX_VERTS,
//     faster_convex_cell.cuh:21), instead of depending on clip order.
//   * coincident points (q == s in all three coordinates) never clip each
//     other, as in the reference (its too-far test skips them when
//     |q - s| = 0, faster_convex_cell.cuh:398-407).
//
// Candidate enumeration: a median-split kd-tree with per-node max weight,
// visited best-first; a node is skipped when no point inside it can place a
// plane closer to the seed than the farthest cell vertex (the security radius
// of voronoi_bvh.cuh:149-288 / pwr_bvh.cuh:217-356, here with a rigorous
// radius bound). "brute" mode instead enumerates every plane triple against
// every plane (no traversal, no clipping) for small N.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <queue>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace pgo
{

static const int kMaxVerts = 64; // reference MAX_VERTS (faster_convex_cell.cuh:21)

enum Status
{
    kSuccess = 0,
    kPlaneOverflow = 1,
    kVertexOverflow = 2,
    kEmptyCell = 3,
    kSecurityRadiusNotReached = 4,
    kInconsistentBoundary = 5,
};

// ============================================================================
// Arbitrary precision signed integers (sign + base-2^32 magnitude).
// ============================================================================
struct Big
{
    int s = 0;                 // -1, 0, +1
    std::vector<uint32_t> m;   // little-endian limbs, no leading zero limbs
};

static void trim(Big &a)
{
    while (!a.m.empty() && a.m.back() == 0)
        a.m.pop_back();
    if (a.m.empty())
        a.s = 0;
}

static int cmp_mag(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b)
{
    if (a.size() != b.size())
        return a.size() < b.size() ? -1 : 1;
    for (size_t i = a.size(); i-- > 0;)
        if (a[i] != b[i])
            return a[i] < b[i] ? -1 : 1;
    return 0;
}

static std::vector<uint32_t> add_mag(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b)
{
    const std::vector<uint32_t> &x = a.size() >= b.size() ? a : b;
    const std::vector<uint32_t> &y = a.size() >= b.size() ? b : a;
    std::vector<uint32_t> r(x.size() + 1, 0);
    uint64_t carry = 0;
    for (size_t i = 0; i < x.size(); ++i)
    {
        uint64_t t = (uint64_t)x[i] + (i < y.size() ? y[i] : 0) + carry;
        r[i] = (uint32_t)t;
        carry = t >> 32;
    }
    r[x.size()] = (uint32_t)carry;
    return r;
}

// |a| - |b| with |a| >= |b|
static std::vector<uint32_t> sub_mag(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b)
{
    std::vector<uint32_t> r(a.size(), 0);
    int64_t borrow = 0;
    for (size_t i = 0; i < a.size(); ++i)
    {
        int64_t t = (int64_t)a[i] - (i < b.size() ? (int64_t)b[i] : 0) - borrow;
        borrow = t < 0 ? 1 : 0;
        if (t < 0)
            t += ((int64_t)1 << 32);
        r[i] = (uint32_t)t;
    }
    return r;
}

static Big add(const Big &a, const Big &b)
{
    if (a.s == 0)
        return b;
    if (b.s == 0)
        return a;
    Big r;
    if (a.s == b.s)
    {
        r.m = add_mag(a.m, b.m);
        r.s = a.s;
    }
    else
    {
        int c = cmp_mag(a.m, b.m);
        if (c == 0)
            return Big();
        if (c > 0)
        {
            r.m = sub_mag(a.m, b.m);
            r.s = a.s;
        }
        else
        {
            r.m = sub_mag(b.m, a.m);
            r.s = b.s;
        }
    }
    trim(r);
    return r;
}

static Big neg(Big a)
{
    a.s = -a.s;
    return a;
}

static Big sub(const Big &a, const Big &b) { return add(a, neg(b)); }

static Big mul(const Big &a, const Big &b)
{
    if (a.s == 0 || b.s == 0)
        return Big();
    Big r;
    r.m.assign(a.m.size() + b.m.size(), 0);
    for (size_t i = 0; i < a.m.size(); ++i)
    {
        uint64_t carry = 0;
        for (size_t j = 0; j < b.m.size(); ++j)
        {
            uint64_t t = (uint64_t)a.m[i] * b.m[j] + r.m[i + j] + carry;
            r.m[i + j] = (uint32_t)t;
            carry = t >> 32;
        }
        r.m[i + b.m.size()] = (uint32_t)carry;
    }
    r.s = a.s * b.s;
    trim(r);
    return r;
}

static Big shl(const Big &a, int bits)
{
    if (a.s == 0 || bits == 0)
        return a;
    Big r;
    r.s = a.s;
    int limbs = bits / 32, rem = bits % 32;
    r.m.assign(a.m.size() + limbs + 1, 0);
    for (size_t i = 0; i < a.m.size(); ++i)
    {
        uint64_t v = (uint64_t)a.m[i] << rem;
        r.m[i + limbs] |= (uint32_t)v;
        r.m[i + limbs + 1] |= (uint32_t)(v >> 32);
    }
    trim(r);
    return r;
}

static Big from_u64(uint64_t v, int sign)
{
    Big r;
    if (v == 0)
        return r;
    r.s = sign;
    r.m.push_back((uint32_t)v);
    r.m.push_back((uint32_t)(v >> 32));
    trim(r);
    return r;
}

// Exact integer value of f * 2^149 (every finite float is an integer multiple of 2^-149).
static Big from_float(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    uint32_t E = (u >> 23) & 0xFFu, F = u & 0x7FFFFFu;
    int sign = (u >> 31) ? -1 : 1;
    if (E == 0)
        return from_u64(F, sign); // subnormal: F * 2^-149
    return shl(from_u64(F | 0x800000u, sign), (int)E - 1); // (F|2^23) * 2^(E-150) * 2^149
}

// ============================================================================
// Planes of one cell.
//
// Coordinates are relative to the seed s. A plane is the set 2 a.x = beta:
//   bisector of s and q : a = q - s,  beta = |q - s|^2 - (w_q - w_s)
//   box plane x_i = b   : a = e_i,    beta = 2 (b - s_i)
// Interior side: 2 a.x <= beta (closer, in power distance, to s than to q).
// ============================================================================
struct Plane
{
    double a[3];
    double beta;
    double dbeta;   // bound on |beta_double - beta_exact|
    bool exact_a;   // a[] holds the exact differences
    int pt;         // neighbour point index, or -1 for a box plane
    int box;        // 0..5 for box planes (axis*2 + side), -1 otherwise
};

static const double kU = 1.1102230246251565e-16; // 2^-53

// exact difference test (TwoDiff error term == 0)
static inline bool diff_exact(double x, double y, double d)
{
    double bv = x - d;
    double av = d + bv;
    double br = bv - y;
    double ar = x - av;
    return (ar + br) == 0.0;
}

struct Ctx
{
    int64_t n;
    const float *pts; // n*3
    const float *w;   // n or nullptr
    float lo[3], hi[3];
    float wmax;
};

static inline float weight_of(const Ctx &c, int64_t i) { return c.w ? c.w[i] : 0.0f; }

static void make_bisector(const Ctx &c, int64_t s, int64_t q, Plane &p)
{
    bool ex = true;
    double n2 = 0.0;
    for (int k = 0; k < 3; ++k)
    {
        double qs = c.pts[q * 3 + k], ss = c.pts[s * 3 + k];
        p.a[k] = qs - ss;
        ex = ex && diff_exact(qs, ss, p.a[k]);
        n2 += p.a[k] * p.a[k];
    }
    double wq = weight_of(c, q), ws = weight_of(c, s);
    double dw = wq - ws;
    ex = ex && diff_exact(wq, ws, dw);
    p.beta = n2 - dw;
    p.dbeta = 8.0 * kU * (n2 + std::fabs(dw));
    p.exact_a = ex;
    p.pt = (int)q;
    p.box = -1;
}

static float box_value(const Ctx &c, int code) { return (code & 1) ? c.hi[code >> 1] : c.lo[code >> 1]; }

// Box planes are oriented outward like the bisectors (interior 2 a.x <= beta):
// the low face x_i >= lo is a = -e_i, beta = 2 (s_i - lo); the high face
// x_i <= hi is a = +e_i, beta = 2 (hi - s_i).
static void make_box(const Ctx &c, int64_t s, int code, Plane &p)
{
    int ax = code >> 1;
    double sg = (code & 1) ? 1.0 : -1.0;
    p.a[0] = p.a[1] = p.a[2] = 0.0;
    p.a[ax] = sg;
    double b = box_value(c, code), ss = c.pts[s * 3 + ax];
    double d = b - ss;
    p.beta = 2.0 * sg * d;
    p.dbeta = diff_exact(b, ss, d) ? 0.0 : 4.0 * kU * std::fabs(p.beta);
    p.exact_a = true;
    p.pt = -1;
    p.box = code;
}

// exact (integer) row matching a Plane: 2 A.X = B with X = x * 2^149
struct ExactRow
{
    Big A[3];
    Big B;
    int pt;
};

static void exact_row(const Ctx &c, int64_t s, const Plane &p, ExactRow &r)
{
    r.pt = p.pt;
    if (p.pt >= 0)
    {
        for (int k = 0; k < 3; ++k)
            r.A[k] = sub(from_float(c.pts[(int64_t)p.pt * 3 + k]), from_float(c.pts[s * 3 + k]));
        Big n2 = add(add(mul(r.A[0], r.A[0]), mul(r.A[1], r.A[1])), mul(r.A[2], r.A[2]));
        Big dw = sub(from_float(weight_of(c, p.pt)), from_float(weight_of(c, s)));
        r.B = sub(n2, shl(dw, 149));
    }
    else
    {
        int ax = p.box >> 1;
        int sg = (p.box & 1) ? 1 : -1;
        for (int k = 0; k < 3; ++k)
            r.A[k] = from_u64(k == ax ? 1 : 0, sg);
        Big d = shl(sub(from_float(box_value(c, p.box)), from_float(c.pts[s * 3 + ax])), 1);
        r.B = sg > 0 ? d : neg(d);
    }
}

static Big det3_big(const Big *m[3][3])
{
    Big t0 = sub(mul(*m[1][1], *m[2][2]), mul(*m[1][2], *m[2][1]));
    Big t1 = sub(mul(*m[1][0], *m[2][2]), mul(*m[1][2], *m[2][0]));
    Big t2 = sub(mul(*m[1][0], *m[2][1]), mul(*m[1][1], *m[2][0]));
    return add(sub(mul(*m[0][0], t0), mul(*m[0][1], t1)), mul(*m[0][2], t2));
}

// Exact decision: is the vertex of rows r[0..2] strictly on the far side of
// candidate row r[3] (to be removed)?  det4 * D < 0, with SoS for det4 == 0.
static bool exact_removed(const ExactRow *r[4], int64_t seed)
{
    Big C[4];
    for (int i = 0; i < 4; ++i)
    {
        const Big *m[3][3];
        int rr = 0;
        for (int k = 0; k < 4; ++k)
        {
            if (k == i)
                continue;
            for (int j = 0; j < 3; ++j)
                m[rr][j] = &r[k]->A[j];
            ++rr;
        }
        Big d = det3_big(m);
        C[i] = ((i + 3) & 1) ? neg(d) : d;
    }
    const Big &D = C[3];
    if (D.s == 0)
        return false;
    Big det4;
    for (int i = 0; i < 4; ++i)
        det4 = add(det4, mul(r[i]->B, C[i]));
    int s4 = det4.s;
    if (s4 == 0)
    {
        // Simulation of Simplicity on the weights.
        struct Term
        {
            int64_t idx;
            Big coef;
        };
        std::vector<Term> terms;
        Big S;
        bool any = false;
        for (int i = 0; i < 4; ++i)
            if (r[i]->pt >= 0)
            {
                S = add(S, C[i]);
                terms.push_back({(int64_t)r[i]->pt, neg(C[i])});
                any = true;
            }
        if (any)
            terms.push_back({seed, S});
        std::sort(terms.begin(), terms.end(), [](const Term &a, const Term &b) { return a.idx < b.idx; });
        for (const Term &t : terms)
            if (t.coef.s != 0)
            {
                s4 = t.coef.s;
                break;
            }
        if (s4 == 0)
            return false;
    }
    return s4 * D.s < 0;
}

// ============================================================================
// Vertices (double cofactors with rigorous error bounds).
// ============================================================================
struct Vtx
{
    int p[3];       // plane slots, consistently oriented
    double c[4];    // det4 = c . (a_x, a_y, a_z, beta) of a candidate row
    double e[4];    // |c_double - c_exact| bounds (INFINITY = unusable)
    double X[3];    // position relative to the seed (approximate)
    double ex;      // upper bound on |X - X_exact|
    double rad;     // upper bound on |X_exact|
};

// det of 3x3 (rows) where only column `ecol` carries entry errors err[3].
static double det3_err(const double m[3][3], int ecol, const double err[3], double *bound)
{
    double p00 = m[1][1] * m[2][2], p01 = m[1][2] * m[2][1];
    double p10 = m[1][0] * m[2][2], p11 = m[1][2] * m[2][0];
    double p20 = m[1][0] * m[2][1], p21 = m[1][1] * m[2][0];
    double d = m[0][0] * (p00 - p01) - m[0][1] * (p10 - p11) + m[0][2] * (p20 - p21);
    double perm = std::fabs(m[0][0]) * (std::fabs(p00) + std::fabs(p01)) +
                  std::fabs(m[0][1]) * (std::fabs(p10) + std::fabs(p11)) +
                  std::fabs(m[0][2]) * (std::fabs(p20) + std::fabs(p21));
    double b = 8.0 * kU * perm;
    if (ecol >= 0)
    {
        for (int i = 0; i < 3; ++i)
        {
            if (err[i] == 0.0)
                continue;
            int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
            int j1 = (ecol + 1) % 3, j2 = (ecol + 2) % 3;
            double cp = std::fabs(m[i1][j1] * m[i2][j2]) + std::fabs(m[i1][j2] * m[i2][j1]);
            b += err[i] * cp * (1.0 + 8.0 * kU) + err[i] * err[i];
        }
    }
    *bound = b * (1.0 + 16.0 * kU);
    return d;
}

static void make_vertex(const std::vector<Plane> &pl, int p0, int p1, int p2, Vtx &v)
{
    v.p[0] = p0;
    v.p[1] = p1;
    v.p[2] = p2;
    const Plane *r[3] = {&pl[p0], &pl[p1], &pl[p2]};
    bool exact_a = r[0]->exact_a && r[1]->exact_a && r[2]->exact_a;
    double derr[3] = {r[0]->dbeta, r[1]->dbeta, r[2]->dbeta};
    // columns: 0 ax, 1 ay, 2 az, 3 beta; c_j = (-1)^(3+j) det(rows, column j removed)
    for (int j = 0; j < 4; ++j)
    {
        double m[3][3];
        int ecol = -1;
        for (int i = 0; i < 3; ++i)
        {
            int cc = 0;
            for (int col = 0; col < 4; ++col)
            {
                if (col == j)
                    continue;
                m[i][cc] = col == 3 ? r[i]->beta : r[i]->a[col];
                if (col == 3)
                    ecol = cc;
                ++cc;
            }
        }
        double bound;
        double d = det3_err(m, ecol, derr, &bound);
        double sgn = ((j + 3) & 1) ? -1.0 : 1.0;
        v.c[j] = sgn * d;
        v.e[j] = exact_a ? bound : INFINITY;
    }
    double c3 = v.c[3];
    double den = 2.0 * (std::fabs(c3) - v.e[3]);
    double x2 = 0.0, e2 = 0.0;
    bool ok = std::isfinite(den) && den > 0.0;
    for (int k = 0; k < 3; ++k)
    {
        v.X[k] = c3 != 0.0 ? -v.c[k] / (2.0 * c3) : 0.0;
        double ex = ok ? (v.e[k] + std::fabs(v.X[k]) * 2.0 * v.e[3]) / den + 4.0 * kU * std::fabs(v.X[k]) : INFINITY;
        x2 += v.X[k] * v.X[k];
        e2 += ex * ex;
    }
    v.ex = ok ? std::sqrt(e2) * (1.0 + 1e-12) : INFINITY;
    v.rad = ok ? (std::sqrt(x2) + v.ex) * (1.0 + 1e-12) : INFINITY;
}

// ============================================================================
// One cell (incremental clipping).
// ============================================================================
struct Cell
{
    std::vector<Plane> planes;
    std::vector<Vtx> verts;
    std::vector<Vtx> nverts;
    std::vector<char> removed;
    std::vector<std::pair<int, int>> edges;
    bool empty = false;
    bool inconsistent = false;
    int64_t exact_calls = 0;
    int64_t tests = 0;
};

// side test: true iff vertex v is strictly on the candidate's side of plane q
static bool removed_test(const Ctx &c, int64_t s, const Cell &cell, const Vtx &v, const Plane &q, int64_t *exact_calls)
{
    if (q.exact_a && std::isfinite(v.e[0]) && std::isfinite(v.e[1]) && std::isfinite(v.e[2]) && std::isfinite(v.e[3]))
    {
        double r[4] = {q.a[0], q.a[1], q.a[2], q.beta};
        double val = 0.0, mag = 0.0, bnd = 0.0;
        for (int j = 0; j < 4; ++j)
        {
            val += v.c[j] * r[j];
            mag += std::fabs(v.c[j] * r[j]);
            bnd += v.e[j] * std::fabs(r[j]);
        }
        bnd += (std::fabs(v.c[3]) + v.e[3]) * q.dbeta + 8.0 * kU * mag;
        bnd *= (1.0 + 16.0 * kU);
        if (std::fabs(v.c[3]) > v.e[3] && std::fabs(val) > bnd)
            return (val > 0.0) != (v.c[3] > 0.0);
    }
    ++*exact_calls;
    ExactRow rows[4];
    for (int i = 0; i < 3; ++i)
        exact_row(c, s, cell.planes[v.p[i]], rows[i]);
    exact_row(c, s, q, rows[3]);
    const ExactRow *rp[4] = {&rows[0], &rows[1], &rows[2], &rows[3]};
    return exact_removed(rp, s);
}

static void cell_init(const Ctx &c, int64_t s, Cell &cell)
{
    cell.planes.clear();
    cell.verts.clear();
    cell.empty = false;
    cell.inconsistent = false;
    for (int code = 0; code < 6; ++code)
    {
        Plane p;
        make_box(c, s, code, p);
        cell.planes.push_back(p);
    }
    // 8 corners; triples ordered so that the outward normals have a positive
    // triple product (one consistent orientation of the dual triangulation).
    for (int corner = 0; corner < 8; ++corner)
    {
        int sx = corner & 1, sy = (corner >> 1) & 1, sz = (corner >> 2) & 1;
        int px = 0 * 2 + sx, py = 1 * 2 + sy, pz = 2 * 2 + sz;
        // outward normal signs: side 0 (low) -> -1, side 1 (high) -> +1
        int sign = (sx ? 1 : -1) * (sy ? 1 : -1) * (sz ? 1 : -1);
        Vtx v;
        if (sign > 0)
            make_vertex(cell.planes, px, py, pz, v);
        else
            make_vertex(cell.planes, py, px, pz, v);
        cell.verts.push_back(v);
    }
}

// Clip by the bisector of s and q.  Returns true if the cell changed.
static bool cell_clip(const Ctx &c, int64_t s, Cell &cell, int64_t q)
{
    if (cell.empty || cell.inconsistent)
        return false;
    const float *ps = c.pts + s * 3, *pq = c.pts + q * 3;
    if (ps[0] == pq[0] && ps[1] == pq[1] && ps[2] == pq[2])
        return false; // coincident points never clip each other
    Plane p;
    make_bisector(c, s, q, p);
    size_t nv = cell.verts.size();
    cell.removed.assign(nv, 0);
    size_t nrem = 0;
    for (size_t i = 0; i < nv; ++i)
    {
        ++cell.tests;
        if (removed_test(c, s, cell, cell.verts[i], p, &cell.exact_calls))
        {
            cell.removed[i] = 1;
            ++nrem;
        }
    }
    if (nrem == 0)
        return false;
    if (nrem == nv)
    {
        cell.empty = true;
        cell.verts.clear();
        return true;
    }
    // boundary edges: directed edges of removed triangles whose reverse edge is
    // not an edge of another removed triangle
    cell.edges.clear();
    for (size_t i = 0; i < nv; ++i)
    {
        if (!cell.removed[i])
            continue;
        const int *t = cell.verts[i].p;
        for (int e = 0; e < 3; ++e)
        {
            int x = t[e], y = t[(e + 1) % 3];
            bool interior = false;
            for (size_t k = 0; k < nv && !interior; ++k)
            {
                if (!cell.removed[k] || k == i)
                    continue;
                const int *u = cell.verts[k].p;
                for (int f = 0; f < 3; ++f)
                    if (u[f] == y && u[(f + 1) % 3] == x)
                    {
                        interior = true;
                        break;
                    }
            }
            if (!interior)
                cell.edges.push_back({x, y});
        }
    }
    // consistency: the boundary must be one simple cycle
    {
        size_t ne = cell.edges.size();
        bool ok = ne >= 3;
        for (size_t i = 0; i < ne && ok; ++i)
        {
            int nsrc = 0, ndst = 0;
            for (size_t k = 0; k < ne; ++k)
            {
                nsrc += cell.edges[k].first == cell.edges[i].first;
                ndst += cell.edges[k].second == cell.edges[i].first;
            }
            ok = nsrc == 1 && ndst == 1;
        }
        if (ok)
        {
            size_t len = 0;
            int cur = cell.edges[0].first;
            do
            {
                int nxt = -1;
                for (size_t k = 0; k < ne; ++k)
                    if (cell.edges[k].first == cur)
                        nxt = cell.edges[k].second;
                cur = nxt;
                ++len;
            } while (cur != cell.edges[0].first && cur >= 0 && len <= ne);
            ok = (cur == cell.edges[0].first) && len == ne;
        }
        if (!ok)
        {
            cell.inconsistent = true;
            return true;
        }
    }
    int P = (int)cell.planes.size();
    cell.planes.push_back(p);
    cell.nverts.clear();
    for (size_t i = 0; i < nv; ++i)
        if (!cell.removed[i])
            cell.nverts.push_back(cell.verts[i]);
    for (auto &e : cell.edges)
    {
        Vtx v;
        make_vertex(cell.planes, P, e.first, e.second, v);
        cell.nverts.push_back(v);
    }
    cell.verts.swap(cell.nverts);
    return true;
}

static double cell_radius(const Cell &cell)
{
    double r = 0.0;
    for (const Vtx &v : cell.verts)
        r = std::max(r, v.rad);
    return r;
}

// ============================================================================
// kd-tree (median split, leaf <= 8) with per-node box and max weight.
// ============================================================================
struct KdNode
{
    float lo[3], hi[3];
    float maxw;
    int left, right; // child node ids, -1 for leaves
    int begin, end;  // range into perm
};

struct KdTree
{
    std::vector<KdNode> nodes;
    std::vector<int> perm;
};

static int kd_build_rec(const Ctx &c, KdTree &t, int begin, int end)
{
    KdNode nd;
    for (int k = 0; k < 3; ++k)
    {
        nd.lo[k] = INFINITY;
        nd.hi[k] = -INFINITY;
    }
    nd.maxw = -INFINITY;
    for (int i = begin; i < end; ++i)
    {
        int64_t p = t.perm[i];
        for (int k = 0; k < 3; ++k)
        {
            nd.lo[k] = std::min(nd.lo[k], c.pts[p * 3 + k]);
            nd.hi[k] = std::max(nd.hi[k], c.pts[p * 3 + k]);
        }
        nd.maxw = std::max(nd.maxw, weight_of(c, p));
    }
    nd.begin = begin;
    nd.end = end;
    nd.left = nd.right = -1;
    int id = (int)t.nodes.size();
    t.nodes.push_back(nd);
    if (end - begin > 8)
    {
        int ax = 0;
        float ext = -1.0f;
        for (int k = 0; k < 3; ++k)
            if (nd.hi[k] - nd.lo[k] > ext)
            {
                ext = nd.hi[k] - nd.lo[k];
                ax = k;
            }
        int mid = (begin + end) / 2;
        std::nth_element(t.perm.begin() + begin, t.perm.begin() + mid, t.perm.begin() + end,
                         [&](int a, int b) { return c.pts[(int64_t)a * 3 + ax] < c.pts[(int64_t)b * 3 + ax]; });
        int l = kd_build_rec(c, t, begin, mid);
        int r = kd_build_rec(c, t, mid, end);
        t.nodes[id].left = l;
        t.nodes[id].right = r;
    }
    return id;
}

static void kd_build(const Ctx &c, KdTree &t)
{
    t.nodes.clear();
    t.perm.resize(c.n);
    for (int64_t i = 0; i < c.n; ++i)
        t.perm[i] = (int)i;
    t.nodes.reserve(2 * (c.n / 4 + 1));
    if (c.n > 0)
        kd_build_rec(c, t, 0, (int)c.n);
}

static double box_dist2(const KdNode &nd, const float *p)
{
    double d2 = 0.0;
    for (int k = 0; k < 3; ++k)
    {
        double v = p[k];
        double d = 0.0;
        if (v < nd.lo[k])
            d = (double)nd.lo[k] - v;
        else if (v > nd.hi[k])
            d = v - (double)nd.hi[k];
        d2 += d * d;
    }
    return d2 * (1.0 - 1e-12);
}

// can a point inside this node carry a plane closer than R to the seed?
static bool node_may_clip(const KdNode &nd, double d2, double ws, double R)
{
    if (!std::isfinite(R))
        return true;
    double R2 = R * R * (1.0 + 1e-9);
    double dmax = (double)nd.maxw - ws;
    if (dmax <= 0.0)
        return !(d2 > 4.0 * R2);
    double num = d2 - dmax;
    if (num <= 0.0)
        return true;
    return !(num * num > 4.0 * d2 * R2);
}

// Tighter test: q in the node can remove vertex v only if
// |v - q|^2 < |v - s|^2 + (w_q - w_s); bound |v - q| below by the distance of
// v to the node box and w_q by the node's max weight.
static bool node_may_clip_verts(const KdNode &nd, const Cell &cell, const float *ps, double ws)
{
    double dmax = (double)nd.maxw - ws;
    for (const Vtx &v : cell.verts)
    {
        if (!std::isfinite(v.rad))
            return true;
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k)
        {
            double x = (double)ps[k] + v.X[k];
            double d = 0.0;
            if (x < nd.lo[k])
                d = (double)nd.lo[k] - x;
            else if (x > nd.hi[k])
                d = x - (double)nd.hi[k];
            d2 += d * d;
        }
        double md = std::sqrt(d2) * (1.0 - 1e-12) - v.ex - 1e-300;
        double lhs = md > 0.0 ? md * md : 0.0;
        double rhs = (v.rad * v.rad + dmax) * (1.0 + 1e-9) + 1e-300;
        if (lhs < rhs)
            return true;
    }
    return false;
}

struct CellResult
{
    int status;
    int nverts;
    std::vector<int> row;
    int64_t exact_calls;
    int64_t tests;
};

static void build_cell_incremental(const Ctx &c, const KdTree &t, int64_t s, Cell &cell, CellResult &out)
{
    cell_init(c, s, cell);
    cell.exact_calls = 0;
    cell.tests = 0;
    const float *ps = c.pts + s * 3;
    double ws = weight_of(c, s);
    typedef std::pair<double, int> QE;
    std::priority_queue<QE, std::vector<QE>, std::greater<QE>> pq;
    if (!t.nodes.empty())
        pq.push({box_dist2(t.nodes[0], ps), 0});
    double R = cell_radius(cell);
    while (!pq.empty() && !cell.empty && !cell.inconsistent)
    {
        QE top = pq.top();
        pq.pop();
        const KdNode &nd = t.nodes[top.second];
        if (!node_may_clip(nd, top.first, ws, R) || !node_may_clip_verts(nd, cell, ps, ws))
            continue;
        if (nd.left < 0)
        {
            bool changed = false;
            for (int i = nd.begin; i < nd.end; ++i)
            {
                int64_t q = t.perm[i];
                if (q == s)
                    continue;
                changed |= cell_clip(c, s, cell, q);
            }
            if (changed)
                R = cell_radius(cell);
        }
        else
        {
            const KdNode &l = t.nodes[nd.left], &r = t.nodes[nd.right];
            double dl = box_dist2(l, ps), dr = box_dist2(r, ps);
            if (node_may_clip(l, dl, ws, R))
                pq.push({dl, nd.left});
            if (node_may_clip(r, dr, ws, R))
                pq.push({dr, nd.right});
        }
    }
    out.exact_calls = cell.exact_calls;
    out.tests = cell.tests;
    out.row.clear();
    if (cell.inconsistent)
    {
        out.status = kInconsistentBoundary;
        out.nverts = (int)cell.verts.size();
        return;
    }
    if (cell.empty)
    {
        out.status = kEmptyCell;
        out.nverts = 0;
        return;
    }
    std::vector<char> used(cell.planes.size(), 0);
    for (const Vtx &v : cell.verts)
        for (int k = 0; k < 3; ++k)
            used[v.p[k]] = 1;
    for (size_t i = 0; i < cell.planes.size(); ++i)
        if (used[i] && cell.planes[i].pt >= 0)
            out.row.push_back(cell.planes[i].pt);
    std::sort(out.row.begin(), out.row.end());
    out.nverts = (int)cell.verts.size();
    out.status = out.nverts > kMaxVerts ? kVertexOverflow : kSuccess;
}

// Brute force: planes = box + every other (non-coincident) point; a triple is
// a vertex iff no plane strictly removes it.  O(N^4) per cell: small N only.
static void build_cell_brute(const Ctx &c, int64_t s, CellResult &out)
{
    std::vector<Plane> pl;
    for (int code = 0; code < 6; ++code)
    {
        Plane p;
        make_box(c, s, code, p);
        pl.push_back(p);
    }
    const float *ps = c.pts + s * 3;
    for (int64_t q = 0; q < c.n; ++q)
    {
        if (q == s)
            continue;
        const float *pq = c.pts + q * 3;
        if (ps[0] == pq[0] && ps[1] == pq[1] && ps[2] == pq[2])
            continue;
        Plane p;
        make_bisector(c, s, q, p);
        pl.push_back(p);
    }
    int P = (int)pl.size();
    std::vector<ExactRow> er(P);
    for (int i = 0; i < P; ++i)
        exact_row(c, s, pl[i], er[i]);
    std::vector<char> used(P, 0);
    int nverts = 0;
    out.exact_calls = 0;
    out.tests = 0;
    Cell dummy;
    dummy.planes = pl; // removed_test reads the vertex plane definitions from here
    for (int i = 0; i < P; ++i)
        for (int j = i + 1; j < P; ++j)
            for (int k = j + 1; k < P; ++k)
            {
                Vtx v;
                make_vertex(pl, i, j, k, v);
                // skip singular triples exactly
                {
                    const Big *m[3][3];
                    const ExactRow *rr[3] = {&er[i], &er[j], &er[k]};
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b)
                            m[a][b] = &rr[a]->A[b];
                    if (det3_big(m).s == 0)
                        continue;
                }
                bool alive = true;
                for (int l = 0; l < P && alive; ++l)
                {
                    if (l == i || l == j || l == k)
                        continue;
                    ++out.tests;
                    bool rem;
                    if (pl[l].pt >= 0)
                        rem = removed_test(c, s, dummy, v, pl[l], &out.exact_calls);
                    else
                    {
                        const ExactRow *rp[4] = {&er[i], &er[j], &er[k], &er[l]};
                        rem = exact_removed(rp, s);
                    }
                    if (rem)
                        alive = false;
                }
                if (alive)
                {
                    used[i] = used[j] = used[k] = 1;
                    ++nverts;
                }
            }
    out.row.clear();
    for (int i = 0; i < P; ++i)
        if (used[i] && pl[i].pt >= 0)
            out.row.push_back(pl[i].pt);
    std::sort(out.row.begin(), out.row.end());
    out.nverts = nverts;
    if (nverts == 0)
    {
        out.status = kEmptyCell;
        out.row.clear();
    }
    else
        out.status = nverts > kMaxVerts ? kVertexOverflow : kSuccess;
}

static void compute_box(Ctx &c)
{
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    float wm = -INFINITY;
    for (int64_t i = 0; i < c.n; ++i)
    {
        for (int k = 0; k < 3; ++k)
        {
            mn[k] = std::min(mn[k], c.pts[i * 3 + k]);
            mx[k] = std::max(mx[k], c.pts[i * 3 + k]);
        }
        wm = std::max(wm, weight_of(c, i));
    }
    for (int k = 0; k < 3; ++k)
    {
        // FP32 arithmetic, as the reference: (min - 1.0f) - 1e-5f, (max + 1.0f) + 1e-5f
        volatile float a = mn[k] - 1.0f;
        volatile float b = mx[k] + 1.0f;
        volatile float lo = a - 1e-5f;
        volatile float hi = b + 1e-5f;
        c.lo[k] = lo;
        c.hi[k] = hi;
    }
    c.wmax = wm;
}

} // namespace pgo

// ============================================================================
// C ABI (used by oracle/pg_oracle.py only)
// ============================================================================
extern "C" {

struct pgo_result
{
    int64_t n_cells;      // cells computed: [cell_begin, cell_end)
    int32_t *status;      // [n_cells]
    int32_t *nverts;      // [n_cells]
    int64_t *row_offsets; // [n_cells + 1]
    int32_t *rows;        // directed rows, sorted, original ids
    int64_t exact_calls;  // number of side tests decided by big integers
    int64_t tests;        // number of side tests
    double seconds;       // wall time of the cell computation (excludes tree build)
    double tree_seconds;  // wall time of the kd-tree build
    int threads;          // OpenMP threads used
};

int pgo_build(int64_t n, const float *points, const float *weights, int mode, int64_t cell_begin, int64_t cell_end,
              int threads, pgo_result *res)
{
    using namespace pgo;
    if (n < 0 || !points || !res || cell_begin < 0 || cell_end > n || cell_begin > cell_end)
        return -1;
    Ctx c;
    c.n = n;
    c.pts = points;
    c.w = weights;
    compute_box(c);
#ifdef _OPENMP
    if (threads > 0)
        omp_set_num_threads(threads);
    int nthreads = omp_get_max_threads();
#else
    int nthreads = 1;
#endif
    auto t0 = std::chrono::steady_clock::now();
    KdTree tree;
    if (mode == 0)
        kd_build(c, tree);
    auto t1 = std::chrono::steady_clock::now();
    int64_t m = cell_end - cell_begin;
    std::vector<CellResult> out(m);
    int64_t exact_calls = 0, tests = 0;
#pragma omp parallel reduction(+ : exact_calls, tests)
    {
        Cell cell;
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < m; ++i)
        {
            if (mode == 0)
                build_cell_incremental(c, tree, cell_begin + i, cell, out[i]);
            else
                build_cell_brute(c, cell_begin + i, out[i]);
            exact_calls += out[i].exact_calls;
            tests += out[i].tests;
        }
    }
    auto t2 = std::chrono::steady_clock::now();
    res->n_cells = m;
    res->status = (int32_t *)std::malloc(sizeof(int32_t) * (m > 0 ? m : 1));
    res->nverts = (int32_t *)std::malloc(sizeof(int32_t) * (m > 0 ? m : 1));
    res->row_offsets = (int64_t *)std::malloc(sizeof(int64_t) * (m + 1));
    int64_t tot = 0;
    res->row_offsets[0] = 0;
    for (int64_t i = 0; i < m; ++i)
    {
        res->status[i] = out[i].status;
        res->nverts[i] = out[i].nverts;
        tot += (int64_t)out[i].row.size();
        res->row_offsets[i + 1] = tot;
    }
    res->rows = (int32_t *)std::malloc(sizeof(int32_t) * (tot > 0 ? tot : 1));
    for (int64_t i = 0; i < m; ++i)
        if (!out[i].row.empty())
            std::memcpy(res->rows + res->row_offsets[i], out[i].row.data(), sizeof(int32_t) * out[i].row.size());
    res->exact_calls = exact_calls;
    res->tests = tests;
    res->seconds = std::chrono::duration<double>(t2 - t1).count();
    res->tree_seconds = std::chrono::duration<double>(t1 - t0).count();
    res->threads = nthreads;
    return 0;
}

void pgo_free_result(pgo_result *res)
{
    if (!res)
        return;
    std::free(res->status);
    std::free(res->nverts);
    std::free(res->row_offsets);
    std::free(res->rows);
    res->status = nullptr;
    res->nverts = nullptr;
    res->row_offsets = nullptr;
    res->rows = nullptr;
}

// Symmetrisation with the reference rule (adjacency.cuh:78-159), rows sorted.
// in: directed CSR over all n cells. out_offsets [n+1]; out_adj capacity 2*E_in.
int pgo_symmetrize(int64_t n, const int64_t *off, const int32_t *adj, int64_t *out_off, int32_t *out_adj,
                   int64_t *out_len)
{
    std::vector<std::vector<int32_t>> rows(n);
    for (int64_t u = 0; u < n; ++u)
    {
        for (int64_t k = off[u]; k < off[u + 1]; ++k)
        {
            int32_t v = adj[k];
            if (off[v + 1] - off[v] <= 0)
                continue;
            rows[u].push_back(v);
            bool has = std::binary_search(adj + off[v], adj + off[v + 1], (int32_t)u);
            if (!has)
            {
                // rows of the directed CSR are sorted; a linear search would also do
                rows[v].push_back((int32_t)u);
            }
        }
    }
    int64_t tot = 0;
    out_off[0] = 0;
    for (int64_t u = 0; u < n; ++u)
    {
        std::sort(rows[u].begin(), rows[u].end());
        for (int32_t v : rows[u])
            out_adj[tot++] = v;
        out_off[u + 1] = tot;
    }
    *out_len = tot;
    return 0;
}

// Exact side test on explicit rows, exposed for the predicate unit tests:
// vertex planes given as (kind,id) pairs (kind 0: bisector with point id,
// kind 1: box plane code id), candidate point q. Returns 1 if removed.
int pgo_side_test(int64_t n, const float *points, const float *weights, int64_t seed, const int32_t *kinds,
                  const int32_t *ids, int64_t q, int32_t *used_exact)
{
    using namespace pgo;
    Ctx c;
    c.n = n;
    c.pts = points;
    c.w = weights;
    compute_box(c);
    std::vector<Plane> pl(3);
    for (int i = 0; i < 3; ++i)
    {
        if (kinds[i] == 0)
            make_bisector(c, seed, ids[i], pl[i]);
        else
            make_box(c, seed, ids[i], pl[i]);
    }
    Vtx v;
    make_vertex(pl, 0, 1, 2, v);
    Plane pq;
    make_bisector(c, seed, q, pq);
    Cell cell;
    cell.planes = pl;
    int64_t ex = 0;
    bool r = removed_test(c, seed, cell, v, pq, &ex);
    if (used_exact)
        *used_exact = (int32_t)ex;
    return r ? 1 : 0;
}

int pgo_box(int64_t n, const float *points, float *lo, float *hi)
{
    pgo::Ctx c;
    c.n = n;
    c.pts = points;
    c.w = nullptr;
    pgo::compute_box(c);
    for (int k = 0; k < 3; ++k)
    {
        lo[k] = c.lo[k];
        hi[k] = c.hi[k];
    }
    return 0;
}

} // extern "C"
