// pg_exact.cuh -- exact side test used when the FP32 filter of the cell
// clipper cannot decide.
//
// The clipper's decision (faster_convex_cell.cuh:280-285 CCVertexIsInHalfSpace
// in the reference, there in FP32 fast-math) is: "is cell vertex v strictly
// closer, in power distance, to candidate point p than to the seed s?".
// With coordinates relative to s, every plane is a row (a, beta) of the
// equation 2 a.x = beta:
//   bisector with point q : a = q - s, beta = |q - s|^2 - (w_q - w_s)
//   box face x_i >= lo    : a = -e_i,  beta = 2 (s_i - lo)
//   box face x_i <= hi    : a = +e_i,  beta = 2 (hi - s_i)
// A vertex is the intersection of three rows r0, r1, r2; the candidate is r3.
// With C_i = (-1)^(i+3) det3(a-parts of the rows other than i),
//   det4 = sum_i beta_i C_i,  D = C_3 = det3(a_0, a_1, a_2),
// the vertex is removed iff det4 * D < 0.
//
// Evaluation cascade:
//   1. double precision with a rigorous forward error bound (cofactors of the
//      vertex rows against the candidate row);
//   2. exact evaluation with floating-point expansions: Two-Sum, Two-Product,
//      Grow-Expansion, Scale-Expansion and Compress from J. R. Shewchuk,
//      "Adaptive Precision Floating-Point Arithmetic and Fast Robust
//      Geometric Predicates", Discrete & Computational Geometry 18, 1997;
//   3. if det4 == 0 exactly: Simulation of Simplicity (H. Edelsbrunner and
//      E. P. Muecke, ACM Transactions on Graphics 9, 1990) on the weights,
//      w_j -> w_j + eps_j with eps_i >> eps_j for original index i < j:
//      det4(eps) = det4 + eps_s * sum_{bisector rows i} C_i
//                       - sum_{bisector rows i} eps_{q_i} C_i,
//      whose sign is the sign of the coefficient of the largest eps present.
//
// The header compiles as host code too (g++), so the exact machinery is
// unit-tested on the CPU against an independent big-integer evaluation.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define PG_HD __host__ __device__ __forceinline__
#define PG_HD_NOINLINE __host__ __device__ __noinline__
#else
#define PG_HD inline
#define PG_HD_NOINLINE
#endif

namespace pg
{
namespace exact
{

constexpr int kMaxTerms = 48; // capacity of one expansion buffer

// ---------------------------------------------------------------------------
// Error-free transformations and expansion arithmetic (Shewchuk 1997).
// Expansions are stored with increasing magnitude, zero components removed.
// ---------------------------------------------------------------------------
PG_HD void two_sum(double a, double b, double &x, double &y)
{
    x = a + b;
    double bv = x - a;
    double av = x - bv;
    double br = b - bv;
    double ar = a - av;
    y = ar + br;
}

PG_HD void fast_two_sum(double a, double b, double &x, double &y)
{
    x = a + b;
    double bv = x - a;
    y = b - bv;
}

PG_HD void two_diff(double a, double b, double &x, double &y)
{
    x = a - b;
    double bv = a - x;
    double av = x + bv;
    double br = bv - b;
    double ar = a - av;
    y = ar + br;
}

PG_HD void two_product(double a, double b, double &x, double &y)
{
    x = a * b;
#if defined(__CUDA_ARCH__)
    y = fma(a, b, -x);
#else
    y = std::fma(a, b, -x);
#endif
}

// h = e + b (h may alias e; h needs room for n + 1 terms)
PG_HD int grow(const double *e, int n, double b, double *h)
{
    double q = b;
    int hn = 0;
    for (int i = 0; i < n; ++i)
    {
        double qn, hh;
        two_sum(q, e[i], qn, hh);
        q = qn;
        if (hh != 0.0)
            h[hn++] = hh;
    }
    if (q != 0.0 || hn == 0)
        h[hn++] = q;
    return hn;
}

// h = e + f (h must not alias f); returns length, or -1 on capacity overflow
PG_HD int sum(const double *e, int ne, const double *f, int nf, double *h)
{
    if (ne + nf > kMaxTerms)
        return -1;
    for (int i = 0; i < ne; ++i)
        h[i] = e[i];
    int hn = ne;
    for (int j = 0; j < nf; ++j)
        hn = grow(h, hn, f[j], h);
    return hn;
}

// h = e * b; returns length, or -1 on capacity overflow
PG_HD int scale(const double *e, int n, double b, double *h)
{
    if (n == 0 || b == 0.0)
    {
        h[0] = 0.0;
        return 1;
    }
    if (2 * n > kMaxTerms)
        return -1;
    double q, hh;
    int hn = 0;
    two_product(e[0], b, q, hh);
    if (hh != 0.0)
        h[hn++] = hh;
    for (int i = 1; i < n; ++i)
    {
        double p1, p0, s;
        two_product(e[i], b, p1, p0);
        two_sum(q, p0, s, hh);
        if (hh != 0.0)
            h[hn++] = hh;
        fast_two_sum(p1, s, q, hh);
        if (hh != 0.0)
            h[hn++] = hh;
    }
    if (q != 0.0 || hn == 0)
        h[hn++] = q;
    return hn;
}

// in-place compression; returns the new length
PG_HD int compress(double *e, int m)
{
    if (m <= 1)
        return m;
    double g[kMaxTerms];
    double q = e[m - 1];
    int bottom = m - 1;
    for (int i = m - 2; i >= 0; --i)
    {
        double qn, qq;
        fast_two_sum(q, e[i], qn, qq);
        if (qq != 0.0)
        {
            g[bottom--] = qn;
            q = qq;
        }
        else
            q = qn;
    }
    g[bottom] = q;
    int top = 0;
    for (int i = bottom + 1; i < m; ++i)
    {
        double qn, qq;
        fast_two_sum(g[i], q, qn, qq);
        if (qq != 0.0)
            e[top++] = qq;
        q = qn;
    }
    e[top++] = q;
    return top;
}

PG_HD int sign_of(const double *e, int n)
{
    for (int i = n - 1; i >= 0; --i)
        if (e[i] != 0.0)
            return e[i] > 0.0 ? 1 : -1;
    return 0;
}

PG_HD void negate(double *e, int n)
{
    for (int i = 0; i < n; ++i)
        e[i] = -e[i];
}

// h = e * f, compressed; h must not alias e or f. Returns -1 on overflow.
PG_HD int mul(const double *e, int ne, const double *f, int nf, double *h)
{
    double t[kMaxTerms];
    double acc[kMaxTerms];
    int na = 0;
    for (int j = 0; j < nf; ++j)
    {
        int nt = scale(e, ne, f[j], t);
        if (nt < 0)
            return -1;
        int nn = sum(acc, na, t, nt, h);
        if (nn < 0)
            return -1;
        nn = compress(h, nn);
        for (int i = 0; i < nn; ++i)
            acc[i] = h[i];
        na = nn;
    }
    if (na == 0)
    {
        h[0] = 0.0;
        return 1;
    }
    for (int i = 0; i < na; ++i)
        h[i] = acc[i];
    return na;
}

// h = e - f, compressed; h must not alias f. Returns -1 on overflow.
PG_HD int diff(const double *e, int ne, const double *f, int nf, double *h)
{
    double nfv[kMaxTerms];
    if (nf > kMaxTerms)
        return -1;
    for (int i = 0; i < nf; ++i)
        nfv[i] = -f[i];
    int n = sum(e, ne, nfv, nf, h);
    return n < 0 ? -1 : compress(h, n);
}

// ---------------------------------------------------------------------------
// Plane rows built from the FP32 inputs.
// ---------------------------------------------------------------------------
struct PlaneSrc
{
    float x, y, z, w; // bisector: the neighbour point and weight; box: value in x
    int box;          // -1 for a bisector, else 0..5 (axis*2 + side, side 1 = high)
    int oid;          // original index of the neighbour (SoS order), -1 for a box face
};

struct Row
{
    double a[3][2];
    int na[3];
    double b[16];
    int nb;
    int oid;
};

// exact FP32 difference as an expansion of <= 2 terms
PG_HD int diff_f(float p, float q, double *out)
{
    double x, y;
    two_diff((double)p, (double)q, x, y);
    int n = 0;
    if (y != 0.0)
        out[n++] = y;
    if (x != 0.0 || n == 0)
        out[n++] = x;
    return n;
}

PG_HD bool make_row(const PlaneSrc &p, float sx, float sy, float sz, float sw, Row &r)
{
    r.oid = p.oid;
    if (p.box < 0)
    {
        float sc[3] = {sx, sy, sz};
        float qc[3] = {p.x, p.y, p.z};
        double acc[kMaxTerms];
        int nacc = 0;
        for (int k = 0; k < 3; ++k)
        {
            r.na[k] = diff_f(qc[k], sc[k], r.a[k]);
            double sq[kMaxTerms], t[kMaxTerms];
            int ns = mul(r.a[k], r.na[k], r.a[k], r.na[k], sq);
            if (ns < 0)
                return false;
            int nt = sum(acc, nacc, sq, ns, t);
            if (nt < 0)
                return false;
            for (int i = 0; i < nt; ++i)
                acc[i] = t[i];
            nacc = nt;
        }
        double dw[2];
        int ndw = diff_f(p.w, sw, dw);
        double t[kMaxTerms];
        int nt = diff(acc, nacc, dw, ndw, t);
        if (nt < 0 || nt > 16)
            return false;
        for (int i = 0; i < nt; ++i)
            r.b[i] = t[i];
        r.nb = nt;
    }
    else
    {
        int ax = p.box >> 1;
        double sg = (p.box & 1) ? 1.0 : -1.0;
        for (int k = 0; k < 3; ++k)
        {
            r.a[k][0] = k == ax ? sg : 0.0;
            r.na[k] = 1;
        }
        float sc = ax == 0 ? sx : (ax == 1 ? sy : sz);
        double d[2];
        int nd = (p.box & 1) ? diff_f(p.x, sc, d) : diff_f(sc, p.x, d);
        for (int i = 0; i < nd; ++i)
            r.b[i] = 2.0 * d[i];
        r.nb = nd;
    }
    return true;
}

// det3 of the a-parts of three rows; returns length or -1
PG_HD int det3(const Row &r0, const Row &r1, const Row &r2, double *out)
{
    double p[kMaxTerms], q[kMaxTerms], m[3][kMaxTerms];
    int nm[3];
    // minors of rows 1,2: m0 = yz, m1 = xz, m2 = xy
    const int ci[3][2] = {{1, 2}, {0, 2}, {0, 1}};
    for (int t = 0; t < 3; ++t)
    {
        int j = ci[t][0], k = ci[t][1];
        int np = mul(r1.a[j], r1.na[j], r2.a[k], r2.na[k], p);
        int nq = mul(r1.a[k], r1.na[k], r2.a[j], r2.na[j], q);
        if (np < 0 || nq < 0)
            return -1;
        nm[t] = diff(p, np, q, nq, m[t]);
        if (nm[t] < 0)
            return -1;
    }
    double acc[kMaxTerms], t[kMaxTerms];
    int na = 0;
    for (int c = 0; c < 3; ++c)
    {
        int np = mul(r0.a[c], r0.na[c], m[c], nm[c], p);
        if (np < 0)
            return -1;
        if (c == 1)
            negate(p, np);
        int nt = sum(acc, na, p, np, t);
        if (nt < 0)
            return -1;
        nt = compress(t, nt);
        for (int i = 0; i < nt; ++i)
            acc[i] = t[i];
        na = nt;
    }
    for (int i = 0; i < na; ++i)
        out[i] = acc[i];
    return na;
}

// ---------------------------------------------------------------------------
// Stage 1: double precision with a forward error bound. Returns +1 (removed),
// 0 (kept) or -1 (undecided).
// ---------------------------------------------------------------------------
struct DRow
{
    double a[3];
    double b;
    double eb;
    bool ok; // a[] exact
};

PG_HD bool exact_diff_d(double p, double q, double d)
{
    double x, y;
    two_diff(p, q, x, y);
    return y == 0.0 && x == d;
}

PG_HD void make_drow(const PlaneSrc &p, float sx, float sy, float sz, float sw, DRow &r)
{
    const double u = 1.1102230246251565e-16;
    if (p.box < 0)
    {
        double qc[3] = {p.x, p.y, p.z}, sc[3] = {sx, sy, sz};
        bool ok = true;
        double n2 = 0.0;
        for (int k = 0; k < 3; ++k)
        {
            r.a[k] = qc[k] - sc[k];
            ok = ok && exact_diff_d(qc[k], sc[k], r.a[k]);
            n2 += r.a[k] * r.a[k];
        }
        double dw = (double)p.w - (double)sw;
        ok = ok && exact_diff_d(p.w, sw, dw);
        r.b = n2 - dw;
        r.eb = 8.0 * u * (n2 + fabs(dw));
        r.ok = ok;
    }
    else
    {
        int ax = p.box >> 1;
        double sg = (p.box & 1) ? 1.0 : -1.0;
        r.a[0] = r.a[1] = r.a[2] = 0.0;
        r.a[ax] = sg;
        double sc = ax == 0 ? sx : (ax == 1 ? sy : sz);
        double d = (double)p.x - sc;
        r.b = 2.0 * sg * d;
        r.eb = 0.0;
        r.ok = exact_diff_d(p.x, sc, d);
    }
}

PG_HD int fp64_stage(const DRow v[3], const DRow &c)
{
    const double u = 1.1102230246251565e-16;
    if (!(v[0].ok && v[1].ok && v[2].ok && c.ok))
        return -1;
    double cf[4], ce[4];
    for (int j = 0; j < 4; ++j)
    {
        double m[3][3], e[3];
        int ecol = -1;
        for (int i = 0; i < 3; ++i)
        {
            int cc = 0;
            for (int col = 0; col < 4; ++col)
            {
                if (col == j)
                    continue;
                if (col == 3)
                {
                    m[i][cc] = v[i].b;
                    ecol = cc;
                }
                else
                    m[i][cc] = v[i].a[col];
                ++cc;
            }
            e[i] = v[i].eb;
        }
        double p00 = m[1][1] * m[2][2], p01 = m[1][2] * m[2][1];
        double p10 = m[1][0] * m[2][2], p11 = m[1][2] * m[2][0];
        double p20 = m[1][0] * m[2][1], p21 = m[1][1] * m[2][0];
        double d = m[0][0] * (p00 - p01) - m[0][1] * (p10 - p11) + m[0][2] * (p20 - p21);
        double perm = fabs(m[0][0]) * (fabs(p00) + fabs(p01)) + fabs(m[0][1]) * (fabs(p10) + fabs(p11)) +
                      fabs(m[0][2]) * (fabs(p20) + fabs(p21));
        double bnd = 8.0 * u * perm;
        if (ecol >= 0)
            for (int i = 0; i < 3; ++i)
            {
                if (e[i] == 0.0)
                    continue;
                int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (ecol + 1) % 3, j2 = (ecol + 2) % 3;
                bnd += e[i] * (fabs(m[i1][j1] * m[i2][j2]) + fabs(m[i1][j2] * m[i2][j1])) * (1.0 + 8.0 * u) +
                       e[i] * e[i];
            }
        cf[j] = ((j + 3) & 1) ? -d : d;
        ce[j] = bnd * (1.0 + 16.0 * u);
    }
    if (!(fabs(cf[3]) > ce[3]))
        return -1;
    double r[4] = {c.a[0], c.a[1], c.a[2], c.b};
    double val = 0.0, mag = 0.0, bnd = 0.0;
    for (int j = 0; j < 4; ++j)
    {
        val += cf[j] * r[j];
        mag += fabs(cf[j] * r[j]);
        bnd += ce[j] * fabs(r[j]);
    }
    bnd += (fabs(cf[3]) + ce[3]) * c.eb + 8.0 * u * mag;
    bnd *= (1.0 + 16.0 * u);
    if (!(fabs(val) > bnd))
        return -1;
    return ((val > 0.0) != (cf[3] > 0.0)) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Stage 2 + 3: exact expansions and SoS. Returns +1 removed, 0 kept,
// -2 on internal capacity overflow (reported as an error by the caller).
// ---------------------------------------------------------------------------
PG_HD_NOINLINE int expansion_stage(const PlaneSrc *vp, const PlaneSrc &cp, float sx, float sy, float sz, float sw,
                                   int seed_oid)
{
    Row rows[4];
    for (int i = 0; i < 3; ++i)
        if (!make_row(vp[i], sx, sy, sz, sw, rows[i]))
            return -2;
    if (!make_row(cp, sx, sy, sz, sw, rows[3]))
        return -2;
    double C[4][24];
    int nC[4];
    for (int i = 0; i < 4; ++i)
    {
        const Row *o[3];
        int k = 0;
        for (int j = 0; j < 4; ++j)
            if (j != i)
                o[k++] = &rows[j];
        double t[kMaxTerms];
        int n = det3(*o[0], *o[1], *o[2], t);
        if (n < 0 || n > 24)
            return -2;
        if ((i + 3) & 1)
            negate(t, n);
        for (int q = 0; q < n; ++q)
            C[i][q] = t[q];
        nC[i] = n;
    }
    int sD = sign_of(C[3], nC[3]);
    if (sD == 0)
        return 0;
    double acc[kMaxTerms], t[kMaxTerms], h[kMaxTerms];
    int na = 0;
    for (int i = 0; i < 4; ++i)
    {
        int nt = mul(rows[i].b, rows[i].nb, C[i], nC[i], t);
        if (nt < 0)
            return -2;
        int nh = sum(acc, na, t, nt, h);
        if (nh < 0)
            return -2;
        nh = compress(h, nh);
        for (int q = 0; q < nh; ++q)
            acc[q] = h[q];
        na = nh;
    }
    int s4 = sign_of(acc, na);
    if (s4 == 0)
    {
        // Simulation of Simplicity on the weights
        double S[kMaxTerms];
        int nS = 0;
        bool any = false;
        for (int i = 0; i < 4; ++i)
        {
            if (rows[i].oid < 0)
                continue;
            int nh = sum(S, nS, C[i], nC[i], h);
            if (nh < 0)
                return -2;
            nh = compress(h, nh);
            for (int q = 0; q < nh; ++q)
                S[q] = h[q];
            nS = nh;
            any = true;
        }
        // visit the perturbation terms by increasing original index
        int done = 0; // bitmask of rows consumed (bit 4 = seed)
        for (int step = 0; step < 5 && s4 == 0; ++step)
        {
            int best = -1;
            long long bid = 0x7fffffffffffffffLL;
            for (int i = 0; i < 4; ++i)
                if (rows[i].oid >= 0 && !(done & (1 << i)) && (long long)rows[i].oid < bid)
                {
                    bid = rows[i].oid;
                    best = i;
                }
            if (any && !(done & 16) && (long long)seed_oid < bid)
            {
                best = 4;
                bid = seed_oid;
            }
            if (best < 0)
                break;
            done |= 1 << best;
            if (best == 4)
                s4 = sign_of(S, nS);
            else
                s4 = -sign_of(C[best], nC[best]);
        }
        if (s4 == 0)
            return 0;
    }
    return (s4 * sD < 0) ? 1 : 0;
}

// Full cascade. Returns +1 removed, 0 kept, -2 internal overflow.
PG_HD int side_test(const PlaneSrc *vp, const PlaneSrc &cp, float sx, float sy, float sz, float sw, int seed_oid,
                    int *used_expansions)
{
    DRow dv[3], dc;
    for (int i = 0; i < 3; ++i)
        make_drow(vp[i], sx, sy, sz, sw, dv[i]);
    make_drow(cp, sx, sy, sz, sw, dc);
    int r = fp64_stage(dv, dc);
    if (r >= 0)
        return r;
    if (used_expansions)
        *used_expansions = 1;
    return expansion_stage(vp, cp, sx, sy, sz, sw, seed_oid);
}

} // namespace exact
} // namespace pg
