// pg_cells.cu -- per-cell convex clipping, one warp per cell.
//
// Reference counterpart: compute_bvh_voronoi_kernel (voronoi_ultra.cu:39-141)
// and compute_bvh_power_diagram_kernel (laguerre_ultra.cu:43-174): one thread
// per cell, polyhedron state in a strided global scratch (ConvexCellMemory,
// faster_convex_cell.cuh:33-70), clipping by CCClipByPlane
// (faster_convex_cell.cuh:411-512) during a shrinking-radius BVH traversal
// (pwr_bvh.cuh:217-356).
//
// Here one warp owns a cell. The polyhedron lives in shared memory
// (struct CellMem: planes, vertices, plane ids, node queue, edge table); lanes
// own vertex slots (slot = k * 32 + lane). Candidates come in batches of up to
// 32 (one per lane): the caller's initial guesses, if any, then BVH leaves,
// best first from the seed's own leaf. A batch is filtered by a
// security-radius test, then by an FP32 vertex test with a rigorous error
// bound; the surviving candidates clip one at a time, nearest first:
//   1. every lane classifies its vertices (FP32 filter; undecided tests go to
//      the exact cascade of pg_exact.cuh);
//   2. the removed vertices' triangles (in the dual: each vertex is a triangle
//      of its three planes) give the boundary edges of the new face: a
//      directed edge x->y of a removed triangle whose reverse is not an edge
//      of another removed triangle (found through a per-warp bit table of
//      the removed triangles' edges); each boundary edge x->y makes the new
//      vertex (P, x, y) -- the reference builds the same cycle sequentially
//      in CCComputeBoundary (faster_convex_cell.cuh:322-388);
//   3. new vertices fill the freed slots (ballot / popc ranks), are computed
//      in FP32 by Cramer's rule with an a-posteriori error bound (residuals of
//      the exact planes at the computed point, per adjugate column), rebuilt
//      in FP64 when that bound is large.
// A BVH node is visited only if some vertex v could be removed by a point of
// the node's box: dist(v, box)^2 < |v - s|^2 + (max weight in box - w_s),
// tested lane-parallel over the vertices.
//
// A cell that needs more than 64 vertex / plane slots is deferred to a second
// launch with 128 slots in shared memory, and one that outgrows those to a
// third with 256 slots, also in shared memory (then 512 in a global slab); its status is then
// vertex_overflow (2) if the final cell has more than 64 vertices (the
// reference MAX_VERTS) and plane_overflow (1) only if even 512 slots overflow.
//
// With a geometry output, each final cell is also integrated before it is
// discarded (integrate_cell: volume and centroid from a fan of signed
// tetrahedra per face).
#include <atomic>
#include <cfloat>
#include <climits>
#include <type_traits>

#include "pg_common.cuh"
#include "pg_exact.cuh"
#include "pg_kernels.cuh"

namespace pg
{

constexpr float kEps = 5.9604645e-8f; // 2^-24
// resident blocks per SM of the two register budgets of the cell kernel (blocks_per_sm 2 and 3)
#ifndef PG_MINB_LO
#define PG_MINB_LO 2
#endif
#ifndef PG_MINB_HI
#define PG_MINB_HI 3
#endif
constexpr int kMinBlocksLo = PG_MINB_LO, kMinBlocksHi = PG_MINB_HI;
// A vertex whose FP32 error radius exceeds this fraction of its L1 norm is rebuilt in FP64.
#ifndef PG_VERTEX64_REL
#define PG_VERTEX64_REL 3e-4f
#endif
constexpr float kVertex64Rel = PG_VERTEX64_REL;
constexpr unsigned kFull = 0xFFFFFFFFu;

// A vertex is the triangle of its three plane slots, packed in 10-bit fields;
// a boundary edge (x, y) packs its two plane slots in 16-bit fields.
__host__ __device__ __forceinline__ unsigned tri_pack(unsigned a, unsigned b, unsigned c)
{
    return a | (b << 10) | (c << 20);
}
__host__ __device__ __forceinline__ unsigned tri_get(unsigned t, int e) { return (t >> (10 * e)) & 1023u; }

template <int CAP, int STACK> struct CellMem
{
    float4 pl[CAP];   // plane (n.x, n.y, n.z, h): interior n.x <= h (relative to the seed)
    float4 vx[CAP];   // vertex (X.x, X.y, X.z, psi), psi bounds the FP32 side-test error
    float pe[CAP];    // bound on |h - h_exact|
    float vr[CAP];    // (|X| + psi)^2, upper bound on |X_exact|^2
    int pid[CAP];     // >= 0: sorted point index; < 0: -1 - box code
    unsigned vt[CAP]; // plane slots of the vertex, tri_pack(p0, p1, p2) (oriented)
    unsigned eb[CAP]; // boundary edges x | y << 16 of the clip in progress, by rank
    int stk[STACK];   // pending BVH references (unordered)
    float skey[STACK]; // lower bound of the bisector distance of any point of the pending node
    unsigned long long cnt[kNumStats]; // per-warp statistics (written by lane 0)
    unsigned long long cnt0[3];        // nodes, leaves, candidates at the start of the current cell
    float cap;  // search radius of the current pass (learned / given; +inf without one)
    float done; // search radius of the finished first pass (-inf during the first pass)
    unsigned et[CAP * CAP / 32];       // edge table of the clip in progress (all zero between clips)
};

// Clear a warp's edge table (once, before its first clip).
template <int CAP, int STACK> __device__ __forceinline__ void clear_edges(CellMem<CAP, STACK> &m, int lane)
{
    for (int k = lane; k < CAP * CAP / 32; k += 32)
        m.et[k] = 0u;
    __syncwarp();
}

struct CellArgs
{
    const float4 *pts;
    const int *oid;
    const int *rank;
    const float4 *rec;
    const float *box;        // 8 floats per cloud: reference box lo xyz, hi xyz, max weight
    const int *cloud_off;    // [clouds + 1]
    const int *cloud_root;   // [clouds]
    int num_clouds;
    int n;
    int window;
    const int *guesses;
    const int *guess_off;
    int *rows;
    int *deg;
    int *status;
    int *big_list;
    int *big_list2; // cells that outgrew the middle tier too, and their deferred-row slots
    int *big_slot2;
    int *big_rows;
    int *counters;
    unsigned long long *stats;
    int64_t begin, end;
    int big_pass;
    int64_t big_cap;
    char *huge_slabs;
    float *radius_out; // optional per-cell diagnostics (original ids)
    int4 *work_out;
    float4 *geometry_out; // optional per-cell centroid and volume (original ids)
    int vertex_cap;            // optional vertex export (original ids)
    float4 *vertices_out;
    int *vertex_planes_out;
    int *vertex_count_out;
    const float *hint; // search radius per sorted slot (learned or given), or nullptr
    const int *rparent; // record node -> entry in its parent's record
    const int *pleaf;   // sorted point -> entry of its leaf
    int fp32_only;      // undecided FP32 side tests take the FP32 sign (no exact cascade)
};

enum Flag : int
{
    kFlagEmpty = 1,
    kFlagDefer = 2,
    kFlagError = 4,
};

template <int CAP> struct WarpState
{
    static constexpr int W = CAP / 32;
    unsigned valid[W];
    int np;
    float4 s;
    int si, soid;
    const float *box; // the cell's cloud box
    int root;         // the cell's cloud BVH root
    float rsafe;
    int flags;
    int peak; // longest node queue of the current cell
};

// statistics live in the warp's shared-memory block, not in registers
// The value is evaluated by every lane (it may contain warp-collective calls).
#define PG_COUNT(m, lane, idx, v)                                                                                      \
    do                                                                                                                 \
    {                                                                                                                  \
        unsigned long long pg_count_v_ = (unsigned long long)(v);                                                      \
        if ((lane) == 0)                                                                                               \
            (m).cnt[idx] += pg_count_v_;                                                                               \
    } while (0)

// Optional per-phase SM cycle counters (compile with -DPG_PHASE_CYCLES).
#ifdef PG_PHASE_CYCLES
#define PG_T0(t) long long t = clock64()
#define PG_T1(m, lane, idx, t) PG_COUNT(m, lane, idx, clock64() - (t))
#else
#define PG_T0(t)
#define PG_T1(m, lane, idx, t)
#endif

struct Cand
{
    float nx, ny, nz, h;
    float nrm;  // upper bound on |q - s|
    float cerr; // constant part of the side-test error bound
    float eh;   // bound on |h - h_exact|
    int id;     // sorted index
};

__device__ __forceinline__ Cand make_cand(float4 s, float4 q, int id)
{
    Cand c;
    c.nx = q.x - s.x;
    c.ny = q.y - s.y;
    c.nz = q.z - s.z;
    float n2 = __fmaf_rn(c.nx, c.nx, __fmaf_rn(c.ny, c.ny, __fmul_rn(c.nz, c.nz)));
    float dw = q.w - s.w;
    c.h = 0.5f * __fsub_rn(n2, dw);
    c.eh = 2.0f * kEps * (fabsf(c.h) + 3.0f * n2 + fabsf(dw));
    c.nrm = n2 * rsqrtf(n2) * (1.0f + 4e-6f); // rsqrtf: <= 2 ulp
    c.cerr = (3.0f * kEps * fabsf(c.h) + c.eh) * (1.0f + 8.0f * kEps);
    if (!(n2 > 1e-30f && n2 < 1e30f))
        c.cerr = INFINITY; // out of the filter's range: always exact
    c.id = id;
    return c;
}

__device__ __forceinline__ Cand shfl_cand(const Cand &c, int src)
{
    Cand r;
    r.nx = __shfl_sync(kFull, c.nx, src);
    r.ny = __shfl_sync(kFull, c.ny, src);
    r.nz = __shfl_sync(kFull, c.nz, src);
    r.h = __shfl_sync(kFull, c.h, src);
    r.nrm = __shfl_sync(kFull, c.nrm, src);
    r.cerr = __shfl_sync(kFull, c.cerr, src);
    r.eh = __shfl_sync(kFull, c.eh, src);
    r.id = __shfl_sync(kFull, c.id, src);
    return r;
}

// +1 removed, 0 kept, -1 undecided
__device__ __forceinline__ int side_fp32(float4 X, const Cand &q)
{
    float g = __fmaf_rn(q.nx, X.x, __fmaf_rn(q.ny, X.y, __fmaf_rn(q.nz, X.z, -q.h)));
    float b = __fmaf_rn(q.nrm, X.w, q.cerr) * (1.0f + 1e-6f);
    return g > b ? 1 : (g < -b ? 0 : -1);
}

// Source of plane `pid` (a sorted point index, or -1 - box code) of a cell
// whose cloud box is `box`.
// Sign of the FP32 side value alone (1 removed, 0 kept), for FP32-only predicates.
__device__ __forceinline__ int side_fp32_sign(float4 X, const Cand &q)
{
    float g = __fmaf_rn(q.nx, X.x, __fmaf_rn(q.ny, X.y, __fmaf_rn(q.nz, X.z, -q.h)));
    return g > 0.0f ? 1 : 0;
}

__device__ __forceinline__ exact::PlaneSrc plane_src(int pid, const float4 *__restrict__ pts,
                                                     const int *__restrict__ oid, const float *__restrict__ box)
{
    exact::PlaneSrc r;
    if (pid >= 0)
    {
        float4 p = pts[pid];
        r.x = p.x;
        r.y = p.y;
        r.z = p.z;
        r.w = p.w;
        r.box = -1;
        r.oid = oid[pid];
    }
    else
    {
        int code = -1 - pid;
        r.x = box[(code & 1) * 3 + (code >> 1)];
        r.y = r.z = r.w = 0.0f;
        r.box = code;
        r.oid = -1;
    }
    return r;
}

// Exact cascade for one undecided test. Takes plain values so that no
// per-warp state has its address taken (which would move it to local memory).
__device__ __noinline__ int side_exact(int p0, int p1, int p2, int qid, const float4 *__restrict__ pts,
                                       const int *__restrict__ oid, const float *__restrict__ box, float4 s, int soid,
                                       int *used)
{
    exact::PlaneSrc vp[3] = {plane_src(p0, pts, oid, box), plane_src(p1, pts, oid, box), plane_src(p2, pts, oid, box)};
    exact::PlaneSrc cp = plane_src(qid, pts, oid, box);
    return exact::side_test(vp, cp, s.x, s.y, s.z, s.w, soid, used);
}

// Vertex of three planes (FP32 Cramer) with its side-test error radius psi.
__device__ __forceinline__ float4 make_vertex(float4 a, float ea, float4 b, float eb, float4 c, float ec, float &vr)
{
    float u0x = b.y * c.z - b.z * c.y, u0y = b.z * c.x - b.x * c.z, u0z = b.x * c.y - b.y * c.x;
    float u1x = c.y * a.z - c.z * a.y, u1y = c.z * a.x - c.x * a.z, u1z = c.x * a.y - c.y * a.x;
    float u2x = a.y * b.z - a.z * b.y, u2y = a.z * b.x - a.x * b.z, u2z = a.x * b.y - a.y * b.x;
    float D = a.x * u0x + a.y * u0y + a.z * u0z;
    float nx = a.w * u0x + b.w * u1x + c.w * u2x;
    float ny = a.w * u0y + b.w * u1y + c.w * u2y;
    float nz = a.w * u0z + b.w * u1z + c.w * u2z;
    // any FP32 point is acceptable here: the bound below is a-posteriori
    float rD = __frcp_rn(D);
    float X = nx * rD, Y = ny * rD, Z = nz * rD;
    float x2 = X * X + Y * Y + Z * Z;
    float xn = x2 > 0.0f ? x2 * rsqrtf(x2) * (1.0f + 4e-6f) : 0.0f;
    float la = fabsf(a.x) + fabsf(a.y) + fabsf(a.z);
    float lb = fabsf(b.x) + fabsf(b.y) + fabsf(b.z);
    float lc = fabsf(c.x) + fabsf(c.y) + fabsf(c.z);
    float ra = fabsf(__fmaf_rn(a.x, X, __fmaf_rn(a.y, Y, __fmaf_rn(a.z, Z, -a.w)))) + 4.0f * kEps * (la * xn + fabsf(a.w)) + ea;
    float rb = fabsf(__fmaf_rn(b.x, X, __fmaf_rn(b.y, Y, __fmaf_rn(b.z, Z, -b.w)))) + 4.0f * kEps * (lb * xn + fabsf(b.w)) + eb;
    float rc = fabsf(__fmaf_rn(c.x, X, __fmaf_rn(c.y, Y, __fmaf_rn(c.z, Z, -c.w)))) + 4.0f * kEps * (lc * xn + fabsf(c.w)) + ec;
    // X - X_exact = adj(A) r / D with the columns u0, u1, u2 of adj(A) and the residuals r, so
    // |X - X_exact| <= (ra |u0| + rb |u1| + rc |u2|) / |D|, each |u_i| bounded with its rounding
    // error (2 eps per product pair). Per-plane weighting keeps the bound tight for a vertex far
    // along a thin prism, whose large-offset box plane only moves it along the prism axis.
    float q0 = u0x * u0x + u0y * u0y + u0z * u0z;
    float q1 = u1x * u1x + u1y * u1y + u1z * u1z;
    float q2 = u2x * u2x + u2y * u2y + u2z * u2z;
    float U0 = (q0 > 0.0f ? q0 * rsqrtf(q0) * (1.0f + 4e-6f) : 0.0f) + 8.0f * kEps * lb * lc;
    float U1 = (q1 > 0.0f ? q1 * rsqrtf(q1) * (1.0f + 4e-6f) : 0.0f) + 8.0f * kEps * lc * la;
    float U2 = (q2 > 0.0f ? q2 * rsqrtf(q2) * (1.0f + 4e-6f) : 0.0f) + 8.0f * kEps * la * lb;
    float num = (ra * U0 + rb * U1 + rc * U2) * (1.0f + 4e-6f);
    float den = fabsf(D) - 8.0f * kEps * la * lb * lc;
    float ex = den > 0.0f ? __fdividef(num, den) * (1.0f + 4e-6f) : INFINITY;
    float psi = (2.0f * ex + 4.0f * kEps * xn) * (1.0f + 1e-6f);
    if (!(psi < 1e30f) || !(xn < 1e30f))
        psi = INFINITY;
    float r = xn + psi;
    vr = r * r * (1.0f + 1e-6f);
    return make_float4(X, Y, Z, psi);
}

// Vertex of three planes rebuilt in FP64 from the planes' sources (the FP32
// plane coefficients are themselves rounded), for a vertex whose FP32 error
// radius is large: three nearly dependent planes, e.g. two bisectors of
// near-coplanar points meeting a third along a long thin cell. Returns the FP32
// point with psi = 2 * (FP64 a-posteriori bound) + |X32 - X64| + the FP32
// side-test rounding term, or `fallback` when a plane is not exact in FP64.
__device__ __noinline__ float4 make_vertex64(int pid0, int pid1, int pid2, const float4 *__restrict__ pts,
                                             const int *__restrict__ oid, const float *__restrict__ box, float4 s,
                                             float4 fallback, float fallback_vr, float &vr)
{
    const double u = 1.1102230246251565e-16; // 2^-53
    exact::DRow r[3];
    exact::make_drow(plane_src(pid0, pts, oid, box), s.x, s.y, s.z, s.w, r[0]);
    exact::make_drow(plane_src(pid1, pts, oid, box), s.x, s.y, s.z, s.w, r[1]);
    exact::make_drow(plane_src(pid2, pts, oid, box), s.x, s.y, s.z, s.w, r[2]);
    if (!(r[0].ok && r[1].ok && r[2].ok))
    {
        vr = fallback_vr;
        return fallback;
    }
    // plane i: a_i . X = b_i / 2 with |b_i - b_i exact| <= eb_i
    const double *a = r[0].a, *b = r[1].a, *c = r[2].a;
    double u0x = b[1] * c[2] - b[2] * c[1], u0y = b[2] * c[0] - b[0] * c[2], u0z = b[0] * c[1] - b[1] * c[0];
    double u1x = c[1] * a[2] - c[2] * a[1], u1y = c[2] * a[0] - c[0] * a[2], u1z = c[0] * a[1] - c[1] * a[0];
    double u2x = a[1] * b[2] - a[2] * b[1], u2y = a[2] * b[0] - a[0] * b[2], u2z = a[0] * b[1] - a[1] * b[0];
    double D = a[0] * u0x + a[1] * u0y + a[2] * u0z;
    double h0 = 0.5 * r[0].b, h1 = 0.5 * r[1].b, h2 = 0.5 * r[2].b;
    double X = (h0 * u0x + h1 * u1x + h2 * u2x) / D;
    double Y = (h0 * u0y + h1 * u1y + h2 * u2y) / D;
    double Z = (h0 * u0z + h1 * u1z + h2 * u2z) / D;
    double la = fabs(a[0]) + fabs(a[1]) + fabs(a[2]);
    double lb = fabs(b[0]) + fabs(b[1]) + fabs(b[2]);
    double lc = fabs(c[0]) + fabs(c[1]) + fabs(c[2]);
    double xn = sqrt(X * X + Y * Y + Z * Z) * (1.0 + 1e-14);
    double ra = fabs(fma(a[0], X, fma(a[1], Y, fma(a[2], Z, -h0)))) + 4.0 * u * (la * xn + fabs(h0)) + 0.5 * r[0].eb;
    double rb = fabs(fma(b[0], X, fma(b[1], Y, fma(b[2], Z, -h1)))) + 4.0 * u * (lb * xn + fabs(h1)) + 0.5 * r[1].eb;
    double rc = fabs(fma(c[0], X, fma(c[1], Y, fma(c[2], Z, -h2)))) + 4.0 * u * (lc * xn + fabs(h2)) + 0.5 * r[2].eb;
    double U0 = sqrt(u0x * u0x + u0y * u0y + u0z * u0z) * (1.0 + 1e-14) + 4.0 * u * lb * lc;
    double U1 = sqrt(u1x * u1x + u1y * u1y + u1z * u1z) * (1.0 + 1e-14) + 4.0 * u * lc * la;
    double U2 = sqrt(u2x * u2x + u2y * u2y + u2z * u2z) * (1.0 + 1e-14) + 4.0 * u * la * lb;
    double den = fabs(D) - 8.0 * u * la * lb * lc;
    if (!(den > 0.0) || !(xn < 1e30))
    {
        vr = fallback_vr;
        return fallback;
    }
    double ex = (ra * U0 + rb * U1 + rc * U2) / den * (1.0 + 1e-13);
    float fx = (float)X, fy = (float)Y, fz = (float)Z;
    double dx = (double)fx - X, dy = (double)fy - Y, dz = (double)fz - Z;
    double e32 = sqrt(dx * dx + dy * dy + dz * dz) * (1.0 + 1e-14);
    float x2 = fx * fx + fy * fy + fz * fz;
    float xnf = x2 > 0.0f ? x2 * rsqrtf(x2) * (1.0f + 4e-6f) : 0.0f;
    float psi = (float)((2.0 * ex + e32) * (1.0 + 1e-6)) * (1.0f + 1e-6f) + 4.0f * kEps * xnf;
    if (!(psi < fallback.w))
    {
        vr = fallback_vr;
        return fallback;
    }
    float rr = xnf + psi;
    vr = rr * rr * (1.0f + 1e-6f);
    return make_float4(fx, fy, fz, psi);
}

template <int CAP, int STACK>
__device__ __forceinline__ void cell_init(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, const CellArgs &A, int lane)
{
    // 6 box planes (code = axis * 2 + side, side 1 = high face)
    if (lane < 6)
    {
        int ax = lane >> 1, hi = lane & 1;
        float sc = ax == 0 ? ws.s.x : (ax == 1 ? ws.s.y : ws.s.z);
        float b = ws.box[hi * 3 + ax];
        float h = hi ? __fsub_rn(b, sc) : __fsub_rn(sc, b);
        float sg = hi ? 1.0f : -1.0f;
        m.pl[lane] = make_float4(ax == 0 ? sg : 0.0f, ax == 1 ? sg : 0.0f, ax == 2 ? sg : 0.0f, h);
        m.pe[lane] = kEps * fabsf(h);
        m.pid[lane] = -1 - lane;
    }
    __syncwarp();
    // 8 corners; triples ordered so the outward normals have a positive triple product
    if (lane < 8)
    {
        int sx = lane & 1, sy = (lane >> 1) & 1, sz = (lane >> 2) & 1;
        int px = sx, py = 2 + sy, pz = 4 + sz;
        int sign = (sx ? 1 : -1) * (sy ? 1 : -1) * (sz ? 1 : -1);
        int p0 = sign > 0 ? px : py, p1 = sign > 0 ? py : px, p2 = pz;
        // a corner of the box: each coordinate is a plane offset (n = +-e_axis), exact up to that
        // offset's own error bound pe; psi as in make_vertex (2 x position bound + FP32 side-test term)
        float X = sx ? m.pl[px].w : -m.pl[px].w, Y = sy ? m.pl[py].w : -m.pl[py].w,
              Z = sz ? m.pl[pz].w : -m.pl[pz].w;
        float ex = (m.pe[px] + m.pe[py] + m.pe[pz]) * (1.0f + 1e-6f);
        float x2 = X * X + Y * Y + Z * Z;
        float xn = x2 > 0.0f ? x2 * rsqrtf(x2) * (1.0f + 4e-6f) : 0.0f;
        float psi = (2.0f * ex + 4.0f * kEps * xn) * (1.0f + 1e-6f);
        float rr = xn + psi;
        m.vx[lane] = make_float4(X, Y, Z, psi);
        m.vr[lane] = rr * rr * (1.0f + 1e-6f);
        m.vt[lane] = tri_pack((unsigned)p0, (unsigned)p1, (unsigned)p2);
    }
    __syncwarp();
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < WarpState<CAP>::W; ++k)
        ws.valid[k] = k == 0 ? 0xFFu : 0u;
    ws.np = 6;
    ws.flags = 0;
    float vr = lane < 8 ? m.vr[lane] : 0.0f;
    ws.rsafe = sqrtf(__uint_as_float(__reduce_max_sync(kFull, __float_as_uint(vr)))) * (1.0f + 1e-6f);
}

template <int W> __device__ __forceinline__ int count_bits(const unsigned (&m)[W])
{
    int c = 0;
#pragma unroll(W > 8 ? 1 : W)
    for (int k = 0; k < W; ++k)
        c += __popc(m[k]);
    return c;
}

// Drop planes no valid vertex references; renumber vertex triples.
template <int CAP, int STACK> __device__ __forceinline__ void gc_planes(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, int lane)
{
    constexpr int W = CAP / 32;
    unsigned lm[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        lm[k] = 0;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if ((ws.valid[k] >> lane) & 1u)
        {
            unsigned t = m.vt[k * 32 + lane];
            unsigned p[3] = {tri_get(t, 0), tri_get(t, 1), tri_get(t, 2)};
#pragma unroll
            for (int e = 0; e < 3; ++e)
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
                for (int kk = 0; kk < W; ++kk)
                    if ((int)(p[e] >> 5) == kk)
                        lm[kk] |= 1u << (p[e] & 31u);
        }
    unsigned live[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        live[k] = __reduce_or_sync(kFull, lm[k]);
    int pre[W];
    int acc = 0;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        pre[k] = acc;
        acc += __popc(live[k]);
    }
    float4 tpl[W];
    float tpe[W];
    int tpid[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        int p = k * 32 + lane;
        if (p < ws.np && ((live[k] >> lane) & 1u))
        {
            tpl[k] = m.pl[p];
            tpe[k] = m.pe[p];
            tpid[k] = m.pid[p];
        }
    }
    __syncwarp();
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        int p = k * 32 + lane;
        if (p < ws.np && ((live[k] >> lane) & 1u))
        {
            int q = pre[k] + __popc(live[k] & ((1u << lane) - 1u));
            m.pl[q] = tpl[k];
            m.pe[q] = tpe[k];
            m.pid[q] = tpid[k];
        }
    }
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if ((ws.valid[k] >> lane) & 1u)
        {
            unsigned t = m.vt[k * 32 + lane];
            unsigned out = 0;
#pragma unroll
            for (int e = 0; e < 3; ++e)
            {
                unsigned p = tri_get(t, e);
                unsigned q = 0;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
                for (int kk = 0; kk < W; ++kk)
                    if ((int)(p >> 5) == kk)
                        q = pre[kk] + __popc(live[kk] & ((1u << (p & 31u)) - 1u));
                out |= q << (10 * e);
            }
            m.vt[k * 32 + lane] = out;
        }
    ws.np = acc;
    __syncwarp();
}

// per-word vertex masks passed by value (an array whose address is taken lives in local memory)
template <int W> struct VMask
{
    unsigned w[W];
};

enum ClipResult : int
{
    kClipNone = 0,
    kClipChanged = 1,
    kClipEmptied = 2,
    kClipDefer = 3,
};

template <int CAP, int STACK>
__device__ __forceinline__ int clip(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, const Cand &q, const CellArgs &A, int lane)
{
    constexpr int W = CAP / 32;
    unsigned rem[W];
    unsigned tri[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        int r = 0;
        tri[k] = 0;
        if ((ws.valid[k] >> lane) & 1u)
        {
            int slot = k * 32 + lane;
            float4 X = m.vx[slot];
            r = side_fp32(X, q);
            if (r < 0 && A.fp32_only)
                r = side_fp32_sign(X, q);
            if (r < 0)
            {
                unsigned t = m.vt[slot];
                int used = 0;
                r = side_exact(m.pid[tri_get(t, 0)], m.pid[tri_get(t, 1)], m.pid[tri_get(t, 2)], q.id, A.pts, A.oid,
                               ws.box, ws.s, ws.soid, &used);
                atomicAdd(&m.cnt[kStatFp64], 1ull);
                if (used)
                    atomicAdd(&m.cnt[kStatExpansion], 1ull);
                if (r < 0)
                {
                    ws.flags |= kFlagError;
                    r = 0;
                }
            }
            if (r)
                tri[k] = m.vt[slot];
        }
        rem[k] = __ballot_sync(kFull, r == 1);
    }
    PG_COUNT(m, lane, kStatTests, count_bits(ws.valid));
    bool any = false, all = true;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        any = any || rem[k] != 0u;
        all = all && rem[k] == ws.valid[k];
    }
    if (!any)
        return kClipNone;
    if (all)
    {
        ws.flags |= kFlagEmpty;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
        for (int k = 0; k < W; ++k)
            ws.valid[k] = 0;
        return kClipEmptied;
    }
    if (ws.np >= CAP)
    {
        gc_planes(m, ws, lane);
        if (ws.np >= CAP)
            return kClipDefer;
        // plane slots were renumbered: reload the removed triangles
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
        for (int k = 0; k < W; ++k)
            if ((rem[k] >> lane) & 1u)
                tri[k] = m.vt[k * 32 + lane];
    }
    int P = ws.np++;
    if (lane == 0)
    {
        m.pl[P] = make_float4(q.nx, q.ny, q.nz, q.h);
        m.pe[P] = q.eh;
        m.pid[P] = q.id;
    }
    // boundary edges of the removed region: the directed edge x->y of a removed
    // triangle is a boundary edge iff y->x is not an edge of another removed
    // triangle. The removed triangles mark their edges in the warp's edge table
    // (bit x * CAP + y), each lane tests the reverses of its own edges, then the
    // marks are cleared (the table is all zero between clips).
    using Bits = typename std::conditional<(3 * W > 32), unsigned long long, unsigned>::type;
    Bits bf = 0; // bit k*3+e: edge e of my removed vertex in word k is a boundary edge
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if ((rem[k] >> lane) & 1u)
        {
            unsigned t = tri[k];
#pragma unroll
            for (int e = 0; e < 3; ++e)
            {
                unsigned bit = tri_get(t, e) * CAP + tri_get(t, (e + 1) % 3);
                atomicOr(&m.et[bit >> 5], 1u << (bit & 31u));
            }
        }
    __syncwarp();
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if ((rem[k] >> lane) & 1u)
        {
            unsigned t = tri[k];
#pragma unroll
            for (int e = 0; e < 3; ++e)
            {
                unsigned rbit = tri_get(t, (e + 1) % 3) * CAP + tri_get(t, e);
                if (!((m.et[rbit >> 5] >> (rbit & 31u)) & 1u))
                    bf |= (Bits)1u << (3 * k + e);
            }
        }
    __syncwarp();
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if ((rem[k] >> lane) & 1u)
        {
            unsigned t = tri[k];
#pragma unroll
            for (int e = 0; e < 3; ++e)
                m.et[(tri_get(t, e) * CAP + tri_get(t, (e + 1) % 3)) >> 5] = 0u;
        }
    // list the boundary edges in the warp's edge buffer, lane by lane (exclusive scan of the counts)
    int mine = 0;
    if constexpr (3 * W > 32)
        mine = __popcll(bf);
    else
        mine = __popc((unsigned)bf);
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        int v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += v;
    }
    const int nb = __shfl_sync(kFull, incl, 31);
    {
        int at = incl - mine;
#pragma unroll(W > 8 ? 1 : 3 * W)
        for (int f = 0; f < 3 * W; ++f)
            if ((bf >> f) & 1u)
            {
                unsigned my = tri[f / 3];
                m.eb[at++] = tri_get(my, f % 3) | (tri_get(my, (f % 3 + 1) % 3) << 16);
            }
    }
    int nv_new = count_bits(ws.valid) - count_bits(rem) + nb;
    if (nv_new > CAP)
        return kClipDefer;
    unsigned fr[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        fr[k] = ~ws.valid[k] | rem[k];
    __syncwarp(); // edge list, plane P and all reads of removed triangles are done
    float4 pP = m.pl[P];
    float eP = m.pe[P];
    unsigned nbits[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        nbits[k] = 0;
    bool ill = false; // a vertex built by this lane needs the FP64 rebuild
    // lane r builds the vertex (P, x, y) of the r-th boundary edge in the r-th free slot
    for (int r0 = 0; r0 < nb; r0 += 32)
    {
        int r = r0 + lane;
        if (r < nb)
        {
            unsigned xy = m.eb[r];
            unsigned x = xy & 0xFFFFu, y = xy >> 16;
            int rr = r, slot = -1;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
            for (int k = 0; k < W; ++k)
            {
                int c = __popc(fr[k]);
                if (slot < 0 && rr < c)
                    slot = k * 32 + (int)__fns(fr[k], 0, rr + 1);
                else if (slot < 0)
                    rr -= c;
            }
            if (slot >= 0 && slot < CAP)
            {
                float vr;
                float4 X = make_vertex(pP, eP, m.pl[x], m.pe[x], m.pl[y], m.pe[y], vr);
                ill = ill || !(X.w <= kVertex64Rel * (fabsf(X.x) + fabsf(X.y) + fabsf(X.z)));
                m.vx[slot] = X;
                m.vr[slot] = vr;
                m.vt[slot] = tri_pack((unsigned)P, x, y);
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
                for (int k = 0; k < W; ++k)
                    if ((slot >> 5) == k)
                        nbits[k] |= 1u << (slot & 31);
            }
            else
                ws.flags |= kFlagError; // unreachable: capacity was checked above
        }
    }
    // ill-conditioned in FP32: rebuild in FP64 so that the empty sphere stays tight
    if (__any_sync(kFull, ill))
    {
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
        for (int k = 0; k < W; ++k)
        {
            unsigned mm = nbits[k];
            while (mm)
            {
                int slot = k * 32 + __ffs(mm) - 1;
                mm &= mm - 1;
                float4 X = m.vx[slot];
                if (!(X.w <= kVertex64Rel * (fabsf(X.x) + fabsf(X.y) + fabsf(X.z))))
                {
                    unsigned t = m.vt[slot];
                    float vr = m.vr[slot];
                    m.vx[slot] = make_vertex64(m.pid[tri_get(t, 0)], m.pid[tri_get(t, 1)], m.pid[tri_get(t, 2)], A.pts, A.oid,
                                               ws.box, ws.s, X, vr, vr);
                    m.vr[slot] = vr;
                    atomicAdd(&m.cnt[kStatVertex64], 1ull);
                }
            }
        }
    }
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        ws.valid[k] = (ws.valid[k] & ~rem[k]) | __reduce_or_sync(kFull, nbits[k]);
    __syncwarp();
    PG_COUNT(m, lane, kStatClips, 1);
    return kClipChanged;
}

// Radius of the current cell: no vertex lies farther from the seed (with its error bound).
template <int CAP, int STACK> __device__ __forceinline__ float cell_radius(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, int lane)
{
    float mx = 0.0f;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < CAP / 32; ++k)
        if ((ws.valid[k] >> lane) & 1u)
            mx = fmaxf(mx, m.vr[k * 32 + lane]);
    return sqrtf(__uint_as_float(__reduce_max_sync(kFull, __float_as_uint(mx)))) * (1.0f + 1e-6f);
}

// The pruning radius: the cell's radius, capped by the pass's search radius (HINT)
template <int CAP, int STACK, bool HINT>
__device__ __forceinline__ void update_rsafe(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, int lane)
{
    float r = cell_radius(m, ws, lane);
    ws.rsafe = HINT ? fminf(r, m.cap) : r;
}

// Process one batch of candidates (one per lane, `have` marks real ones).
// Returns false when the cell is finished early (empty or deferred).
template <int CAP, int STACK, bool HINT>
__device__ __forceinline__ bool run_batch(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, bool have, const Cand &q, float key,
                                          const CellArgs &A, int lane, VMask<CAP / 32> vmask, bool masked,
                                          bool old_leaf = false)
{
    // security radius: no vertex can be removed when h - eh > |a| * rsafe (the pruning radius)
    if (have && (q.h - q.eh) > q.nrm * ws.rsafe * (1.0f + 1e-6f))
        have = false;
    // second pass of a capped cell: in a leaf the first pass visited, the candidates within
    // the first pass's radius were clipped then (or could not clip: the cell only shrinks)
    if (HINT && old_leaf && have && !((q.h - q.eh) > q.nrm * m.done * (1.0f + 1e-6f)))
        have = false;
    unsigned hv = __ballot_sync(kFull, have);
    if (hv == 0u)
        return true;
    PG_COUNT(m, lane, kStatCandidates, __popc(hv));
    if (masked)
    {
        // FP32 pre-check restricted to the vertices whose empty sphere reaches the
        // leaf's box: a point of the leaf can remove no other vertex.
        bool may = false;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
        for (int k = 0; k < CAP / 32; ++k)
        {
            unsigned mm = vmask.w[k] & ws.valid[k];
            while (mm)
            {
                int b = __ffs(mm) - 1;
                mm &= mm - 1;
                float4 X = m.vx[k * 32 + b];
                if (have && !may)
                    may = side_fp32(X, q) != 0;
            }
        }
        have = have && may;
    }
    unsigned todo = __ballot_sync(kFull, have);
    bool changed = false;
    while (todo)
    {
        unsigned kk = ((todo >> lane) & 1u) ? ((__float_as_uint(key) & ~31u) | (unsigned)lane) : 0xFFFFFFFFu;
        unsigned mn = __reduce_min_sync(kFull, kk);
        int src = (int)(mn & 31u);
        todo &= ~(1u << src);
        Cand c = shfl_cand(q, src);
        PG_T0(tc);
        int r = clip(m, ws, c, A, lane);
        PG_T1(m, lane, kStatCycClips, tc);
        if (r == kClipEmptied)
            return false;
        if (r == kClipDefer)
        {
            ws.flags |= kFlagDefer;
            PG_COUNT(m, lane, kStatDeferVerts, 1);
            return false;
        }
        changed = changed || r == kClipChanged;
    }
    if (changed)
        update_rsafe<CAP, STACK, HINT>(m, ws, lane);
    return true;
}

// Lower bound of the bisector distance t = (|a|^2 - dw) / (2 |a|) over the points
// of a box (relative to the seed), and the quick security-radius rejection.
template <int CAP>
__device__ __forceinline__ bool box_key(const WarpState<CAP> &ws, float lx, float ly, float lz, float hx, float hy,
                                        float hz, float mw, float &key)
{
    float rlx = lx - ws.s.x, rly = ly - ws.s.y, rlz = lz - ws.s.z;
    float rhx = hx - ws.s.x, rhy = hy - ws.s.y, rhz = hz - ws.s.z;
    float dx = fmaxf(fmaxf(rlx, -rhx), 0.0f), dy = fmaxf(fmaxf(rly, -rhy), 0.0f), dz = fmaxf(fmaxf(rlz, -rhz), 0.0f);
    float d2 = (dx * dx + dy * dy + dz * dz) * (1.0f - 1e-6f);
    float dm = mw - ws.s.w;
    float d = d2 > 0.0f ? d2 * rsqrtf(d2) * (1.0f - 4e-6f) : 0.0f; // lower bound of the box distance
    float t;
    if (dm <= 0.0f)
        t = 0.5f * d;
    else
    {
        float num = d2 - dm * (1.0f + 1e-6f);
        t = (num > 0.0f && d > 0.0f) ? __fdividef(num, 2.0f * d) * (1.0f - 4e-6f) : 0.0f;
    }
    key = t * (1.0f - 1e-5f);
    return !(key > ws.rsafe);
}

// Vertices whose empty sphere reaches the box: q in the box can remove v only
// if |v - q|^2 < |v - s|^2 + (w_q - w_s); per-word ballots in vm[].
template <int CAP, int STACK>
__device__ __forceinline__ bool node_vertex_mask(const CellMem<CAP, STACK> &m, const WarpState<CAP> &ws, float lx,
                                                 float ly, float lz, float hx, float hy, float hz, float mw, int lane,
                                                 VMask<CAP / 32> &vm)
{
    float rlx = lx - ws.s.x, rly = ly - ws.s.y, rlz = lz - ws.s.z;
    float rhx = hx - ws.s.x, rhy = hy - ws.s.y, rhz = hz - ws.s.z;
    float dm = mw - ws.s.w;
    float dmu = dm > 0.0f ? dm * (1.0f + 1e-6f) : dm * (1.0f - 1e-6f);
    bool any = false;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < CAP / 32; ++k)
    {
        bool may = false;
        if ((ws.valid[k] >> lane) & 1u)
        {
            int slot = k * 32 + lane;
            float4 X = m.vx[slot];
            float e = X.w + 1e-6f * (fabsf(X.x) + fabsf(X.y) + fabsf(X.z) + fabsf(rlx) + fabsf(rly) + fabsf(rlz) +
                                     fabsf(rhx) + fabsf(rhy) + fabsf(rhz));
            float ax = fmaxf(fmaxf(rlx - e - X.x, X.x - rhx - e), 0.0f);
            float ay = fmaxf(fmaxf(rly - e - X.y, X.y - rhy - e), 0.0f);
            float az = fmaxf(fmaxf(rlz - e - X.z, X.z - rhz - e), 0.0f);
            float lhs = (ax * ax + ay * ay + az * az) * (1.0f - 1e-6f);
            may = lhs < m.vr[slot] + dmu;
        }
        vm.w[k] = __ballot_sync(kFull, may);
        any = any || vm.w[k] != 0u;
    }
    return any;
}

// Returns false when the row does not fit the fast-pass row width (the cell
// is then deferred to the large-capacity pass).
template <int CAP, int STACK>
__device__ __forceinline__ bool write_outputs(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, const CellArgs &A, int lane,
                                              bool big)
{
    constexpr int W = CAP / 32;
    int oi = ws.soid;
    if (ws.flags & kFlagEmpty)
    {
        if (lane == 0)
        {
            A.deg[oi] = 0;
            A.status[oi] = kEmptyCell;
        }
        return true;
    }
    unsigned lm[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        lm[k] = 0;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if ((ws.valid[k] >> lane) & 1u)
        {
            unsigned t = m.vt[k * 32 + lane];
#pragma unroll
            for (int e = 0; e < 3; ++e)
            {
                unsigned p = tri_get(t, e);
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
                for (int kk = 0; kk < W; ++kk)
                    if ((int)(p >> 5) == kk)
                        lm[kk] |= 1u << (p & 31u);
            }
        }
    int o[W];
    unsigned has[W];
    int cnt = 0;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        unsigned live = __reduce_or_sync(kFull, lm[k]);
        int p = k * 32 + lane;
        o[k] = INT_MAX;
        if (p < ws.np && ((live >> lane) & 1u))
        {
            int id = m.pid[p];
            if (id >= 0)
                o[k] = A.oid[id];
        }
        has[k] = __ballot_sync(kFull, o[k] != INT_MAX);
        cnt += __popc(has[k]);
    }
    int rnk[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        rnk[k] = 0;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        unsigned mm = has[k];
        while (mm)
        {
            int b = __ffs(mm) - 1;
            mm &= mm - 1;
            int v = __shfl_sync(kFull, o[k], b);
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
            for (int kk = 0; kk < W; ++kk)
                rnk[kk] += (v < o[kk]);
        }
    }
    if (!big && cnt > kRowWidth)
        return false;
    int nverts = count_bits(ws.valid);
    int st = nverts > kMaxVertsRef ? kVertexOverflow : kSuccess;
    if (ws.flags & kFlagDefer)
        st = kPlaneOverflow; // only reachable in the large-capacity pass
    if (big && cnt > kBigRowWidth)
    {
        st = kPlaneOverflow; // more faces than a deferred row holds: keep the first ones
        cnt = kBigRowWidth;
    }
    int *row;
    if (big)
    {
        int bi = ws.si; // index in the deferred list
        row = A.big_rows + (size_t)bi * kBigRowWidth;
        if (lane == 0)
        {
            A.rows[(size_t)oi * kRowWidth] = bi;
            A.deg[oi] = cnt | (int)kBigFlag;
        }
    }
    else
    {
        row = A.rows + (size_t)oi * kRowWidth;
        if (lane == 0)
            A.deg[oi] = cnt;
    }
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if (o[k] != INT_MAX && rnk[k] < cnt)
            row[rnk[k]] = o[k];
    if (lane == 0)
        A.status[oi] = st;
    return true;
}

// One BVH leaf as a candidate batch (one point per lane).
template <int CAP, int STACK, bool GUESS, bool HINT>
__device__ __forceinline__ bool leaf_batch(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, int ref, int i,
                                           const CellArgs &A, int lane, VMask<CAP / 32> vm, bool old_leaf)
{
    PG_COUNT(m, lane, kStatLeaves, 1);
    int first = leaf_first(ref), count = leaf_count(ref);
    int j = first + lane;
    bool have = lane < count && j != i;
    Cand q;
    float qkey = 0.0f;
    if (have)
    {
        float4 p = A.pts[j];
        have = !(p.x == ws.s.x && p.y == ws.s.y && p.z == ws.s.z);
        q = make_cand(ws.s, p, j);
        qkey = q.nrm;
        if (GUESS)
            for (int t = 0; t < ws.np && have; ++t)
                have = m.pid[t] != j;
    }
    return run_batch<CAP, STACK, HINT>(m, ws, have, q, qkey, A, lane, vm, true, old_leaf);
}

// Best-first BVH traversal of one cell. A pending entry is (parent << 1 | side)
// with a lower bound of the bisector distance of the child's points; the
// entry with the smallest bound is popped, dropped if the bound exceeds the
// pruning radius (the radius of the since shrunk cell; with a search radius,
// at most that), else its box is tested against every vertex's empty sphere
// and, for a leaf, only the vertices that pass are pre-tested. Returns false
// when the cell finished early (emptied or deferred).
template <int CAP, int STACK, bool GUESS, bool HINT>
__device__ __forceinline__ bool traverse(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, int i, const CellArgs &A, int lane)
{
    const float4 *rec = A.rec;
    // Start at the seed's own leaf (bound 0) and queue the sibling of every node
    // on its path up to the cloud's root with its bound, instead of descending
    // from the root. A cloud whose root is a leaf starts with entry -2 (that
    // leaf, unbounded box).
    int sp = 1;
    if (ref_is_leaf(ws.root))
    {
        if (lane == 0)
        {
            m.stk[0] = -2;
            m.skey[0] = 0.0f;
        }
    }
    else
    {
        int e = A.pleaf[i];
        if (lane == 0)
        {
            m.stk[0] = e;
            m.skey[0] = 0.0f;
        }
        for (int lvl = 0; lvl < STACK - 1; ++lvl)
        {
            int parent = e >> 1, side = e & 1;
            if (e < 0 || parent >= A.n - 1)
            {
                ws.flags |= kFlagError; // unreachable: the path always meets the cloud's root
                break;
            }
            const float4 *r = rec + 4 * (size_t)parent;
            float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
            float k;
            bool p = side == 1 ? box_key(ws, r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r3.z, k)
                               : box_key(ws, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w, r3.w, k);
            if (p)
            {
                if (lane == 0)
                {
                    m.stk[sp] = (parent << 1) | (side ^ 1);
                    m.skey[sp] = k;
                }
                ++sp;
            }
            if (parent == ws.root)
                break;
            e = A.rparent[parent];
        }
    }
    ws.peak = max(ws.peak, sp);
    __syncwarp();
    while (sp > 0)
    {
        PG_T0(tn);
        int jb = sp - 1;
        float floor_key = 0.0f; // lower bound of every pending bound (best-first only)
        if (sp <= STACK - 64)
        {
            unsigned best = 0xFFFFFFFFu;
            for (int j = lane; j < sp; j += 32)
                best = min(best, (__float_as_uint(m.skey[j]) & ~(unsigned)(STACK - 1)) | (unsigned)j);
            best = __reduce_min_sync(kFull, best);
            jb = (int)(best & (unsigned)(STACK - 1));
            floor_key = __uint_as_float(best & ~(unsigned)(STACK - 1));
        }
        // else: a nearly full queue continues depth first (newest entry), which adds at most one
        // pending entry per tree level; the order of visits never changes the cell.
        int ent = m.stk[jb];
        float key = m.skey[jb];
        __syncwarp();
        if (lane == 0)
        {
            m.stk[jb] = m.stk[sp - 1];
            m.skey[jb] = m.skey[sp - 1];
        }
        --sp;
        __syncwarp();
        if (key > ws.rsafe)
        {
            PG_T1(m, lane, kStatCycNodes, tn);
            if (floor_key > ws.rsafe)
                break; // every pending bound exceeds the radius: the cell is final
            continue;
        }
        PG_COUNT(m, lane, kStatNodes, 1);
        float lx, ly, lz, hx, hy, hz, mw;
        int ref;
        if (ent < 0)
        {
            // the root leaf of a small cloud: every vertex may be removed by its points
            lx = ly = lz = -INFINITY;
            hx = hy = hz = INFINITY;
            mw = ws.box[6];
            ref = ws.root;
        }
        else
        {
            int parent = ent >> 1, side = ent & 1;
            const float4 *r = rec + 4 * (size_t)parent;
            float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
            if (side == 0)
            {
                lx = r0.x; ly = r0.y; lz = r0.z; hx = r0.w; hy = r1.x; hz = r1.y; mw = r3.z;
                ref = __float_as_int(r3.x);
            }
            else
            {
                lx = r1.z; ly = r1.w; lz = r2.x; hx = r2.y; hy = r2.z; hz = r2.w; mw = r3.w;
                ref = __float_as_int(r3.y);
            }
        }
        VMask<CAP / 32> vm;
        bool any = node_vertex_mask(m, ws, lx, ly, lz, hx, hy, hz, mw, lane, vm);
        PG_T1(m, lane, kStatCycNodes, tn);
        if (!any)
            continue;
        if (ref_is_leaf(ref))
        {
            PG_T0(tl);
            bool go = leaf_batch<CAP, STACK, GUESS, HINT>(m, ws, ref, i, A, lane, vm, HINT && !(key > m.done));
            PG_T1(m, lane, kStatCycLeaves, tl);
            if (!go)
                return false;
            continue;
        }
        PG_T0(tn2);
        // internal: queue both children with their distance bounds
        const float4 *rc = rec + 4 * (size_t)ref;
        float4 c0 = rc[0], c1 = rc[1], c2 = rc[2], c3 = rc[3];
        float k0, k1;
        bool p0 = box_key(ws, c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c3.z, k0);
        bool p1 = box_key(ws, c1.z, c1.w, c2.x, c2.y, c2.z, c2.w, c3.w, k1);
        if (sp + 2 > STACK)
        {
            ws.flags |= kFlagDefer;
            PG_COUNT(m, lane, kStatDeferStack, 1);
            return false;
        }
        if (lane == 0)
        {
            if (p0)
            {
                m.stk[sp] = ref << 1;
                m.skey[sp] = k0;
            }
            if (p1)
            {
                m.stk[sp + (p0 ? 1 : 0)] = (ref << 1) | 1;
                m.skey[sp + (p0 ? 1 : 0)] = k1;
            }
        }
        sp += (p0 ? 1 : 0) + (p1 ? 1 : 0);
        ws.peak = max(ws.peak, sp);
        __syncwarp();
        PG_T1(m, lane, kStatCycNodes, tn2);
    }    return true;
}

template <int CAP, int STACK, bool GUESS, bool HINT>
__device__ __forceinline__ void process_cell(CellMem<CAP, STACK> &m, WarpState<CAP> &ws, int i, const CellArgs &A, int lane)
{
    ws.s = A.pts[i];
    ws.si = i;
    ws.soid = A.oid[i];
    {
        int c = cloud_of(A.cloud_off, A.num_clouds, i);
        ws.box = A.box + 8 * c;
        ws.root = A.cloud_root[c];
    }
    cell_init(m, ws, A, lane);
    ws.peak = 0;
    if (A.work_out != nullptr && lane == 0)
    {
        m.cnt0[0] = m.cnt[kStatNodes];
        m.cnt0[1] = m.cnt[kStatLeaves];
        m.cnt0[2] = m.cnt[kStatCandidates];
    }
    const int n = A.n;
    const bool guessing = GUESS;
    PG_T0(tw);
    // 1. warm start: curve-order neighbours (or the caller's initial guesses)
    if (guessing)
    {
        int g0 = A.guess_off[ws.soid], g1 = A.guess_off[ws.soid + 1];
        for (int g = g0; g < g1; g += 32)
        {
            int j = -1;
            if (g + lane < g1)
            {
                int o = A.guesses[g + lane];
                if (o >= 0 && o < n)
                    j = A.rank[o];
            }
            bool have = j >= 0 && j != i;
            Cand q;
            float key = 0.0f;
            if (have)
            {
                float4 p = A.pts[j];
                have = !(p.x == ws.s.x && p.y == ws.s.y && p.z == ws.s.z);
                q = make_cand(ws.s, p, j);
                key = q.nrm;
                for (int t = 0; t < ws.np && have; ++t)
                    have = m.pid[t] != j;
            }
            // deduplicate within the batch: keep the first lane holding a point
            unsigned peers = __match_any_sync(kFull, have ? j : -2 - lane);
            if (have && (__ffs(peers) - 1) != lane)
                have = false;
            if (!run_batch<CAP, STACK, false>(m, ws, have, q, key, A, lane, VMask<CAP / 32>{}, false))
                return;
        }
    }
    PG_T1(m, lane, kStatCycWarm, tw);
    // 2. BVH traversal, best first (traverse). With a search radius R (learned or
    // given), the first pass prunes nodes and candidates at min(cell radius, R):
    // whatever lies beyond R cannot cut a cell whose radius is within R, so the
    // pass is certified when the final cell's radius is <= R (and it skips the
    // transient clips by points beyond R). Otherwise a second pass completes the
    // cell without the cap; in the leaves the first pass visited it takes only
    // the candidates beyond R.
    if (!HINT)
    {
        traverse<CAP, STACK, GUESS, false>(m, ws, i, A, lane);
        return;
    }
    float cap = INFINITY;
    if (A.hint != nullptr)
    {
        float rq = A.hint[i];
        if (rq > 0.0f && rq < 1e30f)
            cap = rq;
    }
    if (lane == 0)
    {
        m.cap = cap;
        m.done = -INFINITY;
    }
    __syncwarp();
    ws.rsafe = fminf(ws.rsafe, cap);
    for (int pass = 0;; ++pass) // one inlined copy of the traversal for both passes
    {
        if (!traverse<CAP, STACK, GUESS, true>(m, ws, i, A, lane))
            return;
        float r = cell_radius(m, ws, lane);
        ws.rsafe = r;
        if (pass == 1 || cap == INFINITY)
            return;
        if (r <= cap)
        {
            PG_COUNT(m, lane, kStatHintHit, 1);
            return;
        }
        PG_COUNT(m, lane, kStatHintMiss, 1);
        if (lane == 0)
        {
            m.cap = INFINITY;
            m.done = cap;
        }
        __syncwarp();
    }
}


// Optional per-cell diagnostics: certified radius and traversal work.
// The vertex of three planes solved in FP64 from the planes' sources (the
// bisector coefficients are exact differences of FP32 values), without the
// error bound of make_vertex64: a vertex of the cell geometry. Returns X
// unchanged when the planes do not give exact FP64 rows or a usable solve.
__device__ __noinline__ float4 vertex64_plain(int pid0, int pid1, int pid2, const float4 *__restrict__ pts,
                                              const int *__restrict__ oid, const float *__restrict__ box, float4 s,
                                              float4 X)
{
    exact::DRow r[3];
    exact::make_drow(plane_src(pid0, pts, oid, box), s.x, s.y, s.z, s.w, r[0]);
    exact::make_drow(plane_src(pid1, pts, oid, box), s.x, s.y, s.z, s.w, r[1]);
    exact::make_drow(plane_src(pid2, pts, oid, box), s.x, s.y, s.z, s.w, r[2]);
    if (!(r[0].ok && r[1].ok && r[2].ok))
        return X;
    const double *a = r[0].a, *b = r[1].a, *c = r[2].a;
    double u0x = b[1] * c[2] - b[2] * c[1], u0y = b[2] * c[0] - b[0] * c[2], u0z = b[0] * c[1] - b[1] * c[0];
    double u1x = c[1] * a[2] - c[2] * a[1], u1y = c[2] * a[0] - c[0] * a[2], u1z = c[0] * a[1] - c[1] * a[0];
    double u2x = a[1] * b[2] - a[2] * b[1], u2y = a[2] * b[0] - a[0] * b[2], u2z = a[0] * b[1] - a[1] * b[0];
    double D = a[0] * u0x + a[1] * u0y + a[2] * u0z;
    if (!(fabs(D) > 0.0))
        return X;
    double q = 0.5 / D;
    double x = (r[0].b * u0x + r[1].b * u1x + r[2].b * u2x) * q;
    double y = (r[0].b * u0y + r[1].b * u1y + r[2].b * u2y) * q;
    double z = (r[0].b * u0z + r[1].b * u1z + r[2].b * u2z) * q;
    return make_float4((float)x, (float)y, (float)z, X.w);
}

// Volume and centroid of the final cell (the cell's geometry, which the
// reference computes and discards: voronoi_ultra.cu:125-138). Each face a is
// fanned from the foot f_a of the perpendicular from an apex o onto its plane,
// so the cell is the signed union of the tetrahedra (o, f_a, v_t, v_u) over
// the directed edges v_t -> v_u of its faces. The vertex triangles are
// oriented consistently (each plane pair appears once in each direction), so
// the edge of face a that leaves vertex t = (a, b, c) ends at the vertex whose
// triangle holds the directed pair a -> c, and all terms share one sign.
// Writes (centroid x, y, z, volume); a deferred cell writes NaN (the larger
// pass overwrites it), an empty cell volume 0 and a NaN centroid.
// (the valid-slot masks arrive in m.eb, free once the cell is final)
template <int CAP, int STACK>
__device__ __forceinline__ void integrate_cell(CellMem<CAP, STACK> &m, const CellArgs &A, int lane, int soid, float4 s,
                                            const float *box)
{
    constexpr int W = WarpState<CAP>::W;
    unsigned valid[W];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        valid[k] = m.eb[k];
    // the directed plane pair (a -> c) that each of this lane's vertices needs, per rotation
    unsigned want[W][3];
    int succ[W][3];
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        unsigned t = m.vt[k * 32 + lane];
#pragma unroll
        for (int r = 0; r < 3; ++r)
        {
            want[k][r] = ((valid[k] >> lane) & 1u) ? (tri_get(t, r) << 10 | tri_get(t, (r + 2) % 3)) : ~0u;
            succ[k][r] = -1;
        }
    }
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int kj = 0; kj < W; ++kj)
    {
        unsigned vm = valid[kj];
        while (vm)
        {
            int j = kj * 32 + __ffs(vm) - 1;
            vm &= vm - 1;
            unsigned tj = m.vt[j];
            unsigned x0 = tri_get(tj, 0), x1 = tri_get(tj, 1), x2 = tri_get(tj, 2);
            unsigned e0 = x0 << 10 | x1, e1 = x1 << 10 | x2, e2 = x2 << 10 | x0;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
            for (int k = 0; k < W; ++k)
#pragma unroll
                for (int r = 0; r < 3; ++r)
                    if (want[k][r] == e0 || want[k][r] == e1 || want[k][r] == e2)
                        succ[k][r] = j;
        }
    }
    // apex: the mean vertex (inside the cell), not the seed, which a power cell may lie far from;
    // tetrahedra from a distant apex would cancel to the cell's small volume
    float ox = 0.0f, oy = 0.0f, oz = 0.0f, on = 0.0f;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
        if ((valid[k] >> lane) & 1u)
        {
            float4 v = m.vx[k * 32 + lane];
            ox += v.x;
            oy += v.y;
            oz += v.z;
            on += 1.0f;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        ox += __shfl_xor_sync(kFull, ox, o);
        oy += __shfl_xor_sync(kFull, oy, o);
        oz += __shfl_xor_sync(kFull, oz, o);
        on += __shfl_xor_sync(kFull, on, o);
    }
    ox /= on;
    oy /= on;
    oz /= on;
    float S = 0.0f, cx = 0.0f, cy = 0.0f, cz = 0.0f;
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
    for (int k = 0; k < W; ++k)
    {
        if (!((valid[k] >> lane) & 1u))
            continue;
        int slot = k * 32 + lane;
        unsigned t = m.vt[slot];
        float4 v = m.vx[slot];
        v.x -= ox;
        v.y -= oy;
        v.z -= oz;
#pragma unroll
        for (int r = 0; r < 3; ++r)
        {
            if (succ[k][r] < 0)
                continue;
            float4 p = m.pl[tri_get(t, r)];
            float4 u = m.vx[succ[k][r]];
            u.x -= ox;
            u.y -= oy;
            u.z -= oz;
            // foot of the perpendicular from the apex onto the plane n.x <= h
            float sc = (p.w - (p.x * ox + p.y * oy + p.z * oz)) / (p.x * p.x + p.y * p.y + p.z * p.z);
            float fx = p.x * sc, fy = p.y * sc, fz = p.z * sc;
            float d = fx * (v.y * u.z - v.z * u.y) + fy * (v.z * u.x - v.x * u.z) + fz * (v.x * u.y - v.y * u.x);
            S += d;
            cx += d * (fx + v.x + u.x);
            cy += d * (fy + v.y + u.y);
            cz += d * (fz + v.z + u.z);
        }
    }
    double dS = S, dx = cx, dy = cy, dz = cz;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        dS += __shfl_xor_sync(kFull, dS, o);
        dx += __shfl_xor_sync(kFull, dx, o);
        dy += __shfl_xor_sync(kFull, dy, o);
        dz += __shfl_xor_sync(kFull, dz, o);
    }
    if (lane == 0)
    {
        double q = 0.25 / dS;
        A.geometry_out[soid] =
            make_float4((float)((double)s.x + (double)ox + dx * q), (float)((double)s.y + (double)oy + dy * q),
                        (float)((double)s.z + (double)oz + dz * q), (float)(fabs(dS) / 6.0));
    }
}

// Vertex export of a final cell: its valid vertices (masks in m.eb) in slot
// order, relative to the seed with their error radius psi, which bounds the
// distance to the exact vertex, and their planes as original point ids (box
// planes -1 - code).
template <int CAP, int STACK>
__device__ __forceinline__ void write_vertices(CellMem<CAP, STACK> &m, const CellArgs &A, int lane, int soid)
{
    constexpr int W = WarpState<CAP>::W;
    const int cap = A.vertex_cap;
    int base = 0;
    for (int k = 0; k < W; ++k)
    {
        unsigned v = m.eb[k];
        if ((v >> lane) & 1u)
        {
            int rank = base + __popc(v & ((1u << lane) - 1u));
            if (rank < cap)
            {
                int slot = k * 32 + lane;
                size_t o = (size_t)soid * cap + rank;
                if (A.vertices_out != nullptr)
                    A.vertices_out[o] = m.vx[slot];
                if (A.vertex_planes_out != nullptr)
                {
                    unsigned t = m.vt[slot];
                    for (int e = 0; e < 3; ++e)
                    {
                        int pid = m.pid[tri_get(t, e)];
                        A.vertex_planes_out[o * 3 + e] = pid >= 0 ? A.oid[pid] : pid;
                    }
                }
            }
        }
        base += __popc(v);
    }
    if (lane == 0 && A.vertex_count_out != nullptr)
        A.vertex_count_out[soid] = base;
}

// The FP32 vertices are only as accurate as the side tests need (psi); before an
// export, rebuild in FP64 the ones whose bound exceeds 32 ulps of their size, so
// that each vertex is within about 2^-19 |v| of the exact one (a power cell far
// from its seed amplifies that by |v| / size). psi stays a valid bound.
template <int CAP, int STACK>
__device__ __forceinline__ void refine_vertices(CellMem<CAP, STACK> &m, const CellArgs &A, int lane, float4 s,
                                                const float *box)
{
    constexpr int W = WarpState<CAP>::W;
    for (int k = 0; k < W; ++k)
        if ((m.eb[k] >> lane) & 1u)
        {
            int slot = k * 32 + lane;
            float4 X = m.vx[slot];
            if (!(X.w <= 32.0f * kEps * (fabsf(X.x) + fabsf(X.y) + fabsf(X.z))))
            {
                unsigned t = m.vt[slot];
                m.vx[slot] = vertex64_plain(m.pid[tri_get(t, 0)], m.pid[tri_get(t, 1)], m.pid[tri_get(t, 2)], A.pts,
                                            A.oid, box, s, X);
            }
        }
    __syncwarp();
}

// Geometry and vertex export of a final cell (valid-slot masks in m.eb). A cell
// deferred to the larger pass writes NaN geometry and no vertices (that pass
// writes them); an empty cell volume 0, a NaN centroid and no vertices.
// (one non-inlined call site: the cell kernels keep their register allocation
// and code size when no export is asked for)
template <int CAP, int STACK>
__device__ __noinline__ void export_cell(CellMem<CAP, STACK> &m, const CellArgs &A, int lane, int soid, float4 s,
                                         const float *box, int flags)
{
    if (!(flags & (kFlagDefer | kFlagEmpty)))
        refine_vertices(m, A, lane, s, box);
    if (A.geometry_out != nullptr)
    {
        if (flags & (kFlagDefer | kFlagEmpty))
        {
            if (lane == 0)
            {
                float nan = __int_as_float(0x7fc00000);
                A.geometry_out[soid] = make_float4(nan, nan, nan, (flags & kFlagDefer) ? nan : 0.0f);
            }
        }
        else
            integrate_cell(m, A, lane, soid, s, box);
    }
    if ((A.vertex_count_out != nullptr || A.vertices_out != nullptr || A.vertex_planes_out != nullptr) &&
        !(flags & kFlagDefer))
        write_vertices(m, A, lane, soid);
}

template <int CAP, int STACK>
__device__ __forceinline__ void write_diagnostics(CellMem<CAP, STACK> &m, const WarpState<CAP> &ws,
                                                  const CellArgs &A, int lane)
{
    constexpr int W = WarpState<CAP>::W;
    if (A.geometry_out != nullptr || A.vertex_count_out != nullptr || A.vertices_out != nullptr ||
        A.vertex_planes_out != nullptr)
    {
        if (lane == 0)
        {
#pragma unroll(CAP > 256 ? 1 : CAP / 32)
            for (int k = 0; k < W; ++k)
                m.eb[k] = ws.valid[k];
        }
        __syncwarp();
        export_cell(m, A, lane, ws.soid, ws.s, ws.box, ws.flags);
    }
    if (lane != 0)
        return;
    if (A.radius_out != nullptr)
        A.radius_out[ws.soid] = (ws.flags & kFlagEmpty) ? 0.0f : ws.rsafe;
    if (A.work_out != nullptr)
        A.work_out[ws.soid] = make_int4((int)(m.cnt[kStatNodes] - m.cnt0[0]), (int)(m.cnt[kStatLeaves] - m.cnt0[1]),
                                        (int)(m.cnt[kStatCandidates] - m.cnt0[2]), ws.peak);
}

template <int CAP, int STACK> __device__ void flush_stats(CellMem<CAP, STACK> &m, const CellArgs &A, int lane)
{
    __syncwarp();
    if (lane < kNumStats && m.cnt[lane])
        atomicAdd(&A.stats[lane], m.cnt[lane]);
}

// The per-phase cycle counters describe the first pass; a deferred tier reports
// only its total (kStatCycBig).
template <int CAP, int STACK> __device__ __forceinline__ void deferred_phase_counters(CellMem<CAP, STACK> &m, int lane)
{
#ifdef PG_PHASE_CYCLES
    if (lane >= kStatCycCell && lane <= kStatCycOut)
        m.cnt[lane] = 0;
    __syncwarp();
#endif
}

// Rebuild cell i with 512 vertex / plane slots and a 2048-entry queue: the
// rare cell that outgrew the 256 slots (long cells of surface data reach a
// few hundred vertices). Its state lives in one of kHugeSlabs global slabs,
// one per such cell and build; returns false when they are used up (the
// caller keeps its plane-overflow result).
__device__ __noinline__ bool huge_cell(const CellArgs &A, int i, int lane, int slot)
{
    int hs = 0;
    if (lane == 0)
        hs = atomicAdd(&A.counters[4], 1);
    hs = __shfl_sync(kFull, hs, 0);
    if (hs >= kHugeSlabs)
        return false;
    auto &m = *reinterpret_cast<CellMem<kCapHuge, kStackHuge> *>(A.huge_slabs +
                                                                  hs * sizeof(CellMem<kCapHuge, kStackHuge>));
    WarpState<kCapHuge> ws;
    if (lane < kNumStats)
        m.cnt[lane] = 0;
    clear_edges(m, lane);
    process_cell<kCapHuge, kStackHuge, false, false>(m, ws, i, A, lane);
    write_diagnostics(m, ws, A, lane);
    if (__any_sync(kFull, ws.flags & kFlagError) && lane == 0)
        atomicExch(&A.counters[2], 1);
    ws.si = slot;
    write_outputs(m, ws, A, lane, true);
    deferred_phase_counters(m, lane);
    flush_stats(m, A, lane);
    return true;
}

template <int CAP, int STACK, bool GUESS, bool HINT>
__device__ __forceinline__ void cells_body(CellMem<CAP, STACK> &m, const CellArgs &A, int lane)
{
    WarpState<CAP> ws;
    if (lane < kNumStats)
        m.cnt[lane] = 0;
    clear_edges(m, lane);
    int64_t count = A.big_pass ? min((int64_t)A.counters[1], A.big_cap) : (A.end - A.begin);
    int *ctr = A.big_pass ? &A.counters[3] : &A.counters[0];
    for (;;)
    {
        int t = 0;
        if (lane == 0)
            t = atomicAdd(ctr, 1);
        t = __shfl_sync(kFull, t, 0);
        if (t >= count)
            break;
        int i = A.big_pass ? A.big_list[t] : (int)(A.begin + t);
        // a cell the learned model routed to the 128-slot tier (listed by the prediction)
        if (HINT && A.hint != nullptr && A.hint[i] < 0.0f)
            continue;
        PG_T0(tcell);
        process_cell<CAP, STACK, GUESS, HINT>(m, ws, i, A, lane);
        write_diagnostics(m, ws, A, lane);
        if (A.big_pass)
            ws.si = t; // the deferred-row slot
        if (__any_sync(kFull, ws.flags & kFlagError)) // a flag may be set on any lane
        {
            if (lane == 0)
                atomicExch(&A.counters[2], 1);
            ws.flags &= ~kFlagError;
        }
        if (A.big_pass && (ws.flags & kFlagDefer) && ws.si < A.big_cap && huge_cell(A, i, lane, ws.si))
            continue; // outgrew the 256 slots too: rebuilt with 512
        if (!(ws.flags & kFlagDefer) || A.big_pass)
        {
            PG_T0(to);
            bool done = write_outputs(m, ws, A, lane, A.big_pass != 0);
            PG_T1(m, lane, kStatCycOut, to);
            if (done)
            {
                PG_T1(m, lane, kStatCycCell, tcell);
                continue;
            }
        }
        PG_T1(m, lane, kStatCycCell, tcell);
        PG_COUNT(m, lane, kStatDeferred, 1);
        // deferred: placeholder outputs (an empty row) until the large-capacity pass
        if (lane == 0)
        {
            A.deg[ws.soid] = 0;
            A.status[ws.soid] = kPlaneOverflow;
            int d = atomicAdd(&A.counters[1], 1);
            A.big_list[d] = i;
        }
    }
    flush_stats(m, A, lane);
}

template <int MINB, bool GUESS, bool HINT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, MINB) k_cells_fast(CellArgs A)
{
    __shared__ CellMem<kCapFast, kStackFast> mem[kWarpsPerBlock];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    cells_body<kCapFast, kStackFast, GUESS, HINT>(mem[w], A, lane);
}


// Rebuild cell i with 256 vertex / plane slots and a 1024-entry queue in this
// warp's share of the block's shared memory: a cell that outgrew the 128 slots
// of the middle tier. A cell that outgrows the 256 slots too is rebuilt once
// more by huge_cell.
template <bool GUESS>
__device__ __forceinline__ void big_cell(CellMem<kCapBig, kStackBig> &m, const CellArgs &A, int i, int lane, int slot)
{
    WarpState<kCapBig> ws;
    if (lane < kNumStats)
        m.cnt[lane] = 0;
    PG_T0(tb);
    clear_edges(m, lane);
    process_cell<kCapBig, kStackBig, GUESS, false>(m, ws, i, A, lane);
    write_diagnostics(m, ws, A, lane);
    if (__any_sync(kFull, ws.flags & kFlagError) && lane == 0)
        atomicExch(&A.counters[2], 1);
    if (!((ws.flags & kFlagDefer) && huge_cell(A, i, lane, slot)))
    {
        ws.si = slot;
        write_outputs(m, ws, A, lane, true); // plane_overflow when even the 512 slots ran out
    }
    PG_T1(m, lane, kStatCycBig, tb);
    deferred_phase_counters(m, lane);
    flush_stats(m, A, lane);
}

// The middle tier's loop: the cells the first pass deferred (list index t =
// their deferred-row slot), with 128 slots; a cell that outgrows them is listed
// again for the 256-slot tier. A separate body from the first pass's, whose
// code (one inlined copy of traversal and clip) is kept as it is.
template <bool GUESS> __device__ __forceinline__ void mid_body(CellMem<kCapMid, kStackMid> &m, const CellArgs &A, int lane)
{
    WarpState<kCapMid> ws;
    if (lane < kNumStats)
        m.cnt[lane] = 0;
    clear_edges(m, lane);
    const int64_t count = min((int64_t)A.counters[1], A.big_cap);
    for (;;)
    {
        int t = 0;
        if (lane == 0)
            t = atomicAdd(&A.counters[3], 1);
        t = __shfl_sync(kFull, t, 0);
        if (t >= count)
            break;
        int i = A.big_list[t];
        PG_T0(tb);
        process_cell<kCapMid, kStackMid, GUESS, false>(m, ws, i, A, lane);
        write_diagnostics(m, ws, A, lane);
        if (__any_sync(kFull, ws.flags & kFlagError) && lane == 0)
            atomicExch(&A.counters[2], 1);
        ws.flags &= ~kFlagError;
        if (ws.flags & kFlagDefer)
        {
            // outgrew the 128 slots too: listed, with its row slot, for the launch after this one
            if (lane == 0)
            {
                int d = atomicAdd(&A.counters[5], 1);
                A.big_list2[d] = i;
                A.big_slot2[d] = t;
            }
            PG_T1(m, lane, kStatCycBig, tb);
            continue;
        }
        ws.si = t;
        write_outputs(m, ws, A, lane, true);
        PG_T1(m, lane, kStatCycBig, tb);
    }
    deferred_phase_counters(m, lane);
    flush_stats(m, A, lane);
}

// Third tier: the cells that outgrew the middle tier, one per warp at a time, each
// warp's 256-slot state in shared memory (kBigWarps warps per block; the 512-slot
// rebuilds keep theirs in global slabs).
template <bool GUESS> __global__ void __launch_bounds__(kBigWarps * 32, 2) k_cells_big(CellArgs A)
{
    extern __shared__ __align__(16) unsigned char big_smem[];
    auto *m = reinterpret_cast<CellMem<kCapBig, kStackBig> *>(big_smem) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    const int64_t count = min((int64_t)A.counters[5], A.big_cap);
    for (;;)
    {
        int t = 0;
        if (lane == 0)
            t = atomicAdd(&A.counters[6], 1);
        t = __shfl_sync(kFull, t, 0);
        if (t >= count)
            break;
        big_cell<GUESS>(*m, A, A.big_list2[t], lane, A.big_slot2[t]);
    }
}

// Middle tier: the cells that outgrew 64 slots, with 128 slots and a 512-entry
// queue in shared memory (its own launch, so its larger shared-memory carve-out
// does not shrink the first pass's L1).
template <bool GUESS> __global__ void __launch_bounds__(kMidWarps * 32, kMidBlocksPerSM) k_cells_mid(CellArgs A)
{
    extern __shared__ __align__(16) unsigned char mid_smem[];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto *m = reinterpret_cast<CellMem<kCapMid, kStackMid> *>(mid_smem) + w;
    mid_body<GUESS>(*m, A, lane);
}

int big_warps() { return 148 * kMaxWarpsPerSM; } // upper bound of resident cell warps
size_t huge_slab_bytes() { return sizeof(CellMem<kCapHuge, kStackHuge>) * (size_t)kHugeSlabs; }

static CellArgs make_args(const Workspace &ws, const CellLaunch &cl)
{
    CellArgs A;
    A.pts = ws.pts;
    A.oid = ws.oid;
    A.rank = ws.rank;
    A.rec = ws.records;
    A.box = ws.box;
    A.cloud_off = ws.cloud_off;
    A.cloud_root = ws.cloud_root;
    A.num_clouds = cl.num_clouds;
    A.n = (int)cl.n;
    A.window = cl.window;
    A.guesses = cl.guesses;
    A.guess_off = cl.guess_off;
    A.rows = ws.rows;
    A.deg = ws.deg;
    A.status = nullptr;
    A.big_list = ws.big_list;
    A.big_list2 = ws.big_list2;
    A.big_slot2 = ws.big_slot2;
    A.big_rows = ws.big_rows;
    A.counters = ws.counters;
    A.stats = ws.stats;
    A.begin = cl.cell_begin;
    A.end = cl.cell_end;
    A.big_pass = 0;
    A.big_cap = 0;
    A.huge_slabs = (char *)ws.huge_slabs;
    A.radius_out = cl.radius_out;
    A.work_out = reinterpret_cast<int4 *>(cl.work_out);
    A.geometry_out = reinterpret_cast<float4 *>(cl.geometry_out);
    A.vertex_cap = cl.vertex_cap;
    A.vertices_out = reinterpret_cast<float4 *>(cl.vertices_out);
    A.vertex_planes_out = cl.vertex_planes_out;
    A.vertex_count_out = cl.vertex_count_out;
    A.hint = cl.use_hint ? ws.hint : nullptr;
    A.rparent = ws.rparent;
    A.fp32_only = cl.fp32_only;
    A.pleaf = ws.pleaf;
    return A;
}

void cells_launch(const Workspace &ws, const CellLaunch &cl, int *status, int num_sms, cudaStream_t st)
{
    CellArgs A = make_args(ws, cl);
    A.status = status;
    cudaMemsetAsync(ws.counters, 0, sizeof(int), st); // work counter
    int64_t cells = cl.cell_end - cl.cell_begin;
    // variants: register budget (2 or 3 blocks per SM), initial guesses, search radius per cell
    void (*kern)(CellArgs);
    if (cl.guesses)
        kern = cl.use_hint ? k_cells_fast<kMinBlocksLo, true, true> : k_cells_fast<kMinBlocksLo, true, false>;
    else if (cl.use_hint)
        kern = cl.min_blocks == 3 ? k_cells_fast<kMinBlocksHi, false, true> : k_cells_fast<kMinBlocksLo, false, true>;
    else
        kern = cl.min_blocks == 3 ? k_cells_fast<kMinBlocksHi, false, false> : k_cells_fast<kMinBlocksLo, false, false>;
    // resident blocks per SM of this variant, queried once per (variant, device) and thread
    struct Occ
    {
        void (*kern)(CellArgs);
        int dev, blocks;
    };
    static thread_local Occ occ[16];
    static thread_local int occ_n = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    int blocks_per_sm = 0;
    for (int k = 0; k < occ_n; ++k)
        if (occ[k].kern == kern && occ[k].dev == dev)
            blocks_per_sm = occ[k].blocks;
    if (blocks_per_sm == 0)
    {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, kWarpsPerBlock * 32, 0);
        if (blocks_per_sm < 1)
            blocks_per_sm = 1;
        if (occ_n < 16)
            occ[occ_n++] = Occ{kern, dev, blocks_per_sm};
    }
    A.big_cap = cl.big_cap;
    int64_t grid = std::min<int64_t>((int64_t)num_sms * blocks_per_sm, big_warps() / kWarpsPerBlock);
    int64_t need = (cells + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (grid > need)
        grid = need;
    if (grid < 1)
        grid = 1;
    ++g_launches;
    kern<<<(unsigned)grid, kWarpsPerBlock * 32, 0, st>>>(A);
}

// The deferred counts stay on the device: fixed grids read them. The middle
// tier (shared memory) rebuilds the cells the first pass deferred; the global
// tier (256, then 512 slots) the ones that outgrow it.
void cells_big_launch(const Workspace &ws, const CellLaunch &cl, int *status, int64_t big_cap, cudaStream_t st)
{
    CellArgs A = make_args(ws, cl);
    A.status = status;
    A.big_cap = big_cap;
    const size_t mid_smem = sizeof(CellMem<kCapMid, kStackMid>) * kMidWarps;
    void (*mid)(CellArgs) = cl.guesses ? k_cells_mid<true> : k_cells_mid<false>;
    // the shared-memory opt-in is a per-device attribute of the kernel: set once per device
    static std::atomic<unsigned long long> mid_ready[2];
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(mid_ready[cl.guesses ? 1 : 0].load() & bit))
    {
        cudaFuncSetAttribute(mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mid_smem);
        mid_ready[cl.guesses ? 1 : 0].fetch_or(bit);
    }
    ++g_launches;
    mid<<<(unsigned)(148 * kMidBlocksPerSM), kMidWarps * 32, mid_smem, st>>>(A);
    // 2 blocks of kBigWarps warps per SM, 256-slot state in shared memory
    const size_t big_smem = sizeof(CellMem<kCapBig, kStackBig>) * kBigWarps;
    void (*bigk)(CellArgs) = cl.guesses ? k_cells_big<true> : k_cells_big<false>;
    static std::atomic<unsigned long long> big_ready[2];
    if (!(big_ready[cl.guesses ? 1 : 0].load() & bit))
    {
        cudaFuncSetAttribute(bigk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem);
        big_ready[cl.guesses ? 1 : 0].fetch_or(bit);
    }
    ++g_launches;
    bigk<<<(unsigned)(148 * 2), kBigWarps * 32, big_smem, st>>>(A);
}

} // namespace pg
