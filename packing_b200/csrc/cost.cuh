// cost.cuh -- batched tree-pair + boundary cost and gradient.
//
// One CTA evaluates one packing (instance).  Work per instance:
//   phase 0  thread per tree: pose -> (x, y, cos, sin), piece AABBs relative to
//            the tree centre, and the boundary term (pack_cuda.py:550-642).
//   phase A  every unordered pair {i, j} once (not both orders as the
//            reference's 2-threads-per-ref-tree loop does, pack_cuda.py:404-464),
//            centre cull at (2R)^2, then the 16 piece-pair AABB tests; the
//            surviving piece pairs are appended to a shared-memory work list
//            (warp ballot + one shared atomic per warp).
//   phase B  thread per listed piece pair: intersection area (or SAT
//            penetration) with the gradient of BOTH trees' poses, added into
//            per-tree int64 fixed-point accumulators (order-independent, so
//            deterministic), flushed whenever the list fills.
//   phase C  per-tree gradients out; totals by fixed-order reductions.
// Coordinates are taken relative to tree i's centre so the clipper works on
// O(1) numbers whatever the packing's extent.
#pragma once
#include "common.cuh"

struct PkCostSmem {
    float4* pose;       // [n_max] x, y, cos, sin
    float* theta;       // [n_max]
    float4* aabb;       // [4*n_max] per piece: minx, maxx, miny, maxy (centre-relative)
    unsigned* acc_lo;   // [3*n_max] fixed-point gradient, low words
    unsigned* acc_hi;   // [3*n_max] fixed-point gradient, high words
    float4* bnd;        // [n_max] boundary: cost, dh0, dh1, dh2 (unweighted)
    uint32_t* items;    // [cap_items] piece pairs: i | j << 11 | pi << 22 | pj << 24
    uint32_t* near;     // [cap_near] centre-culled pairs: i | j << 11
    int* count;         // items in the list
    double* red;        // [32]
    long long* redl;    // [32]
    float2* piece;      // [16]
    float4* piece4;     // [8] per piece: (x0, x1, x2, x3), (y0, y1, y2, y3)
    int* piece_nv;      // [4]
    unsigned int* cnt;  // [4] candidate pairs tested, near pairs, piece pairs, evaluations; then
                        // [4] kept near list: state (-1 off, 0 build next, 1 valid), length,
                        // filter flag, list distance (pk_nlist)
    int* cell_start;    // [grid_cap + 1] first sorted slot of each grid cell
    int* cell_fill;     // [grid_cap] trees per cell, then a scratch cursor
    int* sorted;        // [n_max] tree indices ordered by cell
    int* tcell;         // [n_max] cell of each tree
    int* near_cnt;      // [n_max] near pairs of each sorted position
    int* near_start;    // [n_max + 1] their offsets (exclusive scan)
    int cap_items, cap_near, grid_cap, n_cap;
};

// Cells of the broad-phase grid (each at least the interaction distance
// wide): two per tree, at least 64, at most 1024.
__host__ __device__ inline int pk_grid_cap(int n_max) { return n_max < 32 ? 64 : (n_max > 512 ? 1024 : 2 * n_max); }

// List capacities.  The near list takes 8 T pairs, at least the n_max - 1
// pairs of one tree for every n_max that pk_cost_threads gives T for; an
// expansion chunk appends at most 16 T piece pairs to the item list, which is
// flushed before the next chunk could overflow it (the LUT's items are the
// near pairs themselves).
__host__ __device__ inline void pk_caps(int T, int mode, int* cap_near, int* cap_items)
{
    *cap_near = 8 * T;
    *cap_items = mode == PK_PAIR_LUT ? 0 : 20 * T;
}

// keep: room for the kept near list's state (the fused relaxation only; a
// one-shot evaluation keeps the smaller footprint, which lets the smallest
// size classes fit one more CTA per SM).
__host__ __device__ inline size_t pk_cost_smem_bytes(int n_max, int cap_near, int cap_items, bool keep = false)
{
    size_t b = 0;
    b += (size_t)n_max * 16;        // pose
    b += (size_t)n_max * 16;        // bnd
    b += (size_t)n_max * 64;        // aabb
    b += (size_t)n_max * 24;        // acc
    b += (size_t)n_max * 4;         // theta
    b += (size_t)cap_items * 4;     // items
    b += (size_t)cap_near * 4;      // near pairs
    b += (size_t)(2 * pk_grid_cap(n_max) + 1) * 4 + (size_t)n_max * 16 + 4;   // grid
    b += 32 * 8 + 32 * 8 + 16 * 8 + 4 * 4 + 16 + 16 + 16 + 16 + 128;
    if (keep) b += 16 + 32 * 4;   // pk_nlist, pk_disp
    return (b + 15) & ~(size_t)15;   // whatever follows starts 16-byte aligned
}

__device__ inline PkCostSmem pk_cost_carve(unsigned char* base, int n_max, int cap_near, int cap_items,
                                           bool keep = false)
{
    PkCostSmem s;
    unsigned char* p = base;
    s.pose = (float4*)p; p += (size_t)n_max * 16;
    s.bnd = (float4*)p; p += (size_t)n_max * 16;
    s.aabb = (float4*)p; p += (size_t)n_max * 64;
    s.piece4 = (float4*)p; p += 8 * 16;   // 16-byte aligned: every offset so far is a multiple of 16
    // 8-byte arrays next: every offset up to here is a multiple of 16
    s.red = (double*)p; p += 32 * 8;
    s.redl = (long long*)p; p += 32 * 8;
    if (keep) p += 32 * 4;   // pk_disp
    s.acc_lo = (unsigned*)p; p += (size_t)n_max * 12;
    s.acc_hi = (unsigned*)p; p += (size_t)n_max * 12;
    s.piece = (float2*)p; p += 16 * 8;
    s.theta = (float*)p; p += (size_t)n_max * 4;
    s.items = (uint32_t*)p; p += (size_t)cap_items * 4;
    s.near = (uint32_t*)p; p += (size_t)cap_near * 4;
    s.piece_nv = (int*)p; p += 16;
    s.count = (int*)p; p += 16;
    s.cnt = (unsigned int*)p; p += 16;
    if (keep) p += 16;   // pk_nlist
    s.grid_cap = pk_grid_cap(n_max);
    s.cell_start = (int*)p; p += (size_t)(s.grid_cap + 1) * 4;
    s.cell_fill = (int*)p; p += (size_t)s.grid_cap * 4;
    s.sorted = (int*)p; p += (size_t)n_max * 4;
    s.tcell = (int*)p; p += (size_t)n_max * 4;
    s.near_cnt = (int*)p; p += (size_t)n_max * 4;
    s.near_start = (int*)p; p += (size_t)n_max * 4 + 4;
    p += 16;
    s.cap_items = cap_items;
    s.cap_near = cap_near;
    s.n_cap = n_max;
    return s;
}

// Arrays placed right after cnt and redl by a carve with keep; derived from
// them rather than held as pointers of their own (fewer live registers around
// the clipper).
__device__ __forceinline__ int* pk_nlist(const PkCostSmem& sm) { return (int*)(sm.cnt + 4); }
__device__ __forceinline__ float* pk_disp(const PkCostSmem& sm) { return (float*)(sm.redl + 32); }

// ---------------------------------------------------------------------------
// Convex piece intersection area with the gradient of both rigid poses.
//
// The reference clips the subject piece against the clip piece edge by edge
// (Sutherland-Hodgman, pack_cuda_primitives.py:238-296, 348-538) and back-
// propagates through every stage for the subject's vertex gradient.  Here the
// same area is assembled from the boundary of P n Q directly: each edge of P
// is clipped to the part inside Q (parametric interval against Q's half-
// planes, inside = cross >= 0 as in :263-264) and each edge of Q to the part
// inside P.  With both pieces CCW, the area is sum 1/2 cross(a', b') over
// those portions (Green's theorem).  A rigid motion of P moves only the P
// portions, so dA/d(x, y) = sum of their outward normals N = len * n_hat and
// dA/dtheta = sum cross(midpoint - centre, N) (exact for straight edges).
// Collinear edges: a P edge lying on a Q edge line is excluded; a Q edge on a
// P edge line is kept only if both run the same way, so a shared boundary
// segment is counted once and touching pieces contribute zero.
// ---------------------------------------------------------------------------
// Near-collinear edges (all four endpoints within 2e-6 tree units of the
// other edge's line) are classified from the same four numbers on both
// passes, so the two passes can never disagree about a shared boundary.
#define PK_COLLINEAR_TOL2 4e-12f   // (2e-6)^2

// (b - a) x (c - a) with fixed rounding, so that the same four points give
// the same value wherever it is evaluated.
__device__ __forceinline__ float pk_cross3_rn(float2 a, float2 b, float2 c)
{
    return __fmaf_rn(b.x - a.x, c.y - a.y, -__fmul_rn(b.y - a.y, c.x - a.x));
}

// f[k][v] = cross(Y[k+1] - Y[k], X[v] - Y[k]): X's vertices against Y's
// edge lines (>= 0 inside).
__device__ __forceinline__ void pk_side_values(const float2 (&X)[4], const float2 (&Y)[4], float (&f)[4][4])
{
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int v = 0; v < 4; ++v) f[k][v] = pk_cross3_rn(Y[k], Y[(k + 1) & 3], X[v]);
}

// A convex piece's four vertices packed in pairs for the FP32x2 instructions
// of sm_100 (FFMA2 / FMUL2: two independent FP32 operations, each rounded
// like its scalar form): x01 = (x0, x1), x23 = (x2, x3), likewise y.
struct PkQuad { float2 x01, x23, y01, y23; };

__device__ __forceinline__ float2 pk_qv(const PkQuad& q, int v)
{
    return v == 0 ? make_float2(q.x01.x, q.y01.x) : v == 1 ? make_float2(q.x01.y, q.y01.y)
         : v == 2 ? make_float2(q.x23.x, q.y23.x) : make_float2(q.x23.y, q.y23.y);
}

__device__ __forceinline__ PkQuad pk_quad(const float2 (&V)[4])
{
    PkQuad q;
    q.x01 = make_float2(V[0].x, V[1].x); q.x23 = make_float2(V[2].x, V[3].x);
    q.y01 = make_float2(V[0].y, V[1].y); q.y23 = make_float2(V[2].y, V[3].y);
    return q;
}

// f[k][v] for the four lines of Y, two vertices of X per instruction, with
// the rounding of pk_cross3_rn (the vertex is taken relative to the line's
// first point before the cross product, which keeps small side values
// accurate wherever the pieces lie).
__device__ __forceinline__ void pk_side_values_q(const PkQuad& X, const PkQuad& Y, float (&f)[4][4])
{
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 a = pk_qv(Y, k), b = pk_qv(Y, (k + 1) & 3);
        const float ex = b.x - a.x, ey = b.y - a.y;
        const float2 ex2 = make_float2(ex, ex), ney2 = make_float2(-ey, -ey);
        const float2 nax2 = make_float2(-a.x, -a.x), nay2 = make_float2(-a.y, -a.y);   // x - a = x + (-a), exactly
        const float2 f01 = __ffma2_rn(ex2, __fadd2_rn(X.y01, nay2), __fmul2_rn(ney2, __fadd2_rn(X.x01, nax2)));
        const float2 f23 = __ffma2_rn(ex2, __fadd2_rn(X.y23, nay2), __fmul2_rn(ney2, __fadd2_rn(X.x23, nax2)));
        f[k][0] = f01.x; f[k][1] = f01.y; f[k][2] = f23.x; f[k][3] = f23.y;
    }
}

// One pass of the assembly: the portions of X's edges inside Y, added to A2
// (twice the area) and to g (gradient of X's rigid pose about centre ctr).
// f holds X's vertices against Y's lines.  Per vertex, a 4-bit mask of the
// lines it is outside of decides most edges without arithmetic: an edge
// with both ends outside one line is empty, an edge with neither end
// outside any line is whole, and only the lines it crosses get a crossing
// parameter.  Returns false when some line of Y has every vertex of X
// outside (separating axis: the pieces are disjoint).  KEEP_SAME_DIR: a
// collinear edge of X is kept when it runs the same way as Y's (X = Q) or
// always dropped (X = P).
template <bool KEEP_SAME_DIR>
__device__ __forceinline__ bool pk_clip_pass(const float2 (&X)[4], bool x_tri, const float2 (&Y)[4], bool y_tri,
                                             const float (&f)[4][4], float2 ctr, float& A2, float3& g)
{
    const float tiny = c_geom.coll_tiny;
    const unsigned lines = y_tri ? 0x7u : 0xFu;
    unsigned out[4], nearm[4] = {0u, 0u, 0u, 0u};
    float mn = 3.4e38f;   // smallest |f| against Y's real lines
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        unsigned o = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            o |= (unsigned)(f[k][v] < 0.f) << k;
            mn = fminf(mn, (k == 3 && y_tri) ? 3.4e38f : fabsf(f[k][v]));
        }
        out[v] = o & lines;
    }
    if (out[0] & out[1] & out[2] & out[3]) return false;
    if (mn <= tiny) {
        // some vertex lies within the tolerance of a line: the per-vertex
        // masks of near lines (rarely needed, so built only here)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            unsigned nm = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) nm |= (unsigned)(fabsf(f[k][v]) <= tiny) << k;
            nearm[v] = nm & lines;
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        if (v == 3 && x_tri) break;
        const int vb = (v + 1) & 3;
        const float2 a = X[v], b = X[vb];
        unsigned skip = 0;
        bool empty = false;
        const unsigned coll = nearm[v] & nearm[vb];
        if (coll) {
            // both ends within tolerance of some line of Y: confirm collinearity
            // with the symmetric four-number test (the other pass sees the same numbers)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!((coll >> k) & 1u)) continue;
                const float fa = f[k][v], fb = f[k][vb];
                const float2 ya = Y[k], yb = Y[(k + 1) & 3];
                const float2 ey = make_float2(yb.x - ya.x, yb.y - ya.y), ex = make_float2(b.x - a.x, b.y - a.y);
                const float ty = PK_COLLINEAR_TOL2 * __fmaf_rn(ey.x, ey.x, __fmul_rn(ey.y, ey.y));
                const float tx = PK_COLLINEAR_TOL2 * __fmaf_rn(ex.x, ex.x, __fmul_rn(ex.y, ex.y));
                const float ra = pk_cross3_rn(a, b, ya), rb = pk_cross3_rn(a, b, yb);
                if (fa * fa <= ty && fb * fb <= ty && ra * ra <= tx && rb * rb <= tx) {
                    if (!KEEP_SAME_DIR || ex.x * ey.x + ex.y * ey.y <= 0.f) empty = true;
                    skip |= 1u << k;
                }
            }
        }
        const unsigned oa = out[v] & ~skip, ob = out[vb] & ~skip;
        if (empty || (oa & ob)) continue;
        const unsigned crossm = oa | ob;
        float tin = 0.f, tout = 1.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if ((crossm >> k) & 1u) {
                const float fa = f[k][v], fb = f[k][vb];
                const float t = __fdividef(fa, fa - fb);
                if ((oa >> k) & 1u) tin = fmaxf(tin, t);    // entering
                else tout = fminf(tout, t);                 // leaving
            }
        }
        if (tin < tout) {
            const float dt = tout - tin;
            const float2 e = make_float2(b.x - a.x, b.y - a.y);
            A2 += dt * pk_cross(a, b);
            const float2 N = make_float2(dt * e.y, -dt * e.x);
            const float tm = 0.5f * (tin + tout);
            const float2 m = make_float2(a.x + tm * e.x - ctr.x, a.y + tm * e.y - ctr.y);
            g.x += N.x;
            g.y += N.y;
            g.z += pk_cross(m, N);
        }
    }
    return true;
}

__device__ __forceinline__ void pk_piece_area_grad_q(const PkQuad& PQ, bool p_tri, const PkQuad& QQ, bool q_tri,
                                                     float2 d, float& area, float3& gP, float3& gQ)
{
    float A2 = 0.f;   // twice the area
    gP = make_float3(0.f, 0.f, 0.f);
    gQ = make_float3(0.f, 0.f, 0.f);
    area = 0.f;
    const float2 P[4] = {pk_qv(PQ, 0), pk_qv(PQ, 1), pk_qv(PQ, 2), pk_qv(PQ, 3)};
    const float2 Q[4] = {pk_qv(QQ, 0), pk_qv(QQ, 1), pk_qv(QQ, 2), pk_qv(QQ, 3)};
    float f[4][4];
    pk_side_values_q(PQ, QQ, f);
    if (!pk_clip_pass<false>(P, p_tri, Q, q_tri, f, make_float2(0.f, 0.f), A2, gP)) return;
    pk_side_values_q(QQ, PQ, f);
    if (!pk_clip_pass<true>(Q, q_tri, P, p_tri, f, d, A2, gQ)) {
        gP = make_float3(0.f, 0.f, 0.f);
        return;
    }
    area = 0.5f * A2;
    if (!(area > 0.f)) {   // empty or numerically vanishing overlap
        area = 0.f;
        gP = make_float3(0.f, 0.f, 0.f);
        gQ = make_float3(0.f, 0.f, 0.f);
    }
}

__device__ __forceinline__ void pk_piece_area_grad(const float2 (&P)[4], bool p_tri,
                                                   const float2 (&Q)[4], bool q_tri, float2 d,
                                                   float& area, float3& gP, float3& gQ)
{
    pk_piece_area_grad_q(pk_quad(P), p_tri, pk_quad(Q), q_tri, d, area, gP, gQ);
}

// ---------------------------------------------------------------------------
// SAT penetration depth (sat_separation_with_grad_pose,
// pack_cuda_primitives.py:544-828) with the pose gradient of both pieces.
// Axes: P's edge normals, then Q's; a separating axis returns 0; the
// smallest overlap wins (strict <), pen1 <= pen2 selects case 1.  The
// reference evaluates each ordered pair and keeps the ref gradient; the
// other piece's gradient here is the same expression with the roles swapped
// (translation: the negative; rotation: its own extreme vertex, plus the
// axis-rotation term when the axis is one of its edges).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pk_piece_sat_grad(const float2 (&P)[4], bool p_tri, const float2 (&Q)[4],
                                                  bool q_tri, float2 d, float& sep, float3& gP,
                                                  float3& gQ)
{
    sep = 0.f;
    gP = make_float3(0.f, 0.f, 0.f);
    gQ = make_float3(0.f, 0.f, 0.f);
    float best = 1.0e30f;
    bool found = false, from1 = false;
    float sigma = 1.f;
    float2 bn = make_float2(0.f, 0.f), bv = bn, bw = bn;
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const bool tri = pass == 0 ? p_tri : q_tri;
            if (k == 3 && tri) continue;
            const float2 a = pass == 0 ? P[k] : Q[k];
            const float2 b = pass == 0 ? P[(k + 1) & 3] : Q[(k + 1) & 3];
            float2 nr = make_float2(-(b.y - a.y), b.x - a.x);
            const float len = sqrtf(nr.x * nr.x + nr.y * nr.y);
            if (len < 1.0e-12f) continue;
            nr.x /= len;
            nr.y /= len;
            float p1[4], p2[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                p1[v] = P[v].x * nr.x + P[v].y * nr.y;
                p2[v] = Q[v].x * nr.x + Q[v].y * nr.y;
            }
            float mn1 = p1[0], mx1 = p1[0], mn2 = p2[0], mx2 = p2[0];
#pragma unroll
            for (int v = 1; v < 4; ++v) {
                mn1 = fminf(mn1, p1[v]); mx1 = fmaxf(mx1, p1[v]);
                mn2 = fminf(mn2, p2[v]); mx2 = fmaxf(mx2, p2[v]);
            }
            if (mx1 < mn2 || mx2 < mn1) return;   // separating axis: no overlap
            found = true;
            const float pen1 = mx1 - mn2, pen2 = mx2 - mn1;
            const float pen = pen1 < pen2 ? pen1 : pen2;
            if (pen < best) {
                best = pen;
                bn = nr;
                from1 = pass == 0;
                const bool c1 = pen1 <= pen2;
                sigma = c1 ? 1.f : -1.f;
                // first vertex attaining the extreme, like the reference scans
                float2 v = P[0], w = Q[0];
                float pv = p1[0], pw = p2[0];
#pragma unroll
                for (int q = 1; q < 4; ++q) {
                    if (c1 ? (p1[q] > pv) : (p1[q] < pv)) { pv = p1[q]; v = P[q]; }
                    if (c1 ? (p2[q] < pw) : (p2[q] > pw)) { pw = p2[q]; w = Q[q]; }
                }
                bv = v;
                bw = w;
            }
        }
    }
    if (!found || best <= 1.0e-12f) return;
    sep = best;
    const float2 gv = make_float2(sigma * bn.x, sigma * bn.y);
    const float2 rn = make_float2(-bn.y, bn.x);                     // d n / d theta
    const float2 vw = make_float2(bv.x - bw.x, bv.y - bw.y);
    const float axis_term = sigma * (vw.x * rn.x + vw.y * rn.y);
    const float2 rq = make_float2(bw.x - d.x, bw.y - d.y);
    gP.x = gv.x;
    gP.y = gv.y;
    gP.z = gv.x * -bv.y + gv.y * bv.x + (from1 ? axis_term : 0.f);
    gQ.x = -gv.x;
    gQ.y = -gv.y;
    gQ.z = -(gv.x * -rq.y + gv.y * rq.x) + (from1 ? 0.f : axis_term);
}

// ---------------------------------------------------------------------------
// LUT lookup with analytic gradient (lut_lookup_with_grad,
// pack_cuda_lut.py:298-415), FP32 with the reference's operation order.
// Indices are clamped into the table (the reference can read one cell out of
// range when a trimmed theta range is mirrored).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float pk_lut_lookup(const PkLut& L, float x, float y, float th, float3& g)
{
    g = make_float3(0.f, 0.f, 0.f);
    if (x < -L.x_max || x > L.x_max || y < L.y_min || y > L.y_max || th < L.t_min || th > L.t_max)
        return 0.f;
    const float xt = x >= 0.f ? x : -x;
    const float tt = x >= 0.f ? th : -th;
    const float gx = (xt - L.x_min) / (L.x_max - L.x_min) * (float)(L.nx - 1);
    const float gy = (y - L.y_min) / (L.y_max - L.y_min) * (float)(L.ny - 1);
    const float gt = (tt - L.t_min) / (L.t_max - L.t_min) * (float)(L.nt - 1);
    int ix0 = (int)floorf(gx), iy0 = (int)floorf(gy), it0 = (int)floorf(gt);
    const float fx = gx - ix0, fy = gy - iy0, ft = gt - it0;
    ix0 = min(max(ix0, 0), L.nx - 1);
    iy0 = min(max(iy0, 0), L.ny - 1);
    it0 = min(max(it0, 0), L.nt - 1);
    const int ix1 = min(ix0 + 1, L.nx - 1), iy1 = min(iy0 + 1, L.ny - 1), it1 = min(it0 + 1, L.nt - 1);
    const size_t sy = (size_t)L.nt, sx = (size_t)L.ny * L.nt;
    const float* V = L.vals;
    const float v000 = __ldg(V + ix0 * sx + iy0 * sy + it0), v001 = __ldg(V + ix0 * sx + iy0 * sy + it1);
    const float v010 = __ldg(V + ix0 * sx + iy1 * sy + it0), v011 = __ldg(V + ix0 * sx + iy1 * sy + it1);
    const float v100 = __ldg(V + ix1 * sx + iy0 * sy + it0), v101 = __ldg(V + ix1 * sx + iy0 * sy + it1);
    const float v110 = __ldg(V + ix1 * sx + iy1 * sy + it0), v111 = __ldg(V + ix1 * sx + iy1 * sy + it1);
    const float v00 = v000 * (1.0f - ft) + v001 * ft, v01 = v010 * (1.0f - ft) + v011 * ft;
    const float v10 = v100 * (1.0f - ft) + v101 * ft, v11 = v110 * (1.0f - ft) + v111 * ft;
    const float v0 = v00 * (1.0f - fy) + v01 * fy, v1 = v10 * (1.0f - fy) + v11 * fy;
    const float val = v0 * (1.0f - fx) + v1 * fx;
    const float dfx = v1 - v0;
    const float dfy = (1.0f - fx) * (v01 - v00) + fx * (v11 - v10);
    const float d0 = (v001 - v000) * (1.0f - fy) + (v011 - v010) * fy;
    const float d1 = (v101 - v100) * (1.0f - fy) + (v111 - v110) * fy;
    const float dft = d0 * (1.0f - fx) + d1 * fx;
    g.x = dfx * ((float)(L.nx - 1) / (L.x_max - L.x_min));
    g.y = dfy * ((float)(L.ny - 1) / (L.y_max - L.y_min));
    g.z = dft * ((float)(L.nt - 1) / (L.t_max - L.t_min));
    if (x < 0.f) { g.x = -g.x; g.z = -g.z; }
    return val;
}

// Adds v to the int64 at a (shared memory) with two 32-bit atomics: the low
// word's old value gives the carry, which travels with the high word.  The
// sum stays exact modulo 2^64 whatever the interleaving (the carries total
// floor((lo0 + sum lo_k) / 2^32) in any order), and a high-word add of zero
// -- small values of either sign -- is skipped.  On this GPU a 64-bit
// shared atomic costs several times two 32-bit ones.
__device__ __forceinline__ void pk_fx_add(long long* a, long long v)
{
    unsigned* w = (unsigned*)a;   // little endian: w[0] low word, w[1] high word
    const unsigned lo = (unsigned)v, hi = (unsigned)((unsigned long long)v >> 32);
    const unsigned old = atomicAdd(&w[0], lo);
    const unsigned up = hi + (unsigned)(old + lo < old);
    if (up) atomicAdd(&w[1], up);
}

// The same add on a split accumulator: low words in one array, high words
// in another, so consecutive accumulators use consecutive banks.
__device__ __forceinline__ void pk_fx_add2(unsigned* lo_w, unsigned* hi_w, long long v)
{
    const unsigned lo = (unsigned)v, hi = (unsigned)((unsigned long long)v >> 32);
    const unsigned old = atomicAdd(lo_w, lo);
    const unsigned up = hi + (unsigned)(old + lo < old);
    if (up) atomicAdd(hi_w, up);
}

__device__ __forceinline__ void pk_acc_add2(const PkCostSmem& sm, int t, float3 g)
{
    pk_fx_add2(&sm.acc_lo[3 * t + 0], &sm.acc_hi[3 * t + 0], pk_to_fx(g.x));
    pk_fx_add2(&sm.acc_lo[3 * t + 1], &sm.acc_hi[3 * t + 1], pk_to_fx(g.y));
    pk_fx_add2(&sm.acc_lo[3 * t + 2], &sm.acc_hi[3 * t + 2], pk_to_fx(g.z));
}

__device__ __forceinline__ long long pk_acc_get(const PkCostSmem& sm, int k)
{
    return (long long)(((unsigned long long)sm.acc_hi[k] << 32) | (unsigned long long)sm.acc_lo[k]);
}

__device__ __forceinline__ void pk_acc_add(long long* acc, int t, float3 g)
{
    pk_fx_add(&acc[3 * t + 0], pk_to_fx(g.x));
    pk_fx_add(&acc[3 * t + 1], pk_to_fx(g.y));
    pk_fx_add(&acc[3 * t + 2], pk_to_fx(g.z));
}

__device__ __forceinline__ void pk_load_piece(const PkCostSmem& sm, int p, float c, float s, float ox,
                                              float oy, float2 (&V)[4])
{
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float2 l = sm.piece[p * 4 + v];
        V[v] = make_float2(c * l.x - s * l.y + ox, s * l.x + c * l.y + oy);
    }
}

// Piece p of a tree rotated by (c, s) and moved by (ox, oy), from the SoA
// table: two vertices per instruction.
__device__ __forceinline__ PkQuad pk_load_quad(const PkCostSmem& sm, int p, float c, float s, float ox, float oy)
{
    const float4 X = sm.piece4[2 * p], Y = sm.piece4[2 * p + 1];
    const float2 c2 = make_float2(c, c), s2 = make_float2(s, s), ns2 = make_float2(-s, -s);
    const float2 ox2 = make_float2(ox, ox), oy2 = make_float2(oy, oy);
    const float2 x01 = make_float2(X.x, X.y), x23 = make_float2(X.z, X.w);
    const float2 y01 = make_float2(Y.x, Y.y), y23 = make_float2(Y.z, Y.w);
    PkQuad q;
    q.x01 = __fadd2_rn(__ffma2_rn(c2, x01, __fmul2_rn(ns2, y01)), ox2);
    q.x23 = __fadd2_rn(__ffma2_rn(c2, x23, __fmul2_rn(ns2, y23)), ox2);
    q.y01 = __fadd2_rn(__ffma2_rn(s2, x01, __fmul2_rn(c2, y01)), oy2);
    q.y23 = __fadd2_rn(__ffma2_rn(s2, x23, __fmul2_rn(c2, y23)), oy2);
    return q;
}

// Centre-distance cull, rounded the same way wherever it is evaluated.  Swapping A and B
// gives the same answer: rounding is symmetric under negation.
__device__ __forceinline__ int pk_is_near(float4 A, float4 B, float cutoff)
{
    const float dx = __fsub_rn(B.x, A.x), dy = __fsub_rn(B.y, A.y);
    return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) <= cutoff;
}

// Phase B: evaluate every listed item; returns this thread's fixed-point
// pair total.  Items: i (11 bits) | j (11 bits) | pi (2) | pj (2).
// filter (LUT only): the list is a kept near list, so a pair is looked up only
// if it passes the centre cull now; the kept pairs are counted.
template <int MODE>
__device__ __forceinline__ long long pk_process_items(const PkCostSmem& sm, const uint32_t* list, int count,
                                                      float w_pair, const PkLut& lut, bool filter = false,
                                                      float cutoff = 0.f)
{
    long long tot = 0;
    unsigned kept = 0;
    const int nwarps = blockDim.x >> 5;
    for (int base = 0; base < count; base += blockDim.x) {
        // Analytic modes, full rounds: a warp's lanes take items nwarps apart.
        // Consecutive items share trees (a near pair's piece pairs, a tree's
        // near pairs), and spread over warps their accumulator atomics stop
        // hitting the same addresses within a warp (1 % at 4096 x n = 200;
        // the same bits).  The LUT's lookups keep the contiguous order.
        const int w = MODE != PK_PAIR_LUT && base + (int)blockDim.x <= count
                          ? base + (int)(threadIdx.x & 31) * nwarps + (int)(threadIdx.x >> 5)
                          : base + (int)threadIdx.x;
        if (w >= count) continue;
        const uint32_t it = list[w];
        const int i = it & 2047, j = (it >> 11) & 2047;
        const float4 A = sm.pose[i], B = sm.pose[j];
        if (MODE == PK_PAIR_LUT && filter) {
            if (!pk_is_near(A, B, cutoff)) continue;
            ++kept;
        }
        const float2 d = make_float2(B.x - A.x, B.y - A.y);
        float val;
        float3 gi, gj;
        if (MODE == PK_PAIR_LUT) {
            // ref = lower index, as the reference's triangular loop (pack_cuda_lut.py:437)
            const int r = i < j ? i : j, o = i < j ? j : i;
            const float4 R = sm.pose[r], O = sm.pose[o];
            const float dxw = O.x - R.x, dyw = O.y - R.y;
            const float dxl = R.z * dxw + R.w * dyw;
            const float dyl = -R.w * dxw + R.z * dyw;
            const float dth = pk_wrap_angle(sm.theta[o] - sm.theta[r]);
            float3 gl;
            val = pk_lut_lookup(lut, dxl, dyl, dth, gl);
            if (lut.quadratic) {
                if (val > 0.f) {
                    gl.x *= 2.0f * val; gl.y *= 2.0f * val; gl.z *= 2.0f * val;
                    val = val * val;
                } else {
                    val = 0.f;
                    gl = make_float3(0.f, 0.f, 0.f);
                }
            }
            float3 gr = make_float3(-gl.x * R.z + gl.y * R.w, -gl.x * R.w - gl.y * R.z,
                                    gl.x * dyl - gl.y * dxl - gl.z);
            float3 go = make_float3(gl.x * R.z - gl.y * R.w, gl.x * R.w + gl.y * R.z, gl.z);
            gi = (r == i) ? gr : go;
            gj = (r == i) ? go : gr;
        } else {
            const int pi = (it >> 22) & 3, pj = (it >> 24) & 3;
            const bool pt = sm.piece_nv[pi] == 3, qt = sm.piece_nv[pj] == 3;
            if (MODE == PK_PAIR_AREA) {
                const PkQuad PQ = pk_load_quad(sm, pi, A.z, A.w, 0.f, 0.f);
                const PkQuad QQ = pk_load_quad(sm, pj, B.z, B.w, d.x, d.y);
                pk_piece_area_grad_q(PQ, pt, QQ, qt, d, val, gi, gj);
            } else {
                float2 P[4], Q[4];
                pk_load_piece(sm, pi, A.z, A.w, 0.f, 0.f, P);
                pk_load_piece(sm, pj, B.z, B.w, d.x, d.y, Q);
                float sp;
                pk_piece_sat_grad(P, pt, Q, qt, d, sp, gi, gj);
                const float f = 2.0f * sp;
                gi = make_float3(f * gi.x, f * gi.y, f * gi.z);
                gj = make_float3(f * gj.x, f * gj.y, f * gj.z);
                val = sp * sp;
            }
        }
        if (val != 0.f || gi.x != 0.f || gi.y != 0.f || gi.z != 0.f) {
            tot += pk_to_fx(w_pair * val);
            pk_acc_add2(sm, i, make_float3(w_pair * gi.x, w_pair * gi.y, w_pair * gi.z));
            pk_acc_add2(sm, j, make_float3(w_pair * gj.x, w_pair * gj.y, w_pair * gj.z));
        }
    }
    if (MODE == PK_PAIR_LUT && filter) {
        kept = __reduce_add_sync(PK_FULL_MASK, kept);
        if ((threadIdx.x & 31) == 0 && kept) { atomicAdd(&sm.cnt[1], kept); atomicAdd(&sm.cnt[2], kept); }
    }
    return tot;
}

// Sorted-position ranges [b0, b1) and [b2, b3) of the half neighbourhood of
// sorted position a (grid of gx x gy cells, row-major cell order).
__device__ __forceinline__ void pk_half_neighbourhood(const PkCostSmem& sm, int a, int gx, int gy, int& b0, int& b1,
                                                      int& b2, int& b3)
{
    const int c = sm.tcell[sm.sorted[a]];
    const int cy = c / gx, cx = c - cy * gx;
    b0 = a + 1;
    b1 = sm.cell_start[cy * gx + min(cx + 2, gx)];
    if (cy + 1 < gy) {
        const int r = (cy + 1) * gx;
        b2 = sm.cell_start[r + max(cx - 1, 0)];
        b3 = sm.cell_start[r + min(cx + 2, gx)];
    } else {
        b2 = b3 = b1;
    }
}

// Processes the cn near pairs of the list: the LUT looks them up directly;
// the analytic modes expand each into the piece pairs whose boxes overlap and
// evaluate those in chunks.  With KEEP the list may be a kept near list
// (pk_nlist(sm)[2] set), whose pairs were within cutoff + skin when it was
// built: each pair is then first tested against the centre cutoff at the
// current poses, and the pairs that pass are counted.  The flag is read where
// it is used, so nothing extra stays live across the clipper.  Otherwise every
// listed pair is near.  All threads call it; it ends with a barrier.
template <int MODE, bool KEEP>
__device__ __forceinline__ long long pk_flush_near(const PkCostSmem& sm, int cn, const PkCostSpec& spec, int T)
{
    long long tot = 0;
    const int lane = threadIdx.x & 31;
    if (MODE == PK_PAIR_LUT) {
        const bool filter = KEEP && pk_nlist(sm)[2] != 0;
        if (threadIdx.x == 0 && !filter) sm.cnt[2] += (unsigned)cn;
        tot += pk_process_items<MODE>(sm, sm.near, cn, spec.w_pair, spec.lut, filter, c_geom.cutoff_sq);
    } else {
        for (int c0 = 0; c0 < cn; c0 += T) {
            const int w = c0 + threadIdx.x;
            const bool filter = KEEP && pk_nlist(sm)[2] != 0;
            uint32_t mask = 0, ij = 0;
            bool keep = false;
            float4 A, B;
            if (w < cn) {
                ij = sm.near[w];
                A = sm.pose[ij & 2047];
                B = sm.pose[(ij >> 11) & 2047];
                keep = !filter || pk_is_near(A, B, c_geom.cutoff_sq);
            }
            if (filter) {
                const unsigned kb = __ballot_sync(PK_FULL_MASK, keep);
                if (lane == 0 && kb) atomicAdd(&sm.cnt[1], (unsigned)__popc(kb));
            }
            if (keep) {
                const int i = ij & 2047, j = (ij >> 11) & 2047;
                const float dx = B.x - A.x, dy = B.y - A.y;
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const float4 a = sm.aabb[p * sm.n_cap + i];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 b = sm.aabb[q * sm.n_cap + j];
                        const bool ov = !(a.y < b.x + dx || b.y + dx < a.x || a.w < b.z + dy || b.w + dy < a.z);
                        mask |= (uint32_t)ov << (4 * p + q);
                    }
                }
            }
            const int cnt = __popc(mask);
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(PK_FULL_MASK, incl, o);
                if (lane >= o) incl += v;
            }
            const int wtot = __shfl_sync(PK_FULL_MASK, incl, 31);
            int wbase = 0;
            if (lane == 31 && wtot) {
                wbase = atomicAdd(sm.count, wtot);
                atomicAdd(&sm.cnt[2], (unsigned)wtot);
            }
            wbase = __shfl_sync(PK_FULL_MASK, wbase, 31);
            int pos = wbase + incl - cnt;
            while (mask) {
                const int b = __ffs(mask) - 1;
                mask &= mask - 1;
                sm.items[pos++] = ij | ((uint32_t)(b >> 2) << 22) | ((uint32_t)(b & 3) << 24);
            }
            __syncthreads();
            const int ci = *sm.count;
            __syncthreads();
            if (ci > sm.cap_items - 16 * T || c0 + T >= cn) {
                tot += pk_process_items<MODE>(sm, sm.items, ci, spec.w_pair, spec.lut);
                __syncthreads();
                if (threadIdx.x == 0) *sm.count = 0;
                __syncthreads();
            }
        }
    }
    __syncthreads();
    return tot;
}

// Sums of the four components of bnd[0..n) in an order fixed by n alone
// (not by blockDim): lane l of warp 0 adds its contiguous chunk in double,
// then a fixed shuffle tree.  Called by warp 0 only; lane 0 gets the sums.
__device__ __forceinline__ double4 pk_canonical_sum4(int n, const float4* bnd)
{
    double4 s = make_double4(0.0, 0.0, 0.0, 0.0);
    const int k = (n + 31) >> 5;
    const int b = threadIdx.x * k, e = min(n, b + k);
    for (int t = b; t < e; ++t) {
        const float4 v = bnd[t];
        s.x += (double)v.x; s.y += (double)v.y; s.z += (double)v.z; s.w += (double)v.w;
    }
    s.x = pk_warp_sum(s.x); s.y = pk_warp_sum(s.y); s.z = pk_warp_sum(s.z); s.w = pk_warp_sum(s.w);
    return s;
}

// Images per genotype tree of a symmetric packing (spec.symmetry): 1, 2
// (SolutionCollectionSquareSymmetric180, kaggle_support.py:1272-1393) or 4
// (SolutionCollectionSquareSymmetric90, :1039-1195).
__host__ __device__ inline int pk_symmetry(const PkCostSpec& spec) { return spec.symmetry > 1 ? spec.symmetry : 1; }

// Pose of phenotype tree t = k ng + g: image k of genotype tree g, as the
// reference expands it in float32 (the angle offsets are pi / 2, pi and
// 3 pi / 2 rounded to float32 before the add):
//   180: (x, y, th), (-x, -y, th + pi)
//   90:  (x, y, th), (-y, x, th + pi/2), (-x, -y, th + pi), (y, -x, th + 3pi/2)
__device__ __forceinline__ void pk_image_pose(const float* X, int ng, int sym, int t, float& x, float& y, float& th)
{
    const int k = sym == 1 ? 0 : t / ng, g = t - k * ng;
    const float gx = X[3 * g], gy = X[3 * g + 1], gt = X[3 * g + 2];
    const float hpi = (float)(3.14159265358979323846 / 2.0), pi = (float)3.14159265358979323846,
                tpi = (float)(3.0 * 3.14159265358979323846 / 2.0);
    if (k == 0) { x = gx; y = gy; th = gt; }
    else if (sym == 2 || k == 2) { x = -gx; y = -gy; th = gt + pi; }
    else if (k == 1) { x = -gy; y = gx; th = gt + hpi; }
    else { x = gy; y = -gx; th = gt + tpi; }
}

struct PkEvalOut {
    double cost;
};

// Skin of the kept near lists (below), as a fraction of the cutoff distance.
// 0.22 relaxed 4096 x n = 200 (max_step 0.01) fastest of 0.12, 0.17, 0.22, 0.26.
#define PK_NEAR_SKIN 0.22f   // skin / cutoff distance

__device__ __forceinline__ float pk_near_skin() { return PK_NEAR_SKIN * sqrtf(c_geom.cutoff_sq); }

// Broad phase on a uniform grid of cells at least the interaction distance
// wide: tree i only meets trees of the 3 x 3 cells around its own, and each
// pair is found once, from its lower index.  Builds the grid (sm.cell_start,
// sm.sorted, sm.tcell), counts each sorted position's near pairs (pass 1)
// and scans the counts into sm.near_start; returns the grid's (gx, gy).
// build: take pairs within cutoff + skin for a kept list, falling back to the
// cutoff (and to no kept lists from then on) when they do not fit the near
// list in one piece.  Leaves pk_nlist(sm)[2] (list kept) and [3] (the
// distance pass 2 must use) for the caller, visible after its barriers.
// KEEP: the caller keeps near lists (the flags above); without it build is
// false and nothing is left in pk_nlist.  All threads call it.
template <bool KEEP>
__device__ __forceinline__ int2 pk_broad_phase(const PkCostSmem& sm, int n, bool build)
{
    const int T = blockDim.x;
    const float cutoff = c_geom.cutoff_sq;
    float cut_list = cutoff;
    if (build) {
        const float r = sqrtf(cutoff) + pk_near_skin();
        cut_list = r * r;
    }
    int gx = 1, gy = 1;
    float4 bb = make_float4(-3.4e38f, -3.4e38f, -3.4e38f, -3.4e38f);   // (-min x, max x, -min y, max y)
    for (int t = threadIdx.x; t < n; t += T) {
        const float4 A = sm.pose[t];
        bb.x = fmaxf(bb.x, -A.x); bb.y = fmaxf(bb.y, A.x);
        bb.z = fmaxf(bb.z, -A.y); bb.w = fmaxf(bb.w, A.y);
    }
    bb = pk_block_max4(bb, (float*)sm.red);
    const float x0 = -bb.x, y0 = -bb.z;
    const float wx = fmaxf(bb.y - x0, 0.f), wy = fmaxf(bb.w - y0, 0.f);
    // 1 % wider than the interaction distance, so rounding in the cell
    // index never puts two interacting trees two cells apart
    float cs = sqrtf(cut_list) * 1.01f;
    for (int tries = 0; tries < 64; ++tries) {
        gx = (int)fminf(wx / cs, 2048.f) + 1;
        gy = (int)fminf(wy / cs, 2048.f) + 1;
        if (gx * gy <= sm.grid_cap) break;
        cs *= 1.25f;
    }
    if (gx * gy > sm.grid_cap) { gx = 1; gy = 1; cs = 3.4e38f; }   // non-finite extent: one cell
    const float inv = 1.0f / cs;
    const int ncell = gx * gy;
    for (int c = threadIdx.x; c < ncell; c += T) sm.cell_fill[c] = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += T) {
        const float4 A = sm.pose[t];
        const int cx = min(gx - 1, max(0, (int)((A.x - x0) * inv)));
        const int cy = min(gy - 1, max(0, (int)((A.y - y0) * inv)));
        const int c = cy * gx + cx;
        sm.tcell[t] = c;
        atomicAdd(&sm.cell_fill[c], 1);
    }
    __syncthreads();
    pk_block_exclusive_scan(sm.cell_fill, sm.cell_start, ncell, (int*)sm.redl);
    for (int c = threadIdx.x; c < ncell; c += T) sm.cell_fill[c] = sm.cell_start[c];
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += T) sm.sorted[atomicAdd(&sm.cell_fill[sm.tcell[t]], 1)] = t;
    __syncthreads();

    // Half neighbourhood of sorted position a in cell (cx, cy): the rest
    // of its own cell and the cell to its right (one contiguous range of
    // the sorted order), and cells cx-1..cx+1 of the row above (another).
    // Every pair of trees in touching cells is found exactly once.
    // Pass 1 counts the near pairs of each position, a scan turns the
    // counts into list offsets, and pass 2 writes them in chunks that fit
    // the near list, each chunk flushed before the next is written.
    unsigned tested = 0;
    for (int pass = 0; pass < 2; ++pass) {
        for (int a = threadIdx.x; a < n; a += T) {
            int b0, b1, b2, b3;
            pk_half_neighbourhood(sm, a, gx, gy, b0, b1, b2, b3);
            tested += (unsigned)(b1 - b0 + b3 - b2);
            const float4 A = sm.pose[sm.sorted[a]];
            int k = 0;
            for (int b = b0; b < b1; ++b) k += pk_is_near(A, sm.pose[sm.sorted[b]], cut_list);
            for (int b = b2; b < b3; ++b) k += pk_is_near(A, sm.pose[sm.sorted[b]], cut_list);
            sm.near_cnt[a] = k;
        }
        if (KEEP && threadIdx.x == 0) {
            // read by pass 2 and by the flush (after the scan's barriers)
            pk_nlist(sm)[2] = build;
            ((float*)pk_nlist(sm))[3] = cut_list;
        }
        __syncthreads();
        pk_block_exclusive_scan(sm.near_cnt, sm.near_start, n, (int*)sm.redl);
        // a kept list must fit the near list in one piece; when it does
        // not, count again at the cutoff and keep no lists from now on
        if (!KEEP || !build || sm.near_start[n] <= sm.cap_near) break;
        build = false;
        cut_list = cutoff;
        if (threadIdx.x == 0) pk_nlist(sm)[0] = -1;
    }
    atomicAdd(&sm.cnt[0], tested);
    return make_int2(gx, gy);
}

// The fused relaxation calls the broad phase and pass 2 out of line: with
// kept lists they run once per several evaluations, and their code then stays
// out of the hot loop's way.  A one-shot cost evaluation inlines them.  The
// out-of-line forms take the carve's sizes, not the caller's PkCostSmem (whose
// address would pin it to local memory), and carve the dynamic shared memory
// again: every kernel that evaluates costs places the cost arrays at its base.
__device__ __noinline__ int2 pk_broad_phase_outlined(int n_cap, int cap_near, int cap_items, int n, bool build)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const PkCostSmem sm = pk_cost_carve(pk_smem, n_cap, cap_near, cap_items, true);
    return pk_broad_phase<true>(sm, n, build);
}

// Pass 2: writes the near pairs of the longest run of sorted positions from
// a0 whose pairs fit the near list into sm.near, and keeps the list when
// pk_broad_phase built a kept one (the run is then every position).  Returns
// (end of the run, pairs written).  All threads call it; the pairs are
// written (behind a barrier) when it returns.
template <bool KEEP>
__device__ __forceinline__ int2 pk_write_near(const PkCostSmem& sm, int n, int a0, int gx, int gy)
{
    const int T = blockDim.x;
    // the longest run of positions from a0 whose pairs fit the list
    // (a single position's pairs always do: cap_near >= n_max)
    int lo = a0 + 1, hi = n;
    const int lim = sm.near_start[a0] + sm.cap_near;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sm.near_start[mid] <= lim) lo = mid; else hi = mid - 1;
    }
    const int a1 = lo, base = sm.near_start[a0];
    const int cn = sm.near_start[a1] - base;
    const float cut2 = KEEP ? ((const float*)pk_nlist(sm))[3] : c_geom.cutoff_sq;   // pass 1's distance
    for (int a = a0 + threadIdx.x; a < a1; a += T) {
        int b0, b1, b2, b3;
        pk_half_neighbourhood(sm, a, gx, gy, b0, b1, b2, b3);
        const int ia = sm.sorted[a];
        const float4 A = sm.pose[ia];
        uint32_t* out = sm.near + (sm.near_start[a] - base);
        const int kmax = sm.near_cnt[a];
        int k = 0;
        for (int b = b0; b < b3 && k < kmax; ++b) {
            if (b == b1) { b = b2; if (b >= b3) break; }
            const int ib = sm.sorted[b];
            if (pk_is_near(A, sm.pose[ib], cut2))
                out[k++] = (uint32_t)min(ia, ib) | ((uint32_t)max(ia, ib) << 11);
        }
    }
    __syncthreads();
    if (KEEP && pk_nlist(sm)[2]) {
        // the whole list is this one chunk: keep it, with the
        // positions it was built at in the grid's arrays (dead from here)
        for (int t = threadIdx.x; t < n; t += T) {
            const float4 A = sm.pose[t];
            ((float*)sm.sorted)[t] = A.x;
            ((float*)sm.tcell)[t] = A.y;
        }
        if (threadIdx.x == 0) { pk_nlist(sm)[0] = 1; pk_nlist(sm)[1] = cn; }
    } else if (threadIdx.x == 0) {
        sm.cnt[1] += (unsigned)cn;
    }
    return make_int2(a1, cn);
}

__device__ __noinline__ int2 pk_write_near_outlined(int n_cap, int cap_near, int cap_items, int n, int a0, int gx,
                                                   int gy)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const PkCostSmem sm = pk_cost_carve(pk_smem, n_cap, cap_near, cap_items, true);
    return pk_write_near<true>(sm, n, a0, gx, gy);
}

// The piece table in shared memory (SoA and AoS), from constant memory.
__device__ __forceinline__ void pk_load_piece_table(const PkCostSmem& sm)
{
    if (threadIdx.x < 16) {
        const float2 v = c_geom.piece[threadIdx.x >> 2][threadIdx.x & 3];
        sm.piece[threadIdx.x] = v;
        float* soa = (float*)sm.piece4;   // piece p: x at [8p + v], y at [8p + 4 + v]
        soa[8 * (threadIdx.x >> 2) + (threadIdx.x & 3)] = v.x;
        soa[8 * (threadIdx.x >> 2) + 4 + (threadIdx.x & 3)] = v.y;
    }
    if (threadIdx.x < 4) sm.piece_nv[threadIdx.x] = c_geom.piece_nv[threadIdx.x];
}

// Evaluate one instance.  X: 3n floats (global or shared), H: 3 floats or
// NULL.  G: 3n floats or NULL (written, not accumulated); GH: 3 floats or
// NULL.  Must be called by every thread of the block.
// SYM: the packing may be symmetric (spec.symmetry > 1); the plain
// instantiation keeps no symmetry state in registers.
// Kept near lists (KEEP, the fused relaxation only).  The list built by
// one evaluation holds every pair within cutoff + skin; a later evaluation
// reuses it, without building the cell grid, while no tree has moved by
// more than skin / (2 sqrt 2) per coordinate since, re-applying the exact
// centre cull to each listed pair.  Any pair near now was then within
// cutoff + skin, so the pairs evaluated are the same as a fresh grid's, and
// the fixed-point sums make the result independent of their order.
template <int MODE, bool SYM, bool KEEP = false>
__device__ double pk_eval_instance(const float* X, int ng, const float* H, const PkCostSpec& spec,
                                   float* G, float* GH, const PkCostSmem& sm)
{
    // ng genotype trees in X (3 ng floats); the cost is that of the n
    // phenotype trees, and G receives the genotype gradient
    const int sym = SYM ? pk_symmetry(spec) : 1;
    const int n = sym * ng;
    const int T = blockDim.x;
    const bool do_bnd = spec.w_boundary != 0.f && H != nullptr;
    float half = 0.f, hox = 0.f, hoy = 0.f;
    if (H) { half = H[0] * 0.5f; hox = H[1]; hoy = H[2]; }
    // piece table into shared memory first: phase 0 reads it (the fused
    // relaxation loads it once, before its first evaluation)
    if (!KEEP) {
        pk_load_piece_table(sm);
    }
    // kept list state, written by the last evaluation that built the grid
    const int nstate = KEEP ? pk_nlist(sm)[0] : -1;
    float disp = 0.f;   // largest coordinate change of this thread's trees since the list was built
    if (!KEEP) __syncthreads();
    // ---- phase 0: per tree -------------------------------------------------
    for (int t = threadIdx.x; t < n; t += T) {
        float x, y, th;
        pk_image_pose(X, ng, sym, t, x, y, th);
        if (nstate == 1) {
            // positions when the list was built, kept in the grid's dead arrays
            const float dm = fmaxf(fabsf(__fsub_rn(x, ((const float*)sm.sorted)[t])),
                                   fabsf(__fsub_rn(y, ((const float*)sm.tcell)[t])));
            disp = dm <= 1e30f ? fmaxf(disp, dm) : 3.4e38f;   // NaN or infinite: rebuild
        }
        float s, c;
        sincosf(th, &s, &c);
        sm.pose[t] = make_float4(x, y, c, s);
        sm.theta[t] = th;
        long long a0 = 0, a1 = 0, a2 = 0;
        float4 bnd = make_float4(0.f, 0.f, 0.f, 0.f);
        if (MODE == PK_PAIR_AREA || MODE == PK_PAIR_SEP) {
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                float2 V[4];
                pk_load_piece(sm, p, c, s, 0.f, 0.f, V);
                float4 bb = make_float4(V[0].x, V[0].x, V[0].y, V[0].y);
#pragma unroll
                for (int v = 1; v < 4; ++v) {
                    bb.x = fminf(bb.x, V[v].x); bb.y = fmaxf(bb.y, V[v].x);
                    bb.z = fminf(bb.z, V[v].y); bb.w = fmaxf(bb.w, V[v].y);
                }
                const float eps = 1e-6f;
                sm.aabb[p * sm.n_cap + t] = make_float4(bb.x - eps, bb.y + eps, bb.z - eps, bb.w + eps);
            }
        }
        if (do_bnd) {
            // boundary_distance_tree, pack_cuda.py:550-642
            float best = 0.f;
            int bi = 0;
            for (int v = 0; v < c_geom.n_tree; ++v) {
                const float2 l = c_geom.tree[v];
                const float vx = c * l.x - s * l.y + x - hox;
                const float vy = s * l.x + c * l.y + y - hoy;
                const float ax = fabsf(vx), ay = fabsf(vy);
                const float dx = ax > half ? ax - half : 0.f;
                const float dy = ay > half ? ay - half : 0.f;
                const float dd = dx * dx + dy * dy;
                if (dd > best) { best = dd; bi = v; }
            }
            const float2 l = c_geom.tree[bi];
            const float vx = c * l.x - s * l.y + x - hox;
            const float vy = s * l.x + c * l.y + y - hoy;
            const float ax = fabsf(vx), ay = fabsf(vy);
            const float dx = ax > half ? ax - half : 0.f;
            const float dy = ay > half ? ay - half : 0.f;
            const float gvx = dx > 0.f ? 2.0f * dx * (vx >= 0.f ? 1.f : -1.f) : 0.f;
            const float gvy = dy > 0.f ? 2.0f * dy * (vy >= 0.f ? 1.f : -1.f) : 0.f;
            const float gth = gvx * (-s * l.x - c * l.y) + gvy * (c * l.x - s * l.y);
            const float wb = spec.w_boundary;
            a0 = pk_to_fx(wb * gvx);
            a1 = pk_to_fx(wb * gvy);
            a2 = pk_to_fx(wb * gth);
            bnd = make_float4(best, -(dx + dy), -gvx, -gvy);
        }
        sm.acc_lo[3 * t] = (unsigned)a0;
        sm.acc_hi[3 * t] = (unsigned)((unsigned long long)a0 >> 32);
        sm.acc_lo[3 * t + 1] = (unsigned)a1;
        sm.acc_hi[3 * t + 1] = (unsigned)((unsigned long long)a1 >> 32);
        sm.acc_lo[3 * t + 2] = (unsigned)a2;
        sm.acc_hi[3 * t + 2] = (unsigned)((unsigned long long)a2 >> 32);
        sm.bnd[t] = bnd;
    }
    if (threadIdx.x == 0) {
        *sm.count = 0;
        sm.cnt[3] += 1;
    }
    if (nstate == 1) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) disp = fmaxf(disp, __shfl_xor_sync(PK_FULL_MASK, disp, o));
        if ((threadIdx.x & 31) == 0) pk_disp(sm)[threadIdx.x >> 5] = disp;
    }
    __syncthreads();
    bool reuse = false;
    if (nstate == 1) {
        float dm = 0.f;
        for (int w = 0; w < (T >> 5); ++w) dm = fmaxf(dm, pk_disp(sm)[w]);
        // a pair's distance moved by at most 2 sqrt 2 dm; 1e-4 covers the rounding
        reuse = 2.8285f * dm + 1e-4f < pk_near_skin();
    }

    // ---- phases A + B: pairs -------------------------------------------------
    long long pair_tot = 0;
    if (MODE != PK_PAIR_NONE && n > 1) {
        int gx = 1, gy = 1;
        int a0 = reuse ? -1 : 0;   // -1: flush the kept list
        if (!reuse) {
            // without a kept list to reuse, build one this time (nstate >= 0)
            const int2 g = KEEP ? pk_broad_phase_outlined(sm.n_cap, sm.cap_near, sm.cap_items, n, nstate >= 0)
                                : pk_broad_phase<false>(sm, n, false);
            gx = g.x;
            gy = g.y;
        }
        while (a0 < n) {
            int cn;
            if (a0 < 0) {
                // the kept list (pk_nlist(sm)[2] is still set from when it was built)
                cn = pk_nlist(sm)[1];
                if (threadIdx.x == 0) sm.cnt[0] += (unsigned)cn;
                a0 = n;
            } else {
                const int2 r = KEEP ? pk_write_near_outlined(sm.n_cap, sm.cap_near, sm.cap_items, n, a0, gx, gy)
                                    : pk_write_near<false>(sm, n, a0, gx, gy);
                a0 = r.x;
                cn = r.y;
            }
            if (cn > 0) pair_tot += pk_flush_near<MODE, KEEP>(sm, cn, spec, T);
        }
    }

    // ---- phase C: outputs ----------------------------------------------------
    if (G) {
        // genotype gradient: the images' gradients through the symmetry's
        // rotations (backprop_phenotype, kaggle_support.py:1366-1393 and
        // :1155-1195), combined exactly in fixed point
        for (int t = threadIdx.x; t < ng; t += T) {
            long long gx = pk_acc_get(sm, 3 * t), gy = pk_acc_get(sm, 3 * t + 1), gt = pk_acc_get(sm, 3 * t + 2);
            if (sym == 2) {
                const int u = 3 * (t + ng);
                gx -= pk_acc_get(sm, u); gy -= pk_acc_get(sm, u + 1); gt += pk_acc_get(sm, u + 2);
            } else if (sym == 4) {
                const int u1 = 3 * (t + ng), u2 = 3 * (t + 2 * ng), u3 = 3 * (t + 3 * ng);
                gx = gx + pk_acc_get(sm, u1 + 1) - pk_acc_get(sm, u2) - pk_acc_get(sm, u3 + 1);
                gy = gy - pk_acc_get(sm, u1) - pk_acc_get(sm, u2 + 1) + pk_acc_get(sm, u3);
                gt = gt + pk_acc_get(sm, u1 + 2) + pk_acc_get(sm, u2 + 2) + pk_acc_get(sm, u3 + 2);
            }
            G[3 * t] = (float)((double)gx * PK_FX_INV);
            G[3 * t + 1] = (float)((double)gy * PK_FX_INV);
            G[3 * t + 2] = (float)((double)gt * PK_FX_INV);
        }
    }
    // one barrier for every total: per-warp pair partials (int64: exact in
    // any order) and the boundary sums of warp 0
    {
        const long long wsum = pk_warp_sum(pair_tot);
        if ((threadIdx.x & 31) == 0) sm.redl[threadIdx.x >> 5] = wsum;
        if (do_bnd && threadIdx.x < 32) {
            const double4 b4 = pk_canonical_sum4(n, sm.bnd);
            if (threadIdx.x == 0) { sm.red[0] = b4.x; sm.red[1] = b4.y; sm.red[2] = b4.z; sm.red[3] = b4.w; }
        }
        __syncthreads();
    }
    long long ptot = 0;
    for (int w = 0; w < (T >> 5); ++w) ptot += sm.redl[w];
    double total = (double)ptot * PK_FX_INV;
    double h0 = H ? (double)H[0] : 0.0;
    if (do_bnd) {
        total += (double)spec.w_boundary * sm.red[0];
        if (GH && threadIdx.x == 0) {
            GH[0] = (float)(spec.w_boundary * sm.red[1] + (double)spec.w_area * 2.0 * h0);
            GH[1] = (float)(spec.w_boundary * sm.red[2]);
            GH[2] = (float)(spec.w_boundary * sm.red[3]);
        }
    } else if (GH && threadIdx.x == 0) {
        GH[0] = (float)((double)spec.w_area * 2.0 * h0);
        GH[1] = 0.f;
        GH[2] = 0.f;
    }
    if (GH && spec.fixed_h && threadIdx.x == 0) { GH[0] = 0.f; GH[1] = 0.f; GH[2] = 0.f; }
    // AreaCost is zero with a fixed side, its gradient too (use_fixed_h,
    // pack_cost.py:1276-1282; every term's h gradient is zeroed, :178-189)
    if (!spec.fixed_h) total += (double)spec.w_area * h0 * h0;
    __syncthreads();
    return total;
}

// CTA b costs instance order[b] (instance b without an order).  The LUT
// mode has no clipper: it fits 64 registers without spilling, so four CTAs of
// 256 threads share an SM and one CTA's broad phase overlaps the others'
// gathers (4096 x n = 200: 0.201 -> 0.183 ms, the same bits).
template <int MODE, bool SYM>
__global__ void __launch_bounds__(256, MODE == PK_PAIR_LUT ? 4 : 3) pk_cost_kernel(const float* __restrict__ xyt, const int* __restrict__ offsets,
                               const int* __restrict__ order, int E,
                               int n_max, const float* __restrict__ h, PkCostSpec spec,
                               float* __restrict__ cost, float* __restrict__ grad,
                               float* __restrict__ grad_h, int cap_near, int cap_items)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const int e = order ? order[blockIdx.x] : blockIdx.x;
    if (e < 0 || e >= E) return;
    const int base = offsets ? offsets[e] : e * n_max;
    const int n = offsets ? offsets[e + 1] - base : n_max;
    if (n < 0 || n > n_max) {
        if (threadIdx.x == 0) cost[e] = __int_as_float(0x7fc00000);   // NaN marks a bad offset
        return;
    }
    PkCostSmem sm = pk_cost_carve(pk_smem, n_max * (SYM ? pk_symmetry(spec) : 1), cap_near, cap_items);
    if (threadIdx.x < 4) sm.cnt[threadIdx.x] = 0;
    __syncthreads();
    const double tot = pk_eval_instance<MODE, SYM>(xyt + (size_t)base * 3, n, h ? h + 3 * e : nullptr, spec,
                                              grad ? grad + (size_t)base * 3 : nullptr,
                                              grad_h ? grad_h + 3 * e : nullptr, sm);
    if (threadIdx.x == 0) cost[e] = (float)tot;
}

// Threads per CTA as a function of the instance size only (so a packing's
// result never depends on what else is in the batch).
static inline int pk_cost_threads(int n_max)
{
    if (n_max <= 48) return 64;
    if (n_max <= 128) return 128;
    return 256;
}


// count entries of the launch order (all E instances when order is NULL);
// threads 0 = pk_cost_threads of the size bound.
static int pk_launch_cost(const float* xyt, const int* offsets, const int* order, int count, int E, int n_max,
                          const float* h, const PkCostSpec* spec, int threads, float* cost, float* grad,
                          float* grad_h, cudaStream_t st)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (!spec) return pk_fail(PK_EINVAL, "pk_cost: spec is NULL%s");
    if (E < 0 || n_max < 0) return pk_fail(PK_EINVAL, "pk_cost: negative size%s");
    if (count < 0 || count > E) return pk_fail(PK_EINVAL, "pk_cost: order count must be in [0, E]%s");
    if (count < E && !order) return pk_fail(PK_EINVAL, "pk_cost: a partial launch needs an order%s");
    if (E == 0 || count == 0) return PK_OK;
    if (spec && spec->symmetry != 0 && spec->symmetry != 1 && spec->symmetry != 2 && spec->symmetry != 4)
        return pk_fail(PK_EINVAL, "pk_cost: symmetry must be 0, 1, 2 or 4%s");
    if (n_max > PK_MAX_TREES || (spec && (long long)n_max * pk_symmetry(*spec) > PK_MAX_TREES))
        return pk_fail(PK_ERANGE, "pk_cost: more than 1024 (phenotype) trees per instance%s");
    if (!cost || (!xyt && n_max > 0)) return pk_fail(PK_EINVAL, "pk_cost: xyt and cost are required%s");
    if (spec->w_boundary != 0.f && !h) return pk_fail(PK_EINVAL, "pk_cost: boundary term needs h%s");
    if (spec->w_area != 0.f && !h) return pk_fail(PK_EINVAL, "pk_cost: area term needs h%s");
    if (spec->pair_mode == PK_PAIR_LUT) {
        const PkLut& L = spec->lut;
        if (!L.vals || L.nx < 2 || L.ny < 2 || L.nt < 2)
            return pk_fail(PK_EINVAL, "pk_cost: LUT needs vals and at least 2 points per axis%s");
    }
    int T = pk_cost_threads(n_max * pk_symmetry(*spec));
    if (threads != 0) {
        if (threads < 32 || threads > 256 || (threads & 31) || 8 * threads < n_max * pk_symmetry(*spec) - 1)
            return pk_fail(PK_EINVAL, "pk_cost: threads must be 0 or a multiple of 32 in [32, 256] with "
                                      "8 * threads >= n - 1%s");
        T = threads;
    }
    int cap_near, cap_items;
    pk_caps(T, spec->pair_mode, &cap_near, &cap_items);
    const size_t smem = pk_cost_smem_bytes(n_max * pk_symmetry(*spec), cap_near, cap_items);
    cudaError_t err = cudaSuccess;
    switch (spec->pair_mode) {
#define PK_CASE(M)                                                                                  \
    case M:                                                                                         \
        if (spec->symmetry > 1) {                                                                   \
            err = cudaFuncSetAttribute(pk_cost_kernel<M, true>,                                     \
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
            if (err == cudaSuccess)                                                                 \
                pk_cost_kernel<M, true><<<count, T, smem, st>>>(xyt, offsets, order, E, n_max, h, *spec, \
                                                                cost, grad, grad_h, cap_near, cap_items); \
        } else {                                                                                    \
            err = cudaFuncSetAttribute(pk_cost_kernel<M, false>,                                    \
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
            if (err == cudaSuccess)                                                                 \
                pk_cost_kernel<M, false><<<count, T, smem, st>>>(xyt, offsets, order, E, n_max, h,    \
                                                                 *spec, cost, grad, grad_h, cap_near, \
                                                                 cap_items);                          \
        }                                                                                           \
        if (err == cudaSuccess) err = cudaGetLastError();                                           \
        break;
        PK_CASE(PK_PAIR_NONE)
        PK_CASE(PK_PAIR_AREA)
        PK_CASE(PK_PAIR_SEP)
        PK_CASE(PK_PAIR_LUT)
#undef PK_CASE
        default:
            return pk_fail(PK_EINVAL, "pk_cost: unknown pair_mode%s");
    }
    return pk_cuda_check(err, "pk_cost launch");
}

extern "C" int pk_cost(const float* xyt, const int* offsets, int E, int n_uniform, const float* h,
                       const PkCostSpec* spec, float* cost, float* grad, float* grad_h, void* stream)
{
    return pk_launch_cost(xyt, offsets, nullptr, E, E, n_uniform, h, spec, 0, cost, grad, grad_h,
                          (cudaStream_t)stream);
}

extern "C" int pk_cost_ordered(const float* xyt, const int* offsets, const int* order, int count, int E, int n_max,
                               const float* h, const PkCostSpec* spec, int threads, float* cost, float* grad,
                               float* grad_h, void* stream)
{
    if (!order) return pk_fail(PK_EINVAL, "pk_cost_ordered: order is required%s");
    return pk_launch_cost(xyt, offsets, order, count, E, n_max, h, spec, threads, cost, grad, grad_h,
                          (cudaStream_t)stream);
}

extern "C" int pk_overlap(const float* xyt, int E, int n, int use_separation, float* cost, float* grad,
                          void* stream)
{
    PkCostSpec s;
    memset(&s, 0, sizeof(s));
    s.pair_mode = use_separation ? PK_PAIR_SEP : PK_PAIR_AREA;
    s.w_pair = 1.f;
    return pk_launch_cost(xyt, nullptr, nullptr, E, E, n, nullptr, &s, 0, cost, grad, nullptr, (cudaStream_t)stream);
}

extern "C" int pk_boundary(const float* xyt, const float* h, int E, int n, float* cost, float* grad,
                           float* grad_h, void* stream)
{
    PkCostSpec s;
    memset(&s, 0, sizeof(s));
    s.pair_mode = PK_PAIR_NONE;
    s.w_boundary = 1.f;
    return pk_launch_cost(xyt, nullptr, nullptr, E, E, n, h, &s, 0, cost, grad, grad_h, (cudaStream_t)stream);
}

extern "C" int pk_overlap_lut(const float* xyt, const int* offsets, int E, int n_uniform, const PkLut* lut,
                              float* cost, float* grad, void* stream)
{
    if (!lut) return pk_fail(PK_EINVAL, "pk_overlap_lut: lut is NULL%s");
    PkCostSpec s;
    memset(&s, 0, sizeof(s));
    s.pair_mode = PK_PAIR_LUT;
    s.w_pair = 1.f;
    s.lut = *lut;
    return pk_launch_cost(xyt, offsets, nullptr, E, E, n_uniform, nullptr, &s, 0, cost, grad, nullptr,
                          (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// LUT construction from the analytic pair cost: vals[ix, iy, it] = cost of
// a tree at the origin (theta 0) and one at (X[ix], Y[iy], T[it]) -- the
// eval_fn of CollisionCost._ensure_lut_initialized (pack_cost.py:333-377),
// which evaluates 2-tree ensembles with the kernel cost.  Thread per grid
// point; all 16 piece pairs after the centre and AABB culls.
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void pk_lut_build_kernel(const float* __restrict__ X, int nx, const float* __restrict__ Y, int ny,
                                    const float* __restrict__ Tt, int nt, float* __restrict__ vals)
{
    const size_t total = (size_t)nx * ny * nt;
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < total; w += (size_t)gridDim.x * blockDim.x) {
        const int it = (int)(w % nt);
        const int iy = (int)((w / nt) % ny);
        const int ix = (int)(w / ((size_t)nt * ny));
        const float2 d = make_float2(X[ix], Y[iy]);
        float acc = 0.f;
        if (d.x * d.x + d.y * d.y <= c_geom.cutoff_sq) {
            float s, c;
            sincosf(Tt[it], &s, &c);
#pragma unroll 1
            for (int p = 0; p < 4; ++p) {
                float2 P[4];
                float4 bp = make_float4(1e30f, -1e30f, 1e30f, -1e30f);
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    P[v] = c_geom.piece[p][v];
                    bp.x = fminf(bp.x, P[v].x); bp.y = fmaxf(bp.y, P[v].x);
                    bp.z = fminf(bp.z, P[v].y); bp.w = fmaxf(bp.w, P[v].y);
                }
#pragma unroll 1
                for (int q = 0; q < 4; ++q) {
                    float2 Q[4];
                    float4 bq = make_float4(1e30f, -1e30f, 1e30f, -1e30f);
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const float2 l = c_geom.piece[q][v];
                        Q[v] = make_float2(c * l.x - s * l.y + d.x, s * l.x + c * l.y + d.y);
                        bq.x = fminf(bq.x, Q[v].x); bq.y = fmaxf(bq.y, Q[v].x);
                        bq.z = fminf(bq.z, Q[v].y); bq.w = fmaxf(bq.w, Q[v].y);
                    }
                    if (bp.y < bq.x || bq.y < bp.x || bp.w < bq.z || bq.w < bp.z) continue;
                    float val;
                    float3 gp, gq;
                    const bool pt = c_geom.piece_nv[p] == 3, qt = c_geom.piece_nv[q] == 3;
                    if (MODE == PK_PAIR_AREA) {
                        pk_piece_area_grad(P, pt, Q, qt, d, val, gp, gq);
                    } else {
                        float sp;
                        pk_piece_sat_grad(P, pt, Q, qt, d, sp, gp, gq);
                        val = sp * sp;
                    }
                    acc += val;
                }
            }
        }
        vals[w] = acc;
    }
}

extern "C" int pk_lut_build(const float* X, int nx, const float* Y, int ny, const float* T, int nt, int pair_mode,
                            float* vals, void* stream)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (nx < 1 || ny < 1 || nt < 1) return pk_fail(PK_EINVAL, "pk_lut_build: empty grid%s");
    if (!X || !Y || !T || !vals) return pk_fail(PK_EINVAL, "pk_lut_build: NULL pointer%s");
    const size_t total = (size_t)nx * ny * nt;
    const int blocks = (int)((total + 255) / 256 < 148 * 32 ? (total + 255) / 256 : 148 * 32);
    cudaStream_t st = (cudaStream_t)stream;
    if (pair_mode == PK_PAIR_AREA)
        pk_lut_build_kernel<PK_PAIR_AREA><<<blocks, 256, 0, st>>>(X, nx, Y, ny, T, nt, vals);
    else if (pair_mode == PK_PAIR_SEP)
        pk_lut_build_kernel<PK_PAIR_SEP><<<blocks, 256, 0, st>>>(X, nx, Y, ny, T, nt, vals);
    else
        return pk_fail(PK_EINVAL, "pk_lut_build: pair_mode must be AREA or SEP%s");
    return pk_cuda_check(cudaGetLastError(), "pk_lut_build launch");
}
