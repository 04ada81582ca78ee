// moves.cuh -- GA offspring moves (core/pack_move.py) in one launch.
//
// The reference applies a MoveSelector (pack_move.py:119-158) by drawing a
// move per offspring, then, per move type, masking the offspring of that
// type and running the type's vectorised cupy code on them: about a dozen
// elementwise / argsort / gather / scatter launches per move type and a host
// synchronisation per type.  Here one CTA per offspring row chooses its move
// and applies it: the row's trees and its mate's trees sit in shared memory,
// nearest-tree orderings are stable ranks counted in shared memory, and the
// row is written back once.
//
// Random draws: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011), key = seed, counter = (draw / 2,
// row position, call low, call high); each 128-bit block gives two float64
// uniforms with 53 random bits.  Draw k of a row is the same whatever the
// batch, so a call is reproducible and a host restatement can replay it.
// The draws are this library's own stream (the reference's cupy generator
// cannot be reproduced); given the draws, every move follows the
// reference's arithmetic: float64 draws, float32 poses, and float32
// operations where the reference combines float32 arrays with Python
// scalars.
#pragma once
#include "common.cuh"

#define PK_MV_THREADS 128
#define PK_MV_REJECT_LIMIT 100000   // draws of a rejection sampler before it reports and stops

struct PkMvRng {
    uint32_t k0, k1;       // seed
    uint32_t c1, c2, c3;   // row position, call (low, high)
    uint32_t next;         // next draw of the sequential stream
};

__device__ __forceinline__ void pk_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// draw k of a row: uniform in [0, 1) with 53 bits
__device__ __forceinline__ double pk_mv_draw(const PkMvRng& g, uint32_t k)
{
    uint32_t c[4] = {k >> 1, g.c1, g.c2, g.c3};
    pk_philox4x32_10(c, g.k0, g.k1);
    const uint32_t a = (k & 1u) ? c[2] : c[0], b = (k & 1u) ? c[3] : c[1];
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double pk_mv_u(PkMvRng& g) { return pk_mv_draw(g, g.next++); }

// low + (high - low) u, the form of numpy's / cupy's uniform
__device__ __forceinline__ double pk_mv_lerp(double lo, double hi, double u)
{
    return __dadd_rn(lo, __dmul_rn(__dsub_rn(hi, lo), u));
}

__device__ __forceinline__ double pk_mv_uniform(PkMvRng& g, double lo, double hi)
{
    return pk_mv_lerp(lo, hi, pk_mv_u(g));
}

// integer in [lo, hi_excl)
__device__ __forceinline__ int pk_mv_integers(PkMvRng& g, int lo, int hi_excl)
{
    const int span = hi_excl - lo;
    int k = (int)floor(__dmul_rn(pk_mv_u(g), (double)span));
    k = k < 0 ? 0 : (k > span - 1 ? span - 1 : k);
    return lo + k;
}

// numpy's remainder (sign of the divisor), float64 and float32
__device__ __forceinline__ double pk_mv_pymod(double a, double b)
{
    double m = fmod(a, b);
    if (m != 0.0) {
        if ((b < 0.0) != (m < 0.0)) m = __dadd_rn(m, b);
    } else {
        m = copysign(0.0, b);
    }
    return m;
}

__device__ __forceinline__ float pk_mv_pymodf(float a, float b)
{
    float m = fmodf(a, b);
    if (m != 0.0f) {
        if ((b < 0.0f) != (m < 0.0f)) m = __fadd_rn(m, b);
    } else {
        m = copysignf(0.0f, b);
    }
    return m;
}

// EdgeSpacerBasic._check_valid (kaggle_support.py:497-513) in float32;
// EdgeSpacerDummy accepts everything.
__device__ __forceinline__ bool pk_mv_spacer_ok(const PkGenotype& G, float x, float y, float h0)
{
    if (G.spacer == 0) return true;
    const float half = __fmul_rn(h0, 0.5f), mg = (float)G.margin;
    const float tx = __fsub_rn(__fsub_rn(half, (float)G.dist_x), mg);
    const float ty = __fsub_rn(__fsub_rn(half, (float)G.dist_y), mg);
    if (fabsf(x) >= tx || fabsf(y) >= ty) return true;
    const float hs = __fsub_rn(half, mg), dc = (float)G.dist_corner;
    const float xm = fabsf(__fsub_rn(x, hs)), xp = fabsf(__fadd_rn(x, hs));
    const float ym = fabsf(__fsub_rn(y, hs)), yp = fabsf(__fadd_rn(y, hs));
    return __fadd_rn(xm, ym) <= dc || __fadd_rn(xp, ym) <= dc || __fadd_rn(xm, yp) <= dc || __fadd_rn(xp, yp) <= dc;
}

// generate_move_centers of the population's class: SolutionCollectionSquare
// (kaggle_support.py:881-1030), ...Symmetric90 (:1211-1268), ...Symmetric180
// (:1409-1620).  ec < 0 means edge_clearance None.  Centres are float32, as
// the reference stores them.  err bit 0: a rejection sampler hit its limit;
// bit 1: a configuration the reference rejects by assertion.
__device__ void pk_mv_centers(const PkGenotype& G, bool filter, double ec, float h0, float h1, float h2, PkMvRng& g,
                              float& cx, float& cy, int& err)
{
    const bool analytic = G.spacer == 1 && G.dist_corner == 0.0 && filter;
    if (G.kind == PK_GENO_SQUARE) {
        if (ec >= 0.0) {
            const float size = (float)__dsub_rn((double)h0, __dmul_rn(ec, 2.0));
            const double hs = (double)__fmul_rn(size, 0.5f);
            const float ux = (float)pk_mv_uniform(g, -hs, hs);
            const float uy = (float)pk_mv_uniform(g, -hs, hs);
            cx = __fadd_rn(ux, h1);
            cy = __fadd_rn(uy, h2);
            return;
        }
        if (analytic) {   // the O-ring of valid locations as four rectangles
            const float size = h0, half = __fmul_rn(size, 0.5f), mg = (float)G.margin;
            const float xt = __fsub_rn(__fsub_rn(half, (float)G.dist_x), mg);
            const float yt = __fsub_rn(__fsub_rn(half, (float)G.dist_y), mg);
            const float aA = __fmul_rn(__fsub_rn(half, xt), size);
            const float aC = __fmul_rn(__fmul_rn(2.0f, xt), __fsub_rn(half, yt));
            const float tot = __fadd_rn(__fadd_rn(__fadd_rn(aA, aA), aC), aC);
            const float safe = fmaxf(tot, 1e-10f);
            const float pA = __fdiv_rn(aA, safe), pAB = __fdiv_rn(__fadd_rn(aA, aA), safe);
            const float pABC = __fdiv_rn(__fadd_rn(__fadd_rn(aA, aA), aC), safe);
            const double sel = pk_mv_u(g);
            const double H = half, X = xt, Y = yt;
            double x, y;
            if (sel < (double)pA) {
                x = pk_mv_uniform(g, -H, -X);
                y = pk_mv_uniform(g, -H, H);
            } else if (sel < (double)pAB) {
                x = pk_mv_uniform(g, X, H);
                y = pk_mv_uniform(g, -H, H);
            } else if (sel < (double)pABC) {
                x = pk_mv_uniform(g, -X, X);
                y = pk_mv_uniform(g, Y, H);
            } else {
                x = pk_mv_uniform(g, -X, X);
                y = pk_mv_uniform(g, -H, -Y);
            }
            cx = __fadd_rn((float)x, h1);
            cy = __fadd_rn((float)y, h2);
            return;
        }
        const double hs = (double)__fmul_rn(h0, 0.5f);
        for (int t = 0;; ++t) {
            const float x = __fadd_rn((float)pk_mv_uniform(g, -hs, hs), h1);
            const float y = __fadd_rn((float)pk_mv_uniform(g, -hs, hs), h2);
            if (!filter || pk_mv_spacer_ok(G, x, y, h0) || t >= PK_MV_REJECT_LIMIT) {
                if (t >= PK_MV_REJECT_LIMIT) err |= 1;
                cx = x;
                cy = y;
                return;
            }
        }
    }
    if (G.kind == PK_GENO_SYM90) {   // canonical quadrant x, y <= 0 away from the origin corner
        if (filter) err |= 2;
        const double e = ec >= 0.0 ? ec : 0.0;
        const float size = ec >= 0.0 ? (float)__dsub_rn((double)h0, __dmul_rn(ec, 2.0)) : h0;
        if (!((double)h0 >= __dmul_rn(4.0, e))) err |= 2;
        const double lo = -(double)__fmul_rn(size, 0.5f), lim = -__dmul_rn(2.0, e);
        for (int t = 0;; ++t) {
            const double x = pk_mv_uniform(g, lo, 0.0), y = pk_mv_uniform(g, lo, 0.0);
            if (__dadd_rn(x, y) <= lim || t >= PK_MV_REJECT_LIMIT) {
                if (t >= PK_MV_REJECT_LIMIT) err |= 1;
                cx = (float)__dadd_rn(x, (double)h1);
                cy = (float)__dadd_rn(y, (double)h2);
                return;
            }
        }
    }
    // PK_GENO_SYM180: canonical half plane x <= 0
    if (ec >= 0.0) {   // an L of three rectangles, areas in float64
        const float size = (float)__dsub_rn((double)h0, __dmul_rn(ec, 2.0)), half = __fmul_rn(size, 0.5f);
        if (!((double)h0 >= __dmul_rn(4.0, ec))) err |= 2;
        const double H = half;
        const double aA = __dmul_rn(__dsub_rn(H, ec), (double)size), aB = __dmul_rn(ec, __dsub_rn(H, ec));
        const double tot = __dadd_rn(__dadd_rn(aA, aB), aB);
        const double pA = __ddiv_rn(aA, tot), pAB = __ddiv_rn(__dadd_rn(aA, aB), tot);
        const double sel = pk_mv_u(g);
        double x, y;
        if (sel < pA) {
            x = pk_mv_uniform(g, -H, -ec);
            y = pk_mv_uniform(g, -H, H);
        } else if (sel < pAB) {
            x = pk_mv_uniform(g, -ec, 0.0);
            y = pk_mv_uniform(g, ec, H);
        } else {
            x = pk_mv_uniform(g, -ec, 0.0);
            y = pk_mv_uniform(g, -H, -ec);
        }
        cx = __fadd_rn((float)x, h1);
        cy = __fadd_rn((float)y, h2);
        return;
    }
    if (analytic) {   // three rectangles, areas in float32
        const float size = h0, half = __fmul_rn(size, 0.5f), mg = (float)G.margin;
        const float xt = __fsub_rn(__fsub_rn(half, (float)G.dist_x), mg);
        const float yt = __fsub_rn(__fsub_rn(half, (float)G.dist_y), mg);
        const float aA = __fmul_rn(__fsub_rn(half, xt), size), aB = __fmul_rn(xt, __fsub_rn(half, yt));
        const float tot = __fadd_rn(__fadd_rn(aA, aB), aB);
        const float safe = fmaxf(tot, 1e-10f);
        const float pA = __fdiv_rn(aA, safe), pAB = __fdiv_rn(__fadd_rn(aA, aB), safe);
        const double sel = pk_mv_u(g);
        const double H = half, X = xt, Y = yt;
        double x, y;
        if (sel < (double)pA) {
            x = pk_mv_uniform(g, -H, -X);
            y = pk_mv_uniform(g, -H, H);
        } else if (sel < (double)pAB) {
            x = pk_mv_uniform(g, -X, 0.0);
            y = pk_mv_uniform(g, Y, H);
        } else {
            x = pk_mv_uniform(g, -X, 0.0);
            y = pk_mv_uniform(g, -H, -Y);
        }
        cx = __fadd_rn((float)x, h1);
        cy = __fadd_rn((float)y, h2);
        return;
    }
    const double hs = (double)__fmul_rn(h0, 0.5f);
    for (int t = 0;; ++t) {
        const double x = pk_mv_uniform(g, -hs, 0.0), y = pk_mv_uniform(g, -hs, hs);
        const float fx = (float)__dadd_rn(x, (double)h1), fy = (float)__dadd_rn(y, (double)h2);
        if (!filter || pk_mv_spacer_ok(G, fx, fy, h0) || t >= PK_MV_REJECT_LIMIT) {
            if (t >= PK_MV_REJECT_LIMIT) err |= 1;
            cx = fx;
            cy = fy;
            return;
        }
    }
}

// _sample_trees_to_mutate (pack_move.py:58-116): a uniform tree, or the r-th
// tree the edge spacer accepts (all trees when it accepts none).
__device__ int pk_mv_sample_tree(const PkGenotype& G, bool filter, const float* sx, const float* sy, int n, float h0,
                                 PkMvRng& g)
{
    if (!filter) return pk_mv_integers(g, 0, n);
    int cnt = 0;
    for (int i = 0; i < n; ++i) cnt += pk_mv_spacer_ok(G, sx[i], sy[i], h0);
    const bool all = cnt == 0;
    if (all) cnt = n;
    int r = (int)__dmul_rn(pk_mv_u(g), (double)cnt);
    if (r > cnt - 1) r = cnt - 1;
    for (int i = 0, seen = 0; i < n; ++i) {
        if (all || pk_mv_spacer_ok(G, sx[i], sy[i], h0)) {
            if (seen == r) return i;
            ++seen;
        }
    }
    return n - 1;
}

// stable ascending order with NaN last: does (a, i) come before (b, j)?
__device__ __forceinline__ bool pk_mv_before(double a, int i, double b, int j)
{
    const bool na = isnan(a), nb = isnan(b);
    if (na || nb) return na == nb ? i < j : nb;
    return a < b || (a == b && i < j);
}

// ord[r] = the tree of rank r for r < limit (argsort, stable); the order is
// total, so the ranks are a permutation and fill every slot.  Starts and
// ends with a barrier.
__device__ void pk_mv_rank(const double* key, int n, short* ord, int limit)
{
    for (int r = threadIdx.x; r < limit; r += blockDim.x) ord[r] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double ki = key[i];
        int r = 0;
        for (int j = 0; j < n; ++j) r += pk_mv_before(key[j], j, ki, i);
        if (r < limit) ord[r] = (short)i;
    }
    __syncthreads();
}

__device__ __forceinline__ float pk_mv_linf(float x, float y, float cx, float cy)
{
    return fmaxf(fabsf(__fsub_rn(x, cx)), fabsf(__fsub_rn(y, cy)));
}

// phenotype trees per genotype tree
__device__ __forceinline__ int pk_mv_mult(int kind) { return kind == PK_GENO_SYM90 ? 4 : (kind == PK_GENO_SYM180 ? 2 : 1); }

struct PkMvShared {
    int move, tree, nrep, rot, mirror, maxj, err, use_f64;
    uint32_t kbase;
    float fc[4];     // float32 centres / line points
    double dc[8];    // float64 parameters
};

// One CTA per offspring row.  Shared memory: the row's trees (3 n float),
// the mate's trees (3 n float), two sort keys (2 n double), two orders
// (2 n short), two validity masks (2 n byte).
__global__ void __launch_bounds__(PK_MV_THREADS) pk_moves_kernel(
    float* __restrict__ xyt, const float* __restrict__ h, int E, int n, const int* __restrict__ inds, int C,
    const float* __restrict__ mxyt, const float* __restrict__ mh, int M, const int* __restrict__ inds_mate,
    const PkMoveSet set,
    uint32_t k0, uint32_t k1, uint32_t call_lo, uint32_t call_hi, int* __restrict__ chosen, int* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    double* kd = (double*)pk_smem;
    double* km = kd + n;
    float* sx = (float*)(km + n);
    float* sy = sx + n;
    float* st = sy + n;
    float* mx = st + n;
    float* my = mx + n;
    float* mt = my + n;
    short* oi = (short*)(mt + n);
    short* om = oi + n;
    unsigned char* vi = (unsigned char*)(om + n);
    unsigned char* vm = vi + n;
    __shared__ PkMvShared S;

    const int c = blockIdx.x;
    if (c >= C) return;
    const int row = inds[c];
    bool needs_mate = false;
    for (int m = 0; m < set.n_moves; ++m)
        needs_mate |= set.moves[m].type == PK_MOVE_CROSSOVER || set.moves[m].type == PK_MOVE_CROSSOVER2;
    const int mrow_checked = needs_mate ? inds_mate[c] : 0;
    if (row < 0 || row >= E || (needs_mate && (mrow_checked < 0 || mrow_checked >= M))) {   // bad index: report, skip
        if (threadIdx.x == 0) {
            if (status) atomicOr(status, 4);
            if (chosen) chosen[c] = -1;
        }
        return;
    }
    const PkGenotype& G = set.geno;
    PkMvRng g;
    g.k0 = k0;
    g.k1 = k1;
    g.c1 = (uint32_t)c;
    g.c2 = call_lo;
    g.c3 = call_hi;
    g.next = 0;
    float* X = xyt + (size_t)row * n * 3;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        sx[i] = X[3 * i];
        sy[i] = X[3 * i + 1];
        st[i] = X[3 * i + 2];
    }
    const float h0 = h[3 * row], h1 = h[3 * row + 1], h2 = h[3 * row + 2];
    if (threadIdx.x == 0) {
        const double u = pk_mv_u(g);
        int m = 0;
        while (m < set.n_moves && set.cum_prob[m] < u) ++m;   // searchsorted, side left
        S.move = m < set.n_moves ? m : -1;
        S.err = 0;
        if (chosen) chosen[c] = S.move;
    }
    __syncthreads();
    if (S.move < 0) return;
    const PkMove& mv = set.moves[S.move];
    const bool filter = G.filter && mv.respect_edge_spacer_filter;
    const int type = mv.type;

    if (type == PK_MOVE_RANDOM_TREE || type == PK_MOVE_JIGGLE_TREE) {   // pack_move.py:161-224
        if (threadIdx.x == 0) {
            int err = 0;
            const int t = pk_mv_sample_tree(G, filter, sx, sy, n, h0, g);
            if (type == PK_MOVE_RANDOM_TREE) {
                float cx, cy;
                pk_mv_centers(G, filter, -1.0, h0, h1, h2, g, cx, cy, err);
                const double th = pk_mv_uniform(g, -M_PI, M_PI);
                sx[t] = cx;
                sy[t] = cy;
                st[t] = (float)th;
            } else {
                const double ox = pk_mv_uniform(g, -mv.max_xy_move, mv.max_xy_move);
                const double oy = pk_mv_uniform(g, -mv.max_xy_move, mv.max_xy_move);
                const double ot = pk_mv_uniform(g, -mv.max_theta_move, mv.max_theta_move);
                sx[t] = (float)__dadd_rn((double)sx[t], ox);
                sy[t] = (float)__dadd_rn((double)sy[t], oy);
                st[t] = (float)__dadd_rn((double)st[t], ot);
            }
            S.err = err;
        }
    } else if (type == PK_MOVE_JIGGLE_CLUSTER) {   // pack_move.py:227-298
        if (threadIdx.x == 0) {
            int err = 0;
            float cx, cy;
            pk_mv_centers(G, filter, -1.0, h0, h1, h2, g, cx, cy, err);
            const int maxj = min(mv.max_n_trees, n), minj = min(mv.min_n_trees, n);
            S.nrep = pk_mv_integers(g, minj, maxj + 1);
            S.maxj = maxj;
            S.kbase = g.next;
            S.fc[0] = cx;
            S.fc[1] = cy;
            S.err = err;
        }
        __syncthreads();
        const float cx = S.fc[0], cy = S.fc[1];
        const int maxj = S.maxj, nj = S.nrep;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float dx = __fsub_rn(sx[i], cx), dy = __fsub_rn(sy[i], cy);
            kd[i] = (double)__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        }
        __syncthreads();
        pk_mv_rank(kd, n, oi, maxj);
        for (int r = threadIdx.x; r < maxj; r += blockDim.x) {
            const int t = oi[r];
            const double mask = r < nj ? 1.0 : 0.0;
            const double ox = __dmul_rn(pk_mv_lerp(-mv.max_xy_move, mv.max_xy_move, pk_mv_draw(g, S.kbase + r)), mask);
            const double oy = __dmul_rn(pk_mv_lerp(-mv.max_xy_move, mv.max_xy_move, pk_mv_draw(g, S.kbase + maxj + r)), mask);
            const double ot = __dmul_rn(pk_mv_lerp(-mv.max_theta_move, mv.max_theta_move,
                                                   pk_mv_draw(g, S.kbase + 2 * maxj + r)), mask);
            sx[t] = (float)__dadd_rn((double)sx[t], ox);
            sy[t] = (float)__dadd_rn((double)sy[t], oy);
            st[t] = (float)__dadd_rn((double)st[t], ot);
        }
    } else if (type == PK_MOVE_TRANSLATE) {   // pack_move.py:301-333
        if (threadIdx.x == 0) {
            const double hs = (double)__fmul_rn(h0, 0.5f);
            S.dc[0] = pk_mv_uniform(g, -hs, hs);
            S.dc[1] = pk_mv_uniform(g, -hs, hs);
        }
        __syncthreads();
        const double ox = S.dc[0], oy = S.dc[1], H = h0, half = (double)__fmul_rn(h0, 0.5f);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            sx[i] = (float)__dsub_rn(pk_mv_pymod(__dadd_rn((double)sx[i], ox), H), half);
            sy[i] = (float)__dsub_rn(pk_mv_pymod(__dadd_rn((double)sy[i], oy), H), half);
        }
    } else if (type == PK_MOVE_TWIST) {   // pack_move.py:336-382
        if (threadIdx.x == 0) {
            int err = 0;
            float cx, cy;
            pk_mv_centers(G, filter, -1.0, h0, h1, h2, g, cx, cy, err);
            S.fc[0] = cx;
            S.fc[1] = cy;
            S.dc[0] = pk_mv_uniform(g, -M_PI, M_PI);
            S.dc[1] = pk_mv_uniform(g, mv.min_radius, mv.max_radius);
            S.err = err;
        }
        __syncthreads();
        const float cx = S.fc[0], cy = S.fc[1];
        const double a = S.dc[0], rad = S.dc[1];
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float dx = __fsub_rn(sx[i], cx), dy = __fsub_rn(sy[i], cy);
            const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
            const double tw = __dmul_rn(a, fmax(0.0, __dsub_rn(1.0, __ddiv_rn((double)dist, rad))));
            double s, co;
            sincos(tw, &s, &co);
            sx[i] = (float)__dsub_rn(__dadd_rn((double)cx, __dmul_rn((double)dx, co)), __dmul_rn((double)dy, s));
            sy[i] = (float)__dadd_rn(__dadd_rn((double)cy, __dmul_rn((double)dx, s)), __dmul_rn((double)dy, co));
            st[i] = (float)__dadd_rn((double)st[i], tw);
        }
    } else if (type == PK_MOVE_CROSSOVER) {   // pack_move.py:406-632
        const int mrow = mrow_checked;
        const float* MX = mxyt + (size_t)mrow * n * 3;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            mx[i] = MX[3 * i];
            my[i] = MX[3 * i + 1];
            mt[i] = MX[3 * i + 2];
        }
        if (threadIdx.x == 0) {
            int err = 0;
            const int mint = min(mv.min_n_trees, n);
            int maxt = min((int)rint(__dmul_rn(mv.max_n_trees_ratio, (double)n)), n);
            if (maxt < mint) maxt = mint;
            const int nrep = pk_mv_integers(g, mint, maxt + 1);
            S.nrep = nrep;
            S.rot = pk_mv_integers(g, 0, 4);
            S.mirror = pk_mv_integers(g, 0, 2) == 1;
            float icx, icy;
            double mcx, mcy;
            if (mv.simple_mate_location) {
                const int NT = n * pk_mv_mult(G.kind);
                const double ss = __dmul_rn((double)h0, sqrt(__ddiv_rn((double)nrep, (double)NT)));
                const double ec = __dmul_rn(ss, 0.5);
                float fx, fy;
                pk_mv_centers(G, filter, ec, h0, h1, h2, g, icx, icy, err);
                pk_mv_centers(G, filter, ec, h0, h1, h2, g, fx, fy, err);
                mcx = fx;
                mcy = fy;
                S.use_f64 = 0;
            } else {
                pk_mv_centers(G, filter, -1.0, h0, h1, h2, g, icx, icy, err);
                const int sgx = pk_mv_integers(g, 0, 2) * 2 - 1, sgy = pk_mv_integers(g, 0, 2) * 2 - 1;
                const float m0 = mh[3 * mrow], m1 = mh[3 * mrow + 1], m2 = mh[3 * mrow + 2];
                const float ratio = __fdiv_rn(m0, h0);
                const float ax = __fmul_rn(fabsf(__fsub_rn(icx, h1)), ratio);
                const float ay = __fmul_rn(fabsf(__fsub_rn(icy, h2)), ratio);
                mcx = __dadd_rn(__dmul_rn((double)ax, (double)sgx), (double)m1);
                mcy = __dadd_rn(__dmul_rn((double)ay, (double)sgy), (double)m2);
                S.use_f64 = 1;
            }
            S.fc[0] = icx;
            S.fc[1] = icy;
            S.dc[0] = mcx;
            S.dc[1] = mcy;
            S.err = err;
        }
        __syncthreads();
        const float icx = S.fc[0], icy = S.fc[1];
        const double mcx = S.dc[0], mcy = S.dc[1];
        const int nrep = S.nrep;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            kd[i] = (double)pk_mv_linf(sx[i], sy[i], icx, icy);
            km[i] = S.use_f64 ? fmax(fabs(__dsub_rn((double)mx[i], mcx)), fabs(__dsub_rn((double)my[i], mcy)))
                              : (double)pk_mv_linf(mx[i], my[i], (float)mcx, (float)mcy);
        }
        __syncthreads();
        pk_mv_rank(kd, n, oi, nrep);
        pk_mv_rank(km, n, om, nrep);
        if (threadIdx.x == 0) {   // centres of mass of the selections, summed in rank order
            float a = 0.f, b = 0.f, p = 0.f, q = 0.f;
            for (int r = 0; r < nrep; ++r) {
                a = __fadd_rn(a, sx[oi[r]]);
                b = __fadd_rn(b, sy[oi[r]]);
                p = __fadd_rn(p, mx[om[r]]);
                q = __fadd_rn(q, my[om[r]]);
            }
            S.dc[2] = __ddiv_rn((double)a, (double)nrep);
            S.dc[3] = __ddiv_rn((double)b, (double)nrep);
            S.dc[4] = __ddiv_rn((double)p, (double)nrep);
            S.dc[5] = __ddiv_rn((double)q, (double)nrep);
        }
        __syncthreads();
        const double icmx = S.dc[2], icmy = S.dc[3], mcmx = S.dc[4], mcmy = S.dc[5];
        const double ang = __dmul_rn((double)S.rot, M_PI / 2);
        double sa, ca;
        sincos(ang, &sa, &ca);
        for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
            const int j = om[r], t = oi[r];
            double dx = __dsub_rn((double)mx[j], mcmx), dy = __dsub_rn((double)my[j], mcmy);
            double th = mt[j];
            if (S.mirror) {
                dy = -dy;
                th = (double)__fsub_rn((float)M_PI, mt[j]);
            }
            if (S.rot != 0) {
                const double rx = __dsub_rn(__dmul_rn(dx, ca), __dmul_rn(dy, sa));
                const double ry = __dadd_rn(__dmul_rn(dx, sa), __dmul_rn(dy, ca));
                dx = rx;
                dy = ry;
                th = __dadd_rn(th, ang);
            }
            sx[t] = (float)__dadd_rn(icmx, dx);
            sy[t] = (float)__dadd_rn(icmy, dy);
            st[t] = (float)th;
        }
    } else if (type == PK_MOVE_CROSSOVER2) {   // pack_move.py:635-1033
        const int mrow = mrow_checked;
        const float* MX = mxyt + (size_t)mrow * n * 3;
        const float m0 = mh[3 * mrow], m1 = mh[3 * mrow + 1], m2 = mh[3 * mrow + 2];
        if (threadIdx.x == 0) {
            S.rot = mv.do_90_rotation ? pk_mv_integers(g, 0, 4) : 2 * pk_mv_integers(g, 0, 2);
            S.mirror = pk_mv_integers(g, 0, 2) == 1;
        }
        __syncthreads();
        const int rot = S.rot;
        const bool mir = S.mirror;
        const double ang = __dmul_rn((double)rot, M_PI / 2);
        double sa, ca;
        sincos(ang, &sa, &ca);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            // _apply_orientation_preselection (:1003-1033), then the mate class's canonicalize_xyt
            float x = MX[3 * i], y = MX[3 * i + 1], th = MX[3 * i + 2];
            if (mir) {
                y = -y;
                th = __fsub_rn((float)M_PI, th);
            }
            if (rot != 0) {
                const float rx = (float)__dsub_rn(__dmul_rn((double)x, ca), __dmul_rn((double)y, sa));
                const float ry = (float)__dadd_rn(__dmul_rn((double)x, sa), __dmul_rn((double)y, ca));
                th = (float)__dadd_rn((double)th, ang);
                x = rx;
                y = ry;
            }
            if (G.mate_kind == PK_GENO_SYM90) {   // kaggle_support.py:1053-1088
                const bool q1 = x > 0.f && y > 0.f, q2 = x <= 0.f && y > 0.f, q4 = x > 0.f && y <= 0.f;
                const float nx = q1 ? -x : (q2 ? -y : (q4 ? y : x));
                const float ny = q1 ? -y : (q2 ? x : (q4 ? -x : y));
                const float nt = q1 ? __fadd_rn(th, (float)M_PI)
                                    : (q2 ? __fadd_rn(th, (float)(M_PI / 2))
                                          : (q4 ? __fadd_rn(th, (float)(3 * M_PI / 2)) : th));
                x = nx;
                y = ny;
                th = pk_mv_pymodf(nt, (float)(2 * M_PI));
            } else if (G.mate_kind == PK_GENO_SYM180) {   // kaggle_support.py:1287-1310
                const bool r = x > 0.f;
                const float nt = r ? __fadd_rn(th, (float)M_PI) : th;
                x = r ? -x : x;
                y = r ? -y : y;
                th = pk_mv_pymodf(nt, (float)(2 * M_PI));
            }
            mx[i] = x;
            my[i] = y;
            mt[i] = th;
            vi[i] = !filter || pk_mv_spacer_ok(G, sx[i], sy[i], h0);
            vm[i] = !filter || pk_mv_spacer_ok(G, x, y, m0);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int err = 0, ci = 0, cm = 0;
            for (int i = 0; i < n; ++i) {
                ci += vi[i];
                cm += vm[i];
            }
            const int usable = max(min(ci, cm), 0);
            const int mint = min(min(mv.min_n_trees, n), usable);
            int maxt = min((int)floor(__dmul_rn(mv.max_n_trees_ratio, (double)usable)), usable);
            maxt = max(maxt, mint);
            const int span = maxt - mint + 1;
            const int nrep = mint + (int)floor(__dmul_rn(pk_mv_u(g), (double)span));
            S.nrep = nrep;
            float lx, ly, mlx, mly;
            if (!mv.decouple_mate_location) {
                pk_mv_centers(G, filter, -1.0, h0, h1, h2, g, lx, ly, err);
                mlx = __fadd_rn(__fsub_rn(lx, h1), m1);
                mly = __fadd_rn(__fsub_rn(ly, h2), m2);
            } else if (mv.use_edge_clearance_when_decoupled) {
                const int NT = n * pk_mv_mult(G.mate_kind);
                const double ss = __dmul_rn((double)h0, sqrt(__ddiv_rn((double)nrep, (double)NT)));
                const double ec = __dmul_rn(ss, 0.5);
                pk_mv_centers(G, filter, ec, h0, h1, h2, g, lx, ly, err);
                pk_mv_centers(G, filter, ec, h0, h1, h2, g, mlx, mly, err);
            } else {
                pk_mv_centers(G, filter, -1.0, h0, h1, h2, g, lx, ly, err);
                pk_mv_centers(G, filter, -1.0, h0, h1, h2, g, mlx, mly, err);
            }
            S.fc[0] = lx;
            S.fc[1] = ly;
            S.fc[2] = mlx;
            S.fc[3] = mly;
            if (mv.distance_function == PK_XDIST_STRIPE) {
                const double la = pk_mv_uniform(g, 0.0, 2 * M_PI);
                double s, co;
                sincos(la, &s, &co);
                S.dc[0] = -s;
                S.dc[1] = co;
            }
            S.err = err;
        }
        __syncthreads();
        const float lx = S.fc[0], ly = S.fc[1], mlx = S.fc[2], mly = S.fc[3];
        const int df = mv.distance_function;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float x = sx[i], y = sy[i], a = mx[i], b = my[i];
            double di, dm;
            if (df == PK_XDIST_STRIPE) {
                const double nx = S.dc[0], ny = S.dc[1];
                di = fabs(__dadd_rn(__dmul_rn((double)__fsub_rn(x, lx), nx), __dmul_rn((double)__fsub_rn(y, ly), ny)));
                dm = fabs(__dadd_rn(__dmul_rn((double)__fsub_rn(a, mlx), nx), __dmul_rn((double)__fsub_rn(b, mly), ny)));
            } else if (df == PK_XDIST_SQUARE) {
                di = pk_mv_linf(x, y, lx, ly);
                dm = pk_mv_linf(a, b, mlx, mly);
            } else if (df == PK_XDIST_SQUARE90) {   // images (x, y), (-y, x), (-x, -y), (y, -x)
                di = fminf(fminf(pk_mv_linf(x, y, lx, ly), pk_mv_linf(-y, x, lx, ly)),
                           fminf(pk_mv_linf(-x, -y, lx, ly), pk_mv_linf(y, -x, lx, ly)));
                const float d0 = pk_mv_linf(a, b, mlx, mly), d1 = pk_mv_linf(-b, a, mlx, mly);
                const float d2 = pk_mv_linf(-a, -b, mlx, mly), d3 = pk_mv_linf(b, -a, mlx, mly);
                dm = fminf(fminf(d0, d1), fminf(d2, d3));
                int k = 0;
                float best = d0;
                if (d1 < best) { best = d1; k = 1; }
                if (d2 < best) { best = d2; k = 2; }
                if (d3 < best) { best = d3; k = 3; }
                const float t = mt[i];
                if (k == 1) { mx[i] = -b; my[i] = a; mt[i] = __fadd_rn(t, (float)(M_PI / 2)); }
                if (k == 2) { mx[i] = -a; my[i] = -b; mt[i] = __fadd_rn(t, (float)M_PI); }
                if (k == 3) { mx[i] = b; my[i] = -a; mt[i] = __fadd_rn(t, (float)(3 * M_PI / 2)); }
            } else {   // PK_XDIST_SQUARE180: images (x, y), (-x, -y)
                di = fminf(pk_mv_linf(x, y, lx, ly), pk_mv_linf(-x, -y, lx, ly));
                const float d0 = pk_mv_linf(a, b, mlx, mly), d1 = pk_mv_linf(-a, -b, mlx, mly);
                dm = fminf(d0, d1);
                if (d1 < d0) { mx[i] = -a; my[i] = -b; mt[i] = __fadd_rn(mt[i], (float)M_PI); }
            }
            kd[i] = vi[i] ? di : (double)INFINITY;
            km[i] = vm[i] ? dm : (double)INFINITY;
        }
        __syncthreads();
        const int nrep = S.nrep;
        pk_mv_rank(kd, n, oi, nrep);
        pk_mv_rank(km, n, om, nrep);
        const float ox = mv.decouple_mate_location ? __fsub_rn(lx, mlx) : 0.f;
        const float oy = mv.decouple_mate_location ? __fsub_rn(ly, mly) : 0.f;
        for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
            const int j = om[r], t = oi[r];
            sx[t] = mv.decouple_mate_location ? __fadd_rn(mx[j], ox) : mx[j];
            sy[t] = mv.decouple_mate_location ? __fadd_rn(my[j], oy) : my[j];
            st[t] = mt[j];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        X[3 * i] = sx[i];
        X[3 * i + 1] = sy[i];
        X[3 * i + 2] = st[i];
    }
    if (threadIdx.x == 0 && S.err && status) atomicOr(status, S.err);
}

__global__ void pk_move_draws_kernel(uint32_t k0, uint32_t k1, uint32_t c2, uint32_t c3, int row, int first, int count,
                                     double* out)
{
    PkMvRng g;
    g.k0 = k0;
    g.k1 = k1;
    g.c1 = (uint32_t)row;
    g.c2 = c2;
    g.c3 = c3;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        out[i] = pk_mv_draw(g, (uint32_t)(first + i));
}

static size_t pk_moves_smem(int n) { return (size_t)n * (2 * sizeof(double) + 6 * sizeof(float) + 2 * sizeof(short) + 2); }

extern "C" int pk_moves(float* xyt, const float* h, int E, int n, const int* inds_to_do, int C, const float* mate_xyt,
                        const float* mate_h, int M, const int* inds_mate, const PkMoveSet* set, uint64_t seed,
                        uint64_t call, int* chosen, int* status, void* stream)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (!set) return pk_fail(PK_EINVAL, "pk_moves: set is required%s");
    if (E < 0 || C < 0 || M < 0 || n < 1) return pk_fail(PK_EINVAL, "pk_moves: bad sizes%s");
    if (n > PK_MAX_TREES) return pk_fail(PK_ERANGE, "pk_moves: more than 1024 trees%s");
    if (set->n_moves < 1 || set->n_moves > PK_MAX_MOVE_TYPES)
        return pk_fail(PK_EINVAL, "pk_moves: n_moves must be in [1, 16]%s");
    bool needs_mate = false;
    for (int m = 0; m < set->n_moves; ++m) {
        const PkMove& mv = set->moves[m];
        if (mv.type < PK_MOVE_RANDOM_TREE || mv.type > PK_MOVE_CROSSOVER2)
            return pk_fail(PK_EINVAL, "pk_moves: unknown move type%s");
        if (mv.type == PK_MOVE_CROSSOVER2 && (mv.distance_function < PK_XDIST_STRIPE || mv.distance_function > PK_XDIST_SQUARE180))
            return pk_fail(PK_EINVAL, "pk_moves: unknown Crossover2 distance function%s");
        if (mv.type == PK_MOVE_JIGGLE_CLUSTER && (mv.min_n_trees < 0 || mv.max_n_trees < mv.min_n_trees))
            return pk_fail(PK_EINVAL, "pk_moves: JiggleCluster needs 0 <= min_N_trees <= max_N_trees%s");
        needs_mate |= mv.type == PK_MOVE_CROSSOVER || mv.type == PK_MOVE_CROSSOVER2;
    }
    if (set->geno.kind < PK_GENO_SQUARE || set->geno.kind > PK_GENO_SYM180 || set->geno.mate_kind < PK_GENO_SQUARE ||
        set->geno.mate_kind > PK_GENO_SYM180 || set->geno.spacer < 0 || set->geno.spacer > 1)
        return pk_fail(PK_EINVAL, "pk_moves: bad genotype description%s");
    if (C == 0) return PK_OK;
    if (!xyt || !h || !inds_to_do || (needs_mate && (!mate_xyt || !mate_h || !inds_mate)))
        return pk_fail(PK_EINVAL, "pk_moves: NULL pointer%s");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t smem = pk_moves_smem(n);
    cudaError_t err = cudaFuncSetAttribute(pk_moves_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_moves attribute");
    pk_moves_kernel<<<C, PK_MV_THREADS, smem, st>>>(xyt, h, E, n, inds_to_do, C, mate_xyt, mate_h, M, inds_mate, *set,
                                                    (uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)call,
                                                    (uint32_t)(call >> 32), chosen, status);
    return pk_cuda_check(cudaGetLastError(), "pk_moves launch");
}

extern "C" int pk_move_draws(uint64_t seed, uint64_t call, int row, int first, int count, double* out, void* stream)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (count < 0 || first < 0 || row < 0 || (count > 0 && !out)) return pk_fail(PK_EINVAL, "pk_move_draws: bad arguments%s");
    if (count == 0) return PK_OK;
    const int blocks = (count + 255) / 256 < 1024 ? (count + 255) / 256 : 1024;
    pk_move_draws_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>((uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)call,
                                                                   (uint32_t)(call >> 32), row, first, count, out);
    return pk_cuda_check(cudaGetLastError(), "pk_move_draws launch");
}
