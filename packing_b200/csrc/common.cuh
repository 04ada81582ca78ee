// common.cuh -- shared definitions for the packing_b200 CUDA library.
//
// The library is one translation unit (capi.cu includes every *.cuh), so the
// __constant__ / __device__ symbols below exist once per loaded library.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/packb200.h"

#define PK_FULL_MASK 0xffffffffu

// Tree geometry in the form the kernels read it.  Pieces are CCW; a
// triangle is padded to four vertices as [v0, v1, v2, v0], so its edge 3 is
// degenerate (zero length) and is skipped as a clipping line.
struct PkDevGeom {
    float2 piece[PK_NUM_PIECES][4];
    int piece_nv[PK_NUM_PIECES];
    float2 tree[PK_MAX_TREE_VERTS];
    int n_tree;
    float max_radius;
    float cutoff_sq;    // (2 R)^2: farther centres cannot overlap
    float coll_tiny;    // 2e-6 * longest piece edge: bound on |cross| of near-collinear points
};

// FP64 tables: the search tree, and the legality tree of the validator
// (CCW pieces padded like the FP32 ones).
struct PkDevGeom64 {
    double2 piece[PK_NUM_PIECES][4];
    int piece_nv[PK_NUM_PIECES];
    double2 tree[PK_MAX_TREE_VERTS];
    int n_tree;
    double max_radius;
    double2 legal_piece[PK_NUM_PIECES][4];
    double2 legal_tree[PK_MAX_TREE_VERTS];
    double legal_radius;
};

__constant__ PkDevGeom c_geom;
__constant__ PkDevGeom64 c_geom64;

// Fixed-point scale of the pair-gradient accumulators: sums of int64 are
// associative, so the result does not depend on the order in which threads
// add their contributions (batched == single, bit for bit).
#define PK_FX_SCALE 4294967296.0f          // 2^32
#define PK_FX_INV (1.0 / 4294967296.0)

__device__ __forceinline__ long long pk_to_fx(float v)
{
    return __float2ll_rn(v * PK_FX_SCALE);
}

__device__ __forceinline__ float pk_cross(float2 a, float2 b) { return a.x * b.y - a.y * b.x; }

// (B - A) x (C - A): >= 0 means C is on or left of the directed line A->B.
__device__ __forceinline__ float pk_cross3(float2 a, float2 b, float2 c)
{
    return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x);
}

template <typename T>
__device__ __forceinline__ T pk_warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(PK_FULL_MASK, v, o);
    return v;
}

// Deterministic block-wide sum: fixed warp-shuffle tree, then warp 0 sums the
// per-warp partials in warp order.  scratch needs blockDim.x/32 entries.
// Every thread gets the result.
template <typename T>
__device__ __forceinline__ T pk_block_sum(T v, T* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = pk_warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T r = (lane < nw) ? scratch[lane] : T(0);
    if (warp == 0) {
        r = pk_warp_sum(r);
        if (lane == 0) scratch[0] = r;
    }
    __syncthreads();
    r = scratch[0];
    __syncthreads();
    return r;
}

template <typename T>
__device__ __forceinline__ T pk_block_max(T v, T* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(PK_FULL_MASK, v, o));
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T r = (lane < nw) ? scratch[lane] : scratch[0];
    if (warp == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = max(r, __shfl_xor_sync(PK_FULL_MASK, r, o));
        if (lane == 0) scratch[0] = r;
    }
    __syncthreads();
    r = scratch[0];
    __syncthreads();
    return r;
}

// Block-wide maximum of four floats at once (one round trip through
// shared memory); scratch needs 4 * warps floats.  All threads get the result.
__device__ __forceinline__ float4 pk_block_max4(float4 v, float* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x = fmaxf(v.x, __shfl_xor_sync(PK_FULL_MASK, v.x, o));
        v.y = fmaxf(v.y, __shfl_xor_sync(PK_FULL_MASK, v.y, o));
        v.z = fmaxf(v.z, __shfl_xor_sync(PK_FULL_MASK, v.z, o));
        v.w = fmaxf(v.w, __shfl_xor_sync(PK_FULL_MASK, v.w, o));
    }
    __syncthreads();
    if (lane == 0) {
        scratch[4 * warp + 0] = v.x; scratch[4 * warp + 1] = v.y;
        scratch[4 * warp + 2] = v.z; scratch[4 * warp + 3] = v.w;
    }
    __syncthreads();
    float4 r = v;
    for (int w = 0; w < nw; ++w) {
        r.x = fmaxf(r.x, scratch[4 * w + 0]); r.y = fmaxf(r.y, scratch[4 * w + 1]);
        r.z = fmaxf(r.z, scratch[4 * w + 2]); r.w = fmaxf(r.w, scratch[4 * w + 3]);
    }
    __syncthreads();
    return r;
}

// Exclusive prefix sum of in[0..count) into out[0..count], out[count] = total.
// scratch needs 32 ints.  Called by all threads; ends with a barrier.
__device__ __forceinline__ void pk_block_exclusive_scan(const int* in, int* out, int count, int* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int carry = 0;
    for (int base = 0; base < count; base += blockDim.x) {
        const int k = base + threadIdx.x;
        const int v = k < count ? in[k] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(PK_FULL_MASK, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) scratch[warp] = incl;
        __syncthreads();
        int woff = 0, tot = 0;
        for (int w = 0; w < nw; ++w) {
            const int s = scratch[w];
            woff += w < warp ? s : 0;
            tot += s;
        }
        if (k < count) out[k] = carry + woff + incl - v;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[count] = carry;
    __syncthreads();
}

// Elementwise arithmetic rounded after every operation (never contracted
// into an FMA), as the reference's separate tensor operations round
// (lbfgs_torch_parallel.py:546-690).
__device__ __forceinline__ float pk_rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double pk_rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float pk_radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double pk_radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float pk_rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double pk_rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float pk_rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double pk_rdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float pk_rsqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double pk_rsqrt(double a) { return __dsqrt_rn(a); }

// Order-fixed vector reductions.  Element k belongs to group k / 128 and
// lane k % 32; thread (warp w, lane l) OWNS the elements of the groups
// g = w, w + nwarps, ... with lane l, and PK_OWN_LOOP visits exactly those.
// Vector updates written with the same ownership need no barrier before the
// next reduction.  pk_canon_sum adds each group's per-lane partial in k
// order, then the groups in order, then a fixed shuffle tree, so the sum
// depends on N alone, not on blockDim.  red: two buffers of 64 * ngroups
// entries, alternated by `flip` (one barrier per reduction: a thread can only
// write a buffer again after the next reduction's barrier, by which time every
// thread has finished reading it).  All threads call these and all get the
// result.
#define PK_CANON_GROUP 128
#define PK_OWN_LOOP(k, N)                                                                      \
    for (int _g = (int)(threadIdx.x >> 5); _g * PK_CANON_GROUP < (N); _g += (int)(blockDim.x >> 5)) \
        for (int k = _g * PK_CANON_GROUP + (int)(threadIdx.x & 31);                             \
             k < min((N), (_g + 1) * PK_CANON_GROUP); k += 32)

__host__ __device__ inline int pk_canon_groups(int N) { return (N + PK_CANON_GROUP - 1) / PK_CANON_GROUP; }

template <typename T>
__device__ __forceinline__ T* pk_canon_buf(int ng, T* red, int& flip)
{
    T* buf = red + (flip ? 64 * ng : 0);
    flip ^= 1;
    return buf;
}

// Second half of a canonical sum: barrier, the groups' per-lane partials in
// group order, then the shuffle tree.  buf holds ng * 32 partials.
template <typename T>
__device__ __forceinline__ T pk_canon_finish(const T* buf, int ng)
{
    const int lane = threadIdx.x & 31;
    __syncthreads();
    T r = T(0);
    for (int grp = 0; grp < ng; ++grp) r = pk_radd(r, buf[grp * 32 + lane]);
    return pk_warp_sum(r);
}

template <typename T, typename Get>
__device__ __forceinline__ T pk_canon_sum(int N, Get get, T* red, int& flip)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const int ng = pk_canon_groups(N);
    T* buf = pk_canon_buf(ng, red, flip);
    for (int grp = warp; grp < ng; grp += nw) {
        T s = T(0);
        const int end = min(N, (grp + 1) * PK_CANON_GROUP);
        for (int k = grp * PK_CANON_GROUP + lane; k < end; k += 32) s = pk_radd(s, get(k));
        buf[grp * 32 + lane] = s;
    }
    return pk_canon_finish(buf, ng);
}

// Two canonical sums with one barrier; each is bit-identical to its own
// pk_canon_sum.
template <typename T, typename Get>
__device__ __forceinline__ void pk_canon_sum2(int N, Get get, T* red, int& flip, T& r0, T& r1)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const int ng = pk_canon_groups(N);
    T* buf = pk_canon_buf(ng, red, flip);
    for (int grp = warp; grp < ng; grp += nw) {
        T s0 = T(0), s1 = T(0);
        const int end = min(N, (grp + 1) * PK_CANON_GROUP);
        for (int k = grp * PK_CANON_GROUP + lane; k < end; k += 32) {
            T a, b;
            get(k, a, b);
            s0 = pk_radd(s0, a);
            s1 = pk_radd(s1, b);
        }
        buf[grp * 32 + lane] = s0;
        buf[(ng + grp) * 32 + lane] = s1;
    }
    __syncthreads();
    T a = T(0), b = T(0);
    for (int grp = 0; grp < ng; ++grp) {
        a = pk_radd(a, buf[grp * 32 + lane]);
        b = pk_radd(b, buf[(ng + grp) * 32 + lane]);
    }
    r0 = pk_warp_sum(a);
    r1 = pk_warp_sum(b);
}

// Maxima of two element functions over the owned elements with one barrier
// (a maximum does not depend on the order).  Starts from 0: the callers
// reduce absolute values.
template <typename T, typename Get>
__device__ __forceinline__ void pk_canon_max2(int N, Get get, T* red, int& flip, T& r0, T& r1)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    T* buf = pk_canon_buf(pk_canon_groups(N), red, flip);
    T a = T(0), b = T(0);
    PK_OWN_LOOP(k, N) {
        T u, v;
        get(k, u, v);
        a = fmax(a, u);
        b = fmax(b, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(PK_FULL_MASK, a, o));
        b = fmax(b, __shfl_xor_sync(PK_FULL_MASK, b, o));
    }
    if (lane == 0) {
        buf[2 * warp] = a;
        buf[2 * warp + 1] = b;
    }
    __syncthreads();
    for (int w = 0; w < nw; ++w) {
        a = fmax(a, buf[2 * w]);
        b = fmax(b, buf[2 * w + 1]);
    }
    r0 = a;
    r1 = b;
}

// Both buffers of the canonical reductions (2 x 64 per group; a block of at
// most 32 warps fits the per-warp maxima in one buffer).
__host__ __device__ inline int pk_canon_red_len(int N) { return 2 * 64 * pk_canon_groups(N); }

// Bounded wrap of an angle difference into [-pi, pi], following the
// reference's subtract-2pi loop (pack_cuda_lut.py:289-293) in FP32.  Angles
// beyond +-64 pi are reduced with remainderf first so the loop stays short.
__device__ __forceinline__ float pk_wrap_angle(float t)
{
    const float PI = 3.14159265358979323846f;
    if (!(fabsf(t) < 64.0f * PI)) t = remainderf(t, 2.0f * PI);
    while (t > PI) t -= 2.0f * PI;
    while (t < -PI) t += 2.0f * PI;
    return t;
}
