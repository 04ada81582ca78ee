// crystal.cuh -- periodic (crystal) form of the pair cost: trees interact
// with the images of every tree under the lattice translations
// cx A + cy B, cx, cy in [-N, N] (overlap_ref_with_list_piece with
// use_crystal and overlap_list_total, pack_cuda.py:254-464; wrapper
// :1040-1183).
//
// The reference visits every ordered (ref tree i, tree j, cell c) from i and
// keeps i's gradient, then halves the total.  Here each unordered
// {i, j + c} with i < j is evaluated once with the gradients of both trees
// (its two ordered visits are the same geometry), and the images of a tree
// itself (j = i, c != 0) add half their value and no gradient, as the
// reference (:350-351) leaves their gradient out.  With only_self the sum
// keeps the self images only, at full weight (:455-460).  The centre cutoff
// applies to each image (:159-168).  Accumulation is fixed-point, so the
// result does not depend on the order of the work.
#pragma once
#include "common.cuh"
#include "cost.cuh"

__host__ __device__ inline size_t pk_crystal_smem_bytes(int n)
{
    return (size_t)n * (16 + 64 + 24) + 16 * 8 + 16 + 32 * 8;
}

// i <= j from the index p of the pair in row-major upper-triangular order.
__device__ __forceinline__ void pk_tri_decode(long long p, int n, int& i, int& j)
{
    const double b = 2.0 * n + 1.0;
    int r = (int)floor((b - sqrt(b * b - 8.0 * (double)p)) * 0.5);
    // row r starts at r n - r (r - 1) / 2; fix rounding at row boundaries
    auto start = [&](int row) { return (long long)row * n - (long long)row * (row - 1) / 2; };
    if (r < 0) r = 0;
    if (r > n - 1) r = n - 1;
    while (r > 0 && start(r) > p) --r;
    while (r < n - 1 && start(r + 1) <= p) ++r;
    i = r;
    j = r + (int)(p - start(r));
}

template <int MODE>
__global__ void __launch_bounds__(256) pk_crystal_kernel(const float* __restrict__ xyt, const float* __restrict__ axes,
                                                         int E, int n, int only_self, int np_,
                                                         float* __restrict__ cost, float* __restrict__ grad)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const int e = blockIdx.x;
    if (e >= E) return;
    const int T = blockDim.x;
    unsigned char* p = pk_smem;
    float4* pose = (float4*)p; p += (size_t)n * 16;
    float4* aabb = (float4*)p; p += (size_t)n * 64;
    long long* acc = (long long*)p; p += (size_t)n * 24;
    long long* redl = (long long*)p; p += 32 * 8;
    float2* piece = (float2*)p; p += 16 * 8;
    int* piece_nv = (int*)p;
    PkCostSmem sm{};
    sm.piece = piece;
    if (threadIdx.x < 16) piece[threadIdx.x] = c_geom.piece[threadIdx.x >> 2][threadIdx.x & 3];
    if (threadIdx.x < 4) piece_nv[threadIdx.x] = c_geom.piece_nv[threadIdx.x];
    __syncthreads();
    const float* X = xyt + (size_t)e * n * 3;
    for (int t = threadIdx.x; t < n; t += T) {
        const float x = X[3 * t], y = X[3 * t + 1], th = X[3 * t + 2];
        float s, c;
        sincosf(th, &s, &c);
        pose[t] = make_float4(x, y, c, s);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float2 V[4];
            pk_load_piece(sm, q, c, s, 0.f, 0.f, V);
            float4 bb = make_float4(V[0].x, V[0].x, V[0].y, V[0].y);
#pragma unroll
            for (int v = 1; v < 4; ++v) {
                bb.x = fminf(bb.x, V[v].x); bb.y = fmaxf(bb.y, V[v].x);
                bb.z = fminf(bb.z, V[v].y); bb.w = fmaxf(bb.w, V[v].y);
            }
            const float eps = 1e-6f;
            aabb[4 * t + q] = make_float4(bb.x - eps, bb.y + eps, bb.z - eps, bb.w + eps);
        }
        acc[3 * t] = acc[3 * t + 1] = acc[3 * t + 2] = 0;
    }
    __syncthreads();
    const float ax = axes[4 * e], ay = axes[4 * e + 1], bx = axes[4 * e + 2], by = axes[4 * e + 3];
    const int side = 2 * np_ + 1, ncell = side * side;
    const long long npairs = only_self ? (long long)n : (long long)n * (n + 1) / 2;
    const long long units = npairs * ncell;
    const float cutoff = c_geom.cutoff_sq;
    long long tot = 0;
    for (long long u = threadIdx.x; u < units; u += T) {
        const long long pr = u / ncell;
        const int cidx = (int)(u - pr * ncell);
        const int cx = cidx / side - np_, cy = cidx % side - np_;
        int i, j;
        if (only_self) { i = j = (int)pr; }
        else pk_tri_decode(pr, n, i, j);
        const bool self = i == j;
        if (self && cx == 0 && cy == 0) continue;
        const float4 A = pose[i], B = pose[j];
        const float sx = (float)cx * ax + (float)cy * bx, sy = (float)cx * ay + (float)cy * by;
        const float2 d = make_float2((B.x + sx) - A.x, (B.y + sy) - A.y);
        if (__fadd_rn(__fmul_rn(d.x, d.x), __fmul_rn(d.y, d.y)) > cutoff) continue;
        const float wself = only_self ? 1.f : 0.5f;
        for (int pi = 0; pi < 4; ++pi) {
            const float4 a = aabb[4 * i + pi];
            for (int pj = 0; pj < 4; ++pj) {
                const float4 b = aabb[4 * j + pj];
                if (a.y < b.x + d.x || b.y + d.x < a.x || a.w < b.z + d.y || b.w + d.y < a.z) continue;
                float2 P[4], Q[4];
                pk_load_piece(sm, pi, A.z, A.w, 0.f, 0.f, P);
                pk_load_piece(sm, pj, B.z, B.w, d.x, d.y, Q);
                const bool pt = piece_nv[pi] == 3, qt = piece_nv[pj] == 3;
                float val;
                float3 gi, gj;
                if (MODE == PK_PAIR_AREA) {
                    pk_piece_area_grad(P, pt, Q, qt, d, val, gi, gj);
                } else {
                    float sp;
                    pk_piece_sat_grad(P, pt, Q, qt, d, sp, gi, gj);
                    const float f = 2.0f * sp;
                    gi = make_float3(f * gi.x, f * gi.y, f * gi.z);
                    gj = make_float3(f * gj.x, f * gj.y, f * gj.z);
                    val = sp * sp;
                }
                if (self) {
                    tot += pk_to_fx(wself * val);
                } else if (val != 0.f || gi.x != 0.f || gi.y != 0.f || gi.z != 0.f) {
                    tot += pk_to_fx(val);
                    if (grad) {
                        pk_acc_add(acc, i, gi);
                        pk_acc_add(acc, j, gj);
                    }
                }
            }
        }
    }
    const long long wsum = pk_warp_sum(tot);
    if ((threadIdx.x & 31) == 0) redl[threadIdx.x >> 5] = wsum;
    __syncthreads();
    if (grad) {
        float* G = grad + (size_t)e * n * 3;
        for (int k = threadIdx.x; k < 3 * n; k += T) G[k] = (float)((double)acc[k] * PK_FX_INV);
    }
    if (threadIdx.x == 0) {
        long long s = 0;
        for (int w = 0; w < (T >> 5); ++w) s += redl[w];
        cost[e] = (float)((double)s * PK_FX_INV);
    }
}

extern "C" int pk_overlap_crystal(const float* xyt, int E, int n, int use_separation, const float* crystal_axes,
                                  int only_self, int n_periodic, float* cost, float* grad, void* stream)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (E < 0 || n < 0) return pk_fail(PK_EINVAL, "pk_overlap_crystal: negative size%s");
    if (E == 0) return PK_OK;
    if (n > PK_MAX_TREES) return pk_fail(PK_ERANGE, "pk_overlap_crystal: more than 1024 trees per instance%s");
    if (n_periodic < 0 || n_periodic > 16) return pk_fail(PK_EINVAL, "pk_overlap_crystal: N_periodic must be in [0, 16]%s");
    if (!cost || !crystal_axes || (!xyt && n > 0)) return pk_fail(PK_EINVAL, "pk_overlap_crystal: NULL pointer%s");
    const int T = 256;
    const size_t smem = pk_crystal_smem_bytes(n);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err;
    if (use_separation) {
        err = cudaFuncSetAttribute(pk_crystal_kernel<PK_PAIR_SEP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err == cudaSuccess)
            pk_crystal_kernel<PK_PAIR_SEP><<<E, T, smem, st>>>(xyt, crystal_axes, E, n, only_self, n_periodic, cost, grad);
    } else {
        err = cudaFuncSetAttribute(pk_crystal_kernel<PK_PAIR_AREA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err == cudaSuccess)
            pk_crystal_kernel<PK_PAIR_AREA><<<E, T, smem, st>>>(xyt, crystal_axes, E, n, only_self, n_periodic, cost, grad);
    }
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_overlap_crystal attribute");
    return pk_cuda_check(cudaGetLastError(), "pk_overlap_crystal launch");
}
