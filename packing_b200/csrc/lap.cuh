// lap.cuh -- batched linear assignment (Hungarian) and GA diversity kernels.
//
// One warp solves one N x N problem.  The reference runs the same
// shortest-augmenting-path Kuhn-Munkres on ONE thread per problem
// (lap_batch.py:62-165); here the N columns are spread over the 32 lanes
// (column j lives in lane j % 32, slot j / 32) so each Dijkstra step is a
// parallel slack update plus a warp argmin.  Every per-element float
// operation is the reference's, in the same order, and the argmin keeps the
// lowest column among equal slacks (the reference's strict '<' scan), so
// the assignment and the total are bit-identical to the sequential kernel.
#pragma once
#include "common.cuh"

#define PK_LAP_WARPS 4
// dynamic shared memory one CTA may hold on sm_100a (227 KB)
#define PK_LAP_SMEM_MAX ((size_t)227 * 1024)

// Warp-cooperative Hungarian for problem b.  u and rm are this warp's shared
// arrays of N entries.  costfn(row, col) returns C[row][col] for this
// problem (called for the lane's own columns only).  Returns false (and
// leaves rm at -1 for unmatched rows) if a step finds no finite slack.
// PREFETCH: load the next step's cost row as soon as the argmin names it,
// before the step's dual updates, so that an L2 load latency overlaps them
// (2048 x 100^2 from L2: 1.76 -> 1.27 ms).  Costs read from shared memory or
// computed in registers are fetched at the start of their step instead
// (earlier loads measured slower there).  Same operations, same results.
template <int CPL, bool PREFETCH, typename CostFn>
__device__ __forceinline__ bool pk_hungarian_warp(int N, float* u, int* rm, CostFn costfn)
{
    const int lane = threadIdx.x & 31;
    float v[CPL], minv[CPL];
    int p[CPL], cm[CPL];
    unsigned used = 0;
#pragma unroll
    for (int k = 0; k < CPL; ++k) { v[k] = 0.f; cm[k] = -1; }
    for (int r = lane; r < N; r += 32) { u[r] = 0.f; rm[r] = -1; }
    __syncwarp();
    for (int i = 0; i < N; ++i) {
#pragma unroll
        for (int k = 0; k < CPL; ++k) { minv[k] = 1e30f; p[k] = -1; }
        used = 0;
        int cur_row = i, cur_col = -1;
        float crow[CPL];   // the lane's costs in the row this step scans
#pragma unroll
        for (int k = 0; k < CPL; ++k) {
            const int j = lane + 32 * k;
            crow[k] = (PREFETCH && j < N) ? costfn(cur_row, j) : 0.f;
        }
        for (int step = 0; step < N; ++step) {
            if (!PREFETCH) {
#pragma unroll
                for (int k = 0; k < CPL; ++k) {
                    const int j = lane + 32 * k;
                    if (j < N && !((used >> k) & 1u)) crow[k] = costfn(cur_row, j);
                }
            }
            const float urow = u[cur_row];
            float lbv = 1e30f;
            int lbj = 0x7fffffff;
#pragma unroll
            for (int k = 0; k < CPL; ++k) {
                const int j = lane + 32 * k;
                if (j < N && !((used >> k) & 1u)) {
                    float red = crow[k] - urow;
                    red = red - v[k];
                    if (red < minv[k]) { minv[k] = red; p[k] = cur_row; }
                    if (minv[k] < lbv) { lbv = minv[k]; lbj = j; }
                }
            }
            // Warp argmin in two redux.sync steps: the smallest slack as an
            // order-preserving unsigned key (-0 folded into +0, so equal
            // floats give equal keys), then the lowest column among the
            // lanes holding it.  Slacks are never NaN: a NaN cost fails the
            // '<' above and leaves minv untouched.
            {
                const unsigned bits = __float_as_uint(__fadd_rn(lbv, 0.f));
                const unsigned key = (bits & 0x80000000u) ? ~bits : (bits | 0x80000000u);
                const unsigned kmin = __reduce_min_sync(PK_FULL_MASK, key);
                lbj = (int)__reduce_min_sync(PK_FULL_MASK, key == kmin ? (unsigned)lbj : 0xffffffffu);
            }
            if (lbj == 0x7fffffff) return false;   // no finite slack: infeasible input
            // the winning lane's own slack, bit for bit
            const float delta = __shfl_sync(PK_FULL_MASK, lbv, lbj & 31);
            // the row matched to the chosen column is the next step's row
            const int owner = lbj & 31, slot = lbj >> 5;
            int nxt = -1;
#pragma unroll
            for (int k = 0; k < CPL; ++k)
                if (k == slot && lane == owner) nxt = cm[k];
            const int next_row = __shfl_sync(PK_FULL_MASK, nxt, owner);
            const unsigned used_next = used | (lane == owner ? 1u << slot : 0u);
            if (PREFETCH && next_row >= 0) {
#pragma unroll
                for (int k = 0; k < CPL; ++k) {
                    const int j = lane + 32 * k;
                    if (j < N && !((used_next >> k) & 1u)) crow[k] = costfn(next_row, j);
                }
            }
#pragma unroll
            for (int k = 0; k < CPL; ++k) {
                const int j = lane + 32 * k;
                if (j < N) {
                    if ((used >> k) & 1u) {
                        u[cm[k]] += delta;
                        v[k] -= delta;
                    } else {
                        minv[k] -= delta;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) u[i] += delta;
            __syncwarp();
            used = used_next;
            cur_col = lbj;
            cur_row = next_row;
            if (cur_row < 0) break;
        }
        // flip the alternating path (lap_batch.py:157-163)
        for (int guard = 0; cur_col >= 0 && guard <= N; ++guard) {
            const int owner = cur_col & 31, slot = cur_col >> 5;
            int prow = 0;
#pragma unroll
            for (int k = 0; k < CPL; ++k)
                if (k == slot && lane == owner) prow = p[k];
            prow = __shfl_sync(PK_FULL_MASK, prow, owner);
            const int pcol = rm[prow];
            __syncwarp();
#pragma unroll
            for (int k = 0; k < CPL; ++k)
                if (k == slot && lane == owner) cm[k] = prow;
            if (lane == 0) rm[prow] = cur_col;
            __syncwarp();
            cur_col = pcol;
        }
    }
    return true;
}

// One warp per problem, PK_LAP_WARPS problems per CTA.  The minimum of one
// CTA per SM in the launch bounds lets ptxas give every CPL the registers it
// needs (up to 88, no spills); without it, it capped CPL = 5..7 at 64 with
// spills and scheduled the rest tighter (2048 x 100^2: 1.28 -> 1.04 ms with
// it, 512 x 200^2: 3.56 -> 2.55 ms).
template <int CPL>
__global__ void __launch_bounds__(32 * PK_LAP_WARPS, 1)
pk_hungarian_kernel(const float* __restrict__ C, int B, int N, int* __restrict__ row_match,
                    float* __restrict__ total, int* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * PK_LAP_WARPS + warp;
    if (b >= B) return;
    float* u = (float*)pk_smem + (size_t)warp * 2 * N;
    int* rm = (int*)(u + N);
    const float* Cb = C + (size_t)b * N * N;
    const bool ok = pk_hungarian_warp<CPL, true>(N, u, rm, [&](int r, int j) { return __ldg(Cb + (size_t)r * N + j); });
    __syncwarp();
    for (int r = lane; r < N; r += 32) row_match[(size_t)b * N + r] = ok ? rm[r] : -1;
    if (lane == 0) {
        // compute_costs (lap_batch.py:173-196): sequential float sum over rows
        float t = 0.f;
        if (ok) {
            for (int r = 0; r < N; ++r) {
                const int col = rm[r];
                if (col >= 0 && col < N) t += __ldg(Cb + (size_t)r * N + col);
            }
        } else {
            t = __int_as_float(0x7fc00000);
        }
        total[b] = t;
        if (status) status[b] = ok ? 0 : 1;
    }
}

// The same solver with the problem's N x N costs copied into shared memory
// first.  Each Dijkstra step reads one cost row, and which row is only known
// when the previous step ends, so every step waits a full load latency: from
// shared memory that wait is a few tens of cycles instead of an L2 round trip.
// One warp per CTA; the CTAs beyond those resident start as others finish,
// which balances problems of very different step counts.
template <int CPL>
__global__ void __launch_bounds__(32)
pk_hungarian_smem_kernel(const float* __restrict__ C, int B, int N, int* __restrict__ row_match,
                         float* __restrict__ total, int* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const int lane = threadIdx.x;
    const int b = blockIdx.x;
    if (b >= B) return;
    const size_t nn = (size_t)N * N;
    float* Cs = (float*)pk_smem;
    float* u = Cs + ((nn + 3) & ~(size_t)3);
    int* rm = (int*)(u + N);
    const float* Cb = C + (size_t)b * nn;
    if ((((uintptr_t)Cb) & 15) == 0) {
        const size_t n4 = nn >> 2;
        const float4* src = (const float4*)Cb;
        float4* dst = (float4*)Cs;
#pragma unroll 8
        for (size_t k = lane; k < n4; k += 32) dst[k] = __ldg(src + k);
        for (size_t k = (n4 << 2) + lane; k < nn; k += 32) Cs[k] = __ldg(Cb + k);
    } else {
        for (size_t k = lane; k < nn; k += 32) Cs[k] = __ldg(Cb + k);
    }
    __syncwarp();
    const bool ok = pk_hungarian_warp<CPL, false>(N, u, rm, [&](int r, int j) { return Cs[r * N + j]; });
    __syncwarp();
    for (int r = lane; r < N; r += 32) row_match[(size_t)b * N + r] = ok ? rm[r] : -1;
    if (lane == 0) {
        float t = 0.f;
        if (ok) {
            for (int r = 0; r < N; ++r) {
                const int col = rm[r];
                if (col >= 0 && col < N) t += Cs[r * N + col];
            }
        } else {
            t = __int_as_float(0x7fc00000);
        }
        total[b] = t;
        if (status) status[b] = ok ? 0 : 1;
    }
}

// Shared memory of the staged solver for N: the matrix (rounded up to whole
// float4s), u and the row matches.
static size_t pk_lap_smem_bytes(int N)
{
    return (((size_t)N * N + 3) & ~(size_t)3) * 4 + (size_t)N * 8;
}

// Launches the staged solver when every problem can be resident at once
// (staging trades concurrency for latency: with fewer problems in flight
// than the SMs could hold from L2, the L2 form finishes first).  Returns 1
// if launched, 0 if the L2 form should run, or a status on failure.
template <int CPL>
static int pk_lap_try_smem(const float* C, int B, int N, int* rm, float* tot, int* status, cudaStream_t st)
{
    const size_t ssm = pk_lap_smem_bytes(N);
    if (ssm > PK_LAP_SMEM_MAX) return 0;
    cudaError_t err = cudaFuncSetAttribute(pk_hungarian_smem_kernel<CPL>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm);
    int dev = 0, sms = 0, per_sm = 0;
    if (err == cudaSuccess) err = cudaGetDevice(&dev);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (err == cudaSuccess)
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk_hungarian_smem_kernel<CPL>, 32, ssm);
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_lap_solve occupancy");
    if ((long long)per_sm * sms < (long long)B) return 0;
    pk_hungarian_smem_kernel<CPL><<<B, 32, ssm, st>>>(C, B, N, rm, tot, status);
    const int rc = pk_cuda_check(cudaGetLastError(), "pk_lap_solve launch");
    return rc == PK_OK ? 1 : rc;
}

static int pk_lap_dispatch(const float* C, int B, int N, int* rm, float* tot, int* status, cudaStream_t st)
{
    const int cpl = (N + 31) / 32;
    int staged = 0;
    switch (cpl) {
#define PK_L(K) case K: staged = pk_lap_try_smem<K>(C, B, N, rm, tot, status, st); break;
        PK_L(1) PK_L(2) PK_L(3) PK_L(4) PK_L(5) PK_L(6) PK_L(7) PK_L(8)
#undef PK_L
        default: return pk_fail(PK_ERANGE, "pk_lap_solve: N beyond 256%s");
    }
    if (staged == 1) return PK_OK;
    if (staged != 0) return staged;
    const dim3 grid((B + PK_LAP_WARPS - 1) / PK_LAP_WARPS), block(32 * PK_LAP_WARPS);
    const size_t smem = (size_t)PK_LAP_WARPS * 2 * N * 4;
    switch (cpl) {
#define PK_L(K) case K: pk_hungarian_kernel<K><<<grid, block, smem, st>>>(C, B, N, rm, tot, status); break;
        PK_L(1) PK_L(2) PK_L(3) PK_L(4) PK_L(5) PK_L(6) PK_L(7) PK_L(8)
#undef PK_L
        default: return pk_fail(PK_ERANGE, "pk_lap_solve: N beyond 256%s");
    }
    return pk_cuda_check(cudaGetLastError(), "pk_lap_solve launch");
}

extern "C" int pk_lap_solve(const float* C, int B, int N, int* row_match, float* total, int* status,
                            void* stream)
{
    if (B < 0 || N < 0) return pk_fail(PK_EINVAL, "pk_lap_solve: negative size%s");
    if (N > PK_MAX_LAP_N) return pk_fail(PK_ERANGE, "pk_lap_solve: N beyond 256%s");
    if (B == 0) return PK_OK;
    if (N == 0) {
        // empty assignments: totals are 0 (lap_batch.py:173-196 with N = 0)
        return pk_cuda_check(cudaMemsetAsync(total, 0, sizeof(float) * B, (cudaStream_t)stream),
                             "pk_lap_solve memset");
    }
    if (!C || !row_match || !total) return pk_fail(PK_EINVAL, "pk_lap_solve: NULL pointer%s");
    return pk_lap_dispatch(C, B, N, row_match, total, status, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// GA diversity: 8 symmetry transforms of the reference packing
// (kaggle_support.py:2061-2071), cost sqrt(dx^2 + dy^2 + wrap(dtheta)^2)
// (:2105-2112), one LAP per transform, minimum over transforms (:2126).
// The reference materialises a (8 * N_pop * N_ref, N, N) tensor and calls
// solve_lap_batch; here each CTA of 8 warps handles one (pop, ref) pair,
// warp t solving transform t with its cost rows generated on the fly, and
// the minimum is taken in shared memory.  No intermediate tensor.
// ---------------------------------------------------------------------------

// Transformed reference pose (kaggle_support.py:2080-2099), FP32.
__device__ __forceinline__ float3 pk_div_transform(float x, float y, float th, int t)
{
    const float PI = 3.14159265358979323846f;
    if (t >= 4) { y = -y; th = PI - th; }
    const int r = t & 3;
    const float ca[4] = {1.f, 0.f, -1.f, 0.f};
    const float sa[4] = {0.f, 1.f, 0.f, -1.f};
    const float ang[4] = {0.f, 1.5707963267948966f, 3.141592653589793f, 4.71238898038469f};
    float nx = x, ny = y;
    if (r != 0) {
        // explicit roundings: the fused and the materialised paths must agree bit for bit
        nx = __fsub_rn(__fmul_rn(x, ca[r]), __fmul_rn(y, sa[r]));
        ny = __fadd_rn(__fmul_rn(x, sa[r]), __fmul_rn(y, ca[r]));
        th = __fadd_rn(th, ang[r]);
    }
    // remainder(th + pi, 2 pi) - pi, result in [-pi, pi)
    float m = fmodf(__fadd_rn(th, PI), 2.f * PI);
    if (m < 0.f) m = __fadd_rn(m, 2.f * PI);
    return make_float3(nx, ny, __fsub_rn(m, PI));
}

// fmodf(x, 2 pi) (2 pi rounded to float), exactly: |x| < 2 pi is its own
// remainder, and for 2 pi <= |x| < 4 pi the remainder |x| - 2 pi is exact
// (Sterbenz) and takes the sign of x; anything else goes to fmodf.  The
// cost rows of the fused diversity solver are generated inside its Dijkstra
// steps, where the general fmodf was most of a step's arithmetic.
__device__ __forceinline__ float pk_fmod_2pi(float x)
{
    const float T = 2.f * 3.14159265358979323846f;
    const float ax = fabsf(x);
    if (ax < T) return x;
    if (ax < 2.f * T) return copysignf(__fsub_rn(ax, T), x);
    return fmodf(x, T);
}

__device__ __forceinline__ float pk_div_cost(float px, float py, float pt, float3 r)
{
    const float PI = 3.14159265358979323846f;
    const float dx = __fsub_rn(px, r.x), dy = __fsub_rn(py, r.y);
    float dt = pk_fmod_2pi(__fadd_rn(__fsub_rn(pt, r.z), PI));
    if (dt < 0.f) dt = __fadd_rn(dt, 2.f * PI);
    dt = __fsub_rn(dt, PI);
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dt, dt)));
}

// Dense cost matrices of every (transform, pop, ref) problem, in the
// reference's stacking order (transform, pop, ref) -> (N, N), for checking
// the fused kernel and for callers that want the matrices.
__global__ void pk_diversity_costs_kernel(const float* __restrict__ pop, const float* __restrict__ ref, int Np,
                                          int Nr, int n, int ntf, float* __restrict__ out)
{
    const size_t total = (size_t)ntf * Np * Nr * n * n;
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < total; w += (size_t)gridDim.x * blockDim.x) {
        const int col = (int)(w % n);
        const int row = (int)((w / n) % n);
        const size_t prob = w / ((size_t)n * n);
        const int r = (int)(prob % Nr), p = (int)((prob / Nr) % Np), t = (int)(prob / ((size_t)Np * Nr));
        const float* R = ref + ((size_t)r * n + col) * 3;
        const float* P = pop + ((size_t)p * n + row) * 3;
        out[w] = pk_div_cost(P[0], P[1], P[2], pk_div_transform(R[0], R[1], R[2], t));
    }
}

template <int CPL>
__global__ void __launch_bounds__(256)
pk_diversity_lap_kernel(const float* __restrict__ pop, const float* __restrict__ ref, int Np, int Nr, int n,
                        int ntf, float* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pr = blockIdx.x;
    const int p = pr / Nr, r = pr % Nr;
    float* s_tot = (float*)pk_smem;                       // [8]
    float* s_pop = s_tot + 8;                             // [3n]
    float* base = s_pop + 3 * n;
    const float* P = pop + (size_t)p * n * 3;
    for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) s_pop[k] = P[k];
    __syncthreads();
    if (warp < ntf) {
        float* u = base + (size_t)warp * 2 * n;
        int* rm = (int*)(u + n);
        // this lane's transformed reference columns
        float3 rc[CPL];
        const float* R = ref + (size_t)r * n * 3;
#pragma unroll
        for (int k = 0; k < CPL; ++k) {
            const int j = lane + 32 * k;
            rc[k] = j < n ? pk_div_transform(R[3 * j], R[3 * j + 1], R[3 * j + 2], warp) : make_float3(0, 0, 0);
        }
        const bool ok = pk_hungarian_warp<CPL, false>(n, u, rm, [&](int row, int j) {
            float3 c = rc[0];
#pragma unroll
            for (int k = 1; k < CPL; ++k)
                if ((j >> 5) == k) c = rc[k];
            return pk_div_cost(s_pop[3 * row], s_pop[3 * row + 1], s_pop[3 * row + 2], c);
        });
        __syncwarp();
        if (lane == 0) {
            float t = 0.f;
            if (ok) {
                for (int row = 0; row < n; ++row) {
                    const int col = rm[row];
                    const float3 c = pk_div_transform(R[3 * col], R[3 * col + 1], R[3 * col + 2], warp);
                    t += pk_div_cost(s_pop[3 * row], s_pop[3 * row + 1], s_pop[3 * row + 2], c);
                }
            } else {
                t = __int_as_float(0x7fc00000);
            }
            s_tot[warp] = t;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = s_tot[0];
        for (int t = 1; t < ntf; ++t) m = fminf(m, s_tot[t]);
        out[pr] = m;
    }
}

// Shared argument checks of the diversity entry points: sizes, the (pop, ref)
// pair count of a one-CTA-per-pair grid (computed in 64 bits), and the
// pointers of a launch that has work.
static int pk_diversity_args(const char* who, const float* pop, const float* ref, int Np, int Nr, int n,
                             const float* out)
{
    if (Np < 0 || Nr < 0 || n < 0) {
        snprintf(g_pk_err, sizeof(g_pk_err), "%s: negative size", who);
        return PK_EINVAL;
    }
    if ((long long)Np * (long long)Nr > 0x7fffffffLL) {
        snprintf(g_pk_err, sizeof(g_pk_err), "%s: Np * Nr = %lld pairs exceeds the grid limit 2^31 - 1", who,
                 (long long)Np * (long long)Nr);
        return PK_ERANGE;
    }
    if ((long long)Np * Nr > 0 && (!out || (n > 0 && (!pop || !ref)))) {
        snprintf(g_pk_err, sizeof(g_pk_err), "%s: NULL pointer", who);
        return PK_EINVAL;
    }
    return PK_OK;
}

extern "C" int pk_diversity_costs(const float* pop, const float* ref, int Np, int Nr, int n, int transform,
                                  float* out, void* stream)
{
    int rc = pk_diversity_args("pk_diversity_costs", pop, ref, Np, Nr, n, out);
    if (rc) return rc;
    const int ntf = transform ? 8 : 1;
    const size_t total = (size_t)ntf * Np * Nr * n * n;
    if (total == 0) return PK_OK;
    const int blocks = (int)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
    pk_diversity_costs_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(pop, ref, Np, Nr, n, ntf, out);
    return pk_cuda_check(cudaGetLastError(), "pk_diversity_costs launch");
}

extern "C" int pk_diversity_matrix(const float* pop, const float* ref, int Np, int Nr, int n, int transform,
                                   float* out, void* stream)
{
    int rc = pk_diversity_args("pk_diversity_matrix", pop, ref, Np, Nr, n, out);
    if (rc) return rc;
    if (n > PK_MAX_LAP_N) return pk_fail(PK_ERANGE, "pk_diversity_matrix: more than 256 trees%s");
    if (Np == 0 || Nr == 0) return PK_OK;
    if (n == 0) return pk_cuda_check(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)Np * Nr, (cudaStream_t)stream),
                                     "pk_diversity_matrix memset");
    const int ntf = transform ? 8 : 1;
    const int cpl = (n + 31) / 32;
    const size_t smem = 8 * 4 + (size_t)3 * n * 4 + (size_t)8 * 2 * n * 4;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaSuccess;
    switch (cpl) {
#define PK_D(K)                                                                                        \
    case K:                                                                                            \
        err = cudaFuncSetAttribute(pk_diversity_lap_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                   (int)smem);                                                         \
        if (err == cudaSuccess) pk_diversity_lap_kernel<K><<<Np * Nr, 256, smem, st>>>(pop, ref, Np, Nr, n, ntf, out); \
        break;
        PK_D(1) PK_D(2) PK_D(3) PK_D(4) PK_D(5) PK_D(6) PK_D(7) PK_D(8)
#undef PK_D
        default: return pk_fail(PK_ERANGE, "pk_diversity_matrix: more than 256 trees%s");
    }
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_diversity_matrix attribute");
    return pk_cuda_check(cudaGetLastError(), "pk_diversity_matrix launch");
}

// diversity_shortcut_kernel (lap_batch.py:216-331): transform of the
// reference by (cos_a, sin_a, mirror), then for every population tree the
// nearest transformed reference tree; sum of those distances.  One CTA per
// (pop, ref) pair; the sum runs over trees in index order like the reference.
__global__ void pk_diversity_shortcut_kernel(const float* __restrict__ pop, const float* __restrict__ ref, int Np,
                                             int Nr, int n, float cos_a, float sin_a, int mirror,
                                             float* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    float* rx = (float*)pk_smem;
    float* ry = rx + n;
    float* rt = ry + n;
    float* part = rt + n;
    const float PI = 3.14159265358979323846f, TWO_PI = 2.0f * PI;
    const int b = blockIdx.x;
    const int pi = b / Nr, ri = b % Nr;
    const float* P = pop + (size_t)pi * n * 3;
    const float* R = ref + (size_t)ri * n * 3;
    const float rot = atan2f(sin_a, cos_a);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float x = R[3 * k], y = R[3 * k + 1], t = R[3 * k + 2];
        if (mirror) { y = -y; t = PI - t; }
        const float xr = x * cos_a - y * sin_a, yr = x * sin_a + y * cos_a;
        float tr = t + rot;
        tr = fmodf(tr + PI, TWO_PI);
        if (tr < 0) tr += TWO_PI;
        tr -= PI;
        rx[k] = xr; ry[k] = yr; rt[k] = tr;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const float px = P[3 * k], py = P[3 * k + 1], pt = P[3 * k + 2];
        float best = 1e30f;
        for (int j = 0; j < n; ++j) {
            const float dx = px - rx[j], dy = py - ry[j];
            float dt = pt - rt[j];
            dt = fmodf(dt + PI, TWO_PI);
            if (dt < 0) dt += TWO_PI;
            dt -= PI;
            const float sq = dx * dx + dy * dy + dt * dt;
            if (sq < best) best = sq;
        }
        part[k] = sqrtf(best);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < n; ++k) t += part[k];
        out[b] = t;
    }
}

extern "C" int pk_diversity_shortcut(const float* pop, const float* ref, int Np, int Nr, int n, float cos_a,
                                     float sin_a, int mirror, float* out, void* stream)
{
    int rc = pk_diversity_args("pk_diversity_shortcut", pop, ref, Np, Nr, n, out);
    if (rc) return rc;
    if (n > 3072) return pk_fail(PK_ERANGE, "pk_diversity_shortcut: more than 3072 trees (48 KB of shared memory)%s");
    if (Np == 0 || Nr == 0) return PK_OK;
    if (n == 0) return pk_cuda_check(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)Np * Nr, (cudaStream_t)stream),
                                     "pk_diversity_shortcut memset");
    const int T = n < 32 ? 32 : (n > 256 ? 256 : ((n + 31) / 32) * 32);
    pk_diversity_shortcut_kernel<<<Np * Nr, T, (size_t)4 * n * 4, (cudaStream_t)stream>>>(pop, ref, Np, Nr, n, cos_a,
                                                                                         sin_a, mirror, out);
    return pk_cuda_check(cudaGetLastError(), "pk_diversity_shortcut launch");
}
