// wolfe.cuh -- batched strong-Wolfe line search for the drop-in L-BFGS
// (_strong_wolfe_batched and _cubic_interpolate_batch,
// lbfgs_torch_parallel.py:30-407; called from the main loop at :613-624).
//
// The search is a per-system state machine split into phases at the points
// where the reference evaluates the objective: the host runs the phases and,
// between them, calls the caller's objective on exactly the rows the
// reference passes to it (all systems of the search first, then the systems
// still active), so the objective sees the same sequence of calls.  One CTA
// per system; vector work uses the order-fixed reductions of common.cuh.
// Every rule follows the reference as written, including its bookkeeping:
// after an interpolation the previous step becomes the new trial step
// (:218-221); the zoom starts with low_pos = 1 when bracket_f[0] <= f[1]
// (:257-258); a system that runs out of evaluations in the bracketing
// phase keeps bracket_gtd from before (:236-246); one evaluation counter is
// shared by the batch (:146, :229, :308).
#pragma once
#include "common.cuh"

template <typename F>
struct PkWolfeState {
    const F *x, *d, *g, *f;          // point, direction, gradient, loss of the outer iteration
    F* gtd;                          // g . d (computed by the init phase)
    F* t;                            // trial step; the accepted step at the end
    F *x_new, *g_new, *f_new, *gtd_new;
    F *g_prev, *f_prev, *gtd_prev, *t_prev;
    F *bg, *bt, *bf, *bgtd;          // bracket: gradients (M, 2, N); steps, losses, g . d (M, 2)
    F *d_norm, *t_new;
    int *bsize, *done, *active, *low, *insuf, *evals, *in_ls, *flag;
    int M, N;
};

// torch.clamp / min / max semantics: a NaN operand gives NaN.
template <typename F>
__device__ __forceinline__ F pk_nmax(F a, F b) { return (a != a || b != b) ? (a != a ? a : b) : (a > b ? a : b); }
template <typename F>
__device__ __forceinline__ F pk_nmin(F a, F b) { return (a != a || b != b) ? (a != a ? a : b) : (a < b ? a : b); }

// _cubic_interpolate_batch (:30-66) for one system: the reference's
// operations in its order, each rounded on its own (no FMA contraction).
template <typename F>
__device__ __forceinline__ F pk_cubic_interpolate(F x1, F f1, F g1, F x2, F f2, F g2, F lo, F hi)
{
    const F d1 = pk_rsub(pk_radd(g1, g2), pk_rdiv(pk_rmul((F)3, pk_rsub(f1, f2)), pk_rsub(x1, x2)));
    const F d2sq = pk_rsub(pk_rmul(d1, d1), pk_rmul(g1, g2));
    const F d2 = pk_rsqrt(d2sq > (F)0 ? d2sq : (F)0);
    F mp;
    if (x1 <= x2)
        mp = pk_rsub(x2, pk_rmul(pk_rsub(x2, x1), pk_rdiv(pk_rsub(pk_radd(g2, d2), d1),
                                                         pk_radd(pk_rsub(g2, g1), pk_rmul((F)2, d2)))));
    else
        mp = pk_rsub(x1, pk_rmul(pk_rsub(x1, x2), pk_rdiv(pk_rsub(pk_radd(g1, d2), d1),
                                                         pk_radd(pk_rsub(g1, g2), pk_rmul((F)2, d2)))));
    if (d2sq >= (F)0) return pk_nmin(pk_nmax(mp, lo), hi);
    return pk_rdiv(pk_radd(lo, hi), (F)2.0);
}

// f + c1 t gtd, rounded as the reference's tensor expression (:150, :311)
template <typename F>
__device__ __forceinline__ F pk_armijo_bound(F f, F c1, F t, F gtd)
{
    return pk_radd(f, pk_rmul(pk_rmul(c1, t), gtd));
}

template <typename F>
__device__ __forceinline__ void pk_wolfe_set_slot(const PkWolfeState<F>& s, int b, int slot, F t, F f, const F* g,
                                                  F gtd, bool set_gtd)
{
    const int N = s.N;
    F* dst = s.bg + ((size_t)b * 2 + slot) * N;
    PK_OWN_LOOP(k, N) dst[k] = g[k];
    if (threadIdx.x == 0) {
        s.bt[2 * b + slot] = t;
        s.bf[2 * b + slot] = f;
        if (set_gtd) s.bgtd[2 * b + slot] = gtd;
    }
}

// Phase 0 (:117-140): start of the search, first trial point x + t d.
template <typename F>
__global__ void pk_wolfe_init_kernel(PkWolfeState<F> s)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    F* red = (F*)pk_smem;
    int flip = 0;
    const int b = blockIdx.x, N = s.N;
    if (!s.in_ls[b]) {
        // not searched this time: no flag of an earlier search may survive
        if (threadIdx.x == 0) { s.active[b] = 0; s.done[b] = 0; s.bsize[b] = 0; }
        return;
    }
    const F* d = s.d + (size_t)b * N;
    const F* g = s.g + (size_t)b * N;
    const F* x = s.x + (size_t)b * N;
    F dn, unused;
    pk_canon_max2<F>(N, [&](int k, F& u, F& v) { u = (F)fabs(d[k]); v = (F)0; }, red, flip, dn, unused);
    const F gtd = pk_canon_sum<F>(N, [&](int k) { return pk_rmul(g[k], d[k]); }, red, flip);
    const F t = s.t[b];
    F* xn = s.x_new + (size_t)b * N;
    F* gp = s.g_prev + (size_t)b * N;
    PK_OWN_LOOP(k, N) {
        xn[k] = pk_radd(x[k], pk_rmul(t, d[k]));
        gp[k] = g[k];
    }
    if (threadIdx.x == 0) {
        s.gtd[b] = gtd;
        s.d_norm[b] = dn;
        s.t_prev[b] = 0;
        s.f_prev[b] = s.f[b];
        s.gtd_prev[b] = gtd;
        for (int q = 0; q < 2; ++q) s.bt[2 * b + q] = s.bf[2 * b + q] = s.bgtd[2 * b + q] = 0;
        s.bsize[b] = 0;
        s.done[b] = 0;
        s.active[b] = 1;
        s.insuf[b] = 0;
        s.evals[b] = 1;
        s.low[b] = 0;
        s.t_new[b] = 0;
    }
}

// After an evaluation (:134, :229-230, :307-308): g_new . d of the rows just
// evaluated (all systems of the search first, then the active ones) and
// their evaluation count.
template <typename F>
__global__ void pk_wolfe_after_eval_kernel(PkWolfeState<F> s, int first)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    F* red = (F*)pk_smem;
    int flip = 0;
    const int b = blockIdx.x, N = s.N;
    if (!s.in_ls[b] || (!first && !s.active[b])) return;
    const F* gn = s.g_new + (size_t)b * N;
    const F* d = s.d + (size_t)b * N;
    const F gtd = pk_canon_sum<F>(N, [&](int k) { return pk_rmul(gn[k], d[k]); }, red, flip);
    if (threadIdx.x == 0) {
        s.gtd_new[b] = gtd;
        if (!first) s.evals[b] += 1;
    }
}

// One pass of the bracketing loop up to its evaluation (:146-221): the
// Armijo / non-decrease, curvature and positive-slope tests, then for the
// systems still searching the next trial step by cubic interpolation and the
// "previous" state.  Sets *flag if any system is still searching.
template <typename F>
__global__ void pk_wolfe_bracket_kernel(PkWolfeState<F> s, int ls_iter, F c1, F c2)
{
    const int b = blockIdx.x, N = s.N;
    if (!s.in_ls[b]) return;
    __shared__ int act_s;
    const F f = s.f[b], gtd = s.gtd[b], t = s.t[b];
    const F fn = s.f_new[b], gn = s.gtd_new[b];
    const F tp = s.t_prev[b], fp = s.f_prev[b], gp = s.gtd_prev[b];
    int act = s.active[b];
    int size = s.bsize[b];
    const F* gnew = s.g_new + (size_t)b * N;
    const F* gprev = s.g_prev + (size_t)b * N;
    if (act) {
        const bool armijo_fail = fn > pk_armijo_bound(f, c1, t, gtd);
        const bool not_decreasing = ls_iter > 1 && fn >= fp;
        if ((armijo_fail || not_decreasing) && size == 0) {
            pk_wolfe_set_slot(s, b, 0, tp, fp, gprev, gp, true);
            pk_wolfe_set_slot(s, b, 1, t, fn, gnew, gn, true);
            size = 2;
            act = 0;
        }
    }
    if (act && (F)fabs(gn) <= pk_rmul(-c2, gtd)) {
        pk_wolfe_set_slot(s, b, 0, t, fn, gnew, gn, false);
        size = 1;
        if (threadIdx.x == 0) s.done[b] = 1;
        act = 0;
    }
    if (act && gn >= (F)0) {
        pk_wolfe_set_slot(s, b, 0, tp, fp, gprev, gp, true);
        pk_wolfe_set_slot(s, b, 1, t, fn, gnew, gn, true);
        size = 2;
        act = 0;
    }
    F tt = t;
    if (act)
        tt = pk_cubic_interpolate<F>(tp, fp, gp, t, fn, gn, pk_radd(t, pk_rmul((F)0.01, pk_rsub(t, tp))),
                                     pk_rmul(t, (F)10));
    if (threadIdx.x == 0) act_s = act;
    __syncthreads();   // slot copies read g_prev; it is overwritten below
    F* gpw = s.g_prev + (size_t)b * N;
    PK_OWN_LOOP(k, N) gpw[k] = gnew[k];
    if (act) {
        const F* x = s.x + (size_t)b * N;
        const F* d = s.d + (size_t)b * N;
        F* xn = s.x_new + (size_t)b * N;
        PK_OWN_LOOP(k, N) xn[k] = pk_radd(x[k], pk_rmul(tt, d[k]));
    }
    if (threadIdx.x == 0) {
        s.t[b] = tt;
        s.t_prev[b] = tt;
        s.f_prev[b] = fn;
        s.gtd_prev[b] = gn;
        s.bsize[b] = size;
        s.active[b] = act_s;
        if (act_s) atomicOr(s.flag, 1);
    }
}

// Systems that used up the evaluations without a bracket (:236-246), then
// the zoom's start (:250-258).
template <typename F>
__global__ void pk_wolfe_zoom_init_kernel(PkWolfeState<F> s, int out_of_evals)
{
    const int b = blockIdx.x;
    if (!s.in_ls[b]) return;
    int size = s.bsize[b];
    if (out_of_evals && size == 0) {
        pk_wolfe_set_slot(s, b, 0, (F)0, s.f[b], s.g + (size_t)b * s.N, (F)0, false);
        pk_wolfe_set_slot(s, b, 1, s.t[b], s.f_new[b], s.g_new + (size_t)b * s.N, (F)0, false);
        size = 2;
    }
    if (threadIdx.x == 0) {
        s.bsize[b] = size;
        s.active[b] = size == 2 && !s.done[b];
        s.low[b] = s.bf[2 * b] <= s.bf[2 * b + 1] ? 1 : 0;
        s.insuf[b] = 0;
    }
}

// One zoom pass up to its evaluation (:260-305): bracket-width stop, cubic
// trial inside the bracket, the insufficient-progress adjustment, the trial
// point.  Sets *flag if any system is still zooming.
template <typename F>
__global__ void pk_wolfe_zoom_pre_kernel(PkWolfeState<F> s, F tol_change)
{
    const int b = blockIdx.x, N = s.N;
    if (!s.in_ls[b]) return;
    const F b0 = s.bt[2 * b], b1 = s.bt[2 * b + 1];
    const F width = (F)fabs(pk_rsub(b1, b0));
    int act = s.active[b];
    if (act && pk_rmul(width, s.d_norm[b]) < tol_change) act = 0;
    const F bmin = pk_nmin(b0, b1), bmax = pk_nmax(b0, b1);
    F tn = 0;
    if (act)
        tn = pk_cubic_interpolate<F>(b0, s.bf[2 * b], s.bgtd[2 * b], b1, s.bf[2 * b + 1], s.bgtd[2 * b + 1], bmin,
                                     bmax);
    const F eps = pk_rmul((F)0.1, width);
    const F dist = pk_nmin(pk_rsub(bmax, tn), pk_rsub(tn, bmin));
    const bool close = dist < eps && act;
    int insuf = s.insuf[b];
    const bool need = close && (insuf || tn >= bmax || tn <= bmin);
    if (need) {
        tn = (F)fabs(pk_rsub(tn, bmax)) < (F)fabs(pk_rsub(tn, bmin)) ? pk_rsub(bmax, eps) : pk_radd(bmin, eps);
        insuf = 0;
    }
    if (close && !need) insuf = 1;
    if (!close) insuf = 0;
    if (act) {
        const F* x = s.x + (size_t)b * N;
        const F* d = s.d + (size_t)b * N;
        F* xn = s.x_new + (size_t)b * N;
        PK_OWN_LOOP(k, N) xn[k] = pk_radd(x[k], pk_rmul(tn, d[k]));
    }
    if (threadIdx.x == 0) {
        s.t_new[b] = tn;
        s.insuf[b] = insuf;
        s.active[b] = act;
        if (act) atomicOr(s.flag, 1);
    }
}

// The zoom's bracket update after its evaluation (:310-389).
template <typename F>
__global__ void pk_wolfe_zoom_post_kernel(PkWolfeState<F> s, F c1, F c2)
{
    const int b = blockIdx.x, N = s.N;
    if (!s.in_ls[b] || !s.active[b]) return;
    const F f = s.f[b], gtd = s.gtd[b], tn = s.t_new[b];
    const F fn = s.f_new[b], gn = s.gtd_new[b];
    const F* gnew = s.g_new + (size_t)b * N;
    int low = s.low[b];
    const int high = 1 - low;
    const bool todo1 = fn > pk_armijo_bound(f, c1, tn, gtd) || fn >= s.bf[2 * b + low];
    int act = 1;
    if (todo1) {
        pk_wolfe_set_slot(s, b, high, tn, fn, gnew, gn, true);
        __syncthreads();
        low = s.bf[2 * b] <= s.bf[2 * b + 1] ? 0 : 1;
    } else {
        const bool wolfe = (F)fabs(gn) <= pk_rmul(-c2, gtd);
        if (wolfe) {
            act = 0;
            if (threadIdx.x == 0) s.done[b] = 1;
        } else if (pk_rmul(gn, pk_rsub(s.bt[2 * b + high], s.bt[2 * b + low])) >= (F)0) {
            // the old low end becomes the high end
            pk_wolfe_set_slot(s, b, high, s.bt[2 * b + low], s.bf[2 * b + low], s.bg + ((size_t)b * 2 + low) * N,
                              s.bgtd[2 * b + low], true);
            __syncthreads();
        }
        pk_wolfe_set_slot(s, b, low, tn, fn, gnew, gn, true);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s.low[b] = low;
        s.active[b] = act;
    }
}

// Result (:391-407): the accepted step, loss and gradient of each system.
template <typename F>
__global__ void pk_wolfe_final_kernel(PkWolfeState<F> s)
{
    const int b = blockIdx.x, N = s.N;
    if (!s.in_ls[b]) return;
    const int slot = s.bsize[b] == 1 ? 0 : s.low[b];
    const F* src = s.bg + ((size_t)b * 2 + slot) * N;
    F* gn = s.g_new + (size_t)b * N;
    PK_OWN_LOOP(k, N) gn[k] = src[k];
    if (threadIdx.x == 0) {
        s.t[b] = s.bt[2 * b + slot];
        s.f_new[b] = s.bf[2 * b + slot];
    }
}

template <typename F>
static int pk_wolfe_phase_t(int phase, const PkWolfeState<F>& s, int ls_iter, double c1, double c2, double tol_change,
                            int flag_arg, cudaStream_t st)
{
    if (s.M == 0) return PK_OK;
    const int T = pk_lbfgs_threads(s.N);
    const size_t smem = (size_t)pk_canon_red_len(s.N) * sizeof(F);
    switch (phase) {
        case 0: pk_wolfe_init_kernel<F><<<s.M, T, smem, st>>>(s); break;
        case 1: pk_wolfe_after_eval_kernel<F><<<s.M, T, smem, st>>>(s, flag_arg); break;
        case 2: pk_wolfe_bracket_kernel<F><<<s.M, T, 0, st>>>(s, ls_iter, (F)c1, (F)c2); break;
        case 3: pk_wolfe_zoom_init_kernel<F><<<s.M, T, 0, st>>>(s, flag_arg); break;
        case 4: pk_wolfe_zoom_pre_kernel<F><<<s.M, T, 0, st>>>(s, (F)tol_change); break;
        case 5: pk_wolfe_zoom_post_kernel<F><<<s.M, T, 0, st>>>(s, (F)c1, (F)c2); break;
        case 6: pk_wolfe_final_kernel<F><<<s.M, T, 0, st>>>(s); break;
        default: return pk_fail(PK_EINVAL, "pk_wolfe_phase: unknown phase%s");
    }
    return pk_cuda_check(cudaGetLastError(), "pk_wolfe_phase launch");
}

extern "C" int pk_wolfe_phase(int phase, int dtype_bytes, void* const* arrays, int M, int N, int ls_iter, double c1,
                              double c2, double tol_change, int flag_arg, void* stream)
{
    if (!arrays) return pk_fail(PK_EINVAL, "pk_wolfe_phase: arrays is NULL%s");
    if (M < 0 || N < 1) return pk_fail(PK_EINVAL, "pk_wolfe_phase: bad sizes%s");
    cudaStream_t st = (cudaStream_t)stream;
#define PK_WFILL(F)                                                                                     \
    PkWolfeState<F> s;                                                                                  \
    s.x = (const F*)arrays[0]; s.d = (const F*)arrays[1]; s.g = (const F*)arrays[2];                    \
    s.f = (const F*)arrays[3]; s.gtd = (F*)arrays[4]; s.t = (F*)arrays[5];                              \
    s.x_new = (F*)arrays[6]; s.g_new = (F*)arrays[7]; s.f_new = (F*)arrays[8]; s.gtd_new = (F*)arrays[9]; \
    s.g_prev = (F*)arrays[10]; s.f_prev = (F*)arrays[11]; s.gtd_prev = (F*)arrays[12];                  \
    s.t_prev = (F*)arrays[13]; s.bg = (F*)arrays[14]; s.bt = (F*)arrays[15]; s.bf = (F*)arrays[16];     \
    s.bgtd = (F*)arrays[17]; s.d_norm = (F*)arrays[18]; s.t_new = (F*)arrays[19];                       \
    s.bsize = (int*)arrays[20]; s.done = (int*)arrays[21]; s.active = (int*)arrays[22];                 \
    s.low = (int*)arrays[23]; s.insuf = (int*)arrays[24]; s.evals = (int*)arrays[25];                   \
    s.in_ls = (int*)arrays[26]; s.flag = (int*)arrays[27];                                              \
    s.M = M; s.N = N;
    if (dtype_bytes == 4) {
        PK_WFILL(float)
        return pk_wolfe_phase_t<float>(phase, s, ls_iter, c1, c2, tol_change, flag_arg, st);
    } else if (dtype_bytes == 8) {
        PK_WFILL(double)
        return pk_wolfe_phase_t<double>(phase, s, ls_iter, c1, c2, tol_change, flag_arg, st);
    }
#undef PK_WFILL
    return pk_fail(PK_EINVAL, "pk_wolfe_phase: dtype must be float32 or float64%s");
}

// The outer iteration after a search (:621-624, :632): the searched systems
// take the accepted step and its loss and gradient; evaluation counts are
// set up so that the history / convergence phase (which adds one) ends with
// func_evals += ls_evals for them and += 0 for the others.
template <typename F>
__global__ void pk_wolfe_apply_kernel(F* x, F* g, F* loss, int* evals, const F* d, const F* t, const F* f_new,
                                      const F* g_new, const int* in_ls, const int* ls_evals, int M, int N)
{
    const int b = blockIdx.x;
    if (b >= M) return;
    if (!in_ls[b]) {
        if (threadIdx.x == 0) evals[b] -= 1;
        return;
    }
    const F tb = t[b];
    F* xb = x + (size_t)b * N;
    F* gb = g + (size_t)b * N;
    const F* db = d + (size_t)b * N;
    const F* gn = g_new + (size_t)b * N;
    PK_OWN_LOOP(k, N) {
        xb[k] = pk_radd(xb[k], pk_rmul(tb, db[k]));
        gb[k] = gn[k];
    }
    if (threadIdx.x == 0) {
        loss[b] = f_new[b];
        evals[b] += ls_evals[b] - 1;
    }
}

extern "C" int pk_wolfe_apply(int dtype_bytes, void* x, void* g, void* loss, int* evals, const void* d, const void* t,
                              const void* f_new, const void* g_new, const int* in_ls, const int* ls_evals, int M,
                              int N, void* stream)
{
    if (M < 0 || N < 1) return pk_fail(PK_EINVAL, "pk_wolfe_apply: bad sizes%s");
    if (M == 0) return PK_OK;
    const int T = pk_lbfgs_threads(N);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype_bytes == 4)
        pk_wolfe_apply_kernel<float><<<M, T, 0, st>>>((float*)x, (float*)g, (float*)loss, evals, (const float*)d,
                                                      (const float*)t, (const float*)f_new, (const float*)g_new,
                                                      in_ls, ls_evals, M, N);
    else if (dtype_bytes == 8)
        pk_wolfe_apply_kernel<double><<<M, T, 0, st>>>((double*)x, (double*)g, (double*)loss, evals,
                                                       (const double*)d, (const double*)t, (const double*)f_new,
                                                       (const double*)g_new, in_ls, ls_evals, M, N);
    else
        return pk_fail(PK_EINVAL, "pk_wolfe_apply: dtype must be float32 or float64%s");
    return pk_cuda_check(cudaGetLastError(), "pk_wolfe_apply launch");
}
