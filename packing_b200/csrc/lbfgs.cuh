// lbfgs.cuh -- batched L-BFGS (lbfgs_torch_parallel.py:411-729, no line search).
//
// Two forms share the per-system arithmetic below:
//  * the drop-in kernels (pk_lbfgs_direction / _step / _update) run one
//    iteration phase each for M independent systems while the objective
//    stays a caller-supplied function (the reference's `func`);
//  * pk_relax_kernel runs whole relaxations: one CTA per packing keeps x,
//    the gradient and the direction in shared memory, evaluates the compound
//    cost with the cost kernel's device code and iterates to max_iter in a
//    single launch.
// Both use the same order-fixed reductions (pk_canon_sum), so given the same
// objective values they produce the same iterates bit for bit.
// History is a ring buffer (logical entry i of a system lives in slot
// (start + i) % m), which is equivalent to the reference's shift-left-and-
// append (:676-690) without moving memory.
#pragma once
#include "common.cuh"
#include "cost.cuh"

#include <mutex>

// Two-loop recursion (:533-572) for one system: d = -H g with the valid
// history entries in logical order; al is shared scratch of m entries.
// Every elementwise operation rounds as the reference's tensor operations do
// (q - y a, s (al - be), products before the sums); the dot products use the
// canonical order.  Vector work uses element ownership (PK_OWN_LOOP): no
// barrier besides the one inside each reduction.
//
// When every warp owns at most one group (N <= 128 x warps), each thread
// holds its <= 4 elements of q in registers and loads the next history entry
// while the current dot product is being reduced, so the chain of 2 hlen
// dependent reductions does not also wait for a memory round trip per step.
// Both paths perform the same operations in the same order.
template <typename F>
__device__ void pk_two_loop(const F* g, F* d, int N, const F* S, const F* Y, const F* ro, int m, int hlen,
                            int hstart, F Hdiag, F* al, F* red, int& flip)
{
    const int ng = pk_canon_groups(N);
    const int nw = blockDim.x >> 5;
    if (ng > nw) {
        PK_OWN_LOOP(k, N) d[k] = -g[k];
        for (int i = hlen - 1; i >= 0; --i) {
            const int slot = (hstart + i) % m;
            const F* s = S + (size_t)slot * N;
            const F* y = Y + (size_t)slot * N;
            const F a = pk_rmul(pk_canon_sum<F>(N, [&](int k) { return pk_rmul(s[k], d[k]); }, red, flip), ro[slot]);
            if (threadIdx.x == 0) al[i] = a;
            PK_OWN_LOOP(k, N) d[k] = pk_rsub(d[k], pk_rmul(y[k], a));
        }
        PK_OWN_LOOP(k, N) d[k] = pk_rmul(d[k], Hdiag);
        __syncthreads();   // al[] visible
        for (int i = 0; i < hlen; ++i) {
            const int slot = (hstart + i) % m;
            const F* s = S + (size_t)slot * N;
            const F* y = Y + (size_t)slot * N;
            const F be = pk_rmul(pk_canon_sum<F>(N, [&](int k) { return pk_rmul(y[k], d[k]); }, red, flip), ro[slot]);
            const F c = pk_rsub(al[i], be);
            PK_OWN_LOOP(k, N) d[k] = pk_radd(d[k], pk_rmul(s[k], c));
        }
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k0 = warp * PK_CANON_GROUP + lane;   // >= N for a warp that owns no group
    // this lane's elements are k0 + 32 j for j < nv
    const int nv = k0 < N ? min(4, (N - k0 + 31) >> 5) : 0;
    const ptrdiff_t yoff = Y - S;                  // Y entry = S entry + yoff
    F q[4], sc[4], yc[4], sn[4], yn[4];
    F rc = 0, rn = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        q[j] = j < nv ? -g[k0 + 32 * j] : F(0);
        sc[j] = yc[j] = sn[j] = yn[j] = F(0);
    }
#define PK_TL_FETCH(SV, YV, P)                         \
    {                                                  \
        _Pragma("unroll") for (int j = 0; j < 4; ++j)  \
            if (j < nv) {                              \
                SV[j] = (P)[32 * j];                   \
                YV[j] = (P)[yoff + 32 * j];            \
            }                                          \
    }
    // first loop: newest entry first; the slot steps down with wraparound
    int slot = hlen > 0 ? (hstart + hlen - 1) % m : 0;
    const F* pcur = S + (size_t)slot * N + k0;
    if (hlen > 0) {
        PK_TL_FETCH(sc, yc, pcur)
        rc = ro[slot];
    }
    for (int i = hlen - 1; i >= 0; --i) {
        const int nslot = slot == 0 ? m - 1 : slot - 1;
        const F* pnext = slot == 0 ? pcur + (size_t)(m - 1) * N : pcur - N;
        if (i > 0) {
            PK_TL_FETCH(sn, yn, pnext)
            rn = ro[nslot];
        }
        F* buf = pk_canon_buf(ng, red, flip);
        if (warp < ng) {
            F p = F(0);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < nv) p = pk_radd(p, pk_rmul(sc[j], q[j]));
            buf[warp * 32 + lane] = p;
        }
        const F a = pk_rmul(pk_canon_finish(buf, ng), rc);
        if (threadIdx.x == 0) al[i] = a;
#pragma unroll
        for (int j = 0; j < 4; ++j) q[j] = pk_rsub(q[j], pk_rmul(yc[j], a));
        if (i > 0) {   // entry 0 stays in hand: the second loop starts with it
#pragma unroll
            for (int j = 0; j < 4; ++j) { sc[j] = sn[j]; yc[j] = yn[j]; }
            rc = rn;
            slot = nslot;
            pcur = pnext;
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) q[j] = pk_rmul(q[j], Hdiag);
    __syncthreads();   // al[] visible
    // second loop: oldest entry first; the slot steps up with wraparound
    for (int i = 0; i < hlen; ++i) {
        const int nslot = slot == m - 1 ? 0 : slot + 1;
        const F* pnext = slot == m - 1 ? pcur - (size_t)(m - 1) * N : pcur + N;
        if (i + 1 < hlen) {
            PK_TL_FETCH(sn, yn, pnext)
            rn = ro[nslot];
        }
        F* buf = pk_canon_buf(ng, red, flip);
        if (warp < ng) {
            F p = F(0);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < nv) p = pk_radd(p, pk_rmul(yc[j], q[j]));
            buf[warp * 32 + lane] = p;
        }
        const F be = pk_rmul(pk_canon_finish(buf, ng), rc);
        const F c = pk_rsub(al[i], be);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            q[j] = pk_radd(q[j], pk_rmul(sc[j], c));
            sc[j] = sn[j];
            yc[j] = yn[j];
        }
        rc = rn;
        slot = nslot;
        pcur = pnext;
    }
#undef PK_TL_FETCH
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (j < nv) d[k0 + 32 * j] = q[j];
}

// max_k |v[k] * scale| and max_k |w[k] * wscale| with one barrier.
template <typename F>
__device__ __forceinline__ void pk_own_absmax2(int N, const F* v, F scale, const F* w, F wscale, F* red, int& flip,
                                               F& rv, F& rw)
{
    pk_canon_max2<F>(N, [&](int k, F& a, F& b) {
        a = (F)fabs(pk_rmul(v[k], scale));
        b = (F)fabs(pk_rmul(w[k], wscale));
    }, red, flip, rv, rw);
}

// ---------------------------------------------------------------------------
// Drop-in kernels.  Per-system state (all device arrays of M entries):
//   loss, prev_loss, loss0 (F); t, H (F); hlen, hstart, evals, active (int)
// ---------------------------------------------------------------------------
template <typename F>
struct PkLbfgsState {
    F* x; F* g; F* loss; F* d; F* pg; F* ploss; F* loss0;
    F* S; F* Y; F* ro; F* H; F* t;
    int* hlen; int* hstart; int* evals; int* active; int* any_active;
    int M, N, m;
};

// Phase 1 of an iteration (:531-612): direction, initial step, max_step
// clamp, directional-derivative stop.  Sets *any_active if a system remains.
template <typename F>
__global__ void pk_lbfgs_direction_kernel(PkLbfgsState<F> s, int n_iter, F lr, F max_step, int has_max_step,
                                          F tol_change)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const int N = s.N;
    F* al = (F*)pk_smem;
    F* red = al + s.m;
    int flip = 0;
    const int b = blockIdx.x;
    const F* g = s.g + (size_t)b * N;
    F* d = s.d + (size_t)b * N;
    F* pg = s.pg + (size_t)b * N;
    int active = s.active[b];
    F Hd = s.H[b];
    if (n_iter == 1) {
        PK_OWN_LOOP(k, N) d[k] = -g[k];
        Hd = 1;
    } else {
        pk_two_loop<F>(g, d, N, s.S + (size_t)b * s.m * N, s.Y + (size_t)b * s.m * N, s.ro + (size_t)b * s.m, s.m,
                       s.hlen[b], s.hstart[b], Hd, al, red, flip);
    }
    PK_OWN_LOOP(k, N) pg[k] = g[k];
    F t;
    if (n_iter == 1) {
        const F gs = pk_canon_sum<F>(N, [&](int k) { return (F)fabs(g[k]); }, red, flip);
        t = (F)1 / gs;
        t = (t < (F)1 ? t : (F)1) * lr;   // torch.minimum(1, 1/sum|g|) * lr
        if (!active) t = 0;
    } else {
        t = lr;
    }
    if (has_max_step) {
        F pc, unused;
        pk_own_absmax2<F>(N, d, t, d, t, red, flip, pc, unused);
        if (pc > max_step) t = t * (max_step / pc);
    }
    const F gtd = pk_canon_sum<F>(N, [&](int k) { return pk_rmul(g[k], d[k]); }, red, flip);
    if (gtd > -tol_change) active = 0;
    if (threadIdx.x == 0) {
        s.t[b] = t;
        s.H[b] = Hd;
        s.ploss[b] = s.loss[b];
        s.active[b] = active;
        if (active) atomicOr(s.any_active, 1);
    }
}

// Phase 2 (:631): x += t d for every system (inactive ones too, as the
// reference does while any system is active).
template <typename F>
__global__ void pk_lbfgs_step_kernel(F* x, const F* d, const F* t, int M, int N)
{
    const size_t total = (size_t)M * N;
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < total; w += (size_t)gridDim.x * blockDim.x)
        x[w] = pk_radd(x[w], pk_rmul(t[w / N], d[w]));
}

// Phase 3 (:636-724): history update with the curvature guard, then the
// convergence tests.  g / loss are the values at the new x (unchanged when
// the objective was not re-evaluated on the last iteration).
template <typename F>
__global__ void pk_lbfgs_update_kernel(PkLbfgsState<F> s, int n_iter, F tol_grad, F tol_change, F tol_rel,
                                       int stop_on_increase, int max_eval)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    F* red = (F*)pk_smem;
    int flip = 0;
    const int b = blockIdx.x;
    const int N = s.N, m = s.m;
    const F* g = s.g + (size_t)b * N;
    const F* pg = s.pg + (size_t)b * N;
    const F* d = s.d + (size_t)b * N;
    const F t = s.t[b];
    int active = s.active[b];
    int evals = s.evals[b] + 1;
    if (n_iter > 1) {
        F ys, yy;
        pk_canon_sum2<F>(N, [&](int k, F& a, F& c) {
            const F y = pk_rsub(g[k], pg[k]);
            a = pk_rmul(y, pk_rmul(d[k], t));
            c = pk_rmul(y, y);
        }, red, flip, ys, yy);
        if (active && ys > (F)1e-10) {
            int hl = s.hlen[b], hs = s.hstart[b], slot;
            if (hl < m) { slot = (hs + hl) % m; ++hl; }
            else { slot = hs; hs = (hs + 1) % m; }
            F* S = s.S + ((size_t)b * m + slot) * N;
            F* Y = s.Y + ((size_t)b * m + slot) * N;
            PK_OWN_LOOP(k, N) {
                Y[k] = pk_rsub(g[k], pg[k]);
                S[k] = pk_rmul(d[k], t);
            }
            if (threadIdx.x == 0) {
                s.H[b] = ys / yy;
                s.ro[(size_t)b * m + slot] = (F)1 / ys;
                s.hlen[b] = hl;
                s.hstart[b] = hs;
            }
        }
    }
    F gmax, pc;
    pk_own_absmax2<F>(N, g, (F)1, d, t, red, flip, gmax, pc);
    if (threadIdx.x == 0) {
        if (gmax <= tol_grad) active = 0;
        if (evals >= max_eval) active = 0;
        if (pc <= tol_change && active) active = 0;
        const F loss = s.loss[b], ploss = s.ploss[b];
        const F lc = fabs(loss - ploss);
        if (lc < tol_change && active) active = 0;
        if (tol_rel > 0 && n_iter > m) {
            if (lc / (fabs(ploss) + (F)1e-12) < tol_rel && active) active = 0;
        }
        if (stop_on_increase && loss > s.loss0[b] && active) active = 0;
        s.active[b] = active;
        s.evals[b] = evals;
    }
}

// Initial activity (:493-500): active unless max|g| <= tol_grad.
template <typename F>
__global__ void pk_lbfgs_init_kernel(PkLbfgsState<F> s, F tol_grad)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    F* red = (F*)pk_smem;
    int flip = 0;
    const int b = blockIdx.x;
    const F* g = s.g + (size_t)b * s.N;
    F gm, unused;
    pk_own_absmax2<F>(s.N, g, (F)1, g, (F)1, red, flip, gm, unused);
    if (threadIdx.x == 0) {
        const int a = gm <= tol_grad ? 0 : 1;
        s.active[b] = a;
        s.hlen[b] = 0;
        s.hstart[b] = 0;
        s.evals[b] = 1;
        s.H[b] = 1;
        s.loss0[b] = s.loss[b];
        if (a) atomicOr(s.any_active, 1);
    }
}

// One warp per canonical group (so the two-loop keeps its elements in
// registers), between 2 and 8 warps.
static inline int pk_lbfgs_threads(int N)
{
    const int ng = pk_canon_groups(N);
    return 32 * (ng < 2 ? 2 : (ng > 8 ? 8 : ng));
}

template <typename F>
static int pk_lbfgs_phase(int phase, const PkLbfgsState<F>& s, int n_iter, double a, double b_, double c, double d_,
                          int i1, int i2, cudaStream_t st)
{
    const int T = pk_lbfgs_threads(s.N);
    const size_t smem = ((size_t)s.m + pk_canon_red_len(s.N)) * sizeof(F);
    if (s.M == 0) return PK_OK;
    cudaError_t err = cudaSuccess;
    switch (phase) {
        case 0:
        case 1:
        case 3: {
            const void* fn = phase == 0 ? (const void*)pk_lbfgs_init_kernel<F>
                           : phase == 1 ? (const void*)pk_lbfgs_direction_kernel<F>
                                        : (const void*)pk_lbfgs_update_kernel<F>;
            err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (err != cudaSuccess) return pk_cuda_check(err, "pk_lbfgs attribute");
            if (phase == 0) pk_lbfgs_init_kernel<F><<<s.M, T, smem, st>>>(s, (F)a);
            else if (phase == 1) pk_lbfgs_direction_kernel<F><<<s.M, T, smem, st>>>(s, n_iter, (F)a, (F)b_, i1, (F)c);
            else pk_lbfgs_update_kernel<F><<<s.M, T, smem, st>>>(s, n_iter, (F)a, (F)b_, (F)c, i1, i2);
            break;
        }
        case 2: {
            const size_t total = (size_t)s.M * s.N;
            const int blocks = (int)((total + 255) / 256 < 148 * 8 ? (total + 255) / 256 : 148 * 8);
            pk_lbfgs_step_kernel<F><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(s.x, s.d, s.t, s.M, s.N);
            break;
        }
        default: return pk_fail(PK_EINVAL, "pk_lbfgs: unknown phase%s");
    }
    (void)d_;
    return pk_cuda_check(cudaGetLastError(), "pk_lbfgs launch");
}

// C-ABI: the state struct is passed as pointers to device arrays.
extern "C" int pk_lbfgs_phase(int phase, int dtype_bytes, void* const* arrays, int M, int N, int m, int n_iter,
                              double p0, double p1, double p2, double p3, int i1, int i2, void* stream)
{
    if (!arrays) return pk_fail(PK_EINVAL, "pk_lbfgs_phase: arrays is NULL%s");
    if (M < 0 || N < 1 || m < 1) return pk_fail(PK_EINVAL, "pk_lbfgs_phase: bad sizes%s");
    cudaStream_t st = (cudaStream_t)stream;
#define PK_FILL(F)                                                                                     \
    PkLbfgsState<F> s;                                                                                 \
    s.x = (F*)arrays[0]; s.g = (F*)arrays[1]; s.loss = (F*)arrays[2]; s.d = (F*)arrays[3];             \
    s.pg = (F*)arrays[4]; s.ploss = (F*)arrays[5]; s.loss0 = (F*)arrays[6]; s.S = (F*)arrays[7];        \
    s.Y = (F*)arrays[8]; s.ro = (F*)arrays[9]; s.H = (F*)arrays[10]; s.t = (F*)arrays[11];             \
    s.hlen = (int*)arrays[12]; s.hstart = (int*)arrays[13]; s.evals = (int*)arrays[14];                \
    s.active = (int*)arrays[15]; s.any_active = (int*)arrays[16];                                      \
    s.M = M; s.N = N; s.m = m;
    if (dtype_bytes == 4) {
        PK_FILL(float)
        return pk_lbfgs_phase<float>(phase, s, n_iter, p0, p1, p2, p3, i1, i2, st);
    } else if (dtype_bytes == 8) {
        PK_FILL(double)
        return pk_lbfgs_phase<double>(phase, s, n_iter, p0, p1, p2, p3, i1, i2, st);
    }
#undef PK_FILL
    return pk_fail(PK_EINVAL, "pk_lbfgs_phase: dtype must be float32 or float64%s");
}

// ---------------------------------------------------------------------------
// Fused relaxation: one CTA per packing runs the L-BFGS loop with the
// compound cost evaluated in place.  x = [xyt (3n), h (3)] as in
// pack_dynamics.py:76-83.  Per-instance stop: an instance that becomes
// inactive stops stepping (the reference keeps stepping inactive systems
// while another system of the same batch is still active, so with this form
// an instance's result never depends on the rest of the batch).  The cost is
// evaluated at one place in the loop.
// ---------------------------------------------------------------------------
struct PkRelaxVars {
    int it, evals, hlen, hstart, active;
    float H, loss, loss0, ploss, t;
};

// Runs iterations until the relaxation finishes (returns true) or, after the
// history update of iteration it_stop, pauses (returns false) with x, g, the
// history and v complete, so a later call with resume = true continues
// exactly where this one stopped.  resume = false starts from x (evaluates
// it first).  All threads of the block call it.
template <int MODE, bool SYM>
__device__ bool pk_relax_iterate(float* x, float* g, float* pg, float* d, float* al, float* ro, float* red, int& flip,
                                 float* S, float* Y, int n, bool use_h, const PkCostSpec& spec,
                                 const PkRelaxParams& prm, const PkCostSmem& sm, PkRelaxVars& v, bool resume,
                                 int it_stop, unsigned long long& hist_streamed)
{
    const int N = 3 * n + 3;
    const int m = prm.history;
    bool need_eval = !resume, final_pending = false, want_grad = true, skip_update = resume;
    // Kept near lists when the step bound lets a list serve at least four
    // evaluations (every coordinate moves at most max_step per step); the
    // first evaluation of this call builds one.
    if (threadIdx.x == 0)
        pk_nlist(sm)[0] = (prm.has_max_step && 4.f * 2.8285f * prm.max_step + 1e-4f < pk_near_skin()) ? 0 : -1;
    pk_load_piece_table(sm);   // read after the next barrier; evaluations do not reload it
    for (;;) {
        if (need_eval) {
            __syncthreads();   // x complete
            const double L = pk_eval_instance<MODE, SYM, true>(x, n, use_h ? x + 3 * n : nullptr, spec,
                                                          want_grad ? g : nullptr,
                                                          (want_grad && use_h) ? g + 3 * n : nullptr, sm);
            v.loss = (float)L;
        }
        if (final_pending) return true;
        if (!skip_update) {
            if (v.it == 0) {
                // initial point (:489-500)
                v.loss0 = v.loss;
                float gm, unused;
                pk_own_absmax2<float>(N, g, 1.f, g, 1.f, red, flip, gm, unused);
                v.active = !(gm <= prm.tol_grad);
            } else {
                // after a step (:632-724)
                ++v.evals;
                if (v.it > 1) {
                    const float t = v.t;
                    float ys, yy;
                    pk_canon_sum2<float>(N, [&](int k, float& a, float& c) {
                        const float y = pk_rsub(g[k], pg[k]);
                        a = pk_rmul(y, pk_rmul(d[k], t));
                        c = pk_rmul(y, y);
                    }, red, flip, ys, yy);
                    if (ys > 1e-10f) {
                        int slot;
                        if (v.hlen < m) { slot = (v.hstart + v.hlen) % m; ++v.hlen; }
                        else { slot = v.hstart; v.hstart = (v.hstart + 1) % m; }
                        float* Sd = S + (size_t)slot * N;
                        float* Yd = Y + (size_t)slot * N;
                        PK_OWN_LOOP(k, N) {
                            Yd[k] = pk_rsub(g[k], pg[k]);
                            Sd[k] = pk_rmul(d[k], t);
                        }
                        v.H = ys / yy;
                        if (threadIdx.x == 0) ro[slot] = 1.f / ys;
                    }
                }
                float gmax, pc;
                pk_own_absmax2<float>(N, g, 1.f, d, v.t, red, flip, gmax, pc);
                if (gmax <= prm.tol_grad) v.active = 0;
                if (v.evals >= prm.max_eval) v.active = 0;
                if (pc <= prm.tol_change) v.active = 0;
                const float lc = fabsf(v.loss - v.ploss);
                if (lc < prm.tol_change) v.active = 0;
                if (prm.tol_rel_change > 0.f && v.it > m && lc / (fabsf(v.ploss) + 1e-12f) < prm.tol_rel_change)
                    v.active = 0;
                if (prm.stop_on_cost_increase && v.loss > v.loss0) v.active = 0;
            }
        }
        skip_update = false;
        if (!v.active || v.it >= prm.max_iter) return true;
        if (v.it >= it_stop) return false;
        // ---- next step (:531-631) ----
        ++v.it;
        if (v.it == 1) {
            PK_OWN_LOOP(k, N) d[k] = -g[k];
            v.H = 1.f;
        } else {
            pk_two_loop<float>(g, d, N, S, Y, ro, m, v.hlen, v.hstart, v.H, al, red, flip);
            hist_streamed += (unsigned long long)v.hlen;
        }
        PK_OWN_LOOP(k, N) pg[k] = g[k];
        v.ploss = v.loss;
        float t;
        if (v.it == 1) {
            const float gs = pk_canon_sum<float>(N, [&](int k) { return fabsf(g[k]); }, red, flip);
            t = 1.f / gs;
            t = (t < 1.f ? t : 1.f) * prm.lr;
        } else {
            t = prm.lr;
        }
        if (prm.has_max_step) {
            float pc, unused;
            pk_own_absmax2<float>(N, d, t, d, t, red, flip, pc, unused);
            if (pc > prm.max_step) t = t * (prm.max_step / pc);
        }
        v.t = t;
        const float gtd = pk_canon_sum<float>(N, [&](int k) { return pk_rmul(g[k], d[k]); }, red, flip);
        if (gtd > -prm.tol_change) { v.active = 0; --v.it; return true; }
        PK_OWN_LOOP(k, N) x[k] = pk_radd(x[k], pk_rmul(t, d[k]));
        need_eval = v.it != prm.max_iter;
        if (!need_eval && prm.final_eval) {
            // the last step is not evaluated by the reference loop; evaluate once for the final loss
            need_eval = true;
            want_grad = false;
            final_pending = true;
        }
    }
}

// Drops the 128-byte L2 lines wholly inside [p, p + nbytes) without writing
// them back (PTX discard.global.L2).  A one-shot relaxation's history is
// scratch of its launch: without this, every finished packing's 2 m N floats
// stay dirty in L2 and are written to HBM when later packings evict them
// (315 MB per 4096 x n = 200 launch at m = 10).  A line shared with the
// neighbouring packing's history is left alone.  The caller has synchronised
// the block after the last access; the region's contents are undefined
// afterwards, and every history slot is written before it is read.
__device__ __forceinline__ void pk_discard_l2(const void* p, size_t nbytes)
{
    const size_t g = __cvta_generic_to_global(p);
    const size_t b = (g + 127) & ~(size_t)127;
    const size_t e = (g + nbytes) & ~(size_t)127;
    for (size_t a = b + (size_t)threadIdx.x * 128; a < e; a += (size_t)blockDim.x * 128)
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(a) : "memory");
}

// Relaxes instance e (all threads of the block call it; e is uniform).
template <int MODE, bool SYM>
__device__ void pk_relax_instance(int e, const float* __restrict__ xyt_in, const float* __restrict__ h_in,
                                  const int* __restrict__ offsets, int E, int n_max, const PkCostSpec& spec,
                                  const PkRelaxParams& prm, float* __restrict__ xyt_out, float* __restrict__ h_out,
                                  float* __restrict__ loss_out, int* __restrict__ iters_out, float* __restrict__ work,
                                  int cap_near, int cap_items, unsigned char* smem)
{
    if (e < 0 || e >= E) return;
    const int base = offsets ? offsets[e] : e * n_max;
    const int n = offsets ? offsets[e + 1] - base : n_max;
    if (n < 0 || n > n_max) {
        if (threadIdx.x == 0) { loss_out[e] = __int_as_float(0x7fc00000); if (iters_out) iters_out[e] = -1; }
        return;
    }
    const int N = 3 * n + 3;
    const int NM = 3 * n_max + 3;
    const int m = prm.history;
    const int nps = n_max * (SYM ? pk_symmetry(spec) : 1);   // phenotype trees sized in shared memory
    PkCostSmem sm = pk_cost_carve(smem, nps, cap_near, cap_items, true);
    if (threadIdx.x < 4) sm.cnt[threadIdx.x] = 0;
    float* x = (float*)(smem + pk_cost_smem_bytes(nps, cap_near, cap_items, true));
    float* g = x + NM;
    float* pg = g + NM;
    float* d = pg + NM;
    float* al = d + NM;
    float* ro = al + m;
    float* red = ro + m;
    int flip = 0;
    // history of this instance: work + 2 m * (3 * base + 3 * e) floats
    float* S = work + (size_t)2 * m * (3 * (size_t)base + 3 * (size_t)e);
    float* Y = S + (size_t)m * N;
    for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) x[k] = xyt_in[(size_t)base * 3 + k];
    if (threadIdx.x < 3) x[3 * n + threadIdx.x] = h_in ? h_in[3 * e + threadIdx.x] : 0.f;
    if (threadIdx.x < 3) g[3 * n + threadIdx.x] = 0.f;
    PkRelaxVars v;
    v.it = 0; v.evals = 1; v.hlen = 0; v.hstart = 0; v.active = 1;
    v.H = 1.f; v.loss = 0.f; v.loss0 = 0.f; v.ploss = 0.f; v.t = 0.f;
    unsigned long long hist_streamed = 0;
    pk_relax_iterate<MODE, SYM>(x, g, pg, d, al, ro, red, flip, S, Y, n, h_in != nullptr, spec, prm, sm, v, false,
                           prm.max_iter, hist_streamed);
    __syncthreads();
    pk_discard_l2(S, (size_t)2 * m * N * sizeof(float));
    for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) xyt_out[(size_t)base * 3 + k] = x[k];
    if (h_out && threadIdx.x < 3) h_out[3 * e + threadIdx.x] = x[3 * n + threadIdx.x];
    if (threadIdx.x == 0) {
        loss_out[e] = v.loss;
        if (iters_out) iters_out[e] = v.it;
        if (prm.counters) {
            for (int k = 0; k < 4; ++k) atomicAdd(&prm.counters[k], (unsigned long long)sm.cnt[k]);
            atomicAdd(&prm.counters[4], (unsigned long long)v.it);
            atomicAdd(&prm.counters[5], hist_streamed * (unsigned long long)N);
        }
    }
}

// One CTA per entry of the launch order (count entries), or (persistent) one
// CTA per resident slot walking the order with a stride of the grid: CTA b
// relaxes order[b], order[b + G], ...; largest-first orders keep the CTAs'
// loads even.  Instances are indexed 0 .. E-1 whatever part of the order a
// launch covers.
template <int MODE, bool PERSISTENT, bool SYM>
__global__ void __launch_bounds__(256, 3) pk_relax_kernel(const float* __restrict__ xyt_in, const float* __restrict__ h_in,
                                const int* __restrict__ offsets, const int* __restrict__ order, int count, int E,
                                int n_max, PkCostSpec spec, PkRelaxParams prm, float* __restrict__ xyt_out,
                                float* __restrict__ h_out, float* __restrict__ loss_out, int* __restrict__ iters_out,
                                float* __restrict__ work, int cap_near, int cap_items)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    if (!PERSISTENT) {   // the grid is exactly count CTAs
        pk_relax_instance<MODE, SYM>(order ? order[blockIdx.x] : blockIdx.x, xyt_in, h_in, offsets, E, n_max, spec, prm,
                                xyt_out, h_out, loss_out, iters_out, work, cap_near, cap_items, pk_smem);
    } else {
        for (int k = blockIdx.x; k < count; k += gridDim.x) {
            pk_relax_instance<MODE, SYM>(order ? order[k] : k, xyt_in, h_in, offsets, E, n_max, spec, prm, xyt_out, h_out,
                                    loss_out, iters_out, work, cap_near, cap_items, pk_smem);
            __syncthreads();   // shared state is reused by the next instance
        }
    }
}

// ---------------------------------------------------------------------------
// Resumable relaxation of device-resident jobs (the serving loop's engine).
// Each job keeps x = [xyt, h], its gradient, its L-BFGS history and scalars
// in a device pool between launches; one launch advances every listed job by
// up to chunk_iters iterations.  Because the pause point is the end of an
// iteration and every reduction is order-fixed, a job's result is the same
// whatever other jobs share its launches and however its iterations are
// split into chunks.
// ---------------------------------------------------------------------------
template <int MODE, bool SYM>
__global__ void __launch_bounds__(256, 3) pk_relax_jobs_kernel(PkJob* __restrict__ jobs, const int* __restrict__ list,
                                     int njobs, float* __restrict__ pool, int n_max, PkCostSpec spec,
                                     PkRelaxParams prm, int chunk_iters, int cap_near, int cap_items)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    PkJob* J = &jobs[list[blockIdx.x]];
    const int n = J->n;
    if (J->status == PK_JOB_DONE || n < 0 || n > n_max) return;
    const int N = 3 * n + 3;
    const int NM = 3 * n_max + 3;
    const int m = prm.history;
    const int nps = n_max * (SYM ? pk_symmetry(spec) : 1);
    PkRelaxParams p = prm;
    p.max_iter = J->max_iter;
    p.max_eval = J->max_iter * 5 / 4;
    p.final_eval = 1;
    PkCostSmem sm = pk_cost_carve(pk_smem, nps, cap_near, cap_items, true);
    if (threadIdx.x < 4) sm.cnt[threadIdx.x] = 0;
    float* x = (float*)(pk_smem + pk_cost_smem_bytes(nps, cap_near, cap_items, true));
    float* g = x + NM;
    float* pg = g + NM;
    float* d = pg + NM;
    float* al = d + NM;
    float* ro = al + m;
    float* red = ro + m;
    int flip = 0;
    float* gx = pool + J->x_off;        // x (N), g (N), ro (m)
    float* S = pool + J->h_off;         // S (m N), Y (m N)
    float* Y = S + (size_t)m * N;
    const bool resume = J->status == PK_JOB_RUNNING;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        x[k] = gx[k];
        if (resume) g[k] = gx[N + k];
    }
    if (threadIdx.x < m && resume) ro[threadIdx.x] = gx[2 * N + threadIdx.x];
    if (threadIdx.x < 3 && !resume) g[3 * n + threadIdx.x] = 0.f;
    // a resumed job goes straight to the two-loop recursion, whose threads
    // read elements of g and ro that other threads loaded
    __syncthreads();
    PkRelaxVars v;
    v.it = J->it; v.evals = J->evals; v.hlen = J->hlen; v.hstart = J->hstart; v.active = 1;
    v.H = J->H; v.loss = J->loss; v.loss0 = J->loss0; v.ploss = 0.f; v.t = 0.f;
    if (!resume) { v.it = 0; v.evals = 1; v.hlen = 0; v.hstart = 0; v.H = 1.f; }
    unsigned long long hs = 0;
    const int it_stop = min(p.max_iter, v.it + max(chunk_iters, 1));
    const bool finished = pk_relax_iterate<MODE, SYM>(x, g, pg, d, al, ro, red, flip, S, Y, n, true, spec, p, sm, v,
                                                 resume, it_stop, hs);
    __syncthreads();
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        gx[k] = x[k];
        gx[N + k] = g[k];
    }
    if (threadIdx.x < m) gx[2 * N + threadIdx.x] = ro[threadIdx.x];
    if (threadIdx.x == 0) {
        J->it = v.it; J->evals = v.evals; J->hlen = v.hlen; J->hstart = v.hstart;
        J->H = v.H; J->loss = v.loss; J->loss0 = v.loss0;
        J->status = finished ? PK_JOB_DONE : PK_JOB_RUNNING;
    }
}

// n_max genotype trees (the L-BFGS vectors), sym images of each (the cost's
// per-tree arrays).
static size_t pk_relax_smem_bytes(int n_max, int sym, int cap_near, int cap_items, int m)
{
    const int NM = 3 * n_max + 3;
    return pk_cost_smem_bytes(n_max * sym, cap_near, cap_items, true) +
           ((size_t)4 * NM + 2 * (size_t)m + pk_canon_red_len(NM)) * 4;
}

// Threads per CTA of the relaxation kernels: the caller's choice (an
// autotuned value) or the default for the instance size.  Any multiple of 32
// up to 256 gives the same results (every reduction has an order fixed by
// the instance alone); the near list (8 T pairs) must hold one tree's n_max - 1.
static int pk_relax_threads(int n_max, int want, int* T, const char* who)
{
    if (want == 0) {
        *T = pk_cost_threads(n_max);
        return PK_OK;
    }
    if (want < 32 || want > 256 || (want & 31)) {
        snprintf(g_pk_err, sizeof(g_pk_err), "%s: threads must be 0 or a multiple of 32 in [32, 256], got %d", who,
                 want);
        return PK_EINVAL;
    }
    if (8 * want < n_max - 1) {
        snprintf(g_pk_err, sizeof(g_pk_err), "%s: %d threads are too few for %d trees (need 8 * threads >= n - 1)",
                 who, want, n_max);
        return PK_EINVAL;
    }
    *T = want;
    return PK_OK;
}

// Raises a kernel's dynamic shared memory limit only when a launch needs more
// than any earlier one on this device, so warmed-up launches make no
// attribute call (they can then be captured into a CUDA graph).
static cudaError_t pk_set_smem(const void* fn, int slot, size_t smem)
{
    static size_t done[64][32];
    static std::mutex mu;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= 64 || slot < 0 || slot >= 32) return cudaErrorInvalidValue;
    std::lock_guard<std::mutex> lock(mu);
    if (smem <= done[dev][slot]) return cudaSuccess;
    err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err == cudaSuccess) done[dev][slot] = smem;
    return err;
}

// Grid of a persistent launch: every CTA the GPU can keep resident, at most
// E.  The occupancy of a (kernel, threads, shared memory) shape is queried
// once per device and remembered, so warmed-up launches make no query.
static cudaError_t pk_resident_grid(const void* fn, int threads, size_t smem, int E, int* grid)
{
    struct Entry { const void* fn; int threads; size_t smem; int resident; };
    static Entry cache[64][32];
    static int used[64];
    static std::mutex mu;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidValue;
    int resident = -1;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (int k = 0; k < used[dev]; ++k) {
            const Entry& c = cache[dev][k];
            if (c.fn == fn && c.threads == threads && c.smem == smem) { resident = c.resident; break; }
        }
    }
    if (resident < 0) {
        int sms = 0, per_sm = 0;
        err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (err == cudaSuccess) err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
        if (err != cudaSuccess) return err;
        resident = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
        std::lock_guard<std::mutex> lock(mu);
        if (used[dev] < 32) cache[dev][used[dev]++] = Entry{fn, threads, smem, resident};
    }
    *grid = resident < E ? resident : E;
    return cudaSuccess;
}

extern "C" size_t pk_relax_workspace_floats(const int* sizes_host, int E, int n_uniform, int history)
{
    size_t tot = 0;
    if (sizes_host) {
        for (int e = 0; e < E; ++e) tot += 3 * (size_t)sizes_host[e] + 3;
    } else {
        tot = (size_t)E * (3 * (size_t)n_uniform + 3);
    }
    return 2 * (size_t)history * tot;
}

// The launch behind pk_relax and pk_relax_ordered: count entries of the
// launch order (all E instances when order is NULL).
static int pk_relax_launch(const float* xyt_in, const float* h_in, const int* offsets, const int* order, int count,
                           int E, int n_max, const PkCostSpec* spec, const PkRelaxParams* prm, float* xyt_out,
                           float* h_out, float* loss_out, int* iters_out, float* work, void* stream)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (!spec || !prm) return pk_fail(PK_EINVAL, "pk_relax: spec and params are required%s");
    if (E < 0 || n_max < 0) return pk_fail(PK_EINVAL, "pk_relax: negative size%s");
    if (count < 0 || count > E) return pk_fail(PK_EINVAL, "pk_relax: order count must be in [0, E]%s");
    if (count < E && !order) return pk_fail(PK_EINVAL, "pk_relax: a partial launch needs an order%s");
    if (E == 0 || count == 0) return PK_OK;
    if (n_max > PK_MAX_TREES) return pk_fail(PK_ERANGE, "pk_relax: more than 1024 trees per instance%s");
    if (prm->history < 1 || prm->history > 64) return pk_fail(PK_EINVAL, "pk_relax: history must be in [1, 64]%s");
    if (!xyt_in || !xyt_out || !loss_out || !work) return pk_fail(PK_EINVAL, "pk_relax: NULL pointer%s");
    if ((spec->w_boundary != 0.f || spec->w_area != 0.f) && !h_in)
        return pk_fail(PK_EINVAL, "pk_relax: boundary / area terms need h%s");
    if (spec->pair_mode == PK_PAIR_LUT && !spec->lut.vals) return pk_fail(PK_EINVAL, "pk_relax: LUT without vals%s");
    int T = 0;
    if (spec->symmetry != 0 && spec->symmetry != 1 && spec->symmetry != 2 && spec->symmetry != 4)
        return pk_fail(PK_EINVAL, "pk_relax: symmetry must be 0, 1, 2 or 4%s");
    const int sym = pk_symmetry(*spec);
    if ((long long)n_max * sym > PK_MAX_TREES) return pk_fail(PK_ERANGE, "pk_relax: more than 1024 phenotype trees%s");
    rc = pk_relax_threads(n_max * sym, prm->threads, &T, "pk_relax");
    if (rc) return rc;
    int cap_near, cap_items;
    pk_caps(T, spec->pair_mode, &cap_near, &cap_items);
    const size_t smem = pk_relax_smem_bytes(n_max, sym, cap_near, cap_items, prm->history);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaSuccess;
    int grid = count;
    switch (spec->pair_mode) {
#define PK_R3(M, P, S)                                                                                   \
    {                                                                                                    \
        err = pk_set_smem((const void*)pk_relax_kernel<M, P, S>, 4 + M + 4 * (P) + 8 * (S), smem);      \
        if (err == cudaSuccess && (P))                                                                   \
            err = pk_resident_grid((const void*)pk_relax_kernel<M, P, S>, T, smem, count, &grid);        \
        if (err == cudaSuccess)                                                                          \
            pk_relax_kernel<M, P, S><<<grid, T, smem, st>>>(xyt_in, h_in, offsets, order, count, E, n_max, *spec, \
                                                            *prm,                                        \
                                                            xyt_out, h_out, loss_out, iters_out, work, cap_near, \
                                                            cap_items);                                  \
    }
#define PK_R(M)                                                                                          \
    case M:                                                                                              \
        if (prm->persistent) {                                                                           \
            if (sym > 1) PK_R3(M, true, true) else PK_R3(M, true, false)                                 \
        } else {                                                                                         \
            if (sym > 1) PK_R3(M, false, true) else PK_R3(M, false, false)                               \
        }                                                                                                \
        break;
        PK_R(PK_PAIR_NONE)
        PK_R(PK_PAIR_AREA)
        PK_R(PK_PAIR_SEP)
        PK_R(PK_PAIR_LUT)
#undef PK_R
#undef PK_R3
        default: return pk_fail(PK_EINVAL, "pk_relax: unknown pair_mode%s");
    }
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_relax attribute");
    return pk_cuda_check(cudaGetLastError(), "pk_relax launch");
}

extern "C" int pk_relax(const float* xyt_in, const float* h_in, const int* offsets, const int* order, int E,
                        int n_max, const PkCostSpec* spec, const PkRelaxParams* prm, float* xyt_out, float* h_out,
                        float* loss_out, int* iters_out, float* work, void* stream)
{
    return pk_relax_launch(xyt_in, h_in, offsets, order, E, E, n_max, spec, prm, xyt_out, h_out, loss_out, iters_out,
                           work, stream);
}

extern "C" int pk_relax_ordered(const float* xyt_in, const float* h_in, const int* offsets, const int* order,
                                int count, int E, int n_max, const PkCostSpec* spec, const PkRelaxParams* prm,
                                float* xyt_out, float* h_out, float* loss_out, int* iters_out, float* work,
                                void* stream)
{
    if (!order) return pk_fail(PK_EINVAL, "pk_relax_ordered: order is required%s");
    return pk_relax_launch(xyt_in, h_in, offsets, order, count, E, n_max, spec, prm, xyt_out, h_out, loss_out,
                           iters_out, work, stream);
}

extern "C" int pk_relax_jobs(PkJob* jobs, const int* list, int njobs, float* pool, int n_max, const PkCostSpec* spec,
                             const PkRelaxParams* prm, int chunk_iters, void* stream)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (!spec || !prm) return pk_fail(PK_EINVAL, "pk_relax_jobs: spec and params are required%s");
    if (njobs < 0 || n_max < 0) return pk_fail(PK_EINVAL, "pk_relax_jobs: negative size%s");
    if (njobs == 0) return PK_OK;
    if (n_max > PK_MAX_TREES) return pk_fail(PK_ERANGE, "pk_relax_jobs: more than 1024 trees per job%s");
    if (prm->history < 1 || prm->history > 64) return pk_fail(PK_EINVAL, "pk_relax_jobs: history must be in [1, 64]%s");
    if (!jobs || !list || !pool) return pk_fail(PK_EINVAL, "pk_relax_jobs: NULL pointer%s");
    if (spec->pair_mode == PK_PAIR_LUT && !spec->lut.vals) return pk_fail(PK_EINVAL, "pk_relax_jobs: LUT without vals%s");
    int T = 0;
    if (spec->symmetry != 0 && spec->symmetry != 1 && spec->symmetry != 2 && spec->symmetry != 4)
        return pk_fail(PK_EINVAL, "pk_relax_jobs: symmetry must be 0, 1, 2 or 4%s");
    const int sym = pk_symmetry(*spec);
    if ((long long)n_max * sym > PK_MAX_TREES) return pk_fail(PK_ERANGE, "pk_relax_jobs: more than 1024 phenotype trees%s");
    rc = pk_relax_threads(n_max * sym, prm->threads, &T, "pk_relax_jobs");
    if (rc) return rc;
    int cap_near, cap_items;
    pk_caps(T, spec->pair_mode, &cap_near, &cap_items);
    const size_t smem = pk_relax_smem_bytes(n_max, sym, cap_near, cap_items, prm->history);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaSuccess;
    switch (spec->pair_mode) {
#define PK_J(M)                                                                                          \
    case M:                                                                                              \
        if (sym > 1) {                                                                                   \
            err = pk_set_smem((const void*)pk_relax_jobs_kernel<M, true>, 24 + M, smem);                  \
            if (err == cudaSuccess)                                                                      \
                pk_relax_jobs_kernel<M, true><<<njobs, T, smem, st>>>(jobs, list, njobs, pool, n_max, *spec, \
                                                                      *prm, chunk_iters, cap_near, cap_items); \
            break;                                                                                       \
        }                                                                                                \
        err = pk_set_smem((const void*)pk_relax_jobs_kernel<M, false>, 20 + M, smem);                     \
        if (err == cudaSuccess)                                                                          \
            pk_relax_jobs_kernel<M, false><<<njobs, T, smem, st>>>(jobs, list, njobs, pool, n_max, *spec, *prm, chunk_iters, \
                                                            cap_near, cap_items);                        \
        break;
        PK_J(PK_PAIR_NONE)
        PK_J(PK_PAIR_AREA)
        PK_J(PK_PAIR_SEP)
        PK_J(PK_PAIR_LUT)
#undef PK_J
        default: return pk_fail(PK_EINVAL, "pk_relax_jobs: unknown pair_mode%s");
    }
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_relax_jobs attribute");
    return pk_cuda_check(cudaGetLastError(), "pk_relax_jobs launch");
}

// ---------------------------------------------------------------------------
// Allocation-free relaxation: pk_relax with its L-BFGS history kept in a
// fixed device array compiled into this library instead of a caller buffer.
// The array is a file-scope __device__ symbol; host code may not use its name
// as a pointer, so the device address is fetched once per device with
// cudaGetSymbolAddress (on the first call made with that device current).
// ---------------------------------------------------------------------------
#include <mutex>

#define PK_NOALLOC_HISTORY_FLOATS (4u * 1024u * 1024u)   // 16 MiB per device

static __device__ __align__(256) float pk_noalloc_history[PK_NOALLOC_HISTORY_FLOATS];
static float* g_pk_noalloc_ptr[64];
static unsigned g_pk_noalloc_gen[64];   // g_pk_init_gen when the address was fetched
static std::mutex g_pk_noalloc_mu;

extern "C" int pk_relax_noalloc(const float* xyt_in, const float* h_in, int E, int n, const PkCostSpec* spec,
                                const PkRelaxParams* params, float* xyt_out, float* h_out, float* loss_out,
                                int* iters_out, void* stream)
{
    // the geometry must be on this device before anything touches it (and a
    // call before pk_init must not create or query a context)
    int rc = pk_check_init();
    if (rc) return rc;
    if (!params) return pk_fail(PK_EINVAL, "pk_relax_noalloc: params is NULL%s");
    if (E < 0 || n < 0) return pk_fail(PK_EINVAL, "pk_relax_noalloc: negative size%s");
    if (params->history < 1 || params->history > 64)
        return pk_fail(PK_EINVAL, "pk_relax_noalloc: history must be in [1, 64]%s");
    const unsigned long long need = 2ull * (unsigned long long)params->history * (unsigned long long)E *
                                    (3ull * (unsigned long long)n + 3ull);
    if (need > PK_NOALLOC_HISTORY_FLOATS) {
        snprintf(g_pk_err, sizeof(g_pk_err),
                 "pk_relax_noalloc: batch needs %llu history floats (2 * history * E * (3 n + 3)); the built-in "
                 "array holds %u -- use pk_relax with a caller buffer or a smaller batch",
                 need, (unsigned)PK_NOALLOC_HISTORY_FLOATS);
        return PK_ERANGE;
    }
    int dev = 0;
    rc = pk_cuda_check(cudaGetDevice(&dev), "pk_relax_noalloc: cudaGetDevice");
    if (rc) return rc;
    if (dev < 0 || dev >= 64) return pk_fail(PK_ERANGE, "pk_relax_noalloc: device id beyond 63%s");
    float* hist = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pk_noalloc_mu);
        if (!g_pk_noalloc_ptr[dev] || g_pk_noalloc_gen[dev] != g_pk_init_gen[dev]) {
            void* p = nullptr;
            rc = pk_cuda_check(cudaGetSymbolAddress(&p, pk_noalloc_history),
                               "pk_relax_noalloc: cudaGetSymbolAddress");
            if (rc) return rc;
            g_pk_noalloc_ptr[dev] = (float*)p;
            g_pk_noalloc_gen[dev] = g_pk_init_gen[dev];
        }
        hist = g_pk_noalloc_ptr[dev];
    }
    return pk_relax(xyt_in, h_in, nullptr, nullptr, E, n, spec, params, xyt_out, h_out, loss_out, iters_out, hist,
                    stream);
}
