// minkowski.cuh -- exact signed separation of two trees, tabulated on the GPU
// (pack_minkowski.separation_distance, pack_minkowski.py:210-266, which the
// reference evaluates with shapely per theta slice to build the lookup table
// of CollisionCostExactSeparation, pack_cost.py:1144-1215).
//
// Tree 1 sits at the origin unrotated, tree 2 at t = (x, y) rotated by theta.
// Their configuration-space obstacle is Z = union over piece pairs (p, q) of
// the convex Minkowski differences P_p - Q_q(theta) = hull{a - b}
// (pack_minkowski.py:34-62, :103-137).  The value at t is +dist(t, boundary
// of Z) when t is strictly inside Z (the trees overlap) and
// -dist(t, boundary of Z) otherwise (:253-264).
//
// Slice kernel, one CTA per theta: the 16 hulls (Andrew's monotone chain)
// and the boundary of their union: every hull edge minus the parts strictly
// inside another hull.  Grid kernel: tiles of 16 x 16 grid points; per tile
// the boundary pieces that can hold a point's nearest boundary point are
// kept (distance from the tile centre within the smallest such distance
// plus the tile diagonal), then every point tests the hulls whose boxes hold
// it and takes the smallest distance to the kept pieces.  All of it is FP64
// with every operation rounded on its own (no contraction); the table
// stores float32.
//
// Rotation angle: the reference turns tree 2 by shapely's affinity.rotate of
// np.degrees(theta) for a float32 theta, so under NumPy 2 the angle actually
// used is fl32(fl32(fl32(theta * fl32(180 / pi)) * fl32(pi)) / 180).  The
// slice kernel uses that angle; cos and sin are taken in FP64.
//
// Z of two connected trees is connected, so shapely returns one polygon and
// the reference measures to its exterior ring; the distance here is to the
// whole union boundary.  The two differ only where Z has a hole.
#pragma once
#include "common.cuh"

#define PK_MK_REGIONS 16
#define PK_MK_MAXV 16         // hull vertices per region (a hull of 16 points)
#define PK_MK_MAXSEG 2048     // union-boundary pieces per slice
#define PK_MK_TILE 16         // grid points per tile side
#define PK_MK_BATCH 256       // slices per batch of the builder

struct PkMkSlice {
    int nseg;
    int nv[PK_MK_REGIONS];
    double4 bbox[PK_MK_REGIONS];              // (xmin, xmax, ymin, ymax) per hull
    double2 v[PK_MK_REGIONS][PK_MK_MAXV];     // CCW hull vertices
    double4 seg[PK_MK_MAXSEG];                // (ax, ay, bx, by)
};

// (a - o) x (b - o), each operation rounded on its own
__device__ __forceinline__ double pk_mk_cross(double2 o, double2 a, double2 b)
{
    return __dsub_rn(__dmul_rn(__dsub_rn(a.x, o.x), __dsub_rn(b.y, o.y)),
                     __dmul_rn(__dsub_rn(a.y, o.y), __dsub_rn(b.x, o.x)));
}

// Convex hull (CCW, collinear points dropped) of n <= 16 points into out
// (PK_MK_MAXV entries); returns the vertex count, or -1 if it would not fit.
__device__ int pk_mk_hull(double2* pts, int n, double2* out)
{
    for (int i = 1; i < n; ++i) {   // lexicographic insertion sort
        const double2 p = pts[i];
        int j = i - 1;
        while (j >= 0 && (pts[j].x > p.x || (pts[j].x == p.x && pts[j].y > p.y))) {
            pts[j + 1] = pts[j];
            --j;
        }
        pts[j + 1] = p;
    }
    double2 H[2 * 16 + 1];
    int k = 0;
    for (int i = 0; i < n; ++i) {
        while (k >= 2 && pk_mk_cross(H[k - 2], H[k - 1], pts[i]) <= 0.0) --k;
        H[k++] = pts[i];
    }
    for (int i = n - 2, t = k + 1; i >= 0; --i) {
        while (k >= t && pk_mk_cross(H[k - 2], H[k - 1], pts[i]) <= 0.0) --k;
        H[k++] = pts[i];
    }
    const int m = k > 1 ? k - 1 : k;
    if (m > PK_MK_MAXV) return -1;
    for (int i = 0; i < m; ++i) out[i] = H[i];
    return m;
}

// The rotation angle the reference's shapely call applies for a float32 theta.
__device__ __forceinline__ double pk_mk_angle(float theta)
{
    const float deg = __fmul_rn(theta, 57.295776f);            // np.degrees on float32
    return (double)__fdiv_rn(__fmul_rn(deg, 3.1415927f), 180.0f);
}

__global__ void __launch_bounds__(128) pk_mk_slice_kernel(const float* __restrict__ theta, int nt,
                                                          PkMkSlice* __restrict__ slices, int* __restrict__ overflow)
{
    __shared__ double2 sv[PK_MK_REGIONS][PK_MK_MAXV];
    __shared__ int snv[PK_MK_REGIONS];
    __shared__ int scount;
    const int it = blockIdx.x;
    if (it >= nt) return;
    PkMkSlice* S = slices + it;
    if (threadIdx.x == 0) scount = 0;
    if (threadIdx.x < PK_MK_REGIONS) {
        double sn, cs;
        sincos(pk_mk_angle(theta[it]), &sn, &cs);
        const int p = threadIdx.x >> 2, q = threadIdx.x & 3;
        const int np = c_geom64.piece_nv[p], nq = c_geom64.piece_nv[q];
        double2 pts[16];
        int n = 0;
        for (int i = 0; i < np; ++i)
            for (int j = 0; j < nq; ++j) {
                const double2 a = c_geom64.piece[p][i], b = c_geom64.piece[q][j];
                const double bx = __dsub_rn(__dmul_rn(cs, b.x), __dmul_rn(sn, b.y));
                const double by = __dadd_rn(__dmul_rn(sn, b.x), __dmul_rn(cs, b.y));
                pts[n++] = make_double2(__dsub_rn(a.x, bx), __dsub_rn(a.y, by));
            }
        double2 hv[PK_MK_MAXV];
        int m = pk_mk_hull(pts, n, hv);
        if (m < 0) {
            atomicOr(overflow, 1);
            m = 0;
        }
        snv[threadIdx.x] = m;
        double4 bb = make_double4(1e300, -1e300, 1e300, -1e300);
        for (int i = 0; i < PK_MK_MAXV; ++i) {
            const double2 w = i < m ? hv[i] : make_double2(0.0, 0.0);
            sv[threadIdx.x][i] = w;
            S->v[threadIdx.x][i] = w;
            if (i < m) {
                bb.x = fmin(bb.x, w.x); bb.y = fmax(bb.y, w.x);
                bb.z = fmin(bb.z, w.y); bb.w = fmax(bb.w, w.y);
            }
        }
        S->nv[threadIdx.x] = m;
        S->bbox[threadIdx.x] = bb;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < PK_MK_REGIONS * PK_MK_MAXV; e += blockDim.x) {
        const int r = e / PK_MK_MAXV, k = e % PK_MK_MAXV;
        if (k >= snv[r]) continue;
        const double2 a = sv[r][k], b = sv[r][k + 1 < snv[r] ? k + 1 : 0];
        // open parameter intervals of a + s (b - a) strictly inside the other hulls
        double lo[PK_MK_REGIONS], hi[PK_MK_REGIONS];
        int ni = 0;
        for (int o = 0; o < PK_MK_REGIONS; ++o) {
            if (o == r || snv[o] < 3) continue;
            double l = 0.0, h = 1.0;
            bool empty = false;
            for (int j = 0; j < snv[o] && !empty; ++j) {
                const double2 u = sv[o][j], w = sv[o][j + 1 < snv[o] ? j + 1 : 0];
                const double f0 = pk_mk_cross(u, w, a), f1 = pk_mk_cross(u, w, b);
                if (f0 <= 0.0 && f1 <= 0.0) empty = true;
                else if (f0 > 0.0 && f1 <= 0.0) h = fmin(h, __ddiv_rn(f0, __dsub_rn(f0, f1)));
                else if (f0 <= 0.0 && f1 > 0.0) l = fmax(l, __ddiv_rn(f0, __dsub_rn(f0, f1)));
                if (l >= h) empty = true;
            }
            if (!empty) { lo[ni] = l; hi[ni] = h; ++ni; }
        }
        for (int i = 1; i < ni; ++i) {   // intervals by start
            const double l = lo[i], h = hi[i];
            int j = i - 1;
            while (j >= 0 && lo[j] > l) { lo[j + 1] = lo[j]; hi[j + 1] = hi[j]; --j; }
            lo[j + 1] = l;
            hi[j + 1] = h;
        }
        // walk [0, 1] and keep the uncovered pieces
        const double dx = __dsub_rn(b.x, a.x), dy = __dsub_rn(b.y, a.y);
        double cur = 0.0;
        for (int i = 0; i <= ni; ++i) {
            const double nxt = i < ni ? lo[i] : 1.0;
            if (nxt > cur) {
                const int slot = atomicAdd(&scount, 1);
                if (slot < PK_MK_MAXSEG)
                    S->seg[slot] = make_double4(cur == 0.0 ? a.x : __dadd_rn(a.x, __dmul_rn(cur, dx)),
                                                cur == 0.0 ? a.y : __dadd_rn(a.y, __dmul_rn(cur, dy)),
                                                nxt == 1.0 ? b.x : __dadd_rn(a.x, __dmul_rn(nxt, dx)),
                                                nxt == 1.0 ? b.y : __dadd_rn(a.y, __dmul_rn(nxt, dy)));
            }
            if (i < ni) cur = fmax(cur, hi[i]);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        S->nseg = scount < PK_MK_MAXSEG ? scount : PK_MK_MAXSEG;
        if (scount > PK_MK_MAXSEG) atomicOr(overflow, 1);
    }
}

// squared distance from t to the segment s, each operation rounded on its own
__device__ __forceinline__ double pk_mk_seg_d2(double2 t, double4 s)
{
    const double ex = __dsub_rn(s.z, s.x), ey = __dsub_rn(s.w, s.y);
    const double px = __dsub_rn(t.x, s.x), py = __dsub_rn(t.y, s.y);
    const double ll = __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey));
    const double pe = __dadd_rn(__dmul_rn(px, ex), __dmul_rn(py, ey));
    double u = ll > 0.0 ? __ddiv_rn(pe, ll) : 0.0;
    u = fmin(fmax(u, 0.0), 1.0);
    const double qx = __dsub_rn(px, __dmul_rn(u, ex)), qy = __dsub_rn(py, __dmul_rn(u, ey));
    return __dadd_rn(__dmul_rn(qx, qx), __dmul_rn(qy, qy));
}

// minimum over the block (blockDim.x / 32 <= 8 warps); every thread gets it
__device__ __forceinline__ double pk_mk_block_min(double v, double* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(PK_FULL_MASK, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double r = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmin(r, red[w]);
    __syncthreads();
    return r;
}

// blockIdx.y = slice of the batch; the CTAs of a slice stride over its tiles.
// vals points at the table entry (0, 0, first slice of the batch); the slice
// index is the fastest of the table's axes, nt entries apart.
__global__ void __launch_bounds__(256) pk_mk_grid_kernel(const float* __restrict__ X, int nx,
                                                         const float* __restrict__ Y, int ny,
                                                         const PkMkSlice* __restrict__ slices, int nt,
                                                         float* __restrict__ vals)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    double4* seg = (double4*)pk_smem;                                    // PK_MK_MAXSEG
    unsigned short* keep = (unsigned short*)(seg + PK_MK_MAXSEG);        // PK_MK_MAXSEG
    __shared__ double2 sv[PK_MK_REGIONS][PK_MK_MAXV];
    __shared__ double4 sbb[PK_MK_REGIONS];
    __shared__ int snv[PK_MK_REGIONS];
    __shared__ double red[8];
    __shared__ double4 rect;
    __shared__ int nkeep;
    __shared__ unsigned hmask;
    const PkMkSlice* S = slices + blockIdx.y;
    const int nseg = S->nseg;
    for (int i = threadIdx.x; i < nseg; i += blockDim.x) seg[i] = S->seg[i];
    for (int i = threadIdx.x; i < PK_MK_REGIONS * PK_MK_MAXV; i += blockDim.x)
        sv[i / PK_MK_MAXV][i % PK_MK_MAXV] = S->v[i / PK_MK_MAXV][i % PK_MK_MAXV];
    if (threadIdx.x < PK_MK_REGIONS) {
        snv[threadIdx.x] = S->nv[threadIdx.x];
        sbb[threadIdx.x] = S->bbox[threadIdx.x];
    }
    const int tx = (nx + PK_MK_TILE - 1) / PK_MK_TILE, ty = (ny + PK_MK_TILE - 1) / PK_MK_TILE;
    const int lx = threadIdx.x / PK_MK_TILE, ly = threadIdx.x % PK_MK_TILE;
    for (int tile = blockIdx.x; tile < tx * ty; tile += gridDim.x) {
        const int ix0 = (tile / ty) * PK_MK_TILE, iy0 = (tile % ty) * PK_MK_TILE;
        __syncthreads();   // the previous tile is done with rect, keep and hmask
        if (threadIdx.x < 32) {
            // lanes 0-15 read the tile's X values, lanes 16-31 its Y values;
            // min and max within each half by shuffles
            const int l = threadIdx.x & 15;
            const bool isx = threadIdx.x < 16;
            const int idx = (isx ? ix0 : iy0) + l;
            const bool ok = idx < (isx ? nx : ny);
            const double v = ok ? (double)(isx ? X[idx] : Y[idx]) : 0.0;
            double lo = ok ? v : 1e300, hi = ok ? v : -1e300;
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) {
                lo = fmin(lo, __shfl_xor_sync(PK_FULL_MASK, lo, o));
                hi = fmax(hi, __shfl_xor_sync(PK_FULL_MASK, hi, o));
            }
            const double ylo = __shfl_sync(PK_FULL_MASK, lo, 16), yhi = __shfl_sync(PK_FULL_MASK, hi, 16);
            if (threadIdx.x == 0) {
                rect = make_double4(lo, hi, ylo, yhi);
                nkeep = 0;
                hmask = 0u;
            }
        }
        __syncthreads();
        const double4 r = rect;
        const double2 c = make_double2(0.5 * (r.x + r.y), 0.5 * (r.z + r.w));
        const double hd = 0.5 * sqrt((r.y - r.x) * (r.y - r.x) + (r.w - r.z) * (r.w - r.z));
        if (threadIdx.x < PK_MK_REGIONS) {
            const double4 b = sbb[threadIdx.x];
            if (snv[threadIdx.x] >= 3 && !(b.y < r.x || r.y < b.x || b.w < r.z || r.w < b.z))
                atomicOr(&hmask, 1u << threadIdx.x);
        }
        // pieces whose distance from the centre is within the tile diagonal of the smallest
        double dmin = 1e300;
        for (int i = threadIdx.x; i < nseg; i += blockDim.x) dmin = fmin(dmin, pk_mk_seg_d2(c, seg[i]));
        dmin = sqrt(pk_mk_block_min(dmin, red));
        const double lim = dmin + 2.0 * hd + 1e-9;
        const double lim2 = lim * lim;
        for (int i = threadIdx.x; i < nseg; i += blockDim.x)
            if (pk_mk_seg_d2(c, seg[i]) <= lim2) keep[atomicAdd(&nkeep, 1)] = (unsigned short)i;
        __syncthreads();
        const int ix = ix0 + lx, iy = iy0 + ly;
        if (ix < nx && iy < ny) {
            const double2 t = make_double2((double)X[ix], (double)Y[iy]);
            bool inside = false;
            unsigned mk = hmask;
            while (mk && !inside) {
                const int h = __ffs(mk) - 1;
                mk &= mk - 1;
                const double4 b = sbb[h];
                if (t.x <= b.x || t.x >= b.y || t.y <= b.z || t.y >= b.w) continue;
                bool in = true;
                const int m = snv[h];
                for (int j = 0; j < m && in; ++j) in = pk_mk_cross(sv[h][j], sv[h][j + 1 < m ? j + 1 : 0], t) > 0.0;
                inside = in;
            }
            double best = 1e300;
            const int nk = nkeep;
            for (int i = 0; i < nk; ++i) best = fmin(best, pk_mk_seg_d2(t, seg[keep[i]]));
            const double dist = nseg > 0 ? __dsqrt_rn(best) : 0.0;
            vals[((size_t)ix * ny + iy) * nt + blockIdx.y] = (float)(inside ? dist : -dist);
        }
    }
}

static size_t pk_mk_grid_smem() { return (sizeof(double4) + sizeof(unsigned short)) * PK_MK_MAXSEG; }

// Table vals[ix, iy, it] (float32, C order) of the signed separation over the
// grid X x Y x T.  Synchronises the stream before it returns.
extern "C" int pk_lut_build_exact_sep(const float* X, int nx, const float* Y, int ny, const float* T, int nt,
                                      float* vals, void* stream)
{
    int rc = pk_check_init();
    if (rc) return rc;
    if (nx < 1 || ny < 1 || nt < 1) return pk_fail(PK_EINVAL, "pk_lut_build_exact_sep: empty grid%s");
    if (!X || !Y || !T || !vals) return pk_fail(PK_EINVAL, "pk_lut_build_exact_sep: NULL pointer%s");
    cudaStream_t st = (cudaStream_t)stream;
    const int batch = nt < PK_MK_BATCH ? nt : PK_MK_BATCH;
    const size_t slice_bytes = sizeof(PkMkSlice) * (size_t)batch;
    unsigned char* buf = nullptr;
    cudaError_t err = cudaMallocAsync((void**)&buf, slice_bytes + 16, st);
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_lut_build_exact_sep allocation");
    PkMkSlice* sl = (PkMkSlice*)buf;
    int* overflow = (int*)(buf + slice_bytes);
    err = cudaMemsetAsync(overflow, 0, sizeof(int), st);
    const size_t smem = pk_mk_grid_smem();
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(pk_mk_grid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long long tiles = (long long)((nx + PK_MK_TILE - 1) / PK_MK_TILE) * ((ny + PK_MK_TILE - 1) / PK_MK_TILE);
    const int per_slice = (int)(tiles < 64 ? tiles : 64);   // 256 slices x 64 CTAs fill the GPU many times over
    for (int t0 = 0; t0 < nt && err == cudaSuccess; t0 += batch) {
        const int nb = nt - t0 < batch ? nt - t0 : batch;
        pk_mk_slice_kernel<<<nb, 128, 0, st>>>(T + t0, nb, sl, overflow);
        pk_mk_grid_kernel<<<dim3(per_slice, nb), 256, smem, st>>>(X, nx, Y, ny, sl, nt, vals + t0);
        err = cudaGetLastError();
    }
    int ov = 0;
    if (err == cudaSuccess) err = cudaMemcpyAsync(&ov, overflow, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    const cudaError_t e2 = cudaFreeAsync(buf, st);
    if (err == cudaSuccess) err = e2;
    if (err != cudaSuccess) return pk_cuda_check(err, "pk_lut_build_exact_sep");
    if (ov) return pk_fail(PK_ERANGE, "pk_lut_build_exact_sep: a slice's hulls or boundary pieces overflowed their buffers%s");
    return PK_OK;
}
