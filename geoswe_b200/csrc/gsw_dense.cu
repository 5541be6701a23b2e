// gsw_dense.cu -- dense-grid kernels of the GeoSWE step for sm_100a and their C ABI:
// the fused step and residual (the column march of gsw_dense_march.cuh), the standalone
// wave speed, the ghost fill, the stage boundary.
#include "gsw_dense_march.cuh"
#include "gsw_fast.h"

namespace gsw {

// Standalone wave speed of the current state over the interior (lammax_fp32_lean).
template <typename T>
__global__ void __launch_bounds__(256) dense_lammax_kernel(DenseK<T> p, unsigned long long* out) {
    const int nx = p.nxp - 2 * p.ngh, ny = p.nyp - 2 * p.ngh;
    const int64_t N = (int64_t)nx * ny;
    unsigned long long lam = 0ull;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < N;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (p.cfl_skip != nullptr && p.cfl_skip[k] != 0) continue;
        const int ix = (int)(k / ny), iy = (int)(k - (int64_t)ix * ny);
        const int64_t o = (int64_t)(ix + p.ngh) * p.pitch + (iy + p.ngh);
        const unsigned long long lb = lam_dense_bits(p.q0[o], p.q1[o], p.q2[o], p.g, p.h_cfl);
        lam = lb > lam ? lb : lam;
    }
    block_max_to(lam, out);
}

// Ghost fill (bc.py:50-172). apply_bc_2d fills the x faces over all columns, then the
// y faces over all rows, so a corner ends up as the y rule applied to the x-filled cell
// of its row. One launch computes every ghost directly from interior cells: x-ghost
// rows over interior columns, y-ghost columns over interior rows, and the corners by
// composing the two rules, which is what the two passes produce.
__device__ __forceinline__ int bc_src(int kind, int g, int n, int ngh) {
    // source index of ghost g along an axis of length n, for EXTRAPOLATE/WALL/PERIODIC
    if (g < ngh) {
        const int k = g;
        return kind == GSW_BC_WALL ? (2 * ngh - 1 - k) : kind == GSW_BC_PERIODIC ? (n - 2 * ngh + k) : ngh;
    }
    const int k = g - (n - ngh);
    return kind == GSW_BC_WALL ? (n - ngh - 1 - k) : kind == GSW_BC_PERIODIC ? (ngh + k) : (n - ngh - 1);
}

template <typename T>
__global__ void bc_fill_kernel(T* q0, T* q1, T* q2, int nxp, int nyp, int ngh, int64_t pitch,
                               int kxm, int kxp, int kym, int kyp, const GswLoopState* st) {
    if (st != nullptr && st->done) return;
    const int nyi = nyp - 2 * ngh, nxi = nxp - 2 * ngh;
    const int64_t nX = (int64_t)2 * ngh * nyi;      // x-ghost cells at interior columns
    const int64_t nY = (int64_t)2 * ngh * nxi;      // y-ghost cells at interior rows
    const int64_t nC = (int64_t)4 * ngh * ngh;      // corners
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nX + nY + nC;
         t += (int64_t)gridDim.x * blockDim.x) {
        int gi, gj, kx = GSW_BC_NONE, ky = GSW_BC_NONE;
        if (t < nX) {
            const int side = (int)(t / ((int64_t)ngh * nyi));
            const int64_t rem = t - (int64_t)side * ngh * nyi;
            const int k = (int)(rem / nyi);
            gj = ngh + (int)(rem - (int64_t)k * nyi);
            gi = side == 0 ? k : nxp - ngh + k;
            kx = side == 0 ? kxm : kxp;
        } else if (t < nX + nY) {
            const int64_t u = t - nX;
            const int side = (int)(u / ((int64_t)ngh * nxi));
            const int64_t rem = u - (int64_t)side * ngh * nxi;
            const int k = (int)(rem / nxi);
            gi = ngh + (int)(rem - (int64_t)k * nxi);
            gj = side == 0 ? k : nyp - ngh + k;
            ky = side == 0 ? kym : kyp;
            if (ky == GSW_BC_NONE) continue;
        } else {
            const int64_t u = t - nX - nY;
            const int c = (int)(u / ((int64_t)ngh * ngh));
            const int rem = (int)(u - (int64_t)c * ngh * ngh);
            const int a = rem / ngh, bb = rem - a * ngh;
            gi = (c & 1) ? nxp - ngh + a : a;
            gj = (c & 2) ? nyp - ngh + bb : bb;
            kx = (c & 1) ? kxp : kxm;
            ky = (c & 2) ? kyp : kym;
            if (ky == GSW_BC_NONE && kx == GSW_BC_NONE) continue;
        }
        const int64_t go = (int64_t)gi * pitch + gj;
        // value of the x pass at (row gi, column cj)
        auto xval = [&](int cj, T& a, T& u, T& v) {
            if (kx == GSW_BC_NONE) { const int64_t o = (int64_t)gi * pitch + cj; a = q0[o]; u = q1[o]; v = q2[o]; return; }
            if (kx == GSW_BC_FALL) { a = (T)0; u = (T)0; v = (T)0; return; }
            const int64_t o = (int64_t)bc_src(kx, gi, nxp, ngh) * pitch + cj;
            a = q0[o]; u = q1[o]; v = q2[o];
            if (kx == GSW_BC_WALL) u = -u;
        };
        T a, u, v;
        if (t < nX) {
            xval(gj, a, u, v);
            if (kx == GSW_BC_NONE) continue;
        } else if (ky == GSW_BC_NONE) {            // corner left to the x pass
            xval(gj, a, u, v);
        } else if (ky == GSW_BC_FALL) {
            a = (T)0; u = (T)0; v = (T)0;
        } else {
            const int sj = bc_src(ky, gj, nyp, ngh);
            if (t < nX + nY) {
                const int64_t o = (int64_t)gi * pitch + sj;
                a = q0[o]; u = q1[o]; v = q2[o];
            } else {
                xval(sj, a, u, v);
            }
            if (ky == GSW_BC_WALL) v = -v;
        }
        q0[go] = a; q1[go] = u; q2[go] = v;
    }
}

// Stage boundary (forcing.py:315-377): eta(t_new) by clamped linear interpolation.
__device__ __forceinline__ double stage_eta(const double* ts, const double* ss, int n, double t) {
    if (t <= ts[0]) return ss[0];
    if (t >= ts[n - 1]) return ss[n - 1];
    int lo = 0, hi = n;                   // bisect_left
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (ts[mid] < t) lo = mid + 1; else hi = mid; }
    const int i = lo;
    const double t0 = ts[i - 1], t1 = ts[i], s0 = ss[i - 1], s1 = ss[i];
    const double w = __ddiv_rn(__dsub_rn(t, t0), __dsub_rn(t1, t0));
    return __dadd_rn(s0, __dmul_rn(w, __dsub_rn(s1, s0)));
}

template <typename T>
__global__ void stage_kernel(GswStageArgs a) {
    if (a.state->done) return;
    const double eta = stage_eta(a.time_s, a.stage_m, a.n_knots, a.state->t_new);
    T* q0 = (T*)a.q0; T* q1 = (T*)a.q1; T* q2 = (T*)a.q2;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_cells; k += gridDim.x * blockDim.x) {
        T hn;
        if (a.bed_is_f32) {
            const float d = (float)eta - (float)a.bed64[k];
            hn = (T)(d > 0.0f ? d : 0.0f);
        } else {
            const double d = eta - a.bed64[k];
            hn = (T)(d > 0.0 ? d : 0.0);
        }
        const int64_t o = a.cell_off[k];
        q0[o] = hn; q1[o] = (T)0; q2[o] = (T)0;
    }
}

// Fold the wave speed of listed cells into the loop's target (after all stage writes).
template <typename T>
__global__ void lam_cells_kernel(const T* q0, const T* q1, const T* q2, const int64_t* off, int n,
                                 const uint8_t* excl, T g, T h_cfl, unsigned long long* target,
                                 const GswLoopState* st) {
    if (st != nullptr && st->done) return;
    unsigned long long lam = 0ull;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (excl != nullptr && excl[k]) continue;
        const int64_t o = off[k];
        const unsigned long long lb = lam_dense_bits(q0[o], q1[o], q2[o], g, h_cfl);
        lam = lb > lam ? lb : lam;
    }
    block_max_to(lam, target);
}

}  // namespace gsw

using namespace gsw;

// Exact, portable or fast arithmetic; fast is binary32 only.
static int check_arith(const GswDenseArgs* a) {
    if (a->arith != GSW_ARITH_EXACT && a->arith != GSW_ARITH_FAST && a->arith != GSW_ARITH_PORTABLE)
        return set_error(GSW_ERR_INVALID, "dense: bad arith %d", a->arith);
    if (a->arith == GSW_ARITH_FAST && a->dtype != GSW_F32)
        return set_error(GSW_ERR_INVALID, "dense: fast arithmetic is binary32 only");
    return GSW_OK;
}

extern "C" int gsw_dense_step(const GswDenseArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_arith(a)) return rc;
    if (a->arith == GSW_ARITH_FAST) return gsw_fast_dense_launch(a, true, (cudaStream_t)stream);
    if (a->dtype == GSW_F32) return launch_march<float, true>(a, (cudaStream_t)stream);
    if (a->dtype == GSW_F64) return launch_march<double, true>(a, (cudaStream_t)stream);
    return set_error(GSW_ERR_INVALID, "dense step: bad dtype %d", a->dtype);
}

template <typename T>
static int launch_rhs(const GswDenseArgs* a, cudaStream_t s) {
    // cells outside the computed box (and ghost rows) read as 0
    const size_t rowb = (size_t)a->nyp * sizeof(T);
    for (void* o : {a->qn0, a->qn1, a->qn2}) {
        if (!o) return set_error(GSW_ERR_INVALID, "dense rhs: null output");
        if (cudaMemset2DAsync(o, (size_t)a->pitch * sizeof(T), 0, rowb, (size_t)a->nxp, s) != cudaSuccess)
            return set_error(GSW_ERR_CUDA, "dense rhs: cudaMemset2DAsync failed");
    }
    if (a->arith == GSW_ARITH_FAST) return gsw_fast_dense_launch(a, false, s);
    return launch_march<T, false>(a, s);
}

extern "C" int gsw_dense_rhs(const GswDenseArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_arith(a)) return rc;
    if (a->dtype == GSW_F32) return launch_rhs<float>(a, (cudaStream_t)stream);
    if (a->dtype == GSW_F64) return launch_rhs<double>(a, (cudaStream_t)stream);
    return set_error(GSW_ERR_INVALID, "dense rhs: bad dtype %d", a->dtype);
}

template <typename T>
static int launch_lammax(const GswDenseArgs* a, uint64_t* out, cudaStream_t s) {
    DenseK<T> k;
    int rc = fill_dense<T>(a, k, false);
    if (rc) return rc;
    if (!out) return set_error(GSW_ERR_INVALID, "lammax: null output");
    const int64_t N = (int64_t)(k.nxp - 2 * k.ngh) * (k.nyp - 2 * k.ngh);
    const int grid = (int)std::min<int64_t>(sm_count() * 8, (N + 255) / 256);
    dense_lammax_kernel<T><<<grid, 256, 0, s>>>(k, (unsigned long long*)out);
    return check_launch("dense_lammax");
}

extern "C" int gsw_dense_lammax(const GswDenseArgs* a, uint64_t* lam_bits, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->dtype == GSW_F32) return launch_lammax<float>(a, lam_bits, (cudaStream_t)stream);
    if (a->dtype == GSW_F64) return launch_lammax<double>(a, lam_bits, (cudaStream_t)stream);
    return set_error(GSW_ERR_INVALID, "lammax: bad dtype %d", a->dtype);
}

extern "C" int gsw_bc_fill(const GswBcArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->ngh < 1 || 2 * a->ngh >= a->nxp || 2 * a->ngh >= a->nyp || a->pitch < a->nyp)
        return set_error(GSW_ERR_INVALID, "bc: bad extents");
    for (int f = 0; f < 4; ++f)
        if (a->kinds[f] < 0 || a->kinds[f] > GSW_BC_NONE) return set_error(GSW_ERR_INVALID, "bc: bad kind %d", a->kinds[f]);
    const int64_t n = (int64_t)2 * a->ngh * (a->nyp - 2 * a->ngh) + (int64_t)2 * a->ngh * (a->nxp - 2 * a->ngh) +
                      (int64_t)4 * a->ngh * a->ngh;
    const int grid = (int)std::min<int64_t>(sm_count() * 4, (n + 255) / 256);
    cudaStream_t s = (cudaStream_t)stream;
    if (a->dtype == GSW_F32)
        bc_fill_kernel<float><<<grid, 256, 0, s>>>((float*)a->q0, (float*)a->q1, (float*)a->q2, a->nxp, a->nyp,
                                                   a->ngh, a->pitch, a->kinds[0], a->kinds[1], a->kinds[2],
                                                   a->kinds[3], a->state);
    else if (a->dtype == GSW_F64)
        bc_fill_kernel<double><<<grid, 256, 0, s>>>((double*)a->q0, (double*)a->q1, (double*)a->q2, a->nxp, a->nyp,
                                                    a->ngh, a->pitch, a->kinds[0], a->kinds[1], a->kinds[2],
                                                    a->kinds[3], a->state);
    else return set_error(GSW_ERR_INVALID, "bc: bad dtype");
    return check_launch("bc_fill");
}

extern "C" int gsw_stage_apply(const GswStageArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->n_cells <= 0) return GSW_OK;
    if (!a->cell_off || !a->bed64 || !a->time_s || !a->stage_m || a->n_knots < 1 || !a->state)
        return set_error(GSW_ERR_INVALID, "stage: null table or state");
    if (a->lam_target && !(a->h_cfl > 0.0))
        return set_error(GSW_ERR_INVALID, "stage: h_cfl (%g) must be > 0 (the wave speed's divisor floor)", a->h_cfl);
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = std::min(sm_count() * 4, (a->n_cells + 255) / 256);
    if (a->dtype == GSW_F32) stage_kernel<float><<<grid, 256, 0, s>>>(*a);
    else if (a->dtype == GSW_F64) stage_kernel<double><<<grid, 256, 0, s>>>(*a);
    else return set_error(GSW_ERR_INVALID, "stage: bad dtype");
    int rc = check_launch("stage");
    if (rc || !a->lam_target) return rc;
    if (a->dtype == GSW_F32)
        lam_cells_kernel<float><<<grid, 256, 0, s>>>((const float*)a->q0, (const float*)a->q1, (const float*)a->q2,
                                                     a->cell_off, a->n_cells, a->cfl_ghost, (float)a->g,
                                                     (float)a->h_cfl, (unsigned long long*)a->lam_target, a->state);
    else
        lam_cells_kernel<double><<<grid, 256, 0, s>>>((const double*)a->q0, (const double*)a->q1, (const double*)a->q2,
                                                      a->cell_off, a->n_cells, a->cfl_ghost, a->g, a->h_cfl,
                                                      (unsigned long long*)a->lam_target, a->state);
    return check_launch("stage_lam");
}

extern "C" int gsw_lam_cells(const GswStageArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->n_cells <= 0) return GSW_OK;
    if (!a->cell_off || !a->lam_target) return set_error(GSW_ERR_INVALID, "lam_cells: null list or target");
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = std::min(sm_count() * 4, (a->n_cells + 255) / 256);
    if (a->dtype == GSW_F32)
        lam_cells_kernel<float><<<grid, 256, 0, s>>>((const float*)a->q0, (const float*)a->q1, (const float*)a->q2,
                                                     a->cell_off, a->n_cells, a->cfl_ghost, (float)a->g,
                                                     (float)a->h_cfl, (unsigned long long*)a->lam_target, a->state);
    else if (a->dtype == GSW_F64)
        lam_cells_kernel<double><<<grid, 256, 0, s>>>((const double*)a->q0, (const double*)a->q1, (const double*)a->q2,
                                                      a->cell_off, a->n_cells, a->cfl_ghost, a->g, a->h_cfl,
                                                      (unsigned long long*)a->lam_target, a->state);
    else return set_error(GSW_ERR_INVALID, "lam_cells: bad dtype");
    return check_launch("lam_cells");
}
