// gsw_dense.cu -- dense-grid kernels of the GeoSWE step for sm_100a and their C ABI.
//
// Column march. A warp owns a strip of 32 adjacent columns (lane = column, so every
// load of a row is one coalesced 128-byte access) and walks it down `tile_rows` rows.
// Lanes 1..30 are output columns, lanes 0 and 31 are the strip's halo columns.
//   * x-faces (between rows i and i+1) are computed once per row and carried down the
//     column in registers: the face below row i is the face above row i+1;
//   * y-faces (between columns) are computed once by the left lane and handed to the
//     right lane with one warp shuffle;
// so each face is evaluated once instead of twice, and no shared memory or block
// barrier is needed on the step path. The new state's wave speed is reduced in
// registers, then per block, then with one 64-bit atomicMax.
#include "gsw_common.cuh"

namespace gsw {

template <typename T>
struct DenseK {
    const T* q0; const T* q1; const T* q2;
    T* o0; T* o1; T* o2;
    const T* b;
    const uint8_t* mask; int64_t mpitch;
    int nxp, nyp, lo;            // cells [lo, n-lo) are computed (lo = ngh, or 2 for the residual)
    int ngh;
    int64_t pitch;
    T inv_dx, inv_dy, half_dx, half_dy, g, h_min;
    const GswLoopState* st;
    unsigned long long* lam;
    int rain_kind; const T* rain;
    int friction_kind; const uint8_t* ncls; int64_t cpitch; const T* ntab; const T* nfield;
    T vcap; int quad; int keep_h;
    T* max_h;
    const uint8_t* cfl_skip;
    T h_cfl;
    int tile_rows;
};

template <typename T>
__device__ __forceinline__ T ldg_at(const T* a, int64_t pitch, int i, int j) {
    return __ldg(a + (int64_t)i * pitch + j);
}

// Central y-gradient of the bed at (row, lane column): neighbours come from the
// adjacent lanes; the strip's edge lanes read their outer neighbour directly.
template <typename T>
__device__ __forceinline__ T grad_y(const DenseK<T>& p, T bc, int row, int c, int lane) {
    T bl = __shfl_up_sync(0xffffffffu, bc, 1);
    T br = __shfl_down_sync(0xffffffffu, bc, 1);
    if (lane == 0)  bl = ldg_at(p.b, p.pitch, row, max(c - 1, 0));
    if (lane == 31) br = ldg_at(p.b, p.pitch, row, min(c + 1, p.nyp - 1));
    return (T)0.5 * (br - bl) * p.inv_dy;
}

template <typename T>
__device__ __forceinline__ void load_cell(const DenseK<T>& p, Cell<T>& c, int row, int col) {
    c.h = ldg_at(p.q0, p.pitch, row, col);
    c.hu = ldg_at(p.q1, p.pitch, row, col);
    c.hv = ldg_at(p.q2, p.pitch, row, col);
}

template <typename T>
__device__ __forceinline__ Cell<T> shfl_cell_down(const Cell<T>& c) {
    Cell<T> r;
    r.h = __shfl_down_sync(0xffffffffu, c.h, 1);
    r.u = __shfl_down_sync(0xffffffffu, c.u, 1);
    r.v = __shfl_down_sync(0xffffffffu, c.v, 1);
    r.eta = __shfl_down_sync(0xffffffffu, c.eta, 1);
    r.b = __shfl_down_sync(0xffffffffu, c.b, 1);
    r.gy = __shfl_down_sync(0xffffffffu, c.gy, 1);
    r.gx = r.gy; r.hu = r.h; r.hv = r.h;   // unused by a y-face
    return r;
}

template <typename T>
__device__ __forceinline__ Face<T> shfl_face_up(const Face<T>& f) {
    Face<T> r;
    r.Fh = __shfl_up_sync(0xffffffffu, f.Fh, 1);
    r.Fn = __shfl_up_sync(0xffffffffu, f.Fn, 1);
    r.Ft = __shfl_up_sync(0xffffffffu, f.Ft, 1);
    r.srcR = __shfl_up_sync(0xffffffffu, f.srcR, 1);
    r.srcL = r.srcR;
    r.wet = __shfl_up_sync(0xffffffffu, (int)f.wet, 1) != 0;
    return r;
}

template <typename T>
__device__ __forceinline__ T dt_of(const GswLoopState* st);
template <> __device__ __forceinline__ float  dt_of<float>(const GswLoopState* st)  { return st->dt_f32; }
template <> __device__ __forceinline__ double dt_of<double>(const GswLoopState* st) { return st->dt; }

// STEP = false: residual into o0..o2. STEP = true: updated state into o0..o2.
template <typename T, bool STEP, int MINB>
__global__ void __launch_bounds__(256, MINB) dense_march_kernel(DenseK<T> p) {
    if (STEP && p.st->done) return;                       // grid-uniform
    const int lane = threadIdx.x;
    const int strip = blockIdx.x * blockDim.y + threadIdx.y;
    const int jend = p.nyp - p.lo;
    const int col0 = p.lo + strip * 30;
    const bool warp_active = col0 < jend;
    const int c = col0 - 1 + lane;
    const int cl = min(c, p.nyp - 1);
    const bool out_lane = warp_active && lane >= 1 && lane <= 30 && c < jend;
    const int i0 = p.lo + blockIdx.y * p.tile_rows;
    const int i1 = min(i0 + p.tile_rows, p.nxp - p.lo);
    unsigned long long lam_local = 0ull;

    T dt = (T)0;
    T rate = (T)0;
    const T* frame = nullptr;
    if (STEP) {
        dt = dt_of<T>(p.st);
        if (p.rain_kind == GSW_RAIN_UNIFORM) rate = p.rain[p.st->rain_idx];
        if (p.rain_kind == GSW_RAIN_GRIDDED)
            frame = p.rain + (int64_t)p.st->rain_idx * (int64_t)(p.nxp - 2 * p.ngh) * (p.nyp - 2 * p.ngh);
    }

    if (warp_active && i0 < i1) {
        Cell<T> cur, nx;
        const T b_m2 = ldg_at(p.b, p.pitch, i0 - 2, cl);
        load_cell(p, cur, i0 - 1, cl);
        cur.b = ldg_at(p.b, p.pitch, i0 - 1, cl);
        load_cell(p, nx, i0, cl);
        nx.b = ldg_at(p.b, p.pitch, i0, cl);
        T b_next = ldg_at(p.b, p.pitch, i0 + 1, cl);
        // prefetch of the row after next: its loads are in flight during this row's faces
        T pf_h = ldg_at(p.q0, p.pitch, i0 + 1, cl);
        T pf_hu = ldg_at(p.q1, p.pitch, i0 + 1, cl);
        T pf_hv = ldg_at(p.q2, p.pitch, i0 + 1, cl);
        T pf_b = ldg_at(p.b, p.pitch, i0 + 2, cl);
        make_prims(cur, p.h_min);
        make_prims(nx, p.h_min);
        cur.gx = (T)0.5 * (nx.b - b_m2) * p.inv_dx;
        cur.gy = (T)0;
        nx.gx = (T)0.5 * (b_next - cur.b) * p.inv_dx;
        nx.gy = grad_y(p, nx.b, i0, c, lane);
        Face<T> Wf;
        srm_face<T, true>(cur, nx, p.half_dx, p.inv_dx, p.g, p.h_min, Wf);
        cur = nx;

        for (int r = i0; r < i1; ++r) {
            nx.h = pf_h; nx.hu = pf_hu; nx.hv = pf_hv;
            nx.b = b_next;
            const T b_p2 = pf_b;
            if (r + 1 < i1) {           // rows r+2 / r+3 exist: the strip ends at i1 <= nxp - lo
                pf_h = ldg_at(p.q0, p.pitch, r + 2, cl);
                pf_hu = ldg_at(p.q1, p.pitch, r + 2, cl);
                pf_hv = ldg_at(p.q2, p.pitch, r + 2, cl);
                pf_b = ldg_at(p.b, p.pitch, r + 3, cl);
            }
            make_prims(nx, p.h_min);
            nx.gx = (T)0.5 * (b_p2 - cur.b) * p.inv_dx;
            nx.gy = grad_y(p, nx.b, r + 1, c, lane);

            Face<T> Ef;
            srm_face<T, true>(cur, nx, p.half_dx, p.inv_dx, p.g, p.h_min, Ef);
            const Cell<T> rn = shfl_cell_down(cur);
            Face<T> Nf;
            srm_face<T, false>(cur, rn, p.half_dy, p.inv_dy, p.g, p.h_min, Nf);
            const Face<T> Sf = shfl_face_up(Nf);

            if (out_lane) {
                T rh, rhu, rhv;
                accumulate(Ef, Wf, Nf, Sf, rh, rhu, rhv);
                const bool inside = (p.mask == nullptr) || (p.mask[(int64_t)r * p.mpitch + c] != 0);
                if (!inside) { rh = (T)0; rhu = (T)0; rhv = (T)0; }
                const int64_t o = (int64_t)r * p.pitch + c;
                if (!STEP) {
                    p.o0[o] = rh; p.o1[o] = rhu; p.o2[o] = rhv;
                } else {
                    T rr0 = rh;
                    if (inside) {
                        if (p.rain_kind == GSW_RAIN_UNIFORM) rr0 = rh + rate;
                        else if (p.rain_kind == GSW_RAIN_GRIDDED)
                            rr0 = rh + frame[(int64_t)(r - p.ngh) * (p.nyp - 2 * p.ngh) + (c - p.ngh)];
                    }
                    T h = cur.h + dt * rr0;
                    T hu = cur.hu + dt * rhu;
                    T hv = cur.hv + dt * rhv;
                    T n = (T)0;
                    if (p.friction_kind == GSW_FRICTION_TABLE)
                        n = p.ncls ? p.ntab[p.ncls[(int64_t)r * p.cpitch + c]] : p.ntab[0];
                    else if (p.friction_kind == GSW_FRICTION_FIELD) n = p.nfield[o];
                    wetdry_friction<T>(h, hu, hv, p.friction_kind != GSW_FRICTION_NONE, n, dt, p.g,
                                       p.h_min, p.vcap, p.quad != 0, p.keep_h != 0);
                    p.o0[o] = h; p.o1[o] = hu; p.o2[o] = hv;
                    if (p.max_h != nullptr && h > p.max_h[o]) p.max_h[o] = h;
                    if (p.lam != nullptr) {
                        const bool skip = (p.cfl_skip != nullptr) &&
                            p.cfl_skip[(int64_t)(r - p.ngh) * (p.nyp - 2 * p.ngh) + (c - p.ngh)] != 0;
                        if (!skip) {
                            const unsigned long long lb = lam_dense_bits(h, hu, hv, p.g, p.h_cfl);
                            lam_local = lb > lam_local ? lb : lam_local;
                        }
                    }
                }
            }
            Wf = Ef;
            cur = nx;
            b_next = b_p2;
        }
    }
    if (STEP && p.lam != nullptr) block_max_to(lam_local, p.lam);
}

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

template <typename T>
static int fill_dense(const GswDenseArgs* a, DenseK<T>& k, bool step) {
    if (a->nxp < 5 || a->nyp < 5 || a->ngh < 2 || 2 * a->ngh >= a->nxp || 2 * a->ngh >= a->nyp)
        return set_error(GSW_ERR_INVALID, "dense: need ngh >= 2 and a non-empty interior (nxp=%d nyp=%d ngh=%d)",
                         a->nxp, a->nyp, a->ngh);
    if (a->pitch < a->nyp) return set_error(GSW_ERR_INVALID, "dense: pitch %lld < nyp %d", (long long)a->pitch, a->nyp);
    if (!a->q0 || !a->q1 || !a->q2 || !a->qn0 || !a->qn1 || !a->qn2 || !a->bed)
        return set_error(GSW_ERR_INVALID, "dense: null state/output/bed pointer");
    if (a->inside_mask && a->mask_pitch < a->nyp) return set_error(GSW_ERR_INVALID, "dense: mask_pitch < nyp");
    k.q0 = (const T*)a->q0; k.q1 = (const T*)a->q1; k.q2 = (const T*)a->q2;
    k.o0 = (T*)a->qn0; k.o1 = (T*)a->qn1; k.o2 = (T*)a->qn2;
    k.b = (const T*)a->bed;
    k.mask = a->inside_mask; k.mpitch = a->mask_pitch;
    k.nxp = a->nxp; k.nyp = a->nyp; k.ngh = a->ngh; k.pitch = a->pitch;
    k.lo = step ? a->ngh : 2;
    k.inv_dx = (T)a->inv_dx; k.inv_dy = (T)a->inv_dy;
    {   // dx = 1/inv_dx evaluated in T, as the reference kernel does (rhs_cuda.py:925-926)
        const T dx = (T)1 / k.inv_dx, dy = (T)1 / k.inv_dy;
        k.half_dx = (T)0.5 * dx; k.half_dy = (T)0.5 * dy;
    }
    k.g = (T)a->g; k.h_min = (T)a->h_min;
    k.st = a->state; k.lam = (unsigned long long*)a->lam_target;
    k.rain_kind = a->rain_kind; k.rain = (const T*)a->rain;
    k.friction_kind = a->friction_kind; k.ncls = a->n_cls; k.cpitch = a->n_cls_pitch;
    k.ntab = (const T*)a->n_tab; k.nfield = (const T*)a->n_field;
    k.vcap = (T)a->vcap; k.quad = a->quadratic; k.keep_h = a->keep_h;
    k.max_h = (T*)a->max_h; k.cfl_skip = a->cfl_skip; k.h_cfl = (T)a->h_cfl;
    k.tile_rows = a->tile_rows > 0 ? a->tile_rows : 32;
    if (step) {
        if (!a->state) return set_error(GSW_ERR_INVALID, "dense step: state (GswLoopState*) is required");
        if (a->rain_kind != GSW_RAIN_NONE && a->rain_kind != GSW_RAIN_UNIFORM && a->rain_kind != GSW_RAIN_GRIDDED)
            return set_error(GSW_ERR_INVALID, "dense step: bad rain_kind %d", a->rain_kind);
        if (a->rain_kind != GSW_RAIN_NONE && !a->rain) return set_error(GSW_ERR_INVALID, "dense step: rain is NULL");
        if (a->friction_kind == GSW_FRICTION_TABLE && (!a->n_tab || a->n_tab_len < 1 ||
                                                        (a->n_cls && a->n_cls_pitch < a->nyp)))
            return set_error(GSW_ERR_INVALID, "dense step: table friction needs n_tab (and n_cls pitch >= nyp)");
        if (a->friction_kind == GSW_FRICTION_FIELD && !a->n_field)
            return set_error(GSW_ERR_INVALID, "dense step: field friction needs n_field");
        if (a->friction_kind < 0 || a->friction_kind > 2) return set_error(GSW_ERR_INVALID, "dense step: bad friction_kind");
    }
    return GSW_OK;
}

template <typename T, bool STEP>
static int launch_march(const GswDenseArgs* a, cudaStream_t s) {
    DenseK<T> k;
    int rc = fill_dense<T>(a, k, STEP);
    if (rc) return rc;
    const int W = a->warps > 0 ? a->warps : 4;
    const int minb = a->min_blocks;
    if (minb != 0 && minb != 4 && minb != 5) return set_error(GSW_ERR_INVALID, "dense: min_blocks must be 0, 4 or 5");
    if (W < 1 || W > 8) return set_error(GSW_ERR_INVALID, "dense: warps must be in [1, 8]");
    const int ncols = k.nyp - 2 * k.lo, nrows = k.nxp - 2 * k.lo;
    const int strips = (ncols + 29) / 30;
    dim3 block(32, W);
    dim3 grid((strips + W - 1) / W, (nrows + k.tile_rows - 1) / k.tile_rows);
    if (grid.y > 65535u) return set_error(GSW_ERR_INVALID, "dense: too many row tiles (%u); raise tile_rows", grid.y);
    if (minb == 0) dense_march_kernel<T, STEP, 1><<<grid, block, 0, s>>>(k);
    else if (minb == 4) dense_march_kernel<T, STEP, 4><<<grid, block, 0, s>>>(k);
    else dense_march_kernel<T, STEP, 5><<<grid, block, 0, s>>>(k);
    return check_launch("dense_march");
}

extern "C" int gsw_dense_step(const GswDenseArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
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
    return launch_march<T, false>(a, s);
}

extern "C" int gsw_dense_rhs(const GswDenseArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
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
