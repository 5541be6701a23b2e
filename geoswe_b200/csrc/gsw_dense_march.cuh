// gsw_dense_march.cuh -- the dense column-march step kernel and its launcher.
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
//
// Included by gsw_dense.cu (exact arithmetic) and gsw_fast.cu (fast arithmetic, with
// namespace gsw renamed), so each compilation has its own kernels.
#pragma once
#include "gsw_common.cuh"

namespace gsw {

template <typename T>
struct DenseK {
    const T* q0; const T* q1; const T* q2;
    T* o0; T* o1; T* o2;
    const T* b;
    const uint8_t* mask; int64_t mpitch;
    int nxp, nyp, lo;            // cells [lo, n-lo) may be computed (lo = ngh, or 2 for the residual)
    int row_lo, row_hi, col_lo, col_hi;   // the window computed, inside [lo, n-lo)
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
    T g_recip;                   // RN(1/g) for the star depth's h / g, or 0 (gsw_core.cuh div_g)
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
    r.wet = true;   // unused: the residual adds a dry face's zeros
    return r;
}

template <typename T>
__device__ __forceinline__ T dt_of(const GswLoopState* st);
template <> __device__ __forceinline__ float  dt_of<float>(const GswLoopState* st)  { return st->dt_f32; }
template <> __device__ __forceinline__ double dt_of<double>(const GswLoopState* st) { return st->dt; }

// STEP = false: residual into o0..o2. STEP = true: updated state into o0..o2.
// REFPOW: Manning's h^(-4/3) by powf (GSW_ARITH_EXACT) instead of pow_m43.
// LEAN: the kernel of the production configuration (no inside mask, no CFL skip mask,
// the wave speed reduced, a Manning class table, quadratic friction, keep-h; rain none
// or uniform), with those choices compiled in rather than tested per cell: 6 % of the
// 8192^2 step. Any other configuration takes the general kernel; both give the same bits.
template <typename T, bool STEP, int MINB, bool REFPOW, bool LEAN>
__global__ void __launch_bounds__(256, MINB) dense_march_kernel(DenseK<T> p) {
    if (STEP && p.st->done) return;                       // grid-uniform
    const int lane = threadIdx.x;
    const int strip = blockIdx.x * blockDim.y + threadIdx.y;
    const int jend = p.col_hi;
    const int col0 = p.col_lo + strip * 30;
    const bool warp_active = col0 < jend;
    const int c = col0 - 1 + lane;
    const int cl = min(c, p.nyp - 1);
    const bool out_lane = warp_active && lane >= 1 && lane <= 30 && c < jend;
    const int i0 = p.row_lo + blockIdx.y * p.tile_rows;
    const int i1 = min(i0 + p.tile_rows, p.row_hi);
    unsigned long long lam_local = 0ull;
    uint32_t lam32 = 0u;        // binary32: the bits of the largest wave speed (lam_dense_bits32)

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
        srm_face<T, true>(cur, nx, p.half_dx, p.inv_dx, p.g, p.h_min, Wf, p.g_recip);
        cur = nx;

#ifdef GSW_FAST_ARITH
#pragma unroll 2      // two rows in flight: 1.76 -> 1.62 ms at 8192^2 fast (the exact step, and the
                      // flat march with either arithmetic, slow down)
#endif
        for (int r = i0; r < i1; ++r) {
            // the update's class id and running maximum, loaded before the faces so that
            // their latency is hidden (the production kernel; the general one loads late)
            uint8_t cls_r = 0;
            T mh_r = (T)0;
            if (LEAN && STEP && out_lane) {
                cls_r = p.ncls[(int64_t)r * p.cpitch + c];
                if (p.max_h != nullptr) mh_r = p.max_h[(int64_t)r * p.pitch + c];
            }
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
            srm_face<T, true>(cur, nx, p.half_dx, p.inv_dx, p.g, p.h_min, Ef, p.g_recip);
            // the residual in the reference's order (E, W, N, S per component; accumulate() in
            // gsw_core.cuh), the E and W parts before the y-face so that W is released early.
            // A dry face (skipped by the reference) holds +0 in every field, and adding or
            // subtracting +0 leaves these sums unchanged: they start at +0 and are never -0
            // (an IEEE sum or difference is -0 only from a -0 left operand; the fast
            // compilation's flush to zero can make one, whose sign may then differ), so no test of
            // the wet flag is needed.
            T rh = (T)0, rhu = (T)0, rhv = (T)0;
            rh = rh - Ef.Fh; rhu = rhu - Ef.Fn; rhv = rhv - Ef.Ft; rhu = rhu - Ef.srcL;
            rh = rh + Wf.Fh; rhu = rhu + Wf.Fn; rhv = rhv + Wf.Ft; rhu = rhu + Wf.srcR;
            Wf = Ef;
            const Cell<T> rn = shfl_cell_down(cur);
            {
                Face<T> Nf;
                srm_face<T, false>(cur, rn, p.half_dy, p.inv_dy, p.g, p.h_min, Nf, p.g_recip);
                const Face<T> Sf = shfl_face_up(Nf);
                rh = rh - Nf.Fh; rhu = rhu - Nf.Ft; rhv = rhv - Nf.Fn; rhv = rhv - Nf.srcL;
                rh = rh + Sf.Fh; rhu = rhu + Sf.Ft; rhv = rhv + Sf.Fn; rhv = rhv + Sf.srcR;
            }

            if (out_lane) {
                const bool inside = LEAN || (p.mask == nullptr) || (p.mask[(int64_t)r * p.mpitch + c] != 0);
                if (!inside) { rh = (T)0; rhu = (T)0; rhv = (T)0; }
                const int64_t o = (int64_t)r * p.pitch + c;
                if (!STEP) {
                    p.o0[o] = rh; p.o1[o] = rhu; p.o2[o] = rhv;
                } else {
                    T rr0 = rh;
                    if (inside) {
                        if (p.rain_kind == GSW_RAIN_UNIFORM) rr0 = rh + rate;
                        else if (!LEAN && p.rain_kind == GSW_RAIN_GRIDDED)
                            rr0 = rh + frame[(int64_t)(r - p.ngh) * (p.nyp - 2 * p.ngh) + (c - p.ngh)];
                    }
                    T h = cur.h + dt * rr0;
                    T hu = ldg_at(p.q1, p.pitch, r, c) + dt * rhu;     // reloaded: not carried down the march
                    T hv = ldg_at(p.q2, p.pitch, r, c) + dt * rhv;
                    T n = (T)0;
                    if (LEAN) n = p.ntab[cls_r];
                    else if (p.friction_kind == GSW_FRICTION_TABLE)
                        n = p.ncls ? p.ntab[p.ncls[(int64_t)r * p.cpitch + c]] : p.ntab[0];
                    else if (p.friction_kind == GSW_FRICTION_FIELD) n = p.nfield[o];
                    wetdry_friction<T>(h, hu, hv, LEAN || p.friction_kind != GSW_FRICTION_NONE, n, dt, p.g,
                                       p.h_min, p.vcap, LEAN || p.quad != 0, LEAN || p.keep_h != 0, REFPOW);
                    p.o0[o] = h; p.o1[o] = hu; p.o2[o] = hv;
                    if (LEAN) { if (p.max_h != nullptr && h > mh_r) p.max_h[o] = h; }
                    else if (p.max_h != nullptr && h > p.max_h[o]) p.max_h[o] = h;
                    if (LEAN || p.lam != nullptr) {
                        const bool skip = !LEAN && (p.cfl_skip != nullptr) &&
                            p.cfl_skip[(int64_t)(r - p.ngh) * (p.nyp - 2 * p.ngh) + (c - p.ngh)] != 0;
                        if (!skip) {
                            if constexpr (sizeof(T) == 4) {
                                lam32 = max(lam32, lam_dense_bits32(h, hu, hv, p.g, p.h_cfl));
                            } else {
                                const unsigned long long lb = lam_dense_bits(h, hu, hv, p.g, p.h_cfl);
                                lam_local = lb > lam_local ? lb : lam_local;
                            }
                        }
                    }
                }
            }
            cur = nx;
            b_next = b_p2;
        }
    }
    if constexpr (sizeof(T) == 4) lam_local = lam_bits_of32(lam32);
    if (STEP && (LEAN || p.lam != nullptr)) block_max_to(lam_local, p.lam);
}

template <typename T>
inline int fill_dense(const GswDenseArgs* a, DenseK<T>& k, bool step) {
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
    // the window: 0 at both ends of an axis is the whole range
    k.row_lo = (a->row_lo == 0 && a->row_hi == 0) ? k.lo : a->row_lo;
    k.row_hi = (a->row_lo == 0 && a->row_hi == 0) ? a->nxp - k.lo : a->row_hi;
    k.col_lo = (a->col_lo == 0 && a->col_hi == 0) ? k.lo : a->col_lo;
    k.col_hi = (a->col_lo == 0 && a->col_hi == 0) ? a->nyp - k.lo : a->col_hi;
    if (k.row_lo < k.lo || k.row_hi > a->nxp - k.lo || k.row_lo >= k.row_hi ||
        k.col_lo < k.lo || k.col_hi > a->nyp - k.lo || k.col_lo >= k.col_hi)
        return set_error(GSW_ERR_INVALID, "dense: window rows [%d, %d) x columns [%d, %d) is empty or leaves "
                         "[%d, %d) x [%d, %d)", a->row_lo, a->row_hi, a->col_lo, a->col_hi, k.lo,
                         a->nxp - k.lo, k.lo, a->nyp - k.lo);
    k.inv_dx = (T)a->inv_dx; k.inv_dy = (T)a->inv_dy;
    {   // dx = 1/inv_dx evaluated in T, as the reference kernel does (rhs_cuda.py:925-926)
        const T dx = (T)1 / k.inv_dx, dy = (T)1 / k.inv_dy;
        k.half_dx = (T)0.5 * dx; k.half_dy = (T)0.5 * dy;
    }
    if (!(a->h_min > 0.0) || !(a->h_cfl > 0.0))     // both are divisor floors of the step
        return set_error(GSW_ERR_INVALID, "dense: h_min (%g) and h_cfl (%g) must be > 0", a->h_min, a->h_cfl);
    k.g = (T)a->g; k.h_min = (T)a->h_min;
    k.g_recip = sizeof(T) == 4 ? (T)div_const_recip((float)a->g) : (T)0;
    k.st = a->state; k.lam = (unsigned long long*)a->lam_target;
    k.rain_kind = a->rain_kind; k.rain = (const T*)a->rain;
    k.friction_kind = a->friction_kind; k.ncls = a->n_cls; k.cpitch = a->n_cls_pitch;
    k.ntab = (const T*)a->n_tab; k.nfield = (const T*)a->n_field;
    k.vcap = (T)a->vcap; k.quad = a->quadratic; k.keep_h = a->keep_h;
    k.max_h = (T*)a->max_h; k.cfl_skip = a->cfl_skip; k.h_cfl = (T)a->h_cfl;
    if (a->tile_rows > 0) {
        k.tile_rows = a->tile_rows;
    } else {   // rows per warp: the longest march (<= 32 rows) that still gives twice the resident warps
        const int64_t strips = (k.col_hi - k.col_lo + 29) / 30, nrows = k.row_hi - k.row_lo;
        const int64_t want = 2LL * sm_count() * 24;
        k.tile_rows = 4;
        for (int tr = 32; tr > 4; tr >>= 1)
            if (strips * ((nrows + tr - 1) / tr) >= want) { k.tile_rows = tr; break; }
    }
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

template <typename T, bool STEP, bool REFPOW, bool LEAN>
inline void launch_march_caps(const DenseK<T>& k, int minb, dim3 grid, dim3 block, cudaStream_t s) {
    // register caps apply to the binary32 step; the residual and binary64 use the compiler's choice
    constexpr bool capped = STEP && sizeof(T) == 4;
    if (capped && minb == 3) dense_march_kernel<T, STEP, capped ? 3 : 1, REFPOW, LEAN><<<grid, block, 0, s>>>(k);
    else if (capped && minb == 4) dense_march_kernel<T, STEP, capped ? 4 : 1, REFPOW, LEAN><<<grid, block, 0, s>>>(k);
    else if (capped && minb == 5) dense_march_kernel<T, STEP, capped ? 5 : 1, REFPOW, LEAN><<<grid, block, 0, s>>>(k);
    else dense_march_kernel<T, STEP, 1, REFPOW, LEAN><<<grid, block, 0, s>>>(k);
}

// The production configuration (the LEAN kernel) or the general kernel.
template <typename T>
inline bool lean_config(const DenseK<T>& k) {
    return k.mask == nullptr && k.cfl_skip == nullptr && k.lam != nullptr && k.friction_kind == GSW_FRICTION_TABLE &&
           k.ncls != nullptr && k.rain_kind != GSW_RAIN_GRIDDED && k.quad != 0 && k.keep_h != 0;
}

template <typename T, bool STEP, bool REFPOW>
inline void launch_march_shape(const DenseK<T>& k, int minb, dim3 grid, dim3 block, cudaStream_t s) {
    constexpr bool can_lean = STEP && sizeof(T) == 4;
    if (can_lean && lean_config(k)) launch_march_caps<T, STEP, REFPOW, can_lean>(k, minb, grid, block, s);
    else launch_march_caps<T, STEP, REFPOW, false>(k, minb, grid, block, s);
}

template <typename T, bool STEP>
inline int launch_march(const GswDenseArgs* a, cudaStream_t s) {
    DenseK<T> k;
    int rc = fill_dense<T>(a, k, STEP);
    if (rc) return rc;
    const int W = a->warps > 0 ? a->warps : 4;
    const int minb = a->min_blocks;
    if (minb != 0 && (minb < 3 || minb > 5)) return set_error(GSW_ERR_INVALID, "dense: min_blocks must be 0, 3, 4 or 5");
    if (W < 1 || W > 8) return set_error(GSW_ERR_INVALID, "dense: warps must be in [1, 8]");
    const int ncols = k.col_hi - k.col_lo, nrows = k.row_hi - k.row_lo;
    const int strips = (ncols + 29) / 30;
    dim3 block(32, W);
    dim3 grid((strips + W - 1) / W, (nrows + k.tile_rows - 1) / k.tile_rows);
    if (grid.y > 65535u) return set_error(GSW_ERR_INVALID, "dense: too many row tiles (%u); raise tile_rows", grid.y);
    constexpr bool can_refpow = kRefPowBuild && STEP && sizeof(T) == 4;
    if (can_refpow && a->arith == GSW_ARITH_EXACT) launch_march_shape<T, STEP, can_refpow>(k, minb, grid, block, s);
    else launch_march_shape<T, STEP, false>(k, minb, grid, block, s);
    return check_launch("dense_march");
}

}  // namespace gsw
