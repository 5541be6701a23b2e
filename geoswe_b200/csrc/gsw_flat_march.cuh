// gsw_flat_march.cuh -- the fused step on the compressed (flat) mesh, brick storage:
// kernel and launcher.
//
// One warp per brick of 30 x brick_h cells, the same column march as the dense kernel
// (gsw_dense_march.cuh): lanes 1..30 are the brick's columns, lane 0 / lane 31 read the
// edge columns of the left / right brick, and the two rows above and below come from
// the bricks above and below. Every face is computed once from the shared core
// (gsw_core.cuh), so active-cell residuals are bit-identical to the dense kernel's.
//
// Included by gsw_flat.cu (exact arithmetic) and gsw_fast.cu (fast arithmetic, with
// namespace gsw renamed).
#pragma once
#include "gsw_flat_brick.cuh"

namespace gsw {

template <typename T, bool STEP, int MINB, bool REFPOW, bool LEAN>
__global__ void __launch_bounds__(256, MINB) flat_march_kernel(FlatK<T> p) {
    if (STEP && p.st->done) return;
    const int64_t item = (int64_t)blockIdx.x * blockDim.y + threadIdx.y;   // (brick, row segment)
    const int64_t rel = item / p.segs;
    const int seg = (int)(item - rel * p.segs);
    const int64_t bidx = p.b0 + rel;
    unsigned long long lam_local = 0ull;
    T dt = (T)0, rate = (T)0;
    const T* frame = nullptr;
    if (STEP) {
        dt = sizeof(T) == 4 ? (T)p.st->dt_f32 : (T)p.st->dt;
        if (p.ph.rain_kind == GSW_RAIN_UNIFORM) rate = p.ph.rain[p.st->rain_idx];
        if (p.ph.rain_kind == GSW_RAIN_GRIDDED) frame = p.ph.rain + (int64_t)p.st->rain_idx * p.ph.nx * p.ph.ny;
        if (p.ph.rain_kind == GSW_RAIN_LOOKUP) frame = p.ph.rain + (int64_t)p.st->rain_idx * p.ph.ncol;
    }
    if (bidx < p.b1)
        lam_local = flat_brick<T, STEP, REFPOW, LEAN>(p.m, p.ph, bidx, seg * p.m.bh / p.segs, (seg + 1) * p.m.bh / p.segs,
                                        dt, rate, frame);
    if (STEP && p.lam != nullptr) block_max_to(lam_local, p.lam);
}

template <typename T>
inline int fill_flat(const GswFlatArgs* a, FlatK<T>& k, bool step) {
    if (a->brick_h < 2 || a->n_bricks < 0 || !a->brick_ij || !a->brick_nbr || !a->flags)
        return set_error(GSW_ERR_INVALID, "flat: bad brick tables (brick_h >= 2)");
    if (!a->q0 || !a->q1 || !a->q2 || !a->bed) return set_error(GSW_ERR_INVALID, "flat: null state/bed");
    FlatMesh<T>& m = k.m;
    m.q0 = (const T*)a->q0; m.q1 = (const T*)a->q1; m.q2 = (const T*)a->q2;
    m.o0 = (T*)a->qn0; m.o1 = (T*)a->qn1; m.o2 = (T*)a->qn2;
    m.b = (const T*)a->bed; m.flags = a->flags; m.ncls = a->n_cls; m.max_h = (T*)a->max_h;
    m.bij = a->brick_ij; m.bnbr = a->brick_nbr; m.nb = a->n_bricks; m.bh = a->brick_h;
    FlatPhys<T>& ph = k.ph;
    ph.inv_dx = (T)a->inv_dx; ph.inv_dy = (T)a->inv_dy;
    ph.half_dx = (T)0.5 * ((T)1 / ph.inv_dx); ph.half_dy = (T)0.5 * ((T)1 / ph.inv_dy);
    if (!(a->h_min > 0.0) || !(a->h_min_cfl > 0.0))  // both are divisor floors of the step
        return set_error(GSW_ERR_INVALID, "flat: h_min (%g) and h_min_cfl (%g) must be > 0", a->h_min, a->h_min_cfl);
    ph.g = (T)a->g; ph.h_min = (T)a->h_min; ph.h_min_cfl = (T)a->h_min_cfl; ph.vcap = (T)a->vcap;
    ph.linf = a->linf; ph.quad = a->quadratic; ph.keep_h = a->keep_h;
    ph.rain_kind = a->rain_kind; ph.rain = (const T*)a->rain; ph.ngh = a->ngh; ph.nx = a->nx; ph.ny = a->ny;
    ph.ntab = (const T*)a->n_tab;
    ph.lookup = a->rain_lookup; ph.ncol = a->rain_ncol;
    ph.g_recip = sizeof(T) == 4 ? (T)div_const_recip((float)a->g) : (T)0;
    ph.ref_pow = a->arith == GSW_ARITH_EXACT ? 1 : 0;
    k.st = a->state; k.lam = (unsigned long long*)a->lam_target;
    k.segs = a->segments > 0 ? a->segments : auto_segments(a->n_bricks, (int64_t)sm_count() * 24, a->brick_h);
    if (k.segs != 1 && k.segs != 2 && k.segs != 4) return set_error(GSW_ERR_INVALID, "flat: segments must be 0, 1, 2 or 4");
    if (a->brick_h % k.segs != 0) return set_error(GSW_ERR_INVALID, "flat: brick_h must be a multiple of segments");
    const bool all = a->brick_lo == 0 && a->brick_hi == 0;
    k.b0 = all ? 0 : a->brick_lo;
    k.b1 = all ? a->n_bricks : a->brick_hi;
    if (k.b0 < 0 || k.b1 < k.b0 || k.b1 > a->n_bricks)
        return set_error(GSW_ERR_INVALID, "flat: brick range [%lld, %lld) outside [0, %lld)", (long long)a->brick_lo,
                         (long long)a->brick_hi, (long long)a->n_bricks);
    if (step) {
        if (!a->state) return set_error(GSW_ERR_INVALID, "flat step: state is required");
        if (!a->n_tab || a->n_tab_len < 1) return set_error(GSW_ERR_INVALID, "flat step: n_tab is required");
        if (a->rain_kind != GSW_RAIN_NONE && !a->rain) return set_error(GSW_ERR_INVALID, "flat step: rain is NULL");
        if (a->rain_kind == GSW_RAIN_GRIDDED && (a->nx <= 0 || a->ny <= 0 || a->ngh < 0))
            return set_error(GSW_ERR_INVALID, "flat step: gridded rain needs ngh, nx, ny");
        if (a->rain_kind == GSW_RAIN_LOOKUP && (!a->rain_lookup || a->rain_ncol < 1))
            return set_error(GSW_ERR_INVALID, "flat step: lookup rain needs rain_lookup and rain_ncol >= 1");
        if (!m.o0 || !m.o1 || !m.o2) return set_error(GSW_ERR_INVALID, "flat step: null output");
    }
    return GSW_OK;
}

template <typename T, bool STEP, bool REFPOW, bool LEAN>
inline void launch_flat_caps(const FlatK<T>& k, int mb, unsigned blocks, int W, cudaStream_t s) {
    constexpr bool capped = STEP && sizeof(T) == 4;   // register caps apply to the binary32 step
    if (capped && mb == 3) flat_march_kernel<T, STEP, capped ? 3 : 1, REFPOW, LEAN><<<blocks, dim3(32, W), 0, s>>>(k);
    else if (capped && mb == 4) flat_march_kernel<T, STEP, capped ? 4 : 1, REFPOW, LEAN><<<blocks, dim3(32, W), 0, s>>>(k);
    else if (capped && mb == 5) flat_march_kernel<T, STEP, capped ? 5 : 1, REFPOW, LEAN><<<blocks, dim3(32, W), 0, s>>>(k);
    else flat_march_kernel<T, STEP, 1, REFPOW, LEAN><<<blocks, dim3(32, W), 0, s>>>(k);
}

// The production configuration (the LEAN kernel: rain none or uniform, quadratic
// friction, keep-h, the L2 norm) or the general kernel.
template <typename T, bool STEP, bool REFPOW>
inline void launch_flat_shape(const FlatK<T>& k, int mb, unsigned blocks, int W, cudaStream_t s) {
    constexpr bool can_lean = STEP && sizeof(T) == 4;
    const bool lean = k.ph.rain_kind != GSW_RAIN_GRIDDED && k.ph.rain_kind != GSW_RAIN_LOOKUP &&
                      k.ph.quad != 0 && k.ph.keep_h != 0 && k.ph.linf == 0;
    if (can_lean && lean) launch_flat_caps<T, STEP, REFPOW, can_lean>(k, mb, blocks, W, s);
    else launch_flat_caps<T, STEP, REFPOW, false>(k, mb, blocks, W, s);
}

template <typename T, bool STEP>
inline int launch_flat(const GswFlatArgs* a, cudaStream_t s) {
    FlatK<T> k;
    int rc = fill_flat<T>(a, k, STEP);
    if (rc) return rc;
    if (k.b1 == k.b0) return GSW_OK;
    const int W = a->warps > 0 ? a->warps : 4;
    if (W < 1 || W > 8) return set_error(GSW_ERR_INVALID, "flat: warps must be in [1, 8]");
    const int64_t blocks = ((k.b1 - k.b0) * k.segs + W - 1) / W;
    if (blocks > 0x7fffffffLL) return set_error(GSW_ERR_INVALID, "flat: too many bricks");
    const int mb = a->min_blocks;
    if (mb != 0 && (mb < 3 || mb > 5)) return set_error(GSW_ERR_INVALID, "flat: min_blocks must be 0, 3, 4 or 5");
    constexpr bool can_refpow = kRefPowBuild && STEP && sizeof(T) == 4;
    if (can_refpow && a->arith == GSW_ARITH_EXACT) launch_flat_shape<T, STEP, can_refpow>(k, mb, (unsigned)blocks, W, s);
    else launch_flat_shape<T, STEP, false>(k, mb, (unsigned)blocks, W, s);
    return check_launch("flat_march");
}

}  // namespace gsw
