// gsw_flat_brick.cuh -- the per-brick march of the compressed mesh (shared by the flat
// solver's kernels and the ensemble's persistent step).
#pragma once
#include "gsw_common.cuh"

namespace gsw {

// Mesh arrays of one brick storage (a compressed mesh, or all members of an ensemble).
template <typename T>
struct FlatMesh {
    const T* q0; const T* q1; const T* q2;
    T* o0; T* o1; T* o2;
    const T* b;
    const uint8_t* flags;
    const uint8_t* ncls;
    T* max_h;
    const int32_t* bij; const int32_t* bnbr;
    int64_t nb; int bh;
};

// Physics of one solver (one ensemble member).
template <typename T>
struct FlatPhys {
    T inv_dx, inv_dy, half_dx, half_dy, g, h_min, h_min_cfl, vcap;
    int linf, quad, keep_h, rain_kind, ngh, nx, ny;
    const T* rain; const T* ntab;
    const int32_t* lookup;   // GSW_RAIN_LOOKUP: per-slot column of the rain row
    int ncol;
    T g_recip;               // RN(1/g) for the star depth's h / g, or 0 (gsw_core.cuh div_g)
    int ref_pow;             // 1: Manning's h^(-4/3) by powf (GSW_ARITH_EXACT), 0: by pow_m43 (read by
                             // the adjoint; the step kernels take it as their REFPOW parameter)
};

// Row segments per brick when the caller leaves the choice to the library: one warp
// per brick once the bricks fill the `warps` that can run at once twice over
// (throughput), else 2 or 4 warps per brick so that fewer bricks still keep enough
// warps busy and each warp's march is shorter (latency). A segment recomputes the
// x-face above its first row and reads two rows past each end.
__host__ __device__ __forceinline__ int auto_segments(int64_t bricks, int64_t warps, int bh) {
    int s = bricks >= 2 * warps ? 1 : (2 * bricks >= warps ? 2 : 4);
    while (s > 1 && bh % s != 0) s >>= 1;
    return s;
}

// For the flat kernels' argument struct
template <typename T>
struct FlatK {
    FlatMesh<T> m; FlatPhys<T> ph; const GswLoopState* st; unsigned long long* lam; int segs;
    int64_t b0, b1;    // bricks [b0, b1) are stepped
};

// Slot of brick-relative (row, lane). Lanes 0/31 of the rows above/below the brick are
// never used by an output cell; they read the zero brick.
struct BrickView {
    int64_t self, up, down, left, right, zero, BS;
    int bh;
    __device__ __forceinline__ int64_t slot(int r, int lane) const {
        if (r >= 0 && r < bh) {
            if (lane == 0) return left * BS + (int64_t)r * GSW_BRICK_PITCH + (GSW_BRICK_W - 1);
            if (lane == 31) return right * BS + (int64_t)r * GSW_BRICK_PITCH;
            return self * BS + (int64_t)r * GSW_BRICK_PITCH + (lane - 1);
        }
        if (lane == 0 || lane == 31) return zero * BS;
        if (r < 0) return up * BS + (int64_t)(bh + r) * GSW_BRICK_PITCH + (lane - 1);
        return down * BS + (int64_t)(r - bh) * GSW_BRICK_PITCH + (lane - 1);
    }
    // outer bed neighbour of the edge lanes, for the y-gradient
    __device__ __forceinline__ int64_t outer_b(int r, int lane) const {
        if (r < 0 || r >= bh) return zero * BS;
        if (lane == 0) return left * BS + (int64_t)r * GSW_BRICK_PITCH + (GSW_BRICK_W - 2);
        return right * BS + (int64_t)r * GSW_BRICK_PITCH + 1;
    }
};

template <typename T>
__device__ __forceinline__ T grad_y_flat(const FlatMesh<T>& m, const FlatPhys<T>& ph, const BrickView& v, T bc,
                                         int r, int lane) {
    T bl = __shfl_up_sync(0xffffffffu, bc, 1);
    T br = __shfl_down_sync(0xffffffffu, bc, 1);
    if (lane == 0)  bl = __ldg(m.b + v.outer_b(r, 0));
    if (lane == 31) br = __ldg(m.b + v.outer_b(r, 31));
    return (T)0.5 * (br - bl) * ph.inv_dy;
}

template <typename T>
__device__ __forceinline__ Cell<T> shfl_down_cell(const Cell<T>& c) {
    Cell<T> r;
    r.h = __shfl_down_sync(0xffffffffu, c.h, 1);
    r.u = __shfl_down_sync(0xffffffffu, c.u, 1);
    r.v = __shfl_down_sync(0xffffffffu, c.v, 1);
    r.eta = __shfl_down_sync(0xffffffffu, c.eta, 1);
    r.b = __shfl_down_sync(0xffffffffu, c.b, 1);
    r.gy = __shfl_down_sync(0xffffffffu, c.gy, 1);
    r.gx = r.gy; r.hu = r.h; r.hv = r.h;
    return r;
}

template <typename T>
__device__ __forceinline__ Face<T> shfl_up_face(const Face<T>& f) {
    Face<T> r;
    r.Fh = __shfl_up_sync(0xffffffffu, f.Fh, 1);
    r.Fn = __shfl_up_sync(0xffffffffu, f.Fn, 1);
    r.Ft = __shfl_up_sync(0xffffffffu, f.Ft, 1);
    r.srcR = __shfl_up_sync(0xffffffffu, f.srcR, 1);
    r.srcL = r.srcR;
    r.wet = true;   // unused: the residual adds a dry face's zeros
    return r;
}

// Rows [r0, r1) of one brick, walked by one warp (T = float; double serves the adjoint's
// fp64 checks). A segment reads rows r0-2 .. r1+1 through the brick view (the bricks
// above and below past the brick's edge) and recomputes the x-face above row r0 from
// the same inputs as the face below row r0-1, so splitting a brick's rows among warps
// changes no value. STEP: the fused step (returns this lane's wave speed bits);
// otherwise the residual. `frame` is the gridded rain frame, or null. REFPOW: Manning's
// h^(-4/3) by powf (GSW_ARITH_EXACT) instead of pow_m43. LEAN: the production
// configuration compiled in (rain none or uniform, quadratic friction, keep-h, the L2
// wave-speed norm); the same bits as the general path.
template <typename T, bool STEP, bool REFPOW, bool LEAN = false>
__device__ __forceinline__ unsigned long long flat_brick(const FlatMesh<T>& m, const FlatPhys<T>& ph, int64_t bidx,
                                                         int r0, int r1, T dt, T rate, const T* frame) {
    const int lane = threadIdx.x;
    unsigned long long lam_local = 0ull;
    uint32_t lam32 = 0u;        // the production kernel's binary32 key (lam_flat_bits32)
    BrickView v;
    v.BS = (int64_t)m.bh * GSW_BRICK_PITCH;
    v.bh = m.bh;
    v.self = bidx;
    v.up = m.bnbr[4 * bidx + 0]; v.down = m.bnbr[4 * bidx + 1];
    v.left = m.bnbr[4 * bidx + 2]; v.right = m.bnbr[4 * bidx + 3];
    v.zero = m.nb;
    const int bi = m.bij[2 * bidx], bj = m.bij[2 * bidx + 1];
    const int bh = m.bh;
    Cell<T> cur, nx;
    const T b_m2 = __ldg(m.b + v.slot(r0 - 2, lane));
    { const int64_t s = v.slot(r0 - 1, lane); cur.h = __ldg(m.q0 + s); cur.hu = __ldg(m.q1 + s); cur.hv = __ldg(m.q2 + s); cur.b = __ldg(m.b + s); }
    { const int64_t s = v.slot(r0, lane); nx.h = __ldg(m.q0 + s); nx.hu = __ldg(m.q1 + s); nx.hv = __ldg(m.q2 + s); nx.b = __ldg(m.b + s); }
    T b_next = __ldg(m.b + v.slot(r0 + 1, lane));
    // prefetch of the row after next (rows up to bh+1 exist: the brick below or the zero brick)
    int64_t sp = v.slot(r0 + 1, lane);
    T pf_h = __ldg(m.q0 + sp), pf_hu = __ldg(m.q1 + sp), pf_hv = __ldg(m.q2 + sp);
    T pf_b = __ldg(m.b + v.slot(r0 + 2, lane));
    make_prims(cur, ph.h_min);
    make_prims(nx, ph.h_min);
    cur.gx = (T)0.5 * (nx.b - b_m2) * ph.inv_dx;
    cur.gy = (T)0;
    nx.gx = (T)0.5 * (b_next - cur.b) * ph.inv_dx;
    nx.gy = grad_y_flat<T>(m, ph, v, nx.b, r0, lane);
    Face<T> Wf;
    srm_face<T, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min, Wf, ph.g_recip);
    cur = nx;
    for (int r = r0; r < r1; ++r) {
        // the update's slot flag, class id and running maximum, loaded before the faces so
        // that their latency is hidden (the production kernel; the general one loads late)
        uint8_t f_r = 0, cls_r = 0;
        T mh_r = (T)0;
        if (LEAN && STEP && lane >= 1 && lane <= 30) {
            const int64_t o = bidx * v.BS + (int64_t)r * GSW_BRICK_PITCH + (lane - 1);
            f_r = m.flags[o];
            if (m.ncls) cls_r = m.ncls[o];
            if (m.max_h != nullptr) mh_r = m.max_h[o];
        }
        nx.h = pf_h; nx.hu = pf_hu; nx.hv = pf_hv;
        nx.b = b_next;
        const T b_p2 = pf_b;
        if (r + 1 < r1) {
            sp = v.slot(r + 2, lane);
            pf_h = __ldg(m.q0 + sp); pf_hu = __ldg(m.q1 + sp); pf_hv = __ldg(m.q2 + sp);
            pf_b = __ldg(m.b + v.slot(r + 3, lane));
        }
        make_prims(nx, ph.h_min);
        nx.gx = (T)0.5 * (b_p2 - cur.b) * ph.inv_dx;
        nx.gy = grad_y_flat<T>(m, ph, v, nx.b, r + 1, lane);
        Face<T> Ef;
        srm_face<T, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min, Ef, ph.g_recip);
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
        const Cell<T> rn = shfl_down_cell<T>(cur);
        {
            Face<T> Nf;
            srm_face<T, false>(cur, rn, ph.half_dy, ph.inv_dy, ph.g, ph.h_min, Nf, ph.g_recip);
            const Face<T> Sf = shfl_up_face<T>(Nf);
            rh = rh - Nf.Fh; rhu = rhu - Nf.Ft; rhv = rhv - Nf.Fn; rhv = rhv - Nf.srcL;
            rh = rh + Sf.Fh; rhu = rhu + Sf.Ft; rhv = rhv + Sf.Fn; rhv = rhv + Sf.srcR;
        }
        if (lane >= 1 && lane <= 30) {
            const int64_t o = bidx * v.BS + (int64_t)r * GSW_BRICK_PITCH + (lane - 1);
            const uint8_t f = (LEAN && STEP) ? f_r : m.flags[o];
            if (f & GSW_SLOT_STORED) {
                const bool active = (f & GSW_SLOT_ACTIVE) != 0;
                if (!STEP) {
                    if (!active) { rh = (T)0; rhu = (T)0; rhv = (T)0; }
                    m.o0[o] = rh; m.o1[o] = rhu; m.o2[o] = rhv;
                } else if (!active) {
                    m.o0[o] = cur.h; m.o1[o] = __ldg(m.q1 + o); m.o2[o] = __ldg(m.q2 + o);
                    if (m.max_h != nullptr && cur.h > (LEAN ? mh_r : m.max_h[o])) m.max_h[o] = cur.h;
                } else {
                    T rr0 = rh;
                    if (ph.rain_kind == GSW_RAIN_UNIFORM) rr0 = rr0 + rate;
                    else if (!LEAN && ph.rain_kind == GSW_RAIN_GRIDDED) {
                        const int i = bi * bh + r, j = bj * GSW_BRICK_W + (lane - 1);
                        rr0 = rr0 + frame[(int64_t)(i - ph.ngh) * ph.ny + (j - ph.ngh)];
                    } else if (!LEAN && ph.rain_kind == GSW_RAIN_LOOKUP) {
                        rr0 = rr0 + frame[ph.lookup[o]];
                    }
                    T h = cur.h + dt * rr0;
                    T hu = __ldg(m.q1 + o) + dt * rhu;       // reloaded: not carried down the march
                    T hv = __ldg(m.q2 + o) + dt * rhv;
                    const T n = m.ncls ? ph.ntab[LEAN ? cls_r : m.ncls[o]] : ph.ntab[0];
                    wetdry_friction<T>(h, hu, hv, true, n, dt, ph.g, ph.h_min, ph.vcap,
                                       LEAN || ph.quad != 0, LEAN || ph.keep_h != 0, REFPOW);
                    m.o0[o] = h; m.o1[o] = hu; m.o2[o] = hv;
                    if (m.max_h != nullptr && h > (LEAN ? mh_r : m.max_h[o])) m.max_h[o] = h;
                    if constexpr (LEAN && sizeof(T) == 4) {
                        lam32 = max(lam32, lam_flat_bits32(h, hu, hv, ph.g, ph.h_min, ph.h_min_cfl));
                    } else {
                        const unsigned long long lb = lam_flat_bits(h, hu, hv, ph.g, ph.h_min, ph.h_min_cfl,
                                                                    !LEAN && ph.linf != 0);
                        lam_local = lb > lam_local ? lb : lam_local;
                    }
                }
            }
        }
        cur = nx;
        b_next = b_p2;
    }
    if constexpr (LEAN && sizeof(T) == 4) lam_local = lam_bits_of32(lam32);
    return lam_local;
}

}  // namespace gsw
