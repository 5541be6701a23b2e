// gsw_flat_brick.cuh -- the per-brick march of the compressed mesh (shared by the flat
// solver's kernels and the ensemble's persistent step).
#pragma once
#include "gsw_common.cuh"

namespace gsw {

// Mesh arrays of one brick storage (a compressed mesh, or all members of an ensemble).
struct FlatMesh {
    const float* q0; const float* q1; const float* q2;
    float* o0; float* o1; float* o2;
    const float* b;
    const uint8_t* flags;
    const uint8_t* ncls;
    float* max_h;
    const int32_t* bij; const int32_t* bnbr;
    int64_t nb; int bh;
};

// Physics of one solver (one ensemble member).
struct FlatPhys {
    float inv_dx, inv_dy, half_dx, half_dy, g, h_min, h_min_cfl, vcap;
    int linf, quad, keep_h, rain_kind, ngh, nx, ny;
    const float* rain; const float* ntab;
};

// For the flat kernels' argument struct
struct FlatK { FlatMesh m; FlatPhys ph; const GswLoopState* st; unsigned long long* lam; };

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

__device__ __forceinline__ float grad_y_flat(const FlatMesh& m, const FlatPhys& ph, const BrickView& v, float bc,
                                             int r, int lane) {
    float bl = __shfl_up_sync(0xffffffffu, bc, 1);
    float br = __shfl_down_sync(0xffffffffu, bc, 1);
    if (lane == 0)  bl = __ldg(m.b + v.outer_b(r, 0));
    if (lane == 31) br = __ldg(m.b + v.outer_b(r, 31));
    return 0.5f * (br - bl) * ph.inv_dy;
}

__device__ __forceinline__ Cell<float> shfl_down_cell(const Cell<float>& c) {
    Cell<float> r;
    r.h = __shfl_down_sync(0xffffffffu, c.h, 1);
    r.u = __shfl_down_sync(0xffffffffu, c.u, 1);
    r.v = __shfl_down_sync(0xffffffffu, c.v, 1);
    r.eta = __shfl_down_sync(0xffffffffu, c.eta, 1);
    r.b = __shfl_down_sync(0xffffffffu, c.b, 1);
    r.gy = __shfl_down_sync(0xffffffffu, c.gy, 1);
    r.gx = r.gy; r.hu = r.h; r.hv = r.h;
    return r;
}

__device__ __forceinline__ Face<float> shfl_up_face(const Face<float>& f) {
    Face<float> r;
    r.Fh = __shfl_up_sync(0xffffffffu, f.Fh, 1);
    r.Fn = __shfl_up_sync(0xffffffffu, f.Fn, 1);
    r.Ft = __shfl_up_sync(0xffffffffu, f.Ft, 1);
    r.srcR = __shfl_up_sync(0xffffffffu, f.srcR, 1);
    r.srcL = r.srcR;
    r.wet = __shfl_up_sync(0xffffffffu, (int)f.wet, 1) != 0;
    return r;
}

// One brick, walked by one warp. STEP: the fused step (returns this lane's wave speed
// bits); otherwise the residual. `frame` is the member's gridded rain frame or null.
template <bool STEP>
__device__ __forceinline__ unsigned long long flat_brick(const FlatMesh& m, const FlatPhys& ph, int64_t bidx,
                                                         float dt, float rate, const float* frame) {
    const int lane = threadIdx.x;
    unsigned long long lam_local = 0ull;
    BrickView v;
    v.BS = (int64_t)m.bh * GSW_BRICK_PITCH;
    v.bh = m.bh;
    v.self = bidx;
    v.up = m.bnbr[4 * bidx + 0]; v.down = m.bnbr[4 * bidx + 1];
    v.left = m.bnbr[4 * bidx + 2]; v.right = m.bnbr[4 * bidx + 3];
    v.zero = m.nb;
    const int bi = m.bij[2 * bidx], bj = m.bij[2 * bidx + 1];
    const int bh = m.bh;
    Cell<float> cur, nx;
    const float b_m2 = __ldg(m.b + v.slot(-2, lane));
    { const int64_t s = v.slot(-1, lane); cur.h = __ldg(m.q0 + s); cur.hu = __ldg(m.q1 + s); cur.hv = __ldg(m.q2 + s); cur.b = __ldg(m.b + s); }
    { const int64_t s = v.slot(0, lane); nx.h = __ldg(m.q0 + s); nx.hu = __ldg(m.q1 + s); nx.hv = __ldg(m.q2 + s); nx.b = __ldg(m.b + s); }
    float b_next = __ldg(m.b + v.slot(1, lane));
    // prefetch of the row after next (rows up to bh+1 exist: the brick below or the zero brick)
    int64_t sp = v.slot(1, lane);
    float pf_h = __ldg(m.q0 + sp), pf_hu = __ldg(m.q1 + sp), pf_hv = __ldg(m.q2 + sp);
    float pf_b = __ldg(m.b + v.slot(2, lane));
    make_prims(cur, ph.h_min);
    make_prims(nx, ph.h_min);
    cur.gx = 0.5f * (nx.b - b_m2) * ph.inv_dx;
    cur.gy = 0.0f;
    nx.gx = 0.5f * (b_next - cur.b) * ph.inv_dx;
    nx.gy = grad_y_flat(m, ph, v, nx.b, 0, lane);
    Face<float> Wf;
    srm_face<float, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min, Wf);
    cur = nx;
    for (int r = 0; r < bh; ++r) {
        nx.h = pf_h; nx.hu = pf_hu; nx.hv = pf_hv;
        nx.b = b_next;
        const float b_p2 = pf_b;
        if (r + 1 < bh) {
            sp = v.slot(r + 2, lane);
            pf_h = __ldg(m.q0 + sp); pf_hu = __ldg(m.q1 + sp); pf_hv = __ldg(m.q2 + sp);
            pf_b = __ldg(m.b + v.slot(r + 3, lane));
        }
        make_prims(nx, ph.h_min);
        nx.gx = 0.5f * (b_p2 - cur.b) * ph.inv_dx;
        nx.gy = grad_y_flat(m, ph, v, nx.b, r + 1, lane);
        Face<float> Ef;
        srm_face<float, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min, Ef);
        const Cell<float> rn = shfl_down_cell(cur);
        Face<float> Nf;
        srm_face<float, false>(cur, rn, ph.half_dy, ph.inv_dy, ph.g, ph.h_min, Nf);
        const Face<float> Sf = shfl_up_face(Nf);
        if (lane >= 1 && lane <= 30) {
            const int64_t o = bidx * v.BS + (int64_t)r * GSW_BRICK_PITCH + (lane - 1);
            const uint8_t f = m.flags[o];
            if (f & GSW_SLOT_STORED) {
                const bool active = (f & GSW_SLOT_ACTIVE) != 0;
                if (!STEP) {
                    float rh = 0.0f, rhu = 0.0f, rhv = 0.0f;
                    if (active) accumulate(Ef, Wf, Nf, Sf, rh, rhu, rhv);
                    m.o0[o] = rh; m.o1[o] = rhu; m.o2[o] = rhv;
                } else if (!active) {
                    m.o0[o] = cur.h; m.o1[o] = cur.hu; m.o2[o] = cur.hv;
                    if (m.max_h != nullptr && cur.h > m.max_h[o]) m.max_h[o] = cur.h;
                } else {
                    float rh, rhu, rhv;
                    accumulate(Ef, Wf, Nf, Sf, rh, rhu, rhv);
                    float rr0 = rh;
                    if (ph.rain_kind == GSW_RAIN_UNIFORM) rr0 = rr0 + rate;
                    else if (ph.rain_kind == GSW_RAIN_GRIDDED) {
                        const int i = bi * bh + r, j = bj * GSW_BRICK_W + (lane - 1);
                        rr0 = rr0 + frame[(int64_t)(i - ph.ngh) * ph.ny + (j - ph.ngh)];
                    }
                    float h = cur.h + dt * rr0;
                    float hu = cur.hu + dt * rhu;
                    float hv = cur.hv + dt * rhv;
                    const float n = m.ncls ? ph.ntab[m.ncls[o]] : ph.ntab[0];
                    wetdry_friction<float>(h, hu, hv, true, n, dt, ph.g, ph.h_min, ph.vcap,
                                           ph.quad != 0, ph.keep_h != 0);
                    m.o0[o] = h; m.o1[o] = hu; m.o2[o] = hv;
                    if (m.max_h != nullptr && h > m.max_h[o]) m.max_h[o] = h;
                    const unsigned long long lb = lam_flat_bits(h, hu, hv, ph.g, ph.h_min, ph.h_min_cfl,
                                                                ph.linf != 0);
                    lam_local = lb > lam_local ? lb : lam_local;
                }
            }
        }
        Wf = Ef;
        cur = nx;
        b_next = b_p2;
    }
    return lam_local;
}

}  // namespace gsw
