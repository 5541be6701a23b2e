// gsw_adjoint.cu -- the reverse of one compressed-mesh step, for gradient-based calibration.
//
// The reference has no adjoint. This file differentiates the flat tier's fused step
// (gsw_flat_brick.cuh) by hand, with dt, the rain frame and the wet/dry/branch pattern
// those of the forward step (recomputed from the same state, so every branch is the
// one the forward pass took). One reverse step is two launches over the brick storage:
//   A  recompute the residual (the forward column march), the Euler update and the
//      wet/dry + Manning tail of every active cell, and run the tail backwards: the
//      adjoint of the new state (lam_in) gives the adjoint of the old state through the
//      identity part of Euler (written to lam_out), the adjoint of the cell's residual
//      (rbar = dt * ...), of its Manning n (per class) and of the rain rate (per step);
//   B  walk the bricks again, recompute every face and push the residual adjoints of its
//      two cells back through it (srm_face_bwd), adding the face's contributions to
//      both cells' lam_out. Each face is visited once, as in the forward march.
// Ring cells carry their state unchanged and hold no parameter, so their adjoint is
// only what the faces give them (the discharge inlet's ghost cells read it).
#include "gsw_flat_brick.cuh"
#include "gsw_adjoint.cuh"
#include "gsw_forcing.cuh"

namespace gsw {

template <typename T>
struct AdjK {
    FlatMesh<T> m;            // q* = the state the step read (inlet ghosts written)
    FlatPhys<T> ph;
    const GswLoopState* st;   // dt, rain frame and step index of the step being reversed
    const T* li0; const T* li1; const T* li2;   // adjoint of the new state
    T* lo0; T* lo1; T* lo2;                      // adjoint of the old state (out)
    T* rb0; T* rb1; T* rb2;                      // residual adjoints (scratch, zero off the stored slots)
    double* n_bar; int n_tab_len;
    double* rate_bar;
    int segs;                 // warps per brick: each marches brick_h / segs rows
};

template <typename T>
__device__ __forceinline__ Bar3<T> load_bar(const T* a0, const T* a1, const T* a2, int64_t s) {
    Bar3<T> b; b.h = a0[s]; b.hu = a1[s]; b.hv = a2[s];
    return b;
}
template <typename T>
__device__ __forceinline__ void add_bar(Bar3<T>& a, const Bar3<T>& b) { a.h += b.h; a.hu += b.hu; a.hv += b.hv; }
template <typename T>
__device__ __forceinline__ Bar3<T> shfl_up_bar(const Bar3<T>& b) {
    Bar3<T> r;
    r.h = __shfl_up_sync(0xffffffffu, b.h, 1);
    r.hu = __shfl_up_sync(0xffffffffu, b.hu, 1);
    r.hv = __shfl_up_sync(0xffffffffu, b.hv, 1);
    return r;
}
template <typename T>
__device__ __forceinline__ Bar3<T> shfl_down_bar(const Bar3<T>& b) {
    Bar3<T> r;
    r.h = __shfl_down_sync(0xffffffffu, b.h, 1);
    r.hu = __shfl_down_sync(0xffffffffu, b.hu, 1);
    r.hv = __shfl_down_sync(0xffffffffu, b.hv, 1);
    return r;
}
template <typename T>
__device__ __forceinline__ bool nonzero(const Bar3<T>& b) { return b.h != (T)0 || b.hu != (T)0 || b.hv != (T)0; }

template <typename T>
__device__ __forceinline__ BrickView brick_view(const FlatMesh<T>& m, int64_t bidx) {
    BrickView v;
    v.BS = (int64_t)m.bh * GSW_BRICK_PITCH;
    v.bh = m.bh;
    v.self = bidx;
    v.up = m.bnbr[4 * bidx + 0]; v.down = m.bnbr[4 * bidx + 1];
    v.left = m.bnbr[4 * bidx + 2]; v.right = m.bnbr[4 * bidx + 3];
    v.zero = m.nb;
    return v;
}

template <typename T>
__device__ __forceinline__ void load_state(const FlatMesh<T>& m, int64_t s, Cell<T>& c) {
    c.h = __ldg(m.q0 + s); c.hu = __ldg(m.q1 + s); c.hv = __ldg(m.q2 + s); c.b = __ldg(m.b + s);
}

// ---------------------------------------------------------------------------- A
template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB) adj_tail_kernel(AdjK<T> p) {
    __shared__ double s_nbar[256];
    __shared__ double s_rate[8];
    const int tid = threadIdx.x + 32 * threadIdx.y;
    const int nth = 32 * blockDim.y;
    for (int k = tid; k < p.n_tab_len; k += nth) s_nbar[k] = 0.0;
    __syncthreads();
    const FlatMesh<T>& m = p.m;
    const FlatPhys<T>& ph = p.ph;
    const int lane = threadIdx.x;
    const int64_t item = (int64_t)blockIdx.x * blockDim.y + threadIdx.y;   // (brick, row segment)
    const int64_t bidx = item / p.segs;
    const int seg = (int)(item - bidx * p.segs);
    double rate_acc = 0.0;
    const T dt = sizeof(T) == 4 ? (T)p.st->dt_f32 : (T)p.st->dt;
    T rate = (T)0;
    const T* frame = nullptr;
    if (ph.rain_kind == GSW_RAIN_UNIFORM) rate = ph.rain[p.st->rain_idx];
    if (ph.rain_kind == GSW_RAIN_GRIDDED) frame = ph.rain + (int64_t)p.st->rain_idx * ph.nx * ph.ny;
    if (bidx < m.nb) {
        const BrickView v = brick_view(m, bidx);
        const int bi = m.bij[2 * bidx], bj = m.bij[2 * bidx + 1];
        const int bh = m.bh;
        const int r0 = seg * bh / p.segs, r1 = (seg + 1) * bh / p.segs;
        Cell<T> cur, nx;
        const T b_m2 = __ldg(m.b + v.slot(r0 - 2, lane));
        load_state(m, v.slot(r0 - 1, lane), cur);
        load_state(m, v.slot(r0, lane), nx);
        T b_next = __ldg(m.b + v.slot(r0 + 1, lane));
        make_prims(cur, ph.h_min);
        make_prims(nx, ph.h_min);
        cur.gx = (T)0.5 * (nx.b - b_m2) * ph.inv_dx;
        cur.gy = (T)0;
        nx.gx = (T)0.5 * (b_next - cur.b) * ph.inv_dx;
        nx.gy = grad_y_flat<T>(m, ph, v, nx.b, r0, lane);
        Face<T> Wf;
        srm_face<T, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min, Wf);
        cur = nx;
        for (int r = r0; r < r1; ++r) {
            {
                const int64_t s = v.slot(r + 1, lane);
                nx.h = __ldg(m.q0 + s); nx.hu = __ldg(m.q1 + s); nx.hv = __ldg(m.q2 + s);
            }
            nx.b = b_next;
            const T b_p2 = __ldg(m.b + v.slot(r + 2, lane));
            make_prims(nx, ph.h_min);
            nx.gx = (T)0.5 * (b_p2 - cur.b) * ph.inv_dx;
            nx.gy = grad_y_flat<T>(m, ph, v, nx.b, r + 1, lane);
            Face<T> Ef;
            srm_face<T, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min, Ef);
            const Cell<T> rn = shfl_down_cell<T>(cur);
            Face<T> Nf;
            srm_face<T, false>(cur, rn, ph.half_dy, ph.inv_dy, ph.g, ph.h_min, Nf);
            const Face<T> Sf = shfl_up_face<T>(Nf);
            if (lane >= 1 && lane <= 30) {
                const int64_t o = bidx * v.BS + (int64_t)r * GSW_BRICK_PITCH + (lane - 1);
                const uint8_t f = m.flags[o];
                if (f & GSW_SLOT_ACTIVE) {
                    T rh, rhu, rhv;
                    accumulate(Ef, Wf, Nf, Sf, rh, rhu, rhv);
                    T rr0 = rh;
                    if (ph.rain_kind == GSW_RAIN_UNIFORM) rr0 = rr0 + rate;
                    else if (ph.rain_kind == GSW_RAIN_GRIDDED) {
                        const int i = bi * bh + r, j = bj * GSW_BRICK_W + (lane - 1);
                        rr0 = rr0 + frame[(int64_t)(i - ph.ngh) * ph.ny + (j - ph.ngh)];
                    }
                    const T h1 = cur.h + dt * rr0;
                    const T hu1 = cur.hu + dt * rhu;
                    const T hv1 = cur.hv + dt * rhv;
                    const int cls = m.ncls ? (int)m.ncls[o] : 0;
                    const T n = ph.ntab[cls];
                    const Bar3<T> out_b = load_bar(p.li0, p.li1, p.li2, o);
                    Bar3<T> in_b;
                    T n_b;
                    wetdry_friction_bwd<T>(h1, hu1, hv1, n, dt, ph.g, ph.h_min, ph.vcap, ph.quad != 0,
                                           ph.keep_h != 0, ph.ref_pow != 0, out_b, in_b, n_b);
                    p.lo0[o] = in_b.h; p.lo1[o] = in_b.hu; p.lo2[o] = in_b.hv;
                    p.rb0[o] = dt * in_b.h; p.rb1[o] = dt * in_b.hu; p.rb2[o] = dt * in_b.hv;
                    if (ph.rain_kind == GSW_RAIN_UNIFORM) rate_acc += (double)(dt * in_b.h);
                    if (n_b != (T)0 && cls < p.n_tab_len) atomicAdd(&s_nbar[cls], (double)n_b);
                } else if (f & GSW_SLOT_STORED) {
                    p.lo0[o] = (T)0; p.lo1[o] = (T)0; p.lo2[o] = (T)0;
                    p.rb0[o] = (T)0; p.rb1[o] = (T)0; p.rb2[o] = (T)0;
                }
            }
            Wf = Ef;
            cur = nx;
            b_next = b_p2;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rate_acc += __shfl_xor_sync(0xffffffffu, rate_acc, o);
    if (lane == 0) s_rate[threadIdx.y] = rate_acc;
    __syncthreads();
    if (tid == 0 && p.rate_bar != nullptr) {
        double t = 0.0;
        for (int w = 0; w < (int)blockDim.y; ++w) t += s_rate[w];
        if (t != 0.0) atomicAdd(p.rate_bar + p.st->steps, t);
    }
    for (int k = tid; k < p.n_tab_len; k += nth)
        if (s_nbar[k] != 0.0) atomicAdd(p.n_bar + k, s_nbar[k]);
}

// ---------------------------------------------------------------------------- B
template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB) adj_face_kernel(AdjK<T> p) {
    const FlatMesh<T>& m = p.m;
    const FlatPhys<T>& ph = p.ph;
    const int lane = threadIdx.x;
    const int64_t item = (int64_t)blockIdx.x * blockDim.y + threadIdx.y;   // (brick, row segment)
    const int64_t bidx = item / p.segs;
    const int seg = (int)(item - bidx * p.segs);
    if (bidx >= m.nb) return;                                  // warp-uniform
    const BrickView v = brick_view(m, bidx);
    const int bh = m.bh;
    const int r0 = seg * bh / p.segs, r1 = (seg + 1) * bh / p.segs;
    Cell<T> cur, nx;
    const T b_m2 = __ldg(m.b + v.slot(r0 - 2, lane));
    int64_t s = v.slot(r0 - 1, lane);
    load_state(m, s, cur);
    Bar3<T> rb_cur = load_bar<T>(p.rb0, p.rb1, p.rb2, s);
    s = v.slot(r0, lane);
    load_state(m, s, nx);
    Bar3<T> rb_nx = load_bar<T>(p.rb0, p.rb1, p.rb2, s);
    T b_next = __ldg(m.b + v.slot(r0 + 1, lane));
    make_prims(cur, ph.h_min);
    make_prims(nx, ph.h_min);
    cur.gx = (T)0.5 * (nx.b - b_m2) * ph.inv_dx;
    cur.gy = (T)0;
    nx.gx = (T)0.5 * (b_next - cur.b) * ph.inv_dx;
    nx.gy = grad_y_flat<T>(m, ph, v, nx.b, r0, lane);
    const Bar3<T> zero3 = {(T)0, (T)0, (T)0};
    Bar3<T> carry = zero3;                   // the x-face above the current row, cell below
    if (nonzero(rb_cur) || nonzero(rb_nx)) {
        Bar3<T> Lb = zero3;
        srm_face_bwd<T, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min,
                              face_bar<T, true>(rb_cur, rb_nx), Lb, carry);
    }
    cur = nx;
    rb_cur = rb_nx;
    for (int r = r0; r < r1; ++r) {
        s = v.slot(r + 1, lane);
        nx.h = __ldg(m.q0 + s); nx.hu = __ldg(m.q1 + s); nx.hv = __ldg(m.q2 + s);
        rb_nx = load_bar<T>(p.rb0, p.rb1, p.rb2, s);
        nx.b = b_next;
        const T b_p2 = __ldg(m.b + v.slot(r + 2, lane));
        make_prims(nx, ph.h_min);
        nx.gx = (T)0.5 * (b_p2 - cur.b) * ph.inv_dx;
        nx.gy = grad_y_flat<T>(m, ph, v, nx.b, r + 1, lane);
        Bar3<T> acc = carry;
        Bar3<T> below = zero3;
        if (nonzero(rb_cur) || nonzero(rb_nx))
            srm_face_bwd<T, true>(cur, nx, ph.half_dx, ph.inv_dx, ph.g, ph.h_min,
                                  face_bar<T, true>(rb_cur, rb_nx), acc, below);
        const Cell<T> rn = shfl_down_cell<T>(cur);
        const Bar3<T> rb_rn = shfl_down_bar<T>(rb_cur);
        Bar3<T> right = zero3;
        if (lane < 31 && (nonzero(rb_cur) || nonzero(rb_rn)))
            srm_face_bwd<T, false>(cur, rn, ph.half_dy, ph.inv_dy, ph.g, ph.h_min,
                                   face_bar<T, false>(rb_cur, rb_rn), acc, right);
        add_bar(acc, shfl_up_bar<T>(right));
        if (lane >= 1 && lane <= 30) {
            const int64_t o = bidx * v.BS + (int64_t)r * GSW_BRICK_PITCH + (lane - 1);
            if (m.flags[o] & GSW_SLOT_STORED) {
                p.lo0[o] += acc.h; p.lo1[o] += acc.hu; p.lo2[o] += acc.hv;
            }
        }
        carry = below;
        cur = nx;
        rb_cur = rb_nx;
        b_next = b_p2;
    }
}

// ----------------------------------------------------------------- discharge inlet
// Reverse of flat_inflow_kernel (gsw_forcing.cu): the adjoint the faces gave the ghost
// slots flows to the inlet's active cells (the copied depth and the depth weights)
// and to Q(t) of this step (q_bar[steps]); the ghost adjoints are then cleared.
template <typename T>
__global__ void adj_inflow_kernel(GswFlatInflowArgs a, T* l0, T* l1, T* l2, double* q_bar) {
    if (threadIdx.x != 0) return;
    const T* q0 = (const T*)a.q0;
    const T* bed = (const T*)a.bed;
    const double Q = np_interp(a.state->t, a.t_knots, a.q_knots, a.n_knots);
    const T sum = pairwise_sum<T>(q0, a.nbr_slot, 0, a.n);
    const T qds = (T)__ddiv_rn(Q, a.ds);
    double Q_b = 0.0;
    if ((double)sum > 0.0) {
        T ssum_b = (T)0;
        for (int k = 0; k < a.n; ++k) {
            const int64_t g = a.ghost_slot[k], src = a.nbr_slot[k];
            const T h = q0[src];
            const T w = h / sum;
            const T qn_b = l1[g] * (T)a.nx_n + l2[g] * (T)a.ny_n;
            Q_b += (double)(qn_b * w) / a.ds;
            const T w_b = qn_b * qds;
            ssum_b -= w_b * w / sum;
            l0[src] += l0[g] + w_b / sum;
        }
        for (int k = 0; k < a.n; ++k) l0[a.nbr_slot[k]] += ssum_b;
    } else {
        T zmin = bed[a.nbr_slot[0]], zmax = zmin;
        for (int k = 1; k < a.n; ++k) {
            const T z = bed[a.nbr_slot[k]];
            zmin = z < zmin ? z : zmin;
            zmax = z > zmax ? z : zmax;
        }
        const double zlo = (double)zmin, zhi = (double)zmax;
        const T seed = (T)__dadd_rn(zlo, __dmul_rn(0.10, __dsub_rn(zhi, zlo)));
        int nlow = 0;
        T hmax = (T)0;
        for (int k = 0; k < a.n; ++k) {
            const T z = bed[a.nbr_slot[k]];
            nlow += (z <= zmin);
            T hf = seed - z;
            hf = hf > (T)0 ? hf : (T)0;
            hmax = (k == 0 || hf > hmax) ? hf : hmax;
        }
        const double nl = nlow > 0 ? (double)nlow : 1.0;
        const bool flat = !((double)hmax > 0.0);
        double dhc_dQ = 0.0;
        if (flat && Q != 0.0) {
            const double qc = fabs(Q) / (nl * a.ds);
            const double hc = pow(qc * qc / 9.80665, 1.0 / 3.0);
            dhc_dQ = (2.0 / 3.0) * hc / Q;
        }
        for (int k = 0; k < a.n; ++k) {
            const int64_t g = a.ghost_slot[k];
            const T z = bed[a.nbr_slot[k]];
            const double w = ((double)z <= zlo) ? 1.0 / nl : 0.0;
            const T qn_b = l1[g] * (T)a.nx_n + l2[g] * (T)a.ny_n;
            Q_b += (double)qn_b * w / a.ds + (double)l0[g] * dhc_dQ;
        }
    }
    for (int k = 0; k < a.n; ++k) {
        const int64_t g = a.ghost_slot[k];
        l0[g] = (T)0; l1[g] = (T)0; l2[g] = (T)0;
    }
    if (q_bar != nullptr) q_bar[a.state->steps] += Q_b;
}

// ------------------------------------------------------------------------ gauges
template <typename T>
__global__ void gauge_record_kernel(GswGaugeArgs a) {
    if (a.state != nullptr && a.state->done) return;
    const int64_t idx = (a.state ? a.state->steps : 0) + a.offset - a.first;
    if (idx < 0 || idx >= a.count) return;
    const T* q0 = (const T*)a.q0;
    double* out = a.series + idx * a.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n; k += gridDim.x * blockDim.x)
        out[k] = (double)q0[a.slots[k]];
}

template <typename T>
__global__ void gauge_adjoint_kernel(GswGaugeArgs a) {
    const int64_t idx = (a.state ? a.state->steps : 0) + a.offset - a.first;
    if (idx < 0 || idx >= a.count) return;
    const T* q0 = (const T*)a.q0;
    T* lam = (T*)a.lam0;
    const double* tgt = a.target + idx * a.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n; k += gridDim.x * blockDim.x) {
        const double d = (double)q0[a.slots[k]] - tgt[k];
        atomicAdd(lam + a.slots[k], (T)(a.weight * 2.0 * d));
    }
}

}  // namespace gsw

using namespace gsw;

template <typename T>
static int fill_adj(const GswFlatAdjArgs* a, AdjK<T>& k) {
    const GswFlatArgs& f = a->f;
    if (f.brick_h < 2 || f.n_bricks < 0 || !f.brick_ij || !f.brick_nbr || !f.flags || !f.q0 || !f.q1 || !f.q2 ||
        !f.bed || !f.state || !f.n_tab || f.n_tab_len < 1)
        return set_error(GSW_ERR_INVALID, "adjoint: bad flat arguments");
    if (f.n_tab_len > 256) return set_error(GSW_ERR_RANGE, "adjoint: at most 256 Manning classes");
    if (f.rain_kind != GSW_RAIN_NONE && !f.rain) return set_error(GSW_ERR_INVALID, "adjoint: rain is NULL");
    if (f.rain_kind == GSW_RAIN_LOOKUP) return set_error(GSW_ERR_INVALID, "adjoint: lookup rain is not differentiated");
    if (f.arith != GSW_ARITH_EXACT && f.arith != GSW_ARITH_PORTABLE)
        return set_error(GSW_ERR_INVALID, "adjoint: the exact or portable step is differentiated (arith)");
    if (!a->lam_in0 || !a->lam_in1 || !a->lam_in2 || !a->lam_out0 || !a->lam_out1 || !a->lam_out2 ||
        !a->rbar0 || !a->rbar1 || !a->rbar2 || !a->n_bar)
        return set_error(GSW_ERR_INVALID, "adjoint: null adjoint buffer");
    FlatMesh<T>& m = k.m;
    m.q0 = (const T*)f.q0; m.q1 = (const T*)f.q1; m.q2 = (const T*)f.q2;
    m.o0 = nullptr; m.o1 = nullptr; m.o2 = nullptr;
    m.b = (const T*)f.bed; m.flags = f.flags; m.ncls = f.n_cls; m.max_h = nullptr;
    m.bij = f.brick_ij; m.bnbr = f.brick_nbr; m.nb = f.n_bricks; m.bh = f.brick_h;
    FlatPhys<T>& ph = k.ph;
    ph.inv_dx = (T)f.inv_dx; ph.inv_dy = (T)f.inv_dy;
    ph.half_dx = (T)0.5 * ((T)1 / ph.inv_dx); ph.half_dy = (T)0.5 * ((T)1 / ph.inv_dy);
    ph.g = (T)f.g; ph.h_min = (T)f.h_min; ph.h_min_cfl = (T)f.h_min_cfl; ph.vcap = (T)f.vcap;
    ph.linf = f.linf; ph.quad = f.quadratic; ph.keep_h = f.keep_h;
    ph.rain_kind = f.rain_kind; ph.rain = (const T*)f.rain; ph.ngh = f.ngh; ph.nx = f.nx; ph.ny = f.ny;
    ph.ntab = (const T*)f.n_tab;
    ph.lookup = f.rain_lookup; ph.ncol = f.rain_ncol;
    ph.g_recip = (T)0;          // the recomputed faces divide (the same bits as the forward's)
    ph.ref_pow = f.arith == GSW_ARITH_EXACT ? 1 : 0;
    k.st = f.state;
    k.li0 = (const T*)a->lam_in0; k.li1 = (const T*)a->lam_in1; k.li2 = (const T*)a->lam_in2;
    k.lo0 = (T*)a->lam_out0; k.lo1 = (T*)a->lam_out1; k.lo2 = (T*)a->lam_out2;
    k.rb0 = (T*)a->rbar0; k.rb1 = (T*)a->rbar1; k.rb2 = (T*)a->rbar2;
    k.n_bar = a->n_bar; k.n_tab_len = f.n_tab_len; k.rate_bar = a->rate_bar;
    return GSW_OK;
}

template <typename T>
static int launch_adj(const GswFlatAdjArgs* a, cudaStream_t s) {
    AdjK<T> k;
    if (int rc = fill_adj<T>(a, k)) return rc;
    if (k.m.nb == 0) return GSW_OK;
    const int W = 4;
    k.segs = auto_segments(k.m.nb, (int64_t)sm_count() * 32, k.m.bh);
    const int64_t blocks = (k.m.nb * k.segs + W - 1) / W;
    if (blocks > 0x7fffffffLL) return set_error(GSW_ERR_INVALID, "adjoint: too many bricks");
    // register cap of the binary32 reverse kernels: 0 (compiler's choice), 6 (80) or 8 (64 registers)
    const int mb = sizeof(T) == 4 ? a->min_blocks : 0;
    if (mb != 0 && mb != 6 && mb != 8) return set_error(GSW_ERR_INVALID, "adjoint: min_blocks must be 0, 6 or 8");
    const dim3 grid((unsigned)blocks), block(32, W);
    if (mb == 6) adj_tail_kernel<T, sizeof(T) == 4 ? 6 : 1><<<grid, block, 0, s>>>(k);
    else if (mb == 8) adj_tail_kernel<T, sizeof(T) == 4 ? 8 : 1><<<grid, block, 0, s>>>(k);
    else adj_tail_kernel<T, 1><<<grid, block, 0, s>>>(k);
    if (int rc = check_launch("adj_tail")) return rc;
    if (mb == 6) adj_face_kernel<T, sizeof(T) == 4 ? 6 : 1><<<grid, block, 0, s>>>(k);
    else if (mb == 8) adj_face_kernel<T, sizeof(T) == 4 ? 8 : 1><<<grid, block, 0, s>>>(k);
    else adj_face_kernel<T, 1><<<grid, block, 0, s>>>(k);
    return check_launch("adj_face");
}

extern "C" int gsw_adj_flat_step(const GswFlatAdjArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    GSW_CHECK_ABI(&a->f);
    if (a->f.dtype == GSW_F32) return launch_adj<float>(a, (cudaStream_t)stream);
    if (a->f.dtype == GSW_F64) return launch_adj<double>(a, (cudaStream_t)stream);
    return set_error(GSW_ERR_INVALID, "adjoint: bad dtype");
}

extern "C" int gsw_adj_flat_inflow(const GswFlatInflowArgs* a, void* lam0, void* lam1, void* lam2,
                                   double* q_bar, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->n <= 0) return GSW_OK;
    if (!a->ghost_slot || !a->nbr_slot || !a->q0 || !a->bed || !a->t_knots || !a->q_knots || a->n_knots < 1 ||
        !a->state || !(a->ds > 0.0) || !lam0 || !lam1 || !lam2)
        return set_error(GSW_ERR_INVALID, "adjoint inflow: null pointer, empty hydrograph or ds <= 0");
    cudaStream_t s = (cudaStream_t)stream;
    if (a->dtype == GSW_F32)
        adj_inflow_kernel<float><<<1, 32, 0, s>>>(*a, (float*)lam0, (float*)lam1, (float*)lam2, q_bar);
    else if (a->dtype == GSW_F64)
        adj_inflow_kernel<double><<<1, 32, 0, s>>>(*a, (double*)lam0, (double*)lam1, (double*)lam2, q_bar);
    else return set_error(GSW_ERR_INVALID, "adjoint inflow: bad dtype");
    return check_launch("adj_inflow");
}

static int check_gauge(const GswGaugeArgs* a) {
    if (a->n < 0 || !a->q0 || (a->n > 0 && !a->slots)) return set_error(GSW_ERR_INVALID, "gauges: bad arguments");
    if (a->dtype != GSW_F32 && a->dtype != GSW_F64) return set_error(GSW_ERR_INVALID, "gauges: bad dtype");
    return GSW_OK;
}

extern "C" int gsw_gauge_record(const GswGaugeArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_gauge(a)) return rc;
    if (!a->series) return set_error(GSW_ERR_INVALID, "gauge record: series is NULL");
    if (a->n == 0) return GSW_OK;
    const int grid = (a->n + 255) / 256;
    if (a->dtype == GSW_F32) gauge_record_kernel<float><<<grid, 256, 0, (cudaStream_t)stream>>>(*a);
    else gauge_record_kernel<double><<<grid, 256, 0, (cudaStream_t)stream>>>(*a);
    return check_launch("gauge_record");
}

extern "C" int gsw_gauge_adjoint(const GswGaugeArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_gauge(a)) return rc;
    if (!a->target || !a->lam0) return set_error(GSW_ERR_INVALID, "gauge adjoint: target/lam0 is NULL");
    if (a->n == 0) return GSW_OK;
    const int grid = (a->n + 255) / 256;
    if (a->dtype == GSW_F32) gauge_adjoint_kernel<float><<<grid, 256, 0, (cudaStream_t)stream>>>(*a);
    else gauge_adjoint_kernel<double><<<grid, 256, 0, (cudaStream_t)stream>>>(*a);
    return check_launch("gauge_adjoint");
}
