// gsw_flat.cu -- the fused step on the compressed (flat) mesh, brick storage.
//
// One warp per brick of 30 x brick_h cells, the same column march as the dense kernel
// (gsw_dense.cu): lanes 1..30 are the brick's columns, lane 0 / lane 31 read the edge
// columns of the left / right brick, and the two rows above and below come from the
// bricks above and below. Every face is computed once from the shared core
// (gsw_core.cuh), so active-cell residuals are bit-identical to the dense kernel's.
//
// Semantics of the reference's flat step (geoswe/compressed_rhs.py:673-865, 990-1118):
// stored cells that are not active (the two-cell ring) keep their state; active cells
// take rain, Euler, the wet/dry floor and Manning from the class table (always, as
// compressed_solver.py:2862-2879 gives a frictionless run the table [0]); the new
// state's wave speed uses the flat norm and floors.
#include "gsw_common.cuh"

namespace gsw {

struct FlatK {
    const float* q0; const float* q1; const float* q2;
    float* o0; float* o1; float* o2;
    const float* b;
    const uint8_t* flags;
    const int32_t* bij; const int32_t* bnbr;
    int64_t nb; int bh;
    float inv_dx, inv_dy, half_dx, half_dy, g, h_min, h_min_cfl;
    int linf;
    const GswLoopState* st; unsigned long long* lam;
    int rain_kind; const float* rain; int ngh, nx, ny;
    const uint8_t* ncls; const float* ntab;
    float vcap; int quad, keep_h;
    float* max_h;
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

__device__ __forceinline__ void load_cell(const FlatK& p, Cell<float>& c, int64_t s) {
    c.h = __ldg(p.q0 + s); c.hu = __ldg(p.q1 + s); c.hv = __ldg(p.q2 + s);
}

__device__ __forceinline__ float grad_y_flat(const FlatK& p, const BrickView& v, float bc, int r, int lane) {
    float bl = __shfl_up_sync(0xffffffffu, bc, 1);
    float br = __shfl_down_sync(0xffffffffu, bc, 1);
    if (lane == 0)  bl = __ldg(p.b + v.outer_b(r, 0));
    if (lane == 31) br = __ldg(p.b + v.outer_b(r, 31));
    return 0.5f * (br - bl) * p.inv_dy;
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

template <bool STEP>
__global__ void __launch_bounds__(256) flat_march_kernel(FlatK p) {
    if (STEP && p.st->done) return;
    const int lane = threadIdx.x;
    const int64_t bidx = (int64_t)blockIdx.x * blockDim.y + threadIdx.y;
    unsigned long long lam_local = 0ull;
    float dt = 0.0f, rate = 0.0f;
    const float* frame = nullptr;
    if (STEP) {
        dt = p.st->dt_f32;
        if (p.rain_kind == GSW_RAIN_UNIFORM) rate = p.rain[p.st->rain_idx];
        if (p.rain_kind == GSW_RAIN_GRIDDED) frame = p.rain + (int64_t)p.st->rain_idx * p.nx * p.ny;
    }
    if (bidx < p.nb) {
        BrickView v;
        v.BS = (int64_t)p.bh * GSW_BRICK_PITCH;
        v.bh = p.bh;
        v.self = bidx;
        v.up = p.bnbr[4 * bidx + 0]; v.down = p.bnbr[4 * bidx + 1];
        v.left = p.bnbr[4 * bidx + 2]; v.right = p.bnbr[4 * bidx + 3];
        v.zero = p.nb;
        const int bi = p.bij[2 * bidx], bj = p.bij[2 * bidx + 1];
        const int bh = p.bh;

        Cell<float> cur, nx;
        const float b_m2 = __ldg(p.b + v.slot(-2, lane));
        { const int64_t s = v.slot(-1, lane); load_cell(p, cur, s); cur.b = __ldg(p.b + s); }
        { const int64_t s = v.slot(0, lane); load_cell(p, nx, s); nx.b = __ldg(p.b + s); }
        float b_next = __ldg(p.b + v.slot(1, lane));
        make_prims(cur, p.h_min);
        make_prims(nx, p.h_min);
        cur.gx = 0.5f * (nx.b - b_m2) * p.inv_dx;
        cur.gy = 0.0f;
        nx.gx = 0.5f * (b_next - cur.b) * p.inv_dx;
        nx.gy = grad_y_flat(p, v, nx.b, 0, lane);
        Face<float> Wf;
        srm_face<float, true>(cur, nx, p.half_dx, p.inv_dx, p.g, p.h_min, Wf);
        cur = nx;
        for (int r = 0; r < bh; ++r) {
            { const int64_t s = v.slot(r + 1, lane); load_cell(p, nx, s); }
            nx.b = b_next;
            const float b_p2 = __ldg(p.b + v.slot(r + 2, lane));
            make_prims(nx, p.h_min);
            nx.gx = 0.5f * (b_p2 - cur.b) * p.inv_dx;
            nx.gy = grad_y_flat(p, v, nx.b, r + 1, lane);
            Face<float> Ef;
            srm_face<float, true>(cur, nx, p.half_dx, p.inv_dx, p.g, p.h_min, Ef);
            const Cell<float> rn = shfl_down_cell(cur);
            Face<float> Nf;
            srm_face<float, false>(cur, rn, p.half_dy, p.inv_dy, p.g, p.h_min, Nf);
            const Face<float> Sf = shfl_up_face(Nf);
            if (lane >= 1 && lane <= 30) {
                const int64_t o = bidx * v.BS + (int64_t)r * GSW_BRICK_PITCH + (lane - 1);
                const uint8_t f = p.flags[o];
                if (f & GSW_SLOT_STORED) {
                    const bool active = (f & GSW_SLOT_ACTIVE) != 0;
                    if (!STEP) {
                        float rh = 0.0f, rhu = 0.0f, rhv = 0.0f;
                        if (active) accumulate(Ef, Wf, Nf, Sf, rh, rhu, rhv);
                        p.o0[o] = rh; p.o1[o] = rhu; p.o2[o] = rhv;
                    } else if (!active) {
                        p.o0[o] = cur.h; p.o1[o] = cur.hu; p.o2[o] = cur.hv;
                        if (p.max_h != nullptr && cur.h > p.max_h[o]) p.max_h[o] = cur.h;
                    } else {
                        float rh, rhu, rhv;
                        accumulate(Ef, Wf, Nf, Sf, rh, rhu, rhv);
                        float rr0 = rh;
                        if (p.rain_kind == GSW_RAIN_UNIFORM) rr0 = rr0 + rate;
                        else if (p.rain_kind == GSW_RAIN_GRIDDED) {
                            const int i = bi * bh + r, j = bj * GSW_BRICK_W + (lane - 1);
                            rr0 = rr0 + frame[(int64_t)(i - p.ngh) * p.ny + (j - p.ngh)];
                        }
                        float h = cur.h + dt * rr0;
                        float hu = cur.hu + dt * rhu;
                        float hv = cur.hv + dt * rhv;
                        const float n = p.ncls ? p.ntab[p.ncls[o]] : p.ntab[0];
                        wetdry_friction<float>(h, hu, hv, true, n, dt, p.g, p.h_min, p.vcap,
                                               p.quad != 0, p.keep_h != 0);
                        p.o0[o] = h; p.o1[o] = hu; p.o2[o] = hv;
                        if (p.max_h != nullptr && h > p.max_h[o]) p.max_h[o] = h;
                        if (p.lam != nullptr) {
                            const unsigned long long lb = lam_flat_bits(h, hu, hv, p.g, p.h_min, p.h_min_cfl,
                                                                        p.linf != 0);
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

__global__ void __launch_bounds__(256) flat_lammax_kernel(FlatK p, int64_t nslots, unsigned long long* out) {
    unsigned long long lam = 0ull;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (!(p.flags[s] & GSW_SLOT_ACTIVE)) continue;
        const unsigned long long lb = lam_flat_bits(p.q0[s], p.q1[s], p.q2[s], p.g, p.h_min, p.h_min_cfl,
                                                    p.linf != 0);
        lam = lb > lam ? lb : lam;
    }
    block_max_to(lam, out);
}

}  // namespace gsw

using namespace gsw;

static int fill_flat(const GswFlatArgs* a, FlatK& k, bool step) {
    if (a->brick_h < 2 || a->n_bricks < 0 || !a->brick_ij || !a->brick_nbr || !a->flags)
        return set_error(GSW_ERR_INVALID, "flat: bad brick tables (brick_h >= 2)");
    if (!a->q0 || !a->q1 || !a->q2 || !a->bed) return set_error(GSW_ERR_INVALID, "flat: null state/bed");
    k.q0 = a->q0; k.q1 = a->q1; k.q2 = a->q2;
    k.o0 = a->qn0; k.o1 = a->qn1; k.o2 = a->qn2;
    k.b = a->bed; k.flags = a->flags; k.bij = a->brick_ij; k.bnbr = a->brick_nbr;
    k.nb = a->n_bricks; k.bh = a->brick_h;
    k.inv_dx = a->inv_dx; k.inv_dy = a->inv_dy;
    k.half_dx = 0.5f * (1.0f / a->inv_dx); k.half_dy = 0.5f * (1.0f / a->inv_dy);
    k.g = a->g; k.h_min = a->h_min; k.h_min_cfl = a->h_min_cfl; k.linf = a->linf;
    k.st = a->state; k.lam = (unsigned long long*)a->lam_target;
    k.rain_kind = a->rain_kind; k.rain = a->rain; k.ngh = a->ngh; k.nx = a->nx; k.ny = a->ny;
    k.ncls = a->n_cls; k.ntab = a->n_tab; k.vcap = a->vcap; k.quad = a->quadratic; k.keep_h = a->keep_h;
    k.max_h = a->max_h;
    if (step) {
        if (!a->state) return set_error(GSW_ERR_INVALID, "flat step: state is required");
        if (!a->n_tab || a->n_tab_len < 1) return set_error(GSW_ERR_INVALID, "flat step: n_tab is required");
        if (a->rain_kind != GSW_RAIN_NONE && !a->rain) return set_error(GSW_ERR_INVALID, "flat step: rain is NULL");
        if (a->rain_kind == GSW_RAIN_GRIDDED && (a->nx <= 0 || a->ny <= 0 || a->ngh < 0))
            return set_error(GSW_ERR_INVALID, "flat step: gridded rain needs ngh, nx, ny");
        if (!k.o0 || !k.o1 || !k.o2) return set_error(GSW_ERR_INVALID, "flat step: null output");
    }
    return GSW_OK;
}

template <bool STEP>
static int launch_flat(const GswFlatArgs* a, cudaStream_t s) {
    FlatK k;
    int rc = fill_flat(a, k, STEP);
    if (rc) return rc;
    if (k.nb == 0) return GSW_OK;
    const int W = a->warps > 0 ? a->warps : 4;
    if (W < 1 || W > 8) return set_error(GSW_ERR_INVALID, "flat: warps must be in [1, 8]");
    const int64_t blocks = (k.nb + W - 1) / W;
    if (blocks > 0x7fffffffLL) return set_error(GSW_ERR_INVALID, "flat: too many bricks");
    flat_march_kernel<STEP><<<(unsigned)blocks, dim3(32, W), 0, s>>>(k);
    return check_launch("flat_march");
}

extern "C" int gsw_flat_step(const GswFlatArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    return launch_flat<true>(a, (cudaStream_t)stream);
}

extern "C" int gsw_flat_rhs(const GswFlatArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (!a->qn0 || !a->qn1 || !a->qn2) return set_error(GSW_ERR_INVALID, "flat rhs: null output");
    const size_t n = (size_t)(a->n_bricks + 1) * a->brick_h * GSW_BRICK_PITCH * sizeof(float);
    for (float* o : {a->qn0, a->qn1, a->qn2})
        if (cudaMemsetAsync(o, 0, n, (cudaStream_t)stream) != cudaSuccess)
            return set_error(GSW_ERR_CUDA, "flat rhs: memset failed");
    return launch_flat<false>(a, (cudaStream_t)stream);
}

extern "C" int gsw_flat_lammax(const GswFlatArgs* a, uint64_t* lam_bits, void* stream) {
    GSW_CHECK_ABI(a);
    FlatK k;
    int rc = fill_flat(a, k, false);
    if (rc) return rc;
    if (!lam_bits) return set_error(GSW_ERR_INVALID, "flat lammax: null output");
    const int64_t nslots = (k.nb + 1) * (int64_t)k.bh * GSW_BRICK_PITCH;
    const int grid = (int)std::min<int64_t>(sm_count() * 8, (nslots + 255) / 256);
    flat_lammax_kernel<<<std::max(grid, 1), 256, 0, (cudaStream_t)stream>>>(k, nslots, (unsigned long long*)lam_bits);
    return check_launch("flat_lammax");
}
