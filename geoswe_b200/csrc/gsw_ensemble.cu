// gsw_ensemble.cu -- a batch of compressed meshes advanced by one persistent kernel per step.
//
// All members' bricks sit in one brick storage. A step is one launch of a persistent
// grid (a few blocks per SM): warps stride over the global brick list, look up the
// brick's member, and advance it with that member's dt, rain rate and Manning table
// (gsw_flat.cu's per-brick march). Each member's new wave speed is reduced into its own
// GswLoopState. The block that finishes last (a ticket counter in scratch memory)
// then evaluates every member's time-step rule for the next launch, so members keep
// their own CFL dt with no grid-wide barrier and no host round trip; a member that
// reaches its end time drops out while the others continue.
#include "gsw_flat_brick.cuh"
#include <mutex>

namespace gsw {

__device__ __forceinline__ FlatPhys<float> member_phys(const GswMember& mb) {
    FlatPhys<float> ph;
    ph.inv_dx = mb.inv_dx; ph.inv_dy = mb.inv_dx;
    ph.half_dx = 0.5f * (1.0f / mb.inv_dx); ph.half_dy = ph.half_dx;
    ph.g = mb.g; ph.h_min = mb.h_min; ph.h_min_cfl = mb.h_min_cfl; ph.vcap = mb.vcap;
    ph.linf = mb.linf; ph.quad = mb.quadratic; ph.keep_h = mb.keep_h;
    ph.rain_kind = mb.rain_kind; ph.rain = mb.rain; ph.ntab = mb.n_tab;
    ph.ngh = 0; ph.nx = 0; ph.ny = 0; ph.lookup = nullptr; ph.ncol = 0;
    return ph;
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) ensemble_step_kernel(GswEnsembleArgs a, FlatMesh<float> m) {
    if (*a.all_done) return;
    const int lane = threadIdx.x;
    const int W = blockDim.y;
    for (int64_t b = (int64_t)blockIdx.x * W + threadIdx.y; b < a.n_bricks; b += (int64_t)gridDim.x * W) {
        const int mi = a.brick_member[b];
        const GswLoopState* st = a.states + mi;
        if (st->done) continue;                                   // warp-uniform
        const GswMember& mb = a.members[mi];
        const FlatPhys<float> ph = member_phys(mb);
        const float dt = st->dt_f32;
        const float rate = (mb.rain_kind == GSW_RAIN_UNIFORM) ? mb.rain[st->rain_idx] : 0.0f;
        unsigned long long lam = flat_brick<float, true>(m, ph, b, dt, rate, nullptr);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, lam, o);
            lam = w > lam ? w : lam;
        }
        if (lane == 0 && lam != 0ull) atomicMax((unsigned long long*)&a.states[mi].lam_bits, lam);
    }
    // the last block to arrive evaluates every member's rule for the next step
    __shared__ int s_last;
    __syncthreads();
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    if (tid == 0) {
        __threadfence();
        const unsigned int ticket = atomicAdd(&a.scratch[0], 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int nth = blockDim.x * blockDim.y;
    __shared__ int s_open;
    if (tid == 0) s_open = 0;
    __syncthreads();
    for (int mi = tid; mi < a.n_members; mi += nth) {
        GswLoopState* st = a.states + mi;
        const unsigned long long lb = atomicAdd((unsigned long long*)&st->lam_bits, 0ull);  // coherent read
        dt_finalize_one(a.members[mi].dt, st, lb);
        if (!st->done) atomicAdd(&s_open, 1);
    }
    __syncthreads();
    if (tid == 0) {
        a.scratch[0] = 0u;
        *a.all_done = (s_open == 0) ? 1 : 0;
    }
}

__global__ void ensemble_finalize_kernel(GswEnsembleArgs a) {
    __shared__ int s_open;
    if (threadIdx.x == 0) s_open = 0;
    __syncthreads();
    for (int mi = threadIdx.x; mi < a.n_members; mi += blockDim.x) {
        GswLoopState* st = a.states + mi;
        dt_finalize_one(a.members[mi].dt, st, st->lam_bits);
        if (!st->done) atomicAdd(&s_open, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a.scratch[0] = 0u;
        *a.all_done = (s_open == 0) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(256) ensemble_lammax_kernel(GswEnsembleArgs a) {
    const int64_t BS = (int64_t)a.brick_h * GSW_BRICK_PITCH;
    const int64_t nslots = a.n_bricks * BS;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (!(a.flags[s] & GSW_SLOT_ACTIVE)) continue;
        const int mi = a.brick_member[s / BS];
        const GswMember& mb = a.members[mi];
        const unsigned long long lb = lam_flat_bits(a.q0[s], a.q1[s], a.q2[s], mb.g, mb.h_min, mb.h_min_cfl,
                                                    mb.linf != 0);
        if (lb != 0ull) atomicMax((unsigned long long*)&a.states[mi].lam_bits, lb);
    }
}

}  // namespace gsw

using namespace gsw;

static int check_ens(const GswEnsembleArgs* a) {
    if (a->n_members <= 0 || a->n_members > 65536 || a->brick_h < 2 || a->n_bricks < 0)
        return set_error(GSW_ERR_INVALID, "ensemble: bad sizes");
    if (!a->brick_ij || !a->brick_nbr || !a->brick_member || !a->flags || !a->q0 || !a->q1 || !a->q2 ||
        !a->bed || !a->members || !a->states || !a->scratch || !a->all_done)
        return set_error(GSW_ERR_INVALID, "ensemble: null pointer");
    return GSW_OK;
}

extern "C" int gsw_ensemble_lammax(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    int rc = check_ens(a);
    if (rc) return rc;
    const int64_t nslots = a->n_bricks * (int64_t)a->brick_h * GSW_BRICK_PITCH;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(sm_count() * 8, (nslots + 255) / 256));
    ensemble_lammax_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(*a);
    return check_launch("ensemble_lammax");
}

extern "C" int gsw_ensemble_finalize(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    int rc = check_ens(a);
    if (rc) return rc;
    ensemble_finalize_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(*a);
    return check_launch("ensemble_finalize");
}

extern "C" int gsw_ensemble_step(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    int rc = check_ens(a);
    if (rc) return rc;
    if (!a->qn0 || !a->qn1 || !a->qn2) return set_error(GSW_ERR_INVALID, "ensemble step: null output");
    const int W = a->warps > 0 ? a->warps : 4;
    if (W < 1 || W > 8) return set_error(GSW_ERR_INVALID, "ensemble: warps must be in [1, 8]");
    const int grid = a->grid > 0 ? a->grid : 2 * sm_count();
    FlatMesh<float> m;
    m.q0 = a->q0; m.q1 = a->q1; m.q2 = a->q2;
    m.o0 = a->qn0; m.o1 = a->qn1; m.o2 = a->qn2;
    m.b = a->bed; m.flags = a->flags; m.ncls = a->n_cls; m.max_h = a->max_h;
    m.bij = a->brick_ij; m.bnbr = a->brick_nbr; m.nb = a->n_bricks; m.bh = a->brick_h;
    cudaStream_t st = (cudaStream_t)stream;
    if (a->min_blocks == 4) ensemble_step_kernel<4><<<grid, dim3(32, W), 0, st>>>(*a, m);
    else if (a->min_blocks == 5) ensemble_step_kernel<5><<<grid, dim3(32, W), 0, st>>>(*a, m);
    else if (a->min_blocks == 0) ensemble_step_kernel<1><<<grid, dim3(32, W), 0, st>>>(*a, m);
    else return set_error(GSW_ERR_INVALID, "ensemble: min_blocks must be 0, 4 or 5");
    return check_launch("ensemble_step");
}

// ---------------------------------------------------------------------------
// gsw_ensemble_step_static: the same launch with the ticket counter in library memory.
static __device__ __align__(256) unsigned int g_ens_static_scratch[GSW_ENS_STATIC_SCRATCH_WORDS];
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
unsigned int* g_static_ptr[kMaxDevices] = {};
}  // namespace

extern "C" int gsw_ensemble_step_static(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (GSW_ENS_SCRATCH_WORDS > GSW_ENS_STATIC_SCRATCH_WORDS)
        return set_error(GSW_ERR_RANGE, "ensemble step (static scratch): needs %d words, the static array "
                         "holds %d", GSW_ENS_SCRATCH_WORDS, GSW_ENS_STATIC_SCRATCH_WORDS);
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(GSW_ERR_CUDA, "ensemble step (static scratch): no device");
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(GSW_ERR_RANGE, "ensemble step (static scratch): device %d >= %d", dev, kMaxDevices);
    unsigned int* ptr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (g_static_ptr[dev] == nullptr) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_ens_static_scratch);
            if (e != cudaSuccess || p == nullptr)
                return set_error(GSW_ERR_CUDA, "ensemble step (static scratch): cudaGetSymbolAddress: %s",
                                 cudaGetErrorString(e));
            e = cudaMemsetAsync(p, 0, sizeof(g_ens_static_scratch), (cudaStream_t)stream);
            if (e != cudaSuccess)
                return set_error(GSW_ERR_CUDA, "ensemble step (static scratch): clearing the ticket: %s",
                                 cudaGetErrorString(e));
            g_static_ptr[dev] = (unsigned int*)p;
        }
        ptr = g_static_ptr[dev];
    }
    GswEnsembleArgs b = *a;
    b.scratch = ptr;
    return gsw_ensemble_step(&b, stream);
}
