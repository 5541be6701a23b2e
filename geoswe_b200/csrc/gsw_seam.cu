// gsw_seam.cu -- seam exchange of a compressed mesh split over ranks.
//
// The reference packs each face of its CompressedHalo with three CuPy fancy-index
// gathers into a dense (3, ngh, P) buffer and unpacks with three scatters
// (geoswe/compressed_solver.py:1069-1132). Here one launch moves all three planes of a
// face in either direction: thread k handles list entry k for the three planes, so the
// slot and position lists are read once.
#include "gsw_common.cuh"

namespace gsw {

template <typename T>
__global__ void __launch_bounds__(256) seam_copy_kernel(GswSeamArgs a) {
    T* q[3] = {(T*)a.q0, (T*)a.q1, (T*)a.q2};
    T* dense = (T*)a.dense;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < a.n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = a.slot[k], p = a.pos[k];
        if (s < 0 || s >= a.nslots || p < 0 || p >= a.stride) continue;
        if (a.scatter) {
#pragma unroll
            for (int c = 0; c < 3; ++c) q[c][s] = dense[c * a.stride + p];
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) dense[c * a.stride + p] = q[c][s];
        }
    }
}

}  // namespace gsw

using namespace gsw;

extern "C" int gsw_seam_copy(const GswSeamArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->n < 0 || a->stride < 1 || a->nslots < 0)
        return set_error(GSW_ERR_INVALID, "seam copy: negative count or stride < 1");
    if (a->n == 0) return GSW_OK;
    if (!a->q0 || !a->q1 || !a->q2 || !a->slot || !a->pos || !a->dense)
        return set_error(GSW_ERR_INVALID, "seam copy: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sm_count() * 8, (a->n + 255) / 256));
    if (a->dtype == GSW_F32) seam_copy_kernel<float><<<grid, 256, 0, s>>>(*a);
    else if (a->dtype == GSW_F64) seam_copy_kernel<double><<<grid, 256, 0, s>>>(*a);
    else return set_error(GSW_ERR_INVALID, "seam copy: bad dtype");
    return check_launch("seam_copy");
}
