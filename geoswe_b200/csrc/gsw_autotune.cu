// gsw_autotune.cu -- launch-shape search for the fused step kernels, in the library.
//
// No counterpart in the reference, whose kernels have fixed launch shapes. Each call
// times the step at every shape of a fixed search space with CUDA events on the
// caller's stream and buffers, and returns the fastest. The step's outputs serve as
// scratch; the wave-speed target and the running maximum are left untouched (the
// timed launches get NULL for both) and the loop state is only read. Results are kept
// per (device, kernel family, arithmetic, binary size, size class) in a table guarded
// by a mutex, so a second call for the same class returns without launching.
#include "gsw_common.cuh"
#include <map>
#include <mutex>
#include <string>

using namespace gsw;

namespace {

std::mutex g_tune_mu;
std::map<std::string, GswTuneResult> g_tune_cache;

std::string tune_key(const char* family, int arith, int dtype, int64_t cells) {
    int dev = -1;
    cudaGetDevice(&dev);
    const char* size = cells < (1LL << 20) ? "small" : (cells < (1LL << 24) ? "medium" : "large");
    return std::string(family) + "|" + std::to_string(dev) + "|" + std::to_string(arith) + "|" +
           std::to_string(dtype) + "|" + size;
}

// The loop state must not be done, or the timed launches would return at once.
int check_not_done(const GswLoopState* st, cudaStream_t s) {
    if (!st) return set_error(GSW_ERR_INVALID, "autotune: the step needs its loop state");
    GswLoopState h;
    if (cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return set_error(GSW_ERR_CUDA, "autotune: reading the loop state failed");
    if (h.done) return set_error(GSW_ERR_INVALID, "autotune: the loop state is done; time a live state");
    return GSW_OK;
}

// Mean time (ms) of `reps` launches of `launch` after one untimed launch; < 0 if the
// shape is refused (an invalid combination), which is skipped.
template <typename F>
float time_shape(F launch, int reps, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    if (launch() != GSW_OK) { cudaGetLastError(); return -1.0f; }
    cudaEventRecord(e0, s);
    for (int k = 0; k < reps; ++k)
        if (launch() != GSW_OK) { cudaGetLastError(); return -1.0f; }
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) return -1.0f;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / (float)reps;
}

}  // namespace

extern "C" int gsw_dense_autotune(const GswDenseArgs* a, int32_t reps, int32_t use_cache, GswTuneResult* out,
                                  void* stream) {
    GSW_CHECK_ABI(a);
    GSW_CHECK_ABI(out);
    if (reps < 1) return set_error(GSW_ERR_INVALID, "autotune: reps must be >= 1");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t cells = (int64_t)(a->nxp - 2 * a->ngh) * (a->nyp - 2 * a->ngh);
    const std::string key = tune_key("dense", a->arith, a->dtype, cells);
    if (use_cache) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) { *out = it->second; return GSW_OK; }
    }
    if (int rc = check_not_done(a->state, s)) return rc;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return set_error(GSW_ERR_CUDA, "autotune: cudaEventCreate failed");
    GswTuneResult best{};
    best.abi_version = GSW_ABI_VERSION;
    best.ms = 3.0e38f;
    const int rows[] = {0, 4, 8, 16, 32, 64}, warps[] = {2, 4, 8}, caps[] = {0, 3, 4, 5};
    for (int tr : rows)
        for (int w : warps)
            for (int mb : caps) {
                GswDenseArgs b = *a;
                b.lam_target = nullptr;
                b.max_h = nullptr;
                b.tile_rows = tr; b.warps = w; b.min_blocks = mb;
                const float ms = time_shape([&] { return gsw_dense_step(&b, stream); }, reps, s, e0, e1);
                if (ms < 0.0f) continue;
                ++best.n_tried;
                if (ms < best.ms) { best.ms = ms; best.tile_rows = tr; best.warps = w; best.min_blocks = mb; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best.n_tried == 0) return set_error(GSW_ERR_INVALID, "autotune: no launch shape ran (%s)", gsw_last_error());
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = best;
    }
    *out = best;
    return GSW_OK;
}

extern "C" int gsw_flat_autotune(const GswFlatArgs* a, int32_t reps, int32_t use_cache, GswTuneResult* out,
                                 void* stream) {
    GSW_CHECK_ABI(a);
    GSW_CHECK_ABI(out);
    if (reps < 1) return set_error(GSW_ERR_INVALID, "autotune: reps must be >= 1");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t slots = (a->n_bricks + 1) * (int64_t)a->brick_h * GSW_BRICK_PITCH;
    const std::string key = tune_key("flat", a->arith, a->dtype, slots);
    if (use_cache) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) { *out = it->second; return GSW_OK; }
    }
    if (int rc = check_not_done(a->state, s)) return rc;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return set_error(GSW_ERR_CUDA, "autotune: cudaEventCreate failed");
    GswTuneResult best{};
    best.abi_version = GSW_ABI_VERSION;
    best.ms = 3.0e38f;
    const int warps[] = {2, 4, 8}, caps[] = {0, 3, 4, 5}, segs[] = {0, 1, 2, 4};
    for (int w : warps)
        for (int mb : caps)
            for (int g : segs) {
                if (g > 0 && a->brick_h % g != 0) continue;
                GswFlatArgs b = *a;
                b.lam_target = nullptr;
                b.max_h = nullptr;
                b.warps = w; b.min_blocks = mb; b.segments = g;
                const float ms = time_shape([&] { return gsw_flat_step(&b, stream); }, reps, s, e0, e1);
                if (ms < 0.0f) continue;
                ++best.n_tried;
                if (ms < best.ms) { best.ms = ms; best.warps = w; best.min_blocks = mb; best.segments = g; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best.n_tried == 0) return set_error(GSW_ERR_INVALID, "autotune: no launch shape ran (%s)", gsw_last_error());
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = best;
    }
    *out = best;
    return GSW_OK;
}
