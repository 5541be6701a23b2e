// gsw_forcing.cuh -- NumPy-order helpers of the forcing kernels (inlet sums, np.interp).
#pragma once
#include "gsw_common.cuh"

namespace gsw {

// numpy's pairwise sum (add.reduce over a contiguous run): < 8 terms sequential;
// <= 128 terms in eight interleaved partial sums combined as ((0+1)+(2+3))+((4+5)+(6+7))
// plus a sequential tail; longer runs split at n/2 rounded down to a multiple of 8.
template <typename T>
__device__ inline T pairwise_sum(const T* q0, const int64_t* off, int64_t a, int64_t n) {
    if (n < 8) {
        T res = (T)0;
        for (int64_t i = 0; i < n; ++i) res = res + q0[off[a + i]];
        return res;
    }
    if (n <= 128) {
        T r[8];
        for (int k = 0; k < 8; ++k) r[k] = q0[off[a + k]];
        int64_t i = 8;
        for (; i < n - (n % 8); i += 8)
            for (int k = 0; k < 8; ++k) r[k] = r[k] + q0[off[a + i + k]];
        T res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res = res + q0[off[a + i]];
        return res;
    }
    int64_t n2 = n / 2;
    n2 -= n2 % 8;
    return pairwise_sum(q0, off, a, n2) + pairwise_sum(q0, off, a + n2, n - n2);
}

// np.interp(x, xp, fp) for one scalar x (numpy/_core/src/multiarray/compiled_base.c).
__device__ inline double np_interp(double x, const double* xp, const double* fp, int n) {
    if (n == 1) return fp[0];
    if (x != x) return x;
    if (x < xp[0]) return fp[0];
    if (x > xp[n - 1]) return fp[n - 1];
    int lo = 0, hi = n;                               // last j with xp[j] <= x
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (xp[mid] <= x) lo = mid + 1; else hi = mid; }
    const int j = lo - 1;
    if (j >= n - 1) return fp[n - 1];
    if (xp[j] == x) return fp[j];
    const double slope = __ddiv_rn(__dsub_rn(fp[j + 1], fp[j]), __dsub_rn(xp[j + 1], xp[j]));
    double r = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[j])), fp[j]);
    if (r != r) {
        r = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[j + 1])), fp[j + 1]);
        if (r != r && fp[j] == fp[j + 1]) r = fp[j];
    }
    return r;
}

}  // namespace gsw
