// gsw_core.cuh -- per-face and per-cell arithmetic of GeoSWE's SRM-HLLC step.
//
// Every expression follows the operand order of the reference kernel text
// (geoswe/rhs_cuda.py:900-1207 for the residual, :1757-1796 for the update tail) and
// is evaluated with separately rounded IEEE operations: the library is compiled with
// --fmad=false and uses no fast-math intrinsics, so the C oracle (oracle/gsw_oracle.c)
// reproduces every value. gsw_fast.cu compiles the binary32 step kernels a second time
// with GSW_FAST_ARITH (FMA contraction, approximate square root and division): the
// opt-in fast arithmetic, held to a stated depth tolerance instead of bit equality.
//
// Face sharing. The reference evaluates the four faces of every cell, so each
// interior face is computed twice, once from each side. From the right-hand cell
// every input of the face is the exact negation or the same value as from the
// left-hand cell (dz_clip and dz flip sign exactly, deta_L/deta_R swap), so the
// flux is bit-identical from both sides; only the bed source differs per side.
// The kernels here compute each face once and hand it to both cells.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gsw {

template <typename T> struct Real;
template <> struct Real<float>  { static __device__ __forceinline__ float  zero() { return 0.0f; } };
template <> struct Real<double> { static __device__ __forceinline__ double zero() { return 0.0; } };

// The reference's max()/min() device calls on floating point (fmaxf/fminf).
__device__ __forceinline__ float  gmax(float a, float b)   { return fmaxf(a, b); }
__device__ __forceinline__ float  gmin(float a, float b)   { return fminf(a, b); }
__device__ __forceinline__ double gmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ double gmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double gsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double gdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float  gabs(float a)   { return fabsf(a); }
__device__ __forceinline__ double gabs(double a)  { return fabs(a); }

#ifndef GSW_FAST_ARITH
// Exact arithmetic (the default compilation): IEEE square root and division.
__device__ __forceinline__ float gsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ float gdiv(float a, float b) { return a / b; }

// x, or 1 where `one` holds, through an opaque select. The substitutions below feed the
// IEEE operation an operand whose result is then discarded; written as a plain
// conditional, the compiler sees that the result is unused there and hands the
// operation the original operand again, which restores the slow path (measured: 2.9 M
// subroutine calls per 4096^2 step, all from exact-zero dividends). An asm select is
// opaque to that reasoning, so the substitution stays.
__device__ __forceinline__ float one_if(bool one, float x) {
    float r;
    asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %2, 0;\n\tselp.f32 %0, 0f3F800000, %1, p;\n\t}"
        : "=f"(r) : "f"(x), "r"((int)one));
    return r;
}
__device__ __forceinline__ double one_if(bool one, double x) {
    double r;
    asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %2, 0;\n\tselp.f64 %0, 0d3FF0000000000000, %1, p;\n\t}"
        : "=d"(r) : "d"(x), "r"((int)one));
    return r;
}

// Exact-zero operands take the IEEE square root's and division's out-of-range path,
// which is a subroutine call; dry faces (sqrt(g * 0)) and fluid at rest (0 / h) hit it
// on most cells. These forms keep every result bit for bit and keep the call off the
// zero case: sqrt(+-0) = +-0, and 0 / b = 0 * b (the same signed zero) for b finite
// and non-zero. Any other operand goes through the IEEE operation itself.
template <typename T>
__device__ __forceinline__ T sqrt_z(T x) {
    const bool zr = (x == (T)0);
    const T r = gsqrt(one_if(zr, x));
    return zr ? x : r;
}
template <typename T>
__device__ __forceinline__ T div_z(T a, T b) {
    const bool zr = (a == (T)0) && (b != (T)0) && (gabs(b) < (T)INFINITY);
    const T q = one_if(zr, a) / b;
    return zr ? a * b : q;
}
// a / b where b is never zero (a wet/dry floor h_min > 0 or a depth above it): only the
// dividend needs the zero test, and b's finiteness (0 / inf is 0, 0 * inf is not).
template <typename T>
__device__ __forceinline__ T div_znz(T a, T b) {
    const bool zr = (a == (T)0) && (gabs(b) < (T)INFINITY);
    const T q = one_if(zr, a) / b;
    return zr ? a * b : q;
}
// Binary32, the whole guard in one asm block: the zero test feeds both selects as a
// predicate, where the forms above pass it through an integer register (a select and
// an integer compare more per guard, 14 guards per cell). sqrt.rn and div.rn are the
// IEEE operations the C operators compile to.
template <>
__device__ __forceinline__ float sqrt_z<float>(float x) {
    float r;
    asm("{\n\t.reg .pred p;\n\t.reg .f32 t;\n\t"
        "setp.eq.f32 p, %1, 0f00000000;\n\t"
        "selp.f32 t, 0f3F800000, %1, p;\n\t"
        "sqrt.rn.f32 t, t;\n\t"
        "selp.f32 %0, %1, t, p;\n\t}"
        : "=f"(r) : "f"(x));
    return r;
}
template <>
__device__ __forceinline__ float div_z<float>(float a, float b) {
    float r;
    asm("{\n\t.reg .pred p;\n\t.reg .f32 t, m;\n\t"
        "abs.f32 m, %2;\n\t"
        "setp.eq.f32 p, %1, 0f00000000;\n\t"
        "setp.lt.and.f32 p, m, 0f7F800000, p;\n\t"
        "setp.gt.and.f32 p, m, 0f00000000, p;\n\t"
        "selp.f32 t, 0f3F800000, %1, p;\n\t"
        "div.rn.f32 t, t, %2;\n\t"
        "mul.rn.f32 m, %1, %2;\n\t"
        "selp.f32 %0, m, t, p;\n\t}"
        : "=f"(r) : "f"(a), "f"(b));
    return r;
}
template <>
__device__ __forceinline__ float div_znz<float>(float a, float b) {
    float r;
    asm("{\n\t.reg .pred p;\n\t.reg .f32 t, m;\n\t"
        "abs.f32 m, %2;\n\t"
        "setp.eq.f32 p, %1, 0f00000000;\n\t"
        "setp.lt.and.f32 p, m, 0f7F800000, p;\n\t"
        "selp.f32 t, 0f3F800000, %1, p;\n\t"
        "div.rn.f32 t, t, %2;\n\t"
        "mul.rn.f32 m, %1, %2;\n\t"
        "selp.f32 %0, m, t, p;\n\t}"
        : "=f"(r) : "f"(a), "f"(b));
    return r;
}
#else
// Fast arithmetic (gsw_fast.cu, compiled with FMA contraction and flush-to-zero):
// binary32 square root and division by the hardware approximations, sqrt.approx
// (relative error about 2^-23) and div.full (at most 2 ulp, full range); no slow path,
// so no zero guards. Binary64 keeps the IEEE operations.
__device__ __forceinline__ float gsqrt(float a) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}
__device__ __forceinline__ float gdiv(float a, float b) {
    float r;
    asm("div.full.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float  sqrt_z(float x) { return gsqrt(x); }
__device__ __forceinline__ float  div_z(float a, float b) { return gdiv(a, b); }
__device__ __forceinline__ float  div_znz(float a, float b) { return gdiv(a, b); }
__device__ __forceinline__ double sqrt_z(double x) { return x == 0.0 ? x : sqrt(x); }
__device__ __forceinline__ double div_z(double a, double b) { return a / b; }
__device__ __forceinline__ double div_znz(double a, double b) { return a / b; }
#endif

// q = h / g for the HLLC star depth, by the constant's reciprocal when the library has
// shown that this is the IEEE quotient: y = RN(1/g), q0 = RN(h y), r = h - g q0 (exact,
// one FMA), q = RN(q0 + r y) -- P. Markstein's correction step ("IA-64 and Elementary
// Functions", 2000), as used for division by a constant by Brisebarre, Muller and
// Raina (IEEE Trans. Computers 53(8), 2004). gsw_rt::div_const_recip checks the
// sequence against the IEEE quotient for every binary32 significand of h with this g
// (rounding commutes with scaling by powers of two, so [1, 2) covers every h whose
// products stay normal, which the range test below ensures) and passes y, else 0.
template <typename T>
__device__ __forceinline__ T div_g(T h, T g, T y) { return gdiv(h, g); }
#ifndef GSW_FAST_ARITH
template <>
__device__ __forceinline__ float div_g<float>(float h, float g, float y) {
    if (y != 0.0f && h >= 0x1p-100f && h <= 0x1p100f) {
        const float q0 = h * y;
        const float r = fmaf(-g, q0, h);
        return fmaf(r, y, q0);
    }
    return h / g;
}
#endif

// Primitive state of one cell (PRIMS macro, rhs_cuda.py:931-938) plus what the
// faces need: free surface and the central bed gradients.
template <typename T>
struct Cell {
    T h, hu, hv;   // conserved state (the update needs hu, hv)
    T u, v;        // velocities, 0 when h <= h_min
    T eta, b;      // free surface h + b and bed
    T gx, gy;      // central bed gradients 0.5*(b+ - b-)*inv_d (rhs_cuda.py:1644-1651)
};

template <typename T>
__device__ __forceinline__ void make_prims(Cell<T>& c, T h_min) {
    const T hs = (c.h > h_min) ? c.h : h_min;
    c.u = (c.h > h_min) ? div_znz(c.hu, hs) : Real<T>::zero();   // hs = h > h_min >= 0 where used
    c.v = (c.h > h_min) ? div_znz(c.hv, hs) : Real<T>::zero();
    c.eta = c.h + c.b;
}

// x^(-4/3) for the Manning coefficient, x >= h_min > 0.
// r = x^(-1/3) from an exponent-splitting first guess (bits(r) ~ (4/3)(127-s)2^23 -
// bits(x)/3 with s = 0.0450466, the log-linear offset of IEEE binary32) refined by
// three Newton steps r <- r + r*(1 - x r^3)/3 on f(r) = r^-3 - x, then x^(-4/3) = r/x.
// Only IEEE +,-,*,/ and integer ops, so C and CUDA give the same bits. Accuracy
// <= 1.85 ulp of the exact x^(-4/3) over [1e-7, 1e3] (the reference's powf evaluates
// x^fl32(-4/3), within ~9 ulp of the exact power).
__device__ __forceinline__ float pow_m43(float x) {
    const uint32_t ix = __float_as_uint(x);
    float r = __uint_as_float(0x54a2fa8du - ix / 3u);
    const float third = 0.333333343267440796f;
#pragma unroll
    for (int it = 0; it < 3; ++it) {
        float t = r * r;
        t = t * r;
        t = x * t;
        t = 1.0f - t;
        t = r * t;
        t = t * third;
        r = r + t;
    }
    return gdiv(r, x);
}
// fp64: the same iteration in double, six steps from the binary32 guess; r/x is within
// ~6 double ulp of x^(-4/3).
__device__ __forceinline__ double pow_m43(double x) {
    const float xf = (float)x;
    const uint32_t ix = __float_as_uint(xf);
    double r = (double)__uint_as_float(0x54a2fa8du - ix / 3u);
    const double third = 0.333333333333333315;
#pragma unroll
    for (int it = 0; it < 6; ++it) {
        double t = r * r;
        t = t * r;
        t = x * t;
        t = 1.0 - t;
        t = r * t;
        t = t * third;
        r = r + t;
    }
    return r / x;
}

// Manning's h^(-4/3) as the reference kernel text evaluates it: powf(hs, -4.0f/3.0f)
// (rhs_cuda.py:1830, compressed_rhs.py:730), CUDA's own powf, called, not restated; the
// library is compiled without contraction, as the reference's strict build. The
// reference's friction is binary32 only; binary64 keeps the iteration above.
__device__ __forceinline__ float pow_m43_ref(float x) { return powf(x, -4.0f / 3.0f); }
__device__ __forceinline__ double pow_m43_ref(double x) { return pow_m43(x); }

// HLLC flux in the face frame (rhs_cuda.py:986-1036) with Sigma = 0 (the no-sigma
// build, rhs_cuda.py:1717-1722): uN normal, uT transverse velocity.
template <typename T>
__device__ __forceinline__ void hllc(T hL, T uNL, T uTL, T hR, T uNR, T uTR,
                                     T g, T h_min, T& Fh, T& FN, T& FT, T g_recip = (T)0) {
    const T z = Real<T>::zero();
    const T half = (T)0.5, quarter = (T)0.25, two = (T)2.0;
    const T aL = sqrt_z(g * (hL > z ? hL : z));
    const T aR = sqrt_z(g * (hR > z ? hR : z));
    const T u_st = half * (uNL + uNR) + aL - aR;
    const T h_rt = half * (aL + aR) + quarter * (uNL - uNR);
    const T h_st = (h_rt > z) ? div_g(h_rt * h_rt, g, g_recip) : z;
    const T a_st = sqrt_z(g * (h_st > z ? h_st : z));
    const T SL_w = gmin(uNL - aL, u_st - a_st);
    const T SR_w = gmax(uNR + aR, u_st + a_st);
    const bool dryL = (hL <= h_min);
    const bool dryR = (hR <= h_min);
    T SL = dryL ? (uNR - two * aR) : SL_w;
    T SR = dryR ? (uNL + two * aL) : SR_w;
    if (dryL && dryR) { SL = z; SR = z; }
    const T denom = hR * (uNR - SR) - hL * (uNL - SL);
    T SM;
    if (gabs(denom) > (T)1.0e-14) {
        SM = div_z(SL * hR * (uNR - SR) - SR * hL * (uNL - SL), denom);
    } else {
        SM = half * (uNL + uNR);
    }
    // The reference returns F_L where SL >= 0, the star flux of the side of the contact
    // (SM >= 0: left) where SL < 0 <= SR or that side is left, else F_R. Each of these
    // reads one side's physical flux only: side P is L where SL >= 0, else the star side
    // K. So the physical flux is evaluated for side P alone, with the reference's
    // expressions for that side (huN = h uN, F_N = huN uN + 0.5 g h h, F_T = huN uT),
    // and one star state for side K: one division, no divergent branches, and the same
    // values wherever the reference's select uses them.
    const bool left = SM >= z;
    const bool useL = SL >= z;
    const bool sideL = useL || left;
    const T hP = sideL ? hL : hR, uNP = sideL ? uNL : uNR, uTP = sideL ? uTL : uTR;
    const T huNP = hP * uNP;
    const T huTP = hP * uTP;
    const T pP = half * g * hP * hP;
    const T FP_h = huNP;
    const T FP_N = huNP * uNP + pP;
    const T FP_T = huNP * uTP;
    // star state of side K (= P wherever it is used: SL < 0 there)
    const T S = left ? SL : SR;
    const T fac = gdiv(S - uNP, S - SM + (T)1.0e-30);
    const T hKs = hP * fac;
    const T huNKs = hKs * SM;
    const T huTKs = hKs * uTP;
    const T Fs_h = FP_h + S * (hKs - hP);
    const T Fs_N = FP_N + S * (huNKs - huNP);
    const T Fs_T = FP_T + S * (huTKs - huTP);
    const bool star = !useL && (left || SR >= z);
    Fh = star ? Fs_h : FP_h;
    FN = star ? Fs_N : FP_N;
    FT = star ? Fs_T : FP_T;
}

// One face between cell L (lower index) and cell R (upper index) along one axis.
// Outputs are already scaled by 1/d, as the reference accumulates F*inv_d:
//   Fh, Fn, Ft : mass, normal-momentum, transverse-momentum flux * inv_d
//   srcL       : SRM bed source of the face for cell L (its +side), * inv_d
//   srcR       : SRM bed source of the face for cell R (its -side), * inv_d
//   wet        : false when both cells are below h_min (the face is skipped)
template <typename T>
struct Face { T Fh, Fn, Ft, srcL, srcR; bool wet; };

template <typename T, bool XAXIS>
__device__ __forceinline__ void srm_face(const Cell<T>& L, const Cell<T>& R,
                                         T half_d, T inv_d, T g, T h_min, Face<T>& F, T g_recip = (T)0) {
    const T z = Real<T>::zero();
    F.wet = !(L.h < h_min && R.h < h_min);
    if (!F.wet) { F.Fh = z; F.Fn = z; F.Ft = z; F.srcL = z; F.srcR = z; return; }
    const T gL = XAXIS ? L.gx : L.gy;
    const T gR = XAXIS ? R.gx : R.gy;
    // rhs_cuda.py:1044-1054 (cell L's frame; cell R's frame is the exact mirror)
    const T zL = L.b + half_d * gL;
    const T zR = R.b - half_d * gR;
    const T zf0 = (L.b > R.b) ? L.b : R.b;
    const T dz_clip = zR - zL;
    const T dz = R.b - L.b - dz_clip;
    const T deta_L = gmax(z, gmin(dz, R.eta - L.eta));
    const T deta_R = gmax(z, gmin(-dz, L.eta - R.eta));
    const T eta_Lf = L.eta + deta_L;
    const T eta_Rf = R.eta + deta_R;
    const T h_Lf = gmax(z, eta_Lf - zf0);
    const T h_Rf = gmax(z, eta_Rf - zf0);
    T Fh, FN, FT;
    if (XAXIS) hllc<T>(h_Lf, L.u, L.v, h_Rf, R.u, R.v, g, h_min, Fh, FN, FT, g_recip);
    else       hllc<T>(h_Lf, L.v, L.u, h_Rf, R.v, R.u, g, h_min, Fh, FN, FT, g_recip);
    F.Fh = Fh * inv_d;
    F.Fn = FN * inv_d;
    F.Ft = FT * inv_d;
    // bed source, cell L (rhs_cuda.py:1062-1072)
    {
        T dzb;
        if (R.h < h_min) dzb = gmax(z, zf0 - L.eta);
        else             dzb = gmax(z, gmin(dz_clip, zf0 - L.eta));
        const T zf = zf0 - dzb;
        const T src = (T)0.5 * g * (h_Lf + L.h) * (zf - L.b);
        F.srcL = src * inv_d;
    }
    // bed source, cell R: its frame has dz_clip' = -dz_clip (rhs_cuda.py:1092-1104)
    {
        T dzb;
        if (L.h < h_min) dzb = gmax(z, zf0 - R.eta);
        else             dzb = gmax(z, gmin(-dz_clip, zf0 - R.eta));
        const T zf = zf0 - dzb;
        const T src = (T)0.5 * g * (h_Rf + R.h) * (zf - R.b);
        F.srcR = src * inv_d;
    }
}

// Residual of one cell from its four faces, accumulated in the reference order:
// x-face i+1/2 (E), x-face i-1/2 (W), y-face j+1/2 (N), y-face j-1/2 (S).
// E and N have this cell on their L side, W and S on their R side.
template <typename T>
__device__ __forceinline__ void accumulate(const Face<T>& E, const Face<T>& W,
                                           const Face<T>& N, const Face<T>& S,
                                           T& rh, T& rhu, T& rhv) {
    rh = Real<T>::zero(); rhu = Real<T>::zero(); rhv = Real<T>::zero();
    if (E.wet) { rh = rh - E.Fh; rhu = rhu - E.Fn; rhv = rhv - E.Ft; rhu = rhu - E.srcL; }
    if (W.wet) { rh = rh + W.Fh; rhu = rhu + W.Fn; rhv = rhv + W.Ft; rhu = rhu + W.srcR; }
    if (N.wet) { rh = rh - N.Fh; rhu = rhu - N.Ft; rhv = rhv - N.Fn; rhv = rhv - N.srcL; }
    if (S.wet) { rh = rh + S.Fh; rhu = rhu + S.Ft; rhv = rhv + S.Fn; rhv = rhv + S.srcR; }
}

// Wet/dry floor and point-implicit Manning friction on an updated cell
// (rhs_cuda.py:1765-1790; solver.py:233-307). friction == false applies the wet/dry
// floor alone, as the reference does when Config.friction is None (solver.py:2952-2962).
// ref_pow: h^(-4/3) by pow_m43_ref (GSW_ARITH_EXACT), else by pow_m43 (GSW_ARITH_PORTABLE
// and the fast arithmetic).
template <typename T>
__device__ __forceinline__ void wetdry_friction(T& h, T& hu, T& hv, bool friction, T n,
                                                T dt, T g, T h_min, T vcap,
                                                bool quadratic, bool keep_h, bool ref_pow) {
    const T z = Real<T>::zero();
    if (h < h_min) {
        h = keep_h ? (h > z ? h : z) : z;
        hu = z; hv = z;
        return;
    }
    if (!friction) return;
    const T hs = (h > h_min) ? h : h_min;
    const T u = div_znz(hu, hs);      // hs >= h_min > 0
    const T v = div_znz(hv, hs);
    const T modU = sqrt_z(u * u + v * v);
    const T h43 = ref_pow ? pow_m43_ref(hs) : pow_m43(hs);
    if (modU > vcap) {
        const T n_cri = gsqrt(gdiv((T)1.0, ((T)1.0e-10 + dt) * g * h43 * (modU + (T)1.0e-30)));
        if (n_cri > n) n = n_cri;
    }
    const T Cf = g * n * n * h43;
    T alpha;
    if (quadratic) {
        const T twodtCfU = (T)2.0 * dt * Cf * modU;
        alpha = gdiv((T)2.0, gsqrt((T)1.0 + (T)2.0 * twodtCfU) + (T)1.0);
    } else {
        alpha = gdiv((T)1.0, (T)1.0 + dt * Cf * modU);
    }
    hu = hu * alpha;
    hv = hv * alpha;
}

// Wave speeds are reduced as the IEEE bits of a non-negative double (unsigned order
// is the float order for non-negative values, and NaN/Inf sit above every finite
// value), so fp32 and fp64 runs share one 64-bit atomicMax target.
//
// Dense loop, fp32 (lammax_fp32_lean, solver.py:152-205): cells with h < h_cfl give
// 0, u = hu/h, non-finite -> +Inf.
__device__ __forceinline__ unsigned long long lam_dense_bits(float h, float hu, float hv,
                                                             float g, float h_cfl) {
    if (h < h_cfl) return 0ull;
    // max(|hu/h|, |hv/h|) with one division: a correctly rounded division by h > 0 is
    // monotonic and symmetric, so it equals max(|hu|, |hv|) / h to the bit (NaN momentum
    // is tested on its own; a NaN or infinite h leaves the quotient non-finite)
    const float ahu = fabsf(hu), ahv = fabsf(hv);
    const float aw = div_znz(ahu > ahv ? ahu : ahv, h);       // h >= h_cfl > 0, or NaN
    const float lam = aw + gsqrt(g * h);
    const bool fin = (hu == hu) && (hv == hv) && (lam <= 3.0e38f) && (aw <= 3.0e38f);
    return fin ? (unsigned long long)__double_as_longlong((double)lam) : 0x7ff0000000000000ull;
}
// The same rule as the bits of the binary32 wave speed: unsigned order of the bits of
// non-negative floats is their order, with +inf (the non-finite case) above every finite
// value, and widening to binary64 is monotonic, so the maximum of these bits, widened
// once, equals the maximum of lam_dense_bits over the same cells. A march keeps one
// 32-bit maximum per thread instead of converting and comparing 64-bit values per cell.
__device__ __forceinline__ uint32_t lam_dense_bits32(float h, float hu, float hv, float g, float h_cfl) {
    if (h < h_cfl) return 0u;
    const float ahu = fabsf(hu), ahv = fabsf(hv);
    const float aw = div_znz(ahu > ahv ? ahu : ahv, h);       // h >= h_cfl > 0, or NaN
    const float lam = aw + gsqrt(g * h);
    const bool fin = (hu == hu) && (hv == hv) && (lam <= 3.0e38f) && (aw <= 3.0e38f);
    return fin ? __float_as_uint(lam) : 0x7f800000u;
}
__device__ __forceinline__ unsigned long long lam_bits_of32(uint32_t b) {
    return (unsigned long long)__double_as_longlong((double)__uint_as_float(b));
}

// Dense loop, fp64 (the generic path, solver.py:2668-2693 with swe.max_wave_speed_2d):
// every cell counts, u = 0 where h <= h_cfl else hu/max(h, h_cfl), c = sqrt(g max(h,0)).
// The all-dry floor sqrt(g h_cfl) is applied by gsw_dt_finalize, so whether cells below
// h_cfl contribute sqrt(g h) < floor or nothing gives the same dt.
__device__ __forceinline__ unsigned long long lam_dense_bits(double h, double hu, double hv,
                                                             double g, double h_cfl) {
    const bool dry = h <= h_cfl;
    const double hs = h > h_cfl ? h : h_cfl;
    const double u = dry ? 0.0 : div_z(hu, hs);
    const double v = dry ? 0.0 : div_z(hv, hs);
    const double c = sqrt(g * (h > 0.0 ? h : 0.0));
    const double au = fabs(u), av = fabs(v);
    const double lam = ((au > av) ? au : av) + c;
    if (!(lam <= 1.0e308)) return 0x7ff0000000000000ull;   // NaN or Inf
    return (unsigned long long)__double_as_longlong(lam);
}

// Flat loop (cfl_lammax_flat_blk_ns, compressed_solver.py:209-244, and the fused
// _LAM_BLOCK, compressed_rhs.py:1027-1039), fp32: NaN depth -> quiet NaN; h < h_min
// -> 0; divisor floored at h_min_cfl; L2 norm, or Linf with cfl_linf.
__device__ __forceinline__ unsigned long long lam_flat_bits(float h, float hu, float hv, float g,
                                                            float h_min, float h_min_cfl,
                                                            bool linf) {
    if (h != h) return 0x7ff8000000000000ull;
    if (h < h_min) return 0ull;
    const float hs = h > h_min_cfl ? h : h_min_cfl;
    const float c = gsqrt(g * (h > 0.0f ? h : 0.0f));
    float speed;
    if (linf) {   // one division, as in lam_dense_bits (fmaxf ignores a NaN operand, as before)
        const float ahu = (hu == hu) ? fabsf(hu) : 0.0f, ahv = (hv == hv) ? fabsf(hv) : 0.0f;
        speed = div_znz(ahu > ahv ? ahu : ahv, hs);             // hs >= h_min_cfl > 0
        if (hu != hu && hv != hv) speed = __int_as_float(0x7fffffff);
    } else {
        const float u = div_znz(hu, hs), v = div_znz(hv, hs);
        speed = sqrt_z(u * u + v * v);
    }
    const float l = speed + c;
    return (unsigned long long)__double_as_longlong((double)l);
}
// The L2 rule as the bits of the binary32 speed (see lam_dense_bits32): NaN depth gives the
// quiet NaN 0x7fc00000, which widens to the 0x7ff8000000000000 above, and widening keeps
// the unsigned order of these bits (positive values, +inf, then NaNs), so the maximum of
// the 32-bit keys, widened once, is the maximum of lam_flat_bits over the same cells.
__device__ __forceinline__ uint32_t lam_flat_bits32(float h, float hu, float hv, float g, float h_min,
                                                    float h_min_cfl) {
    if (h != h) return 0x7fc00000u;
    if (h < h_min) return 0u;
    const float hs = h > h_min_cfl ? h : h_min_cfl;
    const float c = gsqrt(g * (h > 0.0f ? h : 0.0f));
    const float u = div_znz(hu, hs), v = div_znz(hv, hs);
    const float speed = sqrt_z(u * u + v * v);
    return __float_as_uint(speed + c);
}
// The same rule in double (the flat tier is fp32 in the reference; fp64 runs exist for
// the adjoint's finite-difference and autograd checks).
__device__ __forceinline__ unsigned long long lam_flat_bits(double h, double hu, double hv, double g,
                                                            double h_min, double h_min_cfl, bool linf) {
    if (h != h) return 0x7ff8000000000000ull;
    if (h < h_min) return 0ull;
    const double hs = h > h_min_cfl ? h : h_min_cfl;
    const double u = div_z(hu, hs), v = div_z(hv, hs);
    const double c = sqrt(g * (h > 0.0 ? h : 0.0));
    const double speed = linf ? fmax(fabs(u), fabs(v)) : sqrt_z(u * u + v * v);
    return (unsigned long long)__double_as_longlong(speed + c);
}

}  // namespace gsw
