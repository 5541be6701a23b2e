// gsw_adjoint.cuh -- reverse-mode derivatives of the fused step's arithmetic.
//
// Each function recomputes its forward values from the same inputs (so it takes the
// same branches as the forward pass: the wet/dry pattern, the HLLC region, every
// min/max selection) and propagates adjoints back through them. Conventions at
// ties, shared with the plain-PyTorch check implementation:
//   max(0, x)     -> x when x > 0
//   fminf(a, b)   -> a when a <= b;   fmaxf(a, b) -> a when a >= b
//   sqrt(g x)     -> derivative 0 where x <= 0
//   u = hu / h    -> only where h > h_min (else u = 0, a constant)
// h^(-4/3) (powf or pow_m43, as the forward step) is differentiated as the exact power,
// -4/3 h^(-7/3).
// The forward values are recomputed with the forward step's own operations (so every
// branch matches); the adjoint arithmetic itself divides once per denominator and
// multiplies by that reciprocal (a derivative, not a value the forward pass compares).
#pragma once
#include "gsw_core.cuh"

namespace gsw {

template <typename T>
struct Bar3 { T h, hu, hv; };

// F = (h uN, h uN^2 + g h^2 / 2, h uN uT)
template <typename T>
__device__ __forceinline__ void flux_bwd(T h, T uN, T uT, T g, T Fh_b, T FN_b, T FT_b,
                                         T& h_b, T& uN_b, T& uT_b) {
    const T hu = h * uN;
    const T hu_b = Fh_b + FN_b * uN + FT_b * uT;
    uN_b += FN_b * hu + hu_b * h;
    uT_b += FT_b * hu;
    h_b += hu_b * uN + FN_b * g * h;
}

// Reverse of hllc() (gsw_core.cuh), adjoints added into the *_b outputs.
template <typename T>
__device__ __forceinline__ void hllc_bwd(T hL, T uNL, T uTL, T hR, T uNR, T uTR, T g, T h_min,
                                         T Fh_b, T FN_b, T FT_b,
                                         T& hL_b, T& uNL_b, T& uTL_b, T& hR_b, T& uNR_b, T& uTR_b) {
    const T z = Real<T>::zero();
    const T half = (T)0.5, quarter = (T)0.25, two = (T)2.0;
    const T aL = sqrt_z(g * (hL > z ? hL : z));
    const T aR = sqrt_z(g * (hR > z ? hR : z));
    const T u_st = half * (uNL + uNR) + aL - aR;
    const T h_rt = half * (aL + aR) + quarter * (uNL - uNR);
    const T h_st = (h_rt > z) ? (h_rt * h_rt) / g : z;
    const T a_st = sqrt_z(g * (h_st > z ? h_st : z));
    const T A1 = uNL - aL, A2 = u_st - a_st;
    const T B1 = uNR + aR, B2 = u_st + a_st;
    const bool dryL = (hL <= h_min);
    const bool dryR = (hR <= h_min);
    T SL = dryL ? (uNR - two * aR) : gmin(A1, A2);
    T SR = dryR ? (uNL + two * aL) : gmax(B1, B2);
    if (dryL && dryR) { SL = z; SR = z; }
    const T dR = uNR - SR, dL = uNL - SL;
    const T denom = hR * dR - hL * dL;
    const bool big = gabs(denom) > (T)1.0e-14;
    T SM;
    if (big) SM = div_z(SL * hR * dR - SR * hL * dL, denom);
    else     SM = half * (uNL + uNR);
    const bool left = SM >= z;

    T SL_b = z, SR_b = z, SM_b = z;
    if (SL >= z) {
        flux_bwd(hL, uNL, uTL, g, Fh_b, FN_b, FT_b, hL_b, uNL_b, uTL_b);
    } else if (left || SR >= z) {
        const T S = left ? SL : SR;
        const T hK = left ? hL : hR, uNK = left ? uNL : uNR, uTK = left ? uTL : uTR;
        const T huNK = hK * uNK, huTK = hK * uTK;
        const T D = S - SM + (T)1.0e-30;
        const T fac = (S - uNK) / D;
        const T rD = (T)1.0 / D;
        const T hKs = hK * fac;
        const T huNKs = hKs * SM;
        const T huTKs = hKs * uTK;
        T S_b = Fh_b * (hKs - hK) + FN_b * (huNKs - huNK) + FT_b * (huTKs - huTK);
        T hKs_b = Fh_b * S;
        const T huNKs_b = FN_b * S, huTKs_b = FT_b * S;
        T hK_b = -(Fh_b * S), uNK_b = z, uTK_b = z;
        const T huNK_b = -(FN_b * S), huTK_b = -(FT_b * S);
        hKs_b += huTKs_b * uTK; uTK_b += huTKs_b * hKs;
        hKs_b += huNKs_b * SM;  SM_b += huNKs_b * hKs;
        hK_b += hKs_b * fac;
        const T fac_b = hKs_b * hK;
        const T facD_b = fac_b * rD;
        S_b += facD_b * ((T)1.0 - fac);
        uNK_b -= facD_b;
        SM_b += facD_b * fac;
        flux_bwd(hK, uNK, uTK, g, Fh_b, FN_b, FT_b, hK_b, uNK_b, uTK_b);   // the K-side flux
        hK_b += huNK_b * uNK + huTK_b * uTK;
        uNK_b += huNK_b * hK;
        uTK_b += huTK_b * hK;
        if (left) { hL_b += hK_b; uNL_b += uNK_b; uTL_b += uTK_b; SL_b += S_b; }
        else      { hR_b += hK_b; uNR_b += uNK_b; uTR_b += uTK_b; SR_b += S_b; }
    } else {
        flux_bwd(hR, uNR, uTR, g, Fh_b, FN_b, FT_b, hR_b, uNR_b, uTR_b);
    }
    if (SM_b != z) {
        if (big) {
            const T num_b = SM_b / denom;
            const T den_b = -(num_b * SM);
            T dR_b = num_b * SL * hR, dL_b = -(num_b * SR * hL);
            SL_b += num_b * hR * dR;
            hR_b += num_b * SL * dR;
            SR_b -= num_b * hL * dL;
            hL_b -= num_b * SR * dL;
            hR_b += den_b * dR; dR_b += den_b * hR;
            hL_b -= den_b * dL; dL_b -= den_b * hL;
            uNR_b += dR_b; SR_b -= dR_b;
            uNL_b += dL_b; SL_b -= dL_b;
        } else {
            uNL_b += half * SM_b;
            uNR_b += half * SM_b;
        }
    }
    T aL_b = z, aR_b = z, u_st_b = z, a_st_b = z;
    if (!(dryL && dryR)) {
        if (dryL)          { uNR_b += SL_b; aR_b -= two * SL_b; }
        else if (A1 <= A2) { uNL_b += SL_b; aL_b -= SL_b; }
        else               { u_st_b += SL_b; a_st_b -= SL_b; }
        if (dryR)          { uNL_b += SR_b; aL_b += two * SR_b; }
        else if (B1 >= B2) { uNR_b += SR_b; aR_b += SR_b; }
        else               { u_st_b += SR_b; a_st_b += SR_b; }
    }
    const T h_st_b = (h_st > z && a_st > z) ? a_st_b * g / (two * a_st) : z;
    const T h_rt_b = (h_rt > z) ? h_st_b * two * h_rt * ((T)1.0 / g) : z;   // 1/g: loop-invariant
    aL_b += half * h_rt_b; aR_b += half * h_rt_b;
    uNL_b += quarter * h_rt_b; uNR_b -= quarter * h_rt_b;
    uNL_b += half * u_st_b; uNR_b += half * u_st_b;
    aL_b += u_st_b; aR_b -= u_st_b;
    if (hL > z && aL > z) hL_b += aL_b * g / (two * aL);
    if (hR > z && aR > z) hR_b += aR_b * g / (two * aR);
}

// Adjoints of one face's outputs (the quantities srm_face writes, already * inv_d).
template <typename T>
struct FaceBar { T Fh, Fn, Ft, srcL, srcR; };

// Reverse of srm_face<T, XAXIS>: adjoints of cell L's and cell R's (h, hu, hv) added
// into Lb and Rb. L and R carry the forward cell values (h, u, v, eta, b, gx, gy).
template <typename T, bool XAXIS>
__device__ __forceinline__ void srm_face_bwd(const Cell<T>& L, const Cell<T>& R, T half_d, T inv_d, T g,
                                             T h_min, const FaceBar<T>& Fb, Bar3<T>& Lb, Bar3<T>& Rb) {
    const T z = Real<T>::zero();
    if (L.h < h_min && R.h < h_min) return;               // the face is skipped forward
    const T gL = XAXIS ? L.gx : L.gy;
    const T gR = XAXIS ? R.gx : R.gy;
    const T zL = L.b + half_d * gL;
    const T zR = R.b - half_d * gR;
    const T zf0 = (L.b > R.b) ? L.b : R.b;
    const T dz_clip = zR - zL;
    const T dz = R.b - L.b - dz_clip;
    const T eL = R.eta - L.eta, eR = L.eta - R.eta;
    const T mL = gmin(dz, eL), mR = gmin(-dz, eR);
    const T deta_L = gmax(z, mL);
    const T deta_R = gmax(z, mR);
    const T xL = (L.eta + deta_L) - zf0;
    const T xR = (R.eta + deta_R) - zf0;
    const T h_Lf = gmax(z, xL);
    const T h_Rf = gmax(z, xR);
    const T uNL = XAXIS ? L.u : L.v, uTL = XAXIS ? L.v : L.u;
    const T uNR = XAXIS ? R.u : R.v, uTR = XAXIS ? R.v : R.u;
    T hLf_b = z, uNL_b = z, uTL_b = z, hRf_b = z, uNR_b = z, uTR_b = z;
    hllc_bwd<T>(h_Lf, uNL, uTL, h_Rf, uNR, uTR, g, h_min, Fb.Fh * inv_d, Fb.Fn * inv_d, Fb.Ft * inv_d,
                hLf_b, uNL_b, uTL_b, hRf_b, uNR_b, uTR_b);
    T Leta_b = z, Reta_b = z, Lh_b = z, Rh_b = z;
    const T hg = (T)0.5 * g;
    {   // bed source of cell L
        const T y = zf0 - L.eta;
        T dzb;
        bool pass;
        if (R.h < h_min) { dzb = gmax(z, y); pass = y > z; }
        else { const T m = gmin(dz_clip, y); dzb = gmax(z, m); pass = (m > z) && !(dz_clip <= y); }
        const T P = h_Lf + L.h, Q = (zf0 - dzb) - L.b;
        const T sb = Fb.srcL * inv_d;
        const T P_b = sb * hg * Q, Q_b = sb * hg * P;
        hLf_b += P_b; Lh_b += P_b;
        if (pass) Leta_b += Q_b;                          // Q = zf0 - (zf0 - eta) - b
    }
    {   // bed source of cell R (its frame has -dz_clip)
        const T y = zf0 - R.eta;
        T dzb;
        bool pass;
        if (L.h < h_min) { dzb = gmax(z, y); pass = y > z; }
        else { const T m = gmin(-dz_clip, y); dzb = gmax(z, m); pass = (m > z) && !(-dz_clip <= y); }
        const T P = h_Rf + R.h, Q = (zf0 - dzb) - R.b;
        const T sb = Fb.srcR * inv_d;
        const T P_b = sb * hg * Q, Q_b = sb * hg * P;
        hRf_b += P_b; Rh_b += P_b;
        if (pass) Reta_b += Q_b;
    }
    if (xL > z) {
        Leta_b += hLf_b;
        if (mL > z && !(dz <= eL)) { Reta_b += hLf_b; Leta_b -= hLf_b; }
    }
    if (xR > z) {
        Reta_b += hRf_b;
        if (mR > z && !(-dz <= eR)) { Leta_b += hRf_b; Reta_b -= hRf_b; }
    }
    const T Lu_b = XAXIS ? uNL_b : uTL_b, Lv_b = XAXIS ? uTL_b : uNL_b;
    const T Ru_b = XAXIS ? uNR_b : uTR_b, Rv_b = XAXIS ? uTR_b : uNR_b;
    if (L.h > h_min) {
        const T r = (T)1.0 / L.h;
        Lb.hu += Lu_b * r; Lb.hv += Lv_b * r;
        Lh_b -= (Lu_b * L.u + Lv_b * L.v) * r;
    }
    if (R.h > h_min) {
        const T r = (T)1.0 / R.h;
        Rb.hu += Ru_b * r; Rb.hv += Rv_b * r;
        Rh_b -= (Ru_b * R.u + Rv_b * R.v) * r;
    }
    Lb.h += Lh_b + Leta_b;
    Rb.h += Rh_b + Reta_b;
}

// Face adjoints from the residual adjoints of its two cells (the reverse of
// accumulate(): an x-face adds -F to L's (h, hu, hv) and +F to R's, the bed source
// to the normal momentum; a y-face swaps the normal and transverse momentum).
template <typename T, bool XAXIS>
__device__ __forceinline__ FaceBar<T> face_bar(const Bar3<T>& rL, const Bar3<T>& rR) {
    FaceBar<T> f;
    f.Fh = rR.h - rL.h;
    if (XAXIS) { f.Fn = rR.hu - rL.hu; f.Ft = rR.hv - rL.hv; f.srcL = -rL.hu; f.srcR = rR.hu; }
    else       { f.Fn = rR.hv - rL.hv; f.Ft = rR.hu - rL.hu; f.srcL = -rL.hv; f.srcR = rR.hv; }
    return f;
}

// Reverse of wetdry_friction (friction on, the flat tier's Manning table). Inputs: the
// post-Euler state (h1, hu1, hv1) and the adjoints of the updated state; outputs the
// adjoints of (h1, hu1, hv1) and of the cell's Manning n.
template <typename T>
__device__ __forceinline__ void wetdry_friction_bwd(T h1, T hu1, T hv1, T n, T dt, T g, T h_min, T vcap,
                                                    bool quadratic, bool keep_h, bool ref_pow, const Bar3<T>& out_b,
                                                    Bar3<T>& in_b, T& n_b) {
    const T z = Real<T>::zero();
    n_b = z;
    if (h1 < h_min) {
        in_b.h = (keep_h && h1 > z) ? out_b.h : z;
        in_b.hu = z; in_b.hv = z;
        return;
    }
    const bool pass = h1 > h_min;
    const T hs = pass ? h1 : h_min;
    const T u = div_z(hu1, hs), v = div_z(hv1, hs);
    const T modU = sqrt_z(u * u + v * v);
    const T h43 = ref_pow ? pow_m43_ref(hs) : pow_m43(hs);   // the forward step's own value
    T ne = n, K = z, ncri = z;
    bool capped = false;
    if (modU > vcap) {
        K = ((T)1.0e-10 + dt) * g * h43 * (modU + (T)1.0e-30);
        ncri = gsqrt((T)1.0 / K);
        if (ncri > n) { ne = ncri; capped = true; }
    }
    const T Cf = g * ne * ne * h43;
    T alpha, Cf_b, modU_b;
    in_b.h = out_b.h;
    if (quadratic) {
        const T X = (T)2.0 * dt * Cf * modU;
        const T Sq = gsqrt((T)1.0 + (T)2.0 * X);
        alpha = (T)2.0 / (Sq + (T)1.0);
        const T alpha_b = out_b.hu * hu1 + out_b.hv * hv1;
        const T X_b = -(alpha_b * alpha * alpha * (T)0.5) / Sq;
        Cf_b = X_b * (T)2.0 * dt * modU;
        modU_b = X_b * (T)2.0 * dt * Cf;
    } else {
        alpha = (T)1.0 / ((T)1.0 + dt * Cf * modU);
        const T alpha_b = out_b.hu * hu1 + out_b.hv * hv1;
        const T D_b = -(alpha_b * alpha * alpha);
        Cf_b = D_b * dt * modU;
        modU_b = D_b * dt * Cf;
    }
    in_b.hu = out_b.hu * alpha;
    in_b.hv = out_b.hv * alpha;
    const T ne_b = Cf_b * (T)2.0 * g * ne * h43;
    T h43_b = Cf_b * g * ne * ne;
    if (capped) {
        const T K_b = ne_b * (-(T)0.5 * ncri / K);
        h43_b += K_b * ((T)1.0e-10 + dt) * g * (modU + (T)1.0e-30);
        modU_b += K_b * ((T)1.0e-10 + dt) * g * h43;
    } else {
        n_b = ne_b;
    }
    const T rhs = (T)1.0 / hs;
    T hs_b = h43_b * (-(T)4.0 / (T)3.0) * h43 * rhs;
    if (modU > z) {
        const T rU = modU_b / modU;
        const T u_b = rU * u, v_b = rU * v;
        in_b.hu += u_b * rhs;
        in_b.hv += v_b * rhs;
        hs_b -= (u_b * u + v_b * v) * rhs;
    }
    if (pass) in_b.h += hs_b;
}

}  // namespace gsw
