/* gsw_oracle_body.h -- included twice by gsw_oracle.c with R = float / double.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU kernels are compared
 * against; nothing in the product links or calls it.
 *
 * Per-cell restatement of the reference's fused SRM-HLLC kernel text, four faces
 * per cell exactly as the reference evaluates them (geoswe/rhs_cuda.py:900-1207),
 * with the central bed gradients (rhs_cuda.py:1644-1651), Sigma = 0 (:1717-1722),
 * and the fused-step tail (rhs_cuda.py:1757-1796 = solver.py:355-419).
 * Every operation is separately rounded (-ffp-contract=off); operand order is the
 * reference's. h^(-4/3) uses the deterministic Newton form described in
 * gsw_oracle.c (the same one the kernels use).
 */

#define RZ ((R)0)

static inline R SFX(fmx)(R a, R b) { return FMAX(a, b); }
static inline R SFX(fmn)(R a, R b) { return FMIN(a, b); }

/* HLLC macro, rhs_cuda.py:986-1036 (no short-circuit: all states evaluated, then selected) */
static inline void SFX(hllc)(R hL, R uNL, R uTL, R sigL, R hR, R uNR, R uTR, R sigR,
                             R g, R h_min, R* Fh, R* FN, R* FT) {
    const R aL = SQRT(g * (hL > RZ ? hL : RZ));
    const R aR = SQRT(g * (hR > RZ ? hR : RZ));
    const R u_st = (R)0.5 * (uNL + uNR) + aL - aR;
    const R h_rt = (R)0.5 * (aL + aR) + (R)0.25 * (uNL - uNR);
    const R h_st = (h_rt > RZ) ? (h_rt * h_rt) / g : RZ;
    const R a_st = SQRT(g * (h_st > RZ ? h_st : RZ));
    const R SL_w = SFX(fmn)(uNL - aL, u_st - a_st);
    const R SR_w = SFX(fmx)(uNR + aR, u_st + a_st);
    const int dryL = (hL <= h_min);
    const int dryR = (hR <= h_min);
    R SL = dryL ? (uNR - (R)2.0 * aR) : SL_w;
    R SR = dryR ? (uNL + (R)2.0 * aL) : SR_w;
    if (dryL && dryR) { SL = RZ; SR = RZ; }
    const R denom = hR * (uNR - SR) - hL * (uNL - SL);
    R SM;
    if (FABS(denom) > (R)1.0e-14) SM = (SL * hR * (uNR - SR) - SR * hL * (uNL - SL)) / denom;
    else SM = (R)0.5 * (uNL + uNR);
    const R huNL = hL * uNL, huNR = hR * uNR;
    const R huTL = hL * uTL, huTR = hR * uTR;
    const R pL = (R)0.5 * g * hL * hL + sigL;
    const R pR = (R)0.5 * g * hR * hR + sigR;
    const R FL_h = huNL, FL_N = huNL * uNL + pL, FL_T = huNL * uTL;
    const R FR_h = huNR, FR_N = huNR * uNR + pR, FR_T = huNR * uTR;
    const R facL = (SL - uNL) / (SL - SM + (R)1.0e-30);
    const R facR = (SR - uNR) / (SR - SM + (R)1.0e-30);
    const R hLs = hL * facL, hRs = hR * facR;
    const R huNLs = hLs * SM, huNRs = hRs * SM;
    const R huTLs = hLs * uTL, huTRs = hRs * uTR;
    const R FLs_h = FL_h + SL * (hLs - hL);
    const R FLs_N = FL_N + SL * (huNLs - huNL);
    const R FLs_T = FL_T + SL * (huTLs - huTL);
    const R FRs_h = FR_h + SR * (hRs - hR);
    const R FRs_N = FR_N + SR * (huNRs - huNR);
    const R FRs_T = FR_T + SR * (huTRs - huTR);
    if (SL >= RZ)      { *Fh = FL_h;  *FN = FL_N;  *FT = FL_T; }
    else if (SM >= RZ) { *Fh = FLs_h; *FN = FLs_N; *FT = FLs_T; }
    else if (SR >= RZ) { *Fh = FRs_h; *FN = FRs_N; *FT = FRs_T; }
    else               { *Fh = FR_h;  *FN = FR_N;  *FT = FR_T; }
}

/* Residual of one cell from the indices of its 9-point stencil: centre, -i, +i, -2i,
 * +2i, -j, +j, -2j, +2j (dense: row arithmetic; flat: the neighbour table). */
static void SFX(cell_rhs_ix)(const R* q0, const R* q1, const R* q2, const R* b,
                             int64_t idx, int64_t idx_l, int64_t idx_r, int64_t idx_ll, int64_t idx_rr,
                             int64_t idx_b, int64_t idx_t, int64_t idx_bb, int64_t idx_tt,
                             R inv_dx, R inv_dy, R g, R h_min, R* r0, R* r1, R* r2) {
    const R dx = (R)1.0 / inv_dx;
    const R dy = (R)1.0 / inv_dy;
    R h_c, u_c, v_c, h_l, u_l, v_l, h_r, u_r, v_r, h_bo, u_bo, v_bo, h_to, u_to, v_to;
#define PRIMS(II, h, u, v) do { h = q0[II]; { const R _hs = (h > h_min) ? h : h_min; \
        u = (h > h_min) ? q1[II] / _hs : RZ; v = (h > h_min) ? q2[II] / _hs : RZ; } } while (0)
    PRIMS(idx, h_c, u_c, v_c);
    PRIMS(idx_l, h_l, u_l, v_l);
    PRIMS(idx_r, h_r, u_r, v_r);
    PRIMS(idx_b, h_bo, u_bo, v_bo);
    PRIMS(idx_t, h_to, u_to, v_to);
#undef PRIMS
    const R s_c = RZ, s_l = RZ, s_r = RZ, s_bo = RZ, s_to = RZ;
    const R b_c = b[idx], b_l = b[idx_l], b_r = b[idx_r], b_ll = b[idx_ll], b_rr = b[idx_rr];
    const R b_bo = b[idx_b], b_to = b[idx_t], b_bb = b[idx_bb], b_tt = b[idx_tt];
    const R gz_c_x = (R)0.5 * (b_r - b_l) * inv_dx;
    const R gz_l_x = (R)0.5 * (b_c - b_ll) * inv_dx;
    const R gz_r_x = (R)0.5 * (b_rr - b_c) * inv_dx;
    const R gz_c_y = (R)0.5 * (b_to - b_bo) * inv_dy;
    const R gz_bo_y = (R)0.5 * (b_c - b_bb) * inv_dy;
    const R gz_to_y = (R)0.5 * (b_tt - b_c) * inv_dy;
    const R eta_c = h_c + b_c, eta_l = h_l + b_l, eta_r = h_r + b_r;
    const R eta_bo = h_bo + b_bo, eta_to = h_to + b_to;
    R rhs_h = RZ, rhs_hu = RZ, rhs_hv = RZ;
    R Fh, FN, FT;
    /* X-face i+1/2 */
    if (!(h_c < h_min && h_r < h_min)) {
        const R _z_L = b_c + (R)0.5 * dx * gz_c_x;
        const R _z_R = b_r - (R)0.5 * dx * gz_r_x;
        const R z_f0 = (b_c > b_r) ? b_c : b_r;
        const R dz_clip = _z_R - _z_L;
        const R dz = b_r - b_c - dz_clip;
        const R deta_L = SFX(fmx)(RZ, SFX(fmn)(dz, eta_r - eta_c));
        const R deta_R = SFX(fmx)(RZ, SFX(fmn)(-dz, eta_c - eta_r));
        const R h_Lf = SFX(fmx)(RZ, eta_c + deta_L - z_f0);
        const R h_Rf = SFX(fmx)(RZ, eta_r + deta_R - z_f0);
        SFX(hllc)(h_Lf, u_c, v_c, s_c, h_Rf, u_r, v_r, s_r, g, h_min, &Fh, &FN, &FT);
        rhs_h -= Fh * inv_dx; rhs_hu -= FN * inv_dx; rhs_hv -= FT * inv_dx;
        R delta_z;
        if (h_r < h_min) delta_z = SFX(fmx)(RZ, z_f0 - eta_c);
        else delta_z = SFX(fmx)(RZ, SFX(fmn)(dz_clip, z_f0 - eta_c));
        const R z_f = z_f0 - delta_z;
        const R src = (R)0.5 * g * (h_Lf + h_c) * (z_f - b_c);
        rhs_hu -= src * inv_dx;
    }
    /* X-face i-1/2 */
    if (!(h_l < h_min && h_c < h_min)) {
        const R _z_L = b_l + (R)0.5 * dx * gz_l_x;
        const R _z_R = b_c - (R)0.5 * dx * gz_c_x;
        const R z_f0 = (b_l > b_c) ? b_l : b_c;
        const R dz_clip = _z_L - _z_R;
        const R dz = b_l - b_c - dz_clip;
        const R deta_this = SFX(fmx)(RZ, SFX(fmn)(dz, eta_l - eta_c));
        const R deta_neib = SFX(fmx)(RZ, SFX(fmn)(-dz, eta_c - eta_l));
        const R h_Rf = SFX(fmx)(RZ, eta_c + deta_this - z_f0);
        const R h_Lf = SFX(fmx)(RZ, eta_l + deta_neib - z_f0);
        SFX(hllc)(h_Lf, u_l, v_l, s_l, h_Rf, u_c, v_c, s_c, g, h_min, &Fh, &FN, &FT);
        rhs_h += Fh * inv_dx; rhs_hu += FN * inv_dx; rhs_hv += FT * inv_dx;
        R delta_z;
        if (h_l < h_min) delta_z = SFX(fmx)(RZ, z_f0 - eta_c);
        else delta_z = SFX(fmx)(RZ, SFX(fmn)(dz_clip, z_f0 - eta_c));
        const R z_f = z_f0 - delta_z;
        const R src = (R)0.5 * g * (h_Rf + h_c) * (z_f - b_c);
        rhs_hu += src * inv_dx;
    }
    /* Y-face j+1/2 */
    if (!(h_c < h_min && h_to < h_min)) {
        const R _z_L = b_c + (R)0.5 * dy * gz_c_y;
        const R _z_R = b_to - (R)0.5 * dy * gz_to_y;
        const R z_f0 = (b_c > b_to) ? b_c : b_to;
        const R dz_clip = _z_R - _z_L;
        const R dz = b_to - b_c - dz_clip;
        const R deta_L = SFX(fmx)(RZ, SFX(fmn)(dz, eta_to - eta_c));
        const R deta_R = SFX(fmx)(RZ, SFX(fmn)(-dz, eta_c - eta_to));
        const R h_Lf = SFX(fmx)(RZ, eta_c + deta_L - z_f0);
        const R h_Rf = SFX(fmx)(RZ, eta_to + deta_R - z_f0);
        SFX(hllc)(h_Lf, v_c, u_c, s_c, h_Rf, v_to, u_to, s_to, g, h_min, &Fh, &FN, &FT);
        rhs_h -= Fh * inv_dy; rhs_hu -= FT * inv_dy; rhs_hv -= FN * inv_dy;
        R delta_z;
        if (h_to < h_min) delta_z = SFX(fmx)(RZ, z_f0 - eta_c);
        else delta_z = SFX(fmx)(RZ, SFX(fmn)(dz_clip, z_f0 - eta_c));
        const R z_f = z_f0 - delta_z;
        const R src = (R)0.5 * g * (h_Lf + h_c) * (z_f - b_c);
        rhs_hv -= src * inv_dy;
    }
    /* Y-face j-1/2 */
    if (!(h_bo < h_min && h_c < h_min)) {
        const R _z_L = b_bo + (R)0.5 * dy * gz_bo_y;
        const R _z_R = b_c - (R)0.5 * dy * gz_c_y;
        const R z_f0 = (b_bo > b_c) ? b_bo : b_c;
        const R dz_clip = _z_L - _z_R;
        const R dz = b_bo - b_c - dz_clip;
        const R deta_this = SFX(fmx)(RZ, SFX(fmn)(dz, eta_bo - eta_c));
        const R deta_neib = SFX(fmx)(RZ, SFX(fmn)(-dz, eta_c - eta_bo));
        const R h_Rf = SFX(fmx)(RZ, eta_c + deta_this - z_f0);
        const R h_Lf = SFX(fmx)(RZ, eta_bo + deta_neib - z_f0);
        SFX(hllc)(h_Lf, v_bo, u_bo, s_bo, h_Rf, v_c, u_c, s_c, g, h_min, &Fh, &FN, &FT);
        rhs_h += Fh * inv_dy; rhs_hu += FT * inv_dy; rhs_hv += FN * inv_dy;
        R delta_z;
        if (h_bo < h_min) delta_z = SFX(fmx)(RZ, z_f0 - eta_c);
        else delta_z = SFX(fmx)(RZ, SFX(fmn)(dz_clip, z_f0 - eta_c));
        const R z_f = z_f0 - delta_z;
        const R src = (R)0.5 * g * (h_Rf + h_c) * (z_f - b_c);
        rhs_hv += src * inv_dy;
    }
    *r0 = rhs_h; *r1 = rhs_hu; *r2 = rhs_hv;
}

/* Residual of one cell (i, j) of a padded row-major field with row pitch P. */
static void SFX(cell_rhs)(const R* q0, const R* q1, const R* q2, const R* b, int64_t P,
                          int i, int j, R inv_dx, R inv_dy, R g, R h_min,
                          R* r0, R* r1, R* r2) {
    SFX(cell_rhs_ix)(q0, q1, q2, b, (int64_t)i * P + j, (int64_t)(i - 1) * P + j, (int64_t)(i + 1) * P + j,
                     (int64_t)(i - 2) * P + j, (int64_t)(i + 2) * P + j, (int64_t)i * P + (j - 1),
                     (int64_t)i * P + (j + 1), (int64_t)i * P + (j - 2), (int64_t)i * P + (j + 2),
                     inv_dx, inv_dy, g, h_min, r0, r1, r2);
}

/* Wet/dry + friction tail (rhs_cuda.py:1765-1790; friction off: solver.py:2952-2962). */
static inline void SFX(tail)(R* ph, R* phu, R* phv, int friction, R n, R dt, R g, R h_min,
                             R vcap, int quad, int keep_h) {
    R h = *ph, hu = *phu, hv = *phv;
    if (h < h_min) {
        h = keep_h ? (h > RZ ? h : RZ) : RZ; hu = RZ; hv = RZ;
    } else if (friction) {
        const R hs = (h > h_min) ? h : h_min;
        const R u = hu / hs, v = hv / hs;
        const R modU = SQRT(u * u + v * v);
        const R h43 = SFX(pow_m43)(hs);
        if (modU > vcap) {
            const R n_cri = SQRT((R)1.0 / (((R)1.0e-10 + dt) * g * h43 * (modU + (R)1.0e-30)));
            if (n_cri > n) n = n_cri;
        }
        const R Cf = g * n * n * h43;
        R alpha;
        if (quad) {
            const R twodtCfU = (R)2.0 * dt * Cf * modU;
            alpha = (R)2.0 / (SQRT((R)1.0 + (R)2.0 * twodtCfU) + (R)1.0);
        } else {
            alpha = (R)1.0 / ((R)1.0 + dt * Cf * modU);
        }
        hu = hu * alpha; hv = hv * alpha;
    }
    *ph = h; *phu = hu; *phv = hv;
}

/* Residual on cells [2, n-3]^2 (mask == 0 -> 0); everything else 0. */
void SFX(gswo_dense_rhs)(const R* q0, const R* q1, const R* q2, const R* b, int nxp, int nyp,
                         int64_t P, R inv_dx, R inv_dy, R g, R h_min, const uint8_t* mask,
                         R* r0, R* r1, R* r2) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nxp; ++i)
        for (int j = 0; j < nyp; ++j) {
            const int64_t o = (int64_t)i * P + j;
            r0[o] = RZ; r1[o] = RZ; r2[o] = RZ;
            if (i < 2 || i >= nxp - 2 || j < 2 || j >= nyp - 2) continue;
            if (mask && mask[o] == 0) continue;
            SFX(cell_rhs)(q0, q1, q2, b, P, i, j, inv_dx, inv_dy, g, h_min, &r0[o], &r1[o], &r2[o]);
        }
}

/* One fused step over the interior [ngh, n-ngh)^2; other cells of qn are copies of q.
 * rain_kind: 0 none, 1 uniform rate, 2 gridded interior frame.
 * friction_kind: 0 none, 1 table (cls pitch P), 2 field. Returns lambda of the new
 * state (dense semantics) as a double (cells with skip[k] != 0 excluded). */
double SFX(gswo_dense_step)(const R* q0, const R* q1, const R* q2, const R* b, int nxp, int nyp,
                            int ngh, int64_t P, R inv_dx, R inv_dy, R g, R h_min, R dt,
                            const uint8_t* mask, int rain_kind, const R* rain,
                            int friction_kind, const uint8_t* ncls, const R* ntab, const R* nfield,
                            R vcap, int quad, int keep_h, R* qn0, R* qn1, R* qn2, R* max_h,
                            const uint8_t* skip, R h_cfl) {
    const int nx = nxp - 2 * ngh, ny = nyp - 2 * ngh;
    double lam_all = 0.0;
#pragma omp parallel for schedule(static) reduction(max:lam_all)
    for (int i = 0; i < nxp; ++i)
        for (int j = 0; j < nyp; ++j) {
            const int64_t o = (int64_t)i * P + j;
            const int interior = (i >= ngh) && (i < nxp - ngh) && (j >= ngh) && (j < nyp - ngh);
            if (!interior) { qn0[o] = q0[o]; qn1[o] = q1[o]; qn2[o] = q2[o]; continue; }
            R r0 = RZ, r1 = RZ, r2 = RZ;
            const int inside = (mask == NULL) || mask[o] != 0;
            if (inside) SFX(cell_rhs)(q0, q1, q2, b, P, i, j, inv_dx, inv_dy, g, h_min, &r0, &r1, &r2);
            R rr0 = r0;
            if (inside && rain_kind == 1) rr0 = r0 + rain[0];
            else if (inside && rain_kind == 2) rr0 = r0 + rain[(int64_t)(i - ngh) * ny + (j - ngh)];
            R h = q0[o] + dt * rr0;
            R hu = q1[o] + dt * r1;
            R hv = q2[o] + dt * r2;
            R n = RZ;
            if (friction_kind == 1) n = ntab[ncls[o]];
            else if (friction_kind == 2) n = nfield[o];
            SFX(tail)(&h, &hu, &hv, friction_kind != 0, n, dt, g, h_min, vcap, quad, keep_h);
            qn0[o] = h; qn1[o] = hu; qn2[o] = hv;
            if (max_h && h > max_h[o]) max_h[o] = h;
            if (!(skip && skip[(int64_t)(i - ngh) * ny + (j - ngh)])) {
                const double l = SFX(lam_dense)(h, hu, hv, g, h_cfl);   /* never NaN */
                if (l > lam_all) lam_all = l;
            }
        }
    (void)nx;
    return lam_all;
}

double SFX(gswo_dense_lammax)(const R* q0, const R* q1, const R* q2, int nxp, int nyp, int ngh,
                              int64_t P, R g, R h_cfl, const uint8_t* skip) {
    const int ny = nyp - 2 * ngh;
    double lam_all = 0.0;
    for (int i = ngh; i < nxp - ngh; ++i)
        for (int j = ngh; j < nyp - ngh; ++j) {
            if (skip && skip[(int64_t)(i - ngh) * ny + (j - ngh)]) continue;
            const int64_t o = (int64_t)i * P + j;
            const double l = SFX(lam_dense)(q0[o], q1[o], q2[o], g, h_cfl);
            if (l > lam_all) lam_all = l;
        }
    return lam_all;
}

/* Ghost fill (bc.py:50-98 / 101-172), all ghost cells including corners, x faces
 * first then y faces, as apply_bc_2d does. kinds: x-, x+, y-, y+. */
void SFX(gswo_bc)(R* q0, R* q1, R* q2, int nxp, int nyp, int ngh, int64_t P, const int* kinds) {
    R* q[3] = {q0, q1, q2};
    for (int side = 0; side < 2; ++side) {
        const int kind = kinds[side];
        if (kind == 4) continue;
        for (int k = 0; k < ngh; ++k) {
            const int gi = side == 0 ? k : nxp - ngh + k;
            int si;
            if (kind == 1) si = side == 0 ? 2 * ngh - 1 - k : nxp - ngh - 1 - k;
            else if (kind == 3) si = side == 0 ? nxp - 2 * ngh + k : ngh + k;
            else si = side == 0 ? ngh : nxp - ngh - 1;
            for (int j = 0; j < nyp; ++j)
                for (int c = 0; c < 3; ++c) {
                    R v = kind == 2 ? RZ : q[c][(int64_t)si * P + j];
                    if (kind == 1 && c == 1) v = -v;
                    q[c][(int64_t)gi * P + j] = v;
                }
        }
    }
    for (int side = 0; side < 2; ++side) {
        const int kind = kinds[2 + side];
        if (kind == 4) continue;
        for (int k = 0; k < ngh; ++k) {
            const int gj = side == 0 ? k : nyp - ngh + k;
            int sj;
            if (kind == 1) sj = side == 0 ? 2 * ngh - 1 - k : nyp - ngh - 1 - k;
            else if (kind == 3) sj = side == 0 ? nyp - 2 * ngh + k : ngh + k;
            else sj = side == 0 ? ngh : nyp - ngh - 1;
            for (int i = 0; i < nxp; ++i)
                for (int c = 0; c < 3; ++c) {
                    R v = kind == 2 ? RZ : q[c][(int64_t)i * P + sj];
                    if (kind == 1 && c == 2) v = -v;
                    q[c][(int64_t)i * P + gj] = v;
                }
        }
    }
}

#undef RZ
