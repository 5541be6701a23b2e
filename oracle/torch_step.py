"""Plain-PyTorch fp64 restatement of one compressed-mesh step (test infrastructure).

This is the checker of the hand-written adjoint (geoswe_b200/csrc/gsw_adjoint.cu): the
same step as the flat tier's fused kernel (the reference's flat step,
geoswe/compressed_rhs.py:673-865 with the kernel text of geoswe/rhs_cuda.py:900-1207
and :1757-1796; the inlet block of geoswe/compressed_solver.py:2144-2167), written with
differentiable torch operations on the reference's canonical flat arrays (int16
E/W/N/S neighbour deltas, missing -> self), so torch.autograd gives the exact gradient
of the discrete map. Branches are torch.where selections with the conventions the
adjoint uses (max(0, x) passes where x > 0; fmin picks its first argument on ties,
fmax likewise); the operands of non-selected branches are made finite so their
zero gradients stay zero. Only the tests import this module.
"""
from __future__ import annotations

import numpy as np
import torch


def _w(c, a, b):
    return torch.where(c, a, b)


def _sqrt_pos(x):
    """sqrt(x) where x > 0, else 0, with a finite gradient everywhere."""
    pos = x > 0
    return _w(pos, torch.sqrt(_w(pos, x, torch.ones_like(x))), torch.zeros_like(x))


def hllc(hL, uNL, uTL, hR, uNR, uTR, g, h_min):
    z = torch.zeros_like(hL)
    aL = _sqrt_pos(g * _w(hL > 0, hL, z))
    aR = _sqrt_pos(g * _w(hR > 0, hR, z))
    u_st = 0.5 * (uNL + uNR) + aL - aR
    h_rt = 0.5 * (aL + aR) + 0.25 * (uNL - uNR)
    h_st = _w(h_rt > 0, (h_rt * h_rt) / g, z)
    a_st = _sqrt_pos(g * _w(h_st > 0, h_st, z))
    A1, A2 = uNL - aL, u_st - a_st
    B1, B2 = uNR + aR, u_st + a_st
    dryL, dryR = hL <= h_min, hR <= h_min
    SL = _w(dryL, uNR - 2.0 * aR, _w(A1 <= A2, A1, A2))
    SR = _w(dryR, uNL + 2.0 * aL, _w(B1 >= B2, B1, B2))
    both = dryL & dryR
    SL = _w(both, z, SL)
    SR = _w(both, z, SR)
    dR, dL = uNR - SR, uNL - SL
    denom = hR * dR - hL * dL
    big = denom.abs() > 1e-14
    SM = _w(big, (SL * hR * dR - SR * hL * dL) / _w(big, denom, torch.ones_like(denom)), 0.5 * (uNL + uNR))
    huNL, huNR = hL * uNL, hR * uNR
    huTL, huTR = hL * uTL, hR * uTR
    FL = (huNL, huNL * uNL + 0.5 * g * hL * hL, huNL * uTL)
    FR = (huNR, huNR * uNR + 0.5 * g * hR * hR, huNR * uTR)
    left = SM >= 0
    star = (~(SL >= 0)) & (left | (SR >= 0))
    S = _w(left, SL, SR)
    hK, uNK, uTK = _w(left, hL, hR), _w(left, uNL, uNR), _w(left, uTL, uTR)
    huNK, huTK = _w(left, huNL, huNR), _w(left, huTL, huTR)
    FK = [_w(left, a, b) for a, b in zip(FL, FR)]
    D = _w(star, S - SM + 1e-30, torch.ones_like(S))
    fac = (S - uNK) / D
    hKs = hK * fac
    Fs = (FK[0] + S * (hKs - hK), FK[1] + S * (hKs * SM - huNK), FK[2] + S * (hKs * uTK - huTK))
    r0 = SL >= 0
    return [_w(r0, a, _w(star, b, c)) for a, b, c in zip(FL, Fs, FR)]


class TorchFlat:
    """The flat step on canonical arrays. nbr (N, 4) int16 deltas E, W, N, S (i+, i-,
    j+, j-), act (N,) uint8, b (N,), ncls (N,) class ids; scalars as the solver's."""

    def __init__(self, nbr, act, b, ncls, dx, *, g=9.81, h_min=1e-6, vcap=15.0, quad=True, keep_h=True):
        nbr = np.asarray(nbr, np.int64)
        N = nbr.shape[0]
        k = np.arange(N)
        idx = []
        for d in range(4):
            dl = nbr[:, d]
            c = k + dl
            ok = (dl > -32768) & (c >= 0) & (c < N)
            idx.append(torch.from_numpy(np.where(ok, c, k)))
        self.E, self.W, self.Nn, self.S = idx
        self.A = torch.from_numpy(np.nonzero(np.asarray(act) != 0)[0])
        self.b = torch.as_tensor(np.asarray(b, np.float64))
        self.ncls = torch.as_tensor(np.asarray(ncls, np.int64))
        self.inv = 1.0 / dx
        self.half = 0.5 * (1.0 / self.inv)
        self.g, self.h_min, self.vcap, self.quad, self.keep_h = g, h_min, vcap, quad, keep_h
        b = self.b
        self.gx = 0.5 * (b[self.E] - b[self.W]) * self.inv
        self.gy = 0.5 * (b[self.Nn] - b[self.S]) * self.inv

    def _face(self, q, u, v, eta, Li, Ri, xaxis):
        h, g, h_min, inv, half, b = q[0], self.g, self.h_min, self.inv, self.half, self.b
        hL, hR = h[Li], h[Ri]
        gL = (self.gx if xaxis else self.gy)[Li]
        gR = (self.gx if xaxis else self.gy)[Ri]
        bL, bR = b[Li], b[Ri]
        eL_, eR_ = eta[Li], eta[Ri]
        zL = bL + half * gL
        zR = bR - half * gR
        zf0 = torch.maximum(bL, bR)
        dz_clip = zR - zL
        dz = bR - bL - dz_clip
        z = torch.zeros_like(hL)
        eL, eR = eR_ - eL_, eL_ - eR_
        mL = _w(dz <= eL, dz, eL)
        mR = _w(-dz <= eR, -dz, eR)
        xL = (eL_ + _w(mL > 0, mL, z)) - zf0
        xR = (eR_ + _w(mR > 0, mR, z)) - zf0
        hLf, hRf = _w(xL > 0, xL, z), _w(xR > 0, xR, z)
        if xaxis:
            F = hllc(hLf, u[Li], v[Li], hRf, u[Ri], v[Ri], g, h_min)
        else:
            F = hllc(hLf, v[Li], u[Li], hRf, v[Ri], u[Ri], g, h_min)
        yL = zf0 - eL_
        mLs = _w(dz_clip <= yL, dz_clip, yL)
        dzbL = _w(hR < h_min, _w(yL > 0, yL, z), _w(mLs > 0, mLs, z))
        srcL = 0.5 * g * (hLf + hL) * ((zf0 - dzbL) - bL) * inv
        yR = zf0 - eR_
        mRs = _w(-dz_clip <= yR, -dz_clip, yR)
        dzbR = _w(hL < h_min, _w(yR > 0, yR, z), _w(mRs > 0, mRs, z))
        srcR = 0.5 * g * (hRf + hR) * ((zf0 - dzbR) - bR) * inv
        wet = ~((hL < h_min) & (hR < h_min))
        return [_w(wet, f * inv, z) for f in F] + [_w(wet, srcL, z), _w(wet, srcR, z)]

    def step(self, q, ntab, rate, dt):
        """q (3, N) -> the state after one step (active cells updated, ring carried)."""
        h, hu, hv = q[0], q[1], q[2]
        h_min, g = self.h_min, self.g
        wet = h > h_min
        hs = _w(wet, h, torch.ones_like(h))
        u = _w(wet, hu / hs, torch.zeros_like(h))
        v = _w(wet, hv / hs, torch.zeros_like(h))
        eta = h + self.b
        A = self.A
        Fe = self._face(q, u, v, eta, A, self.E[A], True)
        Fw = self._face(q, u, v, eta, self.W[A], A, True)
        Fn = self._face(q, u, v, eta, A, self.Nn[A], False)
        Fs = self._face(q, u, v, eta, self.S[A], A, False)
        rh = -Fe[0] + Fw[0] - Fn[0] + Fs[0]
        rhu = -Fe[1] + Fw[1] - Fn[2] + Fs[2] - Fe[3] + Fw[4]
        rhv = -Fe[2] + Fw[2] - Fn[1] + Fs[1] - Fn[3] + Fs[4]
        h1 = h[A] + dt * (rh + rate)
        hu1 = hu[A] + dt * rhu
        hv1 = hv[A] + dt * rhv
        n = ntab[self.ncls[A]]
        h2, hu2, hv2 = self._tail(h1, hu1, hv1, n, dt)
        out = q.clone()
        out[0, A] = h2
        out[1, A] = hu2
        out[2, A] = hv2
        return out

    def _tail(self, h1, hu1, hv1, n, dt):
        h_min, g = self.h_min, self.g
        z = torch.zeros_like(h1)
        dry = h1 < h_min
        pas = h1 > h_min
        hs = _w(pas, h1, torch.full_like(h1, h_min))
        u, v = hu1 / hs, hv1 / hs
        modU = _sqrt_pos(u * u + v * v)
        h43 = hs ** (-4.0 / 3.0)
        over = modU > self.vcap
        K = _w(over, (1e-10 + dt) * g * h43 * (modU + 1e-30), torch.ones_like(h1))
        ncri = torch.sqrt(1.0 / K)
        capped = over & (ncri > n)
        ne = _w(capped, ncri, n)
        Cf = g * ne * ne * h43
        if self.quad:
            alpha = 2.0 / (torch.sqrt(1.0 + 2.0 * (2.0 * dt * Cf * modU)) + 1.0)
        else:
            alpha = 1.0 / (1.0 + dt * Cf * modU)
        h_dry = _w(h1 > 0, h1, z) if self.keep_h else z
        return _w(dry, h_dry, h1), _w(dry, z, hu1 * alpha), _w(dry, z, hv1 * alpha)


def interp_row(t, xp):
    """Weights w with np.interp(t, xp, fp) == w @ fp."""
    xp = np.asarray(xp, np.float64)
    w = np.zeros(xp.size)
    if xp.size == 1 or t <= xp[0]:
        w[0] = 1.0
    elif t >= xp[-1]:
        w[-1] = 1.0
    else:
        j = int(np.searchsorted(xp, t, "right") - 1)
        a = (t - xp[j]) / (xp[j + 1] - xp[j])
        w[j], w[j + 1] = 1.0 - a, a
    return torch.from_numpy(w)


def inflow(q, b, ghost, nbr, normal, ds, t, t_knots, knots):
    """The flat loop's inlet block (compressed_solver.py:2144-2167) in torch."""
    ghost = torch.as_tensor(ghost)
    nbr = torch.as_tensor(nbr)
    Q = interp_row(t, t_knots) @ knots
    h_a = q[0, nbr]
    ssum = h_a.sum()
    if float(ssum.detach()) > 0.0:
        w = h_a / ssum
        h_face = h_a
    else:
        zb = b[nbr]
        zmin, zmax = float(zb.min()), float(zb.max())
        h_face = torch.clamp(zmin + 0.10 * (zmax - zmin) - zb, min=0.0)
        low = zb <= zmin
        nlow = float(low.sum()) or 1.0
        if float(h_face.max()) <= 0.0:
            qc = Q.abs() / (nlow * ds)
            pos = qc > 0
            qs = _w(pos, qc, torch.ones_like(qc))
            h_face = h_face + _w(pos, (qs * qs / 9.80665) ** (1.0 / 3.0), torch.zeros_like(qc))
        w = _w(low, torch.full_like(zb, 1.0 / nlow), torch.zeros_like(zb))
    qn = (Q / ds) * w
    out = q.clone()
    out[0, ghost] = h_face
    out[1, ghost] = qn * float(normal[0])
    out[2, ghost] = qn * float(normal[1])
    return out


def rollout_loss(tf: TorchFlat, q0, ntab, rain_scale, knots, *, dt_tab, t_tab, rain_t, rain_base,
                 gauges, window, target, inlet=None):
    """Loss of `len(dt_tab)` steps with the given dt schedule (the adjoint's frozen dt):
    sum over the last `window` states of (depth at gauges - target)^2."""
    N = len(dt_tab)
    q = q0
    gauges = torch.as_tensor(gauges)
    loss = torch.zeros((), dtype=torch.float64)
    first = N - window + 1
    for n in range(N):
        t = float(t_tab[n])
        if inlet is not None:
            q = inflow(q, tf.b, inlet["ghost"], inlet["nbr"], inlet["normal"], inlet["ds"], t,
                       inlet["t_knots"], knots)
        i = int(np.clip(np.searchsorted(rain_t, t, "right") - 1, 0, len(rain_t) - 1))
        rate = rain_scale * float(rain_base[i])
        q = tf.step(q, ntab, rate, float(dt_tab[n]))
        if n + 1 >= first:
            d = q[0, gauges] - torch.as_tensor(target[n + 1 - first], dtype=torch.float64)
            loss = loss + (d * d).sum()
    return loss
