"""Seeded synthetic inputs of the benchmark cases (no external data is used).

* dam_break        -- circular dam on a flat bed (r = hypot(i-(n-1)/2, j-(n-1)/2)).
* fractal_bed      -- Gaussian random-phase spectrum with power ~ k^-3 (amplitude
                      k^-3/2, DC removed), real part rescaled to [0, zmax] m, plus a
                      planar slope along x.
* voronoi_classes  -- land-cover classes by nearest of `n_seeds` uniform seeds,
                      one class per seed drawn with rng.integers(n_classes).
* dilate_cross     -- binary dilation with the 4-neighbour cross, as
                      scipy.ndimage.binary_dilation's default structure.
* tidal_case       -- the everywhere-wet sinusoidal-bed case with a tidal stage.
"""
from __future__ import annotations

import numpy as np

MANNING_CLASSES = np.array([0.025, 0.04, 0.06, 0.1], dtype=np.float64)


def dam_break(n=512, radius=64.0, h_in=2.0, h_out=0.5, dtype=np.float64):
    i = np.arange(n, dtype=np.float64)[:, None]
    j = np.arange(n, dtype=np.float64)[None, :]
    r = np.hypot(i - (n - 1) / 2.0, j - (n - 1) / 2.0)
    q0 = np.zeros((3, n, n), dtype=dtype)
    q0[0] = np.where(r < radius, h_in, h_out)
    bed = np.zeros((n, n), dtype=dtype)
    return q0, bed


def fractal_bed(nx, ny, dx, seed=0, zmax=40.0, slope=0.002):
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(nx)[:, None]
    ky = np.fft.fftfreq(ny)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    amp = np.zeros_like(k)
    nz = k > 0
    amp[nz] = k[nz] ** -1.5
    noise = rng.standard_normal((nx, ny)) + 1j * rng.standard_normal((nx, ny))
    z = np.real(np.fft.ifft2(noise * amp))
    z = (z - z.min()) / (z.max() - z.min()) * zmax
    x = (np.arange(nx, dtype=np.float64) + 0.5) * dx
    return z + slope * x[:, None]


def voronoi_classes(nx, ny, n_seeds=256, n_classes=4, seed=0, chunk=1 << 20):
    rng = np.random.default_rng(seed + 7919)
    pts = rng.random((n_seeds, 2)) * np.array([nx, ny], dtype=np.float64)
    cls_of_seed = rng.integers(n_classes, size=n_seeds).astype(np.uint8)
    out = np.empty(nx * ny, dtype=np.uint8)
    ii, jj = np.divmod(np.arange(nx * ny, dtype=np.int64), ny)
    for s0 in range(0, nx * ny, chunk):
        ci = ii[s0:s0 + chunk, None] + 0.5
        cj = jj[s0:s0 + chunk, None] + 0.5
        d2 = (ci - pts[None, :, 0]) ** 2 + (cj - pts[None, :, 1]) ** 2
        out[s0:s0 + chunk] = cls_of_seed[np.argmin(d2, axis=1)]
    return out.reshape(nx, ny)


def voronoi_classes_fast(nx, ny, n_seeds=256, n_classes=4, seed=0):
    """Same classes as voronoi_classes, through a KD-tree (for large grids)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed + 7919)
    pts = rng.random((n_seeds, 2)) * np.array([nx, ny], dtype=np.float64)
    cls_of_seed = rng.integers(n_classes, size=n_seeds).astype(np.uint8)
    tree = cKDTree(pts)
    out = np.empty((nx, ny), dtype=np.uint8)
    jj = np.arange(ny, dtype=np.float64) + 0.5
    rows = max(1, (1 << 22) // ny)
    for i0 in range(0, nx, rows):
        i1 = min(nx, i0 + rows)
        ci = np.repeat(np.arange(i0, i1, dtype=np.float64) + 0.5, ny)
        cj = np.tile(jj, i1 - i0)
        _, idx = tree.query(np.stack([ci, cj], axis=1))
        out[i0:i1] = cls_of_seed[idx].reshape(i1 - i0, ny)
    return out


def voronoi_classes_window(nx, ny, i0, i1, j0, j1, n_seeds=256, n_classes=4, seed=0):
    """Classes of the cells [i0, i1) x [j0, j1) of voronoi_classes(nx, ny, ...): the same
    seeds and nearest-seed rule, evaluated on the window only (a crop of a large case
    without classifying the whole grid)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed + 7919)
    pts = rng.random((n_seeds, 2)) * np.array([nx, ny], dtype=np.float64)
    cls_of_seed = rng.integers(n_classes, size=n_seeds).astype(np.uint8)
    ci, cj = np.meshgrid(np.arange(i0, i1, dtype=np.float64) + 0.5, np.arange(j0, j1, dtype=np.float64) + 0.5,
                         indexing="ij")
    _, idx = cKDTree(pts).query(np.stack([ci.ravel(), cj.ravel()], axis=1))
    return cls_of_seed[idx].reshape(i1 - i0, j1 - j0)


def dilate_cross(mask, iterations):
    """scipy.ndimage.binary_dilation(mask, iterations=k) with the default cross."""
    m = np.asarray(mask, dtype=bool).copy()
    for _ in range(int(iterations)):
        d = m.copy()
        d[1:, :] |= m[:-1, :]
        d[:-1, :] |= m[1:, :]
        d[:, 1:] |= m[:, :-1]
        d[:, :-1] |= m[:, 1:]
        m = d
    return m


def rain_on_terrain(n=8192, dx=3.0, seed=0, pct=60.0, band=8):
    """Rain-on-terrain pluvial case: fractal bed, Voronoi Manning classes, dry start,
    active set z < pct-th percentile dilated `band` times."""
    z = fractal_bed(n, n, dx, seed=seed)
    cls = voronoi_classes_fast(n, n, seed=seed) if n * n > (1 << 22) else voronoi_classes(n, n, seed=seed)
    active = dilate_cross(z < np.percentile(z, pct), band)
    return z, cls, active


def tidal_case(nx, ny, dx=1.0, seed=0, eta0=1.5, noise=0.01, dtype=np.float32):
    """Everywhere-wet case: z = 0.5 sin(2 pi x / 2000) cos(2 pi y / 1500) at cell centres,
    eta = 1.5 + N(0, noise^2), zero velocity."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx, dtype=np.float64) + 0.5) * dx
    y = (np.arange(ny, dtype=np.float64) + 0.5) * dx
    z = 0.5 * np.sin(2 * np.pi * x / 2000.0)[:, None] * np.cos(2 * np.pi * y / 1500.0)[None, :]
    eta = eta0 + noise * rng.standard_normal((nx, ny))
    h = np.maximum(eta - z, 0.0)
    return h.astype(dtype), z.astype(dtype)


def fractal_bed_device(nx, ny, dx, seed=0, zmax=40.0, slope=0.002, device="cuda"):
    """fractal_bed with the same seeded noise, transformed on the GPU (float32 result)."""
    import torch
    rng = np.random.default_rng(seed)
    noise = torch.complex(torch.from_numpy(rng.standard_normal((nx, ny))),
                          torch.from_numpy(rng.standard_normal((nx, ny)))).to(device)
    kx = torch.fft.fftfreq(nx, device=device, dtype=torch.float64)[:, None]
    ky = torch.fft.fftfreq(ny, device=device, dtype=torch.float64)[None, :]
    k = torch.sqrt(kx * kx + ky * ky)
    amp = torch.where(k > 0, k.clamp_min(1e-300) ** -1.5, torch.zeros_like(k))
    z = torch.fft.ifft2(noise * amp).real
    z = (z - z.min()) / (z.max() - z.min()) * zmax
    x = (torch.arange(nx, device=device, dtype=torch.float64) + 0.5) * dx
    return (z + slope * x[:, None]).to(torch.float32)


def voronoi_classes_device(nx, ny, n_seeds=256, n_classes=4, seed=0, device="cuda"):
    """voronoi_classes (same seeds and classes), nearest seed found on the GPU."""
    import torch
    rng = np.random.default_rng(seed + 7919)
    pts = torch.from_numpy(rng.random((n_seeds, 2)) * np.array([nx, ny], dtype=np.float64)).to(device)
    cls_of_seed = torch.from_numpy(rng.integers(n_classes, size=n_seeds).astype(np.uint8)).to(device)
    out = torch.empty((nx, ny), dtype=torch.uint8, device=device)
    jj = torch.arange(ny, device=device, dtype=torch.float64) + 0.5
    rows = max(1, (1 << 22) // max(ny, 1))
    for i0 in range(0, nx, rows):
        i1 = min(nx, i0 + rows)
        ci = (torch.arange(i0, i1, device=device, dtype=torch.float64) + 0.5)[:, None].expand(i1 - i0, ny)
        cj = jj[None, :].expand(i1 - i0, ny)
        c = torch.stack([ci.reshape(-1), cj.reshape(-1)], dim=1)
        d = torch.cdist(c, pts)
        out[i0:i1] = cls_of_seed[d.argmin(dim=1)].reshape(i1 - i0, ny)
    return out


def triangular_hyetograph(peak_mm_h, t_peak_s, t_end_s=3600.0, every_s=60.0):
    """Piecewise-constant samples (every `every_s`, value at each interval's midpoint) of a
    triangle rising from 0 at t=0 to `peak_mm_h` at `t_peak_s` and back to 0 at 2 t_peak."""
    t = np.arange(0.0, t_end_s + every_s, every_s)
    mid = t + 0.5 * every_s
    r = np.where(mid <= t_peak_s, peak_mm_h * mid / t_peak_s,
                 np.maximum(peak_mm_h * (2.0 * t_peak_s - mid) / t_peak_s, 0.0))
    return t, r


def ensemble_specs(n_members=64, seed=0, side_min=256, side_max=4096):
    """Member parameters of the uneven-ensemble case: side ~ exp(U(ln 256, ln 4096)) per axis,
    active fraction ~ U(0.3, 0.9), triangular rain with peak ~ U(20, 120) mm/h at
    t_p ~ U(0.5, 3) h, Manning scale ~ U(0.7, 1.3)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_members):
        nx = int(round(np.exp(rng.uniform(np.log(side_min), np.log(side_max)))))
        ny = int(round(np.exp(rng.uniform(np.log(side_min), np.log(side_max)))))
        out.append(dict(seed=1000 + k, nx=nx, ny=ny, frac=float(rng.uniform(0.3, 0.9)),
                        peak=float(rng.uniform(20.0, 120.0)), t_peak=float(rng.uniform(0.5, 3.0)) * 3600.0,
                        scale=float(rng.uniform(0.7, 1.3))))
    return out


def calibration_case(n=2048, *, seed=0, dx=3.0, frac=0.7, pond=0.3, n_gauges=32, n_knots=16,
                     peak_q=20.0, t_peak=900.0, t_knots_end=3600.0, rain_mm_h=40.0, brick_h=16,
                     base_q=0.0, inlet_gauges=0, device="cuda"):
    """The Manning / rain / inflow calibration case on the compressed mesh: an n x n
    fractal bed (as rain_on_terrain), 4 Voronoi Manning classes, active set z < the
    `frac` quantile (three border rows/columns left out), a pond filling the lowest
    `pond` fraction of the bed to a flat surface at rest, uniform rain of `rain_mm_h`
    times the rain scale, and one point inlet (a single ghost/active pair on the mask
    edge whose ghost bed is not below its neighbour) with an `n_knots` hydrograph
    rising linearly to `peak_q` m^3/s at `t_peak` and falling back to 0 at 2 t_peak,
    never below `base_q`.
    Gauges: `n_gauges` seeded active cells, `inlet_gauges` of them the active cells
    nearest the inlet and the rest among the lower half of the active bed.
    Returns a dict of the CompressedSolver and the pieces FlatAdjoint takes."""
    from . import Config, Mesh2D, Solver2D
    from .adjoint import Inlet
    from .compressed import CompressedSolver
    z = fractal_bed(n, n, dx, seed=seed).astype(np.float32)
    cls = voronoi_classes_fast(n, n, seed=seed) if n * n > (1 << 20) else voronoi_classes(n, n, seed=seed)
    mask = z < np.quantile(z, frac)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    eta0 = np.float32(np.quantile(z, pond))
    h0 = np.where(mask, np.maximum(eta0 - z, 0.0), 0.0).astype(np.float32)
    q0 = np.stack([h0, np.zeros_like(h0), np.zeros_like(h0)])
    s = Solver2D(Mesh2D(nx=n, ny=n, dx=dx, dy=dx, ngh=2), Config(bc_x="fall", bc_y="fall", friction="manning"),
                 q0, z, device=device, track_max_depth=False)
    s.set_inside_mask(mask)
    s.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES)
    cs = CompressedSolver.from_dense(s, brick_h=brick_h)
    del s
    rng = np.random.default_rng(seed + 101)
    g, a = cs.ghost_boundary_pairs()
    ij = cs.ij_active
    b = cs._b[cs._slot].cpu().numpy()
    ok = np.nonzero(b[g] >= b[a])[0]
    k = int(ok[rng.integers(ok.size)])
    d = ij[a[k]] - ij[g[k]]
    inlet_t = np.linspace(0.0, t_knots_end, n_knots)
    inlet_q = np.maximum(base_q, peak_q * (1.0 - np.abs(inlet_t - t_peak) / t_peak))
    inlet = Inlet(ghost=g[k:k + 1], nbr=a[k:k + 1], normal=(float(d[0]), float(d[1])), ds=dx, t_knots=inlet_t)
    act = np.nonzero(cs.is_active != 0)[0]
    near = np.empty(0, np.int64)
    if inlet_gauges > 0:
        dist = np.abs(ij[act] - ij[a[k]]).max(axis=1)
        near = act[np.argsort(dist, kind="stable")[:inlet_gauges]]
    low = np.setdiff1d(act[b[act] <= np.quantile(b[act], 0.5)], near)
    rest = rng.choice(low, size=min(max(n_gauges - near.size, 0), low.size), replace=False)
    gauges = np.sort(np.concatenate([near, rest]))
    return dict(cs=cs, gauges=gauges, inlet=inlet, knots=inlet_q, rain_times=np.array([0.0]),
                rain_base=np.array([rain_mm_h / 3.6e6]), n_tab=MANNING_CLASSES.copy())
