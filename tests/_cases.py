"""Small seeded cases shared by the tests (sizes the oracle finishes in seconds)."""
import numpy as np

from geoswe_b200.synthetic import fractal_bed


def rough_partly_dry(nx, ny, seed=7, dtype=np.float64):
    """The reference's SRM parity fixture shape: rough bed, a lake that leaves part dry,
    small random momentum on wet cells (tests/test_srm_cpu_matches_gpu.py:252-260)."""
    rng = np.random.default_rng(seed)
    bed = rng.random((nx, ny)) * 1.2
    q0 = np.zeros((3, nx, ny))
    q0[0] = np.maximum(0.8 - bed, 0.0)
    wet = q0[0] > 1e-6
    q0[1] = (rng.random((nx, ny)) - 0.5) * 0.04 * wet
    q0[2] = (rng.random((nx, ny)) - 0.5) * 0.04 * wet
    return q0.astype(dtype), bed.astype(dtype)


def flowing(nx, ny, seed=3, dtype=np.float32):
    """Fractal terrain with water at rest-plus-noise, some of it dry: exercises every
    HLLC branch, the dry-face skip and the SRM source clipping."""
    rng = np.random.default_rng(seed)
    bed = fractal_bed(nx, ny, 2.0, seed=seed, zmax=3.0)
    eta = 1.6 + 0.3 * rng.standard_normal((nx, ny))
    h = np.maximum(eta - bed, 0.0)
    h[rng.random((nx, ny)) < 0.05] = 0.0
    u = rng.standard_normal((nx, ny)) * 1.5
    v = rng.standard_normal((nx, ny)) * 1.5
    q0 = np.stack([h, h * u, h * v]).astype(dtype)
    return q0, bed.astype(dtype)


def pad_state(q0, bed, ngh, dtype):
    """Padded (3, nxp, nyp) state and edge-extended padded bed, as Solver2D builds them."""
    nx, ny = bed.shape
    qp = np.zeros((3, nx + 2 * ngh, ny + 2 * ngh), dtype=dtype)
    qp[:, ngh:ngh + nx, ngh:ngh + ny] = q0
    bp = np.zeros((nx + 2 * ngh, ny + 2 * ngh), dtype=dtype)
    bp[ngh:ngh + nx, ngh:ngh + ny] = bed
    bp[:ngh, :] = bp[ngh:ngh + 1, :]
    bp[-ngh:, :] = bp[-ngh - 1:-ngh, :]
    bp[:, :ngh] = bp[:, ngh:ngh + 1]
    bp[:, -ngh:] = bp[:, -ngh - 1:-ngh]
    return qp, bp


def same(a, b):
    """Equal as IEEE values (-0 == +0, NaN == NaN position-wise)."""
    a = np.asarray(a); b = np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
