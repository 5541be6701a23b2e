"""The hand-written adjoint of the compressed-mesh step on the GPU, in float64, against
torch.autograd through the plain-PyTorch restatement of the same step
(oracle/torch_step.py) and against central finite differences of the GPU forward with
the recorded dt schedule replayed (dt frozen, as the adjoint holds it). The loss is a
squared gauge misfit against a run with perturbed parameters (Manning n x 1.2, rain
x 0.9); parameters: the 4 class n values, the rain scale, the inlet's hydrograph knots.
The hydrograph keeps a base flow: at Q = 0 a dry inlet's critical depth, |Q|^(2/3), has
a cusp where no derivative exists (the adjoint and autograd both take 0 there)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from oracle import torch_step  # noqa: E402


def _problem(n, N, window, n_gauges, seed=3, snapshots=6):
    from geoswe_b200.adjoint import FlatAdjoint
    from geoswe_b200.synthetic import calibration_case
    case = calibration_case(n, seed=seed, n_gauges=n_gauges, t_peak=4.0, t_knots_end=16.0, rain_mm_h=80.0,
                           base_q=1.0)
    cs = case["cs"]
    case["gauges"] = np.union1d(case["gauges"], case["inlet"].nbr)   # a gauge the inlet reaches
    prob = FlatAdjoint(cs, gauges=case["gauges"], n_steps=N, window=window, snapshots=snapshots,
                       dtype="float64", rain_times=case["rain_times"], rain_base=case["rain_base"],
                       inlet=case["inlet"])
    return case, prob


def _target(case, prob):
    prob.set_params(case["n_tab"] * 1.2, 0.9, case["knots"])
    return prob.forward().cpu().numpy()


def _torch_setup(case, prob):
    cs = case["cs"]
    slot = cs._slot
    tf = torch_step.TorchFlat(cs.nbr, cs.is_active, cs._b[slot].cpu().numpy().astype(np.float64),
                              cs._ncls[slot].cpu().numpy(), cs.dx, g=cs.g, h_min=cs.h_min, vcap=cs.vcap,
                              quad=cs.quad, keep_h=cs.keep_h)
    q0 = torch.stack([prob.q_init[c][slot].cpu() for c in range(3)]).double()
    inl = case["inlet"]
    inlet = dict(ghost=inl.ghost, nbr=inl.nbr, normal=inl.normal, ds=inl.ds, t_knots=inl.t_knots)
    return tf, q0, inlet


def _torch_grads(case, prob, target, wrt_state=False):
    tf, q0, inlet = _torch_setup(case, prob)
    ntab = torch.tensor(case["n_tab"], dtype=torch.float64, requires_grad=True)
    s = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    knots = torch.tensor(case["knots"], dtype=torch.float64, requires_grad=True)
    q0 = q0.clone().requires_grad_(wrt_state)
    dt = prob.dt_tab.cpu().numpy()[: prob.N]
    loss = torch_step.rollout_loss(tf, q0, ntab, s, knots, dt_tab=dt, t_tab=prob._t_tab, rain_t=prob.rain_t,
                                   rain_base=prob.rain_base, gauges=case["gauges"], window=prob.K,
                                   target=target, inlet=inlet)
    loss.backward()
    return float(loss.detach()), ntab.grad.numpy(), float(s.grad), knots.grad.numpy(), (q0.grad if wrt_state else None)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_one_step_vjp_matches_autograd():
    """One step (window 1): the parameter gradients and the adjoint of the whole initial
    state against torch.autograd."""
    case, prob = _problem(48, 1, 1, 12)
    target = _target(case, prob)
    prob.set_params(case["n_tab"], 1.0, case["knots"])
    prob.forward()
    L = prob.loss(target)
    gn, gs, gk = prob.gradients(target)
    lt, tn, ts, tk, tq = _torch_grads(case, prob, target, wrt_state=True)
    assert abs(L - lt) <= 1e-12 * max(abs(lt), 1e-300)
    assert _rel(gn.cpu().numpy(), tn) < 1e-9
    assert abs(gs - ts) <= 1e-9 * max(abs(ts), 1e-300)
    assert _rel(gk.numpy(), tk) < 1e-9
    slot = case["cs"]._slot
    lam0 = torch.stack([prob.adjoint_state(c)[slot].cpu() for c in range(3)]).numpy()
    assert np.abs(tq.numpy()).max() > 0
    assert _rel(lam0, tq.numpy()) < 1e-9


def test_rollout_gradients_autograd_and_finite_differences():
    """128 x 128 crop, 60 steps with binomial checkpointing (6 snapshots): gradients
    against autograd (1e-8) and against fp64 central differences (1e-3, the stated
    bar) for every parameter with a non-negligible gradient."""
    case, prob = _problem(128, 60, 30, 16)
    target = _target(case, prob)
    base_n, base_k = case["n_tab"].copy(), case["knots"].copy()
    prob.set_params(base_n, 1.0, base_k)
    prob.forward()
    L0 = prob.loss(target)
    gn, gs, gk = prob.gradients(target)
    gn, gk = gn.cpu().numpy(), gk.numpy()
    assert prob.recompute_steps > 0 and prob.max_snapshots <= 6
    lt, tn, ts, tk, _ = _torch_grads(case, prob, target)
    assert abs(L0 - lt) <= 1e-10 * abs(lt)
    assert _rel(gn, tn) < 1e-8
    assert abs(gs - ts) <= 1e-8 * abs(ts)
    assert _rel(gk, tk) < 1e-8

    def loss_at(n_tab, s, knots):
        prob.set_params(n_tab, s, knots)
        prob.forward(replay=True, snapshots=False)
        return prob.loss(target)

    fd = []
    for c in range(4):
        e = 1e-5 * base_n[c]
        up, dn = base_n.copy(), base_n.copy()
        up[c] += e
        dn[c] -= e
        fd.append(("n", c, gn[c], (loss_at(up, 1.0, base_k) - loss_at(dn, 1.0, base_k)) / (2 * e)))
    fd.append(("s", 0, gs, (loss_at(base_n, 1.0 + 1e-5, base_k) - loss_at(base_n, 1.0 - 1e-5, base_k)) / 2e-5))
    for j in range(len(base_k)):
        e = 1e-4
        up, dn = base_k.copy(), base_k.copy()
        up[j] += e
        dn[j] -= e
        fd.append(("k", j, gk[j], (loss_at(base_n, 1.0, up) - loss_at(base_n, 1.0, dn)) / (2 * e)))
    scale = max(abs(x[2]) for x in fd)
    checked = 0
    for name, j, g_adj, g_fd in fd:
        if abs(g_fd) > 1e-6 * scale:
            assert abs(g_adj - g_fd) <= 1e-3 * abs(g_fd), (name, j, g_adj, g_fd)
            checked += 1
        else:
            assert abs(g_adj) <= 1e-5 * scale, (name, j, g_adj, g_fd)
    print(f"\nfinite-difference checks: {checked} of {len(fd)} parameters (others below 1e-6 of the largest)")
    assert checked >= 8
