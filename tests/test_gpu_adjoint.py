"""Discrete adjoint of the FP64 step (pg_adj_*): the restated passes against
the production kernels, and gradients against central finite differences of
the forward run with the same frozen dt schedule.  Needs a B200."""
import numpy as np
import pytest

from penguin_b200 import initial as I
from penguin_b200 import params as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def small_disk(**kw):
    """A 32x96 cut of the adjoint workload: log r in [0.5, 2], h/r 0.05, alpha 1e-3,
    q 5e-4 (full mass: no ramp), orbital advection, no damping."""
    base = dict(q=5.0e-4, alpha=1.0e-3, h=0.05, rmin=0.5, rmax=2.0, ramp_orbits=0.0)
    base.update(kw)
    return P.planet_disk(32, 96, **base).replace(kill_flag=0)


def sigma0_of(p, seed=7, noise=0.0):
    """The disk with a 1 % spiral on top.  A state that is axisymmetric down to
    rounding (no noise, no pattern) sits on the kinks of the PPM limiter and the
    flattening switch in every azimuthal pencil: the derivative there is that of
    rounding-level slopes, and finite differences of any useful step do not
    resolve it.  The spiral makes every pencil generic."""
    st = I.disk_state(p, seed=seed, noise=noise)
    x = I.cell_centres(p)
    y = (np.arange(p.yres) + 0.5) * 2 * np.pi / p.yres
    spiral = 1.0 + 0.01 * np.sin(y[:, None] + 3.0 * np.log(x[None, :]))
    return torch.tensor(st["r"] * spiral, dtype=torch.float64, device="cuda")


def smooth_direction(p, s0):
    x = I.cell_centres(p)
    y = (np.arange(p.yres) + 0.5) * 2 * np.pi / p.yres
    d = np.cos(2 * y[:, None] + 1.0) * np.sin(3 * x[None, :]) + 0.3
    return torch.tensor(d, dtype=torch.float64, device="cuda") * s0


def loss_of(sigma, target):
    return float(((sigma.mean(0) - target) ** 2).sum())


def make(p, nsteps, every=4):
    from penguin_b200.adjoint import DiskAdjoint

    return DiskAdjoint(p, nsteps=nsteps, checkpoint_every=every)


def test_restated_passes_match_production():
    p = small_disk()
    m = make(p, 1)
    err = m.model_error(sigma0_of(p, noise=1e-4))
    m.close()
    assert np.all(err < 1e-12), err


def test_production_passes_replay_exactly():
    """Each production pass re-run on its recorded input reproduces its recorded
    output bit for bit (the recording the adjoint linearises about)."""
    import ctypes

    from penguin_b200._lib import check, lib

    p = small_disk()
    m = make(p, 1)
    s0 = sigma0_of(p, noise=1e-4)
    check(lib().pg_adj_forward(m._h, ctypes.c_void_p(s0.data_ptr()), 0.0, 3, 0, None))
    out = np.zeros(5)
    check(lib().pg_adj_replay_diff(m._h, float(m.schedule()[-1]), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    m.close()
    assert np.all(out == 0.0), out


def test_tangent_matches_production_differences_per_pass():
    """The forward-mode tangent of every restated pass against central differences
    of the production kernel itself, along a smooth direction (relative L2).  The
    restated pass differenced the same way gives the same error: the restatement
    is the production function at the scale of the step.  The azimuthal sweep has
    isolated cells on the azimuthal pressure crest where the flattening
    coefficient (PPM.cu:38-55, the ratio dp1/dp2 with dp2 -> 0) changes on a
    1e-8 scale; there the difference quotient reaches the tangent only as
    eps -> 1e-10, so that pass is held to the restated-vs-production agreement."""
    p = small_disk()
    m = make(p, 1)
    r = m.pass_check(sigma0_of(p), steps_before=1, eps=1.0e-7)
    m.close()
    prod, rest = r[0], r[1]
    assert np.all(np.abs(prod - rest) <= 1e-3 * np.maximum(prod, rest) + 1e-6), (prod, rest)
    for k in (0, 1, 3, 4):  # kick1, sweep_x, advect, kick2
        assert np.all(prod[k] < 1e-4), (k, prod[k])


@pytest.mark.parametrize("visc", [1, 0], ids=["visc", "inviscid"])
def test_adjoint_dot_product_per_pass(visc):
    """<lam, J dir> by forward mode equals <J^T lam, dir> by the gather adjoint,
    pass by pass (kick1, sweep_x, sweep_y + shift, advect, kick2)."""
    p = small_disk().replace(visc_flag=visc)
    m = make(p, 1)
    r = m.dot_test(sigma0_of(p, noise=1e-4))
    m.close()
    for k, (fwd, adj) in enumerate(r):
        assert abs(fwd - adj) <= 1e-10 * max(abs(fwd), 1e-30), (k, fwd, adj)


def test_sigma0_gradient_matches_finite_differences():
    p = small_disk()
    n = 10
    m = make(p, n)
    s0 = sigma0_of(p)
    out = m.forward(s0)
    target = out.mean(0) * 1.01
    g = 2.0 * (out.mean(0) - target) / p.yres
    gs0, _ = m.backward(g[None, :].expand(p.yres, p.xres).contiguous())
    delta = smooth_direction(p, s0)
    ad = float((gs0 * delta).sum())
    # central differences with relative steps 1e-6 and 1e-7: the larger step
    # crosses a few limiter kinks in 10 steps (measured ~6e-6 relative)
    for eps, tol in ((1.0e-6, 1.0e-5), (1.0e-7, 1.0e-6)):
        lp = loss_of(m.forward(s0 + eps * delta, replay=True), target)
        lm = loss_of(m.forward(s0 - eps * delta, replay=True), target)
        fd = (lp - lm) / (2 * eps)
        assert abs(ad - fd) <= tol * abs(fd), (eps, ad, fd)
    m.close()


@pytest.mark.parametrize("k", [0, 1, 2], ids=["q", "alpha", "h"])
def test_theta_gradient_matches_finite_differences(k):
    p = small_disk()
    n = 10
    m = make(p, n)
    s0 = sigma0_of(p)
    theta = [p.planet_mass, p.ss_alpha, p.sc_h]
    out = m.forward(s0)
    target = out.mean(0) * 1.01
    g = 2.0 * (out.mean(0) - target) / p.yres
    _, gth = m.backward(g[None, :].expand(p.yres, p.xres).contiguous())
    # relative step 1e-4: central differences converge to the adjoint there (measured
    # 1e-8..1e-6 relative); at 1e-6 and below the rounding of the rebuilt tables,
    # amplified over 10 steps, dominates (6e-5 relative for h at 1e-6)
    step = 1.0e-4 * theta[k]
    vals = []
    for sgn in (1, -1):
        th = list(theta)
        th[k] += sgn * step
        m.set_theta(*th)
        vals.append(loss_of(m.forward(s0, replay=True), target))
    fd = (vals[0] - vals[1]) / (2 * step)
    m.close()
    assert abs(gth[k] - fd) <= 1e-5 * abs(fd) + 1e-14, (gth[k], fd)


def test_autograd_function_and_checkpoint_segments():
    """torch.autograd through evolve_sigma equals the direct backward, and the
    gradient does not depend on the checkpoint interval."""
    from penguin_b200.adjoint import evolve_sigma

    p = small_disk()
    n = 9
    s0 = sigma0_of(p).requires_grad_(True)
    theta = torch.tensor([p.planet_mass, p.ss_alpha, p.sc_h], dtype=torch.float64, requires_grad=True)
    grads = []
    for every in (2, 4, 64):
        m = make(p, n, every)
        sig = evolve_sigma(s0, theta, m)
        target = sig.detach().mean(0) * 0.99
        loss = ((sig.mean(0) - target) ** 2).sum()
        s0.grad, theta.grad = None, None
        loss.backward()
        grads.append((s0.grad.clone(), theta.grad.clone()))
        m.close()
    for gs, gt in grads[1:]:
        assert torch.allclose(gs, grads[0][0], rtol=1e-12, atol=0.0)
        assert torch.allclose(gt, grads[0][1], rtol=1e-12, atol=0.0)


@pytest.mark.parametrize("visc", [1, 0], ids=["visc", "inviscid"])
def test_hand_reverse_equals_dual_number_sweeps(visc):
    """The sweeps transposed by the hand-written reverse-mode kernels give the
    gradient of the dual-number kernels (the same derivative along the same
    branches) to rounding, for the initial field and for theta."""
    p = small_disk(alpha=1.0e-3 if visc else 1.0e-4).replace(visc_flag=visc)
    s0 = sigma0_of(p, noise=1e-4)
    out = []
    for hand in (False, True):
        m = make(p, 12, 4)
        m.set_sweep_reverse(hand)
        sig = m.forward(s0)
        target = sig.mean(0) * 1.01
        g = 2.0 * (sig.mean(0) - target)[None, :].expand_as(sig) / p.yres
        gs, gth = m.backward(g.contiguous())
        out.append((gs.clone(), np.array(gth)))
        m.close()
    (gd, td), (gh, th) = out
    rel = float((gh - gd).abs().max() / gd.abs().max())
    assert rel < 1e-11, rel
    np.testing.assert_allclose(th, td, rtol=1e-10, atol=0.0)


def test_adjoint_rejects_unsupported_disks():
    from penguin_b200._lib import PG_ERR_CONFIG, PGError
    from penguin_b200.adjoint import DiskAdjoint

    with pytest.raises(PGError) as e:
        DiskAdjoint.check_params(small_disk().replace(kill_flag=1))
    assert e.value.status == PG_ERR_CONFIG
    with pytest.raises(PGError):
        DiskAdjoint.check_params(P.sod_tube(64))
    with pytest.raises(PGError):
        DiskAdjoint.check_params(small_disk().replace(cool_flag=1))
    with pytest.raises(PGError):
        DiskAdjoint.check_params(small_disk().replace(twobd_flag=1))
