"""Gradients of the FP64 step through its discrete adjoint (pg_adj_* C ABI).

The differentiated map takes the initial surface density field Sigma0 and the
disk parameters theta = (q, alpha, h/r) to the surface density after N steps
of main.cu's loop (v_r = 0 and v_phi = the disk's init_C at the start; dt is
the CFL schedule of the first, recorded forward run and stays frozen).  The
backward pass recomputes each segment between checkpoints forward and runs
the adjoint of every pass in reverse order on the GPU.

``DiskAdjoint`` owns one disk; ``evolve_sigma`` is the torch.autograd entry:

    model = DiskAdjoint(params, nsteps=2000)
    sigma = evolve_sigma(sigma0, theta, model)      # theta = tensor([q, alpha, h])
    loss = ((sigma.mean(0) - target) ** 2).sum()
    loss.backward()                                 # sigma0.grad, theta.grad
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .params import Params, PGParams


class DiskAdjoint:
    def __init__(self, params: Params, nsteps: int, t0: float = 0.0, checkpoint_every: int = 64, device: int = 0,
                 stream: int | None = None):
        self.params = params
        self.nsteps, self.t0 = int(nsteps), float(t0)
        self.device = device
        self._P = PGParams.from_params(params)
        h = ctypes.c_void_p()
        check(lib().pg_adj_create(ctypes.byref(self._P), device, ctypes.c_void_p(stream or 0), checkpoint_every,
                                  ctypes.byref(h)))
        self._h = h
        self.theta = (params.planet_mass, params.ss_alpha, params.sc_h)
        self.recorded = False

    @staticmethod
    def check_params(params: Params) -> None:
        P = PGParams.from_params(params)
        check(lib().pg_adj_check_params(ctypes.byref(P)))

    def set_theta(self, q: float, alpha: float, h: float) -> None:
        if (q, alpha, h) != self.theta:
            check(lib().pg_adj_set_params(self._h, q, alpha, h))
            self.theta = (q, alpha, h)

    def forward(self, sigma0, replay: bool | None = None):
        """sigma0: CUDA float64 tensor (yres, xres).  Returns Sigma after nsteps."""
        import torch

        s0 = sigma0.detach().to(torch.float64).contiguous()
        out = torch.empty_like(s0)
        rep = self.recorded if replay is None else replay
        check(lib().pg_adj_forward(self._h, ctypes.c_void_p(s0.data_ptr()), self.t0, self.nsteps, int(rep),
                                   ctypes.c_void_p(out.data_ptr())))
        self.recorded = True
        return out

    def backward(self, grad_sigma):
        """dL/dSigma (CUDA float64 tensor) -> (dL/dSigma0 tensor, dL/dtheta numpy[3])."""
        import torch

        g = grad_sigma.detach().to(torch.float64).contiguous()
        gs0 = torch.empty_like(g)
        gth = np.zeros(3)
        check(lib().pg_adj_backward(self._h, ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(gs0.data_ptr()),
                                    gth.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return gs0, gth

    def model_error(self, sigma0, dt: float | None = None) -> np.ndarray:
        """Runs one step from sigma0, then compares the adjoint's restatement of each
        pass (kick1, sweep_x, sweep_y, advect, kick2) with the production kernels
        over the next step of size dt (default: the first step's)."""
        import torch

        s0 = sigma0.detach().to(torch.float64).contiguous()
        check(lib().pg_adj_forward(self._h, ctypes.c_void_p(s0.data_ptr()), self.t0, 1, 0, None))
        if dt is None:
            dt = float(self.schedule()[0])
        err = np.zeros(5)
        check(lib().pg_adj_model_error(self._h, dt, err.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        self.recorded = False
        return err

    def dot_test(self, sigma0, seed: int = 0) -> np.ndarray:
        """Runs one step from sigma0, then the adjoint dot-product test of every pass
        over the next step (the first step's dt): rows (kick1, sweep_x, sweep_y,
        advect, kick2) of (<lam, J dir> forward mode, <J^T lam, dir> adjoint)."""
        import torch

        s0 = sigma0.detach().to(torch.float64).contiguous()
        check(lib().pg_adj_forward(self._h, ctypes.c_void_p(s0.data_ptr()), self.t0, 1, 0, None))
        dt = float(self.schedule()[0])
        p = self.params
        g = torch.Generator(device="cuda").manual_seed(seed)
        shape = (5, p.yres, p.xres)
        dirs = torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
        lam = torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
        dirs[0] *= s0  # relative perturbations of Sigma
        out = np.zeros(10)
        check(lib().pg_adj_dot_test(self._h, dt, ctypes.c_void_p(dirs.data_ptr()), ctypes.c_void_p(lam.data_ptr()),
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        self.recorded = False
        return out.reshape(5, 2)

    def pass_check(self, sigma0, steps_before: int = 1, eps: float = 1.0e-7, seed: int = 0) -> np.ndarray:
        """Runs steps_before steps from sigma0, then compares the tangent of every pass
        of the next step with central differences of the production kernels along a
        smooth direction: [production, restated] x rows (kick1, sweep_x, sweep_y,
        advect, kick2) x (Sigma, v_r, v_phi) of |fd - tangent|_2 / |tangent|_2.
        Leaves no recorded run."""
        import torch

        s0 = sigma0.detach().to(torch.float64).contiguous()
        check(lib().pg_adj_forward(self._h, ctypes.c_void_p(s0.data_ptr()), self.t0, steps_before, 0, None))
        dt = float(self.schedule()[-1])
        p = self.params
        x = np.log(np.linspace(1.0, 2.0, p.xres))[None, :]
        y = (np.arange(p.yres) + 0.5)[:, None] * 2 * np.pi / p.yres
        rng = np.random.default_rng(seed)
        ph = rng.uniform(0, 2 * np.pi, size=(5, 2))
        dirs = torch.tensor(np.stack([np.cos(2 * y + ph[k, 0]) * np.sin(5 * x + ph[k, 1]) + 0.3 for k in range(5)]),
                            device="cuda", dtype=torch.float64)
        dirs[0] *= s0
        dirs[1:3] *= 1.0e-3
        out = np.zeros(30)
        check(lib().pg_adj_pass_check(self._h, dt, eps, ctypes.c_void_p(dirs.data_ptr()),
                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        self.recorded = False
        return out.reshape(2, 5, 3)

    def schedule(self) -> np.ndarray:
        n = lib().pg_adj_steps(self._h)
        out = np.zeros(n)
        check(lib().pg_adj_schedule(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
        return out

    @property
    def device_bytes(self) -> int:
        return int(lib().pg_adj_device_bytes(self._h))

    def set_sweep_reverse(self, hand: bool) -> None:
        """Transpose the sweeps' face fluxes with the hand-written reverse-mode
        kernels (default) or with the dual-number kernels that check them."""
        check(lib().pg_adj_set_sweep_reverse(self._h, int(bool(hand))))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pg_adj_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _function():
    import torch

    class EvolveSigma(torch.autograd.Function):
        """Sigma0 (yres, xres), theta = (q, alpha, h/r) -> Sigma after the model's nsteps."""

        @staticmethod
        def forward(ctx, sigma0, theta, model):
            q, alpha, h = (float(x) for x in theta.detach().cpu().tolist())
            model.set_theta(q, alpha, h)
            ctx.model = model
            ctx.theta_device = theta.device
            return model.forward(sigma0)

        @staticmethod
        def backward(ctx, grad):
            gs0, gth = ctx.model.backward(grad)
            return gs0, torch.as_tensor(gth, dtype=torch.float64, device=ctx.theta_device), None

    return EvolveSigma


_EVOLVE = None


def evolve_sigma(sigma0, theta, model: DiskAdjoint):
    """Differentiable Sigma after model.nsteps steps (torch.autograd.Function).
    The first call records the dt schedule; later calls replay it."""
    global _EVOLVE
    if _EVOLVE is None:
        _EVOLVE = _function()
    return _EVOLVE.apply(sigma0, theta, model)
