"""Gradient of the emergent spectrum with respect to absorption opacity, by
path replay (sed_diff_* in include/sedona_gpu.h), exposed to torch.

`DiffEngine` drives one context: `forward(theta)` runs the weighted
transport with the absorption opacity of zone z in frequency band k scaled by
theta[z, k] and returns the binned emergent spectrum; `vjp(g)` and
`jacobian()` replay the escaped packets of that forward.

`spectrum_from_absorption(theta, engine, step)` is the same forward as a
torch.autograd.Function (SpectrumFromAbsorption, from autograd_function()):
its backward is the path-replay vector-Jacobian product.  `step` fixes the
Philox step number, so every evaluation with the same step uses the same
deviates (common random numbers) and the spectrum is a smooth function of
theta.

`vjp_density(g)` is the gradient with respect to each zone's density (both
extinctions of the zone scale with it; opacity per unit mass held), and
`spectrum_from_density(r, engine, step)` the torch Function of the per-zone
density factors r: its forward scales the tables of the last opacity build
on the device (sed_diff_scale_extinction), its backward is that replay.

Both torch Functions keep CUDA tensors on the device: theta or r, the
spectrum and the gradients go through the _dev entry points as device
pointers (no host copy); CPU tensors take the host entry points.  The scattering part of the density derivative
is a likelihood-ratio (score) term, since the scattering opacity decides
where a path goes: unbiased, but not a smooth function of r for fixed
deviates, so it is checked against finite differences of the expected
spectrum, not of one set of deviates.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import abi
from .engine import Engine


class DiffEngine(Engine):
    """One context running the weighted forward and its adjoint replay."""

    def __init__(self, workload, n_bands: int, precision: int = abi.PREC_FP64, device: int = 0,
                 n_packets: Optional[int] = None):
        super().__init__(workload, precision=precision, device=device, n_packets=n_packets)
        self.n_bands = int(n_bands)
        self.forward_id = 0          # increments with every forward
        self._have_tables = False
        self._scaled = False         # the context holds density-scaled tables

    def tables(self, dt: float = 1.0):
        """Opacity build (sed_set_opacity); the forward runs on these tables."""
        self.set_opacity(dt)
        self._have_tables = True
        self._scaled = False

    def _unscale(self):
        if self._scaled:  # a density forward left scaled tables: the built ones back
            self._check(self.L.sed_diff_scale_extinction(self.ctx, None), "sed_diff_scale_extinction")
            self._scaled = False

    def forward(self, theta: Optional[np.ndarray] = None, step: Optional[int] = None, dt: float = 1.0):
        """Weighted forward on the tables of the last opacity build; returns
        (flux, click, stats)."""
        if not self._have_tables:
            self.tables(dt)
        self._unscale()
        return self._forward(theta, step, dt)

    def forward_dev(self, theta, step: Optional[int] = None, dt: float = 1.0):
        """forward() with theta a CUDA float64 tensor ([n_zones, n_bands] or
        None); returns the spectrum as a CUDA float64 tensor, on the device
        throughout (sed_diff_forward_dev)."""
        import torch
        if not self._have_tables:
            self.tables(dt)
        self._unscale()
        if step is not None:
            self._check(self.L.sed_set_rng_step(self.ctx, int(step) & 0xFFFFFFFF), "sed_set_rng_step")
        th = None
        if theta is not None:
            theta = _dev_f64(theta, self.nz * self.n_bands, "theta")
        flux = torch.empty(self.nspec, dtype=torch.float64, device=theta.device if theta is not None else "cuda")
        torch.cuda.current_stream().synchronize()  # theta written before the library's stream reads it
        st = abi.StepStats()
        self._check(self.L.sed_diff_forward_dev(self.ctx, dt, theta.data_ptr() if theta is not None else None,
                                                self.n_bands, flux.data_ptr(), C.byref(st)), "sed_diff_forward_dev")
        self.forward_id += 1
        return flux

    def vjp_dev(self, grad_flux, density: bool = False):
        """vjp() / vjp_density() with grad_flux a CUDA float64 tensor; the
        gradient comes back as a CUDA tensor ([n_zones, n_bands] or [n_zones])."""
        import torch
        g = _dev_f64(grad_flux, self.nspec, "grad_flux")
        out = torch.empty(self.nz if density else self.nz * self.n_bands, dtype=torch.float64, device=g.device)
        torch.cuda.current_stream().synchronize()
        st = abi.StepStats()
        fn = self.L.sed_diff_vjp_density_dev if density else self.L.sed_diff_vjp_dev
        self._check(fn(self.ctx, g.data_ptr(), out.data_ptr(), C.byref(st)), "sed_diff_vjp_dev")
        self.last_replay = st.as_dict()
        return out if density else out.reshape(self.nz, self.n_bands)

    def scale_density_dev(self, r):
        """Both extinctions of zone z of the built tables times r[z], r a CUDA
        float64 tensor (sed_diff_scale_extinction_dev)."""
        import torch
        if not self._have_tables:
            self.tables()
        r = _dev_f64(r, self.nz, "r")
        torch.cuda.current_stream().synchronize()
        self._check(self.L.sed_diff_scale_extinction_dev(self.ctx, r.data_ptr()), "sed_diff_scale_extinction_dev")
        self._scaled = True

    def _forward(self, theta, step, dt):
        if step is not None:
            self._check(self.L.sed_set_rng_step(self.ctx, int(step) & 0xFFFFFFFF), "sed_set_rng_step")
        k = abi.Keep()
        th = None
        if theta is not None:
            theta = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
            if theta.size != self.nz * self.n_bands:
                raise ValueError("theta has %d entries, expected %d x %d" % (theta.size, self.nz, self.n_bands))
            th = k.d(theta)
        st = abi.StepStats()
        self._check(self.L.sed_diff_forward(self.ctx, dt, th, self.n_bands, C.byref(st)), "sed_diff_forward")
        self.forward_id += 1
        flux, click = self.spectrum()
        return flux, click, st.as_dict()

    def vjp(self, grad_flux: np.ndarray) -> np.ndarray:
        g = np.ascontiguousarray(grad_flux, dtype=np.float64).reshape(-1)
        if g.size != self.nspec:
            raise ValueError("grad_flux has %d entries, expected %d" % (g.size, self.nspec))
        out = np.zeros(self.nz * self.n_bands)
        st = abi.StepStats()
        self._check(self.L.sed_diff_vjp(self.ctx, g.ctypes.data_as(abi._dp), out.ctypes.data_as(abi._dp),
                                        C.byref(st)), "sed_diff_vjp")
        self.last_replay = st.as_dict()
        return out.reshape(self.nz, self.n_bands)

    def vjp_density(self, grad_flux: np.ndarray) -> np.ndarray:
        """sum_s grad_flux[s] d E[flux[s]] / d ln rho_z of the last forward."""
        g = np.ascontiguousarray(grad_flux, dtype=np.float64).reshape(-1)
        if g.size != self.nspec:
            raise ValueError("grad_flux has %d entries, expected %d" % (g.size, self.nspec))
        out = np.zeros(self.nz)
        st = abi.StepStats()
        self._check(self.L.sed_diff_vjp_density(self.ctx, g.ctypes.data_as(abi._dp), out.ctypes.data_as(abi._dp),
                                                C.byref(st)), "sed_diff_vjp_density")
        self.last_replay = st.as_dict()
        return out

    def forward_density(self, r: np.ndarray, step: Optional[int] = None, dt: float = 1.0):
        """Weighted forward with the extinction of zone z scaled by r[z]
        (the tables of the last opacity build, both absorption and
        scattering); returns (flux, click, stats)."""
        if not self._have_tables:
            self.tables(dt)
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
        if r.size != self.nz:
            raise ValueError("r has %d entries, expected %d" % (r.size, self.nz))
        self._check(self.L.sed_diff_scale_extinction(self.ctx, r.ctypes.data_as(abi._dp)), "sed_diff_scale_extinction")
        self._scaled = True
        return self._forward(None, step, dt)

    def jacobian(self) -> np.ndarray:
        out = np.zeros(self.nspec * self.nz * self.n_bands)
        st = abi.StepStats()
        self._check(self.L.sed_diff_jacobian(self.ctx, out.ctypes.data_as(abi._dp), C.byref(st)),
                    "sed_diff_jacobian")
        self.last_replay = st.as_dict()
        return out.reshape(self.nspec, self.nz, self.n_bands)


def _torch():
    import torch
    return torch


def _dev_f64(t, n: int, what: str):
    """t as a contiguous CUDA float64 tensor of n entries."""
    torch = _torch()
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise TypeError("%s must be a CUDA tensor" % what)
    t = t.detach().to(torch.float64).contiguous().reshape(-1)
    if t.numel() != n:
        raise ValueError("%s has %d entries, expected %d" % (what, t.numel(), n))
    return t


def _make_function():
    torch = _torch()

    class SpectrumFromAbsorption(torch.autograd.Function):
        """flux = F(theta): the weighted transport's binned emergent spectrum
        (float64, [n_spec]) as a function of the (zone, band) absorption
        factors theta ([n_zones, n_bands], float64).  Backward replays the
        packets of the forward; if another forward ran on the engine since,
        this forward is run again first (same theta, same step)."""

        @staticmethod
        def forward(ctx, theta, engine: DiffEngine, step: int):
            ctx.engine = engine
            ctx.step = step
            ctx.save_for_backward(theta)
            if theta.is_cuda:
                flux = engine.forward_dev(theta, step=step)
            else:
                f, _, _ = engine.forward(theta.detach().to(torch.float64).numpy(), step=step)
                flux = torch.from_numpy(f)
            ctx.fid = engine.forward_id
            return flux

        @staticmethod
        def backward(ctx, grad_flux):
            (theta,) = ctx.saved_tensors
            eng = ctx.engine
            if theta.is_cuda:
                if eng.forward_id != ctx.fid:
                    eng.forward_dev(theta, step=ctx.step)
                grad = eng.vjp_dev(grad_flux)
                return grad.to(theta.dtype), None, None
            if eng.forward_id != ctx.fid:
                eng.forward(theta.detach().to(torch.float64).numpy(), step=ctx.step)
            grad = eng.vjp(grad_flux.detach().to("cpu", torch.float64).numpy())
            return torch.from_numpy(grad).to(theta.dtype), None, None

    return SpectrumFromAbsorption


def _make_density_function():
    torch = _torch()

    class SpectrumFromDensity(torch.autograd.Function):
        """flux = F(r): the weighted transport's binned emergent spectrum as a
        function of per-zone density factors r ([n_zones], float64) applied
        to both extinctions of the last opacity build.  Backward:
        d/d r_z = (d/d ln rho_z) / r_z from the density replay."""

        @staticmethod
        def forward(ctx, r, engine: DiffEngine, step: int):
            ctx.engine = engine
            ctx.step = step
            ctx.save_for_backward(r)
            if r.is_cuda:
                flux = _density_forward_dev(engine, r, step)
            else:
                f, _, _ = engine.forward_density(r.detach().to(torch.float64).numpy(), step=step)
                flux = torch.from_numpy(f)
            ctx.fid = engine.forward_id
            return flux

        @staticmethod
        def backward(ctx, grad_flux):
            (r,) = ctx.saved_tensors
            eng = ctx.engine
            if r.is_cuda:
                if eng.forward_id != ctx.fid:
                    _density_forward_dev(eng, r, ctx.step)
                grad = eng.vjp_dev(grad_flux, density=True) / r.detach().to(torch.float64)
                return grad.to(r.dtype), None, None
            rr = r.detach().to(torch.float64).numpy()
            if eng.forward_id != ctx.fid:
                eng.forward_density(rr, step=ctx.step)
            grad = eng.vjp_density(grad_flux.detach().to("cpu", torch.float64).numpy()) / rr
            return torch.from_numpy(grad).to(r.dtype), None, None

    return SpectrumFromDensity


def _density_forward_dev(engine: DiffEngine, r, step: int):
    """Weighted forward on the built tables scaled by r (a CUDA tensor), all on the device."""
    engine.scale_density_dev(r)
    if step is not None:
        engine._check(engine.L.sed_set_rng_step(engine.ctx, int(step) & 0xFFFFFFFF), "sed_set_rng_step")
    import torch
    flux = torch.empty(engine.nspec, dtype=torch.float64, device=r.device)
    st = abi.StepStats()
    engine._check(engine.L.sed_diff_forward_dev(engine.ctx, 1.0, None, engine.n_bands, flux.data_ptr(), C.byref(st)),
                  "sed_diff_forward_dev")
    engine.forward_id += 1
    return flux


_FN = None
_FN_RHO = None


def spectrum_from_density(r, engine: DiffEngine, step: int = 0):
    """torch entry point: the spectrum as a function of per-zone density factors."""
    global _FN_RHO
    if _FN_RHO is None:
        _FN_RHO = _make_density_function()
    return _FN_RHO.apply(r, engine, step)


def spectrum_from_absorption(theta, engine: DiffEngine, step: int = 0):
    """torch entry point: the differentiable spectrum for `theta`."""
    global _FN
    if _FN is None:
        _FN = _make_function()
    return _FN.apply(theta, engine, step)


def autograd_function():
    """The torch.autograd.Function class SpectrumFromAbsorption (built on
    first use, so importing this module does not import torch)."""
    global _FN
    if _FN is None:
        _FN = _make_function()
    return _FN
