"""The differentiable transport on the GPU: weighted forward, path-replay
adjoint, and the torch.autograd.Function over them.

  * the weighted forward draws the oracle's deviates: per packet the same
    integer history and final state (oracle_lib criterion), spectra and
    tallies within the summation-order tolerances;
  * the replayed Jacobian and vector-Jacobian product equal the oracle's
    forward-mode Jacobian (summation order only);
  * central finite differences of the GPU forward (relative step 1e-3, common
    random numbers: the same Philox step) match the adjoint on randomly
    chosen (zone, band) entries, FP64 and mixed tables;
  * the weighted GPU spectrum agrees with the reference's discrete-absorption
    spectrum within Monte Carlo noise;
  * loss.backward() through SpectrumFromAbsorption gives the VJP.
"""
import json
import os

import numpy as np
import pytest
from scipy import stats

from pubsed_b200 import abi, workloads
from pubsed_b200.adjoint import DiffEngine, spectrum_from_absorption
import oracle_lib

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FD_STEP = 1e-3
# analytic in theta for fixed deviates: FD truncation O(h^2), measured ~1e-8
FD_RTOL = 1e-6


def absorbing(n_packets, n_zones=32, n_lines=3000, n_bins=256, spectrum_bins=64, seed=31):
    return workloads.type_ia(n_packets=n_packets, n_zones=n_zones, n_lines=n_lines, n_bins=n_bins,
                             spectrum_bins=spectrum_bins, epsilon=1e-4, radiative_eq=0, seed=seed)


def test_weighted_forward_and_adjoint_match_oracle(sed_lib):
    n, nb = 3000, 16
    w = absorbing(n)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    theta = 1 + 0.2 * np.random.default_rng(3).standard_normal(o.nz * nb)
    for e in (o, g):
        e.set_opacity(1.0)
        e.record(True)
        oracle_lib.diff_forward(e, theta, nb, step=2)
    ro, rg = o.records(n), g.records(n)
    assert np.array_equal(ro["fate"], rg["fate"])
    assert np.array_equal(ro["ind"], rg["ind"])
    assert np.array_equal(ro["draws"], rg["draws"])
    oracle_lib.check_states(rg["state"], ro["state"])
    fo, co = o.spectrum()
    fg, cg = g.spectrum()
    assert np.array_equal(co, cg)
    assert np.abs(fg - fo).max() <= oracle_lib.TALLY_RTOL * np.abs(fo).max()
    To, Tg = o.tallies(), g.tallies()
    for k in ("J_nu", "e_abs", "e_rad", "fx", "fy", "fz", "fr"):
        oracle_lib.zone_tally_close(Tg[k], To[k])
    Jo, Jg = oracle_lib.diff_jacobian(o, nb), oracle_lib.diff_jacobian(g, nb)
    assert np.abs(Jo).max() > 0
    assert np.abs(Jg - Jo).max() <= 1e-10 * np.abs(Jo).max()
    gv = np.random.default_rng(4).standard_normal(o.nspec)
    vg = oracle_lib.diff_vjp(g, gv, nb)
    vo = gv @ Jo
    assert np.abs(vg - vo).max() <= 1e-10 * np.abs(gv) @ np.abs(Jo).max(axis=1)
    o.close()
    g.close()


def test_weighted_forward_and_adjoint_match_oracle_3d(sed_lib):
    """The weighted forward and both replays on an 8^3 Cartesian grid
    against the oracle on the same deviates."""
    n, nb = 3000, 8
    w = workloads.with_params("cart3d", {"transport_radiative_equilibrium": 0}, n_packets=n, n_cells=8,
                              n_lines=3000, n_bins=256, spectrum_bins=64, n_mu=4, epsilon=0.05, seed=11)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    theta = 1 + 0.2 * np.random.default_rng(3).standard_normal(o.nz * nb)
    for e in (o, g):
        e.set_opacity(1.0)
        e.record(True)
        oracle_lib.diff_forward(e, theta, nb, step=2)
    ro, rg = o.records(n), g.records(n)
    assert np.array_equal(ro["fate"], rg["fate"])
    assert np.array_equal(ro["ind"], rg["ind"])
    assert np.array_equal(ro["draws"], rg["draws"])
    oracle_lib.check_states(rg["state"], ro["state"])
    fo, co = o.spectrum()
    fg, cg = g.spectrum()
    assert np.array_equal(co, cg)
    assert np.abs(fg - fo).max() <= oracle_lib.TALLY_RTOL * np.abs(fo).max()
    Jo, Jg = oracle_lib.diff_jacobian(o, nb), oracle_lib.diff_jacobian(g, nb)
    assert np.abs(Jo).max() > 0
    assert np.abs(Jg - Jo).max() <= 1e-10 * np.abs(Jo).max()
    gv = np.random.default_rng(4).standard_normal(o.nspec)
    vg = oracle_lib.diff_vjp(g, gv, nb)
    assert np.abs(vg - gv @ Jo).max() <= 1e-10 * np.abs(gv) @ np.abs(Jo).max(axis=1)
    dg, do = oracle_lib.diff_vjp_density(g, gv), oracle_lib.diff_vjp_density(o, gv)
    assert np.abs(do).max() > 0
    assert np.abs(dg - do).max() <= 1e-9 * np.abs(do).max()
    o.close()
    g.close()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_adjoint_matches_central_differences(sed_lib, precision):
    w = absorbing(100_000, n_zones=64, n_lines=20000, n_bins=1024, spectrum_bins=256, seed=41)
    nb = 64
    eng = DiffEngine(w, n_bands=nb, precision=precision)
    theta = np.ones((eng.nz, nb))
    eng.forward(theta, step=7)
    jac = eng.jacobian().reshape(eng.nspec, -1)
    cols = np.flatnonzero(np.abs(jac).max(axis=0) > 1e-6 * np.abs(jac).max())
    assert cols.size >= 64
    rng = np.random.default_rng(5)
    errs = []
    for q in rng.choice(cols, 12, replace=False):
        tp, tm = theta.copy().reshape(-1), theta.copy().reshape(-1)
        tp[q] += FD_STEP
        tm[q] -= FD_STEP
        fp, _, _ = eng.forward(tp, step=7)
        fm, _, _ = eng.forward(tm, step=7)
        fd = (fp - fm) / (2 * FD_STEP)
        errs.append(np.abs(fd - jac[:, q]).max() / np.abs(jac[:, q]).max())
    assert max(errs) <= FD_RTOL, errs
    eng.close()


def test_weighted_gpu_spectrum_matches_reference(sed_lib):
    ref = np.load(os.path.join(GOLDEN, "free_ia_absorb.npz"))
    kw = json.loads(str(ref["kwargs"]))
    n = 400_000
    kw.update(n_packets=n, seed=7001)
    w = workloads.type_ia(**kw)
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        g = oracle_lib.Engine(sed_lib, "sed_", w, precision=prec)
        g.set_opacity(1.0)
        g.record(True)
        oracle_lib.diff_forward(g, None, 8, step=0)
        f, _ = g.spectrum()
        s1, s2 = oracle_lib.spectrum_second_moment(g, w, n)
        assert np.allclose(s1, f, rtol=1e-10, atol=0)
        r = lambda a: a.reshape(-1, 4).sum(axis=1)
        Fa, Va, Fb, Cb = r(f), r(s2), r(ref["spec_flux"]), r(ref["spec_click"])
        m = (Cb >= 10) & (Va > 0)
        chi2 = float(np.sum((Fa[m] - Fb[m]) ** 2 / (Va[m] + Fb[m] ** 2 / Cb[m])))
        dof = int(m.sum())
        assert dof >= 20 and stats.chi2.sf(chi2, dof) > 0.01, (prec, chi2, dof)
        g.close()


def test_autograd_function_backward_is_the_vjp(sed_lib):
    import torch
    w = absorbing(5000, seed=51)
    nb = 16
    eng = DiffEngine(w, n_bands=nb)
    theta = torch.ones(eng.nz, nb, dtype=torch.float64, requires_grad=True)
    weights = torch.linspace(0.5, 1.5, eng.nspec, dtype=torch.float64)
    flux = spectrum_from_absorption(theta, eng, 9)
    loss = (flux * weights).sum() / flux.detach().sum()
    # another forward in between: backward must replay its own forward
    eng.forward(np.full((eng.nz, nb), 1.3), step=1)
    loss.backward()
    eng.forward(np.ones((eng.nz, nb)), step=9)
    v = eng.vjp((weights / flux.detach().sum()).numpy())
    assert torch.allclose(theta.grad, torch.from_numpy(v), rtol=1e-12, atol=1e-300)
    # a directional derivative against central differences
    d = np.random.default_rng(6).standard_normal((eng.nz, nb))
    h = 1e-4
    fp, _, _ = eng.forward(1 + h * d, step=9)
    fm, _, _ = eng.forward(1 - h * d, step=9)
    s = flux.detach().sum().item()
    dd = float(((fp - fm) / (2 * h)) @ weights.numpy()) / s
    ad = float((theta.grad.numpy() * d).sum())
    assert abs(dd - ad) <= 1e-6 * abs(ad)
    eng.close()


def test_density_vjp_matches_oracle(sed_lib):
    """The density replay on the GPU and the oracle's per-packet estimator on
    the same deviates: the same terms, summed in another order."""
    w = workloads.type_ia(n_packets=20000, n_zones=32, n_lines=3000, n_bins=256, spectrum_bins=64, epsilon=1e-4,
                          radiative_eq=0, seed=23)
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    rng = np.random.default_rng(3)
    gg = rng.normal(size=g.nspec)
    out = []
    for e in (g, o):
        e.set_opacity(1.0)
        oracle_lib.diff_forward(e, np.ones(e.nz * 4), 4, step=2)
        out.append(oracle_lib.diff_vjp_density(e, gg))
    scale = np.abs(out[1]).max()
    assert scale > 0
    assert np.abs(out[0] - out[1]).max() <= 1e-9 * scale
    g.close()
    o.close()


def test_density_gradient_against_finite_differences_at_scale(sed_lib):
    """1e7 packets: the replay's d(total escaped energy)/d ln rho of every
    zone at once, against central differences of the expected spectrum with
    both extinctions scaled by (1 +- 0.05) and common deviates.  The
    scattering score makes the replay estimate noisy (measured: 4% standard
    deviation over Philox steps at 1e7 packets; the finite differences vary
    by 0.5% with the step and by 1% with h from 0.0125 to 0.1), so the replay
    is averaged over four steps and must agree within 6% (3 standard
    deviations of that mean)."""
    w = workloads.type_ia(n_packets=10_000_000, epsilon=1e-4, radiative_eq=0, seed=29)
    e = DiffEngine(w, n_bands=1)
    nz = e.nz
    lr = []
    for step in (7, 8, 9, 10):
        e.forward_density(np.ones(nz), step=step)
        lr.append(e.vjp_density(np.ones(e.nspec)).sum())

    def total(r):
        f, _, _ = e.forward_density(r, step=7)
        return f.sum()

    h = 0.05
    fd = (total(np.full(nz, 1 + h)) - total(np.full(nz, 1 - h))) / (np.log(1 + h) - np.log(1 - h))
    assert fd < 0
    assert abs(np.mean(lr) / fd - 1) < 0.06, (lr, fd)
    e.close()


def test_density_autograd_function(sed_lib):
    import torch
    from pubsed_b200.adjoint import spectrum_from_density
    w = workloads.type_ia(n_packets=200_000, n_zones=32, n_lines=3000, n_bins=256, spectrum_bins=64, epsilon=1e-4,
                          radiative_eq=0, seed=31)
    e = DiffEngine(w, n_bands=1)
    r = torch.full((e.nz,), 1.1, dtype=torch.float64, requires_grad=True)
    flux = spectrum_from_density(r, e, 5)
    g = torch.linspace(0, 1, flux.numel(), dtype=torch.float64)
    (flux * g).sum().backward()
    e.forward_density(np.full(e.nz, 1.1), step=5)
    ref = e.vjp_density(g.numpy()) / 1.1
    assert np.allclose(r.grad.numpy(), ref, rtol=1e-12, atol=0)
    e.close()


def test_density_forward_leaves_the_built_tables(sed_lib):
    """Forwards on the built tables, on density-scaled tables and after a
    rebuild at another temperature interleave: a plain forward always runs on
    the last build, a density forward scales the last build (not an earlier
    one), and a replay after a call that changed the context is refused."""
    w = workloads.type_ia(n_packets=20_000, n_zones=16, n_lines=2000, n_bins=128, spectrum_bins=32, epsilon=1e-4,
                          radiative_eq=0, seed=33)
    e = DiffEngine(w, n_bands=1)
    # the same deviates give the same packet histories: the same spectrum
    # clicks, and fluxes equal up to the order of the FP64 atomic sums
    def same(a, b):
        return np.array_equal(a[1], b[1]) and np.allclose(a[0], b[0], rtol=oracle_lib.TALLY_RTOL, atol=0)

    f0 = e.forward(step=3)
    f1 = e.forward_density(np.full(e.nz, 1.3), step=3)
    assert not same(f0, f1)
    f2 = e.forward(step=3)
    assert same(f0, f2)  # the built tables are back
    w.zones.T = w.zones.T * 1.1
    e.upload_grid()
    e.tables()
    g0 = e.forward(step=3)
    g1 = e.forward_density(np.ones(e.nz), step=3)
    assert same(g0, g1)  # density factor 1 on the new build, not the old one
    assert not same(g0, f0)
    e.tables()  # a rebuild after the forward: nothing left to replay
    with pytest.raises(RuntimeError, match="replay"):
        e.vjp(np.ones(e.nspec))
    e.close()


def test_autograd_functions_keep_cuda_tensors_on_the_device(sed_lib):
    """theta and r as CUDA tensors: the forward returns a CUDA spectrum and
    the backward a CUDA gradient through the device-pointer entry points,
    equal to the host entry points' results (the same device computations,
    only the copies differ)."""
    import torch
    from pubsed_b200.adjoint import spectrum_from_density
    w = absorbing(5000, seed=53)
    nb = 8
    eng = DiffEngine(w, n_bands=nb)
    th = 1 + 0.1 * torch.rand(eng.nz, nb, dtype=torch.float64, generator=torch.Generator().manual_seed(2))
    theta = th.cuda().requires_grad_(True)
    weights = torch.linspace(0.5, 1.5, eng.nspec, dtype=torch.float64, device="cuda")
    flux = spectrum_from_absorption(theta, eng, 4)
    assert flux.is_cuda
    (flux * weights).sum().backward()
    assert theta.grad.is_cuda
    # equal up to the order of FP64 atomic sums, which varies from run to run
    tol = dict(rtol=1e-10, atol=0)
    f_host, _, _ = eng.forward(th.numpy(), step=4)
    assert np.allclose(flux.detach().cpu().numpy(), f_host, **tol)
    v = eng.vjp(weights.cpu().numpy())
    assert np.allclose(theta.grad.cpu().numpy(), v, rtol=1e-10, atol=1e-10 * np.abs(v).max())
    # density factors
    r0 = torch.linspace(0.9, 1.1, eng.nz, dtype=torch.float64)
    r = r0.cuda().requires_grad_(True)
    fr = spectrum_from_density(r, eng, 6)
    (fr * weights).sum().backward()
    assert fr.is_cuda and r.grad.is_cuda
    fr_host, _, _ = eng.forward_density(r0.numpy(), step=6)
    assert np.allclose(fr.detach().cpu().numpy(), fr_host, **tol)
    g_host = eng.vjp_density(weights.cpu().numpy()) / r0.numpy()
    assert np.allclose(r.grad.cpu().numpy(), g_host, rtol=1e-10, atol=1e-10 * np.abs(g_host).max())
    # a plain forward afterwards runs on the built tables again
    f_again, _, _ = eng.forward(th.numpy(), step=4)
    assert np.allclose(f_again, f_host, **tol)
    eng.close()
