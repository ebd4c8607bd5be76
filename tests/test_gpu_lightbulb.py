"""The reference's spherical-lightbulb test (tests/spherical_lightbulb/1D) on
the GPU path: one steady-state iteration of the static vacuum model through
pubsed_b200.transport.run_steady (transport step + radiative-equilibrium
temperature solve), its text outputs read back as the reference's test reads
them, and the reference's acceptance criteria applied:

  * T_gas and T_rad (columns 4 and 5 of plt_00001.dat) within 1% (maximum
    relative error) of the dilution-factor temperature
    T_W = (L W / (4 pi r0^2 sigma))^(1/4), W = (1 - sqrt(1 - r0^2/r^2)) / 2,
    beyond r = 5e14 cm (zone radii shifted to zone centres);
  * the spectrum of spectrum_1.dat within 10% (mean error) of the core
    blackbody L B_nu(T) / (sigma T^4 / pi).
"""
import numpy as np
import pytest

from pubsed_b200 import abi, workloads
from pubsed_b200.transport import run_steady

pytestmark = pytest.mark.gpu

H, C_LIGHT, K, SB, PI = 6.6260755e-27, 2.99792458e10, 1.380658e-16, 5.6704e-5, 3.14159


def rel_errors(y, y_ref, x=None, x_ref=None, use=None):
    """maximum of |y - y_ref| / y_ref and mean |y - y_ref| / mean y_ref, with
    y_ref interpolated to x when both abscissae are given and only the
    entries flagged by `use` counted"""
    if x is not None and x_ref is not None:
        y_ref = np.interp(x, x_ref, y_ref)
    if use is not None:
        y, y_ref = y[use], y_ref[use]
    err = np.abs(y - y_ref)
    return float(np.max(err / y_ref)), float(np.mean(err) / np.mean(y_ref))


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_spherical_lightbulb(sed_lib, tmp_path, precision):
    w = workloads.lightbulb_vacuum(n_packets=200_000, seed=31)
    tr = run_steady(w, outdir=str(tmp_path), precision=precision)
    assert tr.n_unsolved == 0
    T, L, r0 = 1e4, 1e43, 0.5e15
    data = np.loadtxt(str(tmp_path / "plt_00001.dat"), skiprows=2)
    r = data[:, 0]
    r = r - 0.5 * (r[1] - r[0])
    tgas, trad = data[:, 3], data[:, 4]
    rr = np.arange(r0 * 1.01, max(r), 0.05 * r0, dtype=np.float64)
    W = 0.5 * (1 - (1 - r0 ** 2 / rr ** 2) ** 0.5)
    TW = (L * W / (4.0 * PI * r0 ** 2) / SB) ** 0.25
    m_gas, _ = rel_errors(tgas, TW, r, rr, use=r > 5e14)
    m_rad, _ = rel_errors(trad, TW, r, rr, use=r > 5e14)
    assert m_gas <= 0.01, m_gas
    assert m_rad <= 0.01, m_rad
    spec = np.loadtxt(str(tmp_path / "spectrum_1.dat"))
    nu, y = spec[:, 0], spec[:, 1]
    f = 2.0 * H * nu ** 3 / C_LIGHT ** 2 / (np.exp(H * nu / K / T) - 1)
    f = f / (SB * T ** 4 / PI) * L
    _, mean_err = rel_errors(y, f)
    assert mean_err <= 0.1, mean_err
    tr.close()
