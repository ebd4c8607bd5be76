"""The reference's diffusing-pulse test (tests/diffusing_pulse/1D_ddmc) on
the GPU path: a static sphere whose inner 5 cm start at 1e4 K, pure
scattering at rho kappa = 1 / cm, every zone diffusive (method 2 above zone
optical depth 0.1), 1e5 packets of the initial radiation field carried from
step to step by the driver's time loop.  Its criterion: at the 6th, 12th and
18th plot file, the radiation temperature within 10% (mean over zones) of
the diffusion solution of a pulse at r0 = 2.5 cm with D = c / (3 rho kappa),
normalised to the pulse's energy."""
import numpy as np
import pytest

from pubsed_b200 import abi, workloads
from pubsed_b200.transport import run_time_dependent

pytestmark = pytest.mark.gpu


def analytic_T(r, tr, time, r0=2.5, rho=1.0):
    n = r.size
    esum = sum(tr[i] ** 4 * (r[i] ** 3 - r[i - 1] ** 3) * 4.0 / 3.0 * 3.14159 for i in range(1, n - 1))
    D = 3e10 / rho / 3.0
    Ean = np.exp(-1.0 * (r - r0) ** 2 / (4.0 * D * time)) - np.exp(-1.0 * (r + r0) ** 2 / (4.0 * D * time))
    Ean = Ean * r0 / r
    Enorm = sum(Ean[i] * (r[i] ** 3 - r[i - 1] ** 3) * 4.0 / 3.0 * 3.14159 for i in range(1, n - 1))
    return (Ean / Enorm * esum) ** 0.25


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_diffusing_pulse(sed_lib, tmp_path, precision):
    w = workloads.diffusing_pulse(n_initialize=100_000, seed=11)
    r, tr = w.zones.r_out.copy(), w.zones.T.copy()
    got = {}

    def on_write(i, t_write, transport):
        if i in (6, 12, 18):
            got[i] = (t_write, np.loadtxt(str(tmp_path / ("plt_%05d.dat" % i)))[:, 4])  # T_rad column

    tr_ = run_time_dependent(w, str(tmp_path), precision=precision, on_write=on_write)
    assert tr_.n_particles() > 0  # the field is carried between steps
    assert sorted(got) == [6, 12, 18]
    for i, (t_write, T) in got.items():
        Tan = analytic_T(r, tr, t_write)
        mean_err = np.mean(np.abs(T - Tan)) / np.mean(Tan)
        assert mean_err < 0.1, (i, mean_err)
    tr_.close()
