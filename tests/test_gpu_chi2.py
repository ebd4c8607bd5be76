"""Free-running spectra against the reference within Monte Carlo noise.

The fixtures free_*.npz are the reference's own transport::step run with its
own OpenMP packet loop and random streams (tests/golden/make_golden.py).  The
GPU runs the same workload with a different seed and more packets, in both
forms (the FP64 form, and the mixed form: FP32 tables, FP64 transport
without divisions, Philox words as deviates); each
spectrum must agree with the reference's per bin within Monte Carlo noise:
chi^2 = sum (F_a - F_b)^2 / (F_a^2/N_a + F_b^2/N_b) over bins with at least
10 packets in both runs (adjacent bins are merged first), p-value > 0.01.
"""
import json
import os

import numpy as np
import pytest
from scipy import stats

from pubsed_b200 import abi, workloads
import oracle_lib

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
P_MIN = 0.01


def chi2_spectra(Fa, Ca, Fb, Cb, merge=1, min_clicks=10):
    n = (Fa.size // merge) * merge
    f = lambda a: a[:n].reshape(-1, merge).sum(axis=1)
    Fa, Ca, Fb, Cb = f(Fa), f(Ca), f(Fb), f(Cb)
    m = (Ca >= min_clicks) & (Cb >= min_clicks)
    var = Fa[m] ** 2 / Ca[m] + Fb[m] ** 2 / Cb[m]
    chi2 = float(np.sum((Fa[m] - Fb[m]) ** 2 / var))
    dof = int(m.sum())
    return chi2, dof, float(stats.chi2.sf(chi2, dof))


def _gpu_spectrum(sed_lib, w, precision):
    g = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    g.set_opacity(1.0)
    st = g.transport(1.0)
    f, c = g.spectrum()
    g.close()
    return f, c, st


@pytest.mark.parametrize("case,n_packets,seed,merge", [
    ("free_grey_radeq", 1_000_000, 9001, 2),
    ("free_ia", 600_000, 9002, 8),
    ("free_cart3d", 400_000, 9003, 4),
])
def test_free_running_spectrum_matches_reference(sed_lib, case, n_packets, seed, merge):
    ref = np.load(os.path.join(GOLDEN, case + ".npz"))
    kw = json.loads(str(ref["kwargs"]))
    kw.update(n_packets=n_packets, seed=seed)
    w = getattr(workloads, str(ref["generator"]))(**kw)
    results = {}
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        f, c, st = _gpu_spectrum(sed_lib, w, prec)
        chi2, dof, p = chi2_spectra(f, c, ref["spec_flux"], ref["spec_click"], merge=merge)
        results[prec] = (chi2 / max(dof, 1), p)
        assert dof >= 20, dof
        assert p > P_MIN, (case, prec, chi2, dof, p)
    # both forms sit at the same chi^2 against the FP64 reference
    assert abs(results[abi.PREC_FP64][0] - results[abi.PREC_MIXED][0]) < 0.5, results


def test_mixed_and_fp64_forms_agree_within_noise(sed_lib):
    """The mixed form draws its deviates as the 32-bit words of one Philox
    block per segment (and one per interaction), on streams independent of
    the FP64 form's per-draw layout: the two spectra of the same workload
    agree within Monte Carlo noise."""
    w = workloads.type_ia(n_packets=400_000, n_zones=64, n_lines=50000, n_bins=1024, seed=77)
    f64, c64, _ = _gpu_spectrum(sed_lib, w, abi.PREC_FP64)
    f32, c32, _ = _gpu_spectrum(sed_lib, w, abi.PREC_MIXED)
    chi2, dof, p = chi2_spectra(f32, c32, f64, c64, merge=4)
    assert dof >= 20 and p > P_MIN, (chi2, dof, p)
