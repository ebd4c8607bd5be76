"""CPU checks of the batching host logic: the batch workload has the shapes
of the batching configuration, and a batch refuses models that do not share
what a batch shares (checked before any CUDA call)."""
import math

import numpy as np
import pytest

from pubsed_b200 import workloads
from pubsed_b200.batch import BatchEngine


def test_batch64_shapes():
    bw = workloads.batch64()
    assert len(bw.models) == 64
    nz = np.array([m.zones.n_zones for m in bw.models])
    npk = np.array([m.n_packets for m in bw.models])
    vmax = np.array([m.notes["v_max"] for m in bw.models])
    assert nz.min() >= 64 and nz.max() <= 512
    assert npk.min() >= 1e5 and npk.max() <= 1e7
    assert vmax.min() >= 5e8 and vmax.max() <= 2e9
    # log-uniform packet counts: about half the models below the geometric mean
    assert 16 <= int((npk < math.sqrt(1e5 * 1e7)).sum()) <= 48
    # one Philox key per model, one shared line list and grid time
    seeds = {m.params["transport_rng_seed"] for m in bw.models}
    assert len(seeds) == 64
    assert all(m.atoms is bw.models[0].atoms for m in bw.models)
    assert len({m.zones.t_now for m in bw.models}) == 1
    for m in bw.models:
        z = m.zones
        assert np.all(np.diff(z.r_out) > 0) and np.allclose(z.X.sum(axis=1), 1.0)
        # rho0 normalised to the model's mass
        assert abs(float(np.sum(z.rho * z.vol)) / (m.notes["mass_msun"] * workloads.M_SUN) - 1) < 1e-12


def test_batch_rejects_unshared_parameters():
    bw = workloads.batch64(n_models=3, packets=(100, 200), n_lines=100)
    bw.models[2].params["transport_nu_grid"] = [1e14, 3e15, 0.01, 1]
    with pytest.raises(ValueError, match="shared parameter"):
        BatchEngine(bw)
