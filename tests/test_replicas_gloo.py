"""N>1 path on CPU: two gloo ranks each propagate half of the packets with
offset Philox stream ids and average their tallies over ranks; the result
must equal one run with all packets (the reference's MPI packet split)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

N_PER_RANK = 300


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, outdir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch.distributed as dist
    from pubsed_b200 import parallel, workloads
    import oracle_lib

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    w = workloads.lightbulb_grey(n_packets=N_PER_RANK, n_zones=32, n_bins=128, radiative_eq=1, seed=11)
    e = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w,
                          first_packet_id=parallel.first_packet_id(rank, N_PER_RANK))
    e.set_opacity(1.0)
    e.transport(1.0)
    T = e.tallies()
    f, c = e.spectrum()
    avg = parallel.average_over_ranks({"J_nu": T["J_nu"], "e_abs": T["e_abs"], "flux": f, "click": c})
    tmax = parallel.max_over_ranks(float(rank))
    if rank == 0:
        np.savez(os.path.join(outdir, "avg.npz"), tmax=tmax, **avg)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_average_equals_single_run():
    outdir = tempfile.mkdtemp()
    mp.spawn(_rank_main, args=(2, _free_port(), outdir), nprocs=2, join=True)
    avg = np.load(os.path.join(outdir, "avg.npz"))
    assert float(avg["tmax"]) == 1.0

    from pubsed_b200 import workloads
    import oracle_lib
    w = workloads.lightbulb_grey(n_packets=2 * N_PER_RANK, n_zones=32, n_bins=128, radiative_eq=1, seed=11)
    e = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    e.set_opacity(1.0)
    e.transport(1.0)
    T = e.tallies()
    f, c = e.spectrum()
    # packet energies differ by exactly 2 (L dt / n_emit), so the tallies
    # agree up to summation order; clicks are averaged by the reference
    for a, b in ((avg["J_nu"], T["J_nu"]), (avg["e_abs"], T["e_abs"]), (avg["flux"], f)):
        s = np.maximum(np.abs(b), 1e-300)
        assert np.max(np.abs(a - b) / s) <= 1e-12
    assert np.array_equal(2 * avg["click"], c)
