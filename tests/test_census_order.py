"""The order in which packets are carried to the next step (CPU).

transport::clean_up_particle_vector (src/transport/transport.cpp:164-194)
removes escaped and absorbed packets by swapping the last live packet into
each hole from the front.  The census kernels reproduce its result without
running it serially: with E the exclusive sum of "packet exists" flags
(radioactive slots that emitted nothing are not in the reference's vector),
A the exclusive sum of "packet is stopped" flags and n_alive stopped packets
in all, a stopped packet at vector position s < n_alive stays at s, and the
j-th hole below n_alive (counted from the front) takes the j-th stopped
packet counted from the back, i.e. the one with A = n_alive - 1 - j.  This
restates that mapping with numpy and checks it against the reference's loop
on random fates, including all-dead, all-alive and empty vectors."""
import numpy as np
import pytest

MOVING, STOPPED, ESCAPED, ABSORBED = 0, 1, 2, 3


def reference_cleanup(fates):
    """clean_up_particle_vector on a list of (fate, id); returns surviving ids in order."""
    v = [(f, i) for i, f in enumerate(fates) if f != -1]
    dead = lambda f: f in (ESCAPED, ABSORBED)
    i = 0
    while True:
        while v and dead(v[-1][0]):
            v.pop()
        if i >= len(v):
            break
        if dead(v[i][0]):
            v[i] = v[-1]
            v.pop()
        i += 1
    return [idx for _, idx in v]


def scan_mapping(fates):
    """The census kernels' mapping (flags, exclusive sums, front holes, scatter)."""
    f = np.asarray(fates)
    e = (f != -1).astype(np.int64)
    a = (f == STOPPED).astype(np.int64)
    E = np.concatenate([[0], np.cumsum(e)])
    A = np.concatenate([[0], np.cumsum(a)])
    n = f.size
    n_alive = int(A[n])
    front = np.full(n_alive, -1, np.int64)
    for r in range(n):
        if e[r] and not a[r] and E[r] < n_alive:
            front[E[r] - A[r]] = E[r]
    out = np.full(n_alive, -1, np.int64)
    for r in range(n):
        if a[r]:
            dest = E[r] if E[r] < n_alive else front[n_alive - 1 - A[r]]
            out[dest] = r
    return out.tolist()


@pytest.mark.parametrize("seed", range(40))
def test_scan_mapping_is_the_reference_compaction(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(0, 400))
    p = rng.dirichlet(np.ones(4))
    fates = rng.choice([-1, STOPPED, ESCAPED, ABSORBED], size=n, p=p)
    assert scan_mapping(fates) == reference_cleanup(fates)


@pytest.mark.parametrize("fates", [[], [STOPPED] * 7, [ESCAPED] * 5, [ABSORBED, STOPPED, ESCAPED, STOPPED],
                                   [-1, -1, STOPPED], [STOPPED, -1, ABSORBED, -1, STOPPED, STOPPED]])
def test_edge_cases(fates):
    assert scan_mapping(fates) == reference_cleanup(fates)
