"""The serving load generator's request trace (host only): one seed gives one trace, repeats
carry their mesh's previous key and variant, new keys cycle the variants, the tet share and the
repeat share follow their probabilities, and arrivals are Poisson at the rate (closed loops
have none)."""
import numpy as np

from cfd_b200.serving import MeshEntry, request_trace


def _pool():
    pool = []
    for i in range(7):
        pool.append(MeshEntry(i, "box", 100 + i, [None] * 3, [None] * 3, []))
    for i in range(5):
        pool.append(MeshEntry(7 + i, "tet", 600 + i, [None] * 3, [None] * 3, []))
    return pool


def test_same_seed_same_trace():
    pool = _pool()
    a = request_trace(pool, 500.0, 400, seed=11)
    b = request_trace(pool, 500.0, 400, seed=11)
    c = request_trace(pool, 500.0, 400, seed=12)
    key = lambda t: [(r[0], r[1].mesh_id, r[2], r[3], r[4], r[5]) for r in t]  # noqa: E731
    assert key(a) == key(b) and key(a) != key(c)


def test_repeats_keys_and_shares():
    pool = _pool()
    trace = request_trace(pool, 1000.0, 4000, seed=3)
    last = {}
    next_key = 1
    for ta, e, k, mi, bi, rep in trace:
        if rep:
            assert (k, mi) == last[e.mesh_id]
        else:
            assert k == next_key and mi == k % 3
            next_key += 1
            last[e.mesh_id] = (k, mi)
        assert 0 <= bi < 3
    tet = np.mean([e.kind == "tet" for _, e, *_ in trace])
    rep = np.mean([r[5] for r in trace[100:]])
    assert abs(tet - 0.25) < 0.03 and abs(rep - 0.3) < 0.03
    gaps = np.diff([0.0] + [r[0] for r in trace])
    assert abs(np.mean(gaps) - 1e-3) < 1e-4 and np.all(gaps > 0)


def test_closed_loop_has_no_arrivals():
    trace = request_trace(_pool(), 0.0, 50, seed=1, closed_loop=True)
    assert all(r[0] == 0.0 for r in trace)
