"""Serving loop: requests overlap on the device through worker slots, results are identical
alone and in a concurrent mix, warm starts and matrix reuse work, and the HBM budget evicts
idle systems instead of failing."""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _entry(case):
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    return case, diag, up, lo, src


def _cases():
    return [_entry(c) for c in (W.batch_box(10, seed=1), W.tet(6, seed=2), W.batch_box(14, seed=3),
                                W.graded(12, seed=4))]


@pytest.mark.parametrize("schedule", ["fifo", "most_work"])
def test_same_result_alone_and_in_the_mix(gpu, schedule):
    from cfd_b200.serving import Server
    cases = _cases()
    alone = []
    for case, d, u, l, b in cases:
        s = Server(slots=1)
        mid = s.add_mesh(case.n, case.owner, case.neighbour)
        x, st, _ = s.wait(s.submit(mid, 1, d, u, l, b))
        assert st.converged
        alone.append(x)
        s.close()
    s = Server(slots=4, schedule=schedule)
    ids = [s.add_mesh(c.n, c.owner, c.neighbour) for c, *_ in cases]
    tickets = [s.submit(mid, 1, d, u, l, b) for mid, (c, d, u, l, b) in zip(ids, cases)]
    tickets += [s.submit(mid, 1, d, u, l, b) for mid, (c, d, u, l, b) in zip(ids, cases)]
    outs = [s.wait(t) for t in tickets]
    for i, (x, st, times) in enumerate(outs):
        assert st.converged
        assert np.array_equal(x, alone[i % len(cases)])  # bit-identical alone and in the mix
    # requests on different meshes overlapped in time
    spans = [(o[2][1], o[2][2]) for o in outs[:len(cases)]]
    assert any(a[0] < b[1] and b[0] < a[1] for i, a in enumerate(spans) for b in spans[i + 1:])
    s.close()


def test_warm_start_and_budget_eviction(gpu):
    from cfd_b200.serving import Server
    cases = _cases()
    # the budget holds the largest system but not all four, so admission must evict
    s = Server(slots=2, hbm_budget_bytes=2.5e6)
    ids = [s.add_mesh(c.n, c.owner, c.neighbour) for c, *_ in cases]
    (c0, d, u, l, b) = cases[0]
    x1, st1, _ = s.wait(s.submit(ids[0], 7, d, u, l, b))
    x2, st2, _ = s.wait(s.submit(ids[0], 7, d, u, l, b, warm_start=True))
    assert st1.converged and st2.converged and st2.iterations <= 1 < st1.iterations
    for mid, (c, d, u, l, b) in zip(ids, cases):
        x, st, _ = s.wait(s.submit(mid, 1, d, u, l, b))
        assert st.converged
        a = O.ldu_to_csr(O.build_pattern(c.n, c.owner, c.neighbour), d, u, l)
        assert np.linalg.norm(b - a.matvec(x)) <= 1.05e-8 * np.linalg.norm(b)
    info = s.info()
    assert info["evictions"] >= 1 and info["resident_systems"] < len(cases)
    s.close()


@pytest.mark.parametrize("background", [False, True], ids=["inline", "background"])
def test_age_rule_rebuilds(gpu, background):
    """Hierarchies are rebuilt after max_age solves of new matrices, on the request path or by
    the background rebuild thread (swapped in at a later request); every solve meets its
    tolerance against the oracle's matrix-vector product either way."""
    import time

    from cfd_b200 import serving as S
    case, d, u, l, b = _entry(W.tet(6, seed=2))
    s = S.Server(slots=2, max_age=3, background_rebuild=background)
    (e,) = S.make_pool(s, [("tet", case, d, u, l, b)], variants=3, seed=5)
    pat = O.build_pattern(case.n, case.owner, case.neighbour)
    for k in range(1, 16):
        dk, uk, lk = e.matrices[k % 3]
        rhs = e.rhs[k % 3]
        x, st, _ = s.wait(s.submit(e.mesh_id, k, dk, uk, lk, rhs))
        a = O.ldu_to_csr(pat, dk, uk, lk)
        assert st.converged
        assert np.linalg.norm(rhs - a.matvec(x)) <= 1.05e-8 * np.linalg.norm(rhs)
        time.sleep(0.05)  # room for the background build between requests
    info = s.info()
    if background:
        assert info["rebuilds"] == 0 and info["background_rebuilds"] >= 2
    else:
        assert info["rebuilds"] >= 3 and info["background_rebuilds"] == 0
    s.close()
