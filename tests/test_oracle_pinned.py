"""The CPU oracle is pinned to the reference: against the golden fixtures made by the
reference's own host path (tests/golden/make_golden.py), and, where the reference library was
built here, directly against it on fresh inputs. Bit-exact throughout (single-thread sums)."""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _hier(g):
    L = int(g["h_levels"])
    a, p, r = [], [], []
    for l in range(L):
        def m(nm):
            sh = g[f"h_{nm}{l}_shape"]
            return O.Csr(int(sh[0]), int(sh[1]), g[f"h_{nm}{l}_rp"], g[f"h_{nm}{l}_ci"], g[f"h_{nm}{l}_va"])
        a.append(m("a"))
        if l + 1 < L:
            p.append(m("p"))
            r.append(m("r"))
    return a, p, r, g["h_coarse_inverse"]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_reference_goldens(path):
    g = np.load(path)
    n = int(g["n"])
    own, nei = g["owner"], g["neighbour"]
    for conv in (0, 1):
        up, lo, dg, dv = O.assemble(n, own, nei, g["flux"], g["gamma"], g["delta"], float(conv),
                                    diag=np.full(n, 0.5), div=np.zeros(n))
        t = f"asm_c{conv}_"
        for got, key in ((up, "upper"), (lo, "lower"), (dg, "diag"), (dv, "div")):
            assert np.array_equal(got, g[t + key]), key
    pat = O.build_pattern(n, own, nei)
    for got, key in ((pat.row_ptr, "pat_rp"), (pat.col, "pat_col"), (pat.diag_pos, "pat_diag"),
                     (pat.upper_pos, "pat_upper"), (pat.lower_pos, "pat_lower")):
        assert np.array_equal(got, g[key]), key
    a = O.ldu_to_csr(pat, g["ldu_diag"], g["ldu_upper"], g["ldu_lower"])
    h = O.Hierarchy(a)
    ga, gp, gr, gci = _hier(g)
    assert h.levels == len(ga)
    for l in range(h.levels):
        assert np.array_equal(h.a[l].va, ga[l].va) and np.array_equal(h.a[l].ci, ga[l].ci)
        if l + 1 < h.levels:
            assert np.array_equal(h.aggregates[l], g[f"h_agg{l}"])
            assert np.array_equal(h.p[l].va, gp[l].va) and np.array_equal(h.r[l].va, gr[l].va)
    assert np.array_equal(h.coarse_inverse, gci)
    rhs = g["rhs"]
    tol = 1e-10 * np.linalg.norm(rhs)
    x, st = O.amg_cg(ga, gp, gr, gci, rhs, abs_tol=tol, max_iterations=500)
    assert st["iterations"] == int(g["amgcg_iters"]) and np.array_equal(x, g["amgcg_x"])
    assert st["residual"] == float(g["amgcg_res"])
    assert np.array_equal(x, g["ds_x"]) and st["iterations"] == int(g["ds_iters"])
    for meth in (0, 1):
        x, st = O.krylov(a, rhs, method=meth, abs_tol=tol, max_iterations=5000)
        assert st["iterations"] == int(g[f"kry{meth}_iters"]) and np.array_equal(x, g[f"kry{meth}_x"])


@pytest.mark.skipif(O.ref() is None, reason="reference host library not built here")
def test_oracle_matches_reference_live():
    """Fresh random Poisson-like systems: oracle == the reference's compiled host path."""
    from cfd_b200 import workloads as W
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    case = W.graded(10, sigma=1.0, seed=99)
    for conv in (0.0, 1.0):
        r = O.ref_assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma, case.delta, conv)
        o = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma, case.delta, conv)
        assert all(np.array_equal(x, y) for x, y in zip(r, o))
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    pat = O.build_pattern(case.n, case.owner, case.neighbour)
    a = O.ldu_to_csr(pat, diag, up, lo)
    h = O.Hierarchy(a)
    tol = 1e-9 * np.linalg.norm(src)
    x1, s1 = O.amg_cg(h.a, h.p, h.r, h.coarse_inverse, src, abs_tol=tol)
    x2, s2 = O.ref_amg_cg(h.a, h.p, h.r, h.coarse_inverse, src, abs_tol=tol)
    assert s1 == s2 and np.array_equal(x1, x2)


def test_edge_cases_of_the_oracle():
    """Already converged input returns 0 iterations (test_gpu.cpp:93-109); empty face list."""
    # 10 x 10 five-point operator of test_gpu.cpp:14-58 with x = 1
    m = 10
    rp, ci, va = [0], [], []
    for j in range(m):
        for i in range(m):
            for (ii, jj, v) in ((i, j, 4.0), (i - 1, j, -1.0), (i + 1, j, -1.0), (i, j - 1, -1.0),
                                (i, j + 1, -1.0)):
                if 0 <= ii < m and 0 <= jj < m:
                    ci.append(ii + jj * m)
                    va.append(v)
            rp.append(len(ci))
    a = O.Csr(m * m, m * m, np.array(rp, np.int32), np.array(ci, np.int32), np.array(va))
    x = np.ones(m * m)
    b = a.matvec(x)
    x2, st = O.krylov(a, b, x=x, method=0, abs_tol=1e-12, max_iterations=10)
    assert st["converged"] and st["iterations"] == 0
    up, lo, dg, dv = O.assemble(3, [], [], [], [], [], 0.0)
    assert len(up) == 0 and np.array_equal(dg, np.zeros(3))
