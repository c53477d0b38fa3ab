"""Request server (extension) on the GPU: requests of uneven size (3D 7- and
13-point Laplacians with Gaussian wells, Chebyshev and LOBPCG, different nev and
tol) admitted as slots and device memory free up.

  * each result is bit-identical to the same solve run alone through fe_solve
    (the server runs the same device path on its own stream);
  * with four slots and room in the budget, requests overlap in time; with a
    budget smaller than any request, they run one at a time in arrival order;
  * a wait with a zero timeout on a running request reports FE_PENDING;
  * an out-of-range nev fails at submission; a solve that fails in a worker
    reports its error through wait.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def requests():
    from fasteig_b200 import matrices as M
    out = []
    specs = [(14, "star1", "Chebyshev", 12, 1e-8), (12, "star2", "LOBPCG", 6, 1e-8),
             (16, "star1", "Chebyshev", 20, 1e-6), (10, "star2", "Chebyshev", 8, 1e-8),
             (13, "star1", "LOBPCG", 5, 1e-6), (15, "star2", "Chebyshev", 16, 1e-8)]
    for i, (side, st, solver, nev, tol) in enumerate(specs):
        H = M.laplacian_wells(side, wells=6, seed=10 + i, stencil=st)
        out.append((H, solver, nev, tol))
    return out


def options(solver, nev, tol, n):
    from fasteig_b200 import fasteig_options
    o = fasteig_options(n)
    kv = dict(solver=solver, nev=nev, which="SR", tol=tol, maxiter=800, seed=3, degree=10)
    if solver == "Chebyshev":
        kv.update(bounds="ritz", amplification=1e6)
    for k, v in kv.items():
        assert o.set(k, v), k
    return o


def test_server_results_same_alone_and_in_the_mix():
    from fasteig_b200 import CsrMatrix, Server, fasteig_problem
    reqs = requests()
    mats = [CsrMatrix(H.n, H.rowptr, H.colind, H.values) for H, *_ in reqs]
    alone = []
    for (H, solver, nev, tol), A in zip(reqs, mats):
        p = fasteig_problem(A, solver=solver)
        p.solve(options(solver, nev, tol, H.n), want_vectors=False)
        alone.append(p)
    with Server(slots=4) as srv:
        ids = [srv.submit(A, options(solver, nev, tol, H.n))
               for (H, solver, nev, tol), A in zip(reqs * 2, mats * 2)]
        results = [srv.wait(i) for i in ids]
    for k, r in enumerate(results):
        p = alone[k % len(reqs)]
        assert np.array_equal(r["eigenvalues"], p.eigenvalues()), k
        assert np.array_equal(r["residual_norms"], p.residual_norms()), k
        assert r["iterations"] == p.last_iterations()
        tol = reqs[k % len(reqs)][3]
        assert np.all(r["residual_norms"] <= tol)
    # Some requests ran at the same time.
    spans = sorted((r["start_s"], r["end_s"]) for r in results)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))


def test_server_budget_serializes_admission():
    from fasteig_b200 import CsrMatrix, Server
    reqs = requests()[:4]
    mats = [CsrMatrix(H.n, H.rowptr, H.colind, H.values) for H, *_ in reqs]
    with Server(slots=4, memory_budget_bytes=1) as srv:
        ids = [srv.submit(A, options(solver, nev, tol, H.n))
               for (H, solver, nev, tol), A in zip(reqs, mats)]
        results = [srv.wait(i) for i in ids]
    # Nothing fits a 1-byte budget, so each request runs alone, in arrival order.
    for a, b in zip(results, results[1:]):
        assert b["start_s"] >= a["end_s"] - 1e-6
        assert b["queued_s"] > 0.0
    assert all(r["admitted_bytes"] > 1 for r in results)


def test_server_pending_and_bad_options():
    from fasteig_b200 import CsrMatrix, FastEigError, Server, fasteig_options
    from fasteig_b200 import matrices as M
    H = M.laplacian_wells(24, wells=8, seed=1)
    A = CsrMatrix(H.n, H.rowptr, H.colind, H.values)
    with Server(slots=1) as srv:
        rid = srv.submit(A, options("LOBPCG", 24, 1e-10, H.n))
        assert srv.wait(rid, timeout=0.0) is None
        r = srv.wait(rid)
        assert r is not None and len(r["eigenvalues"]) == 24
        bad = fasteig_options(H.n)
        bad.set("nev", 4)
        with pytest.raises(FastEigError, match="solver not available"):
            srv.wait(srv.submit(A, bad, solver="NoSuchSolver"))
        bad2 = fasteig_options(H.n)
        bad2.set("nev", H.n + 1)
        with pytest.raises(FastEigError, match="nev"):
            srv.submit(A, bad2, solver="Chebyshev")


def test_server_grouped_lanes():
    """Requests with group=1 run in grouped lanes (one per width and degree): they
    join a group between cycles, advance together, and each result is the one the
    same problem gets alone in a group (bit-identical for same-stencil groups,
    1e-11 otherwise), meeting tol. Worker-slot requests run beside them."""
    from fasteig_b200 import CsrMatrix, Server, grouped_chebyshev
    from fasteig_b200 import matrices as M
    specs = [(13, "star1", 10), (12, "star1", 12), (14, "star1", 8), (11, "star1", 14),
             (12, "star2", 20), (13, "star2", 24)]
    Hs = [M.laplacian_wells(s, wells=6, seed=50 + i, stencil=st) for i, (s, st, _) in enumerate(specs)]
    mats = [CsrMatrix(H.n, H.rowptr, H.colind, H.values) for H in Hs]

    def gopts(H, nev):
        o = options("Chebyshev", nev, 1e-8, H.n)
        assert o.set("group", 1)
        return o

    def gopts_any(k, H, nev):
        o = gopts(H, nev)
        if k % 2 == 1:
            assert o.set("precision", "mixed")  # FP32-filter group, then the FP64 one
        return o

    gopts_k = [gopts_any(k, H, nev) for k, (H, (_, _, nev)) in enumerate(zip(Hs, specs))]
    alone = [grouped_chebyshev([A], [o])[0][0] for A, o in zip(mats, gopts_k)]
    lob = requests()[1]
    lob_A = CsrMatrix(lob[0].n, lob[0].rowptr, lob[0].colind, lob[0].values)
    with Server(slots=2) as srv:
        ids = [srv.submit(A, o) for A, o in zip(mats, gopts_k)]
        lid = srv.submit(lob_A, options("LOBPCG", lob[2], lob[3], lob[0].n))
        results = [srv.wait(i) for i in ids]
        lres = srv.wait(lid)
        st = srv.stats()
    assert np.all(lres["residual_norms"] <= lob[3])
    assert st["grouped_served"] == len(specs)
    assert st["lanes"] == 2  # widths 32 and 64 at degree 10
    assert st["max_group_members"] >= 2
    assert st["graph_replays"] > 0
    for k, (r, a) in enumerate(zip(results, alone)):
        assert np.all(r["residual_norms"] <= 1e-8), k
        if specs[k][1] == "star1" and specs[k][2] <= 16:  # the all-7-point width-32 lane
            assert np.array_equal(r["eigenvalues"], a["eigenvalues"]), k
            assert r["iterations"] == a["iterations"]
        else:
            np.testing.assert_allclose(r["eigenvalues"], a["eigenvalues"], rtol=1e-11,
                                       atol=1e-12)
    spans = sorted((r["start_s"], r["end_s"]) for r in results)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))


def test_server_destroy_with_queued_grouped_requests():
    """Destroying a server while grouped-lane requests wait (a 1-byte budget admits one
    request at a time) drops the queued ones and returns once the running one is done."""
    import time
    from fasteig_b200 import CsrMatrix, Server
    from fasteig_b200 import matrices as M
    Hs = [M.laplacian_wells(11 + i, wells=4, seed=80 + i) for i in range(4)]
    mats = [CsrMatrix(H.n, H.rowptr, H.colind, H.values) for H in Hs]
    srv = Server(slots=1, memory_budget_bytes=1)
    for H, A in zip(Hs, mats):
        o = options("Chebyshev", 8, 1e-8, H.n)
        assert o.set("group", 1)
        srv.submit(A, o)
    t0 = time.perf_counter()
    srv.close()
    assert time.perf_counter() - t0 < 60.0
