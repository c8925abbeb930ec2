"""Serving on the GPU: continuous batching, admission, and "same result alone
and in the mix"."""
import numpy as np
import pytest

from wind_b200 import lib, networks as W, serve

pytestmark = pytest.mark.gpu


def _requests():
    reqs = serve.request_stream(14, seed=4, max_cells=48, sizes=(5, 16, 32, 64),
                                fractions=(0.4, 0.3, 0.2, 0.1), dt_range=(1e-6, 1e-5))
    k = W.workload_katz96(40, seed=8, atol=1e-8, rtol=1e-6)
    reqs.append(W.Workload(k.net, k.y0, 0.0, 1e10, k.atol, k.rtol, 1, 1, "katz96"))
    return reqs


def test_results_same_alone_and_in_mix(cuda_device):
    reqs = _requests()
    with serve.Server(solver="lu_f64", max_inflight=3) as srv:
        ids = [srv.submit(wl) for wl in reqs]
        res = [srv.poll(i, 300.0) for i in ids]
        stats = srv.stats()
    assert stats["completed"] == len(reqs)
    assert stats["launches"] < len(reqs)  # requests were merged into batches
    for r, wl in zip(res, reqs):
        y = wl.y0.copy()
        _, st, ns = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "lu_f64")
        assert np.array_equal(r.y, y), wl.label
        assert np.array_equal(r.nsteps, ns) and np.array_equal(r.status, st)
        assert r.latency_s > 0


def test_admission_by_footprint(cuda_device):
    """A budget below any request's footprint admits one request at a time."""
    reqs = _requests()[:5]
    with serve.Server(solver="lu_f64", hbm_budget_bytes=1, max_inflight=4) as srv:
        ids = [srv.submit(wl) for wl in reqs]
        res = [srv.poll(i, 300.0) for i in ids]
        stats = srv.stats()
    assert stats["launches"] == len(reqs) and stats["resident_bytes"] == 0
    assert all(r.status.max() == 0 for r in res)


def test_poll_timeout_and_busy(cuda_device):
    slow = W.workload_katz96(8192, seed=9, atol=1e-8, rtol=1e-6)
    quick = _requests()[0]
    with serve.Server(solver="lu_f64", hbm_budget_bytes=1, max_waiting=1) as srv:
        a = srv.submit(slow)
        b = srv.submit(quick)          # waits: the budget is taken
        with pytest.raises(lib.WindError) as e:
            srv.submit(quick)          # max_waiting reached
        assert e.value.code == 6
        assert srv.poll(a, 0.0) is None  # not done yet
        assert srv.poll(a, 300.0) is not None
        assert srv.poll(b, 300.0) is not None
