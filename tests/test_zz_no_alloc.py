"""The allocation-free batch entry point, wind_integrate_batch_noalloc.

Callers that cannot allocate device memory -- codes whose device memory is
owned by another framework's allocator or budget -- get the same kernels as
wind_integrate_batch with the per-group counters in a static device array.
This checks, through the C ABI, that its results equal the allocating entry
point's (bit for bit: the kernels and their order of operations are the same)
on two calls in a row, so the shared array is cleared between calls, and that
a call over the group limit is rejected before anything runs.

Kept in a file that sorts last so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from wind_b200 import _capi, lib, networks as W

pytestmark = pytest.mark.gpu


def _groups():
    k96 = W.workload_katz96(96, atol=1e-8, rtol=1e-6)
    k96 = W.Workload(k96.net, k96.y0, 0.0, 1e9, k96.atol, k96.rtol, 1, 1, "katz96")
    out = [k96]
    out += W.workload_mixed(48, seed=11, sizes=(5, 16), fractions=(0.5, 0.5), dt=1e-5)
    nr = W.workload_nr(32)
    out.append(W.Workload(nr.net, nr.y0, 0.0, 0.005, nr.atol, nr.rtol, 1, 1, "nr"))
    return out


def test_noalloc_matches_allocating_batch_twice(cuda_device):
    groups = _groups()
    want = lib.integrate_batch(groups, "sie", "gje_f64", "device")
    for call in range(2):
        got = lib.integrate_batch(groups, "sie", "gje_f64", "device", noalloc=True)
        for (yw, sw, nw), (yg, sg, ng), wl in zip(want, got, groups):
            assert np.array_equal(yg, yw), f"call {call} {wl.label}: state differs"
            assert np.array_equal(sg, sw), f"call {call} {wl.label}: status differs"
            assert np.array_equal(ng, nw), f"call {call} {wl.label}: step counts differ"
            assert ng.min() > 0


def test_noalloc_rejects_too_many_groups(cuda_device):
    wlib = lib.load()
    n = _capi.NOALLOC_MAX_GROUPS + 1
    arr = (_capi.WindGroup * n)()
    o = lib.options()
    code = wlib.wind_integrate_batch_noalloc(C.byref(o), arr, n, None)
    assert code == _capi.WIND_ERR_ARGUMENT
