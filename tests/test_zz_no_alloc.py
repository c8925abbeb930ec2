"""The allocation-free batch entry point, wind_integrate_batch_noalloc.

Callers that cannot allocate device memory -- codes whose device memory is
owned by another framework's allocator or budget -- get the same kernels as
wind_integrate_batch with the per-group counters in a static device array.
This checks, through the C ABI, that its results equal the allocating entry
point's (bit for bit: the kernels and their order of operations are the same)
on two calls in a row, so the shared array is cleared between calls; that the
CTA-per-system path (N > 32 with the matrix in shared memory) runs without
allocating and agrees bit for bit too; and that a call over the group limit,
or with a group that would need global matrix scratch, is rejected before
anything runs, leaving every group's state untouched.

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


def _cta_groups():
    """A mass-action N = 64 group (CTA kernel, matrix in shared memory) beside
    a small team-kernel group."""
    big = W.workload_mixed(40, seed=41, sizes=(64,), fractions=(1.0,), dt=2e-6, atol=1e-6,
                           rtol=1e-4)[0].subset(slice(0, 4))
    small = W.workload_mixed(40, seed=42, sizes=(16,), fractions=(1.0,), dt=1e-5)[0].subset(slice(0, 8))
    return [big, small]


def test_noalloc_cta_path_matches_allocating_batch(cuda_device):
    groups = _cta_groups()
    for solver in ("lu_f64", "mixed"):
        want = lib.integrate_batch(groups, "sie", solver, "device")
        for call in range(2):
            got = lib.integrate_batch(groups, "sie", solver, "device", noalloc=True)
            for (yw, sw, nw), (yg, sg, ng), wl in zip(want, got, groups):
                assert np.array_equal(yg, yw), f"{solver} call {call} N={wl.net.n_eq}: state differs"
                assert np.array_equal(sg, sw) and np.array_equal(ng, nw)
                assert ng.min() > 0


def test_noalloc_refuses_global_scratch_before_any_launch(cuda_device):
    import torch

    # Gauss-Jordan at N = 64 keeps its matrix pair in global scratch: the call
    # must refuse the whole batch and leave the earlier group untouched
    groups = _cta_groups()[::-1]
    dg = [lib.DeviceGroup(wl, cuda_device) for wl in groups]
    before = [g.y.clone() for g in dg]
    arr = (_capi.WindGroup * len(dg))(*[g.struct() for g in dg])
    o = lib.options("sie", "gje_f64", "device")
    s = torch.cuda.current_stream(cuda_device).cuda_stream
    code = lib.load().wind_integrate_batch_noalloc(C.byref(o), arr, len(dg), s)
    torch.cuda.synchronize(cuda_device)
    assert code == _capi.WIND_ERR_UNSUPPORTED
    for g, y0 in zip(dg, before):
        assert torch.equal(g.y, y0)
        assert int(g.nsteps.abs().sum()) == 0


def test_noalloc_rejects_bad_options(cuda_device):
    wlib = lib.load()
    groups = _cta_groups()
    dg = [lib.DeviceGroup(wl, cuda_device) for wl in groups]
    arr = (_capi.WindGroup * len(dg))(*[g.struct() for g in dg])
    for field, bad in (("method", 7), ("solver", 9), ("controller", -1)):
        o = lib.options()
        setattr(o, field, bad)
        assert wlib.wind_integrate_batch_noalloc(C.byref(o), arr, len(dg), None) == _capi.WIND_ERR_ARGUMENT
        assert wlib.wind_integrate_batch(C.byref(o), arr, len(dg), None) == _capi.WIND_ERR_ARGUMENT
