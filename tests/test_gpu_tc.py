"""GPU parity of the tensor-core MIXED solver (WIND_SOLVER_MIXED_TC: the
blocked Gauss-Jordan inverse's rank-16 updates as tcgen05 kind::tf32 MMAs
with 3xTF32 operands, accumulator in tensor memory) for the CTA kernel's
mass-action sizes, at the mixed path's 1e-5 bar against the FP64 oracle."""
import os

import numpy as np
import pytest

from tests.helpers import mixed_err
from wind_b200 import _capi, lib, networks as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("n", [64, 157])
def test_mixed_tc_config4_classes_vs_oracle(cuda_device, n):
    """The N = 64 and N = 157 classes of the mixed-size batch (config-4
    fixture, oracle outputs) through wind_integrate with MIXED_TC."""
    g = np.load(os.path.join(HERE, "golden", "config4.npz"))
    y_ref, sens = g[f"n{n}_y"], g[f"n{n}_sensitive"]
    wl = W.workload_mixed_class(n, y_ref.shape[0], seed=3, dt=1.0, atol=1e-8, rtol=1e-6)
    y = wl.y0.copy()
    tot, st, ns = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "mixed_tc",
                                "gold")
    ok = ~sens
    err = mixed_err(y[ok], y_ref[ok], wl.atol)
    assert err <= 1e-5, f"N={n}: max rel err {err:.3e} vs the FP64 oracle"
    assert (st & ~_capi.SYS_REFINE_FALLBACK).max() == 0


@pytest.mark.parametrize("n", [40, 100, 130, 176])
def test_mixed_tc_edge_sizes_vs_lu_f64(cuda_device, n):
    """Sizes that are not multiples of 16 (a partial last panel), above 128
    (rows split between tensor and CUDA cores) and near the largest size
    whose matrix and operand staging fit in shared memory together,
    against the plain FP64 path on the same systems (the FP64 LU is checked
    against the oracle by the configuration tests)."""
    wl = W.workload_mixed_class(n, 64, seed=41, dt=1e-4, atol=1e-8, rtol=1e-6)
    y, y_lu = wl.y0.copy(), wl.y0.copy()
    _, st, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "mixed_tc", "gold")
    lib.integrate(wl.net, y_lu, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "lu_f64", "gold")
    err = mixed_err(y, y_lu, wl.atol)
    assert err <= 1e-5, f"N={n}: max rel err {err:.3e} vs LU_F64"
    assert (st & ~_capi.SYS_REFINE_FALLBACK).max() == 0


def test_mixed_tc_matches_simt_mixed_closely(cuda_device):
    """Same systems, MIXED (CUDA-core updates) and MIXED_TC: both refine to
    the FP64 solution, so they agree far inside the 1e-5 bar."""
    wl = W.workload_mixed_class(64, 300, seed=42, dt=1e-2)
    a, b = wl.y0.copy(), wl.y0.copy()
    lib.integrate(wl.net, a, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "mixed", "gold")
    lib.integrate(wl.net, b, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "mixed_tc", "gold")
    fin = np.isfinite(a).all(axis=1) & np.isfinite(b).all(axis=1)
    assert fin.mean() > 0.95
    assert mixed_err(b[fin], a[fin], wl.atol) <= 1e-6


def test_mixed_tc_unsupported_elsewhere(cuda_device):
    # above ~190 species the FP32 matrix and the operand staging no longer
    # fit in one CTA's shared memory together
    huge = W.workload_mixed_class(220, 2, seed=45)
    with pytest.raises(lib.WindError) as e:
        lib.integrate(huge.net, huge.y0.copy(), 0.0, 1e-6, 1e-8, 1e-6, "sie", "mixed_tc", "gold")
    assert e.value.code == _capi.WIND_ERR_UNSUPPORTED
    small = W.workload_mixed_class(16, 4, seed=43)
    with pytest.raises(lib.WindError) as e:
        lib.integrate(small.net, small.y0.copy(), 0.0, 1e-3, 1e-8, 1e-6, "sie", "mixed_tc", "gold")
    assert e.value.code == _capi.WIND_ERR_UNSUPPORTED
    big = W.workload_mixed_class(64, 4, seed=44)
    with pytest.raises(lib.WindError) as e:
        lib.integrate_batch([big], method="sie", solver="mixed_tc", controller="gold")
    assert e.value.code == _capi.WIND_ERR_UNSUPPORTED
