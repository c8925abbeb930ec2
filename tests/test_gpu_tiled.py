"""Tiled builtin networks (the Precompiler's Ntile tiling,
python/ode_systems/ode_base.py:86-88, 219-281) on the GPU.

* the golden tiled Katz96 cases (made by the reference's own c_baseline on
  the tiled plug-in, tiles in different states so tile 0's electron density
  couples them) are reproduced bit for bit by the Gauss-Jordan path;
* tiled systems of every team shape (Ntile 2 .. 64, one or two tiles per
  lane) match the oracle's full N x N elimination bit for bit with both
  controllers, SIE and RK2;
* identical tiles at the largest Ntile integrate exactly as the untiled
  network (a size-independent property);
* LU_F64 and MIXED stay within their tolerances of the oracle;
* the drop-in cudaIntegrateSystem takes Nequations_per_system = 5 Ntile.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.helpers import mixed_err
from wind_b200 import lib, networks as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "golden.npz"))
TILED = sorted({k.split("/")[0] for k in GOLDEN.files if "_t" in k.split("/")[0]})


def varied_tiles(kind: int, nsys: int, ntile: int, seed: int):
    """A tiled workload whose tiles start in different states."""
    rng = np.random.default_rng(seed)
    if kind == W.NET_KATZ96:
        base = W.workload_katz96(nsys, seed=seed)
        y0 = np.tile(base.y0, (1, ntile))
        for t in range(1, ntile):
            x = rng.uniform(0.0, 1.0, nsys)
            h = rng.uniform(0.0, W.Y_HELIUM, nsys)
            y0[:, 5 * t:5 * t + 5] = np.stack([x, 1 - x, h, W.Y_HELIUM - h, np.zeros(nsys)], 1)
        return W.Workload(W.tile_network(base.net, ntile), y0, 0.0, 1e10, 1e-8, 1e-6, 1, 1)
    net = W.nr_test(nsys) if kind == W.NET_NR_TEST else W.stifftrig(nsys)
    y0 = rng.uniform(0.5, 1.5, (nsys, 2 * ntile))
    tend = 0.01 if kind == W.NET_NR_TEST else 0.2
    return W.Workload(W.tile_network(net, ntile), y0, 0.0, tend, 1e-8, 1e-6, 1, 1)


@pytest.mark.parametrize("name", TILED)
def test_tiled_golden_bit_exact(cuda_device, name):
    meta = GOLDEN[f"{name}/meta"]
    kind, n = int(meta[0]), int(meta[1])
    net = W.Network(kind, n, GOLDEN[f"{name}/y0"].shape[0], constants=GOLDEN[f"{name}/constants"])
    y = GOLDEN[f"{name}/y0"].copy()
    method = str(GOLDEN[f"{name}/method"])
    tot, st, _ = lib.integrate(net, y, meta[2], meta[3], meta[4], meta[5], method, "gje_f64",
                               "gold", int(meta[6]))
    assert np.array_equal(y, GOLDEN[f"{name}/y"])
    assert tot == int(meta[7]) and st.max() == 0


# (network, Ntile, interval scale): the oracle eliminates the full N x N
# matrix, N^3 per substep, so the large systems take short intervals;
# Katz96 beyond 32 tiles is covered by the identical-tiles property below
@pytest.mark.parametrize("kind,ntile,scale", [(W.NET_KATZ96, 2, 1.0), (W.NET_KATZ96, 7, 1.0),
                                              (W.NET_NR_TEST, 5, 1.0), (W.NET_NR_TEST, 64, 1e-3),
                                              (W.NET_STIFFTRIG, 16, 0.01)])
@pytest.mark.parametrize("method,controller", [("sie", "gold"), ("sie", "device"),
                                               ("rk2", "device")])
def test_tiled_gje_matches_oracle(cuda_device, kind, ntile, scale, method, controller):
    wl = varied_tiles(kind, 2 if ntile > 32 else 5, ntile, seed=ntile)
    tend = wl.tend * scale * (1.0 if method == "sie" else 1e-4)
    y_o, y = wl.y0.copy(), wl.y0.copy()
    tot_o, st_o, n_o = O.restated(wl.net, y_o, wl.tnow, tend, wl.atol, wl.rtol, method, controller)
    tot, st, n = lib.integrate(wl.net, y, wl.tnow, tend, wl.atol, wl.rtol, method, "gje_f64",
                               controller)
    assert np.array_equal(y, y_o), f"max diff {np.nanmax(np.abs(y - y_o))}"
    assert np.array_equal(n, n_o) and tot == tot_o
    assert np.array_equal(st, st_o)


@pytest.mark.parametrize("ntile", [32, 33, 64])
def test_tiled_identical_tiles_equal_untiled(cuda_device, ntile):
    base = W.workload_katz96(300, seed=11, atol=1e-8, rtol=1e-6)
    y1 = base.y0.copy()
    _, _, n1 = lib.integrate(base.net, y1, 0.0, 1e12, 1e-8, 1e-6, "sie", "gje_f64", "gold")
    t = W.tile_workload(base, ntile)
    yt = t.y0.copy()
    _, st, nt = lib.integrate(t.net, yt, 0.0, 1e12, 1e-8, 1e-6, "sie", "gje_f64", "gold")
    assert np.array_equal(yt, np.tile(y1, (1, ntile)))
    assert np.array_equal(nt, n1) and st.max() == 0


@pytest.mark.parametrize("solver,bar", [("lu_f64", 1e-10), ("mixed", 1e-5)])
def test_tiled_lu_and_mixed_within_tolerance(cuda_device, solver, bar):
    wl = varied_tiles(W.NET_KATZ96, 16, 6, seed=5)
    y_o, y = wl.y0.copy(), wl.y0.copy()
    O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "gold")
    _, st, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver, "gold")
    assert mixed_err(y, y_o, wl.atol) <= bar
    assert (st & ~8).max() == 0


def test_tiled_limits(cuda_device):
    net = W.Network(W.NET_KATZ96, 5 * 65, 1, constants=np.ones((1, 10)))
    with pytest.raises(lib.WindError) as e:
        lib.integrate(net, np.zeros((1, 5 * 65)), 0.0, 1.0, 1e-8, 1e-6)
    assert e.value.code == lib._capi.WIND_ERR_UNSUPPORTED
    net = W.Network(W.NET_KATZ96, 12, 1, constants=np.ones((1, 10)))
    with pytest.raises(lib.WindError) as e:
        lib.integrate(net, np.zeros((1, 12)), 0.0, 1.0, 1e-8, 1e-6)
    assert e.value.code == lib._capi.WIND_ERR_ARGUMENT


def test_tiled_drop_in(cuda_device):
    """The drop-in cudaIntegrateSystem with Nequations_per_system = 5 Ntile
    (the reference's Ntile build), float32 in and out, the reference GPU
    kernel's controller: equal to the oracle on the same float inputs."""
    wl = varied_tiles(W.NET_KATZ96, 6, 4, seed=3)
    c32 = wl.net.constants.astype(np.float32)
    y32 = wl.y0.astype(np.float32)
    fn = lib.legacy("katz96", "sie")
    yy = y32.copy()
    tot = fn(0.0, 1e10, 1, c32.ctypes.data, yy.ctypes.data, 6, 20, 1e-8, 1e-6)
    net = W.Network(W.NET_KATZ96, 20, 6, constants=c32.astype(np.float64))
    y_o = y32.astype(np.float64)
    tot_o, _, _ = O.restated(net, y_o, float(np.float32(0.0)), float(np.float32(1e10)),
                             float(np.float32(1e-8)), float(np.float32(1e-6)), "sie", "device")
    assert tot == tot_o
    assert np.array_equal(yy, y_o.astype(np.float32))


def test_tiled_in_batch_and_output_steps(cuda_device):
    wl = varied_tiles(W.NET_KATZ96, 8, 3, seed=9)
    y_o = wl.y0.copy()
    O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "device")
    other = W.workload_mixed_class(16, 4, dt=1e-3)
    out = lib.integrate_batch([wl, other], solver="gje_f64", controller="device")
    assert np.array_equal(out[0][0], y_o)
    y = wl.y0.copy()
    over, steps = lib.integrate_output_steps(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, 2,
                                             solver="gje_f64")
    assert over.shape == (3, 8, 15) and steps.shape == (2,)
    assert np.array_equal(over[0], wl.y0)
