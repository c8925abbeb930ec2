"""Runtime network plug-ins on the GPU: the reference-contract plug-in
sources that the reference's own c_baseline ran to make the golden vectors
(oracle/plugins/*.c) are compiled with NVRTC and integrated on the B200; the
results equal the reference's outputs bit for bit (GOLD controller) and the
oracle's with the DEVICE controller."""
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.test_plugin import source
from wind_b200 import lib, networks as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "golden.npz"))

CASES = {  # golden case -> (plug-in source, NVRTC options)
    "nr_sie": ("nr_test_gold.c", ""),
    "nr_rk2": ("nr_test_gold.c", ""),
    "katz96_t3_sie": ("katz96_tiled_gold.c", "-DNTILE=3"),
    "katz96_t3_rk2": ("katz96_tiled_gold.c", "-DNTILE=3"),
    "ma_n12_r30_lin_sie": ("mass_action_gold.c", "-DMA_N=12 -DMA_R=30 -DMA_LINEAR=1"),
    "ma_n8_r20_rk2": ("mass_action_gold.c", "-DMA_N=8 -DMA_R=20 -DMA_LINEAR=0"),
}


def golden_net(name):
    meta = GOLDEN[f"{name}/meta"]
    kind, n = int(meta[0]), int(meta[1])
    arr = {k: GOLDEN[f"{name}/{k}"] for k in ("constants", "rates", "species", "linear")
           if f"{name}/{k}" in GOLDEN.files}
    y0 = GOLDEN[f"{name}/y0"]
    return W.Network(kind, n, y0.shape[0], **arr), y0, meta


@pytest.mark.parametrize("name", sorted(CASES))
def test_plugin_reproduces_reference_output(cuda_device, name):
    net, y0, meta = golden_net(name)
    src, opts = CASES[name]
    packed = net.packed_constants()
    p = lib.Plugin(source(src), net.n_eq, packed.shape[1], opts)
    y = y0.copy()
    method = str(GOLDEN[f"{name}/method"])
    tot, st, _ = p.integrate(packed, y, meta[2], meta[3], meta[4], meta[5], method, "gold",
                             int(meta[6]))
    assert np.array_equal(y, GOLDEN[f"{name}/y"])
    assert tot == int(meta[7]) and st.max() == 0


@pytest.mark.parametrize("n,r", [(16, 160), (64, 96)])
def test_plugin_device_controller_matches_oracle(cuda_device, n, r):
    rng = np.random.default_rng(n)
    net = W.random_mass_action(rng, 6, n, r, 1e-3, 1e1)
    y0 = rng.uniform(0.0, 1.0, (6, n))
    y_o = y0.copy()
    tot_o, st_o, n_o = O.restated(net, y_o, 0.0, 1e-3, 1e-6, 1e-4, "sie", "device")
    packed = net.packed_constants()
    p = lib.Plugin(source("mass_action_gold.c"), n, packed.shape[1],
                   f"-DMA_N={n} -DMA_R={r} -DMA_LINEAR=0")
    y = y0.copy()
    tot, st, ns = p.integrate(packed, y, 0.0, 1e-3, 1e-6, 1e-4, "sie", "device")
    assert np.array_equal(y, y_o)
    assert np.array_equal(ns, n_o) and tot == tot_o


def test_plugin_failure_status(cuda_device):
    net, y0, meta = golden_net("katz96_t3_sie")
    p = lib.Plugin(source("katz96_tiled_gold.c"), 15, 10, "-DNTILE=3")
    y = y0.copy()
    y[1, 0] = np.nan
    _, st, _ = p.integrate(net.constants, y, meta[2], meta[3], meta[4], meta[5], "sie", "gold",
                           max_attempts=0)
    assert st[1] & 1 and (st[[0] + list(range(2, len(st)))] == 0).all()
    y = y0.copy()
    _, st, _ = p.integrate(net.constants, y, meta[2], meta[3], meta[4], meta[5], "sie", "gold",
                           max_attempts=2)
    assert (st & 2).all()
