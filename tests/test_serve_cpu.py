"""Host-side pieces of serving that need no GPU."""
import ctypes as C

import numpy as np

from wind_b200 import networks as W, serve


def test_request_stream_is_seeded_and_shaped():
    a = serve.request_stream(20, seed=4, max_cells=1000)
    b = serve.request_stream(20, seed=4, max_cells=1000)
    assert [w.net.nsys for w in a] == [w.net.nsys for w in b]
    for w in a:
        assert 1 <= w.net.nsys <= 1000 and w.net.n_eq in W.MIXED_SIZES
        assert w.net.n_react == 10 * w.net.n_eq and 1e-2 <= w.tend <= 1e2
        assert w.net.species.max() < w.net.n_eq


def test_struct_layouts():
    # int32 x4 + int64 x2 + int32 x2
    assert C.sizeof(serve.WindServerConfig) == 40
    assert serve.WindRequest.y0.offset == C.sizeof(serve._capi.WindNetwork)
