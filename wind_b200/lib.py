"""Python host layer over the native C ABI (include/wind.h).

The native library is the product: this module only marshals arrays and
checks status codes.  There is no CPU fallback -- if ``libwind.so`` is missing
or no GPU is visible, calls raise.

Entry points mirror the reference's caller (python/ode_systems/ode_base.py):
* :func:`integrate` -- one call over [tnow, tend] for a batch of systems
  (``runCudaIntegrator``, ode_base.py:441-469, with FP64 state);
* :func:`integrate_output_steps` -- the outer loop over output intervals
  (``runIntegratorOutput``, ode_base.py:315-397), kept on the device;
* :func:`integrate_batch` -- several network shapes in one persistent launch;
* :func:`legacy` -- the drop-in ``cudaIntegrateSystem`` libraries.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _capi
from .networks import Network

HERE = os.path.dirname(os.path.abspath(__file__))
# WIND_LIBDIR selects another build of the libraries (e.g. an experiment)
LIBDIR = os.environ.get("WIND_LIBDIR", os.path.join(HERE, "lib"))

_lib = None


class WindError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = {0: "ok", 1: "invalid argument", 2: "unsupported configuration",
               3: "CUDA runtime error", 4: "out of device memory", 5: "timed out",
               6: "admission refused", 7: "unknown request"}.get(code, f"status {code}")
        super().__init__(f"{what}: {msg}" if what else msg)


def library_path() -> str:
    return os.path.join(LIBDIR, "libwind.so")


def load() -> C.CDLL:
    """Load libwind.so (raises FileNotFoundError if it was not built)."""
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built: run `python -m wind_b200.build`")
        _lib = _capi.declare_api(C.CDLL(path))
    return _lib


def options(method="sie", solver="gje_f64", controller="device", spec_width=0,
            max_attempts=0, timeout_s=0.0) -> _capi.WindOptions:
    o = _capi.WindOptions()
    o.method = _capi.METHODS[method]
    o.solver = _capi.SOLVERS[solver]
    o.controller = _capi.CONTROLLERS[controller]
    o.spec_width = int(spec_width)
    o.max_attempts = int(max_attempts)
    o.timeout_s = float(timeout_s)
    return o


def _is_torch(a) -> bool:
    return hasattr(a, "data_ptr") and hasattr(a, "is_cuda")


def _check(code: int, what: str):
    if code != _capi.WIND_OK:
        detail = ""
        if code == _capi.WIND_ERR_CUDA:
            detail = " (" + load().wind_last_error().decode() + ")"
        raise WindError(code, what + detail)


def integrate(net: Network, y, tnow: float, tend: float, atol: float, rtol: float,
              method: str = "sie", solver: str = "gje_f64", controller: str = "device",
              n_integration_steps: int = 1, spec_width: int = 0, max_attempts: int = 0,
              timeout_s: float = 0.0, device_arrays: Optional[dict] = None,
              stream: Optional[int] = None, want_status: bool = True):
    """Integrate every system of ``net`` from tnow to tend.

    ``y`` is either a host ``float64 [S, N]`` NumPy array (copied in and out,
    updated in place) or a CUDA ``torch.float64`` tensor, in which case
    ``device_arrays`` must hold the network arrays as CUDA tensors too
    (keys ``constants``, ``rates``, ``species``, ``linear``) and the call is
    asynchronous on ``stream`` except for the returned step total.

    Returns ``(total_substeps, status, nsteps)``: per-system status bits and
    substep counts (host NumPy arrays for host calls, CUDA tensors otherwise).
    """
    lib = load()
    o = options(method, solver, controller, spec_width, max_attempts, timeout_s)
    total = C.c_int64(0)
    if _is_torch(y):
        import torch
        assert y.dtype == torch.float64 and y.is_contiguous()
        device_arrays = device_arrays or {}
        for k in ("constants", "rates", "species", "linear"):
            if getattr(net, k) is not None:
                a = device_arrays.get(k)
                if a is None or not getattr(a, "is_cuda", False):
                    raise ValueError(f"device call: network array '{k}' must be a CUDA tensor")
        ns = _capi.network_struct(net, device_arrays)
        status = torch.zeros(net.nsys, dtype=torch.int32, device=y.device) if want_status else None
        nsteps = torch.zeros(net.nsys, dtype=torch.int64, device=y.device) if want_status else None
        code = lib.wind_integrate(C.byref(o), C.byref(ns), tnow, tend, n_integration_steps,
                                  y.data_ptr(), net.nsys, atol, rtol,
                                  status.data_ptr() if want_status else None,
                                  nsteps.data_ptr() if want_status else None,
                                  C.byref(total), _capi.MEM_DEVICE,
                                  stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        _check(code, "wind_integrate")
        return int(total.value), status, nsteps
    assert isinstance(y, np.ndarray) and y.dtype == np.float64 and y.flags["C_CONTIGUOUS"]
    ns = _capi.network_struct(net)
    status = np.zeros(net.nsys, np.int32) if want_status else None
    nsteps = np.zeros(net.nsys, np.int64) if want_status else None
    code = lib.wind_integrate(C.byref(o), C.byref(ns), tnow, tend, n_integration_steps,
                              y.ctypes.data, net.nsys, atol, rtol,
                              status.ctypes.data if want_status else None,
                              nsteps.ctypes.data if want_status else None,
                              C.byref(total), _capi.MEM_HOST, stream)
    _check(code, "wind_integrate")
    return int(total.value), status, nsteps


def integrate_output_steps(net: Network, y: np.ndarray, tnow: float, tend: float,
                           atol: float, rtol: float, n_output_steps: int,
                           n_integration_steps: int = 1, method="sie", solver="gje_f64",
                           controller="device", spec_width=0):
    """The reference's outer loop (ode_base.py:338-378) on the device: returns
    ``(equations_over_time [n_output_steps+1, S, N], nsteps [n_output_steps])``
    and leaves the final state in ``y``."""
    lib = load()
    o = options(method, solver, controller, spec_width)
    ns = _capi.network_struct(net)
    out = np.zeros((n_output_steps + 1,) + y.shape, np.float64)
    steps = np.zeros(n_output_steps, np.int64)
    code = lib.wind_integrate_output_steps(C.byref(o), C.byref(ns), tnow, tend,
                                           n_integration_steps, n_output_steps, y.ctypes.data,
                                           net.nsys, atol, rtol, out.ctypes.data,
                                           steps.ctypes.data, _capi.MEM_HOST, None)
    _check(code, "wind_integrate_output_steps")
    return out, steps


def integrate_global(net: Network, y: np.ndarray, tnow: float, tend: float, atol: float,
                     rtol: float, solver: str = "gje_f64", n_integration_steps: int = 1):
    """The SIE_host variant (cuda/SIE_host/harness_kernel.cu:248-425): one
    step shared by all systems, refined for all when any system fails.
    ``y`` (host float64 [S, N]) is updated in place; returns
    ``(total_substeps, t_reached)``."""
    lib = load()
    assert isinstance(y, np.ndarray) and y.dtype == np.float64 and y.flags["C_CONTIGUOUS"]
    o = options("sie", solver, "gold")
    ns = _capi.network_struct(net)
    total, t_reached = C.c_int64(0), C.c_double(0.0)
    code = lib.wind_integrate_global(C.byref(o), C.byref(ns), tnow, tend, n_integration_steps,
                                     y.ctypes.data, net.nsys, atol, rtol, C.byref(total),
                                     C.byref(t_reached), _capi.MEM_HOST, None)
    _check(code, "wind_integrate_global")
    return int(total.value), float(t_reached.value)


def legacy_host(network: str):
    """The drop-in ``cudaIntegrateSIE`` of ``lib/<network>/sie_host.so``, bound
    by the reference's mangled name (python/wind_harness.py:27-28)."""
    path = os.path.join(LIBDIR, network, "sie_host.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built")
    fn = getattr(C.CDLL(path), "_Z16cudaIntegrateSIEffiPfS_iiff")
    fn.argtypes = [C.c_float, C.c_float, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                   C.c_float, C.c_float]
    fn.restype = C.c_int
    return fn


class DeviceGroup:
    """One workload's arrays on the device, kept alive for a batch call."""

    def __init__(self, wl, device):
        import torch
        self.wl = wl
        net = wl.net
        self.arrays = {k: torch.from_numpy(np.ascontiguousarray(getattr(net, k))).to(device)
                       for k in ("constants", "rates", "species", "linear")
                       if getattr(net, k) is not None}
        self.y = torch.from_numpy(np.ascontiguousarray(wl.y0)).to(device)
        self.status = torch.zeros(net.nsys, dtype=torch.int32, device=device)
        self.nsteps = torch.zeros(net.nsys, dtype=torch.int64, device=device)

    def struct(self) -> _capi.WindGroup:
        wl = self.wl
        g = _capi.WindGroup()
        g.net = _capi.network_struct(wl.net, self.arrays)
        g.y = self.y.data_ptr()
        g.nsys = wl.net.nsys
        g.tnow, g.tend = wl.tnow, wl.tend
        g.n_integration_steps = wl.n_integration_steps
        g.atol, g.rtol = wl.atol, wl.rtol
        g.sys_status = self.status.data_ptr()
        g.sys_nsteps = self.nsteps.data_ptr()
        return g


def integrate_batch(workloads, method="sie", solver="gje_f64", controller="device",
                    spec_width=0, noalloc=False, device=None, stream=None):
    """Integrate several workloads (one group each) in one batch call.
    Returns a list of ``(y, status, nsteps)`` host arrays, one per workload.
    ``noalloc`` selects wind_integrate_batch_noalloc."""
    import torch
    lib = load()
    device = device or torch.device("cuda", torch.cuda.current_device())
    groups = [DeviceGroup(wl, device) for wl in workloads]
    arr = (_capi.WindGroup * max(1, len(groups)))(*[g.struct() for g in groups])
    o = options(method, solver, controller, spec_width)
    s = stream if stream is not None else torch.cuda.current_stream(device).cuda_stream
    fn = lib.wind_integrate_batch_noalloc if noalloc else lib.wind_integrate_batch
    code = fn(C.byref(o), arr, len(groups), s)
    _check(code, fn.__name__)
    torch.cuda.synchronize(device)
    return [(g.y.cpu().numpy(), g.status.cpu().numpy(), g.nsteps.cpu().numpy()) for g in groups]


def legacy(network: str, method: str):
    """The drop-in ``cudaIntegrateSystem`` of ``lib/<network>/<method>.so``,
    bound by the reference's mangled name (python/wind_harness.py:32-40)."""
    path = os.path.join(LIBDIR, network, f"{method}.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built")
    fn = getattr(C.CDLL(path), "_Z19cudaIntegrateSystemffiPfS_iiff")
    fn.argtypes = [C.c_float, C.c_float, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                   C.c_float, C.c_float]
    fn.restype = C.c_int
    return fn


class Plugin:
    """A runtime network compiled with NVRTC (wind_plugin_create): ``source``
    is the network in the reference's host plug-in contract
    (cuda/include/ode_gold.h:1-12; calculate_dydt / calculate_jacobian over
    ``float``, run in FP64).  ``log`` holds the compiler's output."""

    def __init__(self, source: str, n_eq: int, n_const: int, options: str = ""):
        lib = load()
        h = C.c_void_p()
        buf = C.create_string_buffer(1 << 16)
        code = lib.wind_plugin_create(source.encode(), n_eq, n_const, options.encode() or None,
                                      C.byref(h), buf, len(buf))
        self.log = buf.value.decode(errors="replace")
        if code != _capi.WIND_OK:
            raise WindError(code, "wind_plugin_create: " + self.log[-2000:])
        self.handle, self.n_eq, self.n_const = h, n_eq, n_const

    def close(self):
        if self.handle:
            load().wind_plugin_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def integrate(self, constants: np.ndarray, y: np.ndarray, tnow: float, tend: float,
                  atol: float, rtol: float, method: str = "sie", controller: str = "device",
                  n_integration_steps: int = 1, max_attempts: int = 0, timeout_s: float = 0.0):
        """Host arrays: ``constants`` float64 [S, n_const], ``y`` float64 [S, N]
        updated in place.  Returns (total_substeps, status, nsteps)."""
        lib = load()
        nsys = y.shape[0]
        assert y.dtype == np.float64 and y.flags["C_CONTIGUOUS"] and y.shape[1] == self.n_eq
        c = np.ascontiguousarray(constants, np.float64)
        o = options(method, "gje_f64", controller, 0, max_attempts, timeout_s)
        status = np.zeros(nsys, np.int32)
        nsteps = np.zeros(nsys, np.int64)
        total = C.c_int64(0)
        code = lib.wind_integrate_plugin(C.byref(o), self.handle, tnow, tend, n_integration_steps,
                                         c.ctypes.data, y.ctypes.data, nsys, atol, rtol,
                                         status.ctypes.data, nsteps.ctypes.data, C.byref(total),
                                         _capi.MEM_HOST, None)
        _check(code, "wind_integrate_plugin")
        return int(total.value), status, nsteps


def launch_count() -> int:
    return int(load().wind_launch_count())
