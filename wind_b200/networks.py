"""ODE networks (the ode_system plug-ins) and seeded synthetic workloads.

A :class:`Network` carries what the C ABI's ``wind_network`` needs for a batch
of systems: the kind, the equations per system ``N``, and the per-system
constants / reactions / dense linear term as NumPy arrays.  The kinds mirror
the reference's plug-in instances:

* ``NR_TEST``   -- python/ode_systems/NR_test.py (2 eqs, 4 constants)
* ``KATZ96``    -- cuda/ode_system/ode_gold.c, python/ode_systems/katz96.py
                   (5 species, 10 rate constants)
* ``STIFFTRIG`` -- python/ode_systems/stifftrig.py (2 eqs, 2 constants)
* ``MASS_ACTION`` -- runtime two-body networks A+B -> C+D (no reference
                   instance; the synthetic dense and mixed-size workloads).

The workload builders reproduce the synthetic stand-ins for the reference's
benchmark shapes; every draw is seeded (numpy PCG64 ``default_rng``).
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

NET_NR_TEST = 1
NET_KATZ96 = 2
NET_STIFFTRIG = 3
NET_MASS_ACTION = 4

# Equations of one copy of each builtin network.
BASE_N = {NET_NR_TEST: 2, NET_KATZ96: 5, NET_STIFFTRIG: 2}

NET_NAMES = {NET_NR_TEST: "NR_test", NET_KATZ96: "Katz96",
             NET_STIFFTRIG: "StiffTrig", NET_MASS_ACTION: "MassAction"}

# Helium abundance by number relative to H for mass fraction Y=0.27,
# y_He = Y / (4 (1 - Y)) (python/ode_systems/katz96.py:188-189).
Y_HELIUM = 0.27 / (4.0 * (1.0 - 0.27))


@dataclasses.dataclass
class Network:
    """A batch of systems of one network shape.

    Arrays are C-contiguous; ``constants`` is ``[S, n_const]`` float64,
    ``rates`` ``[S, R]`` float64, ``species`` ``[S, R, 4]`` uint16 (A, B, C, D),
    ``linear`` ``[S, N, N]`` float32 row-major (f_j += L_jk y_k)."""

    kind: int
    n_eq: int
    nsys: int
    constants: Optional[np.ndarray] = None
    rates: Optional[np.ndarray] = None
    species: Optional[np.ndarray] = None
    linear: Optional[np.ndarray] = None

    @property
    def n_const(self) -> int:
        return 0 if self.constants is None else int(self.constants.shape[1])

    @property
    def n_react(self) -> int:
        return 0 if self.rates is None else int(self.rates.shape[1])

    @property
    def name(self) -> str:
        if self.kind == NET_MASS_ACTION:
            lin = "_lin" if self.linear is not None else ""
            return f"ma_n{self.n_eq}_r{self.n_react}{lin}"
        base = {NET_NR_TEST: "nr_test", NET_KATZ96: "katz96", NET_STIFFTRIG: "stifftrig"}[self.kind]
        nt = self.ntile
        return base if nt == 1 else f"{base}_t{nt}"

    @property
    def ntile(self) -> int:
        """Copies of a builtin network in one system (1 for an untiled
        network and for mass action)."""
        if self.kind == NET_MASS_ACTION:
            return 1
        return self.n_eq // BASE_N[self.kind]

    def subset(self, idx) -> "Network":
        """Systems ``idx`` (slice or index array) as a new Network."""
        pick = (lambda a: None if a is None else np.ascontiguousarray(a[idx]))
        n = len(np.arange(self.nsys)[idx])
        return Network(self.kind, self.n_eq, n, pick(self.constants),
                       pick(self.rates), pick(self.species), pick(self.linear))

    def packed_constants(self) -> np.ndarray:
        """Per-system constants in the reference host-contract layout
        (cuda/include/ode_gold.h): builtin kinds pass ``constants``; mass
        action packs ``[rates R | species 4R | L N*N]`` as float64."""
        if self.kind != NET_MASS_ACTION:
            return np.ascontiguousarray(self.constants, dtype=np.float64)
        parts = [self.rates.astype(np.float64),
                 self.species.reshape(self.nsys, -1).astype(np.float64)]
        if self.linear is not None:
            parts.append(self.linear.reshape(self.nsys, -1).astype(np.float64))
        return np.ascontiguousarray(np.concatenate(parts, axis=1))

    def nbytes(self) -> int:
        return sum(a.nbytes for a in (self.constants, self.rates, self.species,
                                      self.linear) if a is not None)


@dataclasses.dataclass
class Workload:
    """A network batch plus its initial state and integration settings."""

    net: Network
    y0: np.ndarray            # [S, N] float64
    tnow: float
    tend: float
    atol: float
    rtol: float
    n_integration_steps: int = 1
    n_output_steps: int = 1
    label: str = ""

    def subset(self, idx) -> "Workload":
        return dataclasses.replace(self, net=self.net.subset(idx),
                                   y0=np.ascontiguousarray(self.y0[idx]))


# --------------------------------------------------------------------------
# builtin networks
# --------------------------------------------------------------------------
def nr_test(nsys: int) -> Network:
    """NR 16.6.1 stiff linear test, constants (998, 1998, -999, -1999)
    (python/ode_systems/NR_test.py:28-29)."""
    c = np.tile(np.array([998.0, 1998.0, -999.0, -1999.0]), (nsys, 1))
    return Network(NET_NR_TEST, 2, nsys, constants=np.ascontiguousarray(c))


def stifftrig(nsys: int, freq: float = 6.0) -> Network:
    """StiffTrig with both constants 2*pi*freq (python/ode_systems/stifftrig.py:29-36)."""
    c = np.full((nsys, 2), 2.0 * np.pi * freq)
    return Network(NET_STIFFTRIG, 2, nsys, constants=c)


def tile_network(net: Network, ntile: int) -> Network:
    """The Precompiler's Ntile tiling (python/ode_systems/ode_base.py:86-88,
    219-281) of a builtin network: each system becomes ntile copies of it
    (n_eq x ntile equations, block-diagonal Jacobian) sharing the system's
    constants; Katz96 copies use tile 0's electron density."""
    if net.kind == NET_MASS_ACTION or net.ntile != 1:
        raise ValueError("tile an untiled builtin network")
    if ntile < 1:
        raise ValueError("ntile >= 1")
    return Network(net.kind, net.n_eq * ntile, net.nsys, constants=net.constants)


def tile_workload(wl: "Workload", ntile: int) -> "Workload":
    """Tile a builtin workload: the network by tile_network and each system's
    initial state repeated ntile times (tileEquations, ode_base.py:225-245)."""
    return dataclasses.replace(wl, net=tile_network(wl.net, ntile),
                               y0=np.ascontiguousarray(np.tile(wl.y0, (1, ntile))),
                               label=f"{wl.label}_t{ntile}")


def katz96_rates(T: np.ndarray, nH: np.ndarray, uv: np.ndarray) -> np.ndarray:
    """The ten Katz96 rate constants per cell, in 1/s, evaluated in FP64 from
    the formulas of python/ode_systems/katz96.py:109-121.  Collisional and
    recombination rates are multiplied by nH (abundances are per nH); the
    photo-ionisation rates take the UV rate for H0 and the reference's fixed
    ratios 3.7e-12/4.4e-11 (He0) and 1.7e-14/4.4e-11 (He+)
    (katz96.py:110,113,115).  Order (cuda/ode_system/ode_gold.c:13-22):
    Gamma_eH0, Gamma_gH0, alpha_H+, Gamma_eHe0, Gamma_gHe0, Gamma_eHe+,
    Gamma_gHe+, alpha_He+, alpha_d, alpha_He++."""
    T = np.asarray(T, np.float64)
    nH = np.asarray(nH, np.float64)
    uv = np.asarray(uv, np.float64)
    sq = np.sqrt(T)
    damp = 1.0 + np.sqrt(T / 1e5)
    c = np.empty((T.size, 10))
    c[:, 0] = 5.85e-11 * sq / damp * np.exp(-157809.1 / T) * nH
    c[:, 1] = uv
    c[:, 2] = 8.4e-11 / sq * (T / 1e3) ** -0.2 / (1 + (T / 1e6) ** 0.7) * nH
    c[:, 3] = 2.38e-11 * sq / damp * np.exp(-285335.4 / T) * nH
    c[:, 4] = uv * (3.7e-12 / 4.4e-11)
    c[:, 5] = 5.68e-12 * sq / damp * np.exp(-631515.0 / T) * nH
    c[:, 6] = uv * (1.7e-14 / 4.4e-11)
    c[:, 7] = 1.5e-10 * T ** -0.6353 * nH
    c[:, 8] = 1.9e-3 * T ** -1.5 * np.exp(-470000.0 / T) * (1 + 0.3 * np.exp(-94000.0 / T)) * nH
    c[:, 9] = 3.36e-10 * T ** -0.5 * (T / 1e3) ** -0.2 / (1 + (T / 1e6) ** 0.7) * nH
    return c


def _log_uniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


# --------------------------------------------------------------------------
# mass-action networks
# --------------------------------------------------------------------------
def random_mass_action(rng, nsys: int, n_eq: int, n_react: int,
                       k_lo: float, k_hi: float) -> Network:
    """Per-system random two-body networks: R reactions A+B -> C+D with rate
    log-uniform in [k_lo, k_hi] and species indices uniform in [0, N)."""
    rates = _log_uniform(rng, k_lo, k_hi, (nsys, n_react))
    species = rng.integers(0, n_eq, size=(nsys, n_react, 4), dtype=np.int64)
    return Network(NET_MASS_ACTION, n_eq, nsys, rates=np.ascontiguousarray(rates),
                   species=np.ascontiguousarray(species.astype(np.uint16)))


def dense_linear(rng, nsys: int, n_eq: int, lam_lo: float, lam_hi: float,
                 chunk: int = 16384) -> np.ndarray:
    """L = Q diag(-lambda) Q^T per system, Q from the QR of a Gaussian matrix
    with the signs of R's diagonal folded into Q, lambda log-uniform; computed
    in FP64 and stored as float32."""
    out = np.empty((nsys, n_eq, n_eq), np.float32)
    for s0 in range(0, nsys, chunk):
        s1 = min(nsys, s0 + chunk)
        g = rng.standard_normal((s1 - s0, n_eq, n_eq))
        q, r = np.linalg.qr(g)
        q = q * np.sign(np.diagonal(r, axis1=1, axis2=2))[:, None, :]
        lam = _log_uniform(rng, lam_lo, lam_hi, (s1 - s0, n_eq))
        out[s0:s1] = np.einsum("sik,sk,sjk->sij", q, -lam, q).astype(np.float32)
    return out


# --------------------------------------------------------------------------
# the five synthetic workloads
# --------------------------------------------------------------------------
def workload_nr(nsys: int = 1024, seed: int = 0) -> Workload:
    """NR stiff linear test: ICs U[0.5,1.5]^2, t = 0..1 in 100 output steps,
    one integration step each, rtol 1e-6, atol 1e-8."""
    rng = np.random.default_rng(seed)
    y0 = rng.uniform(0.5, 1.5, size=(nsys, 2))
    return Workload(nr_test(nsys), y0, 0.0, 1.0, 1e-8, 1e-6, 1, 100, "nr_test")


def nr_analytic(y0: np.ndarray, t: float) -> np.ndarray:
    """Exact solution of the NR test: eigenvectors (2,-1) at -1 and (1,-1) at
    -1000 of the matrix at python/ode_systems/NR_test.py:34-35."""
    u0, v0 = y0[:, 0], y0[:, 1]
    a = u0 + v0
    b = u0 + 2.0 * v0
    e1, e2 = np.exp(-t), np.exp(-1000.0 * t)
    return np.stack([2 * a * e1 - b * e2, -a * e1 + b * e2], axis=1)


def workload_katz96(nsys: int = 65536, seed: int = 1, dt: float = 1e13,
                    atol: float = 5e-3, rtol: float = 5e-3) -> Workload:
    """Katz96 primordial H/He network: T log-U[1e2,1e8] K, nH log-U[1e-4,1e4],
    UV log-U[1e-15,1e-11] 1/s; ICs fully ionised H with singly ionised He,
    [0, 1, 0, y_He, 0] (the pattern of cuda/debug/inputKatz96_1_1_1.h:4);
    one call over dt seconds, n_integration_steps = 1."""
    rng = np.random.default_rng(seed)
    T = _log_uniform(rng, 1e2, 1e8, nsys)
    nH = _log_uniform(rng, 1e-4, 1e4, nsys)
    uv = _log_uniform(rng, 1e-15, 1e-11, nsys)
    net = Network(NET_KATZ96, 5, nsys, constants=katz96_rates(T, nH, uv))
    y0 = np.tile(np.array([0.0, 1.0, 0.0, Y_HELIUM, 0.0]), (nsys, 1))
    return Workload(net, y0, 0.0, dt, atol, rtol, 1, 1, "katz96")


# Seeded synthetic batches are generated in chunks of CHUNK systems, chunk c
# of a workload drawn from its own generator default_rng([seed, ..., c]), so
# system i is the same whichever slice of the workload is asked for (a test
# can take systems 0..63 of the 262,144-system batch without generating it).
CHUNK = 4096


def _chunked(nsys: int, first: int, make):
    """Concatenate make(c) over the chunks covering [first, first + nsys)."""
    c0, c1 = first // CHUNK, (first + nsys + CHUNK - 1) // CHUNK
    parts = [make(c) for c in range(c0, max(c1, c0 + 1))]
    lo = first - c0 * CHUNK
    return parts, slice(lo, lo + nsys)


def _cat_networks(nets, sl) -> Network:
    n0 = nets[0]
    cat = (lambda k: None if getattr(n0, k) is None
           else np.ascontiguousarray(np.concatenate([getattr(n, k) for n in nets])[sl]))
    rates, species, linear = cat("rates"), cat("species"), cat("linear")
    return Network(n0.kind, n0.n_eq, int(rates.shape[0]), rates=rates, species=species,
                   linear=linear)


def workload_dense(nsys: int = 262144, seed: int = 2, n_eq: int = 32,
                   n_react: int = 64, first: int = 0) -> Workload:
    """Dense stiff network: L = Q diag(-lambda) Q^T with lambda log-U[1e-2,1e6]
    plus 64 random two-body reactions with k log-U[1e-3,1e1]; y0 U[0,1];
    dt = 1, rtol 1e-6, atol 1e-8.  Systems [first, first + nsys) of the seeded
    sequence (chunk c drawn from default_rng([seed, c]))."""
    def make(c):
        rng = np.random.default_rng([seed, c])
        net = random_mass_action(rng, CHUNK, n_eq, n_react, 1e-3, 1e1)
        net.linear = dense_linear(rng, CHUNK, n_eq, 1e-2, 1e6)
        return net, rng.uniform(0.0, 1.0, size=(CHUNK, n_eq))
    parts, sl = _chunked(nsys, first, make)
    net = _cat_networks([p[0] for p in parts], sl)
    y0 = np.ascontiguousarray(np.concatenate([p[1] for p in parts])[sl])
    return Workload(net, y0, 0.0, 1.0, 1e-8, 1e-6, 1, 1, f"dense_n{n_eq}")


MIXED_SIZES = (5, 16, 32, 64, 157)
MIXED_FRACTIONS = (0.40, 0.25, 0.20, 0.10, 0.05)


def mixed_counts(nsys: int, fractions=MIXED_FRACTIONS) -> list:
    """Systems per size class: rounded fractions, the last class takes the rest."""
    counts = [int(round(nsys * f)) for f in fractions]
    counts[-1] = nsys - sum(counts[:-1])
    return counts


def workload_mixed_class(n_eq: int, nsys: int, seed: int = 3, dt: float = 1.0,
                         atol: float = 1e-8, rtol: float = 1e-6, first: int = 0) -> Workload:
    """Systems [first, first + nsys) of the N = n_eq class of the mixed-size
    batch: random two-body networks with 10N reactions, k log-U[1e-4,1e4],
    y0 U[0,1] (chunk c drawn from default_rng([seed, n_eq, c]))."""
    def make(c):
        rng = np.random.default_rng([seed, n_eq, c])
        net = random_mass_action(rng, CHUNK, n_eq, 10 * n_eq, 1e-4, 1e4)
        return net, rng.uniform(0.0, 1.0, size=(CHUNK, n_eq))
    parts, sl = _chunked(nsys, first, make)
    net = _cat_networks([p[0] for p in parts], sl)
    y0 = np.ascontiguousarray(np.concatenate([p[1] for p in parts])[sl])
    return Workload(net, y0, 0.0, dt, atol, rtol, 1, 1, f"mixed_n{n_eq}")


def workload_mixed(nsys: int = 200000, seed: int = 3, dt: float = 1.0,
                   atol: float = 1e-8, rtol: float = 1e-6,
                   sizes=MIXED_SIZES, fractions=MIXED_FRACTIONS) -> list:
    """Mixed-size batch: N in {5,16,32,64,157} at 40/25/20/10/5 %, each system
    a random two-body network with 10N reactions, k log-U[1e-4,1e4]; y0 U[0,1].
    Returns one Workload per size class (counts from the fractions); class N
    holds the first systems of :func:`workload_mixed_class` for N."""
    out = []
    for n_eq, cnt in zip(sizes, mixed_counts(nsys, fractions)):
        if cnt > 0:
            out.append(workload_mixed_class(n_eq, cnt, seed, dt, atol, rtol))
    return out
