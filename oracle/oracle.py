"""ctypes face of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  Every function here is a thin numpy wrapper
over ``cw_oracle.c``, which restates the reference's Rust functions (see the
citations in that file); ``compile_network`` restates ``Network::from_spec``
(crates/engine/src/network.rs:283-445) in Python.
"""
from __future__ import annotations

import copy
import ctypes as C
import math
import os

import numpy as np

from . import build as _build

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if not os.path.exists(path):
            _build.build()
        L = C.CDLL(path)
        P = C.c_void_p
        L.or_philox.restype = None
        L.or_philox_batch.argtypes = [C.c_uint32, P, P, P]
        L.or_cw_exp.argtypes = [C.c_double]
        L.or_cw_exp.restype = C.c_double
        L.or_field_relax.argtypes = [P, C.c_double, C.c_int, C.c_double, C.c_int64, C.c_int, P]
        L.or_field_relax.restype = C.c_int
        L.or_field_residual.argtypes = [P]
        L.or_field_residual.restype = C.c_double
        L.or_field_inflow.argtypes = [P]
        L.or_field_inflow.restype = C.c_double
        L.or_field_step_explicit.argtypes = [P, C.c_double]
        L.or_field_step_explicit.restype = C.c_int
        L.or_hold_bath.argtypes = [P, P, C.c_double]
        L.or_hold_bath.restype = C.c_int
        L.or_free_span.argtypes = [P, P]
        L.or_free_span.restype = C.c_int
        L.or_auto_omega.argtypes = [P, P]
        L.or_auto_omega.restype = C.c_double
        L.or_reach.argtypes = [C.c_int, C.c_int, P, P]
        L.or_reach.restype = C.c_int
        L.or_lattice_delta_h.argtypes = [P, C.c_int64, C.c_int32, P]
        L.or_lattice_delta_h.restype = None
        L.or_lattice_mcs_sequential.argtypes = [P, C.c_uint64, C.c_int32]
        L.or_lattice_mcs_sequential.restype = None
        L.or_lattice_divide_across.argtypes = [P, C.c_int32, C.c_double, C.c_double, C.c_double, P]
        L.or_lattice_divide_across.restype = C.c_int32
        L.or_lattice_mcs_checkerboard.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32, C.c_int32,
                                                  C.c_int32]
        L.or_lattice_mcs_checkerboard.restype = None
        L.or_lattice_recount.argtypes = [P, P, P]
        L.or_lattice_recount.restype = None
        L.or_occupied_span.argtypes = [P, P]
        L.or_occupied_span.restype = C.c_int
        L.or_colouring.argtypes = [P, P]
        L.or_colouring.restype = C.c_int
        L.or_colour_order.argtypes = [C.c_int32, C.c_uint32, C.c_uint32, C.c_uint32, P]
        L.or_colour_order.restype = None
        L.or_network_step.argtypes = [P, C.c_int64, P, P, C.c_double, C.c_int32]
        L.or_network_step.restype = None
        L.or_network_mechanics.argtypes = [C.c_int64, C.c_int32, P, C.c_int32, C.c_double, C.c_double, C.c_int,
                                           C.c_uint32, P]
        L.or_network_mechanics.restype = None
        L.or_apply_uptake.argtypes = [C.c_int64, P, C.c_int32, P, P, P]
        L.or_apply_uptake.restype = None
        L.or_apply_background_uptake.argtypes = [C.c_int64, P, C.c_double, P]
        L.or_apply_background_uptake.restype = None
        L.or_apply_production.argtypes = [C.c_int64, P, C.c_int64, P, P]
        L.or_apply_production.restype = None
        L.or_hold_obstacles.argtypes = [C.c_int64, P, C.c_double, P, P]
        L.or_hold_obstacles.restype = None
        L.or_hold_vessels_by.argtypes = [C.c_int32, C.c_int32, P, C.c_double, P, P, P]
        L.or_hold_vessels_by.restype = None
        L.or_mean_per_cell.argtypes = [C.c_int64, P, P, C.c_int32, P]
        L.or_mean_per_cell.restype = None
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------------- RNG
def philox(ctr: np.ndarray, key) -> np.ndarray:
    """Philox4x32-10 of each row of ``ctr`` (n x 4 uint32) under ``key`` (2 words)."""
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros_like(ctr)
    lib().or_philox_batch(len(ctr), _p(ctr), _p(k), _p(out))
    return out


def cw_exp(x: float) -> float:
    return lib().or_cw_exp(float(x))


# --------------------------------------------------------------------- field
class _FieldStruct(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("d", C.c_int32), ("values", C.c_void_p),
                ("held", C.c_void_p), ("uptake", C.c_void_p), ("production", C.c_void_p),
                ("lin_sink", C.c_void_p), ("dcoef", C.c_double), ("decay", C.c_double), ("source", C.c_double)]


class Field:
    """The oracle's ScalarField (crates/engine/src/pde.rs:30-53) over numpy arrays."""

    def __init__(self, w, h, d=1, dcoef=0.2, decay=0.0, initial=0.0, source=0.0):
        n = w * h * d
        self.w, self.h, self.d = w, h, d
        self.values = np.full(n, float(initial))
        self.held = np.zeros(n, np.uint8)
        self.uptake = np.zeros(n)
        self.production = np.zeros(n)
        self.lin_sink = None
        self.dcoef, self.decay, self.source = float(dcoef), float(decay), float(source)

    def _struct(self):
        return _FieldStruct(self.w, self.h, self.d, _p(self.values).value, _p(self.held).value,
                            _p(self.uptake).value, _p(self.production).value,
                            None if self.lin_sink is None else _p(self.lin_sink).value,
                            self.dcoef, self.decay, self.source)

    def relax(self, tol, max_sweeps, omega=0.0, stop=0, threads=0):
        s = self._struct()
        sweeps = np.zeros(1, np.int64)
        rc = lib().or_field_relax(C.byref(s), float(omega), int(stop), float(tol), int(max_sweeps), int(threads),
                                  _p(sweeps))
        return rc, int(sweeps[0])

    def residual(self):
        s = self._struct()
        return lib().or_field_residual(C.byref(s))

    def inflow(self):
        s = self._struct()
        return lib().or_field_inflow(C.byref(s))

    def step(self, dt):
        s = self._struct()
        return lib().or_field_step_explicit(C.byref(s), float(dt))

    def hold_bath(self, open_mask, value):
        s = self._struct()
        o = np.ascontiguousarray(open_mask, dtype=np.uint8).reshape(-1)
        return lib().or_hold_bath(C.byref(s), _p(o), float(value))

    def free_span(self):
        s = self._struct()
        span = np.zeros(6, np.int32)
        ok = lib().or_free_span(C.byref(s), _p(span))
        return tuple(int(v) for v in span) if ok else None

    def auto_omega(self):
        span = np.zeros(6, np.int32)
        s = self._struct()
        if not lib().or_free_span(C.byref(s), _p(span)):
            return None
        return lib().or_auto_omega(C.byref(s), _p(span))


# --------------------------------------------------------------------- lattice
class _LatticeStruct(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("d", C.c_int32), ("grid", C.c_void_p),
                ("ncells", C.c_int32), ("type", C.c_void_p), ("volume", C.c_void_p), ("target", C.c_void_p),
                ("lambda_", C.c_void_p), ("surface", C.c_void_p), ("target_surface", C.c_void_p),
                ("lambda_surface", C.c_void_p), ("K", C.c_int32), ("J", C.c_void_p), ("order", C.c_int32),
                ("temperature", C.c_double), ("copy_moore", C.c_int32)]


def reach(order: int, volume: bool):
    off = np.zeros(3 * 124, np.int32)
    across = np.zeros(1)
    n = lib().or_reach(int(order), int(bool(volume)), _p(off), _p(across))
    return off[: 3 * n].reshape(-1, 3), float(across[0])


class Lattice:
    """The oracle's CpmLattice (crates/engine/src/cpm.rs:187-213) over numpy arrays.

    ``grid`` is int32, -1 for the obstacle; cell records are indexed by id with
    the medium at 0; ``J`` is a K x K table indexed by ``type``.
    """

    def __init__(self, grid, dims, ncells, J, temperature, order=1):
        self.w, self.h, self.d = dims
        self.grid = np.ascontiguousarray(grid, dtype=np.int32).reshape(-1).copy()
        self.ncells = int(ncells)
        self.type = np.zeros(self.ncells, np.int32)
        self.volume = np.zeros(self.ncells, np.int32)
        self.target = np.zeros(self.ncells, np.int32)
        self.lam = np.zeros(self.ncells)
        self.surface = None
        self.target_surface = None
        self.lambda_surface = None
        self.J = np.ascontiguousarray(J, dtype=np.float64)
        self.K = int(self.J.shape[0])
        self.J = self.J.reshape(-1).copy()
        self.order = int(order)
        self.temperature = float(temperature)
        self.copy_moore = False  # copy across faces (cpm.rs:922-944); True: from any Chebyshev neighbour

    def enable_surface(self, target_surface, lambda_surface):
        self.target_surface = np.ascontiguousarray(target_surface, dtype=np.int32).copy()
        self.lambda_surface = np.ascontiguousarray(lambda_surface, dtype=np.float64).copy()
        self.surface = np.zeros(self.ncells, np.int32)
        self.recount()

    def _struct(self):
        return _LatticeStruct(self.w, self.h, self.d, _p(self.grid).value, self.ncells, _p(self.type).value,
                              _p(self.volume).value, _p(self.target).value, _p(self.lam).value,
                              None if self.surface is None else _p(self.surface).value,
                              None if self.target_surface is None else _p(self.target_surface).value,
                              None if self.lambda_surface is None else _p(self.lambda_surface).value,
                              self.K, _p(self.J).value, self.order, self.temperature, int(self.copy_moore))

    def recount(self):
        s = self._struct()
        vol = np.zeros(self.ncells, np.int32)
        surf = None if self.surface is None else np.zeros(self.ncells, np.int32)
        lib().or_lattice_recount(C.byref(s), _p(vol), _p(surf))
        self.volume[:] = vol
        if surf is not None:
            self.surface[:] = surf
        return vol, surf

    def counts(self):
        s = self._struct()
        vol = np.zeros(self.ncells, np.int32)
        surf = None if self.surface is None else np.zeros(self.ncells, np.int32)
        lib().or_lattice_recount(C.byref(s), _p(vol), _p(surf))
        return vol, surf

    def delta_h(self, site: int, dst: int):
        """(contact numerator, contact, volume, surface, adhesion+volume, total) for copying `dst` into `site`."""
        s = self._struct()
        out = np.zeros(6)
        lib().or_lattice_delta_h(C.byref(s), int(site), int(dst), _p(out))
        return out

    def mcs_sequential(self, seed: int, sweeps: int = 1):
        s = self._struct()
        lib().or_lattice_mcs_sequential(C.byref(s), int(seed) & (2**64 - 1), int(sweeps))

    def mcs_checkerboard(self, seed: int, mcs0: int, sweeps: int = 1, snapshot: bool = False, subsweeps: int = 1):
        """The device's sublattice sweeps; `snapshot`: the planted mistake of
        reading one snapshot of the records per pass (statistical tests only);
        `subsweeps`: the device's sub-sweep kinetics."""
        s = self._struct()
        lib().or_lattice_mcs_checkerboard(C.byref(s), int(seed) & 0xFFFFFFFF, (int(seed) >> 32) & 0xFFFFFFFF,
                                          int(mcs0) & 0xFFFFFFFF, int(sweeps), int(bool(snapshot)), int(subsweeps))

    def divide_across(self, cid: int, normal, used: int):
        """divide_across (cpm.rs:1094-1160) with the daughter at record `used`:
        (daughter id or -1, records in use after)."""
        s = self._struct()
        u = np.array([used], np.int32)
        nx, ny, nz = (float(v) for v in (tuple(normal) + (0.0, 0.0, 0.0))[:3])
        d = lib().or_lattice_divide_across(C.byref(s), int(cid), nx, ny, nz, _p(u))
        return int(d), int(u[0])

    def occupied_span(self):
        s = self._struct()
        span = np.zeros(6, np.int32)
        ok = lib().or_occupied_span(C.byref(s), _p(span))
        return tuple(int(v) for v in span) if ok else None

    def colouring(self):
        s = self._struct()
        period = np.zeros(1, np.int32)
        n = lib().or_colouring(C.byref(s), _p(period))
        return n, int(period[0])


def colour_order(ncol, mcs, seed):
    perm = np.zeros(ncol, np.int32)
    lib().or_colour_order(int(ncol), int(mcs) & 0xFFFFFFFF, int(seed) & 0xFFFFFFFF, (int(seed) >> 32) & 0xFFFFFFFF,
                          _p(perm))
    return perm


# --------------------------------------------------------------------- network
INPUT_NAMES = ["oxygen", "egf", "crowding", "stress", "waste", "necrotic_factor"]
TERM_KINDS = ["activated_by", "inhibited_by", "activated_by_absence_of", "produced_by", "decays", "relaxes_to",
              "damaged_below", "damaged_above"]


class CompiledNetwork:
    def __init__(self, **kw):
        self.__dict__.update(kw)


class NetworkConfigError(ValueError):
    pass


def compile_network(spec: dict, reference_volume: int) -> CompiledNetwork:
    """Network::from_spec (crates/engine/src/network.rs:283-445), restated.

    ``spec`` is the parsed network table: ``nodes`` (name, initial, terms),
    ``roles``, ``mechanics``.  Raises NetworkConfigError where the reference
    returns CellweaveError::Config.
    """
    nodes = spec.get("nodes", [])
    if not nodes:
        raise NetworkConfigError("a network needs a node")
    roles = spec.get("roles")
    if roles is None:
        raise NetworkConfigError("the network declares no roles")
    mech = spec.get("mechanics")
    if mech is None:
        raise NetworkConfigError("the network declares no mechanics")
    index = {}
    for i, node in enumerate(nodes):
        if node["name"] in INPUT_NAMES:
            raise NetworkConfigError(f"node `{node['name']}` takes the name of an environment input")
        if node["name"] in index:
            raise NetworkConfigError(f"two nodes are named `{node['name']}`")
        index[node["name"]] = i

    def resolve(name, whose):
        if name in INPUT_NAMES:
            return -1 - INPUT_NAMES.index(name)
        if name in index:
            return index[name]
        raise NetworkConfigError(f"node `{whose}` reads `{name}`, which is neither a node nor an input; "
                                 f"known names are {INPUT_NAMES + [n['name'] for n in nodes]}")

    node_ptr, kind, source, rate, hn, hk, param = [0], [], [], [], [], [], []
    for node in nodes:
        for t in node.get("terms", []):
            k = t["kind"]
            if k not in TERM_KINDS:
                raise NetworkConfigError(f"unknown term kind `{k}`")
            kind.append(TERM_KINDS.index(k))
            rate.append(float(t["rate"]))
            n_, k_ = 0.0, 0.0
            if k in ("activated_by", "inhibited_by") and t.get("hill") is not None:
                n_, k_ = float(t["hill"]["n"]), float(t["hill"]["k"])
                if n_ <= 0.0 or k_ <= 0.0:
                    raise NetworkConfigError(f"node `{node['name']}` has a Hill term with n = {n_} and k = {k_}")
            hn.append(n_)
            hk.append(k_)
            p = 0.0
            if k == "relaxes_to":
                p = float(t["value"])
            elif k in ("damaged_below", "damaged_above"):
                p = float(t["threshold"])
                if p <= 0.0:
                    raise NetworkConfigError(f"node `{node['name']}` is damaged at {p}, which must be positive")
            param.append(p)
            source.append(resolve(t["source"], node["name"]) if k not in ("decays", "relaxes_to") else 0)
        node_ptr.append(len(kind))

    def role(name, which):
        if name not in index:
            raise NetworkConfigError(f"the {which} role names `{name}`, which is not a node")
        return index[name]

    growth = role(roles["growth"], "growth")
    survival = role(roles["survival"], "survival")
    hypoxia = role(roles["hypoxia_response"], "hypoxia response")
    optional = {}
    for r in ("differentiation", "apoptosis", "angiogenic", "evasion"):
        optional[r] = role(roles[r], r) if roles.get(r) is not None else -1
    initial = np.array([min(max(float(n.get("initial", 0.0)), 0.0), 1.0) for n in nodes])
    return CompiledNetwork(
        S=len(nodes), names=[n["name"] for n in nodes], node_ptr=np.array(node_ptr, np.int32),
        kind=np.array(kind, np.int32), source=np.array(source, np.int32), rate=np.array(rate, np.float64),
        hill_n=np.array(hn, np.float64), hill_k=np.array(hk, np.float64), param=np.array(param, np.float64),
        initial=initial, growth=growth, survival=survival, hypoxia=hypoxia, optional=optional,
        growth_coefficient=float(mech["growth_coefficient"]), lambda_volume=float(mech["lambda_volume"]),
        max_target=mech.get("max_target"), reference_volume=int(reference_volume))


class _NetStruct(C.Structure):
    _fields_ = [("S", C.c_int32), ("node_ptr", C.c_void_p), ("kind", C.c_void_p), ("source", C.c_void_p),
                ("rate", C.c_void_p), ("hill_n", C.c_void_p), ("hill_k", C.c_void_p), ("param", C.c_void_p)]


def network_step(net: CompiledNetwork, state: np.ndarray, inputs: np.ndarray, dt: float, substeps: int = 1):
    """rk4 (network.rs:777-799) ``substeps`` times on every row of ``state`` (in place)."""
    assert state.dtype == np.float64 and state.flags.c_contiguous
    inputs = np.ascontiguousarray(inputs, dtype=np.float64)
    s = _NetStruct(net.S, _p(net.node_ptr).value, _p(net.kind).value, _p(net.source).value, _p(net.rate).value,
                   _p(net.hill_n).value, _p(net.hill_k).value, _p(net.param).value)
    lib().or_network_step(C.byref(s), state.shape[0], _p(state), _p(inputs), float(dt), int(substeps))
    return state


# ---------------------------------------------------------------- mutations
MUTATION_SPREAD = 2.0  # network.rs:158
GAINED_RATE = 0.1      # network.rs:163
REWIRED_INPUTS = 4     # network.rs:165-169: oxygen, egf, crowding, stress
NETWORK_INPUTS = ["oxygen", "egf", "crowding", "stress", "waste", "necrotic_factor"]  # core network.rs INPUT_NAMES


def _pick(n: int, u: float) -> int:
    """``((u * n as f64) as usize).min(n.saturating_sub(1))`` (network.rs:488-489, 521)."""
    v = u * n
    k = int(v) if v > 0.0 else 0
    return min(k, max(n - 1, 0))


def mutate_spec(spec: dict, which: float, how: float):
    """Network::mutate (network.rs:479-501) on a network table: one rate of
    every node's terms in file order, picked by ``which``, times
    MUTATION_SPREAD^(2 how - 1).  Returns (new table, record) or (table, None)."""
    spec = copy.deepcopy(spec)
    count = sum(len(n.get("terms", [])) for n in spec["nodes"])
    pick = _pick(count, which)
    factor = math.pow(MUTATION_SPREAD, 2.0 * how - 1.0)
    for node in spec["nodes"]:
        terms = node.get("terms", [])
        if pick < len(terms):
            terms[pick]["rate"] = float(terms[pick]["rate"]) * factor
            return spec, dict(node=node["name"], term=pick, kind=terms[pick]["kind"], change="scaled",
                              factor=factor)
        pick -= len(terms)
    return spec, None


def rewire_spec(spec: dict, draws):
    """Network::rewire (network.rs:503-575) on a network table, draws =
    (mode, which, source, sign, how): a gained activated_by /
    activated_by_absence_of link below one half, a lost term otherwise."""
    mode, which, source, sign, how = draws
    spec = copy.deepcopy(spec)
    nodes = spec["nodes"]
    if mode < 0.5:
        node = nodes[_pick(len(nodes), which)]
        s = _pick(REWIRED_INPUTS + len(nodes), source)
        name = NETWORK_INPUTS[s] if s < REWIRED_INPUTS else nodes[s - REWIRED_INPUTS]["name"]
        rate = GAINED_RATE * math.pow(MUTATION_SPREAD, 2.0 * how - 1.0)
        kind = "activated_by" if sign < 0.5 else "activated_by_absence_of"
        terms = node.setdefault("terms", [])
        terms.append({"kind": kind, "rate": rate, "source": name})
        return spec, dict(node=node["name"], term=len(terms) - 1, kind=kind, change="gained", source=name, rate=rate)
    count = sum(len(n.get("terms", [])) for n in nodes)
    at = _pick(count, which)
    for node in nodes:
        terms = node.get("terms", [])
        if at < len(terms):
            lost = terms.pop(at)
            return spec, dict(node=node["name"], term=at, kind=lost["kind"], change="lost")
        at -= len(terms)
    return spec, None


def mutation_text(rec: dict) -> str:
    """Mutation's Display (network.rs:201-226)."""
    if rec["change"] == "scaled":
        return f"{rec['node']} {rec['kind']} #{rec['term']} x{rec['factor']:.2f}"
    if rec["change"] == "gained":
        return f"{rec['node']} gains {rec['kind']} {rec['source']} @{rec['rate']:.2f}"
    return f"{rec['node']} loses {rec['kind']} #{rec['term']}"


def network_mechanics(net: CompiledNetwork, state: np.ndarray) -> np.ndarray:
    out = np.zeros(state.shape[0], np.uint32)
    mt = net.max_target
    lib().or_network_mechanics(state.shape[0], net.S, _p(np.ascontiguousarray(state)), net.growth,
                               net.growth_coefficient, 0.0 if mt is None else float(mt), int(mt is not None),
                               net.reference_volume, _p(out))
    return out


# --------------------------------------------------------------------- coupling
def apply_uptake(grid, type_, rate_by_type):
    grid = np.ascontiguousarray(grid, np.int32).reshape(-1)
    type_ = np.ascontiguousarray(type_, np.int32)
    rbt = np.ascontiguousarray(rate_by_type, np.float64)
    out = np.zeros(grid.size)
    lib().or_apply_uptake(grid.size, _p(grid), len(type_), _p(type_), _p(rbt), _p(out))
    return out


def apply_background_uptake(grid, rate, uptake):
    grid = np.ascontiguousarray(grid, np.int32).reshape(-1)
    lib().or_apply_background_uptake(grid.size, _p(grid), float(rate), _p(uptake))
    return uptake


def apply_production(grid, per_cell):
    grid = np.ascontiguousarray(grid, np.int32).reshape(-1)
    pc = np.ascontiguousarray(per_cell, np.float64)
    out = np.zeros(grid.size)
    lib().or_apply_production(grid.size, _p(grid), len(pc), _p(pc), _p(out))
    return out


def hold_obstacles(grid, value, held, values):
    grid = np.ascontiguousarray(grid, np.int32).reshape(-1)
    lib().or_hold_obstacles(grid.size, _p(grid), float(value), _p(held), _p(values))


def hold_vessels_by(grid, value, delivery, held, values):
    """hold_vessels_by (coupling.rs:114-150) on a plane grid [h][w]; held and
    values are updated in place (flat, the grid's order)."""
    g = np.ascontiguousarray(grid, np.int32)
    h, w = g.shape
    dl = np.ascontiguousarray(delivery, np.float64).reshape(-1)
    lib().or_hold_vessels_by(w, h, _p(g), float(value), _p(dl), _p(held), _p(values))


def mean_per_cell(grid, values, ncells):
    grid = np.ascontiguousarray(grid, np.int32).reshape(-1)
    values = np.ascontiguousarray(values, np.float64).reshape(-1)
    out = np.zeros(int(ncells))
    lib().or_mean_per_cell(grid.size, _p(grid), _p(values), int(ncells), _p(out))
    return out
