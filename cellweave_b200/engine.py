"""The reference's engine API over the C ABI: CpmLattice, ScalarField,
Network, the coupling functions and a batched Simulation driver.

Names, argument meanings and errors follow crates/engine of the reference
(cpm.rs, pde.rs, network.rs, coupling.rs, simulation.rs); every object may
hold a batch of independent histories (``hist`` picks one), a single history
being a batch of one.  All compute runs in ``libcellweave_b200.so`` on the
GPU; this module only moves arguments across.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import tomllib
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import ConfigError, call, lib, ptr

OBSTACLE = -1
FP64, FP32_DC = 0, 1
WINDOW_AUTO, WINDOW_64, WINDOW_TALL = 0, 1, 2
STOP_MAX_CHANGE, STOP_RESIDUAL = 0, 1
COPY_VON_NEUMANN, COPY_MOORE = 0, 1
VALUES, UPTAKE, PRODUCTION, LIN_SINK = 0, 1, 2, 3


def _check_hist(obj, hist):
    if not 0 <= hist < len(obj.dims):
        raise _lib.NotFoundError(f"no history {hist}")


def _dims(dims):
    dims = [tuple(int(v) for v in (tuple(d) + (1,))[:3]) if len(d) < 3 else tuple(int(v) for v in d) for d in dims]
    w = np.array([d[0] for d in dims], np.uint32)
    h = np.array([d[1] for d in dims], np.uint32)
    z = np.array([d[2] for d in dims], np.uint32)
    return dims, w, h, z


# ============================================================== ScalarField
class ScalarField:
    """ScalarField (crates/engine/src/pde.rs:30-640) of one or more histories."""

    def __init__(self, dims: Sequence[Sequence[int]], d: float, decay: float = 0.0, initial: float = 0.0):
        self.dims, w, h, z = _dims(dims)
        handle = C.c_void_p()
        call("cw_field_create", len(self.dims), ptr(w), ptr(h), ptr(z), float(d), float(decay), float(initial),
             C.byref(handle))
        self._h = handle
        self.d, self.decay = float(d), float(decay)

    @classmethod
    def new(cls, width, height, d, decay=0.0, initial=0.0):
        """ScalarField::new (pde.rs:82-90)."""
        return cls([(width, height, 1)], d, decay, initial)

    @classmethod
    def with_depth(cls, width, height, depth, d, decay=0.0, initial=0.0):
        """ScalarField::with_depth (pde.rs:98-131)."""
        return cls([(width, height, depth)], d, decay, initial)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._LIB is not None:
            lib().cw_field_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def n(self, hist=0):
        _check_hist(self, hist)
        w, h, d = self.dims[hist]
        return w * h * d

    # ---- arrays
    def upload(self, which: int, arr, hist: int = 0):
        a = np.ascontiguousarray(arr, np.float64).reshape(-1)
        if a.size != self.n(hist):
            raise ConfigError(f"expected {self.n(hist)} values, got {a.size}")
        call("cw_field_upload", self._h, hist, which, ptr(a))

    def download(self, which: int = VALUES, hist: int = 0) -> np.ndarray:
        out = np.empty(self.n(hist))
        call("cw_field_download", self._h, hist, which, ptr(out))
        return out

    def values(self, hist=0):
        return self.download(VALUES, hist)

    def set_values(self, arr, hist=0):
        self.upload(VALUES, arr, hist)

    def set_uptake_array(self, arr, hist=0):
        """set_uptake_at over every pixel (pde.rs:170-174): rates floored at zero."""
        self.upload(UPTAKE, np.maximum(np.asarray(arr, np.float64), 0.0), hist)

    def set_production_array(self, arr, hist=0):
        """set_production_at over every pixel (pde.rs:178-182)."""
        self.upload(PRODUCTION, np.maximum(np.asarray(arr, np.float64), 0.0), hist)

    def set_linear_sink(self, arr, hist=0):
        """The first-order sink k_i of D lap c - k_i c (an extension; zero is the reference)."""
        self.upload(LIN_SINK, arr, hist)

    def held(self, hist=0):
        out = np.empty(self.n(hist), np.uint8)
        call("cw_field_download_held", self._h, hist, ptr(out))
        return out

    def set_held(self, mask, hist=0):
        m = np.ascontiguousarray(mask, np.uint8).reshape(-1)
        call("cw_field_upload_held", self._h, hist, ptr(m))

    # ---- reference methods
    def with_source(self, source):
        call("cw_field_set_source", self._h, float(source))
        return self

    def set_diffusion(self, d):
        call("cw_field_set_diffusion", self._h, float(d))
        self.d = float(d)

    def fill(self, value):
        call("cw_field_fill", self._h, float(value))

    def clear_uptake(self):
        call("cw_field_clear", self._h, UPTAKE)

    def clear_production(self):
        call("cw_field_clear", self._h, PRODUCTION)

    def release_all(self):
        call("cw_field_release_all", self._h)

    def hold_where(self, value, mask, hist=0):
        """hold_where (pde.rs:491-498) with a boolean mask."""
        m = np.ascontiguousarray(mask, np.uint8).reshape(-1)
        call("cw_field_hold_mask", self._h, hist, ptr(m), float(value))

    def hold_bath(self, value, open_mask, hist=0):
        """hold_bath_at (pde.rs:550-631) with `open` given as a mask."""
        o = np.ascontiguousarray(open_mask, np.uint8).reshape(-1)
        call("cw_field_hold_bath", self._h, hist, ptr(o), float(value))

    def relax(self, tolerance, max_sweeps, omega=None, stop=STOP_MAX_CHANGE, precision=FP64, inner_sweeps=0,
              block_depth=0, window=WINDOW_AUTO, stats=False, error_tolerance=0.0):
        """relax (pde.rs:245-288): the sweep count of every history (SimulationError if one did not settle)."""
        o = _lib.RelaxOpts(float(omega) if omega else 0.0, int(stop), float(tolerance), int(max_sweeps),
                           int(precision), int(inner_sweeps), int(block_depth), int(window), float(error_tolerance))
        st = (_lib.RelaxStats * len(self.dims))()
        rc = lib().cw_field_relax(self._h, C.byref(o), st)
        result = [dict(sweeps=s.sweeps, last_change=s.last_change, residual=s.residual, status=s.status,
                       omega=s.omega) for s in st]
        if rc != _lib.OK:
            err = _lib._ERRORS.get(rc, _lib.CellweaveError)(lib().cw_last_error().decode())
            err.stats = result
            raise err
        if stats:
            return result
        return result[0]["sweeps"] if len(result) == 1 else [r["sweeps"] for r in result]

    def relax_adjoint(self, dl_dc, tolerance, max_sweeps, omega=None, stop=STOP_RESIDUAL, precision=FP64,
                      inner_sweeps=0, block_depth=0, window=WINDOW_AUTO):
        """lambda with A^T lambda = dl_dc for the field's operator as it stands (zero on held
        pixels); dl_dc and the result hold every history's pixels, one after another."""
        g = np.ascontiguousarray(dl_dc, np.float64).reshape(-1)
        total = sum(w * h * d for w, h, d in self.dims)
        if g.size != total:
            raise ConfigError(f"expected {total} values, got {g.size}")
        o = _lib.RelaxOpts(float(omega) if omega else 0.0, int(stop), float(tolerance), int(max_sweeps),
                           int(precision), int(inner_sweeps), int(block_depth), int(window), 0.0)
        st = (_lib.RelaxStats * len(self.dims))()
        lam = np.empty(total)
        call("cw_field_relax_adjoint", self._h, ptr(g), ptr(lam), C.byref(o), st)
        return lam

    def residual(self):
        out = np.empty(len(self.dims))
        call("cw_field_residual", self._h, ptr(out))
        return out

    def inflow(self):
        """inflow (pde.rs:415-456) of every history."""
        out = np.empty(len(self.dims))
        call("cw_field_inflow", self._h, ptr(out))
        return out if len(out) > 1 else float(out[0])

    def step(self, dt):
        """DiffusionField::step (pde.rs:705-728)."""
        call("cw_field_step", self._h, float(dt))

    def free_count(self, hist=0):
        return int((self.held(hist) == 0).sum())

    def value_at(self, i, hist=0):
        v = self.values(hist)
        return float(v[i]) if 0 <= i < v.size else 0.0

    def concentration_at(self, x, y, hist=0):
        w, h, _ = self.dims[hist]
        if x >= w or y >= h:
            return 0.0
        return self.value_at(y * w + x, hist)


# ============================================================== CpmLattice
class CpmLattice:
    """CpmLattice (crates/engine/src/cpm.rs:187-1041) of one or more histories."""

    def __init__(self, dims, temperature, capacity, order=1, J=None):
        self.dims, w, h, z = _dims(dims)
        cap = np.array(capacity if np.ndim(capacity) else [capacity] * len(self.dims), np.uint32)
        handle = C.c_void_p()
        call("cw_lattice_create", len(self.dims), ptr(w), ptr(h), ptr(z), ptr(cap), float(temperature),
             C.byref(handle))
        self._h = handle
        self.capacity = cap
        self.temperature = float(temperature)
        if J is not None:
            self.set_contact(J, order)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._LIB is not None and getattr(self, "_owned", True):
            lib().cw_lattice_destroy(h)
            self._h = None

    @classmethod
    def borrowed(cls, handle, dims, owner):
        """A view of a lattice another object owns (a Simulation's)."""
        lat = cls.__new__(cls)
        lat._h, lat._owned, lat._owner = handle, False, owner
        lat.dims, w, h, z = _dims(dims)
        nh = C.c_uint32()
        call("cw_lattice_count", handle, C.byref(nh))
        caps = []
        for k in range(nh.value):
            c = C.c_uint32()
            call("cw_lattice_capacity", handle, k, C.byref(c))
            caps.append(c.value)
        lat.capacity = np.array(caps, np.uint32)
        lat.temperature = None
        return lat

    @property
    def handle(self):
        return self._h

    def n(self, hist=0):
        _check_hist(self, hist)
        w, h, d = self.dims[hist]
        return w * h * d

    def set_contact(self, J, order=1):
        """ContactEnergy as a K x K table over types, and set_contact_order (cpm.rs:274-301)."""
        J = np.ascontiguousarray(J, np.float64)
        call("cw_lattice_set_contact", self._h, int(J.shape[0]), ptr(J), int(order))

    def set_temperature(self, t):
        call("cw_lattice_set_temperature", self._h, float(t))

    def divide(self, ids, normals, hist=0):
        """divide_across (cpm.rs:1094-1160) for each of `ids` with its plane's normal
        (rows of 2 or 3 components): the daughters' ids, -1 where nothing changed."""
        ids = np.ascontiguousarray(ids, np.int32).reshape(-1)
        nrm = np.zeros((ids.size, 3))
        given = np.asarray(normals, np.float64).reshape(ids.size, -1)
        nrm[:, :given.shape[1]] = given
        out = np.empty(ids.size, np.int32)
        call("cw_lattice_divide", self._h, hist, ids.size, ptr(ids), ptr(np.ascontiguousarray(nrm)), ptr(out))
        return out

    def cell_count(self, hist=0):
        """Records in use (the medium's included): cell_count + 1 of the reference."""
        n = C.c_uint32()
        call("cw_lattice_cell_count", self._h, hist, C.byref(n))
        return int(n.value)

    def bath(self, hist=0):
        """The pixels hold_medium_bath holds (coupling.rs:156-158): medium joined to the
        box's outer layer through medium; uint8 per pixel, [d, h, w]."""
        w, h, d = self.dims[hist]
        out = np.empty(w * h * d, np.uint8)
        call("cw_lattice_bath", self._h, int(hist), ptr(out))
        return out.reshape(d, h, w)

    def set_subsweeps(self, n: int):
        """n sweeps of every colour a Monte Carlo step, each pixel attempting in
        each with probability 1/n: attempts nearer the Poisson(1) of random pixels."""
        call("cw_lattice_set_subsweeps", self._h, int(n))

    def set_copy_neighbourhood(self, moore: bool):
        """Copies from a face neighbour (try_flip, cpm.rs:797-838; the default) or, with
        moore=True, from any pixel at Chebyshev distance 1 (an extension)."""
        call("cw_lattice_set_copy_nbhd", self._h, COPY_MOORE if moore else COPY_VON_NEUMANN)

    def upload(self, grid, hist=0):
        g = np.ascontiguousarray(grid, np.int32).reshape(-1)
        if g.size != self.n(hist):
            raise ConfigError(f"expected {self.n(hist)} pixels, got {g.size}")
        call("cw_lattice_upload", self._h, hist, ptr(g))

    def grid(self, hist=0):
        out = np.empty(self.n(hist), np.int32)
        call("cw_lattice_download", self._h, hist, ptr(out))
        w, h, d = self.dims[hist]
        return out.reshape(d, h, w)

    def set_cells(self, type_=None, volume=None, target=None, lam=None, hist=0):
        arrs = [None if a is None else np.ascontiguousarray(a, dt) for a, dt in
                ((type_, np.int32), (volume, np.int32), (target, np.int32), (lam, np.float64))]
        n = next(len(a) for a in arrs if a is not None)
        call("cw_cells_set", self._h, hist, n, *[ptr(a) for a in arrs])

    def cells(self, n=None, hist=0):
        n = int(self.capacity[hist]) if n is None else n
        t, v, g = (np.empty(n, np.int32) for _ in range(3))
        lam = np.empty(n)
        call("cw_cells_get", self._h, hist, n, ptr(t), ptr(v), ptr(g), ptr(lam))
        return dict(type=t, volume=v, target=g, lam=lam)

    def volume(self, cid, hist=0):
        return int(self.cells(hist=hist)["volume"][cid])

    def set_surface(self, target_surface, lambda_surface, hist=0):
        ts = np.ascontiguousarray(target_surface, np.int32)
        ls = np.ascontiguousarray(lambda_surface, np.float64)
        call("cw_cells_set_surface", self._h, hist, len(ts), ptr(ts), ptr(ls))

    def surfaces(self, n=None, hist=0):
        n = int(self.capacity[hist]) if n is None else n
        out = np.empty(n, np.int32)
        call("cw_cells_get_surface", self._h, hist, n, ptr(out))
        return out

    def set_seed(self, seed, hist=0):
        call("cw_lattice_set_seed", self._h, hist, int(seed) & (2**64 - 1))

    def set_mcs(self, mcs):
        call("cw_lattice_set_mcs", self._h, int(mcs))

    @property
    def mcs(self):
        v = C.c_uint32()
        call("cw_lattice_get_mcs", self._h, C.byref(v))
        return v.value

    def monte_carlo_step(self, sweeps=1):
        """monte_carlo_step (cpm.rs:748-772), `sweeps` times, on every history."""
        call("cw_lattice_mcs", self._h, int(sweeps))

    def delta_h(self, sites, dsts, hist=0):
        """Delta-H (cpm.rs:841-894) of copying dsts[k] into sites[k]: rows of
        (contact numerator, contact, volume, surface, adhesion+volume, total)."""
        s = np.ascontiguousarray(sites, np.int64)
        d = np.ascontiguousarray(dsts, np.int32)
        out = np.empty((len(s), 6))
        call("cw_lattice_delta_h_batch", self._h, hist, len(s), ptr(s), ptr(d), ptr(out))
        return out

    def records_match_grid(self, hist=0):
        ok = C.c_int32()
        call("cw_lattice_verify", self._h, hist, C.byref(ok))
        return bool(ok.value)

    @classmethod
    def from_grids(cls, grids, records, temperature, J, order=1, seeds=None, capacity=None):
        """A lattice holding the given host grids and Records (seeding.Records), one per history."""
        dims = [(g.shape[2], g.shape[1], g.shape[0]) for g in grids]
        caps = [len(r) if capacity is None else capacity for r in records]
        lat = cls(dims, temperature, caps, order, J)
        for k, (g, r) in enumerate(zip(grids, records)):
            lat.upload(g, k)
            t, v, tg, lam = r.arrays()
            lat.set_cells(t, v, tg, lam, hist=k)
            lat.set_seed(0 if seeds is None else seeds[k], k)
        return lat


# ============================================================== coupling
def apply_uptake(field: ScalarField, lattice: CpmLattice, rate_by_type, first_order=False):
    """apply_uptake (coupling.rs:26-39) with a rate per cell type."""
    r = np.ascontiguousarray(rate_by_type, np.float64)
    call("cw_couple_uptake", field.handle, lattice.handle, len(r), ptr(r), int(bool(first_order)))


def apply_background_uptake(field, lattice, rate):
    """apply_background_uptake (coupling.rs:47-53)."""
    call("cw_couple_background_uptake", field.handle, lattice.handle, float(rate))


def apply_production(field, lattice, per_cell, hist=0):
    """apply_production (coupling.rs:61-73)."""
    pc = np.ascontiguousarray(per_cell, np.float64)
    call("cw_couple_production", field.handle, lattice.handle, hist, len(pc), ptr(pc))


def hold_obstacles_at(field, lattice, value):
    """hold_obstacles_at (coupling.rs:80-82)."""
    call("cw_couple_hold_obstacles", field.handle, lattice.handle, float(value))


def hold_vessels_by(field, lattice, value, delivery):
    """hold_vessels_by (coupling.rs:114-150): `delivery` is each pixel's share
    of a full vessel's supply, one value per pixel of the batch (flat, the
    batch's order), as the reference's `delivery(x, y)` closure gives it."""
    share = np.ascontiguousarray(delivery, np.float64).reshape(-1)
    if share.size != int(sum(int(w) * int(h) * int(d) for w, h, d in field.dims)):
        raise ValueError("hold_vessels_by needs one delivery share per pixel of the batch")
    call("cw_couple_hold_vessels_by", field.handle, lattice.handle, float(value), ptr(share))


def hold_medium_bath(field, lattice, value):
    """hold_medium_bath (coupling.rs:156-158)."""
    call("cw_couple_hold_medium_bath", field.handle, lattice.handle, float(value))


def mean_per_cell(field, lattice, n=None, hist=0):
    """mean_per_cell (coupling.rs:164-182) for ids [0, n)."""
    n = int(lattice.capacity[hist]) if n is None else int(n)
    out = np.empty(n)
    call("cw_couple_mean_per_cell", field.handle, lattice.handle, hist, n, ptr(out))
    return out


# ============================================================== Network
INPUT_NAMES = ["oxygen", "egf", "crowding", "stress", "waste", "necrotic_factor"]
TERM_KINDS = ["activated_by", "inhibited_by", "activated_by_absence_of", "produced_by", "decays", "relaxes_to",
              "damaged_below", "damaged_above"]


MECHANICS_KEYS = ("growth_coefficient", "lambda_volume", "max_target")


def load_network_spec(path: str, _seen=()) -> dict:
    """load_network_chain (crates/io/src/config.rs:416-447): a network file and
    everything it `extends`, youngest laid over oldest by merge_onto
    (crates/core/src/network.rs:269-283)."""
    here = os.path.realpath(path)
    if here in _seen:
        chain = " -> ".join(list(_seen) + [here])
        raise ConfigError(f"a network extends itself round a loop: {chain}")
    try:
        with open(path, "rb") as fh:
            spec = tomllib.load(fh)
    except OSError as e:
        raise ConfigError(f"reading the network {path}: {e}") from e
    except tomllib.TOMLDecodeError as e:
        raise ConfigError(f"{path} is not a network: {e}") from e
    # MechanicsSpec refuses a key it does not read (crates/core/src/network.rs:207-230):
    # a contact energy is the lattice's, not a network's
    for key in (spec.get("mechanics") or {}):
        if key not in MECHANICS_KEYS:
            raise ConfigError(f"{path}: unknown field `{key}` in the mechanics, expected one of "
                              f"{', '.join(MECHANICS_KEYS)}")
    parent = spec.get("extends")
    if parent is None:
        spec.pop("extends", None)
        return spec
    base = load_network_spec(os.path.join(os.path.dirname(path), parent), _seen + (here,))
    return merge_onto(spec, base)


def merge_onto(spec: dict, base: dict) -> dict:
    """NetworkSpec::merge_onto (crates/core/src/network.rs:269-283)."""
    nodes = list(base.get("nodes", []))
    for node in spec.get("nodes", []):
        for k, existing in enumerate(nodes):
            if existing["name"] == node["name"]:
                nodes[k] = node
                break
        else:
            nodes.append(node)
    return {"nodes": nodes, "roles": spec.get("roles") or base.get("roles"),
            "mechanics": spec.get("mechanics") or base.get("mechanics")}


class Network:
    """Network (crates/engine/src/network.rs:247-822), compiled on the library side."""

    ROLE_NAMES = ["growth", "survival", "hypoxia_response", "differentiation", "apoptosis", "angiogenic", "evasion"]

    def __init__(self, handle, names):
        self._h = handle
        self.names = names
        S = C.c_int32()
        roles = np.zeros(7, np.int32)
        init = np.zeros(len(names))
        call("cw_network_info", self._h, C.byref(S), ptr(roles), ptr(init))
        self.S = S.value
        self.roles = {k: int(v) for k, v in zip(self.ROLE_NAMES, roles)}
        self.initial = init

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._LIB is not None:
            lib().cw_network_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @classmethod
    def from_spec(cls, spec: dict, reference_volume: int) -> "Network":
        """Network::from_spec (network.rs:283-445); ConfigError where the reference refuses."""
        nodes = spec.get("nodes", [])
        names = [n["name"] for n in nodes]
        enc = [n.encode() for n in names]
        name_arr = (C.c_char_p * max(1, len(enc)))(*enc)
        initial = np.array([float(n.get("initial", 0.0)) for n in nodes] or [0.0])
        terms, keep = [], []
        for i, node in enumerate(nodes):
            for t in node.get("terms", []):
                kind = t.get("kind")
                if kind not in TERM_KINDS:
                    raise ConfigError(f"node `{node['name']}` has a term of unknown kind `{kind}`")
                src = t.get("source")
                b = None if src is None else src.encode()
                keep.append(b)
                hill = t.get("hill")
                param = t.get("value", t.get("threshold", 0.0))
                terms.append(_lib.TermSpec(i, TERM_KINDS.index(kind), b, float(t["rate"]),
                                           float(hill["n"]) if hill else 0.0, float(hill["k"]) if hill else 0.0,
                                           float(param), 1 if hill else 0))
        tarr = (_lib.TermSpec * max(1, len(terms)))(*terms)
        roles = spec.get("roles") or {}
        mech = spec.get("mechanics")
        if spec.get("roles") is None and nodes:
            raise ConfigError("the network declares no roles, and inherits none: say which node is growth, "
                              "which is survival, and which is the hypoxia response")
        if mech is None and nodes:
            raise ConfigError("the network declares no mechanics, and inherits none: say how the growth node "
                              "becomes a target volume")
        mech = mech or {"growth_coefficient": 0.0, "lambda_volume": 0.0}
        rn = [roles.get(k) for k in cls.ROLE_NAMES]
        handle = C.c_void_p()
        mt = mech.get("max_target")
        call("cw_network_compile", len(nodes), name_arr, ptr(initial), len(terms), tarr,
             *[None if r is None else r.encode() for r in rn], float(mech["growth_coefficient"]),
             float(mech["lambda_volume"]), math.nan if mt is None else float(mt), int(reference_volume),
             C.byref(handle))
        return cls(handle, names)

    @classmethod
    def load(cls, path, reference_volume):
        return cls.from_spec(load_network_spec(path), reference_volume)

    def step_batch(self, state, inputs, dt, substeps=1):
        """rk4 (network.rs:777-799) `substeps` times on every row of state [ncells, S] (in place)."""
        st = np.ascontiguousarray(state, np.float64)
        ins = np.ascontiguousarray(inputs, np.float64)
        call("cw_network_step_batch", self._h, st.shape[0], ptr(st), ptr(ins), float(dt), int(substeps))
        if st is not state:
            state[...] = st
        return state

    def backward_batch(self, state, inputs, dt, substeps, adjoint, nrates=0):
        """The adjoint of step_batch from `state` (the state before the steps): returns
        (dL/d state before, dL/d oxygen input per cell, dL/d rate of the first nrates terms)
        given `adjoint` = dL/d state after."""
        st = np.ascontiguousarray(state, np.float64)
        ins = np.ascontiguousarray(inputs, np.float64)
        adj = np.array(adjoint, np.float64, order="C", copy=True)
        d_o2 = np.zeros(st.shape[0])
        d_rates = np.zeros(max(int(nrates), 1))
        call("cw_network_backward_batch", self._h, st.shape[0], ptr(st), ptr(ins), float(dt), int(substeps), ptr(adj),
             ptr(d_o2), int(nrates), ptr(d_rates))
        return adj, d_o2, d_rates[:int(nrates)]

    INPUT_NAMES = ["oxygen", "egf", "crowding", "stress", "waste", "necrotic_factor"]
    CHANGES = ["scaled", "gained", "lost"]

    def _record(self, r):
        """A Mutation (network.rs:171-199) as a dict, with its Display text."""
        kind = TERM_KINDS[r.kind]
        node = self.names[r.node]
        change = self.CHANGES[r.change]
        rec = dict(node=node, term=int(r.term), kind=kind, change=change)
        if change == "scaled":
            rec["factor"] = r.value
            rec["text"] = f"{node} {kind} #{r.term} x{r.value:.2f}"
        elif change == "gained":
            src = self.INPUT_NAMES[-1 - r.source] if r.source < 0 else self.names[r.source]
            rec.update(source=src, rate=r.value, text=f"{node} gains {kind} {src} @{r.value:.2f}")
        else:
            rec["text"] = f"{node} loses {kind} #{r.term}"
        return rec

    def mutate(self, which, how):
        """Network::mutate (network.rs:479-501) on a copy: (daughter network, mutation record);
        NotFoundError for a network without a single term."""
        h, r = C.c_void_p(), _lib.Mutation()
        call("cw_network_mutate", self._h, float(which), float(how), C.byref(h), C.byref(r))
        return Network(h, self.names), self._record(r)

    def rewire(self, draws):
        """Network::rewire (network.rs:503-575) on a copy, draws = (mode, which, source, sign, how)."""
        d = np.ascontiguousarray(draws, np.float64)
        if d.shape != (5,):
            raise ConfigError("rewiring takes five draws")
        h, r = C.c_void_p(), _lib.Mutation()
        call("cw_network_rewire", self._h, ptr(d), C.byref(h), C.byref(r))
        return Network(h, self.names), self._record(r)

    @staticmethod
    def step_clones(nets, clone, state, inputs, dt, substeps=1):
        """RK4 for cells of many networks at once: row c of state [ncells, S] steps under
        nets[clone[c]] (the per-cell networks of an evolving run), in place."""
        st = np.ascontiguousarray(state, np.float64)
        ins = np.ascontiguousarray(inputs, np.float64)
        cl = np.ascontiguousarray(clone, np.int32)
        handles = (C.c_void_p * len(nets))(*[n.handle.value for n in nets])
        call("cw_network_step_clones", len(nets), handles, st.shape[0], ptr(cl), ptr(st), ptr(ins), float(dt),
             int(substeps))
        if st is not state:
            state[...] = st
        return state

    def mechanics_batch(self, state):
        """mechanics (network.rs:811-821): target volumes and lambdas."""
        st = np.ascontiguousarray(state, np.float64)
        tgt = np.empty(st.shape[0], np.uint32)
        lam = np.empty(st.shape[0])
        call("cw_network_mechanics_batch", self._h, st.shape[0], ptr(st), ptr(tgt), ptr(lam))
        return tgt, lam


# ============================================================== Simulation
class Simulation:
    """A device-resident Simulation<Running>::step (simulation.rs:1129-1350)
    over a batch of histories (the reference's campaign, src/campaign.rs)."""

    def __init__(self, network: Network, dims, ncells, seeds, *, temperature=10.0, J=None, contact_order=2,
                 target_volume=49, lambda_volume=1.0, surface_target=0, lambda_surface=0.0, seeding=0, seed_side=7,
                 nfields=1, o2_dcoef=1.0, o2_sink_by_type=(0.0, 0.01, 0.01), o2_background_sink=0.0, o2_hold=0, signal_dcoef=1.0,
                 signal_decay=0.01, signal_secretion=0.05, hypoxic_level=0.1, tolerance=1e-6, precision=FP32_DC,
                 omega=None, inner_sweeps=0, relax_every=1, dt=0.01, substeps=8, sweeps=1, death_threshold=0.25,
                 necrotic_type=-1, use_graphs=True, divide=True, max_cells=2000, spare_cells=0,
                 waste_production=0.0, necrotic_production=0.0, necrotic_release_for=-1, subsweeps=1,
                 o2_uptake=0.0, divide_every=1, vessel_radius=0, stop_rule=STOP_RESIDUAL, first_tolerance=0.0,
                 cycle_median=0.0, cycle_spread=0.0, debris_loss=0.0, still_medium=0.0, exposure_intensity=0.0,
                 exposure_uptake=0.0, exposure_start=0, exposure_on=0, exposure_off=0, mutation_rate=0.0,
                 rewiring=0.0, field_off=False, differentiated_type=-1, apoptotic_type=-1, lineage=False,
                 error_tolerance=0.0, suppress_before=0, tracing_at=None):
        self.dims, w, h, z = _dims(dims)
        self._keep = [w, h, z]
        nc = np.array(ncells, np.uint32)
        sd = np.array(seeds, np.uint64)
        J = np.ascontiguousarray(J, np.float64)
        sink = np.zeros(8)
        sink[:len(o2_sink_by_type)] = o2_sink_by_type
        self._keep += [nc, sd, J, sink]
        cfg = _lib.SimConfig(len(self.dims), ptr(w).value, ptr(h).value, ptr(z).value, ptr(nc).value, ptr(sd).value,
                             float(temperature), int(J.shape[0]), ptr(J).value, int(contact_order),
                             int(target_volume), float(lambda_volume), int(surface_target), float(lambda_surface),
                             int(seeding), int(seed_side), int(nfields), float(o2_dcoef), ptr(sink).value, float(o2_background_sink),
                             int(o2_hold), float(signal_dcoef), float(signal_decay), float(signal_secretion),
                             float(hypoxic_level), float(tolerance), int(precision), float(omega or 0.0), int(inner_sweeps),
                             int(relax_every), float(dt), int(substeps), int(sweeps), float(death_threshold),
                             int(necrotic_type), int(bool(use_graphs)), int(bool(divide)), int(max_cells),
                             int(spare_cells), float(waste_production), float(necrotic_production),
                             int(necrotic_release_for), int(subsweeps), float(o2_uptake), int(divide_every),
                             int(vessel_radius), int(stop_rule), float(first_tolerance), float(cycle_median),
                             float(cycle_spread), float(debris_loss), float(still_medium), float(exposure_intensity),
                             float(exposure_uptake), int(exposure_start), int(exposure_on), int(exposure_off),
                             float(mutation_rate), float(rewiring), int(bool(field_off)), int(differentiated_type),
                             int(apoptotic_type), int(bool(lineage)), float(error_tolerance), int(suppress_before),
                             int(tracing_at is not None), int(tracing_at or 0))
        handle = C.c_void_p()
        call("cw_sim_create", C.byref(cfg), network.handle, C.byref(handle))
        self._h = handle
        self.network = network

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._LIB is not None:
            lib().cw_sim_destroy(h)
            self._h = None

    def step(self, n=1):
        call("cw_sim_step", self._h, int(n))

    def set_lesion(self, network: "Network", at, radius, centre=None):
        """A lesion (Lesion, simulation.rs:348-360): at the start of step `at`
        every living cell whose centre lies within `radius` of `centre` (the
        box's centre when None) joins one new clone carrying `network`, fresh."""
        cx, cy = (float("nan"), float("nan")) if centre is None else (float(centre[0]), float(centre[1]))
        call("cw_sim_set_lesion", self._h, network.handle, int(at), float(radius), cx, cy)
        self._lesion_network = network  # the simulation reads it until it is destroyed

    def tuning(self):
        """What the autotuner chose: factors per history (oxygen, signal), blocking depth and window, still tuning."""
        n = len(self.dims)
        a, b = np.zeros(n), np.zeros(n)
        depth, window, active = C.c_int32(), C.c_int32(), C.c_int32()
        call("cw_sim_tuning", self._h, ptr(a), ptr(b), C.byref(depth), C.byref(window), C.byref(active))
        return dict(omega_o2=a, omega_signal=b, depth=depth.value, window=window.value, tuning=bool(active.value))

    def graph_info(self):
        """(steps replayed from CUDA graphs, budget misses, outer-iteration budgets)."""
        steps, misses = C.c_uint64(), C.c_uint64()
        budgets = np.zeros(2, np.int32)
        call("cw_sim_graph_info", self._h, C.byref(steps), C.byref(misses), ptr(budgets))
        return steps.value, misses.value, budgets

    def stats(self):
        out = np.empty((len(self.dims), 4))
        call("cw_sim_stats", self._h, ptr(out))
        return out

    def lattice_handle(self):
        h = C.c_void_p()
        call("cw_sim_lattice", self._h, C.byref(h))
        return h

    def field_handle(self, which=0):
        h = C.c_void_p()
        call("cw_sim_field", self._h, int(which), C.byref(h))
        return h

    def grid(self, hist=0):
        w, h, d = self.dims[hist]
        out = np.empty(w * h * d, np.int32)
        call("cw_lattice_download", self.lattice_handle(), hist, ptr(out))
        return out.reshape(d, h, w)

    def lattice(self):
        """The driver's lattice, as a CpmLattice view (owned by this Simulation)."""
        return CpmLattice.borrowed(self.lattice_handle(), self.dims, self)

    def field_values(self, which=0, hist=0):
        w, h, d = self.dims[hist]
        out = np.empty(w * h * d)
        call("cw_field_download", self.field_handle(which), hist, VALUES, ptr(out))
        return out

    def records_match_grid(self, hist=0):
        ok = C.c_int32()
        call("cw_lattice_verify", self.lattice_handle(), hist, C.byref(ok))
        return bool(ok.value)

    def measure(self):
        """Simulation::measure (measure.rs:133-236) of every history: a dict each."""
        arr = (_lib.Measurements * len(self.dims))()
        call("cw_sim_measure", self._h, arr)
        keys = [f for f, _ in _lib.Measurements._fields_]
        return [{k: getattr(m, k) for k in keys} for m in arr]

    def network_state(self, n, hist=0):
        """The protein levels of records 0..n-1 of a history, [n, S]."""
        out = np.empty((int(n), self.network.S))
        call("cw_sim_network_state", self._h, int(hist), int(n), ptr(out))
        return out

    def touches_edge(self):
        """touches_the_edge (simulation.rs:2165-2198) of every history, on the device."""
        out = np.zeros(len(self.dims), np.int32)
        call("cw_sim_touches_edge", self._h, ptr(out))
        return out.astype(bool)

    def clones(self, n, hist=0):
        """The clone of records 0..n-1 of a history (0: the founding network)."""
        out = np.zeros(int(n), np.int32)
        call("cw_sim_clones", self._h, int(hist), int(n), ptr(out))
        return out

    def clone_count(self):
        """Clones in the whole batch: the founders' and every one founded since."""
        n = C.c_uint32()
        call("cw_sim_clone_count", self._h, C.byref(n))
        return n.value

    def traced_clones(self, hist=0):
        """traced_clones (simulation.rs:2407-2421): (mark, cells in the layer
        carrying it) for every mark still carried, in the order of the marks."""
        n = C.c_uint32()
        call("cw_sim_traced", self._h, int(hist), 0, None, None, C.byref(n))
        k = n.value
        marks, cells = np.zeros(max(k, 1), np.uint32), np.zeros(max(k, 1), np.uint64)
        call("cw_sim_traced", self._h, int(hist), k, ptr(marks), ptr(cells), C.byref(n))
        return [(int(marks[i]), int(cells[i])) for i in range(k)]

    def clone_records(self):
        """Every clone founded during the run so far, in order: (parent clone,
        mutation record); a lesion's clone is (-1, {"lesion": True}), a
        suppressed mutation's record carries "suppressed": True."""
        n = C.c_uint32()
        call("cw_sim_clone_records", self._h, C.byref(n), None, None)
        k = n.value
        parent = np.zeros(max(k, 1), np.int32)
        recs = (_lib.Mutation * max(k, 1))()
        call("cw_sim_clone_records", self._h, C.byref(n), ptr(parent), recs)
        out = []
        for i in range(k):
            if recs[i].change < 0:
                out.append((int(parent[i]), {"lesion": True}))
                continue
            rec = self.network._record(recs[i])
            if recs[i].suppressed:
                rec["suppressed"] = True
            out.append((int(parent[i]), rec))
        return out

    def cycle(self, n, hist=0):
        """(began, due) of records 0..n-1 of a history: each cell's cycle."""
        began, due = np.empty(int(n), np.int32), np.empty(int(n), np.int32)
        call("cw_sim_cycle", self._h, int(hist), int(n), ptr(began), ptr(due))
        return began, due


# ============================================================== Fit (adjoint)
class Fit:
    """Loss and gradient of a frozen lattice's step (cw_fit_*): parameters are
    D, the uptake k of types 1..3 and the first `network_params` network rates.
    The reference has no counterpart; see include/cellweave_b200.h."""

    def __init__(self, lattice: CpmLattice, network: Network, *, dcoef=1.0, uptake=(0.01, 0.005, 0.0),
                 vessel_value=1.0, vessel_x=0, egf=0.2, signal_dcoef=1.0, signal_decay=0.01, secretion=0.05,
                 steps=2000, checkpoint_every=100, dt=0.01, nbins=64, bin_width=16.0, hypoxic_level=0.1, tau=0.02,
                 signal_weight=1.0, tolerance=1e-8, adjoint_tolerance=1e-10, precision=FP32_DC, omega=None,
                 network_params=32):
        cfg = _lib.FitConfig(float(dcoef), (C.c_double * 3)(*uptake), float(vessel_value), int(vessel_x),
                             float(egf), float(signal_dcoef), float(signal_decay), float(secretion), int(steps),
                             int(checkpoint_every), float(dt), int(nbins), float(bin_width), float(hypoxic_level),
                             float(tau), float(signal_weight), float(tolerance), float(adjoint_tolerance),
                             int(precision), float(omega or 0.0), int(network_params))
        handle = C.c_void_p()
        call("cw_fit_create", lattice.handle, network.handle, C.byref(cfg), C.byref(handle))
        self._h = handle
        self._keep = (lattice, network)
        self.nbins = int(nbins)
        n = C.c_int32()
        call("cw_fit_nparams", self._h, C.byref(n))
        self.nparams = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._LIB is not None:
            lib().cw_fit_destroy(h)
            self._h = None

    @property
    def params(self):
        p = np.empty(self.nparams)
        call("cw_fit_get_params", self._h, ptr(p))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float64)
        call("cw_fit_set_params", self._h, ptr(p))

    def set_target(self, hypoxic, signal):
        h = np.ascontiguousarray(hypoxic, np.float64)
        g = np.ascontiguousarray(signal, np.float64)
        call("cw_fit_set_target", self._h, ptr(h), ptr(g))

    def forward(self):
        loss = C.c_double()
        h, g = np.empty(self.nbins), np.empty(self.nbins)
        call("cw_fit_forward", self._h, C.byref(loss), ptr(h), ptr(g))
        return loss.value, h, g

    def gradient(self):
        loss = C.c_double()
        g = np.empty(self.nparams)
        call("cw_fit_gradient", self._h, C.byref(loss), ptr(g))
        return loss.value, g
