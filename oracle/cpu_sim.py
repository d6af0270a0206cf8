"""One history of the benchmark workload stepped on the CPU oracle.

TEST INFRASTRUCTURE / CPU BASELINE ONLY: ``bench.py``'s CPU leg and its
reference arm time this; no product path imports it.  Every step runs the
reference's own algorithms as restated in ``cw_oracle.c``: the red-black FP64
SOR of pde.rs:245-405 (residual stopping rule, first-order sink), the
mean_per_cell of coupling.rs:164-182, the RK4 of network.rs:777-799 with the
mechanics of network.rs:811-821, and the sequential random-site Metropolis
sweep of cpm.rs:748-838, in the order of simulation.rs:1129-1350.
"""
from __future__ import annotations

import tomllib

import math

import numpy as np

from . import oracle as O


def seed_history(cfg, w, h, d, n, seed):
    """Squares (cubes) of the workload's side at random free places (seeding 0),
    packed with a gap of two (1), or cubes in a ball (2); types 1..K-1 (the
    necrotic type excluded) drawn at random."""
    rng = np.random.default_rng(seed)
    s = int(cfg.get("seed_side", 7))
    grid = np.zeros((d, h, w), np.int32)
    K = cfg["J"].shape[0]
    nec = cfg.get("necrotic_type", -1)
    ntypes = max(1, (nec - 1) if nec and nec > 0 else K - 1)
    if cfg.get("seeding", 0) == 4:
        # a sheet (Seeding::Sheet, simulation.rs:732-740): side x side blocks of
        # normal tissue (type 2) tiling the box row by row
        types = [0]
        for y in range(0, h, s):
            for x in range(0, w, s):
                grid[0, y:y + s, x:x + s] = len(types)
                types.append(2)
        return grid, np.array(types, np.int32)
    if cfg.get("o2_hold", 0) == 1:
        grid[:, :, w // 2] = -1
    z_, y_, x_ = np.mgrid[0:d, 0:h, 0:w]
    if cfg.get("o2_hold", 0) == 4:
        # a vessel: an obstacle disc at the centre through every slice (add_obstacle_disc, cpm.rs:389-415)
        rv = int(cfg["vessel_radius"])
        grid[(x_ - w // 2) ** 2 + (y_ - h // 2) ** 2 <= rv * rv] = -1
    if cfg.get("seeding", 0) == 3:
        # one cell (Seeding::Single, simulation.rs:666-694; add_ball, cpm.rs:323-354)
        cx = w // 2 + (int(cfg["vessel_radius"]) + s if cfg.get("o2_hold", 0) == 4 else 0)
        ball = ((x_ - cx) ** 2 + (y_ - h // 2) ** 2 + (z_ - d // 2) ** 2 <= s * s) & (grid != -1)
        grid[ball] = 1
        return grid, np.array([0, 1], np.int32)
    types = [0]
    sz = s if d > 1 else 1

    def free(x, y, z):
        return (x + s <= w and y + s <= h and z + sz <= d and not grid[z:z + sz, y:y + s, x:x + s].any())

    def put(x, y, z):
        grid[z:z + sz, y:y + s, x:x + s] = len(types)
        types.append(1 + int(rng.integers(ntypes)))

    mode = cfg.get("seeding", 0)
    if mode == 1:
        pitch = s + 2
        for z in range(0, d - sz + 1, pitch if d > 1 else 1):
            for y in range(1, h - s + 1, pitch):
                for x in range(1, w - s + 1, pitch):
                    if len(types) - 1 < n and free(x, y, z):
                        put(x, y, z)
    elif mode == 2 and d > 1:
        R = (3.0 * n * s ** 3 / (4.0 * np.pi)) ** (1 / 3) + 0.5 * s
        for z in range(0, d - s + 1, s):
            for y in range(0, h - s + 1, s):
                for x in range(0, w - s + 1, s):
                    if ((x + s / 2 - w / 2) ** 2 + (y + s / 2 - h / 2) ** 2 + (z + s / 2 - d / 2) ** 2 <= R * R
                            and len(types) - 1 < n and free(x, y, z)):
                        put(x, y, z)
    else:
        tries = 0
        while len(types) - 1 < n and tries < 200 * n + 1000:
            tries += 1
            x, y = int(rng.integers(w - s + 1)), int(rng.integers(h - s + 1))
            z = int(rng.integers(d - sz + 1)) if d > 1 else 0
            if free(x, y, z):
                put(x, y, z)
    return grid, np.array(types, np.int32)


def lesion_joining(grid, types, volume, leaving, centre, radius):
    """The cells a lesion takes (place_lesion, simulation.rs:1920-1962) on a
    plane grid [h][w]: every cell holding pixels whose type is not one of
    `leaving` (necrotic, differentiated, apoptotic) and whose centre of mass,
    x + 1/2 and y + 1/2 summed in row order over its pixels and divided by
    their count, lies within `radius` of `centre` (the box's centre when
    None).  Record ids in increasing order."""
    g = np.asarray(grid)
    h, w = g.shape
    cx, cy = (w / 2.0, h / 2.0) if centre is None else (float(centre[0]), float(centre[1]))
    ncap = len(types)
    y, x = np.mgrid[0:h, 0:w]
    ok = (g >= 0) & (g < ncap)
    ids = g[ok]
    # bincount adds the weights in array order: the reference's row order
    sx = np.bincount(ids, weights=(x[ok] + 0.5), minlength=ncap)
    sy = np.bincount(ids, weights=(y[ok] + 0.5), minlength=ncap)
    n = np.bincount(ids, minlength=ncap)
    out = []
    for cid in range(1, ncap):
        alive = volume[cid] > 0 and int(types[cid]) not in [t for t in leaving if t >= 0]
        if alive and n[cid] > 0 and math.hypot(sx[cid] / n[cid] - cx, sy[cid] / n[cid] - cy) <= radius:
            out.append(cid)
    return out


def measure_records(grid, types, volume, used, hypoxia, necrotic, o2_hold, mcs, leaving=(), clone=None,
                    clone_lesion=None):
    """measure.rs:133-236 on a lattice's records: counts of cycling (hypoxia
    response under 0.45), quiescent and necrotic cells with pixels, born (every
    record assigned), gone (dead and resorbed to nothing), equivalent radii (a
    disc in the plane, a ball in a volume); viable_depth as measure.rs:171-199
    reads it for the source the hold stands for (bath-like faces and bath: the
    tissue radius less the necrotic one; a held row: the living area over the
    columns living cells hold; a held column: over twice the rows)."""
    d, h, w = grid.shape
    ids = np.arange(1, used)
    vol = volume[1:used].astype(np.int64)
    dead = (types[1:used] == necrotic) if necrotic >= 0 else np.zeros(used - 1, bool)
    # cells leaving the layer or breaking up (differentiated, apoptotic types)
    diff = (types[1:used] == leaving[0]) if len(leaving) > 0 and leaving[0] >= 0 else np.zeros(used - 1, bool)
    apop = (types[1:used] == leaving[1]) if len(leaving) > 1 and leaving[1] >= 0 else np.zeros(used - 1, bool)
    has = vol > 0
    live = has & ~dead & ~diff & ~apop
    cyc = live & (hypoxia[1:used] < 0.45)
    m = dict(mcs=mcs, cycling=int(cyc.sum()), quiescent=int((live & ~cyc).sum()), necrotic=int((has & dead).sum()),
             born=int(used - 1), gone=int((~has & (dead | diff | apop)).sum()),
             differentiating=int((has & diff).sum()), apoptotic=int((has & apop).sum()))
    if clone is not None:
        m["clones"] = int(np.unique(clone[1:used][live]).size)
    else:
        m["clones"] = 1 if live.any() else 0
    # living cells descended from a lesion (lesion_cells, evolution.rs:182-197)
    m["lesion"] = 0
    if clone is not None and clone_lesion is not None:
        flags = np.asarray(clone_lesion, bool)
        m["lesion"] = int(flags[clone[1:used][live]].sum())
    leaving_area = int(vol[has & (diff | apop)].sum())
    m["vessel"] = int((grid == -1).sum()) if o2_hold in (1, 4) else 0
    living_area, dead_area = int(vol[live].sum()), int(vol[has & dead].sum())

    def radius(size):
        if d <= 1:
            return float(np.sqrt(size / np.pi))
        if o2_hold == 4:
            return float(np.sqrt(size / (np.pi * d)))
        return float(np.cbrt(3.0 * size / (4.0 * np.pi)))

    m["tissue_radius"] = radius(m["vessel"] + living_area + dead_area + leaving_area)
    m["necrotic_radius"] = radius(dead_area)
    if o2_hold in (0, 1):
        alive_id = np.zeros(int(types.size), bool)
        alive_id[ids[live]] = True
        g = grid.reshape(d, h, w)
        lv = (g > 0) & alive_id[np.clip(g, 0, None)]
        lines = lv.any(axis=(0, 1)).sum() if o2_hold == 0 else lv.any(axis=(0, 2)).sum()
        m["viable_depth"] = 0.0 if lines == 0 else living_area / (float(lines) * (1.0 if o2_hold == 0 else 2.0))
    elif o2_hold == 4:
        m["viable_depth"] = radius(m["vessel"] + living_area) - radius(m["vessel"])
    else:
        m["viable_depth"] = m["tissue_radius"] - m["necrotic_radius"]
    return m


class CpuHistory:
    def __init__(self, cfg, k):
        from cellweave_b200 import synthetic  # the same synthetic network text the device runs
        self.cfg = cfg
        w, h, d = cfg["dims"][k]
        self.dims = (w, h, d)
        self.seed = int(cfg["seeds"][k])
        grid, types = seed_history(cfg, w, h, d, int(cfg["ncells"][k]), self.seed)
        self.divide = bool(cfg.get("divide", True))
        self.max_cells = int(cfg.get("max_cells", 2000) or 2000)
        spare = int(cfg.get("spare_cells", 0) or self.max_cells) if self.divide else 0
        self.used = len(types)
        self.ncap = len(types) + spare
        J = np.asarray(cfg["J"], float)
        self.lat = O.Lattice(grid, (w, h, d), self.ncap, J, cfg["temperature"], cfg.get("contact_order", 1))
        self.lat.type[:len(types)] = types
        self.lat.recount()
        self.lat.volume[0] = 0
        self.lat.target[:self.used] = cfg["target_volume"]
        if cfg.get("seeding", 0) == 3 or cfg["target_volume"] <= 0:
            self.lat.target[:self.used] = self.lat.volume[:self.used]  # a seeded cell aims at what it holds
        self.lat.target[0] = 0
        self.lat.lam[:self.used] = cfg["lambda_volume"]
        self.lat.lam[0] = 0.0
        if cfg.get("surface_target", 0) > 0:
            self.lat.enable_surface(np.full(self.ncap, cfg["surface_target"], np.int32),
                                    np.full(self.ncap, cfg.get("lambda_surface", 0.0)))
        n = w * h * d
        self.o2 = O.Field(w, h, d, cfg["o2_dcoef"], 0.0, 0.0 if cfg.get("o2_hold", 0) == 4 else 1.0)
        z, y, x = np.mgrid[0:d, 0:h, 0:w]
        hold = cfg.get("o2_hold", 0)
        held = (y == 0) if hold == 0 else (x == w // 2) if hold == 1 else (
            (x == 0) | (y == 0) | (z == 0) | (x == w - 1) | (y == h - 1) | (z == d - 1)) if hold == 2 else (
            grid == -1) if hold == 4 else np.zeros_like(y, bool)  # 4: the vessel; 3: the bath, taken every step
        self.o2.held[:] = held.reshape(-1)
        self.o2.values[self.o2.held == 1] = 1.0
        self.o2.lin_sink = np.zeros(n)
        self.sig = None
        if cfg.get("nfields", 1) == 2:
            self.sig = O.Field(w, h, d, cfg["signal_dcoef"], cfg["signal_decay"], 0.0)
        # the released fields (simulation.rs:2057-2113): they diffuse as oxygen does
        self.wst = O.Field(w, h, d, cfg["o2_dcoef"], 0.0, 0.0) if cfg.get("waste_production", 0.0) > 0 else None
        self.nfc = O.Field(w, h, d, cfg["o2_dcoef"], 0.0, 0.0) if cfg.get("necrotic_production", 0.0) > 0 else None
        self.cell_wst = self.cell_nfc = None
        # an exposure's stress (simulation.rs:802-840): diffusing as oxygen does, from zero
        self.str = O.Field(w, h, d, cfg["o2_dcoef"], 0.0, 0.0) if cfg.get("exposure_intensity", 0.0) > 0 else None
        self.str_level = 0.0
        self.cell_str = None
        spec = cfg.get("network_spec") or tomllib.loads(cfg.get("network_toml") or
                                                          synthetic.network_toml(cfg["S"], cfg["S"]))
        # the network's reference volume: the seeded cell's (simulation.rs:726-733) or the target
        self.refvol = (int(self.lat.volume[1]) if cfg.get("seeding", 0) == 3 else
                       int(cfg["seed_side"]) ** 2 if cfg.get("seeding", 0) == 4 else int(cfg["target_volume"]))
        self.net = O.compile_network(spec, self.refvol)
        self.state = np.tile(self.net.initial, (self.ncap, 1))
        # an evolving history (simulation.rs:1655-1700): every record's clone and
        # each clone's network table, mutated or rewired at divisions
        self.mutation_rate = float(cfg.get("mutation_rate", 0.0) or 0.0)
        self.rewiring = float(cfg.get("rewiring", 0.0) or 0.0)
        self.clone = np.zeros(self.ncap, np.int64)
        self.clone_specs = [spec]
        self.clone_nets = [self.net]
        self.clone_lesion = [False]
        self.suppress_before = int(cfg.get("suppress_before", 0) or 0)
        # a lesion (simulation.rs:348-360): its network, step, radius, centre
        self.lesion_spec = cfg.get("lesion_spec")
        self.lesion_at = int(cfg.get("lesion_at", -1))
        self.lesion_radius = float(cfg.get("lesion_radius", 0.0))
        self.lesion_centre = cfg.get("lesion_centre")
        # lineage tracing (types.rs:208-214): every record's mark, -1 for none
        self.tracing_at = cfg.get("tracing_at")
        self.marks = np.full(self.ncap, -1, np.int64)
        # a lineage (a sheet, simulation.rs:780-785): every seeded cell its own
        # clone; its cells step under the one network
        self.lineage = bool(cfg.get("lineage", False))
        if self.lineage:
            self.clone[:self.used] = np.arange(self.used)
            self.clone_specs = [spec] * self.ncap
            self.clone_nets = [self.net] * self.ncap
            self.clone_lesion = [False] * self.ncap
        self.leaving = (int(cfg.get("differentiated_type", -1)), int(cfg.get("apoptotic_type", -1)))
        self.div_rng = np.random.default_rng(self.seed * 7 + 13)
        # a cell's cycle (simulation.rs:1055-1056): none behind the cells the tissue starts with
        self.began = np.zeros(self.ncap, np.int64)
        self.due = np.zeros(self.ncap, np.int64)
        # debris loss (simulation.rs:1226-1275): the dead kept, the debt to the fluid
        self.kept = np.zeros(self.ncap, bool)
        self.debris_owed = 0.0
        self.bath_level = 1.0  # a still medium's level (simulation.rs:1054)
        sink = np.zeros(8)
        sink[:len(cfg["o2_sink_by_type"])] = cfg["o2_sink_by_type"]
        self.sink = sink
        self.steps = 0
        self.died_at = np.full(self.ncap, -1, np.int64)

    def measure(self):
        """Simulation::measure (measure.rs:103-236) of this history, with the
        device step's reading of viable_depth for each oxygen hold."""
        return measure_records(self.lat.grid.reshape(self.dims[2], self.dims[1], self.dims[0]), self.lat.type,
                               self.lat.volume, self.used, self.state[:, self.net.hypoxia],
                               self.cfg.get("necrotic_type", -1), self.cfg.get("o2_hold", 0), max(self.steps - 1, 0),
                               leaving=self.leaving,
                               clone=self.clone if self._tracked() else None, clone_lesion=self.clone_lesion)

    def _in_layer(self):
        """in_layer (simulation.rs:2400-2405) of every record: holding pixels,
        neither necrotic nor apoptotic."""
        t, vol = self.lat.type, self.lat.volume
        nec, apop = self.cfg.get("necrotic_type", -1), self.leaving[1]
        ok = (vol > 0) & (t != nec) if nec >= 0 else vol > 0
        if apop >= 0:
            ok &= t != apop
        ok = ok.copy()
        ok[0] = False
        return ok

    def _mark_every_cell(self):
        """mark_every_cell (simulation.rs:1908-1918): every cell in the layer
        marked with its slot (its id less one), every other record none."""
        ids = np.arange(self.ncap)
        self.marks = np.where(self._in_layer(), ids - 1, -1)

    def traced_clones(self):
        """traced_clones (simulation.rs:2407-2421): (mark, cells in the layer)."""
        m = self.marks[self._in_layer() & (self.marks >= 0)]
        u, c = np.unique(m, return_counts=True)
        return [(int(a), int(b)) for a, b in zip(u, c)]

    def _tracked(self):
        return (self.lineage or self.mutation_rate > 0 or self.lesion_spec is not None
                or self.tracing_at is not None)

    def _place_lesion(self):
        """place_lesion (simulation.rs:1920-1970): every living cell whose
        centre of mass (x + 1/2, y + 1/2 summed in row order over its pixels,
        over their count) lies within the radius of the centre (the box's
        when none is given) joins one new clone carrying the lesion's
        network, its state that network's initial one."""
        w, h = self.dims[0], self.dims[1]
        leaving = (self.cfg.get("necrotic_type", -1),) + tuple(self.leaving)
        joining = lesion_joining(self.lat.grid.reshape(h, w), self.lat.type, self.lat.volume, leaving,
                                 self.lesion_centre, self.lesion_radius)
        if not joining:
            return
        self.clone_specs.append(self.lesion_spec)
        self.clone_nets.append(O.compile_network(self.lesion_spec, self.refvol))
        self.clone_lesion.append(True)
        k = len(self.clone_specs) - 1
        for cid in joining:
            self.clone[cid] = k
            self.state[cid] = self.clone_nets[k].initial

    def _settle_released(self, field, per_cell):
        """settle_released (simulation.rs:2546-2570): production from the cells
        that release, the bath held at zero, relaxed; the per-cell means."""
        c = self.cfg
        g = self.lat.grid
        field.production = O.apply_production(g, per_cell)
        field.held[:] = 0
        field.hold_bath(g == 0, 0.0)
        field.relax(c["tolerance"], 200_000, omega=c.get("omega") or 0.0, stop=c.get("stop_rule", 1), threads=1)
        return O.mean_per_cell(g, field.values, self.ncap)

    def step(self):
        c = self.cfg
        if self.lesion_spec is not None and self.steps == self.lesion_at:
            self._place_lesion()  # before anything else in the step (simulation.rs:1135-1137)
        if self.tracing_at is not None and self.steps == self.tracing_at:
            self._mark_every_cell()  # simulation.rs:1138-1140
        g = self.lat.grid
        t = self.lat.type
        cells = g > 0
        sink = np.zeros(g.size)
        sink[cells] = self.sink[t[g[cells]]]
        sink[g == 0] = c.get("o2_background_sink", 0.0)
        self.o2.lin_sink = sink
        if c.get("o2_uptake", 0.0) > 0:
            # apply_uptake (coupling.rs:22-40): every living pixel; around a vessel the medium too
            nec0 = c.get("necrotic_type", -1)
            up = np.zeros(g.size)
            live = cells & (t[np.clip(g, 0, None)] != nec0)
            up[live] = c["o2_uptake"]
            if c.get("o2_hold", 0) == 4:
                up[g == 0] = c["o2_uptake"]
            self.o2.uptake = up
        field_off = bool(c.get("field_off", False))
        if c.get("o2_hold", 0) == 3 and not field_off:
            # the bath as the lattice stands (declare_sources, simulation.rs:2138-2146)
            self.o2.held[:] = 0
            self.o2.hold_bath(g == 0, self.bath_level)
        omega = c.get("omega") or 0.0
        tol, most = c["tolerance"], 200_000
        if self.steps == 0 and c.get("first_tolerance", 0.0) > 0:
            tol, most = min(c["first_tolerance"], tol), 2_000_000  # start() (simulation.rs:1068-1083)
        # with the field off nothing consumes: the oxygen stays at its start (simulation.rs:2127-2131)
        rc = 0 if field_off else self.o2.relax(tol, most, omega=omega, stop=c.get("stop_rule", 1), threads=1)[0]
        if c.get("still_medium", 0.0) > 0:
            self._settle_bath_level()
            if most == 2_000_000:
                # start() settled the level after its solve; the first step solves against it
                self.o2.held[:] = 0
                self.o2.hold_bath(g == 0, self.bath_level)
                rc, _ = self.o2.relax(c["tolerance"], 200_000, omega=omega, stop=c.get("stop_rule", 1), threads=1)
                self._settle_bath_level()
        o2m = O.mean_per_cell(g, self.o2.values, self.ncap)
        nec = c.get("necrotic_type", -1)
        ldiff, lapop = self.leaving
        leaving_cell = ((t == ldiff) & (ldiff >= 0)) | ((t == lapop) & (lapop >= 0))
        alive = (self.lat.volume > 0) & (t != nec) & ~leaving_cell
        alive[0] = False
        # cells leaving the layer shed, those breaking up fragment (simulation.rs:1209-1262)
        going = np.nonzero(leaving_cell & (self.lat.volume > 0))[0]
        going = going[going > 0]
        if len(going):
            rate = np.where(t[going] == lapop, 8, 6)
            self.lat.target[going] = np.maximum(self.lat.volume[going] - rate, 0)
            self.lat.lam[going] = c["lambda_volume"]
        if self.str is not None:
            self.cell_str = self._settle_stress()
        if self.sig is not None:
            sec = np.where(alive & (o2m < c["hypoxic_level"]), c["signal_secretion"], 0.0)
            self.sig.production = O.apply_production(g, sec)
            self.sig.relax(c["tolerance"], 200_000, omega=omega, stop=c.get("stop_rule", 1), threads=1)
        if self.wst is not None:
            self.cell_wst = self._settle_released(self.wst, np.where(alive, c["waste_production"], 0.0))
        if self.nfc is not None:
            rel = c.get("necrotic_release_for", -1)
            releasing = (rel < 0) | (self.died_at < 0) | (self.steps <= self.died_at + rel)
            dead = (t == nec) & (self.lat.volume > 0) & releasing
            dead[0] = False
            self.cell_nfc = self._settle_released(self.nfc, np.where(dead, c["necrotic_production"], 0.0))
        # a necrotic cell gives up 2 pixels a step until it is gone (simulation.rs:1230-1262)
        loss = c.get("debris_loss", 0.0)
        if nec >= 0:
            dying = np.nonzero((t == nec) & (self.lat.volume > 0))[0]
            dying = dying[dying > 0]
            if loss > 0:
                # the dead keep what they held when kept (simulation.rs:1226-1244)
                new = dying[~self.kept[dying]]
                self.kept[new] = True
                self.lat.target[new] = self.lat.volume[new]
                self.lat.lam[new] = c["lambda_volume"]
            else:
                self.lat.target[dying] = np.maximum(self.lat.volume[dying] - 2, 0)
                self.lat.lam[dying] = c["lambda_volume"]
        idx = np.nonzero(alive)[0]
        if len(idx):
            ins = np.zeros((len(idx), 6))
            ins[:, 0] = o2m[idx]
            ins[:, 1] = 0.2
            # crowding (simulation.rs:2523-2527): 1 - volume / reference volume, clamped
            ins[:, 2] = np.clip(1.0 - self.lat.volume[idx] / float(max(self.refvol, 1)), 0.0, 1.0)
            if self.cell_str is not None:
                ins[:, 3] = self.cell_str[idx]
            if self.cell_wst is not None:
                ins[:, 4] = self.cell_wst[idx]
            if self.cell_nfc is not None:
                ins[:, 5] = self.cell_nfc[idx]
            st = np.ascontiguousarray(self.state[idx])
            if all(n is self.net for n in self.clone_nets):
                O.network_step(self.net, st, ins, c["dt"], c["substeps"])
            else:
                # every clone's cells under its own network, the cells of
                # clones that share one network stepped together
                nets, which = [], np.empty(len(idx), np.int64)
                for j, k in enumerate(self.clone[idx]):
                    net = self.clone_nets[int(k)]
                    for q, n in enumerate(nets):
                        if n is net:
                            which[j] = q
                            break
                    else:
                        nets.append(net)
                        which[j] = len(nets) - 1
                for q, net in enumerate(nets):
                    sel = np.nonzero(which == q)[0]
                    part = np.ascontiguousarray(st[sel])
                    O.network_step(net, part, np.ascontiguousarray(ins[sel]), c["dt"], c["substeps"])
                    st[sel] = part
            self.state[idx] = st
            tg = O.network_mechanics(self.net, st)
            dead = (st[:, self.net.survival] < c.get("death_threshold", 0.25)) if nec >= 0 else np.zeros(len(idx), bool)
            t[idx[dead]] = nec
            self.died_at[idx[dead]] = self.steps
            if loss > 0:
                # kept from the step it dies (simulation.rs:1264-1275)
                nd = idx[dead]
                self.kept[nd] = True
                self.lat.target[nd] = self.lat.volume[nd]
                self.lat.lam[nd] = c["lambda_volume"]
            # apoptosis, then differentiation, each at its node's level as the
            # cell's chance this step (simulation.rs:1276-1296)
            keep = ~dead
            ra, rd = self.net.optional.get("apoptosis", -1), self.net.optional.get("differentiation", -1)
            for j in np.nonzero(keep)[0]:
                if lapop >= 0 and ra is not None and ra >= 0 and self.div_rng.random() < st[j, ra]:
                    t[idx[j]] = lapop
                    keep[j] = False
                elif ldiff >= 0 and rd is not None and rd >= 0 and self.div_rng.random() < st[j, rd]:
                    t[idx[j]] = ldiff
                    keep[j] = False
            live = idx[keep]
            full = np.minimum(tg[keep], 2**31 - 1).astype(np.int64)
            if c.get("cycle_median", 0.0) > 0:
                # grown (simulation.rs:2534-2540)
                b, e = self.began[live], self.due[live]
                span = np.maximum(e - b, 1)
                passed = np.minimum((self.steps - b) / span, 1.0)
                full = np.where(e > b, np.floor(full * (0.5 + 0.5 * passed) + 0.5), full).astype(np.int64)
            self.lat.target[live] = full.astype(np.int32)
            self.lat.lam[live] = c["lambda_volume"]
        if loss > 0:
            self._break_down_debris(loss)
            self._drain_shut_in()
        self.lat.mcs_sequential(self.seed * 1_000_003 + self.steps, c.get("sweeps", 1))
        every = int(c.get("divide_every", 1) or 1)
        if self.divide and (every <= 1 or self.steps % every == 0):
            self._divide_ready_cells()
        self.steps += 1
        return rc

    def _mutate(self, d):
        """A daughter not quite a copy (simulation.rs:1655-1700): one rate of its
        network scaled (Network::mutate) or, with chance `rewiring`, a link
        gained or lost (Network::rewire); a change made founds a clone."""
        which, how = self.div_rng.random(), self.div_rng.random()
        spec = self.clone_specs[int(self.clone[d])]
        if self.rewiring > 0.0:
            u = self.div_rng.random()
            if u < self.rewiring:
                source, sign = self.div_rng.random(), self.div_rng.random()
                new, rec = O.rewire_spec(spec, (u / self.rewiring, which, source, sign, how))
            else:
                new, rec = O.mutate_spec(spec, which, how)
        else:
            new, rec = O.mutate_spec(spec, which, how)
        if rec is None:
            return
        parent = int(self.clone[d])
        if self.steps < self.suppress_before:
            # drawn and recorded, not made: the clone keeps its parent's network
            # (simulation.rs:1671-1694)
            self.clone_specs.append(spec)
            self.clone_nets.append(self.clone_nets[parent])
        else:
            self.clone_specs.append(new)
            self.clone_nets.append(O.compile_network(new, self.refvol))
        self.clone_lesion.append(self.clone_lesion[parent])
        self.clone[d] = len(self.clone_specs) - 1

    def _level_at(self, mcs):
        """Exposure::level_at (types.rs:319-332)."""
        c = self.cfg
        if mcs < c.get("exposure_start", 0):
            return 0.0
        on, off = c.get("exposure_on", 0), c.get("exposure_off", 0)
        if on > 0 and (mcs - c.get("exposure_start", 0)) % max(on + off, 1) >= on:
            return 0.0
        return c["exposure_intensity"]

    def _settle_stress(self):
        """settle_stress (simulation.rs:2015-2055): zero while off; else taken up
        by the living (and the medium around a vessel), held at the level where
        the oxygen is held, solved from scratch and tightly when the level
        changed; the per-cell means."""
        c = self.cfg
        f = self.str
        level = self._level_at(self.steps)
        if level == 0.0:
            f.values[:] = 0.0
            self.str_level = 0.0
        else:
            g, t = self.lat.grid, self.lat.type
            up = np.zeros(f.values.size)
            up[(g > 0) & (t[np.clip(g, 0, None)] != c.get("necrotic_type", -1))] = c["exposure_uptake"]
            if c.get("o2_hold", 0) == 4:
                up[self.lat.grid == 0] = c["exposure_uptake"]
            f.uptake = up
            f.held[:] = self.o2.held
            f.values[f.held == 1] = level
            tol, most = 0.01 * c["exposure_uptake"], 200_000
            if level != self.str_level:
                tol, most = 1e-8, 2_000_000
            f.relax(tol, most, omega=c.get("omega") or 0.0, stop=c.get("stop_rule", 1), threads=1)
            self.str_level = level
        return O.mean_per_cell(self.lat.grid, f.values, self.ncap)

    def _settle_bath_level(self):
        """settle_bath_level (simulation.rs:2114-2125): 1 - inflow / (4 pi D r), r
        the radius of a ball of the free pixels, at zero at least."""
        taken = self.o2.inflow()
        radius = np.cbrt(3.0 * float((self.o2.held == 0).sum()) / (4.0 * np.pi))
        d = self.cfg["still_medium"]
        self.bath_level = max(1.0 - taken / (4.0 * np.pi * d * radius), 0.0) if radius > 0 else 1.0

    def _faces(self):
        """Per direction: (pixels with a neighbour that way, the neighbour's flat index)."""
        w, h, d = self.lat.w, self.lat.h, self.lat.d
        i = np.arange(w * h * d)
        x, y, z = i % w, (i // w) % h, i // (w * h)
        dirs = [(x > 0, i - 1), (x + 1 < w, i + 1), (y > 0, i - w), (y + 1 < h, i + w)]
        if d > 1:
            dirs += [(z > 0, i - w * h), (z + 1 < d, i + w * h)]
        return [(ok, np.where(ok, j, 0)) for ok, j in dirs]

    def _living_around(self, pix, faces):
        """living_around (cpm.rs:709-722) of each pixel in `pix`: [n, 6] neighbour
        ids that are living tissue of another cell (0 where none), and their count."""
        g, t = self.lat.grid, self.lat.type
        nec = self.cfg.get("necrotic_type", -1)
        own = g[pix]
        ids = np.zeros((len(pix), len(faces)), np.int64)
        for k, (ok, j) in enumerate(faces):
            o = np.where(ok[pix], g[j[pix]], 0)
            good = (o > 0) & (o != own)
            good &= t[np.clip(o, 0, None)] != nec
            ids[:, k] = np.where(good, o, 0)
        return ids, (ids > 0).sum(axis=1)

    def _give(self, pix, ids, n, rng):
        """Each pixel to one of its living neighbours, drawn uniformly."""
        pick = np.minimum((rng.random(len(pix)) * n).astype(np.int64), n - 1)
        order = np.cumsum(ids > 0, axis=1) - 1
        taker = ids[np.arange(len(pix)), np.argmax((order == pick[:, None]) & (ids > 0), axis=1)]
        return taker

    def _break_down_debris(self, loss):
        """break_down_debris (simulation.rs:1746-1808): every whole pixel owed
        taken at the dead tissue's edge, up to EDGE_PASSES passes; within a pass
        a uniform draw of the edge without replacement, each taker drawn against
        the lattice at the pass's start."""
        vol = self.lat.volume
        kept = np.nonzero(self.kept & (vol > 0))[0]
        self.debris_owed += loss * float(vol[kept].sum())
        owed = int(np.floor(self.debris_owed))
        if owed <= 0:
            return
        g = self.lat.grid
        keptmask = np.zeros(len(vol), bool)
        keptmask[kept] = True
        pool = np.nonzero((g > 0) & keptmask[np.clip(g, 0, None)])[0]
        held, paid = len(pool), 0
        given = np.zeros(len(vol), np.int64)
        faces = self._faces()
        for _ in range(8):
            ids, n = self._living_around(pool, faces)
            edge, rest = pool[n > 0], pool[n == 0]
            if len(edge) == 0:
                break
            take = min(owed - paid, len(edge))
            chosen = self.div_rng.permutation(len(edge))[:take]
            pix, pids, pn = edge[chosen], ids[n > 0][chosen], n[n > 0][chosen]
            taker = self._give(pix, pids, pn, self.div_rng)
            dead = g[pix]
            g[pix] = taker
            np.subtract.at(vol, dead, 1)
            np.add.at(vol, taker, 1)
            np.add.at(given, dead, 1)
            paid += take
            if paid == owed:
                break
            left = np.ones(len(edge), bool)
            left[chosen] = False
            pool = np.concatenate([rest, edge[left]])
        self.debris_owed = min(self.debris_owed - paid, float(held - paid))
        lost = np.nonzero(given > 0)[0]
        self.lat.target[lost] = np.maximum(self.lat.target[lost] - given[lost], 0)

    def _drain_shut_in(self):
        """drain_shut_in (simulation.rs:1810-1826): medium the bath does not
        reach, with living tissue across a face, to one of those neighbours,
        each drawn against the lattice as it stood."""
        g = self.lat.grid
        scratch = O.Field(self.lat.w, self.lat.h, self.lat.d)
        scratch.hold_bath(g == 0, 1.0)
        shut = np.nonzero((g == 0) & (scratch.held == 0))[0]
        if len(shut) == 0:
            return
        ids, n = self._living_around(shut, self._faces())
        pix, ids, n = shut[n > 0], ids[n > 0], n[n > 0]
        if len(pix) == 0:
            return
        taker = self._give(pix, ids, n, self.div_rng)
        g[pix] = taker
        np.add.at(self.lat.volume, taker, 1)

    def _cycle_length(self):
        """cycle_length (simulation.rs:1739-1745): median x exp(spread z), z by Box and Muller."""
        c = self.cfg
        u, v = 1.0 - self.div_rng.random(), self.div_rng.random()
        z = np.sqrt(-2.0 * np.log(u)) * np.cos(2.0 * np.pi * v)
        return int(max(np.floor(c["cycle_median"] * np.exp(c.get("cycle_spread", 0.0) * z) + 0.5), 1.0))

    def _divide_ready_cells(self):
        """divide_ready_cells (simulation.rs:1603-1716): the living
        cells of at least 1.4 reference volumes whose hypoxia response is under 0.45 split, in
        id order, while the living stay under max_cells; daughters copy the parent's state."""
        c = self.cfg
        nec = c.get("necrotic_type", -1)
        vol, t = self.lat.volume, self.lat.type
        ldiff, lapop = self.leaving
        alive = (vol > 0) & (t != nec) & ~((t == ldiff) & (ldiff >= 0)) & ~((t == lapop) & (lapop >= 0))
        alive[0] = False
        alive[self.used:] = False
        hyp = self.net.hypoxia
        ready = alive & (vol >= 1.4 * self.refvol)
        if hyp is not None and hyp >= 0:
            ready &= self.state[:, hyp] < 0.45
        if c.get("cycle_median", 0.0) > 0:
            ready[:len(self.due)] &= self.due <= self.steps
        living = int(alive.sum())
        born = 0
        for cid in np.nonzero(ready)[0]:
            if living + born >= self.max_cells:
                break
            angle = self.div_rng.random() * np.pi
            if self.lat.d > 1:
                z = 2.0 * angle / np.pi - 1.0
                around = self.div_rng.random() * 2.0 * np.pi
                r = np.sqrt(max(1.0 - z * z, 0.0))
                normal = (r * np.cos(around), r * np.sin(around), z)
            else:
                normal = (np.cos(angle), np.sin(angle), 0.0)
            d, self.used = self.lat.divide_across(int(cid), normal, self.used)
            if d >= 0:
                self.state[d] = self.state[cid]
                self.clone[d] = self.clone[cid]
                self.marks[d] = self.marks[cid]  # simulation.rs:1711
                if self.mutation_rate > 0.0 and self.div_rng.random() < self.mutation_rate:
                    self._mutate(d)
                if c.get("cycle_median", 0.0) > 0:
                    self.began[cid] = self.began[d] = self.steps
                    self.due[cid] = self.steps + self._cycle_length()
                    self.due[d] = self.steps + self._cycle_length()
                born += 1
