"""A cellweave configuration file (crates/io/src/config.rs) run on the device.

``load_sim_config`` reads a configuration as SimConfig does: its fields with
their defaults (config.rs:12-140 and the serde defaults beside them), the
network named relative to the file with its ``extends`` chain followed
(load_network_chain, config.rs:410-447).  ``simulation_from_config`` sets up
the reference's scenario (Simulation::new, simulation.rs:510-1066) where the
device step can run it: one cell seeded in a bath or against a vessel, the
reference's contact energies between medium, tumour, normal and necrotic
cells (ContactEnergy::default, cpm.rs:63-86), oxygen diffusing at 0.2 and
taken up at ``oxygen_uptake`` by every living pixel (and by the stroma around
a vessel), networks stepped eight units of their time a step, division
checked every 20 steps (every step with a cell cycle of its own); an
exposure's stress, waste, necrotic factor, debris loss, a still medium and
daughters that mutate or rewire their networks (mutation_rate, rewiring)
when configured; a sheet of normal tissue with the field off, every cell the
founder of its clone, cells committing to differentiate (or to apoptosis)
at their network's node's level and leaving the layer; a lesion, whose
cells carry a network of their own from the step it appears at; mutations
suppressed before a step (drawn and recorded, not made).  Every other
feature of the file (capillaries, a list of suppressed clones, angiogenesis,
immunity) is refused by name.  ``run`` steps it for ``mcs`` steps or until the tissue touches the
box's edge, writing measurements.csv and the snapshots as the reference
does.

The oxygen is the reference's relax pixel for pixel: FP64 red-black SOR until
no pixel moves by more than 0.01 x uptake a sweep (simulation.rs:79-99; a
zero-order uptake empties the core, where the reference's update floors the
field at zero, which the FP32 defect correction's linear inner solve does not
follow); the first step's solve goes to 1e-8 from the source's level, as
start() does.  One difference stands: the Monte Carlo step is the device's
sub-sweeps (four by default, the kinetics nearest random pixels).
"""
from __future__ import annotations

import math
import os
import tomllib

import numpy as np

from ._lib import ConfigError
from .engine import FP64, STOP_MAX_CHANGE, Network, Simulation, load_network_spec
from .output import MeasurementLog, TraceLog, snapshot, write_snapshot

# SimConfig's fields without a default (config.rs:12-40) and their defaults
REQUIRED = ("width", "height", "mcs", "temperature", "snapshot_interval", "output_dir")
DEFAULTS = dict(depth=1, max_cells=2000, oxygen_source={"kind": "bath"}, oxygen_uptake=0.00002, network=None,
                mutation_rate=0.0, seed=42, seeding={"kind": "single"}, exposure=None, suppress=[],
                suppress_before=None, rewiring=0.0, hours_per_step=None, lesion=None, angiogenesis=None,
                immunity=None, tracing=None, debris_loss=None, sweeps_per_step=1, cycle=None, contact_order=1,
                waste=None, necrotic_factor=None, still_medium=None)

OXYGEN_DIFFUSION = 0.2       # simulation.rs:77
OXYGEN_TOLERANCE = 0.01      # simulation.rs:85
NETWORK_TIME_PER_MCS = 8     # simulation.rs:115
DEATH_THRESHOLD = 0.25       # simulation.rs:118
DIVISION_CHECK_EVERY = 20    # simulation.rs:55
DIVISION_RATIO = 1.4         # simulation.rs:45
OXYGEN_WARMUP_TOLERANCE = 1e-8  # simulation.rs:95
FIRST_CELL_RADIUS = 8        # simulation.rs:65
FIRST_CELL_RADIUS_3D = 3     # simulation.rs:74
MEDIUM, TUMOR, NORMAL, NECROTIC, DIFFERENTIATED, APOPTOTIC = 0, 1, 2, 3, 4, 5

# ContactEnergy::default (cpm.rs:63-86) between the kinds the device step has;
# a differentiated cell costs what a normal one does, an apoptotic one what a
# necrotic one does (ContactEnergy::index, cpm.rs:116-128)
_BASE = np.array([[0.0, 16.0, 16.0, 12.0],
                  [16.0, 2.0, 11.0, 10.0],
                  [16.0, 11.0, 6.0, 12.0],
                  [12.0, 10.0, 12.0, 8.0]])
_AS = [0, 1, 2, 3, 2, 3]
CONTACT = _BASE[np.ix_(_AS, _AS)]


def load_sim_config(path: str) -> dict:
    """SimConfig::from_file (config.rs:300-311) with its defaults; the
    network's path resolved next to the file (config.rs:396-403)."""
    try:
        with open(path, "rb") as fh:
            raw = tomllib.load(fh)
    except OSError as e:
        raise ConfigError(f"{path}: {e}") from None
    except tomllib.TOMLDecodeError as e:
        raise ConfigError(f"{path}: {e}") from None
    missing = [k for k in REQUIRED if k not in raw]
    if missing:
        raise ConfigError(f"{path}: missing field `{missing[0]}`")
    cfg = dict(DEFAULTS)
    cfg.update(raw)
    cfg["path"] = os.path.abspath(path)
    if cfg["network"] is not None:
        cfg["network_path"] = os.path.join(os.path.dirname(cfg["path"]), cfg["network"])
    return cfg


def _refuse(cfg):
    name = os.path.basename(cfg.get("path", "the configuration"))
    src = cfg["oxygen_source"].get("kind", "bath")
    if src not in ("bath", "vessel"):
        raise ConfigError(f"{name}: the device step runs a bath or a vessel, not a {src}")
    kind = cfg["seeding"].get("kind", "single")
    if kind not in ("single", "sheet"):
        raise ConfigError(f"{name}: the device step seeds one cell or a sheet, not a {kind}")
    if kind == "sheet":
        # simulation.rs:696-731
        side = int(cfg["seeding"].get("side", 0))
        if float(cfg["oxygen_uptake"]) != 0.0:
            raise ConfigError(f"{name}: a sheet fills the box and leaves no medium to supply oxygen; "
                              "set oxygen_uptake = 0 to run it with the field off")
        if side < 4:
            raise ConfigError(f"{name}: a sheet of cells {side} pixels across is too fine for any of them to divide")
        if cfg["width"] % side or cfg["height"] % side:
            raise ConfigError(f"{name}: a sheet of cells {side} pixels across does not tile a "
                              f"{cfg['width']}x{cfg['height']} box; make both sides a multiple of {side}")
        if src == "vessel":
            raise ConfigError(f"{name}: a sheet is a layer of normal tissue with nothing inside it; "
                              "it cannot be laid around a vessel")
        if cfg["depth"] > 1:
            raise ConfigError(f"{name}: a sheet, which is a layer one cell thick, runs only in the plane; "
                              "set depth = 1")
    for key in ("angiogenesis", "immunity"):
        if cfg.get(key) is not None:
            raise ConfigError(f"{name}: `{key}` is not part of the device step")
    if cfg.get("tracing") is not None:
        # Tracing (types.rs:208-214) and its check (simulation.rs:614-619)
        tr = cfg["tracing"]
        missing = [k for k in ("at", "every") if k not in tr]
        if missing:
            raise ConfigError(f"{name}: missing field `{missing[0]}` in the tracing")
        if int(tr["every"]) == 0:
            raise ConfigError(f"{name}: tracing every 0 steps: the clones are written down every so many "
                              "steps, at least one")
    if cfg.get("lesion") is not None:
        # LesionConfig (config.rs:142-160); Lesion checks (simulation.rs:751-770)
        les = cfg["lesion"]
        missing = [k for k in ("network", "at", "radius") if k not in les]
        if missing:
            raise ConfigError(f"{name}: missing field `{missing[0]}` in the lesion")
        if cfg["depth"] > 1:
            raise ConfigError(f"{name}: a lesion is placed in a plane; set depth = 1")
        if les.get("centre") is not None:
            cx, cy = (float(v) for v in les["centre"])
            if not (0.0 <= cx < cfg["width"] and 0.0 <= cy < cfg["height"]):
                raise ConfigError(f"{name}: a lesion centred at ({cx}, {cy}) lies outside the "
                                  f"{cfg['width']}x{cfg['height']} box")
        r = float(les["radius"])
        if not (math.isfinite(r) and r > 0.0):
            raise ConfigError(f"{name}: a lesion of radius {r} holds no cell")
    if cfg["suppress"]:
        raise ConfigError(f"{name}: `suppress` is not part of the device step (its mutations are all made)")
    if not 0.0 <= float(cfg["mutation_rate"]) <= 1.0 or not 0.0 <= float(cfg["rewiring"]) <= 1.0:
        raise ConfigError(f"{name}: mutation_rate and rewiring are chances, in [0, 1]")
    if int(cfg["sweeps_per_step"]) < 1:
        # simulation.rs:511-514
        raise ConfigError(f"{name}: sweeps_per_step is {cfg['sweeps_per_step']}; a step sweeps the lattice at "
                          "least once")
    if cfg["contact_order"] not in (1, 2, 3):
        raise ConfigError(f"{name}: contact_order is {cfg['contact_order']}; it is 1, 2 or 3")
    if cfg["network"] is None:
        raise ConfigError(f"{name}: name the network file; the built-in RAS/ERK network is not carried here")
    if cfg["oxygen_uptake"] < 0:
        raise ConfigError(f"{name}: oxygen_uptake must not be below zero (zero leaves the field off)")


def first_cell_volume(cfg) -> int:
    """The pixels of the seeded ball (add_ball, cpm.rs:323-354): the network's
    reference volume (simulation.rs:726-733)."""
    w, h, d = cfg["width"], cfg["height"], cfg["depth"]
    r = FIRST_CELL_RADIUS_3D if d > 1 else FIRST_CELL_RADIUS
    src = cfg["oxygen_source"]
    cx = w // 2 + (int(src.get("radius", 0)) + r if src.get("kind") == "vessel" else 0)
    cy, cz = h // 2, d // 2
    z, y, x = np.mgrid[0:d, 0:h, 0:w]
    ball = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 <= r * r
    if src.get("kind") == "vessel":
        rv = int(src.get("radius", 0))
        ball &= (x - w // 2) ** 2 + (y - h // 2) ** 2 > rv * rv
    return int(ball.sum())


def simulation_kwargs(cfg, histories=1, seeds=None, subsweeps=4):
    """Simulation's options for the scenario, and the network's reference volume."""
    _refuse(cfg)
    src = cfg["oxygen_source"]
    vessel = src.get("kind") == "vessel"
    sheet = cfg["seeding"].get("kind", "single") == "sheet"
    side = int(cfg["seeding"].get("side", 0)) if sheet else 0
    # the network's reference volume: the seeded cell's, or a sheet cell's
    # (newborn_volume, simulation.rs:742-749)
    refvol = side * side if sheet else first_cell_volume(cfg)
    uptake = float(cfg["oxygen_uptake"])
    kw = dict(dims=[(cfg["width"], cfg["height"], cfg["depth"])] * histories, ncells=[1] * histories,
              seeds=list(seeds) if seeds is not None else [int(cfg["seed"]) + k for k in range(histories)],
              temperature=float(cfg["temperature"]), J=CONTACT, contact_order=int(cfg["contact_order"]),
              target_volume=0, seeding=3,
              seed_side=FIRST_CELL_RADIUS_3D if cfg["depth"] > 1 else FIRST_CELL_RADIUS, nfields=1,
              o2_dcoef=OXYGEN_DIFFUSION, o2_sink_by_type=(0.0, 0.0, 0.0, 0.0), o2_hold=4 if vessel else 3,
              vessel_radius=int(src.get("radius", 0)) if vessel else 0, o2_uptake=uptake,
              tolerance=OXYGEN_TOLERANCE * uptake, precision=FP64, stop_rule=STOP_MAX_CHANGE,
              dt=1.0, substeps=NETWORK_TIME_PER_MCS, sweeps=int(cfg["sweeps_per_step"]),
              death_threshold=DEATH_THRESHOLD, necrotic_type=NECROTIC, divide=True,
              max_cells=int(cfg["max_cells"]), divide_every=DIVISION_CHECK_EVERY, subsweeps=int(subsweeps),
              first_tolerance=OXYGEN_WARMUP_TOLERANCE, differentiated_type=DIFFERENTIATED,
              apoptotic_type=APOPTOTIC)
    if uptake == 0.0:
        # nothing consumes: the field stays at its source's level, unsolved
        # (field_is_off, simulation.rs:786-793, 2127-2131)
        kw.update(field_off=True, tolerance=1e-8, first_tolerance=0.0)
    if sheet:
        # the box tiled with side x side cells of normal tissue, each the
        # founder of its own clone (simulation.rs:696-740, 780-785)
        kw.update(seeding=4, seed_side=side, ncells=[(cfg["width"] // side) * (cfg["height"] // side)] * histories,
                  lineage=True)
    if cfg.get("cycle"):
        cy = cfg["cycle"]
        if "median" not in cy or "spread" not in cy:
            raise ConfigError(f"{os.path.basename(cfg['path'])}: a cycle names its median and its spread")
        median, spread = float(cy["median"]), float(cy["spread"])
        # simulation.rs:522-530
        if not (math.isfinite(median) and median >= 1.0 and math.isfinite(spread) and spread >= 0.0):
            raise ConfigError(f"{os.path.basename(cfg['path'])}: the cycle's median is {median} steps and its "
                              f"spread {spread}; a cycle lasts a step at least, and its spread is not below zero")
        kw.update(cycle_median=median, cycle_spread=spread, divide_every=1)
    if cfg.get("exposure"):
        kw.update(_exposure(cfg))
    if cfg.get("debris_loss") is not None:
        loss = float(cfg["debris_loss"])
        # simulation.rs:543-550
        if not (math.isfinite(loss) and 0.0 < loss <= 1.0):
            raise ConfigError(f"{os.path.basename(cfg['path'])}: debris loss is {loss}; it is the share of a "
                              "dead cell lost per step, above zero and at most one")
        kw["debris_loss"] = loss
    if cfg.get("still_medium"):
        if "diffusion" not in cfg["still_medium"]:
            raise ConfigError(f"{os.path.basename(cfg['path'])}: a still medium names its diffusion")
        kw["still_medium"] = float(cfg["still_medium"]["diffusion"])
    if cfg["mutation_rate"]:
        kw.update(mutation_rate=float(cfg["mutation_rate"]), rewiring=float(cfg["rewiring"]))
    if cfg.get("suppress_before") is not None:
        kw["suppress_before"] = int(cfg["suppress_before"])
    if cfg.get("tracing") is not None:
        kw["tracing_at"] = int(cfg["tracing"]["at"])
    if cfg.get("waste"):
        kw["waste_production"] = float(cfg["waste"]["production"])
    if cfg.get("necrotic_factor"):
        nf = cfg["necrotic_factor"]
        kw["necrotic_production"] = float(nf["production"])
        kw["necrotic_release_for"] = int(nf["release_for"]) if nf.get("release_for") is not None else -1
    return kw, refvol


def _exposure(cfg):
    """Exposure (types.rs:92-104): intensity, uptake, start and a continuous or
    periodic schedule, as Simulation's exposure_* options."""
    name = os.path.basename(cfg["path"])
    e = cfg["exposure"]
    missing = [k for k in ("intensity", "uptake", "start", "schedule") if k not in e]
    if missing:
        raise ConfigError(f"{name}: the exposure names its {missing[0]}")
    sched = e["schedule"]
    kind = sched.get("kind")
    if kind == "continuous":
        on, off = 0, 0
    elif kind == "periodic":
        on, off = int(sched["on"]), int(sched["off"])
        if on == 0:
            raise ConfigError(f"{name}: a periodic exposure that is on for zero steps is never on")
    else:
        raise ConfigError(f"{name}: an exposure's schedule is continuous or periodic, not {kind}")
    return dict(exposure_intensity=float(e["intensity"]), exposure_uptake=float(e["uptake"]),
                exposure_start=int(e["start"]), exposure_on=on, exposure_off=off)


def simulation_from_config(cfg, histories=1, seeds=None, subsweeps=4):
    """(Simulation, Network) for a configuration read by load_sim_config."""
    kw, refvol = simulation_kwargs(cfg, histories, seeds, subsweeps)
    spec = load_network_spec(cfg["network_path"])
    cap = (spec.get("mechanics") or {}).get("max_target")
    if cap is not None and not float(cap) >= DIVISION_RATIO:
        # simulation.rs:621-628
        raise ConfigError(f"{os.path.basename(cfg['path'])}: the network caps a cell's target at {cap} times its "
                          f"reference size, and a cell divides at {DIVISION_RATIO}; no cell could ever divide")
    net = Network.from_spec(spec, refvol)
    kw["lambda_volume"] = _network_lambda(cfg)
    sim = Simulation(net, **kw)
    if cfg.get("lesion") is not None:
        # the lesion's network, beside the configuration like its own, compiled
        # for a newborn cell's volume (simulation.rs:751-770)
        les = cfg["lesion"]
        path = os.path.join(os.path.dirname(cfg["path"]), les["network"])
        lesion_net = Network.from_spec(load_network_spec(path), refvol)
        sim.set_lesion(lesion_net, int(les["at"]), float(les["radius"]), les.get("centre"))
    return sim, net


def _network_lambda(cfg):
    spec = load_network_spec(cfg["network_path"])
    return float((spec.get("mechanics") or {}).get("lambda_volume", 50.0))


def touches_the_edge(grid, vessel=False) -> bool:
    """touches_the_edge (simulation.rs:2165-2198) for a bath or a vessel: a
    cell on the box's sides, or in a volume around no vessel its faces."""
    g = np.asarray(grid)
    d = g.shape[0]
    cell = g > 0
    sides = cell[:, 0, :].any() or cell[:, -1, :].any() or cell[:, :, 0].any() or cell[:, :, -1].any()
    return bool(sides or (d > 1 and not vessel and (cell[0].any() or cell[-1].any())))


def snapshot_of(sim, hist, mcs):
    """Simulation::snapshot (simulation.rs:1980-2003) of one history."""
    lat = sim.lattice()
    n = lat.cell_count(hist)
    rec = lat.cells(n, hist)
    return snapshot(mcs, sim.grid(hist), rec["type"], rec["volume"], sim.network_state(n, hist),
                    sim.field_values(0, hist))


def run(path, out_dir=None, histories=1, seeds=None, subsweeps=4, steps=None, profile_last=False):
    """The reference's run loop (src/main.rs:162-206) on the device: every
    step measured into measurements.csv, a snapshot every
    `snapshot_interval` steps and at the step the tissue touches the edge,
    after which that history stops (one directory per history when there
    are several)."""
    cfg = load_sim_config(path)
    sim, _ = simulation_from_config(cfg, histories, seeds, subsweeps)
    out_dir = out_dir or os.path.join(os.path.dirname(cfg["path"]), cfg["output_dir"])
    dirs = [out_dir] if histories == 1 else [os.path.join(out_dir, f"history-{k}") for k in range(histories)]
    logs = [MeasurementLog(d) for d in dirs]
    tracing = cfg.get("tracing")
    traces = [TraceLog(d) for d in dirs] if tracing else None
    done = [False] * histories
    n = int(cfg["mcs"] if steps is None else steps)
    taken = 0
    for i in range(n):
        if profile_last and i == n - 1:
            from . import _lib
            _lib.check(_lib.lib().cw_profiler_start())
            sim.step(1)
            _lib.check(_lib.lib().cw_profiler_stop())
        else:
            sim.step(1)
        taken += 1
        ms = sim.measure()
        edge = sim.touches_edge()
        for k in range(histories):
            if done[k]:
                continue
            logs[k].record(ms[k])
            mcs = int(ms[k]["mcs"])
            # the marked clones every `every` steps from the marking (src/main.rs:173-178)
            if traces and mcs >= int(tracing["at"]) and (mcs - int(tracing["at"])) % int(tracing["every"]) == 0:
                traces[k].record(mcs, sim.traced_clones(k))
            if edge[k]:
                done[k] = True
                write_snapshot(dirs[k], snapshot_of(sim, k, mcs))
            elif mcs % int(cfg["snapshot_interval"]) == 0:
                write_snapshot(dirs[k], snapshot_of(sim, k, mcs))
        if all(done):
            break
    for lg in logs + (traces or []):
        lg.close()
    return dict(steps=taken, reached_edge=done, directories=dirs)


def main(argv=None):
    """``python -m cellweave_b200 run.toml [--steps N] [--histories H]
    [--out DIR]``: the run loop on the device, then one JSON line: steps taken,
    wall seconds and milliseconds a step (measurements, snapshots and the
    edge test included)."""
    import argparse
    import json
    import time
    p = argparse.ArgumentParser(prog="python -m cellweave_b200")
    p.add_argument("config")
    p.add_argument("--steps", type=int, default=None)
    p.add_argument("--histories", type=int, default=1)
    p.add_argument("--subsweeps", type=int, default=4)
    p.add_argument("--out", default=None)
    p.add_argument("--profile-last", action="store_true",
                   help="bracket the last step with the CUDA profiler's start and stop")
    a = p.parse_args(argv)
    t0 = time.perf_counter()
    out = run(a.config, a.out, histories=a.histories, subsweeps=a.subsweeps, steps=a.steps,
              profile_last=a.profile_last)
    wall = time.perf_counter() - t0
    print(json.dumps(dict(config=os.path.abspath(a.config), histories=a.histories, steps=out["steps"],
                          wall_s=round(wall, 3), ms_per_step=round(1000.0 * wall / max(out["steps"], 1), 3),
                          reached_edge=out["reached_edge"], directories=out["directories"])))

