"""measurements.csv and the JSON snapshots, as the reference writes them
(crates/io/src/output.rs:10-97).

One row per step, the columns of MEASUREMENT_COLUMNS in that order, counts as
integers and the exposure and the three radii to four decimals, so that two
runs of one seed write the same bytes.  The device step has no
angiogenesis or immune cells: those columns are written as the reference
writes them without those features (0); the clones column counts the clones
with a living cell (the founder's alone without mutation, a lineage or a
lesion), the lesion column the living cells descended from a lesion, and a
held column of oxygen is the vessel, all of it perfused.
"""
from __future__ import annotations

import json
import os

import numpy as np

MEASUREMENT_COLUMNS = ("mcs,cycling,quiescent,necrotic,differentiating,apoptotic,exposure,born,gone,clones,lesion,"
                       "vessel,perfused,sprouts,regressed,immune,killed,tissue_radius,necrotic_radius,viable_depth")


def measurement_row(m: dict) -> str:
    """One row of output.rs:72-97 from a Simulation.measure() entry; the
    columns the device step has no counterpart for take their defaults."""
    living = int(m["cycling"]) + int(m["quiescent"])
    full = dict(differentiating=0, apoptotic=0, exposure=0.0, clones=1 if living > 0 else 0, lesion=0,
                perfused=m.get("vessel", 0), sprouts=0, regressed=0, immune=0, killed=0)
    full.update(m)
    ints = ("mcs", "cycling", "quiescent", "necrotic", "differentiating", "apoptotic")
    ints2 = ("born", "gone", "clones", "lesion", "vessel", "perfused", "sprouts", "regressed", "immune", "killed")
    return ",".join([str(int(full[k])) for k in ints] + ["{:.4f}".format(float(full["exposure"]))] +
                    [str(int(full[k])) for k in ints2] +
                    ["{:.4f}".format(float(full[k])) for k in ("tissue_radius", "necrotic_radius", "viable_depth")])


class MeasurementLog:
    """MeasurementLog (output.rs:49-120): measurements.csv in `directory`, its
    header first, then one row per recorded step."""

    def __init__(self, directory: str):
        os.makedirs(directory, exist_ok=True)
        self.path = os.path.join(directory, "measurements.csv")
        self._f = open(self.path, "w", newline="\n")
        self._f.write(MEASUREMENT_COLUMNS + "\n")

    def record(self, m: dict):
        self._f.write(measurement_row(m) + "\n")

    def flush(self):
        self._f.flush()

    def close(self):
        self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


TRACE_COLUMNS = "mcs,mark,cells"


class TraceLog(MeasurementLog):
    """TraceLog (output.rs:115-166): traced.csv in `directory`, its header
    first, then a row per marked clone still in the layer each time the
    clones are written down."""

    def __init__(self, directory: str):
        os.makedirs(directory, exist_ok=True)
        self.path = os.path.join(directory, "traced.csv")
        self._f = open(self.path, "w", newline="\n")
        self._f.write(TRACE_COLUMNS + "\n")

    def record(self, mcs: int, clones):
        for mark, cells in clones:
            self._f.write(f"{int(mcs)},{int(mark)},{int(cells)}\n")


# CellKind (crates/core/src/types.rs:61-76) by the device's type index
KIND_NAMES = ("Medium", "Tumor", "Normal", "Necrotic", "Differentiated", "Apoptotic")


def snapshot(mcs: int, grid, types, volumes, proteins, oxygen) -> dict:
    """Simulation::snapshot (simulation.rs:1980-2003): every cell with pixels,
    in id order, its kind, volume, protein levels, the mean oxygen over its
    pixels now (mean_per_cell, coupling.rs:165-182) and its clone (the
    founder's, 0: the device step does not mutate).  `grid` the lattice,
    `types`/`volumes` the records, `proteins` [records, S], `oxygen` the
    field, both flat or shaped as the lattice."""
    g = np.asarray(grid).reshape(-1)
    n = len(volumes)
    inside = g > 0
    sums = np.bincount(g[inside], weights=np.asarray(oxygen, np.float64).reshape(-1)[inside], minlength=n)[:n]
    count = np.bincount(g[inside], minlength=n)[:n]
    cells = []
    for cid in range(1, n):
        if volumes[cid] <= 0:
            continue
        cells.append(dict(id=cid, kind=KIND_NAMES[int(types[cid])], volume=int(volumes[cid]),
                          proteins=dict(values=[float(v) for v in proteins[cid]]),
                          oxygen=float(sums[cid] / count[cid]) if count[cid] else 0.0, clone=0))
    return dict(mcs=int(mcs), cells=cells)


def write_snapshot(directory: str, snap: dict) -> str:
    """JsonOutput::write_snapshot (output.rs:24-35): snapshot_NNNNNN.json in
    `directory`, pretty-printed with two-space indents.  Numbers are written
    shortest-round-trip, as the reference's are; a float in exponent form
    may be spelled differently (1e-07 for 1e-7) and reads back the same."""
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, "snapshot_{:06d}.json".format(int(snap["mcs"])))
    with open(path, "w") as fh:
        fh.write(json.dumps(snap, indent=2))
    return path
