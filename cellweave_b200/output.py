"""measurements.csv, as the reference writes it (crates/io/src/output.rs:30-97).

One row per step, the columns of MEASUREMENT_COLUMNS in that order, counts as
integers and the exposure and the three radii to four decimals, so that two
runs of one seed write the same bytes.  The device step has no exposure,
differentiation, apoptosis, lesion, angiogenesis or immune cells: those
columns are written as the reference writes them without those features (0),
the clones column counts the founder's clone while anything lives (no
mutation happens inside the device step), and a held column of oxygen is the
vessel, all of it perfused.
"""
from __future__ import annotations

import os

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
