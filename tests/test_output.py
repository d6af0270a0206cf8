"""measurements.csv and the snapshots as the reference writes them (crates/io/src/output.rs), on CPU."""
import os

import numpy as np
import pytest

from cellweave_b200 import output
from cellweave_b200.output import MEASUREMENT_COLUMNS, MeasurementLog, measurement_row


def test_the_table_has_a_header_and_one_fixed_width_row_per_step(tmp_path):
    # output.rs:246-289, the reference's own row
    with MeasurementLog(str(tmp_path)) as log:
        log.record(dict(mcs=7, cycling=3, quiescent=2, necrotic=1, differentiating=0, apoptotic=5, exposure=0.5,
                        born=9, gone=4, clones=2, lesion=6, vessel=113, perfused=113, sprouts=1, regressed=2,
                        immune=3, killed=4, tissue_radius=12.0, necrotic_radius=1.0 / 3.0, viable_depth=11.666_666))
    lines = (tmp_path / "measurements.csv").read_text().splitlines()
    assert lines[0] == MEASUREMENT_COLUMNS
    assert lines[1] == "7,3,2,1,0,5,0.5000,9,4,2,6,113,113,1,2,3,4,12.0000,0.3333,11.6667"
    assert len(lines[0].split(",")) == len(lines[1].split(","))


def test_the_trace_has_a_header_and_a_row_per_marked_clone(tmp_path):
    # TraceLog (output.rs:115-166): mcs,mark,cells, one row per clone each time
    with output.TraceLog(str(tmp_path)) as log:
        log.record(1000, [(3, 1), (17, 2)])
        log.record(1010, [])
        log.record(1020, [(17, 5)])
    assert (tmp_path / "traced.csv").read_text().splitlines() == [
        "mcs,mark,cells", "1000,3,1", "1000,17,2", "1020,17,5"]


def test_a_device_measurement_fills_the_columns_it_has():
    m = dict(mcs=3, cycling=10, quiescent=2, necrotic=4, born=20, gone=1, vessel=0, tissue_radius=5.5,
             necrotic_radius=2.0, viable_depth=3.5)
    assert measurement_row(m) == "3,10,2,4,0,0,0.0000,20,1,1,0,0,0,0,0,0,0,5.5000,2.0000,3.5000"


def test_a_snapshot_lists_the_cells_with_pixels_as_the_reference_serialises_them(tmp_path):
    import json
    grid = np.zeros((1, 4, 5), np.int32)
    grid[0, 0, :2] = 1
    grid[0, 1:3, 3:] = 3
    types = np.array([0, 1, 2, 3], np.int32)
    volumes = np.array([0, 2, 0, 4], np.int32)   # record 2 is gone
    proteins = np.arange(8, dtype=float).reshape(4, 2) / 8
    o2 = np.linspace(0.0, 1.0, 20).reshape(1, 4, 5)
    snap = output.snapshot(40, grid, types, volumes, proteins, o2)
    assert snap["mcs"] == 40 and [c["id"] for c in snap["cells"]] == [1, 3]
    first, dead = snap["cells"]
    assert first["kind"] == "Tumor" and dead["kind"] == "Necrotic" and dead["volume"] == 4
    assert first["proteins"] == {"values": [0.25, 0.375]} and first["clone"] == 0
    assert first["oxygen"] == pytest.approx(o2.reshape(-1)[[0, 1]].mean())
    assert dead["oxygen"] == pytest.approx(o2.reshape(-1)[[8, 9, 13, 14]].mean())
    path = output.write_snapshot(str(tmp_path), snap)
    assert os.path.basename(path) == "snapshot_000040.json"
    text = open(path).read()
    assert json.loads(text) == snap
    # serde_json's pretty form: two-space indents, the fields in declaration order
    assert text.startswith('{\n  "mcs": 40,\n  "cells": [\n    {\n      "id": 1,\n      "kind": "Tumor",')
