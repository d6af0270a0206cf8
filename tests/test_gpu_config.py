"""A configuration file's scenario on the device against the oracle (GPU).

A spheroid and a cord written as the reference's configuration files are
(crates/io/src/config.rs), with the RAS/ERK network of the reference's
examples: one cell in a bath (or against a vessel) grows, divides every 20
steps, starves inside; the device's 32 histories against the oracle stepping
the same scenario with the reference's algorithms (sequential random-pixel
sweep, FP64 SOR, RK4), living and necrotic cells and the tissue's radius and
viable depth inside the oracle's 32-seed band (also with daughters that
mutate or rewire their networks and found clones); and the run loop's
measurements.csv.
"""
import json
import os

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import config as C
from cpm_ensembles import SEEDS, within_band
from oracle.cpu_sim import CpuHistory, lesion_joining

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def ras_erk_toml(tmp_path, stressed=False):
    spec = json.load(open(os.path.join(HERE, "golden", "golden.json")))["networks"]["ras-erk"]
    if stressed:
        # survival damaged by stress above a threshold (DamagedAbove, crates/core/src/network.rs:127-135)
        spec["nodes"][4]["terms"].append({"kind": "damaged_above", "rate": 0.2, "source": "stress", "threshold": 0.3})
    lines = []
    for node in spec["nodes"]:
        lines += ["[[nodes]]", f'name = "{node["name"]}"', f'initial = {node["initial"]}', "terms = ["]
        for t in node["terms"]:
            kv = ", ".join(f'{k} = "{v}"' if isinstance(v, str) else f"{k} = {v}" for k, v in t.items())
            lines.append(f"  {{ {kv} }},")
        lines.append("]")
    lines.append("[roles]")
    lines += [f'{k} = "{v}"' for k, v in spec["roles"].items()]
    lines.append("[mechanics]")
    lines += [f"{k} = {v}" for k, v in spec["mechanics"].items()]
    (tmp_path / "ras-erk.toml").write_text("\n".join(lines) + "\n")
    return spec


def toml_value(v):
    if isinstance(v, str):
        return f'"{v}"'
    if isinstance(v, dict):
        return "{ " + ", ".join(f"{k} = {toml_value(x)}" for k, x in v.items()) + " }"
    return str(v)


def network_file(tmp_path, name, spec):
    lines = []
    for node in spec["nodes"]:
        lines += ["[[nodes]]", f'name = "{node["name"]}"', f'initial = {node["initial"]}', "terms = ["]
        lines += ["  " + toml_value(t) + "," for t in node["terms"]]
        lines.append("]")
    lines.append("[roles]")
    lines += [f'{k} = "{v}"' for k, v in spec["roles"].items()]
    lines.append("[mechanics]")
    lines += [f"{k} = {v}" for k, v in spec["mechanics"].items()]
    (tmp_path / name).write_text("\n".join(lines) + "\n")


def scenario(tmp_path, source, uptake=0.001, stressed=False):
    spec = ras_erk_toml(tmp_path, stressed)
    text = ("width = 120\nheight = 120\nmcs = 140\ntemperature = 10.0\nsnapshot_interval = 20\n"
            f"output_dir = \"out\"\noxygen_uptake = {uptake}\nnetwork = \"ras-erk.toml\"\n" + source)
    p = tmp_path / "run.toml"
    p.write_text(text)
    return str(p), spec


CYCLE = "\n[cycle]\nmedian = 20.0\nspread = 0.3\n"


@pytest.mark.parametrize("source,uptake", [("", 0.001), ("\n[oxygen_source]\nkind = \"vessel\"\nradius = 5\n", 0.0001),
                                           (CYCLE, 0.001), ("debris_loss = 0.05\n", 0.001),
                                           ("mutation_rate = 0.3\nrewiring = 0.3\n", 0.001)])
def test_a_configured_tissue_grows_inside_the_oracle_band(tmp_path, source, uptake):
    path, spec = scenario(tmp_path, source, uptake)
    cfg = C.load_sim_config(path)
    seeds = [7_000 + k for k in range(SEEDS)]
    sim, _ = C.simulation_from_config(cfg, histories=SEEDS, seeds=seeds)
    kw, _ = C.simulation_kwargs(cfg, SEEDS, seeds)
    ocfg = dict(kw, network_spec=spec, lambda_volume=float(spec["mechanics"]["lambda_volume"]), hypoxic_level=0.1)
    ora = [CpuHistory(ocfg, k) for k in range(SEEDS)]
    keys = ("cycling", "quiescent", "necrotic", "tissue_radius", "viable_depth")
    for step in range(1, 141):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (60, 100, 140):
            continue
        dm = sim.measure()
        om = [h.measure() for h in ora]
        for q in keys:
            dv = np.array([float(m[q]) for m in dm])
            rv = np.array([float(m[q]) for m in om])
            assert within_band(dv, rv), (step, q, dv.mean(), rv.mean(), rv.std())
    final = np.array([m["cycling"] + m["quiescent"] for m in sim.measure()])
    assert final.mean() > 8  # it grew
    if "mutation_rate" in source:
        # daughters founded clones, each under its own network, on the device as in the oracle
        founded = sim.clone_records()
        assert len(founded) >= 5 and sum(len(h.clone_specs) - 1 for h in ora) >= 5
        assert {r["change"] for _, r in founded} >= {"scaled", "gained"} or len(founded) < 10
        clones = np.concatenate([sim.clones(200, k) for k in range(SEEDS)])
        assert clones.max() == len(founded)
    for k in range(SEEDS):
        assert sim.records_match_grid(k)


def test_a_sheet_of_epithelium_turns_over_inside_the_oracle_band(tmp_path):
    # Seeding::Sheet with the field off (simulation.rs:696-749): a 60 x 60 box
    # tiled with 10 x 10 cells of normal tissue, each the founder of a clone,
    # under the reference's epithelium network (its NOTCH node the chance to
    # commit to differentiate; committed cells shed until gone).  The device's
    # 32 histories against the oracle's: living and differentiating cells, the
    # cells gone and the clones left inside the 32-seed band
    spec = json.load(open(os.path.join(HERE, "golden", "golden.json")))["networks"]["epithelium"]
    network_file(tmp_path, "epithelium.toml", spec)
    p = tmp_path / "run.toml"
    p.write_text("width = 60\nheight = 60\nmcs = 300\ntemperature = 10.0\nsnapshot_interval = 100\n"
                 "output_dir = \"out\"\noxygen_uptake = 0.0\nnetwork = \"epithelium.toml\"\n"
                 "[seeding]\nkind = \"sheet\"\nside = 10\n")
    cfg = C.load_sim_config(str(p))
    seeds = [9_000 + k for k in range(SEEDS)]
    sim, _ = C.simulation_from_config(cfg, histories=SEEDS, seeds=seeds)
    kw, refvol = C.simulation_kwargs(cfg, SEEDS, seeds)
    assert refvol == 100 and kw["field_off"] and kw["lineage"]
    ocfg = dict(kw, network_spec=spec, lambda_volume=float(spec["mechanics"]["lambda_volume"]), hypoxic_level=0.1)
    ora = [CpuHistory(ocfg, k) for k in range(SEEDS)]
    first = sim.measure()
    assert all(m["clones"] == 36 and m["cycling"] + m["quiescent"] == 36 for m in first)
    keys = ("cycling", "differentiating", "gone", "clones")
    for step in range(1, 301):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (100, 200, 300):
            continue
        dm = sim.measure()
        om = [h.measure() for h in ora]
        for q in keys:
            dv = np.array([float(m[q]) for m in dm])
            rv = np.array([float(m[q]) for m in om])
            assert within_band(dv, rv), (step, q, dv.mean(), rv.mean(), rv.std())
    dm = sim.measure()
    assert np.mean([m["gone"] for m in dm]) > 10 and np.mean([m["clones"] for m in dm]) < 36
    # the oxygen was never solved: every cell read full oxygen
    assert np.all(sim.field_values(0, 0) == 1.0)
    for k in range(SEEDS):
        assert sim.records_match_grid(k)


LESION_SHEET = ("width = 60\nheight = 60\nmcs = 240\ntemperature = 10.0\nsnapshot_interval = 100\n"
                "output_dir = \"out\"\noxygen_uptake = 0.0\nnetwork = \"tissue.toml\"\n"
                "mutation_rate = 0.02\nrewiring = 0.3\n{extra}"
                "[seeding]\nkind = \"sheet\"\nside = 10\n"
                "[lesion]\nnetwork = \"lesion.toml\"\nat = {at}\nradius = 15.0\n")


def lesion_files(tmp_path):
    nets = json.load(open(os.path.join(HERE, "golden", "golden.json")))["networks"]
    network_file(tmp_path, "tissue.toml", nets["epithelium-no-pressing"])
    network_file(tmp_path, "lesion.toml", nets["lesion"])
    return nets["epithelium-no-pressing"], nets["lesion"]


def test_a_lesion_takes_the_cells_whose_centres_lie_within_its_radius(tmp_path):
    # place_lesion (simulation.rs:1920-1970) at step 12 of four sheets: the
    # cells that join are the oracle's choice on the device's lattice just
    # before, each history founds one clone (parent -1), and every record
    # outside it keeps its clone
    lesion_files(tmp_path)
    p = tmp_path / "run.toml"
    p.write_text(LESION_SHEET.format(extra="", at=12))
    cfg = C.load_sim_config(str(p))
    sim, net = C.simulation_from_config(cfg, histories=4, seeds=[31, 32, 33, 34])
    sim.step(12)
    lat = sim.lattice()
    before, want, held = [], [], []
    for k in range(4):
        n = lat.capacity[k]
        rec = lat.cells(n, k)
        grid = sim.grid(k).reshape(60, 60)
        want.append(lesion_joining(grid, rec["type"], rec["volume"], (C.NECROTIC, C.DIFFERENTIATED, C.APOPTOTIC),
                                   None, 15.0))
        before.append(sim.clones(n, k))
        held.append(np.asarray(rec["volume"]) > 0)
        assert 4 <= len(want[k]) < 36
    nrec = len(sim.clone_records())
    sim.step(1)
    recs = sim.clone_records()
    lesions = [r for r in recs[nrec:] if r[1].get("lesion")]
    assert len(lesions) == 4 and all(parent == -1 for parent, _ in lesions)
    founded = set()
    for k in range(4):
        n = lat.capacity[k]
        after = sim.clones(n, k)
        joined = np.zeros(n, bool)
        joined[want[k]] = True
        assert len(set(after[joined])) == 1 and after[joined][0] not in before[k]
        founded.add(int(after[joined][0]))
        # every other cell that held pixels before the step kept its clone
        others = held[k] & ~joined
        np.testing.assert_array_equal(after[others], before[k][others])
    assert len(founded) == 4
    ms = sim.measure()
    for k in range(4):
        assert 0 < ms[k]["lesion"] <= len(want[k]) + 4


def test_a_lesion_in_a_mutating_sheet_grows_inside_the_oracle_band(tmp_path):
    # epithelium-lesion.toml's scenario, scaled to a 60 x 60 sheet: mutations
    # (suppressed before step 60), a lesion of NOTCH-slowed cells at step 40;
    # the device's 32 histories against the oracle's: living cells, the
    # lesion's descendants, the clones left and the cells gone
    tissue, lesion = lesion_files(tmp_path)
    p = tmp_path / "run.toml"
    p.write_text(LESION_SHEET.format(extra="suppress_before = 60\n", at=40))
    cfg = C.load_sim_config(str(p))
    seeds = [7_000 + k for k in range(SEEDS)]
    sim, _ = C.simulation_from_config(cfg, histories=SEEDS, seeds=seeds)
    kw, _ = C.simulation_kwargs(cfg, SEEDS, seeds)
    ocfg = dict(kw, network_spec=tissue, lambda_volume=float(tissue["mechanics"]["lambda_volume"]), hypoxic_level=0.1,
                lesion_spec=lesion, lesion_at=40, lesion_radius=15.0)
    ora = [CpuHistory(ocfg, k) for k in range(SEEDS)]
    keys = ("cycling", "differentiating", "gone", "clones", "lesion")
    for step in range(1, 241):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (41, 120, 240):
            continue
        dm = sim.measure()
        om = [h.measure() for h in ora]
        for q in keys:
            dv = np.array([float(m[q]) for m in dm])
            rv = np.array([float(m[q]) for m in om])
            assert within_band(dv, rv), (step, q, dv.mean(), rv.mean(), rv.std())
    dm = sim.measure()
    assert np.mean([m["lesion"] for m in dm]) > 0
    recs = sim.clone_records()
    assert sum(1 for _, r in recs if r.get("lesion")) == SEEDS
    for k in range(SEEDS):
        assert sim.records_match_grid(k)


SHIPPED_LESION = ("width = 100\nheight = 100\nmcs = 6000\ntemperature = 10.0\nsnapshot_interval = 100\n"
                  "output_dir = \"out\"\noxygen_uptake = 0.0\nmutation_rate = 0.01\nrewiring = 0.3\n"
                  "network = \"tissue.toml\"\nhours_per_step = 0.56\n[seeding]\nkind = \"sheet\"\nside = 10\n"
                  "[lesion]\nnetwork = \"lesion.toml\"\nat = {at}\nradius = 15.0\n")


def test_the_shipped_lesion_turns_the_cells_at_the_centre_into_one_clone_at_its_step(tmp_path):
    # crates/io/tests/lesion.rs:29-49: epithelium-lesion.toml on a 100 x 100 box,
    # the lesion at step 20: nothing before it, then one clone with no parent
    # holding 3 to 12 cells, among them the one at the centre, not the corner's
    lesion_files(tmp_path)
    p = tmp_path / "run.toml"
    p.write_text(SHIPPED_LESION.format(at=20))
    sim, _ = C.simulation_from_config(C.load_sim_config(str(p)))
    sim.step(20)
    assert sim.measure()[0]["lesion"] == 0 and not any(r.get("lesion") for _, r in sim.clone_records())
    sim.step(1)
    recs = sim.clone_records()
    lesions = [j for j, (_, r) in enumerate(recs) if r.get("lesion")]
    assert len(lesions) == 1 and recs[lesions[0]][0] == -1
    base = sim.clone_count() - len(recs)
    founded = base + lesions[0]

    def in_lesion(c):
        # descended from the lesion's clone (parents of clones founded in the run)
        while c >= base:
            if c == founded:
                return True
            c = recs[c - base][0]
        return False

    assert 3 <= sim.measure()[0]["lesion"] <= 12
    grid = sim.grid(0).reshape(100, 100)
    clones = sim.clones(sim.lattice().capacity[0], 0)
    assert in_lesion(int(clones[grid[50, 50]])) and not in_lesion(int(clones[grid[2, 2]]))


def test_a_lesion_that_never_comes_leaves_the_run_as_it_was(tmp_path):
    # crates/io/tests/lesion.rs:51-67: a lesion set for a step never reached
    # draws nothing: the measurements and clones are those of the run without one
    lesion_files(tmp_path)
    runs = []
    for text in (SHIPPED_LESION.format(at=10_000), SHIPPED_LESION.format(at=0).split("[lesion]")[0]):
        p = tmp_path / "run.toml"
        p.write_text(text)
        sim, _ = C.simulation_from_config(C.load_sim_config(str(p)))
        measured = []
        for _ in range(200):
            sim.step(1)
            measured.append(sim.measure()[0])
        runs.append((measured, sim.clone_records(), sim.grid(0).copy()))
    assert runs[0][0] == runs[1][0] and runs[0][1] == runs[1][1]
    np.testing.assert_array_equal(runs[0][2], runs[1][2])


def test_suppressed_mutations_leave_the_run_as_it_was(tmp_path):
    # Scenario::suppress_before (simulation.rs:240-244, 1671-1694): mutations
    # drawn and recorded but not made; the draws take nothing from the step's
    # other draws, so a sheet whose every mutation is suppressed runs as the
    # sheet without mutation, lattice and protein levels to the bit, while its
    # daughters still found (suppressed) clones
    lesion_files(tmp_path)
    runs = {}
    for name, extra in [("plain", "mutation_rate = 0.0\n"), ("suppressed", "suppress_before = 100000\n")]:
        p = tmp_path / f"{name}.toml"
        p.write_text(LESION_SHEET.format(extra="", at=0).split("[lesion]")[0]
                     .replace("mutation_rate = 0.02\n", "mutation_rate = 0.5\n" if name == "suppressed" else extra)
                     .replace("rewiring = 0.3\n", "rewiring = 0.3\n" + (extra if name == "suppressed" else "")))
        cfg = C.load_sim_config(str(p))
        sim, _ = C.simulation_from_config(cfg, histories=4, seeds=[51, 52, 53, 54])
        sim.step(400)  # the sheet's first divisions come after about 200 steps
        runs[name] = sim
    a, b = runs["plain"], runs["suppressed"]
    recs = b.clone_records()
    assert len(recs) >= 8 and all(r.get("suppressed") for _, r in recs)
    assert a.clone_records() == []
    for k in range(4):
        np.testing.assert_array_equal(a.grid(k), b.grid(k))
        n = a.lattice().capacity[k]
        np.testing.assert_array_equal(a.network_state(n, k).view(np.uint64), b.network_state(n, k).view(np.uint64))


TRACED_SHEET = ("width = 60\nheight = 60\nmcs = 400\ntemperature = 10.0\nsnapshot_interval = 100\n"
                "output_dir = \"out\"\noxygen_uptake = 0.0\nnetwork = \"epithelium.toml\"\n"
                "[seeding]\nkind = \"sheet\"\nside = 10\n[tracing]\nat = {at}\nevery = 10\n")


def test_tracing_marks_every_cell_in_the_layer_and_daughters_carry_the_marks(tmp_path):
    # mark_every_cell (simulation.rs:1908-1918) at step 150 of four sheets:
    # every cell in the layer carries its own mark (its id less one) and each
    # mark is one cell; 250 steps on, the marks are carried by the clones the
    # marked cells made, in the layer, and no cell born after carries a mark
    # of its own
    spec = json.load(open(os.path.join(HERE, "golden", "golden.json")))["networks"]["epithelium"]
    network_file(tmp_path, "epithelium.toml", spec)
    p = tmp_path / "run.toml"
    p.write_text(TRACED_SHEET.format(at=150))
    cfg = C.load_sim_config(str(p))
    sim, _ = C.simulation_from_config(cfg, histories=4, seeds=[61, 62, 63, 64])
    sim.step(150)
    assert all(sim.traced_clones(k) == [] for k in range(4))
    lat = sim.lattice()
    layer = []
    for k in range(4):
        rec = lat.cells(lat.capacity[k], k)
        ids = np.nonzero((rec["volume"] > 0) & (rec["type"] != C.NECROTIC) & (rec["type"] != C.APOPTOTIC))[0]
        layer.append(ids[ids > 0])
    sim.step(1)
    for k in range(4):
        tr = sim.traced_clones(k)
        # the step after the marking may have taken a cell or two out of the layer
        marks = {m for m, _ in tr}
        assert all(c == 1 for _, c in tr) and marks <= {int(i) - 1 for i in layer[k]}
        assert len(marks) >= len(layer[k]) - 3
    sim.step(250)
    for k in range(4):
        tr = sim.traced_clones(k)
        assert tr and max(c for _, c in tr) >= 2 and all(m + 1 in set(layer[k].tolist()) for m, _ in tr)


def test_traced_clones_grow_inside_the_oracle_band(tmp_path):
    # epithelium-traced.toml's experiment on a 60 x 60 sheet: every cell marked
    # at step 100, then the number of marked clones left in the layer and
    # their mean size, the device's 32 histories against the oracle's
    spec = json.load(open(os.path.join(HERE, "golden", "golden.json")))["networks"]["epithelium"]
    network_file(tmp_path, "epithelium.toml", spec)
    p = tmp_path / "run.toml"
    p.write_text(TRACED_SHEET.format(at=100))
    cfg = C.load_sim_config(str(p))
    seeds = [8_000 + k for k in range(SEEDS)]
    sim, _ = C.simulation_from_config(cfg, histories=SEEDS, seeds=seeds)
    kw, _ = C.simulation_kwargs(cfg, SEEDS, seeds)
    ocfg = dict(kw, network_spec=spec, lambda_volume=float(spec["mechanics"]["lambda_volume"]), hypoxic_level=0.1)
    ora = [CpuHistory(ocfg, k) for k in range(SEEDS)]
    for step in range(1, 401):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (101, 250, 400):
            continue
        dt = [sim.traced_clones(k) for k in range(SEEDS)]
        ot = [h.traced_clones() for h in ora]
        for name, f in (("clones", len), ("mean size", lambda t: np.mean([c for _, c in t]) if t else 0.0)):
            dv = np.array([float(f(t)) for t in dt])
            rv = np.array([float(f(t)) for t in ot])
            assert within_band(dv, rv), (step, name, dv.mean(), rv.mean(), rv.std())
    assert np.mean([len(t) for t in dt]) < 36


def test_the_run_writes_the_measurements_of_every_step_and_the_snapshots(tmp_path):
    path, spec = scenario(tmp_path, "")
    out = C.run(path, str(tmp_path / "out"), steps=25)
    rows = (tmp_path / "out" / "measurements.csv").read_text().splitlines()
    assert rows[0] == cw.output.MEASUREMENT_COLUMNS
    assert len(rows) == 1 + out["steps"] == 26
    assert rows[1].startswith("0,") and rows[-1].startswith("24,")
    # snapshot_interval 20: steps 0 and 20 (src/main.rs:193-194)
    names = sorted(p.name for p in (tmp_path / "out").iterdir() if p.name.startswith("snapshot_"))
    assert names == ["snapshot_000000.json", "snapshot_000020.json"]
    snap = json.loads((tmp_path / "out" / "snapshot_000020.json").read_text())
    assert snap["mcs"] == 20 and len(snap["cells"]) >= 1
    cell = snap["cells"][0]
    assert cell["id"] == 1 and cell["kind"] == "Tumor" and cell["clone"] == 0
    assert len(cell["proteins"]["values"]) == len(spec["nodes"]) and 0.0 < cell["oxygen"] <= 1.0


def test_cells_with_a_cycle_draw_its_lengths_and_divide_on_their_own_clocks(tmp_path):
    """cycle_lengths_have_the_median_and_spread_asked_for and
    with_a_cycle_of_their_own_cells_stop_dividing_together
    (simulation.rs:2868-2925): the lengths each division draws have the
    median and the spread of their logarithm asked for, and births fall on
    many steps of the 20-step check's period, not on one."""
    path, _ = scenario(tmp_path, CYCLE.replace("20.0", "16.0"), uptake=0.0001)
    cfg = C.load_sim_config(path)
    hists = 32
    sim, _ = C.simulation_from_config(cfg, histories=hists, seeds=[500 + k for k in range(hists)])
    lat = sim.lattice()
    drawn, residues = [], set()
    for step in range(120):
        sim.step(1)
        for k in range(hists):
            began, due = sim.cycle(lat.cell_count(k), k)
            fresh = np.nonzero((began == step) & (due > began))[0]
            if len(fresh):
                drawn += list(due[fresh] - began[fresh])
                residues.add(step % 20)
    logs = np.log(np.array(drawn, float))
    assert len(logs) >= 300, len(logs)
    assert abs(np.exp(np.median(logs)) - 16.0) < 1.5, np.exp(np.median(logs))
    assert abs(logs.std() - 0.3) < 0.05, logs.std()
    assert len(residues) >= 10, residues


def test_a_still_spheroid_in_a_volume_loses_its_debris_inside_the_oracle_band(tmp_path):
    """A small spheroid-3d: a ball of radius 3 in a 40^3 box, 26-neighbour
    contact, four sweeps a step, a cell cycle, a still medium whose level
    falls as the tissue grows, and a debris loss that takes the dead core's
    pixels at its edge; living, quiescent and necrotic cells, the tissue's
    and the necrotic radius inside the oracle's 32-seed band."""
    spec = ras_erk_toml(tmp_path)
    text = ("width = 40\nheight = 40\ndepth = 40\nmcs = 180\ntemperature = 10.0\nsnapshot_interval = 20\n"
            "output_dir = \"out\"\noxygen_uptake = 0.005\ndebris_loss = 0.024\nsweeps_per_step = 4\n"
            "contact_order = 3\nnetwork = \"ras-erk.toml\"\n" + CYCLE + "[still_medium]\ndiffusion = 0.606\n")
    (tmp_path / "run.toml").write_text(text)
    cfg = C.load_sim_config(str(tmp_path / "run.toml"))
    seeds = [9_000 + k for k in range(SEEDS)]
    sim, _ = C.simulation_from_config(cfg, histories=SEEDS, seeds=seeds)
    kw, _ = C.simulation_kwargs(cfg, SEEDS, seeds)
    ocfg = dict(kw, network_spec=spec, lambda_volume=float(spec["mechanics"]["lambda_volume"]), hypoxic_level=0.1)
    ora = [CpuHistory(ocfg, k) for k in range(SEEDS)]
    keys = ("cycling", "quiescent", "necrotic", "tissue_radius", "necrotic_radius")
    for step in range(1, 181):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (100, 140, 180):
            continue
        dm = sim.measure()
        om = [h.measure() for h in ora]
        for q in keys:
            dv = np.array([float(m[q]) for m in dm])
            rv = np.array([float(m[q]) for m in om])
            assert within_band(dv, rv), (step, q, dv.mean(), rv.mean(), rv.std())
    assert np.mean([m["necrotic"] for m in sim.measure()]) > 2  # a core died and is breaking down
    for k in range(SEEDS):
        assert sim.records_match_grid(k)


def test_an_exposure_stresses_the_tissue_inside_the_oracle_band(tmp_path):
    """settle_stress (simulation.rs:2015-2055): a periodic exposure from step
    70, on 20 steps in 40, held where the oxygen comes in and taken up by the
    living, read by a network whose survival is damaged above a stress of
    0.3 (the tissue's rim dies each time it is on); the population inside the
    oracle's band while on and off, the measurements' exposure column the
    schedule's level."""
    src = ("\n[exposure]\nintensity = 1.0\nuptake = 0.004\nstart = 70\n"
           "schedule = { kind = \"periodic\", on = 20, off = 20 }\n")
    path, spec = scenario(tmp_path, src, 0.0005, stressed=True)
    cfg = C.load_sim_config(path)
    seeds = [11_000 + k for k in range(SEEDS)]
    sim, _ = C.simulation_from_config(cfg, histories=SEEDS, seeds=seeds)
    kw, _ = C.simulation_kwargs(cfg, SEEDS, seeds)
    ocfg = dict(kw, network_spec=spec, lambda_volume=float(spec["mechanics"]["lambda_volume"]), hypoxic_level=0.1)
    ora = [CpuHistory(ocfg, k) for k in range(SEEDS)]
    keys = ("cycling", "quiescent", "necrotic", "tissue_radius")
    for step in range(1, 141):
        sim.step(1)
        for h in ora:
            h.step()
        dm = sim.measure()
        mcs = step - 1
        level = 1.0 if mcs >= 70 and (mcs - 70) % 40 < 20 else 0.0
        assert all(m["exposure"] == level for m in dm), (mcs, dm[0]["exposure"])
        if step not in (80, 100, 120, 140):
            continue
        om = [h.measure() for h in ora]
        for q in keys:
            dv = np.array([float(m[q]) for m in dm])
            rv = np.array([float(m[q]) for m in om])
            assert within_band(dv, rv), (step, q, dv.mean(), rv.mean(), rv.std())
    stress = sim.field_values(4, 0)
    assert stress.max() <= 1.0 + 1e-9


@pytest.mark.parametrize("width,source", [(22, ""), (40, "\n[oxygen_source]\nkind = \"vessel\"\nradius = 2\n")])
def test_the_device_edge_test_is_the_reference_s(tmp_path, width, source):
    """touches_the_edge (simulation.rs:2165-2198) on the device against the
    host restatement, every step of small boxes the tissue soon reaches."""
    ras_erk_toml(tmp_path)
    (tmp_path / "run.toml").write_text(f"width = {width}\nheight = 20\nmcs = 40\ntemperature = 10.0\n"
                                       "snapshot_interval = 20\noutput_dir = \"out\"\noxygen_uptake = 0.0001\n"
                                       "network = \"ras-erk.toml\"\n" + source)
    cfg = C.load_sim_config(str(tmp_path / "run.toml"))
    sim, _ = C.simulation_from_config(cfg, histories=8, seeds=list(range(8)))
    vessel = bool(source)
    seen = set()
    for _ in range(40):
        sim.step(1)
        dev = sim.touches_edge()
        host = [C.touches_the_edge(sim.grid(k), vessel) for k in range(8)]
        assert list(dev) == host
        seen |= set(host)
    assert seen == {False, True}
