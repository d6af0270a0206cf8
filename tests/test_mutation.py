"""Per-cell mutated networks: the oracle's restatement of Network::mutate and
Network::rewire (crates/engine/src/network.rs:479-575) pinned on the
reference's own tests of them (network.rs:1398-1530), on CPU."""
import numpy as np
import pytest

from oracle import oracle as O


def ras_erk(golden):
    return golden["networks"]["ras-erk"]


def at(o2, egf):
    # CellInputs of network.rs:839-849: oxygen and EGF, every other input zero
    return np.array([[o2, egf, 0.0, 0.0, 0.0, 0.0]])


def run(spec, steps, o2, egf):
    net = O.compile_network(spec, 200)
    st = net.initial.reshape(1, -1).copy()
    O.network_step(net, st, at(o2, egf), 1.0, steps)
    return net, st[0]


def test_a_mutation_scales_one_rate_and_the_parent_keeps_its_own(golden):
    # network.rs:1398-1425: the last of the eleven terms is BCL2's damage
    # below the anoxia threshold; a draw near one doubles it
    parent = ras_erk(golden)
    daughter, m = O.mutate_spec(parent, 0.99, 0.999_999)
    assert (m["node"], m["term"], m["kind"]) == ("bcl2", 3, "damaged_below")
    assert abs(m["factor"] - O.MUTATION_SPREAD) < 1e-5
    net_p, sp = run(parent, 40, 0.05, 0.2)
    net_d, sd = run(daughter, 40, 0.05, 0.2)
    assert sd[net_d.survival] < sp[net_p.survival], "doubled damage kills faster in the dark"
    assert parent["nodes"][4]["terms"][3]["rate"] == 0.25  # the parent keeps its own


def test_a_draw_in_the_middle_changes_nothing(golden):
    # network.rs:1427-1443
    spec, m = O.mutate_spec(ras_erk(golden), 0.0, 0.5)
    assert (m["node"], m["term"], m["kind"]) == ("ras", 0, "activated_by")
    assert m["factor"] == 1.0
    _, a = run(spec, 5, 0.8, 0.2)
    _, b = run(ras_erk(golden), 5, 0.8, 0.2)
    np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))


def test_a_gained_link_makes_a_node_answer_what_it_ignored(golden):
    # network.rs:1484-1502
    spec, m = O.rewire_spec(ras_erk(golden), [0.0, 0.0, 0.0, 0.0, 0.5])
    assert O.mutation_text(m) == "ras gains activated_by oxygen @0.10"
    assert m["term"] == 2, "added after RAS's two terms"
    assert run(ras_erk(golden), 40, 1.0, 0.0)[1][0] < 0.01
    assert run(spec, 40, 1.0, 0.0)[1][0] > 0.1


def test_a_lost_term_takes_its_answer_away(golden):
    # network.rs:1504-1520
    spec, m = O.rewire_spec(ras_erk(golden), [0.9, 0.0, 0.0, 0.0, 0.0])
    assert O.mutation_text(m) == "ras loses activated_by #0"
    assert m["change"] == "lost"
    assert run(ras_erk(golden), 40, 0.8, 0.2)[1][0] > 0.2, "EGF switches the healthy RAS on"
    assert run(spec, 40, 0.8, 0.2)[1][0] < 0.01, "and nothing switches this one on"


@pytest.mark.parametrize("which", [0.0, 0.3, 0.5, 0.999999])
def test_picks_cover_every_term_and_stay_in_range(golden, which):
    spec = ras_erk(golden)
    count = sum(len(n["terms"]) for n in spec["nodes"])
    _, m = O.mutate_spec(spec, which, 0.25)
    flat = [(n["name"], j) for n in spec["nodes"] for j in range(len(n["terms"]))]
    assert flat[min(int(which * count), count - 1)] == (m["node"], m["term"])
    assert abs(m["factor"] - 2.0 ** -0.5) < 1e-15
    # a network without a single term: nothing to change, nothing to lose
    bare = {"nodes": [{"name": "a", "initial": 0.1}], "roles": spec["roles"], "mechanics": spec["mechanics"]}
    assert O.mutate_spec(bare, which, 0.5)[1] is None
    assert O.rewire_spec(bare, [0.9, which, 0.0, 0.0, 0.0])[1] is None


def test_a_lesion_takes_the_living_cells_whose_centres_lie_within_its_radius():
    # place_lesion (simulation.rs:1920-1962) on a hand-built 20 x 20 plane:
    # centres of mass as x + 1/2, y + 1/2 over the pixels; a dead (necrotic)
    # cell at the centre and a cell with no pixels are left out
    from oracle.cpu_sim import lesion_joining
    grid = np.zeros((20, 20), np.int32)
    grid[8:12, 8:12] = 1      # centre (10, 10): in
    grid[8:12, 13:17] = 2     # centre (15, 10): 5 from the middle, in at radius 5
    grid[0:2, 0:2] = 3        # centre (1, 1): out
    grid[12:14, 8:10] = 4     # necrotic, centre (9, 13): left out
    types = np.array([0, 1, 1, 2, 3, 1], np.int32)
    volume = np.array([0, 16, 16, 4, 4, 0], np.int32)  # record 5 holds no pixel
    assert lesion_joining(grid, types, volume, (3, -1, -1), None, 5.0) == [1, 2]
    assert lesion_joining(grid, types, volume, (3, -1, -1), None, 4.99) == [1]
    assert lesion_joining(grid, types, volume, (3, -1, -1), (1.0, 1.0), 0.5) == [3]


def test_tracing_marks_the_cells_in_the_layer_and_daughters_carry_them():
    # mark_every_cell and traced_clones (simulation.rs:1908-1918, 2407-2421)
    # on the oracle's history: marked at the step, each cell its own mark
    import json
    import os
    from oracle.cpu_sim import CpuHistory
    spec = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))["networks"]["epithelium"]
    cfg = dict(dims=[(40, 40, 1)], ncells=[16], seeds=[3], temperature=10.0,
               J=np.array([[0, 16, 16, 12, 12, 12], [16, 2, 11, 10, 11, 10], [16, 11, 6, 12, 6, 12],
                           [12, 10, 12, 8, 12, 8], [12, 11, 6, 12, 6, 12], [12, 10, 12, 8, 12, 8]], float),
               contact_order=1, target_volume=0, lambda_volume=50.0, seeding=4, seed_side=10, nfields=1,
               o2_dcoef=0.2, o2_sink_by_type=(0, 0, 0, 0), o2_hold=3, tolerance=1e-8, field_off=True, dt=1.0,
               substeps=8, sweeps=1, death_threshold=0.25, necrotic_type=3, divide=True, max_cells=2000,
               differentiated_type=4, apoptotic_type=5, lineage=True, hypoxic_level=0.1, network_spec=spec,
               tracing_at=2)
    h = CpuHistory(cfg, 0)
    h.step()
    h.step()
    assert h.traced_clones() == []
    h.step()
    tr = h.traced_clones()
    assert [m for m, _ in tr] == list(range(16)) and all(c == 1 for _, c in tr)


# ---------------------------------------------------------------- closing over dead tissue and shut-in fluid
# cpm.rs:1702-1803 on the oracle's break_down_debris / drain_shut_in helpers


def _closing(blocks, size=30):
    """A lattice of rectangles (kind, x, y, w, h), kinds 1 tumour and 3
    necrotic, as the reference's add_block lays them; ids from 1 in order."""
    from oracle import cpu_sim
    g = np.zeros((size, size), np.int32)
    kinds = [0]
    for i, (kind, x, y, w, h) in enumerate(blocks, start=1):
        g[y:y + h, x:x + w] = i
        kinds.append(kind)
    lat = O.Lattice(g, (size, size, 1), len(kinds), np.zeros((4, 4)), 10.0)
    lat.type[:] = kinds
    lat.volume[:] = np.bincount(lat.grid.clip(0), minlength=len(kinds))
    lat.volume[0] = 0
    hist = cpu_sim.CpuHistory.__new__(cpu_sim.CpuHistory)  # the helpers read only these
    hist.lat, hist.cfg, hist.div_rng = lat, {"necrotic_type": 3}, np.random.default_rng(3)
    return hist, cpu_sim.CpuHistory


def test_a_pixel_closed_over_goes_to_living_tissue_never_to_the_dead_or_the_medium():
    # cpm.rs:1702-1727: dead block at (10, 10), tumour at (15, 10), dead at (10, 15)
    hist, H = _closing([(3, 10, 10, 5, 5), (1, 15, 10, 5, 5), (3, 10, 15, 5, 5)])
    faces = H._faces(hist)
    at = lambda x, y: y * 30 + x
    ids, n = H._living_around(hist, np.array([at(12, 14), at(12, 12), at(14, 12), at(10, 12)]), faces)
    # against dead tissue alone, inside its own cell, against medium alone: no taker
    assert list(n) == [0, 0, 1, 0]
    # against the living cell and nothing else, the living cell takes it
    assert sorted(ids[2][ids[2] > 0]) == [2]
    assert H._give(hist, np.array([at(14, 12)]), ids[2:3], n[2:3], hist.div_rng)[0] == 2


def test_fluid_shut_in_is_closed_in_by_the_living_only():
    # cpm.rs:1771-1803: four cells around a 4 x 4 hole at x, y 13..16, the right one dead
    hist, H = _closing([(1, 10, 10, 10, 3), (1, 10, 17, 10, 3), (1, 10, 13, 3, 4), (3, 17, 13, 3, 4)])
    hole = [y * 30 + x for y in range(13, 17) for x in range(13, 17)]
    scratch = O.Field(30, 30, 1)
    scratch.hold_bath(hist.lat.grid == 0, 1.0)
    assert list(np.nonzero((hist.lat.grid == 0) & (scratch.held == 0))[0]) == hole
    before = int(hist.lat.volume.sum())
    H._drain_shut_in(hist)
    g = hist.lat.grid.reshape(30, 30)
    # every hole pixel with living tissue across a face went to a living cell;
    # those beside only the dead cell or only more fluid stay fluid
    closed = {(x, y) for y in range(13, 17) for x in range(13, 17) if g[y, x] != 0}
    want = {(x, 13) for x in range(13, 17)} | {(x, 16) for x in range(13, 17)} | {(13, 14), (13, 15)}
    assert closed == want
    assert all(g[y, x] in (1, 2, 3) for x, y in closed)
    assert int(hist.lat.volume.sum()) == before + len(want)
    assert np.array_equal(np.bincount(hist.lat.grid.clip(0), minlength=5)[1:], hist.lat.volume[1:])


def test_an_exposure_is_on_when_its_schedule_says():
    # crates/io/tests/stress.rs:71-84 on the oracle's Exposure::level_at
    from oracle import cpu_sim
    hist = cpu_sim.CpuHistory.__new__(cpu_sim.CpuHistory)
    hist.cfg = {"exposure_intensity": 0.8, "exposure_start": 10, "exposure_on": 3, "exposure_off": 2}
    assert [hist._level_at(m) for m in range(8, 20)] == [0, 0, .8, .8, .8, 0, 0, .8, .8, .8, 0, 0]
    hist.cfg = {"exposure_intensity": 1.0, "exposure_start": 5, "exposure_on": 0, "exposure_off": 0}
    assert hist._level_at(4) == 0.0 and hist._level_at(500) == 1.0


def test_a_sheet_fills_the_box_with_one_cell_per_square():
    # crates/io/tests/epithelium.rs:68-81 on the oracle's seeding: a 40 x 40
    # box tiled by 10 x 10 cells of normal tissue, no medium, 16 cells
    from oracle import cpu_sim
    cfg = {"seeding": 4, "seed_side": 10, "J": np.zeros((4, 4))}
    grid, types = cpu_sim.seed_history(cfg, 40, 40, 1, 0, 1)
    assert (grid != 0).all() and len(types) == 17 and (types[1:] == 2).all()
    assert sorted(np.bincount(grid.reshape(-1))[1:]) == [100] * 16
    assert grid[0, 0, 0] == 1 and grid[0, 0, 39] == 4 and grid[0, 39, 0] == 13
