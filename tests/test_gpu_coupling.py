"""Device coupling (coupling.rs) and the batched driver against the oracle (GPU)."""
import math

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import seeding, synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

J5 = np.array([[0, 16, 16, 12, 12], [16, 2, 11, 10, 6], [16, 11, 6, 12, 11], [12, 10, 12, 8, 10],
               [12, 6, 11, 10, 16]], float)


def cluster():
    """coupling.rs:211-224: one cell ringed by eight, plus an obstacle."""
    grid = seeding.empty(80, 80)
    rec = seeding.Records()
    c = seeding.add_cell(grid, rec, 1, (40, 40), 6)
    ring = [seeding.add_cell(grid, rec, 1 if k % 3 else 3, (round(40 + 13 * math.cos(k * math.tau / 8)),
                                                            round(40 + 13 * math.sin(k * math.tau / 8))), 6)
            for k in range(8)]
    seeding.add_obstacle_disc(grid, rec, (10, 10), 3)
    return grid, rec, c, ring


def test_uptake_production_bath_and_means_match_the_oracle():
    grid, rec, c, ring = cluster()
    types = np.array(rec.type, np.int32)
    rates = np.array([0.0, 0.003, 0.0, 0.0, 0.001])  # necrotic (3) consumes nothing
    lat = cw.CpmLattice.from_grids([grid], [rec], 10.0, J5, 1)
    f = cw.ScalarField.new(80, 80, 0.2, 0.0, 1.0)
    cw.apply_uptake(f, lat, rates)
    up = O.apply_uptake(grid, types, rates)
    np.testing.assert_array_equal(f.download(cw.engine.UPTAKE), up)
    cw.apply_background_uptake(f, lat, 0.0005)
    O.apply_background_uptake(grid, 0.0005, up)
    np.testing.assert_array_equal(f.download(cw.engine.UPTAKE), up)
    per_cell = np.linspace(0, 0.01, len(rec))
    cw.apply_production(f, lat, per_cell)
    np.testing.assert_array_equal(f.download(cw.engine.PRODUCTION), O.apply_production(grid, per_cell))
    # bath, then a relax, then means
    o = O.Field(80, 80, 1, 0.2, 0.0, 1.0)
    o.uptake[:] = up
    o.production[:] = O.apply_production(grid, per_cell)
    o.hold_bath(grid.reshape(-1) == 0, 1.0)
    O.hold_obstacles(grid, 0.5, o.held, o.values)
    cw.hold_medium_bath(f, lat, 1.0)
    cw.hold_obstacles_at(f, lat, 0.5)
    np.testing.assert_array_equal(f.held(), o.held)
    assert o.relax(1e-9, 50_000)[0] == 0
    f.relax(1e-9, 50_000)
    np.testing.assert_array_equal(f.values().view(np.uint64), o.values.view(np.uint64))
    got = cw.mean_per_cell(f, lat, len(rec))
    want = O.mean_per_cell(grid, o.values, len(rec))
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=0)
    assert got[0] == 0.0
    assert got[c] < max(got[r] for r in ring)


def test_vessels_held_by_their_delivery_match_the_oracle():
    """hold_vessels_by (coupling.rs:114-150) on a batch of two planes: vessel
    discs in tissue, a field that is not uniform, shares that are zero,
    negative, partial, above one and NaN; every hold and value equal the
    oracle's, history by history."""
    rng = np.random.default_rng(7)
    grids, recs, shares, fields = [], [], [], []
    for (w, h) in [(64, 48), (90, 90)]:
        grid = seeding.empty(w, h)
        rec = seeding.Records()
        for k in range(6):
            seeding.add_cell(grid, rec, 1 + k % 2, (int(rng.integers(8, w - 8)), int(rng.integers(8, h - 8))), 5)
        for k in range(4):
            seeding.add_obstacle_disc(grid, rec, (int(rng.integers(0, w)), int(rng.integers(0, h))), int(rng.integers(0, 4)))
        share = rng.choice([0.0, -0.5, 0.25, 0.5, 0.9, 1.0, 3.0, np.nan], size=w * h)
        grids.append(grid)
        recs.append(rec)
        shares.append(share)
        fields.append(rng.uniform(0.0, 1.2, size=w * h))
    lat = cw.CpmLattice.from_grids(grids, recs, 10.0, J5, 1)
    f = cw.ScalarField([(64, 48, 1), (90, 90, 1)], 0.2)
    for k in range(2):
        f.set_values(fields[k], k)
    cw.engine.hold_vessels_by(f, lat, 0.8, np.concatenate(shares))
    for k in range(2):
        held, values = np.zeros(fields[k].size, np.uint8), fields[k].copy()
        O.hold_vessels_by(grids[k].reshape(grids[k].shape[-2:]), 0.8, shares[k], held, values)
        assert held.any() and (held.sum() < (grids[k] == -1).sum())  # some held, some left free
        np.testing.assert_array_equal(f.held(k), held)
        np.testing.assert_array_equal(f.values(k).view(np.uint64), values.view(np.uint64))


def test_vessels_held_by_their_delivery_the_reference_cases():
    # coupling.rs:300-331 on the device
    grid = np.zeros((1, 1, 10), np.int32)
    grid[0, 0, :3] = -1
    rec = seeding.Records()
    lat = cw.CpmLattice.from_grids([grid], [rec], 10.0, J5, 1)
    f = cw.ScalarField.new(10, 1, 0.2)
    cw.engine.hold_vessels_by(f, lat, 2.0, [0.0, 0.5, 3.0] + [0.0] * 7)
    assert list(f.values()[:3]) == [0.0, 1.0, 2.0] and list(f.held()[:3]) == [0, 1, 1]
    grid = np.zeros((1, 1, 10), np.int32)
    grid[0, 0, 5] = -1
    lat = cw.CpmLattice.from_grids([grid], [rec], 10.0, J5, 1)
    f = cw.ScalarField.new(10, 1, 0.2, initial=0.9)
    cw.engine.hold_vessels_by(f, lat, 1.0, np.full(10, 0.5))
    assert f.values()[5] == 0.9 and f.held()[5] == 0
    cw.engine.hold_vessels_by(f, lat, 1.0, np.full(10, 1.0))
    assert f.values()[5] == 1.0 and f.held()[5] == 1
    v = cw.ScalarField.with_depth(10, 1, 2, 0.2)
    lv = cw.CpmLattice.from_grids([np.zeros((2, 1, 10), np.int32)], [rec], 10.0, J5, 1)
    with pytest.raises(cw.ConfigError):
        cw.engine.hold_vessels_by(v, lv, 1.0, np.zeros(20))


def small_sim(nh=3, precision=cw.FP32_DC):
    net_text = synthetic.network_toml(8, seed=8)
    import tempfile, os
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "n.toml")
        open(p, "w").write(net_text)
        net = cw.Network.load(p, 49)
    cfg = synthetic.campaign(per_size=1, sizes=(64, 96, 128)[:nh])
    cfg.pop("S")
    cfg["precision"] = precision
    return cw.Simulation(net, **cfg), net


def test_the_driver_steps_a_batch_and_keeps_its_books():
    sim, _ = small_sim()
    sim.step(5)
    st = sim.stats()
    for k in range(3):
        assert sim.records_match_grid(k)
        assert st[k, 0] > 0          # living cells
        assert 0 < st[k, 1] <= 1.0   # mean oxygen over cells
        assert st[k, 3] < 1e-6       # the last solve's residual
    v = sim.field_values(0, 0)
    assert v.min() >= 0 and v.max() <= 1.0 + 1e-12


def test_a_history_in_a_batch_runs_as_it_runs_alone():
    net_text = synthetic.network_toml(8, seed=8)
    import tempfile, os
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "n.toml")
        open(p, "w").write(net_text)
        net = cw.Network.load(p, 49)
    cfg = synthetic.campaign(per_size=1, sizes=(64, 96))
    cfg.pop("S")
    cfg["precision"] = cw.FP64
    cfg["tolerance"] = 1e-10
    both = cw.Simulation(net, **cfg)
    alone_cfg = dict(cfg, dims=cfg["dims"][1:], ncells=cfg["ncells"][1:], seeds=cfg["seeds"][1:])
    alone = cw.Simulation(net, **alone_cfg)
    both.step(3)
    alone.step(3)
    np.testing.assert_array_equal(both.grid(1), alone.grid(0))


def test_graph_replay_gives_the_same_histories():
    net_text = synthetic.network_toml(8, seed=8)
    import tempfile, os
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "n.toml")
        open(p, "w").write(net_text)
        net = cw.Network.load(p, 49)
    cfg = synthetic.campaign(per_size=1, sizes=(64, 96, 128))
    cfg.pop("S")
    cfg["omega"] = 1.9
    plain = cw.Simulation(net, **dict(cfg, use_graphs=False))
    graph = cw.Simulation(net, **dict(cfg, use_graphs=True))
    plain.step(8)
    graph.step(8)
    steps, misses, budgets = graph.graph_info()
    assert steps >= 5 and (budgets > 0).all()
    assert plain.graph_info()[0] == 0
    for k in range(3):
        np.testing.assert_array_equal(plain.grid(k), graph.grid(k))
        np.testing.assert_array_equal(plain.field_values(0, k), graph.field_values(0, k))
        assert graph.records_match_grid(k)
