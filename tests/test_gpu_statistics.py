"""The device's dynamics as distributions over 32 seeds (GPU).

The CPM: 32 histories swept in one batch on the device against the oracle's
restatement of the reference's sequential random-pixel sweep (cpm.rs:748-838)
from the same starting lattices: pooled cell volumes alike (KS test, spread,
mean), the boundary length inside the sequential ensemble's band.

The whole step: 32 histories of a small cord-like campaign stepped by the
device against the CPU oracle stepping the reference's algorithms one
history at a time (sequential sweep, FP64 SOR, RK4; oracle/cpu_sim.py):
population, mean oxygen over the cells, the hypoxic fraction of the living
cells and the hypoxic radius (how many rows from the held source row the
oxygen stays above the hypoxic level) inside the oracle's band at several
steps.
"""
import os
import tempfile

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import synthetic
from cpm_ensembles import J, ORDER, SEEDS, SIZE, T, observables, oracle_ensemble, same_volume_law, sheet, within_band
from oracle import oracle as O
from oracle.cpu_sim import CpuHistory, measure_records

pytestmark = pytest.mark.gpu


def test_device_sweeps_match_the_sequential_ensemble():
    mcs = 60
    sheets = [sheet(k) for k in range(SEEDS)]
    lat = cw.CpmLattice.from_grids([g for g, _ in sheets], [r for _, r in sheets], T, J, ORDER,
                                   seeds=[1_000_003 * k + 17 for k in range(SEEDS)])
    lat.monte_carlo_step(mcs)
    vols, bnd = [], []
    for k in range(SEEDS):
        assert lat.records_match_grid(k)
        g = lat.grid(k).reshape(SIZE, SIZE)
        v, b = observables(g, np.bincount(g[g >= 0].ravel(), minlength=len(sheets[k][1])))
        vols.append(v)
        bnd.append(b)
    dev_v, dev_b = np.concatenate(vols), np.array(bnd, float)
    seq_v, seq_b = oracle_ensemble("sequential", mcs)
    assert same_volume_law(seq_v, dev_v), (seq_v.std(), dev_v.std())
    assert within_band(dev_b, seq_b), (seq_b.mean(), seq_b.std(), dev_b.mean())


def small_cord(n=SEEDS):
    cfg = synthetic.campaign(per_size=n, sizes=(64,), fill=0.45)
    cfg.update(necrotic_type=3, death_threshold=0.25, J=synthetic.contact_table(4, seed=2), dt=0.03,
               o2_sink_by_type=(0.0, 0.03, 0.03, 0.0))
    return cfg


def hypoxic_radius(o2, size, level):
    """How deep the tissue is fed: the distance from the held source row (row
    0) at which the row-mean oxygen first falls under the hypoxic level,
    interpolated between rows (the box's height if it never does)."""
    rows = np.asarray(o2, float).reshape(-1, size).mean(axis=1)
    below = np.flatnonzero(rows < level)
    if not below.size:
        return float(len(rows))
    j = int(below[0])
    if j == 0:
        return 0.0
    return (j - 1) + float((rows[j - 1] - level) / (rows[j - 1] - rows[j]))


def per_history(grid, o2, volume, types, necrotic, level, size=64):
    living = (volume > 0) & (types != necrotic)
    living[0] = False
    means = O.mean_per_cell(grid, o2, len(volume))
    cells = np.flatnonzero(living)
    return (len(cells), float(means[cells].mean()), float((means[cells] < level).mean()),
            hypoxic_radius(o2, size, level))


@pytest.mark.parametrize("subsweeps", [1, 4])
def test_the_step_stays_inside_the_oracle_band(subsweeps):
    # one sweep of every colour a step attempts each pixel once where random
    # pixels attempt it Poisson(1) times: a favoured copy happens at once, not
    # with probability 1 - 1/e, so the necrotic cells' resorption (a target
    # two pixels under their volume each step) runs ahead, and the dead are
    # gone sooner; with four sub-sweeps a step (each pixel attempting in each
    # with probability 1/4) the tissue and necrotic radii and the cells gone
    # come inside the band as well
    cfg = small_cord()
    S = cfg.pop("S")
    d = tempfile.mkdtemp()
    p = os.path.join(d, "n.toml")
    open(p, "w").write(synthetic.network_toml(S, S))
    net = cw.Network.load(p, cfg["target_volume"])
    sim = cw.Simulation(net, **dict(cfg, seeds=[s + 50_000 for s in cfg["seeds"]], subsweeps=subsweeps))
    ora = [CpuHistory(dict(cfg, S=S), k) for k in range(SEEDS)]
    for step in range(1, 31):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (5, 15, 30):
            continue
        dev, ref = [], []
        lat = sim.lattice()
        for k in range(SEEDS):
            cells = lat.cells(hist=k)
            dev.append(per_history(sim.grid(k), sim.field_values(0, k), cells["volume"], cells["type"], 3,
                                   cfg["hypoxic_level"]))
            h = ora[k]
            ref.append(per_history(h.lat.grid, h.o2.values, h.lat.volume, h.lat.type, 3, cfg["hypoxic_level"]))
        # the reference's own geometry (measure.rs): tissue and necrotic radii,
        # and how deep living tissue reaches from the held row
        radii = ("tissue_radius", "necrotic_radius", "gone", "viable_depth") if subsweeps > 1 else ("viable_depth",)
        dm = sim.measure()
        dev = [list(r) + [dm[k][q] for q in radii] for k, r in enumerate(dev)]
        ref = [list(r) + [ora[k].measure()[q] for q in radii] for k, r in enumerate(ref)]
        dev, ref = np.array(dev), np.array(ref)
        for j, name in enumerate(("living", "mean oxygen", "hypoxic fraction", "hypoxic radius") + radii):
            assert within_band(dev[:, j], ref[:, j]), (step, name, dev[:, j].mean(), ref[:, j].mean(),
                                                        ref[:, j].std())


def test_division_grows_the_population_inside_the_oracle_band():
    # cells of the reference volume grow as their growth node rises (growth
    # coefficient 2) and divide at 1.4 times it, up to 40 living cells: the
    # population curve inside the 32-seed band of the oracle's
    # divide_ready_cells.  Sweeps attempt every boundary pixel once per MCS
    # where random pixels attempt it Poisson(1) times, so driven volumes
    # follow their targets faster (a change of probability p per MCS instead
    # of 1 - exp(-p)); the population runs about 7% ahead by step 30, inside
    # the band, which is the test.
    cfg = synthetic.campaign(per_size=SEEDS, sizes=(64,), fill=0.2)
    cfg.update(max_cells=40, dt=0.1)
    S = cfg.pop("S")
    text = synthetic.network_toml(S, S).replace("growth_coefficient = 0.5", "growth_coefficient = 2.0")
    assert "growth_coefficient = 2.0" in text
    d = tempfile.mkdtemp()
    p = os.path.join(d, "n.toml")
    open(p, "w").write(text)
    net = cw.Network.load(p, cfg["target_volume"])
    sim = cw.Simulation(net, **dict(cfg, seeds=[s + 70_000 for s in cfg["seeds"]]))
    ora = [CpuHistory(dict(cfg, S=S, network_toml=text), k) for k in range(SEEDS)]
    start = np.array([sim.lattice().cell_count(k) for k in range(SEEDS)])
    for step in range(1, 31):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (10, 20, 30):
            continue
        lat = sim.lattice()
        dev = np.array([float((lat.cells(hist=k)["volume"][1:] > 0).sum()) for k in range(SEEDS)])
        ref = np.array([float((h.lat.volume[1:h.used] > 0).sum()) for h in ora])
        assert within_band(dev, ref, z=None), (step, dev.mean(), ref.mean(), ref.std())
        assert dev.max() <= 40 + 40  # the limit counts the living before a step's divisions
    for k in range(SEEDS):
        assert sim.records_match_grid(k)
    grown = np.array([sim.lattice().cell_count(k) for k in range(SEEDS)]) - start
    assert grown.mean() > 5


def released_network(S):
    # the synthetic network, its survival node also damaged by the necrotic
    # factor and its growth node inhibited by the waste
    text = synthetic.network_toml(S, S)
    old = '{ kind = "relaxes_to", value = 0.9, rate = 2.0 },'
    assert text.count(old) == 1
    text = text.replace(old, old + '\n  { kind = "damaged_above", source = "necrotic_factor", threshold = 0.02, rate = 1.0 },')
    grow = 'name = "n2"\ninitial = 0.1\nterms = [\n'
    assert text.count(grow) == 1
    text = text.replace(grow, grow + '  { kind = "inhibited_by", source = "waste", rate = 0.5 },\n')
    return text


def test_the_released_fields_stay_inside_the_oracle_band():
    # settle_waste / settle_necrotic_factor (simulation.rs:2057-2113): the
    # waste from every living pixel, the necrotic factor from the dead for 20
    # steps after they died, both held at zero on the bath and read by the
    # network; living cells, their mean oxygen, waste and factor inside the
    # oracle's 32-seed band
    cfg = small_cord()
    cfg.update(waste_production=0.01, necrotic_production=0.05, necrotic_release_for=20)
    S = cfg.pop("S")
    text = released_network(S)
    d = tempfile.mkdtemp()
    p = os.path.join(d, "n.toml")
    open(p, "w").write(text)
    net = cw.Network.load(p, cfg["target_volume"])
    sim = cw.Simulation(net, **dict(cfg, seeds=[s + 90_000 for s in cfg["seeds"]]))
    ora = [CpuHistory(dict(cfg, S=S, network_toml=text), k) for k in range(SEEDS)]
    names = ("living", "mean oxygen", "mean waste", "mean necrotic factor")
    for step in range(1, 31):
        sim.step(1)
        for h in ora:
            h.step()
        if step not in (5, 15, 30):
            continue
        dev, ref = [], []
        lat = sim.lattice()
        for k in range(SEEDS):
            cells = lat.cells(hist=k)
            g = sim.grid(k)
            vol, types = cells["volume"], cells["type"]
            living = np.flatnonzero((vol > 0) & (types != 3) & (np.arange(len(vol)) > 0))
            row = [len(living)]
            for f in (0, 2, 3):
                m = O.mean_per_cell(g, sim.field_values(f, k), len(vol))
                row.append(float(m[living].mean()))
            dev.append(row)
            h = ora[k]
            hl = np.flatnonzero((h.lat.volume > 0) & (h.lat.type != 3) & (np.arange(len(h.lat.volume)) > 0))
            rrow = [len(hl)]
            for fld in (h.o2, h.wst, h.nfc):
                m = O.mean_per_cell(h.lat.grid, fld.values, len(h.lat.volume))
                rrow.append(float(m[hl].mean()))
            ref.append(rrow)
        dev, ref = np.array(dev), np.array(ref)
        assert ref[:, 2].mean() > 1e-3
        # the factor once the first dead have stopped releasing is what the
        # solves' tolerance leaves of a sourceless field: compared while they release
        checked = names if step <= 15 else names[:3]
        if step <= 15:
            assert ref[:, 3].mean() > 1e-3
        for j, name in enumerate(checked):
            assert within_band(dev[:, j], ref[:, j]), (step, name, dev[:, j].mean(), ref[:, j].mean(),
                                                        ref[:, j].std())
    for k in range(SEEDS):
        assert sim.records_match_grid(k)


def test_the_bath_holds_the_oxygen_where_the_medium_reaches_the_edge():
    # declare_sources with a bath (simulation.rs:2138-2146): the medium the
    # bath reaches held at the source's level, the cells taking it up
    cfg = small_cord(4)
    cfg.update(o2_hold=3)
    S = cfg.pop("S")
    d = tempfile.mkdtemp()
    p = os.path.join(d, "n.toml")
    open(p, "w").write(synthetic.network_toml(S, S))
    net = cw.Network.load(p, cfg["target_volume"])
    sim = cw.Simulation(net, **cfg)
    baths = [sim.lattice().bath(k).reshape(-1) for k in range(4)]
    grids = [sim.grid(k).reshape(-1).copy() for k in range(4)]
    sim.step(1)
    for k in range(4):
        v = sim.field_values(0, k)
        bath = baths[k].astype(bool)
        assert bath.sum() > 0
        np.testing.assert_array_equal(v[bath], 1.0)
        assert v[grids[k] > 0].min() < 1.0
        o = O.Field(64, 64, 1, 1.0, 0.0, 0.0)
        o.hold_bath(grids[k] == 0, 1.0)
        np.testing.assert_array_equal(baths[k], o.held.astype(np.uint8))


def test_the_device_measures_as_the_reference_does():
    # Simulation::measure (measure.rs:133-236) on the device against the
    # oracle's restatement applied to the device's own lattice and network
    # state, for each oxygen hold
    for hold in (0, 1, 2, 3):
        cfg = small_cord(4)
        cfg.update(o2_hold=hold)
        S = cfg.pop("S")
        d = tempfile.mkdtemp()
        p = os.path.join(d, "n.toml")
        open(p, "w").write(synthetic.network_toml(S, S))
        net = cw.Network.load(p, cfg["target_volume"])
        sim = cw.Simulation(net, **cfg)
        sim.step(12)
        got = sim.measure()
        lat = sim.lattice()
        hyp = net.roles["hypoxia_response"]
        for k in range(4):
            used = lat.cell_count(k)
            cells = lat.cells(hist=k)
            state = sim.network_state(len(cells["volume"]), k)
            want = measure_records(sim.grid(k), cells["type"], cells["volume"], used, state[:, hyp], 3, hold, 11)
            for key in ("mcs", "cycling", "quiescent", "necrotic", "born", "gone", "vessel"):
                assert got[k][key] == want[key], (hold, k, key, got[k][key], want[key])
            for key in ("tissue_radius", "necrotic_radius", "viable_depth"):
                assert abs(got[k][key] - want[key]) <= 1e-12 * max(1.0, abs(want[key])), (hold, k, key)
            assert got[k]["cycling"] + got[k]["quiescent"] > 0
