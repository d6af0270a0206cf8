"""The device RK4 network against the reference's golden table and the oracle (GPU)."""
import os

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_ras_erk_golden_table(golden):
    # network.rs:866-891, 1e-12
    net = cw.Network.from_spec(golden["networks"]["ras-erk"], 200)
    for row in golden["ras_erk_rk4"]:
        st = net.initial.reshape(1, -1).copy()
        net.step_batch(st, np.array([[row["o2"], row["egf"], 0, 0, 0, 0]], float), 1.0, row["steps"])
        np.testing.assert_allclose(st[0], row["expected"], rtol=0, atol=1e-12, err_msg=row["source"])


def test_mechanics_after_forty_steps(golden):
    # network.rs:893-902, 951-965
    spec = golden["networks"]["ras-erk"]
    net = cw.Network.from_spec(spec, 200)
    st = net.initial.reshape(1, -1).copy()
    net.step_batch(st, np.array([[0.8, 0.2, 0, 0, 0, 0]], float), 1.0, 40)
    tgt, lam = net.mechanics_batch(st)
    assert tgt[0] == 299 and lam[0] == 50.0
    capped = cw.Network.from_spec(dict(spec, mechanics=dict(spec["mechanics"], max_target=1.2)), 200)
    assert capped.mechanics_batch(st)[0][0] == 240


@pytest.mark.parametrize("name", ["ras-erk", "fuller-cell", "stress-response", "epithelium", "ras-erk-mutant"])
def test_shipped_networks_match_the_oracle_bit_for_bit(golden, name):
    spec = golden["networks"][name]
    net = cw.Network.from_spec(spec, 200)
    ref = O.compile_network(spec, 200)
    rng = np.random.default_rng(1)
    n = 300
    st = np.tile(net.initial, (n, 1)) * rng.uniform(0.5, 1.5, (n, net.S))
    st = np.clip(st, 0, 1)
    ins = rng.uniform(0, 1, (n, 6))
    a, b = st.copy(), st.copy()
    net.step_batch(a, ins, 1.0, 8)
    O.network_step(ref, b, ins, 1.0, 8)
    hill = any(t.get("hill") for nd in spec["nodes"] for t in nd.get("terms", []))
    if hill:
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-14)
    else:
        np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("S", [8, 12, 16])
def test_synthetic_hill_networks_match_the_oracle(tmp_path, S):
    text = synthetic.network_toml(S, seed=S)
    path = tmp_path / "net.toml"
    path.write_text(text)
    spec = cw.load_network_spec(str(path))
    net = cw.Network.from_spec(spec, 64)
    ref = O.compile_network(spec, 64)
    rng = np.random.default_rng(2)
    n = 1000
    st = rng.uniform(0, 1, (n, S))
    ins = rng.uniform(0, 1, (n, 6))
    a, b = st.copy(), st.copy()
    net.step_batch(a, ins, 0.01, 8)
    O.network_step(ref, b, ins, 0.01, 8)
    # the device squares for a Hill exponent of two where libm's pow (the
    # reference's powf) may differ by an ulp: equal to 1e-12 relative
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)


def test_refusals_name_the_culprit():
    one = lambda terms: {"nodes": [{"name": "a", "initial": 0.0, "terms": terms}],
                         "roles": {"growth": "a", "survival": "a", "hypoxia_response": "a"},
                         "mechanics": {"growth_coefficient": 1.0, "lambda_volume": 1.0}}
    with pytest.raises(cw.ConfigError, match="p53"):
        cw.Network.from_spec(one([{"kind": "activated_by", "source": "p53", "rate": 1.0}]), 100)
    with pytest.raises(cw.ConfigError, match="oxygen"):
        cw.Network.from_spec({**one([]), "nodes": [{"name": "oxygen"}],
                              "roles": {"growth": "oxygen", "survival": "oxygen", "hypoxia_response": "oxygen"}}, 1)
    with pytest.raises(cw.ConfigError, match="bcl2"):
        cw.Network.from_spec({**one([]), "roles": {"growth": "a", "survival": "bcl2", "hypoxia_response": "a"}}, 1)
    with pytest.raises(cw.ConfigError):
        cw.Network.from_spec(one([{"kind": "activated_by", "source": "egf", "rate": 1.0,
                                   "hill": {"n": 2.0, "k": 0.0}}]), 1)
    with pytest.raises(cw.ConfigError):
        cw.Network.from_spec({**one([]), "nodes": []}, 1)


# ---------------------------------------------------------------- mutated networks
DRAWS = [(0.0, 0.5), (0.99, 0.999_999), (0.37, 0.1), (0.62, 0.93)]
REWIRES = [[0.0, 0.0, 0.0, 0.0, 0.5], [0.9, 0.0, 0.0, 0.0, 0.0], [0.2, 0.7, 0.95, 0.6, 0.3],
           [0.4, 0.99, 0.5, 0.1, 0.8], [0.75, 0.55, 0.0, 0.0, 0.0]]


def same_record(dev, ref):
    keys = ("node", "term", "kind", "change")
    assert tuple(dev[k] for k in keys) == tuple(ref[k] for k in keys)
    assert dev["text"] == O.mutation_text(ref)
    if ref["change"] == "scaled":
        assert dev["factor"] == ref["factor"]
    if ref["change"] == "gained":
        assert dev["source"] == ref["source"] and dev["rate"] == ref["rate"]


def test_mutations_on_the_device_match_the_oracle(golden):
    # Network::mutate / rewire (network.rs:479-575): the same pick, factor,
    # gained source and rate as the oracle's restatement
    spec = golden["networks"]["ras-erk"]
    net = cw.Network.from_spec(spec, 200)
    for which, how in DRAWS:
        _, rec = net.mutate(which, how)
        same_record(rec, O.mutate_spec(spec, which, how)[1])
    for d in REWIRES:
        _, rec = net.rewire(d)
        same_record(rec, O.rewire_spec(spec, d)[1])


def test_a_batch_of_clones_steps_each_cell_under_its_own_network(golden, tmp_path):
    # the per-cell networks of an evolving run: every cell of one launch under
    # the network its clone has, against the oracle stepping each clone's
    # table alone; bit for bit without Hill terms, 1e-12 with them
    for name, spec, dt, exact in [("ras-erk", golden["networks"]["ras-erk"], 1.0, True),
                                  ("synthetic", None, 0.01, False)]:
        if spec is None:
            p = tmp_path / "net.toml"
            p.write_text(synthetic.network_toml(8, seed=8))
            spec = cw.load_network_spec(str(p))
        founder = cw.Network.from_spec(spec, 64)
        nets, specs = [founder], [spec]
        for which, how in DRAWS[1:]:
            n, _ = founder.mutate(which, how)
            nets.append(n)
            specs.append(O.mutate_spec(spec, which, how)[0])
        for d in REWIRES:
            n, _ = nets[-1].rewire(d)
            nets.append(n)
            specs.append(O.rewire_spec(specs[-1], d)[0])
        rng = np.random.default_rng(3)
        ncell = 700
        clone = rng.integers(0, len(nets), ncell).astype(np.int32)
        st = rng.uniform(0, 1, (ncell, founder.S))
        ins = rng.uniform(0, 1, (ncell, 6))
        got = st.copy()
        cw.Network.step_clones(nets, clone, got, ins, dt, 8)
        want = st.copy()
        for k, s in enumerate(specs):
            rows = np.flatnonzero(clone == k)
            sub = want[rows].copy()
            O.network_step(O.compile_network(s, 64), sub, ins[rows], dt, 8)
            want[rows] = sub
        if exact:
            np.testing.assert_array_equal(got.view(np.uint64), want.view(np.uint64), err_msg=name)
        else:
            np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-15, err_msg=name)
        # and one network's cells alone are what step_batch gives
        one = st[clone == 0].copy()
        founder.step_batch(one, ins[clone == 0], dt, 8)
        np.testing.assert_array_equal(one.view(np.uint64), got[clone == 0].view(np.uint64))


def test_mutations_refuse_what_the_reference_cannot_do(golden):
    bare = {"nodes": [{"name": "a", "initial": 0.1}], "roles": {"growth": "a", "survival": "a",
            "hypoxia_response": "a"}, "mechanics": {"growth_coefficient": 0.5, "lambda_volume": 10.0}}
    net = cw.Network.from_spec(bare, 50)
    with pytest.raises(cw.NotFoundError):
        net.mutate(0.5, 0.5)
    with pytest.raises(cw.NotFoundError):
        net.rewire([0.9, 0.0, 0.0, 0.0, 0.0])
    gained, rec = net.rewire([0.1, 0.0, 0.99, 0.0, 0.5])  # a gain needs no term: reads itself
    assert rec["text"] == "a gains activated_by a @0.10"
    ras = cw.Network.from_spec(golden["networks"]["ras-erk"], 200)
    st = np.full((3, ras.S), 0.5)
    with pytest.raises(cw.ConfigError):
        cw.Network.step_clones([ras, gained], np.zeros(3, np.int32), st, np.zeros((3, 6)), 1.0)
    with pytest.raises(cw.ConfigError):
        cw.Network.step_clones([ras], np.array([0, 1, 0], np.int32), st, np.zeros((3, 6)), 1.0)


def test_the_step_feeds_each_cell_its_crowding():
    # cell_inputs / crowding (simulation.rs:2511-2527): a network that reads
    # crowding, 1 - volume / reference volume clamped to [0, 1], steps every
    # living cell from its volume before the step's Monte Carlo sweep
    spec = {"nodes": [{"name": "a", "initial": 0.1, "terms": [
        {"kind": "activated_by", "source": "crowding", "rate": 1.0}, {"kind": "decays", "rate": 0.5}]}],
        "roles": {"growth": "a", "survival": "a", "hypoxia_response": "a"},
        "mechanics": {"growth_coefficient": 0.0, "lambda_volume": 1.0}}
    ref_volume = 60
    net = cw.Network.from_spec(spec, ref_volume)
    J = np.array([[0, 16, 16], [16, 8, 12], [16, 12, 8]], float)
    sim = cw.Simulation(net, [(64, 64, 1)], [20], [7], J=J, target_volume=49, nfields=1, dt=0.25, substeps=4,
                        death_threshold=0.0, divide=False)
    cells = sim.lattice().cells(hist=0)
    n = len(cells["volume"])
    sim.step(1)
    got = sim.network_state(n)
    vol = cells["volume"].astype(float)
    live = np.flatnonzero((vol > 0) & (np.arange(n) > 0))
    assert len(live) > 5
    ins = np.zeros((len(live), 6))
    ins[:, 1] = 0.2
    ins[:, 2] = np.clip(1.0 - vol[live] / ref_volume, 0.0, 1.0)
    want = np.full((len(live), 1), 0.1)
    O.network_step(O.compile_network(spec, ref_volume), want, ins, 0.25, 4)
    np.testing.assert_array_equal(got[live].view(np.uint64), want.view(np.uint64))
    assert (ins[:, 2] > 0.1).all()


def _device_settled(spec, o2, stress, steps=600):
    net = cw.Network.from_spec(spec, 100)
    st = net.initial.reshape(1, -1).copy()
    net.step_batch(st, np.array([[o2, 0.2, 0, stress, 0, 0]], float), 1.0, steps)
    return st[0]


def test_the_fuller_cell_decides_as_the_networks_it_fills_in_on_the_device(golden):
    # crates/io/tests/fuller_cell.rs:69-136, settled by 600 RK4 steps on the
    # device; each settled state equals the oracle's, and the decisions match
    nets = golden["networks"]
    ref = {k: O.compile_network(nets[k], 100) for k in ("fuller-cell", "ras-erk", "stress-response")}
    got = {}
    for k in ref:
        for o2, stress in [(1.0, 0.0), (0.1, 0.0), (0.05, 0.0), (1.0, 0.5), (1.0, 1.0)]:
            dev = _device_settled(nets[k], o2, stress)
            want = ref[k].initial.reshape(1, -1).copy()
            O.network_step(ref[k], want, np.array([[o2, 0.2, 0, stress, 0, 0]], float), 1.0, 600)
            # Hill terms through pow: a few ulps a step, damped as the state settles
            np.testing.assert_allclose(dev, want[0], rtol=1e-10, atol=1e-12)
            got[k, o2, stress] = dev
    f, r, s = ref["fuller-cell"], ref["ras-erk"], ref["stress-response"]
    erk = lambda net, st: st[net.names.index("erk")]
    assert abs(erk(f, got["fuller-cell", 1.0, 0.0]) - erk(r, got["ras-erk", 1.0, 0.0])) < 0.002
    for o2 in (0.1, 0.05):
        assert abs(got["fuller-cell", o2, 0.0][f.survival] - got["ras-erk", o2, 0.0][r.survival]) < 0.002
    for stress in (0.5, 1.0):
        a = got["fuller-cell", 1.0, stress][f.optional["apoptosis"]]
        b = got["stress-response", 1.0, stress][s.optional["apoptosis"]]
        assert abs(a - b) < 0.015


def test_one_node_inputs_reach_the_device_as_the_reference_reads_them():
    # network.rs:1268-1342, 1445-1482: waste, the necrotic factor past its
    # threshold, a node at zero not damaged below it, crowding read by a
    # differentiation node
    def one(terms, initial=0.0):
        return {"nodes": [{"name": "a", "initial": initial, "terms": terms}],
                "roles": {"growth": "a", "survival": "a", "hypoxia_response": "a"},
                "mechanics": {"growth_coefficient": 1.0, "lambda_volume": 1.0}}

    def run(spec, inputs, dt, steps):
        net = cw.Network.from_spec(spec, 100)
        st = net.initial.reshape(1, -1).copy()
        net.step_batch(st, np.array([inputs], float), dt, steps)
        return st[0, 0]
    slope = (run(one([{"kind": "activated_by", "source": "waste", "rate": 2.0}], 0.25),
                 [1, 0, 0, 0, 0.5, 0], 1e-6, 1) - 0.25) / 1e-6
    assert abs(slope - 0.75) < 1e-5
    above = one([{"kind": "damaged_above", "source": "necrotic_factor", "threshold": 0.5, "rate": 2.0}], 0.5)
    assert abs((run(above, [1, 0, 0, 0, 0, 0.4], 1e-6, 1) - 0.5) / 1e-6) < 1e-9
    assert abs((run(above, [1, 0, 0, 0, 0, 1.0], 1e-6, 1) - 0.5) / 1e-6 + 2.0) < 1e-5
    below = one([{"kind": "damaged_below", "source": "oxygen", "threshold": 0.5, "rate": 10.0}])
    assert run(below, [0, 0, 0, 0, 0, 0], 1.0, 50) == 0.0
    crowd = one([{"kind": "activated_by", "source": "crowding", "rate": 1.0}, {"kind": "decays", "rate": 1.0}])
    crowd["roles"]["differentiation"] = "a"
    assert abs(run(crowd, [1, 0, 0.6, 0, 0, 0], 1.0, 40) - 0.6 / 1.6) < 1e-6
