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
