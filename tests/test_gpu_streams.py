"""One stream and one error record per handle (GPU).

The reference's objects are borrowed exclusively by one caller at a time
(simulation.rs:456).  Here every handle queues its work on its own CUDA
stream and keeps its own last error, so that two simulations driven from two
host threads run at once and each gives exactly what it gives alone.
"""
import os
import tempfile
import threading

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import _lib, synthetic

pytestmark = pytest.mark.gpu


def network():
    d = tempfile.mkdtemp()
    p = os.path.join(d, "n.toml")
    open(p, "w").write(synthetic.network_toml(8, seed=8))
    return cw.Network.load(p, 49)


def config(sizes, base_seed):
    cfg = synthetic.campaign(per_size=1, sizes=sizes, base_seed=base_seed)
    cfg.pop("S")
    cfg["omega"] = 1.9  # no tuning: the same factors on every run
    return cfg


def run(net, cfg, steps, out=None, key=None):
    sim = cw.Simulation(net, **cfg)
    sim.step(steps)
    nh = len(cfg["dims"])
    res = ([sim.grid(k) for k in range(nh)], [sim.field_values(0, k) for k in range(nh)])
    if out is not None:
        out[key] = res
    return res


def test_two_simulations_on_two_threads_each_give_their_solo_result():
    net = network()
    cfgs = [config((96, 128), 7000), config((128, 64), 8000)]
    steps = 6
    solo = [run(net, c, steps) for c in cfgs]
    out = {}
    ths = [threading.Thread(target=run, args=(net, c, steps, out, k)) for k, c in enumerate(cfgs)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for k in range(2):
        grids, fields = out[k]
        for h in range(2):
            np.testing.assert_array_equal(grids[h], solo[k][0][h])
            np.testing.assert_allclose(fields[h], solo[k][1][h], rtol=0, atol=1e-12)


def test_each_handle_has_its_own_stream_and_last_error():
    L = _lib.lib()
    net = network()
    a = cw.Simulation(net, **config((64,), 1))
    b = cw.Simulation(net, **config((64,), 2))
    sa, sb = L.cw_sim_get_stream(a._h), L.cw_sim_get_stream(b._h)
    assert sa and sb and sa != sb
    # a simulation's lattice and fields share its stream
    assert L.cw_lattice_get_stream(a.lattice_handle()) == sa
    assert L.cw_field_get_stream(a.field_handle(0)) == sa
    # a failure is recorded on the handle it happened on, and only there
    f1 = cw.ScalarField.new(16, 16, 1.0)
    f2 = cw.ScalarField.new(16, 16, 1.0)
    with pytest.raises(cw.ConfigError):
        f1.relax(-1.0, 10)
    assert b"tolerance" in L.cw_field_last_error(f1.handle)
    assert L.cw_field_last_error(f2.handle) == b""
    # a caller's stream handed in, then one of the handle's own again
    torch = pytest.importorskip("torch")
    s = torch.cuda.Stream()
    _lib.check(L.cw_sim_set_stream(a._h, s.cuda_stream))
    assert L.cw_sim_get_stream(a._h) == s.cuda_stream
    assert L.cw_lattice_get_stream(a.lattice_handle()) == s.cuda_stream
    a.step(2)
    assert a.records_match_grid(0)
    _lib.check(L.cw_sim_set_stream(a._h, None))
    own = L.cw_sim_get_stream(a._h)
    assert own and own != s.cuda_stream
    a.step(1)
    assert a.records_match_grid(0)
