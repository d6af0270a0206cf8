"""Parity at the benchmark configurations' own shapes (GPU).

The other device tests run on small lattices; these run the hot path at the
sizes it is measured on and hold it to the same bars:

* the plain 2D config (256 x 256, 120 cells, Moore contact, FP64 SOR at
  omega 1.85 to residual 1e-10 every 10 steps): the simulation's FP64 oxygen
  solve, from scratch and from the last solve with the lattice moved, equals
  the oracle's relax (pde.rs:245-405) to the bit; the sublattice sweep at
  256 x 256 equals the oracle's restatement of it for 12 Monte Carlo steps;
* a campaign history of 1024 x 1024, the large tumour cord (2048 x 2048,
  about 40,000 cells, oxygen and a secreted signal) and the 3D spheroid
  (256^3, 26-neighbour contact with surfaces): after some steps of the
  simulation, every field its FP32 defect-correction solve left is within
  1e-6 of the oracle's FP64 solve of the same problem (to residual 1e-12),
  relative to the field's largest value, field by field;
* the sweeps at those shapes (cells of 49, 64 and 125 pixels, 4 to 8
  colours, surfaces in the volume) finish every pass inside the round limit
  and keep the books (records_match_grid), and the 1024 x 1024 and 256^3
  sweeps equal the oracle's restatement.

The oracle's solve starts from the device's field: the FP64 solution to
residual 1e-12 does not depend on where SOR starts (it is the unique fixed
point, to about 1e-12 over the operator's smallest eigenvalue), and starting
near it keeps the CPU solve to seconds.
"""
import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# the north star's bound on a field against the FP64 oracle, relative to the
# field's scale (its largest value)
FIELD_REL = 1e-6


def network(S, refvol, tmp_path):
    p = tmp_path / f"synthetic-{S}.toml"
    p.write_text(synthetic.network_toml(S, S))
    return cw.Network.load(str(p), refvol)


def sim_of(cfg, tmp_path, **over):
    cfg = dict(cfg, **over)
    S = cfg.pop("S")
    net = network(S, cfg["target_volume"], tmp_path)
    return cw.Simulation(net, **cfg), cfg, net


def field_problem(sim, which, hist, dcoef, decay):
    """The problem a simulation's field `which` last solved, as an oracle Field
    holding the device's values (its coefficients are not repainted after the
    solve within a step)."""
    fh = sim.field_handle(which)
    w, h, d = sim.dims[hist]
    o = O.Field(w, h, d, dcoef, decay, 0.0)
    lib = cw._lib.lib()
    for which_arr, dest in ((cw.VALUES, "values"), (cw.UPTAKE, "uptake"), (cw.PRODUCTION, "production"),
                            (cw.LIN_SINK, "lin_sink")):
        out = np.empty(w * h * d)
        cw._lib.check(lib.cw_field_download(fh, hist, which_arr, cw._lib.ptr(out)))
        setattr(o, dest, out)
    held = np.empty(w * h * d, np.uint8)
    cw._lib.check(lib.cw_field_download_held(fh, hist, cw._lib.ptr(held)))
    o.held[:] = held
    return o


def field_error(o):
    """max |device - FP64 oracle| / max |oracle| after the oracle relaxes the
    device's field to residual 1e-12."""
    device = o.values.copy()
    rc, _ = o.relax(1e-12, 5_000_000, stop=1)
    assert rc == 0
    assert o.residual() < 1e-12
    return float(np.abs(device - o.values).max() / np.abs(o.values).max())


# ------------------------------------------------------------------ plain 2D
def test_plain_2d_fp64_oxygen_is_the_oracle_bit_for_bit(tmp_path):
    cfg = synthetic.plain_2d()
    sim, cfg, _ = sim_of(cfg, tmp_path)
    n = 256
    grid0 = sim.grid(0).reshape(-1)
    types = sim.lattice().cells()["type"]
    sink_by_type = np.array(cfg["o2_sink_by_type"])
    # step 0 solves from the field's start: 1 everywhere, row 0 held at 1
    o = O.Field(n, n, 1, cfg["o2_dcoef"], 0.0, 1.0)
    o.held[:n] = 1
    o.lin_sink = O.apply_uptake(grid0, types, sink_by_type)
    rc, sweeps = o.relax(cfg["tolerance"], 200_000, omega=cfg["omega"], stop=1)
    assert rc == 0 and sweeps > 100
    sim.step(1)
    np.testing.assert_array_equal(sim.field_values(0).view(np.uint64), o.values.view(np.uint64))
    # steps 1-9 do not solve; step 10 solves from there on the moved lattice
    sim.step(9)
    np.testing.assert_array_equal(sim.field_values(0).view(np.uint64), o.values.view(np.uint64))
    grid10 = sim.grid(0).reshape(-1)
    assert (grid10 != grid0).sum() > 500
    types = sim.lattice().cells()["type"]
    o.lin_sink = O.apply_uptake(grid10, types, sink_by_type)
    rc, sweeps = o.relax(cfg["tolerance"], 200_000, omega=cfg["omega"], stop=1)
    assert rc == 0
    sim.step(1)
    np.testing.assert_array_equal(sim.field_values(0).view(np.uint64), o.values.view(np.uint64))


def lattice_pair(grid, types, volume, target, lam, J, T, order, seed, surface=None):
    d, h, w = grid.shape
    n = len(types)
    o = O.Lattice(grid, (w, h, d), n, J, T, order)
    o.type[:], o.volume[:], o.target[:], o.lam[:] = types, volume, target, lam
    lat = cw.CpmLattice([(w, h, d)], T, [n], order, J)
    lat.upload(grid, 0)
    lat.set_cells(types, volume, target, lam, hist=0)
    lat.set_seed(seed, 0)
    if surface is not None:
        o.enable_surface(*surface)
        lat.set_surface(*surface)
    return o, lat


def records_of(sim, cfg):
    grid = sim.grid(0)
    used = int(grid.max()) + 1
    c = sim.lattice().cells()
    t, v = c["type"][:used], c["volume"][:used]
    tg = np.where(np.arange(used) > 0, cfg["target_volume"], 0).astype(np.int32)
    lam = np.where(np.arange(used) > 0, cfg["lambda_volume"], 0.0)
    return grid, used, t, v, tg, lam


def test_plain_2d_sweeps_are_the_oracle_bit_for_bit(tmp_path):
    sim, cfg, _ = sim_of(synthetic.plain_2d(), tmp_path)
    grid, used, t, v, tg, lam = records_of(sim, cfg)
    assert used == 121
    o, lat = lattice_pair(grid, t, v, tg, lam, cfg["J"], cfg["temperature"], cfg["contact_order"], 0xC0)
    o.mcs_checkerboard(0xC0, 0, 12)
    lat.monte_carlo_step(12)
    np.testing.assert_array_equal(lat.grid().reshape(-1), o.grid)
    np.testing.assert_array_equal(lat.cells()["volume"][1:], o.volume[1:])
    assert lat.records_match_grid()


# ------------------------------------------------------------------ campaign 1024^2
def test_campaign_1024_fields_are_within_1e6_of_the_fp64_oracle(tmp_path):
    sim, cfg, _ = sim_of(synthetic.campaign(per_size=1, sizes=(1024, 128)), tmp_path)
    sim.step(12)
    errs = {}
    for which, name, dc, decay in ((0, "oxygen", cfg["o2_dcoef"], 0.0),
                                   (1, "signal", cfg["signal_dcoef"], cfg["signal_decay"])):
        for hist in (0, 1):
            errs[(name, hist)] = field_error(field_problem(sim, which, hist, dc, decay))
    assert max(errs.values()) < FIELD_REL, errs
    assert sim.records_match_grid(0) and sim.records_match_grid(1)


def test_campaign_1024_sweeps_are_the_oracle_bit_for_bit(tmp_path):
    sim, cfg, _ = sim_of(synthetic.campaign(per_size=1, sizes=(1024,)), tmp_path)
    grid, used, t, v, tg, lam = records_of(sim, cfg)
    o, lat = lattice_pair(grid, t, v, tg, lam, cfg["J"], cfg["temperature"], cfg["contact_order"], 1000)
    o.mcs_checkerboard(1000, 0, 4)
    lat.monte_carlo_step(4)
    np.testing.assert_array_equal(lat.grid().reshape(-1), o.grid)
    np.testing.assert_array_equal(lat.cells()["volume"][1:], o.volume[1:])
    assert lat.records_match_grid()


# ------------------------------------------------------------------ the large cord
def test_cord_2048_fields_are_within_1e6_of_the_fp64_oracle(tmp_path):
    sim, cfg, _ = sim_of(synthetic.tumour_cord(), tmp_path)
    assert 39_000 < int((sim.lattice().cells()["volume"] > 0).sum()) < 41_000
    sim.step(6)
    errs = {}
    for which, name, dc, decay in ((0, "oxygen", cfg["o2_dcoef"], 0.0),
                                   (1, "signal", cfg["signal_dcoef"], cfg["signal_decay"])):
        errs[name] = field_error(field_problem(sim, which, 0, dc, decay))
    assert max(errs.values()) < FIELD_REL, errs
    assert sim.records_match_grid(0)


# ------------------------------------------------------------------ the 3D spheroid
def test_spheroid_256_field_is_within_1e6_of_the_fp64_oracle(tmp_path):
    sim, cfg, _ = sim_of(synthetic.spheroid_3d(), tmp_path)
    sim.step(3)
    err = field_error(field_problem(sim, 0, 0, cfg["o2_dcoef"], 0.0))
    assert err < FIELD_REL, err
    assert sim.records_match_grid(0)


def test_spheroid_256_sweeps_are_the_oracle_bit_for_bit(tmp_path):
    # 125-voxel cells, 26-neighbour contact (8 colours), surfaces: every pass
    # inside the round limit, and the grid, volumes and surfaces the oracle's
    sim, cfg, _ = sim_of(synthetic.spheroid_3d(), tmp_path)
    grid, used, t, v, tg, lam = records_of(sim, cfg)
    assert used > 2000
    ts = np.full(used, cfg["surface_target"], np.int32)
    ls = np.full(used, cfg["lambda_surface"])
    o, lat = lattice_pair(grid, t, v, tg, lam, cfg["J"], cfg["temperature"], cfg["contact_order"], 3,
                          surface=(ts, ls))
    o.mcs_checkerboard(3, 0, 3)
    lat.monte_carlo_step(3)
    np.testing.assert_array_equal(lat.grid().reshape(-1), o.grid)
    np.testing.assert_array_equal(lat.cells()["volume"][1:], o.volume[1:])
    np.testing.assert_array_equal(lat.surfaces()[1:used], o.surface[1:])
    assert lat.records_match_grid()
