"""The device field solve against the oracle (GPU).

FP64 mode must equal the oracle to the bit, values and sweep counts (the
reference's red-black SOR, pde.rs:245-405); the FP32 defect-correction mode
must reach its residual tolerance and sit within 1e-6 relative of the FP64
solution.
"""
import numpy as np
import pytest

import cellweave_b200 as cw
from oracle import oracle as O

pytestmark = pytest.mark.gpu

D = 0.2


def outside_disc(size, radius):
    c = float(size // 2)
    y, x = np.mgrid[0:size, 0:size]
    return (((x - c) ** 2 + (y - c) ** 2) > radius * radius).reshape(-1)


def disc_pair(size, radius, uptake):
    out = outside_disc(size, radius)
    up = np.where(out, 0.0, uptake)
    o = O.Field(size, size, 1, D, 0.0, 1.0)
    o.uptake[:] = up
    o.hold_bath(out, 1.0)
    g = cw.ScalarField.new(size, size, D, 0.0, 1.0)
    g.set_uptake_array(up)
    g.hold_bath(1.0, out)
    return o, g


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("size,radius,uptake,tol", [(30, 6, 0.004, 1e-11), (61, 20, 0.0005, 1e-11),
                                                    (32, 8, 0.003, 1e-9), (45, 11, 0.01, 1e-8)])
def test_fp64_relax_is_bit_exact(size, radius, uptake, tol):
    o, g = disc_pair(size, radius, uptake)
    np.testing.assert_array_equal(g.held(), o.held)
    np.testing.assert_array_equal(bits(g.values()), bits(o.values))
    rc, sweeps = o.relax(tol, 50_000)
    assert rc == 0
    assert g.relax(tol, 50_000) == sweeps
    np.testing.assert_array_equal(bits(g.values()), bits(o.values))


def test_fp64_volume_is_bit_exact():
    # the sphere of pde.rs:1202-1229
    side, r, u = 31, 10.0, 0.006
    z, y, x = np.mgrid[0:side, 0:side, 0:side]
    c = float(side // 2)
    inside = ((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2 <= r * r).reshape(-1)
    o = O.Field(side, side, side, D, 0.0, 1.0)
    o.uptake[inside] = u
    o.hold_bath(~inside, 1.0)
    g = cw.ScalarField.with_depth(side, side, side, D, 0.0, 1.0)
    g.set_uptake_array(np.where(inside, u, 0.0))
    g.hold_bath(1.0, ~inside)
    np.testing.assert_array_equal(g.held(), o.held)
    rc, sweeps = o.relax(1e-10, 1_000_000)
    assert g.relax(1e-10, 1_000_000) == sweeps
    np.testing.assert_array_equal(bits(g.values()), bits(o.values))
    centre = g.values()[(side // 2) * (side * side + side + 1)]
    assert abs(centre - (1 - u * r * r / (6 * D))) < 0.05


def sheet_problem(n, k=0.01, dcoef=1.0, seed=3):
    """C0's field: D lap c - k c 1[cell] = 0, c = 1 held on row 0, cells where a random mask says."""
    rng = np.random.default_rng(seed)
    cells = rng.random(n * n) < 0.6
    held = np.zeros(n * n, np.uint8)
    held[:n] = 1
    sink = np.where(cells, k, 0.0)
    return held, sink, dcoef


def test_fp64_residual_stop_with_a_first_order_sink_is_bit_exact():
    held, sink, dcoef = sheet_problem(48)
    o = O.Field(48, 48, 1, dcoef, 0.0, 0.0)
    o.lin_sink = sink.copy()
    o.held[:] = held
    o.values[held == 1] = 1.0
    rc, sweeps = o.relax(1e-10, 100_000, omega=1.85, stop=1)
    assert rc == 0
    g = cw.ScalarField.new(48, 48, dcoef, 0.0, 0.0)
    g.set_linear_sink(sink)
    g.hold_where(1.0, held)
    s = g.relax(1e-10, 100_000, omega=1.85, stop=cw.STOP_RESIDUAL)
    assert s == sweeps
    np.testing.assert_array_equal(bits(g.values()), bits(o.values))
    assert g.residual()[0] < 1e-10


@pytest.mark.parametrize("n,depth", [(64, 4), (300, 4), (257, 2), (200, 1)])
def test_fp32_defect_correction_reaches_the_fp64_solution(n, depth):
    held, sink, dcoef = sheet_problem(n)
    o = O.Field(n, n, 1, dcoef, 0.0, 0.0)
    o.lin_sink = sink.copy()
    o.held[:] = held
    o.values[held == 1] = 1.0
    assert o.relax(1e-12, 1_000_000, omega=1.9, stop=1)[0] == 0
    g = cw.ScalarField.new(n, n, dcoef, 0.0, 0.0)
    g.set_linear_sink(sink)
    g.hold_where(1.0, held)
    # the residual that buys 1e-6 of the field: the error is A^-1 r, and A's
    # smallest eigenvalue here is about the mean sink (0.006), so 1e-9 of
    # residual leaves under 2e-7 of error
    st = g.relax(1e-9, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, block_depth=depth,
                 stats=True)
    assert st[0]["residual"] < 1e-9
    v = g.values()
    # 1e-6 relative of the FP64 oracle, on the scale of the field (its maximum, 1)
    assert np.abs(v - o.values).max() < 1e-6 * np.abs(o.values).max()


def relaxed_from(values, held, sink, dcoef, n):
    """The oracle's FP64 solution to residual 1e-12, started from `values`
    (the unique fixed point: where SOR starts only shortens the CPU solve)."""
    o = O.Field(n, n, 1, dcoef, 0.0, 0.0)
    o.lin_sink = sink.copy()
    o.held[:] = held
    o.values[:] = values
    assert o.relax(1e-12, 5_000_000, omega=1.9, stop=1)[0] == 0
    return o.values


@pytest.mark.parametrize("n,k", [(512, 0.01), (512, 0.002), (1024, 0.001)])
def test_the_error_estimate_stop_leaves_the_field_within_its_bound(n, k):
    # a loose residual (1e-6) with an error bound of 1e-7 of the field's
    # scale: the solve runs on until the estimate from its last two
    # corrections is under the bound, and the field is within 1e-6 of the
    # FP64 oracle's wherever the residual alone would have stopped
    held, sink, dcoef = sheet_problem(n, k=k)
    g = cw.ScalarField.new(n, n, dcoef, 0.0, 0.0)
    g.set_linear_sink(sink)
    g.hold_where(1.0, held)
    loose = g.relax(1e-6, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, block_depth=8,
                    stats=True)[0]
    g2 = cw.ScalarField.new(n, n, dcoef, 0.0, 0.0)
    g2.set_linear_sink(sink)
    g2.hold_where(1.0, held)
    st = g2.relax(1e-6, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, block_depth=8,
                  error_tolerance=1e-7, stats=True)[0]
    assert st["residual"] < 1e-6 and st["sweeps"] >= loose["sweeps"]
    v = g2.values()
    exact = relaxed_from(v, held, sink, dcoef, n)
    assert np.abs(v - exact).max() < 1e-6 * np.abs(exact).max()
    # solved again from its own solution: two outer iterations give the ratio
    again = g2.relax(1e-6, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, block_depth=8,
                     error_tolerance=1e-7, stats=True)[0]
    assert again["sweeps"] <= st["sweeps"]
    assert np.abs(g2.values() - exact).max() < 1e-6 * np.abs(exact).max()


def test_the_error_tolerance_is_checked():
    g = cw.ScalarField.new(64, 64, 1.0, 0.0, 0.0)
    for bad in (-1e-7, float("inf"), float("nan")):
        with pytest.raises(cw.ConfigError):
            g.relax(1e-6, 1000, precision=cw.FP32_DC, stop=cw.STOP_RESIDUAL, error_tolerance=bad)


def test_fp32_defect_correction_on_a_volume():
    n = 40
    held = np.zeros((n, n, n), np.uint8)
    held[0], held[-1], held[:, 0], held[:, -1], held[:, :, 0], held[:, :, -1] = 1, 1, 1, 1, 1, 1
    sink = np.full(n ** 3, 0.005)
    g = cw.ScalarField.with_depth(n, n, n, 1.0, 0.0, 0.0)
    g.set_linear_sink(sink)
    g.hold_where(1.0, held.reshape(-1))
    st = g.relax(1e-9, 100_000, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, stats=True)
    assert st[0]["residual"] < 1e-9
    o = O.Field(n, n, n, 1.0, 0.0, 0.0)
    o.lin_sink = sink.copy()
    o.held[:] = held.reshape(-1)
    o.values[o.held == 1] = 1.0
    assert o.relax(1e-12, 100_000, stop=1)[0] == 0
    assert np.abs(g.values() - o.values).max() < 1e-6 * np.abs(o.values).max()


def test_not_settling_is_an_error():
    o, g = disc_pair(30, 6, 0.004)
    with pytest.raises(cw.SimulationError):
        g.relax(1e-9, 3)


def test_inflow_matches_the_oracle():
    o, g = disc_pair(30, 6, 0.004)
    o.relax(1e-11, 50_000)
    g.relax(1e-11, 50_000)
    assert abs(g.inflow() - o.inflow()) <= 1e-12 * abs(o.inflow())
    free = g.free_count()
    assert abs(g.inflow() - 0.004 * free) < 1e-6 * 0.004 * free


def test_explicit_step_is_bit_exact_and_refuses_what_the_reference_refuses():
    o = O.Field(20, 20, 1, 0.2, 0.05, 0.0)
    o.values.reshape(20, 20)[2:6, 2:6] = 1.0
    o.uptake[50:60] = 0.01
    g = cw.ScalarField.new(20, 20, 0.2, 0.05, 0.0)
    g.set_values(o.values)
    g.set_uptake_array(o.uptake)
    for _ in range(50):
        o.step(1.0)
        g.step(1.0)
    np.testing.assert_array_equal(bits(g.values()), bits(o.values))
    with pytest.raises(cw.ConfigError):
        cw.ScalarField.new(20, 20, 0.3, 0.0, 1.0).step(1.0)
    with pytest.raises(cw.ConfigError):
        cw.ScalarField.new(20, 20, 0.1, 2.0, 1.0).step(1.0)
    with pytest.raises(cw.ConfigError):
        g.step(0.0)


@pytest.mark.parametrize("wall", ["square", "gap", "diamond"])
def test_bath_matches_the_oracle(wall):
    y, x = np.mgrid[0:11, 0:11]
    dx, dy = x - 5, y - 5
    if wall == "square":
        w = np.maximum(abs(dx), abs(dy)) == 3
    elif wall == "gap":
        w = (np.maximum(abs(dx), abs(dy)) == 3) & ~((x == 5) & (y == 2))
    else:
        w = abs(dx) + abs(dy) == 3
    open_ = ~w.reshape(-1)
    o = O.Field(11, 11, 1, 0.2, 0.0, 0.0)
    o.hold_bath(open_, 1.0)
    g = cw.ScalarField.new(11, 11, 0.2, 0.0, 0.0)
    g.hold_bath(1.0, open_)
    np.testing.assert_array_equal(g.held(), o.held)
    np.testing.assert_array_equal(g.values(), o.values)


def test_bath_through_the_faces_of_a_volume_and_a_random_maze():
    col = np.arange(512) % 64 == 4 * 8 + 4
    g = cw.ScalarField.with_depth(8, 8, 8, 0.2, 0.0, 0.0)
    g.hold_bath(1.0, col)
    v = g.values()
    assert v[3 * 64 + 4 * 8 + 4] == 1.0 and v[3 * 64 + 4 * 8 + 3] == 0.0
    rng = np.random.default_rng(5)
    open_ = rng.random(150 * 120) < 0.62
    o = O.Field(150, 120, 1, 0.2, 0.0, 0.0)
    o.hold_bath(open_, 0.7)
    g = cw.ScalarField([(150, 120, 1)], 0.2, 0.0, 0.0)
    g.hold_bath(0.7, open_)
    np.testing.assert_array_equal(g.held(), o.held)


def test_a_batch_of_uneven_histories_solves_each_as_alone():
    cases = [(30, 6, 0.004), (45, 11, 0.002), (61, 20, 0.0005)]
    probs = [disc_pair(s, r, u) for s, r, u in cases]
    batch = cw.ScalarField([(s, s, 1) for s, _, _ in cases], D, 0.0, 1.0)
    for k, (s, r, u) in enumerate(cases):
        out = outside_disc(s, r)
        batch.set_uptake_array(np.where(out, 0.0, u), k)
        batch.hold_bath(1.0, out, k)
    counts = batch.relax(1e-11, 50_000)
    for k, (o, g) in enumerate(probs):
        rc, sweeps = o.relax(1e-11, 50_000)
        assert counts[k] == sweeps
        np.testing.assert_array_equal(bits(batch.values(k)), bits(o.values))


def inner_corrections(dims, depth, window=cw.WINDOW_AUTO, sweeps=5, seed=3):
    """cw_field_time_inner's FP32 correction for each history of a random
    batch (dims (w, h) for planes, (w, h, d) for volumes)."""
    import ctypes as C
    from cellweave_b200 import _lib
    rng = np.random.default_rng(seed)
    dims = [tuple(x) + (1,) * (3 - len(x)) for x in dims]
    f = cw.ScalarField(dims, D, 0.001, 0.0)
    for k, (w, h, d) in enumerate(dims):
        n = w * h * d
        f.set_values(rng.random(n), k)
        f.set_uptake_array(rng.random(n) * 0.01, k)
        f.hold_where(1.0, (rng.random(n) < 0.05).astype(np.uint8), k)
    ms, launches = C.c_float(), C.c_int64()
    L = _lib.lib()
    _lib.check(L.cw_field_time_inner(f.handle, sweeps, depth, window, 1.9, C.byref(ms), C.byref(launches)))
    out = []
    for k, (w, h, d) in enumerate(dims):
        a = np.empty(w * h * d, np.float32)
        _lib.check(L.cw_field_inner_correction(f.handle, k, a.ctypes.data))
        out.append(a)
    return out, launches.value


@pytest.mark.parametrize("dims", [
    [(70, 37, 9), (130, 40, 11), (33, 19, 6)],   # odd widths, a tile's halo across every axis
    [(96, 96, 96), (64, 200, 40)],               # several slice chunks
])
def test_blocked_volume_sweeps_equal_one_half_sweep_per_launch(dims):
    # the tiles marched along z are exact: two or four half-sweeps a launch,
    # tiles 32 or 16 rows high, give to the bit the in-place half-sweeps of
    # one per launch (5 sweeps: a depth-4 run ends on a launch of 2)
    ref, n1 = inner_corrections(dims, 1)
    assert n1 == 10
    assert all(np.abs(r).max() > 0 for r in ref)
    for window in (cw.WINDOW_AUTO, cw.WINDOW_64):
        for depth in (2, 4):
            got, launches = inner_corrections(dims, depth, window)
            assert launches == (10 + depth - 1) // depth
            for k in range(len(dims)):
                np.testing.assert_array_equal(got[k], ref[k], err_msg=f"window {window}, depth {depth}, {dims[k]}")


@pytest.mark.parametrize("dims", [
    [(128, 128), (200, 96), (260, 130), (1024, 70), (64, 300)],   # rows 16-byte aligned: TMA windows
    [(127, 90), (61, 61), (300, 33)],                               # any width: 64 x 64 windows
])
def test_blocked_fp32_sweeps_equal_one_half_sweep_per_launch(dims):
    # temporal blocking is exact: every depth gives, to the bit, the in-place
    # red-black sweeps of one half-sweep per launch (5 sweeps: 10 half-sweeps,
    # so a depth-8 run ends on a launch of 2)
    ref, n1 = inner_corrections(dims, 1)
    assert n1 == 10
    assert all(np.abs(r).max() > 0 for r in ref)
    for window in (cw.WINDOW_AUTO, cw.WINDOW_TALL, cw.WINDOW_64):
        for depth in (2, 4, 6, 8):
            got, _ = inner_corrections(dims, depth, window)
            for k in range(len(dims)):
                np.testing.assert_array_equal(got[k], ref[k], err_msg=f"window {window}, depth {depth}, {dims[k]}")


@pytest.mark.parametrize("sizes,depth", [([256], 8), ([128, 200, 512], 4), ([64, 1024], 6)])
def test_wide_windows_with_the_fused_correction_equal_the_64_windows(sizes, depth):
    # the 128 x 64 TMA windows add the correction in their last launch and take
    # the residual in one pass; the 64 x 64 windows write the correction and
    # update in two colour passes: the same arithmetic, so the same bits
    fields = []
    for window in (cw.WINDOW_AUTO, cw.WINDOW_64, cw.WINDOW_TALL):
        g = cw.ScalarField([(n, n, 1) for n in sizes], 1.0, 0.0, 0.0)
        for k, n in enumerate(sizes):
            held, sink, _ = sheet_problem(n, seed=k)
            g.set_linear_sink(sink, k)
            g.hold_where(1.0, held, k)
        st = g.relax(1e-6, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, block_depth=depth,
                     window=window, stats=True)
        fields.append((g, st))
    (ga, sa), *rest = fields
    for gb, sb in rest:
        for k in range(len(sizes)):
            assert sa[k]["sweeps"] == sb[k]["sweeps"]
            assert sa[k]["residual"] == sb[k]["residual"] < 1e-6
            np.testing.assert_array_equal(bits(ga.values(k)), bits(gb.values(k)))


# ---------------------------------------------------------------- the reference's field tests, on the device
# pde.rs:951-1200, each case run on the device and on the oracle: the same
# bits, and the reference's own assertions on the device's values


def test_a_field_decays_and_never_goes_negative_on_the_device():
    # pde.rs:951-977
    for (n, d, decay, dt, steps) in [(20, 0.25, 0.1, 0.1, 200), (30, 0.5, 2.0, 0.05, 500)]:
        o = O.Field(n, n, 1, d, decay, 1.0)
        g = cw.ScalarField.new(n, n, d, decay, 1.0)
        for _ in range(steps):
            o.step(dt)
            g.step(dt)
        v = g.values()
        np.testing.assert_array_equal(bits(v), bits(o.values))
        assert v.min() >= 0.0
        if n == 20:
            assert v[10 * 20 + 10] < 0.5


def test_a_held_pixel_does_not_move_and_a_cleared_uptake_refills_on_the_device():
    # pde.rs:1047-1081
    o, g = disc_pair(30, 6, 0.05)
    o.relax(1e-11, 50_000)
    g.relax(1e-11, 50_000)
    for _ in range(200):
        o.step(1.0)
        g.step(1.0)
    v = g.values()
    np.testing.assert_array_equal(bits(v), bits(o.values))
    assert v[0] == 1.0 and v[3 * 30 + 15] == 1.0 and v[15 * 30 + 15] < 0.5
    o, g = disc_pair(30, 6, 0.01)
    o.relax(1e-11, 50_000)
    g.relax(1e-11, 50_000)
    assert g.values()[15 * 30 + 15] < 0.9
    o.uptake[:] = 0.0
    g.clear_uptake()
    rc, sweeps = o.relax(1e-7, 50_000)
    assert g.relax(1e-7, 50_000) == sweeps
    v = g.values()
    np.testing.assert_array_equal(bits(v), bits(o.values))
    assert abs(v[15 * 30 + 15] - 1.0) < 1e-5


def test_a_held_vessel_supplies_from_the_inside_out_on_the_device():
    # pde.rs:1083-1113
    y, x = np.mgrid[0:60, 0:60]
    vessel = (((x - 30) ** 2 + (y - 30) ** 2) <= 9).reshape(-1)
    up = np.where(vessel, 0.0, 0.002)
    o = O.Field(60, 60, 1, D, 0.0, 0.0)
    o.uptake[:] = up
    o.held[vessel] = 1
    o.values[vessel] = 1.0
    g = cw.ScalarField.new(60, 60, D, 0.0, 0.0)
    g.set_uptake_array(up)
    g.hold_where(1.0, vessel)
    rc, sweeps = o.relax(1e-7, 50_000)
    assert rc == 0 and g.relax(1e-7, 50_000) == sweeps
    v = g.values()
    np.testing.assert_array_equal(bits(v), bits(o.values))
    at = lambda r: v[30 * 60 + 30 + r]
    assert at(0) == 1.0 and at(5) > at(10) > at(15) and v[61] < 0.01


def test_release_a_bath_and_a_vessel_and_the_box_swept_on_the_device():
    # pde.rs:1115-1200
    g = cw.ScalarField.new(20, 20, D, 0.0, 1.0)
    g.hold_bath(1.0, np.ones(400, bool))
    g.set_uptake_array(np.full(400, 0.01))
    g.step(1.0)
    assert g.values()[210] == 1.0
    g.release_all()
    g.step(1.0)
    assert g.values()[210] < 1.0

    y, x = np.mgrid[0:30, 0:30]
    tissue = ((x >= 5) & (x < 25) & (y >= 5) & (y < 25)).reshape(-1)
    g = cw.ScalarField.new(30, 30, D, 0.0, 0.0)
    g.hold_bath(1.0, ~tissue)
    g.hold_where(0.5, np.arange(900) == 15 * 30 + 15)
    v = g.values()
    assert v[0] == 1.0 and v[15 * 30 + 15] == 0.5 and v[10 * 30 + 10] == 0.0

    y, x = np.mgrid[0:40, 0:40]
    disc = (((x - 20) ** 2 + (y - 20) ** 2) <= 64).reshape(-1)
    up = np.where(disc, 0.001, 0.0)
    o = O.Field(40, 40, 1, D, 0.0, 1.0)
    o.uptake[:] = up
    o.hold_bath(~disc, 1.0)
    g = cw.ScalarField.new(40, 40, D, 0.0, 1.0)
    g.set_uptake_array(up)
    g.hold_bath(1.0, ~disc)
    rc, sweeps = o.relax(1e-9, 100_000)
    assert rc == 0 and g.relax(1e-9, 100_000) == sweeps
    v = g.values()
    np.testing.assert_array_equal(bits(v), bits(o.values))
    assert (v[~disc] == 1.0).all() and v[20 * 40 + 20] < 1.0
