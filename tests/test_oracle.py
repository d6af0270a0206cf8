"""The CPU oracle against the reference's own known answers (CPU only).

Each test restates one of the reference's tests (file:line given) on the
oracle, so that the oracle is pinned before it is trusted as the checker.
"""
import math

import numpy as np
import pytest

from cellweave_b200 import seeding
from oracle import oracle as O

# ---------------------------------------------------------------- RNG / exp


def test_philox_known_answers():
    # Random123's published known-answer vectors for philox4x32-10.
    ctr = np.array([[0, 0, 0, 0], [0xFFFFFFFF] * 4, [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344]], np.uint32)
    keys = [[0, 0], [0xFFFFFFFF, 0xFFFFFFFF], [0xA4093822, 0x299F31D0]]
    want = [[0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8], [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD],
            [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]]
    for c, k, w in zip(ctr, keys, want):
        assert [int(v) for v in O.philox(c, k)[0]] == w


def test_own_exp_is_within_two_ulp_of_libm():
    xs = np.concatenate([-np.logspace(-12, 2.8, 2000), np.linspace(-700, 0, 2001)])
    for x in xs:
        got, want = O.cw_exp(x), math.exp(x)
        assert abs(got - want) <= 2 * math.ulp(want), (x, got, want)
    assert O.cw_exp(0.0) == 1.0
    assert O.cw_exp(-800.0) == 0.0


# ---------------------------------------------------------------- RK4


def test_ras_erk_golden_table(golden):
    # network.rs:866-891: bit for bit in the reference, 1e-12 here.
    net = O.compile_network(golden["networks"]["ras-erk"], golden["ras_erk_reference_volume"])
    for row in golden["ras_erk_rk4"]:
        state = net.initial.copy().reshape(1, -1)
        inputs = np.array([[row["o2"], row["egf"], 0.0, 0.0, 0.0, 0.0]])
        O.network_step(net, state, inputs, 1.0, row["steps"])
        np.testing.assert_allclose(state[0], row["expected"], rtol=0, atol=1e-12, err_msg=row["source"])


def test_ras_erk_mechanics(golden):
    # network.rs:893-902 and 951-965.
    spec = golden["networks"]["ras-erk"]
    net = O.compile_network(spec, 200)
    state = net.initial.copy().reshape(1, -1)
    O.network_step(net, state, np.array([[0.8, 0.2, 0, 0, 0, 0]]), 1.0, 40)
    assert O.network_mechanics(net, state)[0] == golden["mechanics"]["free_target_after_40"]
    capped = dict(spec, mechanics=dict(spec["mechanics"], max_target=1.2))
    cnet = O.compile_network(capped, 200)
    assert O.network_mechanics(cnet, state)[0] == golden["mechanics"]["capped_target_after_40"]
    assert net.lambda_volume == golden["mechanics"]["lambda"]


def one_node(terms, initial=0.0):
    return {"nodes": [{"name": "a", "initial": initial, "terms": terms}],
            "roles": {"growth": "a", "survival": "a", "hypoxia_response": "a"},
            "mechanics": {"growth_coefficient": 1.0, "lambda_volume": 1.0}}


SLOPE_CASES = [  # network.rs:1071-1155: (term, self, input, documented slope)
    ({"kind": "activated_by", "source": "egf", "rate": 2.0}, 0.25, 0.5, 2.0 * 0.5 * 0.75),
    ({"kind": "inhibited_by", "source": "egf", "rate": 2.0}, 0.6, 0.5, -2.0 * 0.5 * 0.6),
    ({"kind": "activated_by_absence_of", "source": "oxygen", "rate": 1.0}, 0.2, 0.25, 1.0 * 0.75 * 0.8),
    ({"kind": "produced_by", "source": "egf", "rate": 2.0}, 0.9, 0.5, 2.0 * 0.5),
    ({"kind": "decays", "rate": 0.5}, 0.8, 0.0, -0.5 * 0.8),
    ({"kind": "relaxes_to", "value": 0.4, "rate": 2.0}, 0.1, 0.0, -2.0 * (0.1 - 0.4)),
    ({"kind": "damaged_below", "source": "oxygen", "threshold": 0.3, "rate": 3.0}, 0.5, 0.2, -3.0 * 0.1 / 0.3),
    ({"kind": "damaged_above", "source": "egf", "threshold": 0.4, "rate": 3.0}, 0.5, 0.6, -3.0 * 0.2 / 0.4),
]


@pytest.mark.parametrize("term,initial,inp,slope", SLOPE_CASES)
def test_each_term_does_what_its_name_says(term, initial, inp, slope):
    net = O.compile_network(one_node([term], initial), 100)
    st = net.initial.copy().reshape(1, -1)
    ins = np.zeros((1, 6))
    ins[0, 0 if term.get("source") == "oxygen" else 1] = inp
    dt = 1e-6
    O.network_step(net, st, ins, dt, 1)
    assert abs((st[0, 0] - initial) / dt - slope) < 1e-5


def test_hill_inhibition_is_half_at_k():
    # network.rs:1178-1218
    term = {"kind": "inhibited_by", "source": "egf", "rate": 1.0, "hill": {"n": 4.0, "k": 0.4}}
    net = O.compile_network(one_node([term], 0.5), 100)
    for egf, check in [(0.1, lambda s: abs(s) < 0.01), (0.4, lambda s: abs(s + 0.25) < 1e-5),
                       (1.6, lambda s: s < -0.49)]:
        st = net.initial.copy().reshape(1, -1)
        O.network_step(net, st, np.array([[0, egf, 0, 0, 0, 0]]), 1e-6, 1)
        assert check((st[0, 0] - 0.5) / 1e-6)


def _slope(term, initial, inputs, dt=1e-6):
    net = O.compile_network(one_node([term], initial), 100)
    st = net.initial.copy().reshape(1, -1)
    O.network_step(net, st, np.array([inputs], float), dt, 1)
    return (st[0, 0] - initial) / dt


def test_a_node_reads_the_waste_and_the_necrotic_factor_around_its_cell():
    # network.rs:1268-1316; inputs: oxygen, egf, crowding, stress, waste, necrotic factor
    waste = _slope({"kind": "activated_by", "source": "waste", "rate": 2.0}, 0.25, [1, 0, 0, 0, 0.5, 0])
    assert abs(waste - 2.0 * 0.5 * 0.75) < 1e-5
    above = {"kind": "damaged_above", "source": "necrotic_factor", "threshold": 0.5, "rate": 2.0}
    assert abs(_slope(above, 0.5, [1, 0, 0, 0, 0, 0.4])) < 1e-9
    assert abs(_slope(above, 0.5, [1, 0, 0, 0, 0, 1.0]) + 2.0) < 1e-5


def test_a_node_at_zero_cannot_be_damaged_below_zero():
    # network.rs:1327-1342
    net = O.compile_network(one_node([{"kind": "damaged_below", "source": "oxygen", "threshold": 0.5,
                                       "rate": 10.0}], 0.0), 100)
    st = net.initial.copy().reshape(1, -1)
    O.network_step(net, st, np.zeros((1, 6)), 1.0, 50)
    assert st[0, 0] == 0.0


def test_decay_pulls_a_node_down_and_a_hill_term_switches_more_sharply():
    # network.rs:1344-1377
    net = O.compile_network(one_node([{"kind": "decays", "rate": 1.0}], 1.0), 100)
    st = net.initial.copy().reshape(1, -1)
    O.network_step(net, st, np.zeros((1, 6)), 0.1, 1)
    assert 0.85 < st[0, 0] < 1.0

    def run(n, egf):
        term = {"kind": "activated_by", "source": "egf", "rate": 10.0, "hill": {"n": n, "k": 0.5}}
        net = O.compile_network(one_node([term]), 100)
        st = net.initial.copy().reshape(1, -1)
        O.network_step(net, st, np.array([[0, egf, 0, 0, 0, 0]], float), 0.1, 200)
        return st[0, 0]
    assert run(8.0, 0.3) < run(1.0, 0.3) and run(8.0, 0.7) > run(1.0, 0.7)


def test_a_crowded_cell_answers_with_its_differentiation_node(golden):
    # network.rs:1445-1482: k c (1 - a) = a settles at a = c / (1 + c)
    spec = one_node([{"kind": "activated_by", "source": "crowding", "rate": 1.0}, {"kind": "decays", "rate": 1.0}])
    spec["roles"] = dict(spec["roles"], differentiation="a")
    net = O.compile_network(spec, 100)
    st = net.initial.copy().reshape(1, -1)
    O.network_step(net, st, np.array([[1.0, 0, 0.6, 0, 0, 0]]), 1.0, 40)
    assert abs(st[0, net.optional["differentiation"]] - 0.6 / 1.6) < 1e-6
    spec["roles"]["differentiation"] = "nowhere"
    with pytest.raises(O.NetworkConfigError):
        O.compile_network(spec, 100)
    assert O.compile_network(golden["networks"]["ras-erk"], 100).optional["differentiation"] == -1


@pytest.mark.parametrize("spec,fragment", [
    (one_node([{"kind": "activated_by", "source": "p53", "rate": 1.0}]), "p53"),
    ({**one_node([]), "roles": {"growth": "a", "survival": "bcl2", "hypoxia_response": "a"}}, "bcl2"),
    ({**one_node([]), "nodes": []}, "node"),
    (one_node([{"kind": "activated_by", "source": "egf", "rate": 1.0, "hill": {"n": 0.0, "k": 0.5}}]), "Hill"),
    (one_node([{"kind": "damaged_above", "source": "egf", "threshold": 0.0, "rate": 1.0}]), "damaged"),
])
def test_compile_refusals(spec, fragment):
    # network.rs:967-1061, 1317-1325
    with pytest.raises(O.NetworkConfigError, match=fragment):
        O.compile_network(spec, 100)


# ---------------------------------------------------------------- reach / Delta-H


def test_reach_sizes(golden):
    r = golden["reach"]
    assert (len(O.reach(3, True)[0]), O.reach(3, True)[1]) == tuple(r["volume_order3"])
    assert (len(O.reach(2, True)[0]), O.reach(2, True)[1]) == tuple(r["volume_order2"])
    assert (len(O.reach(2, False)[0]), O.reach(2, False)[1]) == tuple(r["plane_order2"])
    assert (len(O.reach(3, False)[0]), O.reach(3, False)[1]) == tuple(r["plane_order3"])
    assert len(O.reach(1, False)[0]) == 0


# The reference's default ContactEnergy (cpm.rs:63-86) as a 5 x 5 table over
# Medium, Tumor, Normal, Necrotic, Immune.
REF_J = np.array([[0, 16, 16, 12, 12], [16, 2, 11, 10, 6], [16, 11, 6, 12, 11], [12, 10, 12, 8, 10],
                  [12, 6, 11, 10, 16]], float)


def block_cell(fw, fh):
    """cpm.rs:1208-1222: a tumour cell over a rectangle, lambda 0."""
    grid = np.zeros((1, 20, 20), np.int32)
    grid[0, :fh, :fw] = 1
    lat = O.Lattice(grid, (20, 20, 1), 2, REF_J, 10.0)
    lat.type[1] = 1
    lat.volume[1] = lat.target[1] = fw * fh
    return lat


def test_delta_h_closed_forms():
    # cpm.rs:1232-1258: a hole costs 4J, an isolated bump 2J, a corner slide 0.
    lat = block_cell(10, 20)
    site = lambda row, col: row * 20 + col
    assert lat.delta_h(site(10, 5), 0)[1] == 4 * 16.0
    assert lat.delta_h(site(10, 10), 1)[1] == 2 * 16.0
    corner = block_cell(10, 10)
    assert corner.delta_h(site(9, 9), 0)[1] == 0.0


def boundary_energy(grid, J, types, order, volume):
    """cpm.rs:1834-1866: the whole boundary energy, each pair counted once."""
    offs, across = O.reach(order, volume)
    if len(offs) == 0:
        offs = np.array([(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)])
        across = 1.0
    d, h, w = grid.shape
    kinds = np.where(grid < 0, 0, types[np.clip(grid, 0, None)])
    total = 0.0
    for dx, dy, dz in offs:
        a = grid[max(0, -dz):d - max(0, dz), max(0, -dy):h - max(0, dy), max(0, -dx):w - max(0, dx)]
        b = grid[max(0, dz):d - max(0, -dz) if dz < 0 else d, max(0, dy):h - max(0, -dy) if dy < 0 else h,
                 max(0, dx):w - max(0, -dx) if dx < 0 else w]
        ka = kinds[max(0, -dz):d - max(0, dz), max(0, -dy):h - max(0, dy), max(0, -dx):w - max(0, dx)]
        kb = kinds[max(0, dz):d - max(0, -dz) if dz < 0 else d, max(0, dy):h - max(0, -dy) if dy < 0 else h,
                   max(0, dx):w - max(0, -dx) if dx < 0 else w]
        total += np.where(a != b, J[ka, kb], 0.0).sum()
    return total / 2.0 / across


@pytest.mark.parametrize("order", [1, 2, 3])
def test_delta_h_is_the_change_of_boundary_energy(order):
    # cpm.rs:1912-1943, on a volume of three balls.
    grid = seeding.empty(14, 14, 14)
    rec = seeding.Records()
    seeding.add_ball(grid, rec, 1, (6, 7, 7), 3)
    seeding.add_ball(grid, rec, 1, (9, 7, 7), 3)
    seeding.add_ball(grid, rec, 3, (7, 9, 6), 2)
    types = np.array(rec.type, np.int32)
    lat = O.Lattice(grid, (14, 14, 14), len(rec), REF_J, 10.0, order=order)
    lat.type[:] = types
    rng = np.random.default_rng(11)
    flat = lat.grid
    for _ in range(150):
        i = int(rng.integers(flat.size))
        x, y, z = i % 14, (i // 14) % 14, i // 196
        nb = []
        if y > 0: nb.append(i - 14)
        if y < 13: nb.append(i + 14)
        if x > 0: nb.append(i - 1)
        if x < 13: nb.append(i + 1)
        if z > 0: nb.append(i - 196)
        if z < 13: nb.append(i + 196)
        j = nb[int(rng.integers(len(nb)))]
        src, dst = int(flat[i]), int(flat[j])
        before = boundary_energy(flat.reshape(14, 14, 14), REF_J, types, order, True)
        predicted = lat.delta_h(i, dst)[1]
        flat[i] = dst
        after = boundary_energy(flat.reshape(14, 14, 14), REF_J, types, order, True)
        flat[i] = src
        assert abs(after - before - predicted) < 1e-9


def test_volume_delta_h_formula():
    lat = block_cell(5, 5)
    lat.lam[1] = 3.0
    lat.target[1] = 30
    site = 2 * 20 + 5  # medium pixel next to the block
    out = lat.delta_h(site, 1)
    v, t = 25.0, 30.0
    assert out[2] == 3.0 * ((v + 1 - t) ** 2 - (v - t) ** 2)


# ---------------------------------------------------------------- CPM sweeps


def sheet(seed=0, size=64, ncell=12, side=7, types=2):
    grid = seeding.empty(size, size)
    rec = seeding.Records()
    rng = np.random.default_rng(seed)
    k = 0
    while len(rec) - 1 < ncell:
        x, y = rng.integers(0, size - side, 2)
        if (grid[0, y:y + side, x:x + side] != 0).any():
            continue
        seeding.add_block(grid, rec, 1 + (k % types), (x, y), side, side, lam=1.0)
        k += 1
    return grid, rec


def lattice_from(grid, rec, J, T, order=1):
    d, h, w = grid.shape
    lat = O.Lattice(grid, (w, h, d), len(rec), J, T, order)
    t, v, tg, lam = rec.arrays()
    lat.type[:], lat.volume[:], lat.target[:], lat.lam[:] = t, v, tg, lam
    return lat


J3 = np.array([[0, 16, 16], [16, 8, 12], [16, 12, 8]], float)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_checkerboard_keeps_the_books_and_the_sizes(order):
    grid, rec = sheet()
    lat = lattice_from(grid, rec, J3, 10.0, order)
    lat.mcs_checkerboard(seed=7, mcs0=0, sweeps=20)
    vol, _ = lat.counts()
    np.testing.assert_array_equal(vol[1:], lat.volume[1:])
    dev = np.abs(lat.volume[1:] - 49) / 49.0
    assert dev.max() < 0.35 and dev.mean() < 0.12


def test_checkerboard_is_deterministic():
    grid, rec = sheet()
    a = lattice_from(grid, rec, J3, 10.0, 2)
    b = lattice_from(grid, rec, J3, 10.0, 2)
    a.mcs_checkerboard(3, 0, 5)
    b.mcs_checkerboard(3, 0, 5)
    np.testing.assert_array_equal(a.grid, b.grid)
    c = lattice_from(grid, rec, J3, 10.0, 2)
    c.mcs_checkerboard(4, 0, 5)
    assert (a.grid != c.grid).any()


def test_colour_order_is_a_permutation():
    for ncol in (2, 4, 8, 9, 27):
        for mcs in range(5):
            p = O.colour_order(ncol, mcs, 12345)
            assert sorted(p.tolist()) == list(range(ncol))


def test_sequential_cell_grows_toward_a_raised_target():
    # cpm.rs:1281-1299
    grid = seeding.empty(120, 120)
    rec = seeding.Records()
    cid = seeding.add_cell(grid, rec, 1, (60, 60), 12)
    start = rec.volume[cid]
    lat = lattice_from(grid, rec, REF_J, 12.0)
    lat.target[cid] = 2 * start
    lat.lam[cid] = 20.0
    lat.mcs_sequential(7, 400)
    assert lat.volume[cid] > start + start // 4
    np.testing.assert_array_equal(lat.counts()[0][1:], lat.volume[1:])


def test_sequential_cell_aiming_at_nothing_shrinks_to_nothing():
    # cpm.rs:1438-1457
    grid = seeding.empty(50, 50)
    rec = seeding.Records()
    cid = seeding.add_cell(grid, rec, 3, (25, 25), 6)
    lat = lattice_from(grid, rec, REF_J, 10.0)
    lat.target[cid] = 0
    lat.mcs_sequential(5, 200)
    assert lat.volume[cid] == 0 and not (lat.grid == cid).any()


def test_obstacle_is_never_taken():
    # cpm.rs:1400-1423
    grid = seeding.empty(60, 60)
    rec = seeding.Records()
    seeding.add_obstacle_disc(grid, rec, (30, 30), 5)
    cid = seeding.add_cell(grid, rec, 1, (30, 30), 12)
    obst = grid.reshape(-1) == -1
    lat = lattice_from(grid, rec, REF_J, 30.0)
    lat.target[cid], lat.lam[cid] = 2000, 50.0
    lat.mcs_sequential(11, 100)
    assert (lat.grid[obst] == -1).all()
    lat.mcs_checkerboard(11, 0, 100)
    assert (lat.grid[obst] == -1).all()
    np.testing.assert_array_equal(lat.counts()[0][1:], lat.volume[1:])


def test_surface_books_follow_the_grid():
    grid, rec = sheet(size=48, ncell=8)
    lat = lattice_from(grid, rec, J3, 10.0, 2)
    lat.enable_surface(np.full(len(rec), 28, np.int32), np.full(len(rec), 0.2))
    lat.mcs_checkerboard(9, 0, 10)
    vol, surf = lat.counts()
    np.testing.assert_array_equal(vol[1:], lat.volume[1:])
    np.testing.assert_array_equal(surf[1:], lat.surface[1:])


# ---------------------------------------------------------------- SOR (pde.rs tests)

D = 0.2


def outside_disc(size, radius):
    c = float(size // 2)
    y, x = np.mgrid[0:size, 0:size]
    return ((x - c) ** 2 + (y - c) ** 2) > radius * radius


def bathed_disc(size, radius, uptake, threads=0):
    """pde.rs:762-775."""
    f = O.Field(size, size, 1, D, 0.0, 1.0)
    out = outside_disc(size, radius).reshape(-1)
    f.uptake[~out] = uptake
    f.hold_bath(out, 1.0)
    rc, _ = f.relax(1e-11, 50_000, threads=threads)
    assert rc == 0
    return f


def centre(f, size):
    return f.values[(size // 2) * size + size // 2]


def test_the_size_of_the_box_does_not_change_the_tissue():
    small, large = centre(bathed_disc(30, 6, 0.004), 30), centre(bathed_disc(60, 6, 0.004), 60)
    assert abs(small - large) < 1e-9
    assert 0.1 < small < 0.9


def test_a_bathed_disc_matches_the_textbook_profile():
    measured = centre(bathed_disc(32, 8, 0.003), 32)
    depth = 0.003 * 64 / (4 * D)
    assert abs(measured - (1 - depth)) / depth < 0.12


def test_the_number_of_threads_does_not_change_a_single_bit():
    a = bathed_disc(61, 20, 0.0005, threads=1).values
    for t in (3, 8):
        assert np.array_equal(a.view(np.uint64), bathed_disc(61, 20, 0.0005, threads=t).values.view(np.uint64))


def test_what_the_bath_hands_a_settled_tissue_is_what_it_takes_up():
    f = bathed_disc(30, 6, 0.004)
    free = int((f.held == 0).sum())
    assert free > 100
    assert abs(f.inflow() - 0.004 * free) < 1e-6 * 0.004 * free


def test_relaxing_a_settled_field_takes_one_sweep():
    f = bathed_disc(30, 6, 0.004)
    before = f.values.copy()
    rc, sweeps = f.relax(1e-11, 50_000)
    assert rc == 0 and sweeps == 1
    assert np.abs(f.values - before).max() < 1e-6


def test_relaxing_refuses_to_pretend():
    f = O.Field(30, 30, 1, D, 0.0, 1.0)
    out = outside_disc(30, 6).reshape(-1)
    f.uptake[~out] = 0.004
    f.hold_bath(out, 1.0)
    rc, _ = f.relax(1e-9, 3)
    assert rc == 2


def wall_field(wall):
    f = O.Field(11, 11, 1, 0.2, 0.0, 0.0)
    y, x = np.mgrid[0:11, 0:11]
    f.hold_bath(~wall(x - 5, y - 5, x, y).reshape(-1), 1.0)
    return f.values.reshape(11, 11)


def test_bath_pockets_gaps_and_corners():
    # pde.rs:832-880
    v = wall_field(lambda dx, dy, x, y: np.maximum(abs(dx), abs(dy)) == 3)
    assert v[5, 5] == 0.0 and v[0, 0] == 1.0
    v = wall_field(lambda dx, dy, x, y: (np.maximum(abs(dx), abs(dy)) == 3) & ~((x == 5) & (y == 2)))
    assert v[5, 5] == 1.0
    v = wall_field(lambda dx, dy, x, y: abs(dx) + abs(dy) == 3)
    assert v[5, 5] == 0.0 and v[0, 0] == 1.0


def test_a_bath_reaches_a_volume_through_its_six_faces():
    # pde.rs:1231-1248
    col = np.arange(512) % 64 == 4 * 8 + 4
    f = O.Field(8, 8, 8, D, 0.0, 0.0)
    f.hold_bath(col, 1.0)
    assert f.values[3 * 64 + 4 * 8 + 4] == 1.0 and f.values[3 * 64 + 4 * 8 + 3] == 0.0
    g = O.Field(8, 8, 1, D, 0.0, 0.0)
    g.hold_bath(col[:64], 1.0)
    assert g.values[4 * 8 + 4] == 0.0


def test_a_starving_ball_settles_where_the_sphere_formula_puts_it():
    # pde.rs:1202-1229
    side, r, u = 31, 10.0, 0.006
    f = O.Field(side, side, side, D, 0.0, 1.0)
    z, y, x = np.mgrid[0:side, 0:side, 0:side]
    c = float(side // 2)
    inside = ((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2 <= r * r).reshape(-1)
    f.uptake[inside] = u
    f.hold_bath(~inside, 1.0)
    rc, _ = f.relax(1e-10, 1_000_000)
    assert rc == 0
    got = f.values[(side // 2) * (side * side + side + 1)]
    assert abs(got - (1 - u * r * r / (6 * D))) < 0.05


def test_a_sweep_is_held_to_the_box_around_what_is_free():
    # pde.rs:1158-1175
    f = O.Field(20, 20, 1, D, 0.0, 0.0)
    y, x = np.mgrid[0:20, 0:20]
    tissue = ((x >= 4) & (x < 9) & (y >= 11) & (y < 14)).reshape(-1)
    f.hold_bath(~tissue, 1.0)
    assert f.free_span() == (4, 8, 11, 13, 0, 0)
    f.held[:] = 1
    assert f.free_span() is None
    assert f.relax(1e-9, 10) == (0, 1)


def test_explicit_step_conserves_and_refuses():
    # pde.rs:882-949
    f = O.Field(20, 20, 1, 0.2, 0.0, 0.0)
    f.values.reshape(20, 20)[2:6, 2:6] = 1.0
    before = f.values.sum()
    for _ in range(500):
        assert f.step(1.0) == 0
    assert abs(f.values.sum() - before) < 1e-9
    assert O.Field(20, 20, 1, 0.3, 0.0, 1.0).step(1.0) == 1
    assert O.Field(20, 20, 1, 0.1, 2.0, 1.0).step(1.0) == 1
    assert O.Field(20, 20, 1, 0.1, 0.0, 1.0).step(0.0) == 1


def test_a_field_decays_and_never_goes_negative():
    # pde.rs:951-977
    f = O.Field(20, 20, 1, 0.25, 0.1, 1.0)
    for _ in range(200):
        assert f.step(0.1) == 0
    assert f.values[10 * 20 + 10] < 0.5
    g = O.Field(30, 30, 1, 0.5, 2.0, 1.0)
    for _ in range(500):
        assert g.step(0.05) == 0
    assert g.values.min() >= 0.0


def test_a_held_pixel_is_a_boundary_condition_and_does_not_move():
    # pde.rs:1047-1066
    f = bathed_disc(30, 6, 0.05)
    for _ in range(200):
        assert f.step(1.0) == 0
    v = f.values.reshape(30, 30)
    assert v[0, 0] == 1.0 and v[3, 15] == 1.0 and v[15, 15] < 0.5


def test_clearing_the_uptake_lets_the_field_refill():
    # pde.rs:1069-1081
    f = bathed_disc(30, 6, 0.01)
    assert centre(f, 30) < 0.9
    f.uptake[:] = 0.0
    assert f.relax(1e-7, 50_000)[0] == 0
    assert abs(centre(f, 30) - 1.0) < 1e-5


def vessel_disc(size=60, r2=9):
    y, x = np.mgrid[0:size, 0:size]
    return (((x - size // 2) ** 2 + (y - size // 2) ** 2) <= r2).reshape(-1)


def test_a_held_vessel_supplies_from_the_inside_out():
    # pde.rs:1083-1113
    f = O.Field(60, 60, 1, D, 0.0, 0.0)
    vessel = vessel_disc()
    f.uptake[~vessel] = 0.002
    f.held[vessel] = 1
    f.values[vessel] = 1.0
    assert f.relax(1e-7, 50_000)[0] == 0
    at = lambda r: f.values[30 * 60 + 30 + r]
    assert at(0) == 1.0 and at(5) > at(10) > at(15)
    assert f.values[1 * 60 + 1] < 0.01


def test_releasing_lets_a_former_bath_pixel_move_again():
    # pde.rs:1115-1138
    f = O.Field(20, 20, 1, D, 0.0, 1.0)
    f.hold_bath(np.ones(400, bool), 1.0)
    f.uptake[:] = 0.01
    assert f.step(1.0) == 0
    assert f.values[10 * 20 + 10] == 1.0
    f.held[:] = 0
    assert f.step(1.0) == 0
    assert f.values[10 * 20 + 10] < 1.0


def test_a_bath_and_a_vessel_can_hold_at_once():
    # pde.rs:1140-1156
    f = O.Field(30, 30, 1, D, 0.0, 0.0)
    y, x = np.mgrid[0:30, 0:30]
    tissue = ((x >= 5) & (x < 25) & (y >= 5) & (y < 25)).reshape(-1)
    f.hold_bath(~tissue, 1.0)
    f.held[15 * 30 + 15] = 1
    f.values[15 * 30 + 15] = 0.5
    assert f.values[0] == 1.0 and f.values[15 * 30 + 15] == 0.5 and f.values[10 * 30 + 10] == 0.0


def test_the_box_swept_leaves_what_lies_outside_it_as_it_was_held():
    # pde.rs:1177-1200
    f = O.Field(40, 40, 1, D, 0.0, 1.0)
    disc = vessel_disc(40, 64)
    f.uptake[disc] = 0.001
    f.hold_bath(~disc, 1.0)
    assert f.relax(1e-9, 100_000)[0] == 0
    assert (f.values[~disc] == 1.0).all() and f.values[20 * 40 + 20] < 1.0


def test_residual_stop_reaches_its_tolerance():
    f = O.Field(40, 40, 1, 1.0, 0.0, 0.0)
    f.lin_sink = np.full(1600, 0.01)
    f.held.reshape(40, 40)[0, :] = 1
    f.values.reshape(40, 40)[0, :] = 1.0
    rc, sweeps = f.relax(1e-10, 100_000, omega=1.85, stop=1)
    assert rc == 0 and f.residual() < 1e-10 and sweeps > 10


# ---------------------------------------------------------------- coupling


def cluster():
    """coupling.rs:211-224: one cell ringed by eight."""
    grid = seeding.empty(80, 80)
    rec = seeding.Records()
    c = seeding.add_cell(grid, rec, 1, (40, 40), 6)
    ring = []
    for k in range(8):
        a = k * math.tau / 8
        ring.append(seeding.add_cell(grid, rec, 1, (round(40 + 13 * math.cos(a)), round(40 + 13 * math.sin(a))), 6))
    return grid, rec, c, ring


def test_a_cell_in_the_middle_reads_less_oxygen_than_one_on_the_rim():
    grid, rec, c, ring = cluster()
    f = O.Field(80, 80, 1, 0.2, 0.0, 1.0)
    f.uptake[:] = O.apply_uptake(grid, np.array(rec.type, np.int32), np.array([0.0, 0.003]))
    f.hold_bath(grid.reshape(-1) == 0, 1.0)
    assert f.relax(1e-7, 50_000)[0] == 0
    o2 = O.mean_per_cell(grid, f.values, len(rec))
    inner, outer = o2[c], max(o2[r] for r in ring)
    assert inner < outer and inner < 0.9 and outer > inner + 0.05
    assert o2[0] == 0.0 and (o2[1:] > 0).all()


def test_a_vessel_delivers_what_its_share_says_and_a_dry_one_nothing():
    # coupling.rs:300-315: three vessel pixels on a 10 x 1 strip, shares 0, 1/2, 3 of 2
    grid = np.zeros((1, 10), np.int32)
    grid[0, :3] = -1
    held, values = np.zeros(10, np.uint8), np.zeros(10)
    O.hold_vessels_by(grid, 2.0, [0.0, 0.5, 3.0] + [0.0] * 7, held, values)
    assert values[0] == 0.0 and not held[0], "a dry vessel is not held"
    assert values[1] == 1.0 and held[1], "half of 2"
    assert values[2] == 2.0 and held[2], "never more than in full"
    assert not held[3:].any()


def test_a_vessel_poorer_than_the_tissue_around_it_takes_nothing_from_it():
    # coupling.rs:317-331
    grid = np.zeros((1, 10), np.int32)
    grid[0, 5] = -1
    held, values = np.zeros(10, np.uint8), np.full(10, 0.9)
    O.hold_vessels_by(grid, 1.0, np.full(10, 0.5), held, values)
    assert values[5] == 0.9 and not held[5], "left free, not held down to half"
    O.hold_vessels_by(grid, 1.0, np.full(10, 1.0), held, values)
    assert values[5] == 1.0 and held[5], "held where it is richer"


def test_moore_copies_need_period_two_with_face_contact():
    # with copies from diagonal neighbours a chessboard colour would hold a
    # copy's source: face contact then takes period 2 (4 colours, 8 in a volume)
    grid = np.zeros((1, 12, 12), np.int32)
    lat = O.Lattice(grid, (12, 12, 1), 1, np.zeros((1, 1)), 10.0, 1)
    assert lat.colouring() == (2, 0)
    lat.copy_moore = True
    assert lat.colouring() == (4, 2)
    vol = O.Lattice(np.zeros((6, 6, 6), np.int32), (6, 6, 6), 1, np.zeros((1, 1)), 10.0, 1)
    vol.copy_moore = True
    assert vol.colouring() == (8, 2)
    vol.order = 3  # the 26-neighbourhood: Chebyshev radius 1, period 2 either way
    assert vol.colouring() == (8, 2)


def _disc_lattice(size, centre, radius, lam=1.0, capacity=8):
    from cellweave_b200 import seeding
    grid = seeding.empty(size, size)
    rec = seeding.Records()
    seeding.add_cell(grid, rec, 1, centre, radius, lam=lam)
    lat = O.Lattice(grid, (size, size, 1), capacity, np.zeros((2, 2)), 10.0, 1)
    t, v, tg, lm = rec.arrays()
    lat.type[:len(rec)], lat.volume[:len(rec)], lat.target[:len(rec)], lat.lam[:len(rec)] = t, v, tg, lm
    return lat, len(rec)


def test_division_hands_every_pixel_to_exactly_one_of_the_two():
    # cpm.rs:1302-1316 and 1319-1332
    lat, used = _disc_lattice(60, (30, 30), 10)
    before = int(lat.volume[1])
    lat.target[1], lat.lam[1] = 500, 33.0
    d, used = lat.divide_across(1, (math.cos(0.3), math.sin(0.3)), used)
    assert d == 2 and used == 3
    p, q = int(lat.volume[1]), int(lat.volume[2])
    assert p + q == before and p > 0 and q > 0
    assert abs(p - q) < before / 5
    assert lat.type[2] == lat.type[1] and lat.target[2] == 500 and lat.lam[2] == 33.0
    vol, _ = lat.counts()
    np.testing.assert_array_equal(vol[1:3], lat.volume[1:3])


def test_a_plane_through_a_ball_halves_it_on_the_side_it_faces():
    # cpm.rs:1645-1673: radius 5 at the centre of a 30^3 box, cut by the +z plane
    grid = seeding.empty(30, 30, 30)
    rec = seeding.Records()
    seeding.add_ball(grid, rec, 1, (15, 15, 15), 5, lam=2.0)
    lat = O.Lattice(grid, (30, 30, 30), 3, REF_J, 10.0)
    t, v, tg, lam = rec.arrays()
    lat.type[:2], lat.volume[:2], lat.target[:2], lat.lam[:2] = t, v, tg, lam
    assert lat.divide_across(1, (0.0, 0.0, 1.0), 2) == (2, 3)
    a, b = int(lat.volume[1]), int(lat.volume[2])
    assert a + b == int((grid == 1).sum()) and a > b and 2 * b > a
    assert np.nonzero(lat.grid.reshape(30, 30, 30) == 2)[0].min() > 15


def test_what_cannot_be_divided_is_left_alone():
    # cpm.rs:1335-1379: a cell under 8 pixels, the medium, an unknown id, and a
    # cut that leaves one side empty change nothing
    lat, used = _disc_lattice(30, (15, 15), 1)
    grid = lat.grid.copy()
    assert lat.divide_across(1, (math.cos(0.5), math.sin(0.5)), used) == (-1, used)
    assert lat.divide_across(0, (1.0, 0.0), used) == (-1, used)
    assert lat.divide_across(42, (1.0, 0.0), used) == (-1, used)
    np.testing.assert_array_equal(lat.grid, grid)
    bar = np.zeros((1, 20, 20), np.int32)
    bar[0, 5:15, 10] = 1
    lat = O.Lattice(bar, (20, 20, 1), 4, np.zeros((2, 2)), 10.0, 1)
    lat.type[1], lat.volume[1], lat.target[1], lat.lam[1] = 1, 10, 10, 1.0
    assert lat.divide_across(1, (1.0, 0.0), 2) == (-1, 2)
    np.testing.assert_array_equal(lat.grid, bar.reshape(-1))


def test_the_fit_oracles_direct_solve_is_the_fixed_point_of_relax():
    # the differentiated fit's CPU loss solves its fields directly; that is the
    # field pde.rs's relax converges to (held pixels, first-order sink, decay,
    # production and uptake, in the plane and in a volume)
    from oracle.fit import solve_direct
    rng = np.random.default_rng(11)
    for w, h, d in ((40, 32, 1), (12, 10, 8)):
        n = w * h * d
        a = O.Field(w, h, d, 0.7, 0.01, 0.5)
        held = (rng.random(n) < 0.05).astype(np.uint8)
        held[:w] = 1
        a.held[:] = held
        a.values[held == 1] = rng.uniform(0.5, 1.5, int(held.sum()))
        a.lin_sink = np.where(rng.random(n) < 0.6, 0.02, 0.0)
        a.production[:] = np.where(rng.random(n) < 0.3, 0.01, 0.0)
        a.uptake[:] = np.where(rng.random(n) < 0.2, 0.001, 0.0)
        b = O.Field(w, h, d, 0.7, 0.01, 0.5)
        b.held[:], b.values[:], b.lin_sink = a.held, a.values, a.lin_sink.copy()
        b.production[:], b.uptake[:] = a.production, a.uptake
        assert a.relax(1e-13, 1_000_000, stop=1)[0] == 0
        solve_direct(b)
        np.testing.assert_allclose(b.values, a.values, rtol=0, atol=1e-10)


# ---------------------------------------------------------------- the fuller cell
# crates/io/tests/fuller_cell.rs: the fuller cell against the networks it fills
# in (the same decisions at the same places), on the oracle's compile and RK4


def _settled(golden, name, o2, stress, edit=None):
    import copy
    spec = copy.deepcopy(golden["networks"][name])
    if edit:
        edit(spec)
    net = O.compile_network(spec, 100)
    st = net.initial.reshape(1, -1).copy()
    ins = np.array([[o2, 0.2, 0.0, stress, 0.0, 0.0]])
    O.network_step(net, st, ins, 1.0, 600)  # 600 steps of one unit (fuller_cell.rs:42-48)
    return net, st[0]


def _level(net, st, name):
    return st[net.names.index(name)]


def _arrest_oxygen(golden, name):
    lo, hi = 0.0, 1.0
    for _ in range(30):
        mid = 0.5 * (lo + hi)
        net, st = _settled(golden, name, mid, 0.0)
        if st[net.hypoxia] >= 0.45:  # QUIESCENCE_THRESHOLD
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def test_the_fuller_cell_asks_for_the_size_the_simpler_one_does(golden):
    # fuller_cell.rs:69-80
    a, sa = _settled(golden, "fuller-cell", 1.0, 0.0)
    b, sb = _settled(golden, "ras-erk", 1.0, 0.0)
    assert abs(_level(a, sa, "erk") - _level(b, sb, "erk")) < 0.002
    ta = O.network_mechanics(a, sa.reshape(1, -1))[0]
    tb = O.network_mechanics(b, sb.reshape(1, -1))[0]
    assert abs(int(ta) - int(tb)) <= 1


def test_the_fuller_cell_stops_dividing_at_the_oxygen_the_simpler_one_does(golden):
    # fuller_cell.rs:82-97
    assert abs(_arrest_oxygen(golden, "fuller-cell") - _arrest_oxygen(golden, "ras-erk")) < 0.005
    fed, sf = _settled(golden, "fuller-cell", 1.0, 0.0)
    assert _level(fed, sf, "rb") < 0.3 and _level(fed, sf, "p27") < 0.01
    starved, ss = _settled(golden, "fuller-cell", 0.1, 0.0)
    assert _level(starved, ss, "p27") > 0.5
    assert _level(starved, ss, "cyclin_e") < _level(fed, sf, "cyclin_e") / 2.0


def test_the_fuller_cell_dies_of_anoxia_where_the_simpler_one_does(golden):
    # fuller_cell.rs:99-110
    for o2 in (0.02, 0.05, 0.1, 0.2, 0.6):
        a, sa = _settled(golden, "fuller-cell", o2, 0.0)
        b, sb = _settled(golden, "ras-erk", o2, 0.0)
        assert abs(sa[a.survival] - sb[b.survival]) < 0.002, o2


def test_the_fuller_cell_answers_a_stress_as_the_stress_response_did(golden):
    # fuller_cell.rs:112-136
    for stress in (0.0, 0.2, 0.5, 1.0):
        a, sa = _settled(golden, "fuller-cell", 1.0, stress)
        b, sb = _settled(golden, "stress-response", 1.0, stress)
        assert abs(sa[a.optional["apoptosis"]] - sb[b.optional["apoptosis"]]) < 0.015, stress
    calm, sc = _settled(golden, "fuller-cell", 1.0, 0.0)
    for name in ("p53", "mdm2", "p21", "bax", "caspase"):
        assert _level(calm, sc, name) == 0.0, name
    a, sa = _settled(golden, "fuller-cell", 1.0, 1.0)
    b, sb = _settled(golden, "stress-response", 1.0, 1.0)
    assert _level(a, sa, "p53") < _level(b, sb, "p53")


def test_a_fuller_cell_starts_where_it_settles(golden):
    # fuller_cell.rs:173-191
    spec = golden["networks"]["fuller-cell"]
    net, st = _settled(golden, "fuller-cell", 1.0, 0.0)
    for node, value in zip(spec["nodes"], st):
        if node["name"] in ("hif1", "vegf", "bcl2"):
            continue
        assert abs(node["initial"] - value) < 0.01, node["name"]
