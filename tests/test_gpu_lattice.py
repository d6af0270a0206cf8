"""The device CPM against the oracle (GPU).

Delta-H of identical proposals is bit-exact (cpm.rs:841-894); the sublattice
sweep the device runs is bit-exact against its CPU restatement in the oracle
(same Philox draws, same colour order, same snapshots); the bookkeeping
invariant records_match_grid (cpm.rs:1272-1279) holds after every sweep.
"""
import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import seeding
from oracle import oracle as O

pytestmark = pytest.mark.gpu

J3 = np.array([[0, 16, 16], [16, 8, 12], [16, 12, 8]], float)
REF_J = np.array([[0, 16, 16, 12, 12], [16, 2, 11, 10, 6], [16, 11, 6, 12, 11], [12, 10, 12, 8, 10],
                  [12, 6, 11, 10, 16]], float)


def sheet(seed=0, size=64, ncell=12, side=7, types=2, lam=1.0):
    grid = seeding.empty(size, size)
    rec = seeding.Records()
    rng = np.random.default_rng(seed)
    k = 0
    while len(rec) - 1 < ncell:
        x, y = rng.integers(0, size - side, 2)
        if (grid[0, y:y + side, x:x + side] != 0).any():
            continue
        seeding.add_block(grid, rec, 1 + (k % types), (x, y), side, side, lam=lam)
        k += 1
    return grid, rec


def ball_volume(size=20):
    grid = seeding.empty(size, size, size)
    rec = seeding.Records()
    c = size // 2
    seeding.add_ball(grid, rec, 1, (c - 3, c, c), 3, lam=2.0)
    seeding.add_ball(grid, rec, 1, (c + 3, c, c), 3, lam=2.0)
    seeding.add_ball(grid, rec, 2, (c, c + 3, c - 1), 2, lam=2.0)
    # add_ball takes voxels from earlier cells without updating their records
    # (cpm.rs:323-354); recount so that the books start true
    rec.volume = list(seeding.recount(grid, len(rec)))
    rec.volume[0] = 0
    return grid, rec


def oracle_of(grid, rec, J, T, order):
    d, h, w = grid.shape
    lat = O.Lattice(grid, (w, h, d), len(rec), J, T, order)
    t, v, tg, lam = rec.arrays()
    lat.type[:], lat.volume[:], lat.target[:], lat.lam[:] = t, v, tg, lam
    return lat


def pair(grid, rec, J, T, order, seed, surface=None):
    o = oracle_of(grid, rec, J, T, order)
    g = cw.CpmLattice.from_grids([grid], [rec], T, J, order, seeds=[seed])
    if surface is not None:
        ts, ls = surface
        o.enable_surface(ts, ls)
        g.set_surface(ts, ls)
    return o, g


def proposals(o, n, rng):
    w, h, d = o.w, o.h, o.d
    sites, dsts = [], []
    for _ in range(n):
        i = int(rng.integers(o.grid.size))
        x, y, z = i % w, (i // w) % h, i // (w * h)
        nb = []
        if y > 0: nb.append(i - w)
        if y + 1 < h: nb.append(i + w)
        if x > 0: nb.append(i - 1)
        if x + 1 < w: nb.append(i + 1)
        if z > 0: nb.append(i - w * h)
        if z + 1 < d: nb.append(i + w * h)
        sites.append(i)
        dsts.append(int(o.grid[nb[int(rng.integers(len(nb)))]]))
    return np.array(sites), np.array(dsts)


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("volume", [False, True])
def test_delta_h_is_bit_exact(order, volume):
    grid, rec = ball_volume() if volume else sheet(seed=order)
    # non-integral energies and lambdas, so rounding order matters
    J = REF_J[:3, :3] * 1.37 if not volume else J3 * 0.91
    o, g = pair(grid, rec, J, 10.0, order, 1, surface=(np.full(len(rec), 40, np.int32), np.full(len(rec), 0.3)))
    o.lam[1:] = 1.7
    g.set_cells(lam=o.lam)
    rng = np.random.default_rng(7 + order)
    sites, dsts = proposals(o, 500, rng)
    got = g.delta_h(sites, dsts)
    want = np.array([o.delta_h(s, dd) for s, dd in zip(sites, dsts)])
    np.testing.assert_array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("order,subsweeps", [(1, 1), (2, 1), (3, 1), (2, 4), (1, 3)])
def test_sweeps_are_bit_exact_with_the_sublattice_oracle_plane(order, subsweeps):
    grid, rec = sheet(seed=order, size=64, ncell=20)
    o, g = pair(grid, rec, J3, 10.0, order, 0xC0FFEE12345)
    g.set_subsweeps(subsweeps)
    o.mcs_checkerboard(0xC0FFEE12345, 0, 25, subsweeps=subsweeps)
    g.monte_carlo_step(25)
    np.testing.assert_array_equal(g.grid().reshape(-1), o.grid)
    np.testing.assert_array_equal(g.cells()["volume"], o.volume)
    assert g.records_match_grid()


@pytest.mark.parametrize("order,subsweeps", [(1, 1), (3, 1), (3, 2)])
def test_sweeps_are_bit_exact_in_a_volume_with_surfaces(order, subsweeps):
    grid, rec = ball_volume(18)
    n = len(rec)
    o, g = pair(grid, rec, J3, 20.0, order, 99, surface=(np.full(n, 60, np.int32), np.full(n, 0.2)))
    g.set_subsweeps(subsweeps)
    o.mcs_checkerboard(99, 0, 12, subsweeps=subsweeps)
    g.monte_carlo_step(12)
    np.testing.assert_array_equal(g.grid().reshape(-1), o.grid)
    # the medium's count (index 0) is untracked by the device, as by the reference
    np.testing.assert_array_equal(g.cells()["volume"][1:], o.volume[1:])
    np.testing.assert_array_equal(g.surfaces(), o.surface)
    assert g.records_match_grid()


@pytest.mark.parametrize("order,volume", [(1, False), (2, False), (3, True)])
def test_moore_copies_are_bit_exact_with_the_oracle(order, volume):
    # copies from any Chebyshev neighbour (an extension; the reference copies
    # across faces): face contact then needs period 2, not the chessboard
    if volume:
        grid, rec = ball_volume(18)
        n = len(rec)
        o, g = pair(grid, rec, J3, 20.0, order, 5, surface=(np.full(n, 60, np.int32), np.full(n, 0.2)))
    else:
        grid, rec = sheet(seed=order + 10, size=64, ncell=20)
        o, g = pair(grid, rec, J3, 10.0, order, 0xBEEF)
    o.copy_moore = True
    g.set_copy_neighbourhood(True)
    assert o.colouring() == ((8 if volume else 4), 2) or order > 1
    seed = 5 if volume else 0xBEEF
    o.mcs_checkerboard(seed, 0, 12)
    g.monte_carlo_step(12)
    np.testing.assert_array_equal(g.grid().reshape(-1), o.grid)
    np.testing.assert_array_equal(g.cells()["volume"][1:], o.volume[1:])
    if volume:
        np.testing.assert_array_equal(g.surfaces(), o.surface)
    assert g.records_match_grid()


def test_a_batch_of_uneven_lattices_sweeps_each_as_alone():
    scenes = [sheet(seed=s, size=sz, ncell=nc) for s, sz, nc in [(1, 40, 6), (2, 64, 20), (3, 96, 30)]]
    seeds = [11, 22, 33]
    batch = cw.CpmLattice.from_grids([g for g, _ in scenes], [r for _, r in scenes], 10.0, J3, 2, seeds=seeds)
    batch.monte_carlo_step(10)
    for k, ((grid, rec), seed) in enumerate(zip(scenes, seeds)):
        o = oracle_of(grid, rec, J3, 10.0, 2)
        o.mcs_checkerboard(seed, 0, 10)
        np.testing.assert_array_equal(batch.grid(k).reshape(-1), o.grid)
        assert batch.records_match_grid(k)


def test_obstacles_hold_and_sizes_stay_near_target():
    grid, rec = sheet(seed=4, size=80, ncell=30)
    seeding.add_obstacle_disc(grid, rec, (40, 40), 5)
    obst = grid.reshape(-1) == -1
    g = cw.CpmLattice.from_grids([grid], [rec], 10.0, J3, 2, seeds=[5])
    g.monte_carlo_step(50)
    out = g.grid().reshape(-1)
    assert (out[obst] == -1).all()
    vol = g.cells()["volume"][1:]
    tgt = np.array(rec.target[1:])
    assert np.abs(vol - tgt).mean() / tgt.mean() < 0.15
    assert g.records_match_grid()


def test_a_cell_aiming_at_nothing_shrinks_to_nothing():
    # cpm.rs:1438-1457 on the device's sweep
    grid = seeding.empty(50, 50)
    rec = seeding.Records()
    cid = seeding.add_cell(grid, rec, 1, (25, 25), 6)
    rec.target[cid] = 0
    g = cw.CpmLattice.from_grids([grid], [rec], 10.0, REF_J[:2, :2], 1, seeds=[5])
    g.monte_carlo_step(200)
    assert g.volume(cid) == 0 and not (g.grid() == cid).any()


def test_bad_input_is_refused():
    with pytest.raises(cw.ConfigError):
        cw.CpmLattice([(0, 10, 1)], 10.0, 4)
    lat = cw.CpmLattice([(10, 10, 1)], 10.0, 4, J=J3)
    with pytest.raises(cw.ConfigError):
        lat.upload(np.full(100, 7, np.int32))
    with pytest.raises(cw.ConfigError):
        lat.set_contact(np.array([[0, 1], [2, 0]], float))
    with pytest.raises(cw.NotFoundError):
        lat.grid(hist=3)


@pytest.mark.parametrize("volume", [False, True])
def test_divisions_are_bit_exact_with_the_oracle(volume):
    # divide_across (cpm.rs:1094-1160) of many cells at once against the
    # oracle's one at a time, in id order; plus what must not divide
    if volume:
        grid, rec = ball_volume(18)
    else:
        grid, rec = sheet(seed=21, size=80, ncell=24)
    n = len(rec)
    cap = 2 * n + 2
    o = oracle_of(grid, rec, J3, 10.0, 1)
    lat = O.Lattice(o.grid, (o.w, o.h, o.d), cap, J3, 10.0, 1)
    lat.type[:n], lat.volume[:n], lat.target[:n], lat.lam[:n] = o.type, o.volume, o.target, o.lam
    g = cw.CpmLattice.from_grids([grid], [rec], 10.0, J3, 1, seeds=[1], capacity=cap)
    rng = np.random.default_rng(4 + volume)
    ids = np.array([0] + list(range(1, n)), np.int32)  # existing cells only, as divide_ready_cells takes them
    v = rng.normal(size=(ids.size, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    if not volume:
        v[:, 2] = 0.0
    got = g.divide(ids, v)
    used = n
    want = []
    for cid, nrm in zip(ids, v):
        d, used = lat.divide_across(int(cid), nrm, used)
        want.append(d)
    np.testing.assert_array_equal(got, want)
    assert (np.array(want) > 0).sum() >= n // 2
    np.testing.assert_array_equal(g.grid().reshape(-1), lat.grid)
    cells = g.cells()
    np.testing.assert_array_equal(cells["volume"][1:used], lat.volume[1:used])
    np.testing.assert_array_equal(cells["type"][:used], lat.type[:used])
    np.testing.assert_array_equal(cells["target"][:used], lat.target[:used])
    assert g.cell_count() == used
    assert g.records_match_grid()


def oracle_bath(grid):
    d, h, w = grid.shape
    o = O.Field(w, h, d, 0.2, 0.0, 0.0)
    o.hold_bath((grid.reshape(-1) == 0), 1.0)
    return o.held.reshape(d, h, w).astype(np.uint8)


def test_the_device_bath_is_the_reference_flood():
    # hold_medium_bath (coupling.rs:156-158 over pde.rs:550-631): the medium
    # joined to the box's outer layer; the device's union-find against the
    # oracle's flood, in a batch of uneven lattices: sheets of cells, a ring
    # that shuts medium in, a random maze, a volume
    rng = np.random.default_rng(9)
    grids = []
    g, _ = sheet(seed=3, size=96, ncell=60)
    grids.append(g)
    ring = seeding.empty(40, 30)
    y, x = np.mgrid[0:30, 0:40]
    ring[0][(np.maximum(abs(x - 20), abs(y - 15)) == 6)] = 1
    ring[0][0, 5:9] = -1
    grids.append(ring)
    maze = np.where(rng.random((1, 70, 130)) < 0.45, 1, 0).astype(np.int32)
    grids.append(maze)
    vol = np.where(rng.random((12, 14, 16)) < 0.4, 2, 0).astype(np.int32)
    grids.append(vol)
    recs = []
    for gr in grids:
        r = seeding.Records()
        n = int(gr.max()) + 1
        r.type = [0] + [1] * (n - 1)
        r.volume = list(seeding.recount(gr, n))
        r.target = [0] + [49] * (n - 1)
        r.lam = [0.0] + [1.0] * (n - 1)
        recs.append(r)
    flat = cw.CpmLattice.from_grids(grids[:3], recs[:3], 10.0, J3, 1, seeds=[1, 2, 3])
    box = cw.CpmLattice.from_grids(grids[3:], recs[3:], 10.0, J3, 1, seeds=[4])  # a batch is flat or a volume
    for k, gr in enumerate(grids):
        lat, hist = (flat, k) if k < 3 else (box, 0)
        np.testing.assert_array_equal(lat.bath(hist), oracle_bath(gr), err_msg=f"lattice {k}")
    # the shut-in medium inside the ring is not bath; the rest of the medium is
    assert flat.bath(1)[0, 15, 20] == 0 and flat.bath(1)[0, 1, 1] == 1


def _volume_records(gr):
    r = seeding.Records()
    n = int(gr.max()) + 1
    r.type = [0] + [1] * (n - 1)
    r.volume = list(seeding.recount(gr, n))
    r.target = [0] + [49] * (n - 1)
    r.lam = [0.0] + [1.0] * (n - 1)
    return r


def test_the_volume_bath_over_the_occupied_span_is_the_reference_flood():
    # In a volume the union-find covers the occupied span only: medium outside
    # it is bath, a component inside is bath when it reaches the span's border
    # or the box's outer layer.  Four boxes where that rule could go wrong,
    # each against the oracle's flood over the whole box.
    n = 40
    z, y, x = np.mgrid[0:n, 0:n, 0:n]
    r = np.sqrt((x - 20) ** 2 + (y - 20) ** 2 + (z - 20) ** 2)
    # (a) a hollow shell: the sealed pocket inside is not bath, all outside is
    shell = np.where((r >= 6) & (r < 8), 1, 0).astype(np.int32)
    # (b) a bowl (the shell's lower half) whose pocket opens upward onto the
    # span's border layer: the pocket is bath through the layer above the span
    cup = np.where(((r >= 6) & (r < 8)) & (z <= 20), 1, 0).astype(np.int32)
    # (c) tissue touching one box face, so the span is clipped by the box, with
    # a pocket sealed two pixels in from that face
    face = np.where((x <= 8) & (y >= 10) & (y < 30) & (z >= 10) & (z < 30), 1, 0).astype(np.int32)
    face[14:26, 14:26, 2:6] = 0
    # (d) all medium: the span is empty, and every pixel is bath
    empty = np.zeros((n, n, n), np.int32)
    for k, gr in enumerate([shell, cup, face, empty]):
        if gr.max() > 0:
            rec = _volume_records(gr)
        else:
            rec = seeding.Records()
            rec.type, rec.volume, rec.target, rec.lam = [0], [0], [0], [0.0]
        box = cw.CpmLattice.from_grids([gr], [rec], 10.0, J3, 1, seeds=[k + 1])
        np.testing.assert_array_equal(box.bath(0), oracle_bath(gr), err_msg=f"box {k}")
    assert oracle_bath(shell)[20, 20, 20] == 0 and oracle_bath(shell)[0, 0, 0] == 1
    assert oracle_bath(cup)[18, 20, 20] == 1 and oracle_bath(face)[20, 20, 3] == 0 and oracle_bath(empty).all()


def test_an_upload_past_the_capacity_is_refused_and_the_grid_kept():
    """The upload check runs on the device: a clean upload becomes the grid,
    one holding an id past its history's capacity (or below the obstacle's
    -1) is refused naming its first such pixel, and the grid stays as it was;
    the all-history calls move every history in one buffer."""
    from cellweave_b200 import _lib
    lat = cw.CpmLattice([(16, 8, 1), (8, 16, 1)], 10.0, [5, 9], order=1, J=np.zeros((2, 2)))
    rng = np.random.default_rng(4)
    a = rng.integers(-1, 5, 16 * 8).astype(np.int32)
    b = rng.integers(-1, 9, 8 * 8 * 2).astype(np.int32)
    lat.upload(a, 0)
    lat.upload(b, 1)
    np.testing.assert_array_equal(lat.grid(0).reshape(-1), a)
    bad = b.copy()
    bad[37], bad[90] = 9, 12
    with pytest.raises(cw.ConfigError, match="pixel 37 holds id 9, past the history's cell capacity 9"):
        lat.upload(bad, 1)
    np.testing.assert_array_equal(lat.grid(1).reshape(-1), b)
    low = a.copy()
    low[3] = -2
    with pytest.raises(cw.ConfigError, match="pixel 3 holds id -2"):
        lat.upload(low, 0)
    both = np.empty(16 * 8 + 8 * 8 * 2, np.int32)
    _lib.check(_lib.lib().cw_lattice_download_all(lat.handle, _lib.ptr(both)))
    np.testing.assert_array_equal(both, np.concatenate([a, b]))
    swapped = np.concatenate([np.clip(a[::-1], -1, 4), b[::-1]]).astype(np.int32)
    _lib.check(_lib.lib().cw_lattice_upload_all(lat.handle, _lib.ptr(swapped)))
    np.testing.assert_array_equal(lat.grid(1).reshape(-1), b[::-1])
    wrong = swapped.copy()
    wrong[16 * 8 + 5] = 9  # history 1's pixel 5
    with pytest.raises(cw.ConfigError, match="pixel 5 holds id 9"):
        _lib.check(_lib.lib().cw_lattice_upload_all(lat.handle, _lib.ptr(wrong)))
    np.testing.assert_array_equal(lat.grid(0).reshape(-1), swapped[:16 * 8])


def test_a_plane_through_a_ball_halves_it_on_the_side_it_faces():
    # cpm.rs:1645-1673: a ball of radius 5 cut by the plane of normal +z
    # through its centre; the centre slice stays with the parent, the
    # daughter is the half above it; and the same cut on the oracle
    grid = seeding.empty(30, 30, 30)
    rec = seeding.Records()
    seeding.add_ball(grid, rec, 1, (15, 15, 15), 5, lam=2.0)
    size = int((grid == 1).sum())
    g = cw.CpmLattice.from_grids([grid], [rec], 10.0, J3, 1, seeds=[1], capacity=3)
    daughter = int(g.divide(np.array([1], np.int32), np.array([[0.0, 0.0, 1.0]]))[0])
    assert daughter == 2
    out = g.grid()
    a, b = int((out == 1).sum()), int((out == 2).sum())
    assert a + b == size and a > b and 2 * b > a
    assert np.nonzero(out == 2)[0].min() > 15
    o = oracle_of(grid, rec, J3, 10.0, 1)
    lat = O.Lattice(o.grid, (30, 30, 30), 3, J3, 10.0, 1)
    lat.type[:2], lat.volume[:2], lat.target[:2], lat.lam[:2] = o.type, o.volume, o.target, o.lam
    assert lat.divide_across(1, (0.0, 0.0, 1.0), 2) == (2, 3)
    np.testing.assert_array_equal(out.reshape(-1), lat.grid)
    assert g.records_match_grid()
