"""Failure detection without a GPU fault (GPU).

Every wait on the device is bounded: a sublattice pass's grid barrier and an
FP32 sweep's wait for its TMA copies give up after a time limit, set an error
record and return, and the host turns the record into CW_ERR_TIMEOUT; a pass
that would need more priority rounds than allowed stops with
CW_ERR_SIMULATION.  Here cw_test_faults makes those waits run out on purpose,
with a limit of a few milliseconds: one block of a pass kept from its
barrier, a sweep that announces copies it never issues, a round limit of 1.
Nothing faults, traps or hangs: each wait ends by its limit, and the next
call on the same handle works (the lattice against the oracle, the field to
its tolerance).
"""
import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import _lib, seeding
from oracle import oracle as O

pytestmark = pytest.mark.gpu

J3 = np.array([[0, 16, 16], [16, 8, 12], [16, 12, 8]], float)
LIMIT_NS = 5_000_000  # 5 ms


def faults(wait_ns=0, withhold=-1, max_rounds=0, skip_tma=0):
    _lib.check(_lib.lib().cw_test_faults(wait_ns, withhold, max_rounds, skip_tma))


@pytest.fixture(autouse=True)
def back_to_defaults():
    faults()
    yield
    faults()


def sheet_pair(seed=3, size=96, ncell=40):
    grid = seeding.empty(size, size)
    rec = seeding.Records()
    rng = np.random.default_rng(seed)
    k = 0
    while len(rec) - 1 < ncell:
        x, y = rng.integers(0, size - 7, 2)
        if (grid[0, y:y + 7, x:x + 7] != 0).any():
            continue
        seeding.add_block(grid, rec, 1 + (k % 2), (x, y), 7, 7, lam=1.0)
        k += 1
    o = O.Lattice(grid, (size, size, 1), len(rec), J3, 10.0, 2)
    t, v, tg, lam = rec.arrays()
    o.type[:], o.volume[:], o.target[:], o.lam[:] = t, v, tg, lam
    g = cw.CpmLattice.from_grids([grid], [rec], 10.0, J3, 2, seeds=[seed])
    return o, g


def test_the_knobs_are_checked():
    with pytest.raises(cw.ConfigError):
        faults(wait_ns=10)
    with pytest.raises(cw.ConfigError):
        faults(max_rounds=-1)


def test_a_block_kept_from_the_grid_barrier_times_out_and_the_next_step_is_the_oracles():
    o, g = sheet_pair()
    before = g.grid().copy()
    faults(wait_ns=LIMIT_NS, withhold=0)
    with pytest.raises(_lib.TimeoutError_):
        g.monte_carlo_step(1)
    # every pass gave up at its first barrier, before any round: nothing moved
    np.testing.assert_array_equal(g.grid(), before)
    assert g.records_match_grid()
    # the failed step still took its step number; the next ones are the oracle's
    faults()
    g.monte_carlo_step(3)
    o.mcs_checkerboard(3, 1, 3)
    np.testing.assert_array_equal(g.grid().reshape(-1), o.grid)
    np.testing.assert_array_equal(g.cells()["volume"][1:], o.volume[1:])
    assert g.records_match_grid()


def test_a_pass_past_its_round_limit_is_a_simulation_error_and_the_books_stay_true():
    o, g = sheet_pair(seed=5)
    faults(max_rounds=1)
    with pytest.raises(cw.SimulationError):
        g.monte_carlo_step(1)
    assert g.records_match_grid()
    faults()
    g.monte_carlo_step(2)
    assert g.records_match_grid()


def test_an_fp32_sweep_whose_copies_never_land_times_out_and_the_next_solve_settles():
    n = 256  # rows of 16-byte multiples: the TMA-fed sweep kernel
    rng = np.random.default_rng(2)
    sink = np.where(rng.random(n * n) < 0.6, 0.01, 0.0)
    held = np.zeros(n * n, np.uint8)
    held[:n] = 1
    f = cw.ScalarField.new(n, n, 1.0, 0.0, 0.0)
    f.set_linear_sink(sink)
    f.hold_where(1.0, held)
    faults(wait_ns=LIMIT_NS, skip_tma=1)
    with pytest.raises(_lib.TimeoutError_):
        f.relax(1e-8, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, block_depth=8)
    faults()
    st = f.relax(1e-9, 1_000_000, omega=1.9, stop=cw.STOP_RESIDUAL, precision=cw.FP32_DC, block_depth=8, stats=True)
    assert st[0]["residual"] < 1e-9
    o = O.Field(n, n, 1, 1.0, 0.0, 0.0)
    o.lin_sink = sink.copy()
    o.held[:] = held
    o.values[held == 1] = 1.0
    assert o.relax(1e-12, 1_000_000, omega=1.9, stop=1)[0] == 0
    assert np.abs(f.values() - o.values).max() < 1e-6
