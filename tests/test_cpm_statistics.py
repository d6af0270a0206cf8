"""The sublattice sweep the device runs (restated in the oracle, to the bit)
against the reference's sequential random-pixel sweep, as distributions.

Attempts of one colour meet only through the records of cells they share;
the device settles them in a per-pass priority order (each sees the volumes
every earlier one left), which keeps the volume distribution of the
sequential sweep.  Reading one snapshot of the volumes per pass instead (the
planted mistake below) widens it by about a fifth, which the test sees.
"""
from cpm_ensembles import oracle_ensemble, same_volume_law, within_band


def test_sublattice_sweeps_keep_the_sequential_volume_distribution():
    for mcs in (20, 60):
        seq_v, seq_b = oracle_ensemble("sequential", mcs)
        sub_v, sub_b = oracle_ensemble("sublattice", mcs)
        assert same_volume_law(seq_v, sub_v), (mcs, seq_v.std(), sub_v.std())
        # the boundary coarsens a little faster under sweeps; the ensemble stays in the band
        assert within_band(sub_b, seq_b), (mcs, seq_b.mean(), seq_b.std(), sub_b.mean())


def test_the_check_sees_a_records_snapshot_per_pass():
    seq_v, _ = oracle_ensemble("sequential", 60)
    snap_v, _ = oracle_ensemble("snapshot", 60)
    assert not same_volume_law(seq_v, snap_v), (seq_v.std(), snap_v.std())


def test_moore_copies_keep_the_sequential_volume_distribution_too():
    seq_v, _ = oracle_ensemble("sequential", 40, moore=True)
    sub_v, _ = oracle_ensemble("sublattice", 40, moore=True)
    assert same_volume_law(seq_v, sub_v), (seq_v.std(), sub_v.std())
