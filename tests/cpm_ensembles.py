"""Ensembles of CPM histories for the statistical tests (test helpers).

The device sweeps each colour class of pixels at once, the reference one
random pixel at a time (cpm.rs:748-838); the two sequences differ, so the
dynamics are compared as distributions over 32 seeds: the pooled cell-volume
distribution by a two-sample KS test, and per-history observables against
the band of the reference's sequential ensemble.
"""
import numpy as np

from cellweave_b200 import seeding
from oracle import oracle as O

J = np.array([[0, 16, 16], [16, 8, 12], [16, 12, 8]], float)  # the plain config's adhesion (medium, two types)
SIZE, NCELL, SIDE, T, ORDER = 96, 40, 7, 10.0, 2
SEEDS = 32


def sheet(seed):
    """NCELL squares of SIDE at random free places of a SIZE^2 lattice, types 1, 2 alternating."""
    grid = seeding.empty(SIZE, SIZE)
    rec = seeding.Records()
    rng = np.random.default_rng(seed)
    k = 0
    while len(rec) - 1 < NCELL:
        x, y = rng.integers(0, SIZE - SIDE, 2)
        if (grid[0, y:y + SIDE, x:x + SIDE] != 0).any():
            continue
        seeding.add_block(grid, rec, 1 + (k % 2), (x, y), SIDE, SIDE, lam=1.0)
        k += 1
    return grid, rec


def oracle_lattice(grid, rec):
    d, h, w = grid.shape
    lat = O.Lattice(grid, (w, h, d), len(rec), J, T, ORDER)
    t, v, tg, lam = rec.arrays()
    lat.type[:], lat.volume[:], lat.target[:], lat.lam[:] = t, v, tg, lam
    return lat


def observables(grid2d, volumes):
    """Cell volumes (ids 1..) and the boundary length (4-neighbour pairs of different ids)."""
    g = grid2d
    boundary = int((g[:, 1:] != g[:, :-1]).sum() + (g[1:, :] != g[:-1, :]).sum())
    return np.asarray(volumes[1:]), boundary


def oracle_ensemble(scheme, mcs, moore=False):
    """(pooled volumes, boundary per history) of SEEDS oracle histories after `mcs` steps.

    scheme: "sequential" (the reference's sweep), "sublattice" (the device's,
    restated) or "snapshot" (the sublattice sweep with the planted mistake of
    one records snapshot per pass); `moore`: copies from any Chebyshev
    neighbour."""
    vols, bnd = [], []
    for k in range(SEEDS):
        grid, rec = sheet(k)
        lat = oracle_lattice(grid, rec)
        lat.copy_moore = moore
        if scheme == "sequential":
            lat.mcs_sequential(7919 * k + 1, mcs)
        else:
            lat.mcs_checkerboard(104729 * k + 3, 0, mcs, snapshot=scheme == "snapshot")
        v, b = observables(lat.grid.reshape(SIZE, SIZE), lat.counts()[0])
        vols.append(v)
        bnd.append(b)
    return np.concatenate(vols), np.array(bnd, float)


def same_volume_law(a, b, p_min=0.01, sd_tol=0.12):
    """Pooled volumes alike: KS p above p_min, spreads within sd_tol, means within half a pixel."""
    from scipy import stats
    return (stats.ks_2samp(a, b).pvalue > p_min and abs(b.std() / a.std() - 1.0) < sd_tol
            and abs(b.mean() - a.mean()) < 0.5)


def within_band(sample, band, z=4.0):
    """The sample's mean lies in the band's 2.5-97.5% range and (unless z is None) within z
    standard errors of the band's mean."""
    lo, hi = np.percentile(band, [2.5, 97.5])
    if not lo <= sample.mean() <= hi:
        return False
    if z is None:
        return True
    se = np.sqrt(band.var(ddof=1) / len(band) + sample.var(ddof=1) / len(sample))
    return bool(abs(sample.mean() - band.mean()) <= z * max(se, 1e-12))
