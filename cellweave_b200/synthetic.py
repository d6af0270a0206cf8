"""Synthetic inputs of the benchmark configurations, as the reference's formats.

Networks are written as network TOML files (the format of the reference's
examples/networks/*.toml, read by crates/io/src/config.rs:388-447), so they go
through the same load and compile path as a hand-written hypothesis.  The
lattice workloads are described as keyword sets for ``engine.Simulation``.
All of it is seeded and deterministic.
"""
from __future__ import annotations

import numpy as np


def network_toml(S: int, seed: int = 1, density: float = 0.3) -> str:
    """An S-species Hill network: rates and half-saturations drawn U[0.1, 2],
    Hill exponent 2, random +1 (activated_by) / -1 (inhibited_by) wiring between
    nodes at `density`, one `decays` per node.  Node 0 reads oxygen, node 1
    rises in its absence (the hypoxia response), node 2 reads EGF (growth),
    node 3 is survival: held near 0.9 and damaged below an oxygen threshold."""
    if S < 4:
        raise ValueError("a synthetic network needs at least four nodes")
    rng = np.random.default_rng(seed)
    U = lambda: float(rng.uniform(0.1, 2.0))
    lines = [f"# Synthetic {S}-species Hill network (seed {seed}, wiring density {density}).", ""]
    for i in range(S):
        terms = []
        if i == 0:
            terms.append(f'{{ kind = "activated_by", source = "oxygen", rate = {U():.6f}, '
                         f'hill = {{ n = 2.0, k = {U():.6f} }} }}')
        elif i == 1:
            terms.append(f'{{ kind = "activated_by_absence_of", source = "oxygen", rate = {U():.6f} }}')
        elif i == 2:
            terms.append(f'{{ kind = "activated_by", source = "egf", rate = {U():.6f}, '
                         f'hill = {{ n = 2.0, k = {U():.6f} }} }}')
        for j in range(S):
            if j == i or rng.random() >= density:
                continue
            kind = "activated_by" if rng.random() < 0.5 else "inhibited_by"
            terms.append(f'{{ kind = "{kind}", source = "n{j}", rate = {U():.6f}, '
                         f'hill = {{ n = 2.0, k = {U():.6f} }} }}')
        if i == 3:
            terms.append('{ kind = "relaxes_to", value = 0.9, rate = 2.0 }')
            terms.append('{ kind = "damaged_below", source = "oxygen", threshold = 0.05, rate = 4.0 }')
        if i == 4:
            # the angiogenic node answers the hypoxia response, as a VEGF-like
            # signal does (fixed parameters: the draws of the rest stay as they were)
            terms.append('{ kind = "activated_by", source = "n1", rate = 1.0, hill = { n = 2.0, k = 0.3 } }')
        terms.append(f'{{ kind = "decays", rate = {U():.6f} }}')
        lines += ["[[nodes]]", f'name = "n{i}"', "initial = 0.5" if i == 3 else "initial = 0.1", "terms = ["]
        lines += [f"  {t}," for t in terms]
        lines += ["]", ""]
    lines += ["[roles]", 'growth = "n2"', 'survival = "n3"', 'hypoxia_response = "n1"']
    if S > 4:
        lines.append('angiogenic = "n4"')
    lines += ["", "[mechanics]", "growth_coefficient = 0.5", "lambda_volume = 1.0", "max_target = 2.0", ""]
    return "\n".join(lines)


def contact_table(K: int, seed: int, lo: int = 4, hi: int = 20) -> np.ndarray:
    """A symmetric K x K table of integer energies drawn U[lo, hi], medium-medium 0."""
    rng = np.random.default_rng(seed)
    J = np.zeros((K, K))
    for a in range(K):
        for b in range(a, K):
            if a == 0 and b == 0:
                continue
            J[a, b] = J[b, a] = float(rng.integers(lo, hi + 1))
    return J


def two_type_table() -> np.ndarray:
    """Medium-cell 16, same type 8, different types 12 (two cell types)."""
    return np.array([[0, 16, 16], [16, 8, 12], [16, 12, 8]], float)


def plain_2d(seed=0):
    """A 256 x 256 lattice, 120 cells as 7 x 7 squares at random places, two types,
    Moore contact, target 49, lambda 1, T 10; oxygen D 1, k 0.01 on cells, held
    at 1 on row 0, FP64 SOR omega 1.85 to residual 1e-10 every 10 steps; 8-species
    network, dt 0.01."""
    return dict(dims=[(256, 256, 1)], ncells=[120], seeds=[seed], temperature=10.0, J=two_type_table(),
                contact_order=2, target_volume=49, lambda_volume=1.0, seeding=0, seed_side=7, nfields=1,
                o2_dcoef=1.0, o2_sink_by_type=(0.0, 0.01, 0.01), o2_hold=0, tolerance=1e-10, precision=0,
                omega=1.85, relax_every=10, dt=0.01, substeps=8, sweeps=1, S=8)


def tumour_cord(n=2048):
    """The large cord: n x n, ~40,000 cells of target 64 (8 x 8 packed squares),
    three types (proliferating, arrested, necrotic) with J drawn U[4, 20], a
    vessel held at 1 down the column x = n/2 with the medium around it
    consuming as stroma (apply_background_uptake, coupling.rs:47-53), oxygen and a signal secreted at
    0.05 by hypoxic cells (c < 0.1), FP32 SOR with FP64 defect correction to
    residual 1e-8 (each field then within 1e-6 of its FP64 solution; residual
    1e-6 left the oxygen 1e-6 to 5e-5 off); 16-species network."""
    return dict(dims=[(n, n, 1)], ncells=[40000 * (n * n) // (2048 * 2048)], seeds=[2], temperature=10.0,
                J=contact_table(4, seed=2), contact_order=2, target_volume=64, lambda_volume=1.0, seeding=1,
                seed_side=8, nfields=2, o2_dcoef=1.0, o2_sink_by_type=(0.0, 0.01, 0.005, 0.0), o2_background_sink=0.001,
                o2_hold=1,
                signal_dcoef=1.0, signal_decay=0.01, signal_secretion=0.05, hypoxic_level=0.1, tolerance=1e-8,
                precision=1, omega=None, relax_every=1, dt=0.01, substeps=8, sweeps=1, death_threshold=0.25,
                necrotic_type=3, S=16)


def campaign(per_size=16, sizes=(128, 256, 512, 1024), fill=0.3, base_seed=1000):
    """The batched campaign: `per_size` histories at each size, seeds 1000+h,
    cells filling 30% at target 49, the plain config's physics with two fields
    solved to residual 1e-8 (each field within 1e-6 of its FP64 solution) and
    an 8-species network."""
    dims, ncells, seeds = [], [], []
    h = 0
    for s in sizes:
        for _ in range(per_size):
            dims.append((s, s, 1))
            ncells.append(int(fill * s * s / 49))
            seeds.append(base_seed + h)
            h += 1
    return dict(dims=dims, ncells=ncells, seeds=seeds, temperature=10.0, J=two_type_table(), contact_order=2,
                target_volume=49, lambda_volume=1.0, seeding=0, seed_side=7, nfields=2, o2_dcoef=1.0,
                o2_sink_by_type=(0.0, 0.01, 0.01), o2_hold=0, signal_dcoef=1.0, signal_decay=0.01,
                signal_secretion=0.05, hypoxic_level=0.1, tolerance=1e-8, precision=1, omega=None, relax_every=1,
                dt=0.01, substeps=8, sweeps=1, S=8)


def spheroid_3d(n=256):
    """The 3D spheroid: n^3, 26-neighbour contact, cells of 5^3 packed in a ball
    of radius 40, T 20, lambda_V 1, surface lambda 0.2 target 150; oxygen held
    at 1 on every face, k 0.005 in cells, solved to residual 1e-9 (the medium
    around the ball consumes nothing, so the error is up to a few hundred
    times the residual); 12-species network."""
    ncell = int(4.0 / 3.0 * np.pi * 40 ** 3 / 125)
    return dict(dims=[(n, n, n)], ncells=[ncell], seeds=[3], temperature=20.0, J=two_type_table(),
                contact_order=3, target_volume=125, lambda_volume=1.0, surface_target=150, lambda_surface=0.2,
                seeding=2, seed_side=5, nfields=1, o2_dcoef=1.0, o2_sink_by_type=(0.0, 0.005, 0.005), o2_hold=2,
                tolerance=1e-9, precision=1, omega=None, relax_every=1, dt=0.01, substeps=8, sweeps=1, S=12)
