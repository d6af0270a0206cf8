"""The differentiated fit's forward loss on the CPU, in FP64 (test infrastructure).

The reference has no loss, no adjoint and no autodiff; this restates the loss
the library's fit (cw_fit_*) differentiates, from the oracle's restatements
of the reference's pieces, so that a gradient can be taken independently of
the device: central differences of this loss.  Each field is the fixed point
the reference's SOR (pde.rs:245-405) converges to, solved directly here (a
sparse LU of the same five-point operator: pde.rs's balance per free pixel,
held neighbours on the right-hand side), so that the loss is a smooth
function of the parameters to FP64's rounding and no stopping point of an
iteration moves it between two nearby parameter sets; the floor at zero is
checked to be idle (every free value positive).

    oxygen  D lap c - k_type c = 0, held at `vessel_value` on the lattice's
            obstacle pixels (hold_obstacles_at, coupling.rs:80-82; the
            first-order sink by type as apply_uptake paints it,
            coupling.rs:26-39);
    o_j     mean_per_cell (coupling.rs:164-182);
    x_j(T)  `steps` RK4 steps (network.rs:777-799) from the network's initial
            state, inputs (o_j, egf, 0, 0, 0, 0), the first `ntheta` term
            rates replaced by the parameters;
    signal  D_s lap s - decay s + p = 0, p = secretion x_j(T)[angiogenic] on
            cell j's pixels (apply_production, coupling.rs:61-73);
    loss    sum over bins b of (h_b - h*_b)^2 + w (g_b - g*_b)^2, with h_b the
            mean of sigmoid((level - c) / tau) and g_b the mean of s over the
            cell pixels (id > 0) whose |x - vessel_x| / bin_width falls in b
            (the last bin takes the rest).

Only tests import this module, as the checker.
"""
from __future__ import annotations

import copy

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import oracle as O


def solve_direct(f):
    """The fixed point of pde.rs's relax for field `f` (an oracle Field): per
    free pixel i, (D n_i + decay + k_i) c_i - D sum of its free neighbours =
    source + production_i - uptake_i + D sum of its held neighbours' values,
    n_i its neighbours inside the box (or_pixel_sums, or_denominator).
    Written into f.values; the floor at zero must be idle."""
    w, h, d = f.w, f.h, f.d
    n = w * h * d
    held = f.held.astype(bool)
    free = np.flatnonzero(~held)
    idx = np.full(n, -1, np.int64)
    idx[free] = np.arange(free.size)
    x = np.arange(n) % w
    y = (np.arange(n) // w) % h
    z = np.arange(n) // (w * h)
    real = np.zeros(n)
    rhs = (f.source + f.production - f.uptake).astype(np.float64)
    rows, cols, vals = [], [], []
    for ok, step in ((x > 0, -1), (x + 1 < w, 1), (y > 0, -w), (y + 1 < h, w), (z > 0, -w * h),
                     (z + 1 < d, w * h)):
        real += ok
        i = free[ok[free]]
        j = i + step
        hj = held[j]
        np.add.at(rhs, i[hj], f.dcoef * f.values[j[hj]])
        rows.append(idx[i[~hj]])
        cols.append(idx[j[~hj]])
        vals.append(np.full((~hj).sum(), -f.dcoef))
    den = real * f.dcoef + f.decay
    if f.lin_sink is not None:
        den = den + f.lin_sink
    rows.append(np.arange(free.size))
    cols.append(np.arange(free.size))
    vals.append(den[free])
    a = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(free.size, free.size))
    c = spla.spsolve(a, rhs[free])
    assert (c > 0).all(), "the floor at zero would act: not the linear problem"
    f.values[free] = c


class FitOracle:
    def __init__(self, grid, types, spec, reference_volume, *, dcoef=1.0, uptake=(0.01, 0.005, 0.0),
                 vessel_value=1.0, vessel_x=0, egf=0.2, signal_dcoef=1.0, signal_decay=0.01, secretion=0.05,
                 steps=200, dt=0.01, nbins=16, bin_width=3.0, hypoxic_level=0.1, tau=0.02, signal_weight=1.0,
                 network_params=8):
        self.grid = np.ascontiguousarray(grid, np.int32)
        self.d, self.h, self.w = self.grid.shape
        self.flat = self.grid.reshape(-1)
        self.types = np.ascontiguousarray(types, np.int32)
        self.nc = len(self.types)
        self.net = O.compile_network(spec, reference_volume)
        self.ntheta = min(int(network_params), 32, len(self.net.rate))
        self.angio = self.net.optional["angiogenic"]
        self.vessel_value, self.vessel_x, self.egf = float(vessel_value), int(vessel_x), float(egf)
        self.sd, self.sdecay, self.secretion = float(signal_dcoef), float(signal_decay), float(secretion)
        self.steps, self.dt = int(steps), float(dt)
        self.nbins, self.width = int(nbins), float(bin_width)
        self.level, self.tau, self.weight = float(hypoxic_level), float(tau), float(signal_weight)
        self.params = np.concatenate([[dcoef], np.asarray(uptake, float), self.net.rate[:self.ntheta]])
        x = np.arange(self.flat.size) % self.w
        b = (np.abs(x - self.vessel_x).astype(np.float64) / self.width).astype(np.int64)
        self.bin = np.minimum(b, self.nbins - 1)
        self.cell = self.flat > 0
        self.cnt = np.bincount(self.bin[self.cell], minlength=self.nbins).astype(np.float64)
        self.target_h = np.zeros(self.nbins)
        self.target_g = np.zeros(self.nbins)

    def profiles(self, p):
        p = np.asarray(p, np.float64)
        # oxygen
        o2 = O.Field(self.w, self.h, self.d, float(p[0]), 0.0, 1.0)
        O.hold_obstacles(self.flat, self.vessel_value, o2.held, o2.values)
        rate = np.zeros(8)
        rate[1:4] = p[1:4]
        o2.lin_sink = O.apply_uptake(self.flat, self.types, rate)
        solve_direct(o2)
        c = o2.values
        means = O.mean_per_cell(self.flat, c, self.nc)
        # the network on every record (the medium's too, as the device does)
        net = copy.copy(self.net)
        net.rate = self.net.rate.copy()
        net.rate[:self.ntheta] = p[4:4 + self.ntheta]
        state = np.tile(net.initial, (self.nc, 1))
        inputs = np.zeros((self.nc, 6))
        inputs[:, 0] = means
        inputs[:, 1] = self.egf
        O.network_step(net, state, inputs, self.dt, self.steps)
        # the signal
        per_cell = np.zeros(self.nc)
        if self.angio >= 0:
            per_cell[1:] = self.secretion * state[1:, self.angio]
        sig = O.Field(self.w, self.h, self.d, self.sd, self.sdecay, 0.0)
        sig.production = O.apply_production(self.flat, per_cell)
        solve_direct(sig)
        s = sig.values
        hyp = 1.0 / (1.0 + np.exp(-(self.level - c) / self.tau))
        hb = np.bincount(self.bin[self.cell], weights=hyp[self.cell], minlength=self.nbins)
        gb = np.bincount(self.bin[self.cell], weights=s[self.cell], minlength=self.nbins)
        ok = self.cnt > 0
        h = np.where(ok, hb / np.where(ok, self.cnt, 1.0), 0.0)
        g = np.where(ok, gb / np.where(ok, self.cnt, 1.0), 0.0)
        return h, g

    def loss(self, p):
        h, g = self.profiles(p)
        ok = self.cnt > 0
        dh, dg = (h - self.target_h)[ok], (g - self.target_g)[ok]
        return float((dh * dh).sum() + self.weight * (dg * dg).sum())

    def gradient(self, p, rel=1e-4, floor=1e-6):
        """Central differences of the loss, parameter by parameter (h = rel |p|,
        or `floor` for a parameter at zero).  Where the two losses differ by
        less than 1e8 units in the last place of the loss (a derivative some
        eight orders below the loss's scale, which the loss's rounding could
        move by 1e-4 of itself), the step grows ten times, up to 1e-2 |p|."""
        p = np.asarray(p, np.float64)
        g = np.zeros_like(p)
        ulp = np.spacing(self.loss(p))
        for k in range(p.size):
            r = rel
            while True:
                step = r * abs(p[k]) if p[k] != 0 else floor
                q = p.copy()
                q[k] += step
                up = self.loss(q)
                q[k] -= 2 * step
                down = self.loss(q)
                if up == down or abs(up - down) >= 1e8 * ulp or r >= 1e-2 or p[k] == 0:
                    break
                r *= 10
            g[k] = (up - down) / (2 * step)
        return g
