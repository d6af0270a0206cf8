"""The hand-written adjoint against central finite differences and an FP64 gradient (GPU).

The fit (cw_fit_*): oxygen D lap c - k_type c = 0 held at a vessel column,
cells' RK4 networks on their mean oxygen with checkpoints, a signal secreted
by the angiogenic node, and a loss on the radial hypoxic-fraction and signal
profiles.  Gradients with respect to D, k (three types) and network rates:

* on a 96 x 96 lattice, against central differences of the device's FP64
  forward (h = 1e-4 relative, every evaluation on a fresh fit) and against
  the CPU oracle's FP64 gradient (oracle/fit.py: the same loss from the
  oracle's restatements of the reference's coupling and RK4 with each field
  solved directly to the fixed point of the reference's relax), each within
  1e-4 of the reference value, relatively, component by component (a
  parameter with no path to the loss has an exact zero on both sides);
* at the differentiated fit's own shape (the 2048 x 2048 cord stepped to MCS
  500 and frozen, 2000 RK4 steps with checkpoints every 100, D, three k and
  32 network rates) against central differences of the device's forward,
  within 1e-4 relative (a derivative too small for a step of 1e-4 of its
  parameter to move the loss by more than FP64 resolves takes a larger step).

A forward pass takes its cell means and bin sums in a fixed order, so it
gives the same loss to the bit every time: the differences then resolve even
the derivatives ten orders below the largest.
"""
import os
import tempfile

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import seeding, synthetic

pytestmark = pytest.mark.gpu

J4 = synthetic.contact_table(4, seed=2)


def geometry(size=96, side=6, seed=4):
    grid = seeding.empty(size, size)
    rec = seeding.Records()
    grid[0, :, size // 2] = -1  # the vessel, an obstacle column
    rng = np.random.default_rng(seed)
    for y in range(1, size - side, side + 1):
        for x in range(1, size - side, side + 1):
            if (grid[0, y:y + side, x:x + side] != 0).any() or rng.random() < 0.15:
                continue
            seeding.add_block(grid, rec, 1 + int(rng.integers(3)), (x, y), side, side, lam=1.0)
    return cw.CpmLattice.from_grids([grid], [rec], 10.0, J4, 2, seeds=[1])


def network(S=8):
    d = tempfile.mkdtemp()
    p = os.path.join(d, "n.toml")
    open(p, "w").write(synthetic.network_toml(S, seed=S))
    return cw.Network.load(p, 36)


def make_fit(lat, net, precision, tol=1e-12, adj=1e-14):
    return cw.Fit(lat, net, dcoef=1.0, uptake=(0.01, 0.005, 0.002), vessel_x=48, steps=200, checkpoint_every=20,
                  dt=0.05, nbins=16, bin_width=3.0, hypoxic_level=0.3, tau=0.05, signal_weight=1.0, tolerance=tol,
                  adjoint_tolerance=adj, precision=precision, network_params=8)


@pytest.fixture(scope="module")
def problem():
    lat, net = geometry(), network()
    fit = make_fit(lat, net, cw.FP32_DC)
    start = fit.params.copy()
    # the target: the same model at D = 1.3 and k = 0.008 for every type
    p = start.copy()
    p[0], p[1:4] = 1.3, 0.008
    fit.params = p
    _, h, g = fit.forward()
    fit.set_target(h, g)
    fit.params = start
    return lat, net, fit, start, h, g


def central_differences(make, start, target, rel=1e-4):
    """Central differences of the loss, each evaluation on a fresh fit (solves
    from the same start, cell means and bin sums in a fixed order: the same
    loss to the bit for the same parameters).  The step is `rel` of the
    parameter; where the two losses then differ by less than 1e8 units in the
    last place of the loss (a derivative some eight orders below the loss's
    scale, whose difference the loss's own rounding could move by 1e-4 of
    itself) it grows ten times, up to 1e-2 of the parameter, so that every
    difference carries the digits the bound asks of it."""
    fd = np.zeros(len(start))

    def loss_at(q):
        f = make()
        f.set_target(*target)
        f.params = q
        v = f.forward()[0]
        del f
        return v

    base = loss_at(start)
    ulp = np.spacing(base)
    for k in range(len(start)):
        r = rel
        while True:
            step = r * abs(start[k]) if start[k] != 0 else 1e-7
            q = start.copy()
            q[k] += step
            up = loss_at(q)
            q[k] -= 2 * step
            down = loss_at(q)
            if up == down or abs(up - down) >= 1e8 * ulp or r >= 1e-2 or start[k] == 0:
                break
            r *= 10
        fd[k] = (up - down) / (2 * step)
    return fd


def test_gradient_matches_central_differences(problem):
    lat, net, fit, start, h, g = problem
    loss, grad = fit.gradient()
    assert loss > 0
    fd = central_differences(lambda: make_fit(lat, net, cw.FP64, tol=1e-13), start, (h, g))
    for k in range(fit.nparams):
        assert abs(grad[k] - fd[k]) <= 1e-4 * abs(fd[k]), (k, grad[k], fd[k])
    fit.params = start


def test_gradient_matches_the_oracles_fp64_gradient(problem):
    # an FP64 gradient that owes nothing to the device: the CPU oracle's loss,
    # differenced centrally, against the device's adjoint with FP64 solves
    import tomllib

    from oracle.fit import FitOracle
    lat, net, fit, start, h, g = problem
    spec = tomllib.loads(synthetic.network_toml(8, seed=8))
    o = FitOracle(lat.grid(), lat.cells()["type"], spec, 36, dcoef=1.0, uptake=(0.01, 0.005, 0.002), vessel_x=48,
                  steps=200, dt=0.05, nbins=16, bin_width=3.0, hypoxic_level=0.3, tau=0.05, signal_weight=1.0,
                  network_params=8)
    np.testing.assert_array_equal(o.params, start)
    o.target_h, o.target_g = h, g
    ref = make_fit(lat, net, cw.FP64, tol=1e-13)
    ref.set_target(h, g)
    ref.params = start
    loss, grad = ref.gradient()
    assert abs(o.loss(start) - loss) <= 1e-9 * loss
    want = o.gradient(start, rel=1e-4)
    for k in range(len(start)):
        assert abs(grad[k] - want[k]) <= 1e-4 * abs(want[k]), (k, grad[k], want[k])


def test_fp32_adjoint_matches_the_fp64_gradient(problem):
    lat, net, fit, start, h, g = problem
    ref = make_fit(lat, net, cw.FP64)
    ref.set_target(h, g)
    ref.params = start
    l64, g64 = ref.gradient()
    l32, g32 = fit.gradient()
    assert abs(l32 - l64) <= 1e-9 * abs(l64)
    np.testing.assert_allclose(g32, g64, rtol=1e-6, atol=1e-9 * np.abs(g64).max())


def test_gradient_descent_lowers_the_loss(problem):
    lat, net, fit, start, h, g = problem
    # steepest descent in the log of the parameters, with backtracking
    p = start.copy()
    fit.params = p
    loss0, grad = fit.gradient()
    loss = loss0
    for _ in range(4):
        d = -grad * p * p  # the gradient in log p, back in p
        alpha = 0.1 / (np.abs(d / np.where(p != 0, p, 1)).max() + 1e-300)
        for _ in range(20):
            q = np.maximum(p + alpha * d, 1e-6)
            fit.params = q
            lq = fit.forward()[0]
            if lq < loss:
                break
            alpha *= 0.5
        p, loss = q, lq
        fit.params = p
        loss, grad = fit.gradient()
    assert loss < loss0
    fit.params = start


def adjoint_field(dims, seed=3):
    rng = np.random.default_rng(seed)
    f = cw.ScalarField(dims, 0.7, 0.001, 0.0)
    for k, (w, h, _) in enumerate(dims):
        f.set_linear_sink(np.where(rng.random(w * h) < 0.6, 0.02, 0.0), k)
        held = np.zeros(w * h, np.uint8)
        held[:w] = 1
        f.hold_where(1.0, held, k)
    return f


def test_field_adjoint_gives_the_derivative_of_a_linear_functional():
    # J(s) = g . c(s), A c = b(s) with a source s m: dJ/ds = lambda . m
    dims = [(48, 40, 1), (30, 30, 1)]
    rng = np.random.default_rng(11)
    m = [rng.random(w * h) for w, h, _ in dims]
    g = np.concatenate([rng.random(w * h) for w, h, _ in dims])

    def J(s):
        f = adjoint_field(dims)
        for k in range(len(dims)):
            f.set_production_array(s * m[k], k)
        f.relax(1e-13, 1_000_000, omega=1.8, stop=cw.STOP_RESIDUAL)
        return float(np.concatenate([f.values(k) for k in range(len(dims))]) @ g)

    f = adjoint_field(dims)
    lam = f.relax_adjoint(g, 1e-13, 1_000_000, omega=1.8)
    held = np.concatenate([f.held(k) for k in range(len(dims))]) == 1
    assert np.all(lam[held] == 0.0)
    s, h = 0.3, 1e-3  # J is linear in s: central differences are exact up to the solves' residual
    fd = (J(s + h) - J(s - h)) / (2 * h)
    assert abs(lam @ np.concatenate(m) - fd) <= 1e-8 * abs(fd)
    # A is symmetric: g2 . lambda(g1) = g1 . lambda(g2), in either precision
    g2 = np.concatenate([rng.random(w * h) for w, h, _ in dims])
    for precision in (cw.FP64, cw.FP32_DC):
        l1 = f.relax_adjoint(g, 1e-12, 1_000_000, omega=1.8, precision=precision)
        l2 = f.relax_adjoint(g2, 1e-12, 1_000_000, omega=1.8, precision=precision)
        assert abs(g2 @ l1 - g @ l2) <= 1e-9 * abs(g @ l2)


def test_network_backward_matches_finite_differences():
    S = 8
    import tomllib
    spec = tomllib.loads(synthetic.network_toml(S, seed=S))
    net = cw.Network.from_spec(spec, 36)
    rng = np.random.default_rng(5)
    n, dt, sub = 40, 0.01, 8
    st = rng.uniform(0.2, 0.8, (n, S))
    ins = np.zeros((n, 6))
    ins[:, 0] = rng.uniform(0.05, 0.95, n)
    ins[:, 1] = 0.2
    w = rng.normal(size=(n, S))

    def L(state, inputs, network=net):
        x = state.copy()
        network.step_batch(x, inputs, dt, sub)
        return float((w * x).sum())

    nterms = sum(len(nd.get("terms", [])) for nd in spec["nodes"])
    nr = min(nterms, 12)
    adj, d_o2, d_rates = net.backward_batch(st, ins, dt, sub, w, nrates=nr)
    h = 1e-6
    for c, i in [(0, 0), (3, 5), (17, 2), (39, 7)]:
        up, dn = st.copy(), st.copy()
        up[c, i] += h
        dn[c, i] -= h
        fd = (L(up, ins) - L(dn, ins)) / (2 * h)
        assert abs(adj[c, i] - fd) <= 1e-6 * max(abs(fd), 1e-3), (c, i, adj[c, i], fd)
    for c in (1, 20):
        up, dn = ins.copy(), ins.copy()
        up[c, 0] += h
        dn[c, 0] -= h
        fd = (L(st, up) - L(st, dn)) / (2 * h)
        assert abs(d_o2[c] - fd) <= 1e-6 * max(abs(fd), 1e-3), (c, d_o2[c], fd)
    # rates: terms in compile order, node by node
    where = [(a, b) for a, nd in enumerate(spec["nodes"]) for b in range(len(nd.get("terms", [])))]
    for t in (0, 3, nr - 1):
        a, b = where[t]
        vals = []
        for sgn in (1, -1):
            sp = tomllib.loads(synthetic.network_toml(S, seed=S))
            rate = sp["nodes"][a]["terms"][b]["rate"]
            sp["nodes"][a]["terms"][b]["rate"] = rate + sgn * h * rate
            vals.append(L(st, ins, cw.Network.from_spec(sp, 36)))
        fd = (vals[0] - vals[1]) / (2 * h * spec["nodes"][a]["terms"][b]["rate"])
        assert abs(d_rates[t] - fd) <= 1e-5 * max(abs(fd), 1e-3), (t, d_rates[t], fd)


def test_the_cord_fit_gradient_matches_central_differences():
    # the differentiated fit's own shape: the 2048 x 2048 cord stepped to MCS
    # 500 and frozen; 2000 RK4 steps checkpointed every 100; D, three uptakes
    # and 32 network rates; the adjoint and the differences (fresh fits, every
    # forward the same to the bit) with the FP32 defect-correction solves
    cfg = synthetic.tumour_cord()
    S = cfg.pop("S")
    d = tempfile.mkdtemp()
    path = os.path.join(d, "n.toml")
    open(path, "w").write(synthetic.network_toml(S, seed=S))
    net = cw.Network.load(path, cfg["target_volume"])
    sim = cw.Simulation(net, **cfg)
    sim.step(500)
    lat = sim.lattice()
    w = cfg["dims"][0][0]

    def fit_of(precision, tol, adj):
        return cw.Fit(lat, net, dcoef=1.0, uptake=(0.01, 0.005, 0.0), vessel_x=w // 2, steps=2000,
                      checkpoint_every=100, dt=0.01, nbins=64, bin_width=w / 128.0, tolerance=tol,
                      adjoint_tolerance=adj, precision=precision, network_params=32)

    fit = fit_of(cw.FP32_DC, 1e-12, 1e-14)
    start = fit.params.copy()
    assert len(start) == 36
    p = start.copy()
    p[0], p[1:4] = 1.3, 0.008
    fit.params = p
    _, h, g = fit.forward()
    fit.set_target(h, g)
    fit.params = start
    loss, grad = fit.gradient()
    assert loss > 0
    fd = central_differences(lambda: fit_of(cw.FP32_DC, 1e-12, 1e-14), start, (h, g))
    for k in range(len(start)):
        assert abs(grad[k] - fd[k]) <= 1e-4 * abs(fd[k]), (k, grad[k], fd[k])
    # D, the uptakes of the living types and the rates upstream of the signal
    assert (fd != 0.0).sum() >= 12
