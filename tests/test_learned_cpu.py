"""CPU checks of the learned-preconditioner oracle (oracle/learned_ref.py).

The network has no reference counterpart, so the oracle's gradient is pinned by
central finite differences of its own loss; the GPU kernels are then checked
against this oracle in tests/test_gpu_learned.py.
"""
import numpy as np
import scipy.sparse.linalg as spla

from axisim import cases
import oracle
import learned_ref as LR


def _net_and_sample(nr=10, nz=50, seed=0):
    case = cases.pipe(nr=nr, nz=nz, max_iter=1, tol=1e-30)
    mesh = oracle.multiblock(case.blocks)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    orc.run()
    levels = orc.mg_levels()
    net = LR.NetRef(LR.hierarchy(mesh, orc.mg_level_maps, len(levels)))
    rng = np.random.default_rng(seed)
    N = int(mesh["nCells"])
    ac, af = LR.random_spd_system(mesh, rng)
    A = LR.matrix(mesh, ac, af)
    b = rng.standard_normal(N)
    t = spla.spsolve(A.tocsc(), b)
    d = 1.0 - (np.asarray(abs(A).sum(1)).ravel() - ac) / ac
    return net, (b, t, ac, d, A), levels


def test_oracle_layout_covers_every_level_and_shares_coarse_weights():
    net, _, levels = _net_and_sample()
    assert net.L == len(levels) >= 3
    keys = [ly["key"] for ly in net.layers]
    assert keys[0] == "in" and keys[-1] == "out"
    assert len(net.layers) == 2 + 2 * (net.L - 1) + 1 + 2 * (net.L - 1) + 1
    spans = sorted((off, off + K * Co + Co) for off, K, Co in net.groups.values())
    assert spans[0][0] == 0 and spans[-1][1] == net.n_params
    assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))


def test_oracle_gradient_matches_finite_differences():
    net, (b, t, ac, d, A), _ = _net_and_sample()
    p = net.init_params(seed=3)
    loss, g = net.loss_and_grad(p, b, t, ac, d, A)
    assert np.isfinite(loss) and 0 < loss <= 1
    rng = np.random.default_rng(1)
    idx = []
    for off, K, Co in net.groups.values():  # every group, shared coarse weights and biases included
        idx += list(rng.integers(off, off + K * Co + Co, size=3))
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (net.loss_and_grad(pp, b, t, ac, d, A)[0] - net.loss_and_grad(pm, b, t, ac, d, A)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7, (i, fd, g[i])


def test_oracle_prediction_is_scale_equivariant():
    net, (b, t, ac, d, A), _ = _net_and_sample()
    p = net.init_params(seed=5)
    np.testing.assert_allclose(net.predict(p, 7.5 * b, ac, d), 7.5 * net.predict(p, b, ac, d), rtol=1e-12,
                               atol=1e-12)


def test_energy_loss_is_one_minus_the_optimal_step_reduction():
    net, (b, t, ac, d, A), _ = _net_and_sample()
    p = net.init_params(seed=7)
    loss, _ = net.loss_and_grad(p, b, t, ac, d, A)
    feat, _ = net.features(b, ac, d)
    y = net.forward(p, feat)[0]["Y"][:, 0]
    a = (y @ b) / (y @ (A @ y))  # the line search of one Krylov step from zero
    e = t - a * y
    assert abs(loss - (e @ (A @ e)) / (t @ (A @ t))) < 1e-10
