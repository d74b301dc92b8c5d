"""Learned warm start on a small bump family (farfield boundaries, a unique
steady state): the network trained on solver fields of some members predicts
another member's field; the warm-started run reaches 1e-6 of the cold run's
iteration-1 residual in fewer iterations, and after 8000 iterations (both at
machine-zero residual) the wall forces and cl, cd of the two runs agree to
0.1 %."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    from aerocfd_b200 import build, solver
    build.build()
    return solver


def test_warm_start_saves_iterations(solver):
    from aerocfd_b200 import warmstart as W
    fam = W.family(15, seed=4, ni=33, nj=17, nk=5)
    train, test = fam[:12], fam[12:]
    hist, _, batch = W.run_batch(solver, train, 3000, chunk=500)
    X = np.concatenate([W.features(c, h, m) for c, h, m in train])
    T = np.concatenate([W.targets(W.member(batch, i, c.cfg)) for i, (c, h, m) in enumerate(train)])
    net = W.Network(width=256, depth=6, batch=2048, seed=7)
    try:
        loss = net.train(X, T, steps=4000, lr=1e-3)
        print("training loss first/last", loss[:3], loss[-3:])
        assert loss[-50:].mean() < 0.1 * loss[:10].mean()
        warm = {i: net.predict(W.features(c, h, m)) for i, (c, h, m) in enumerate(test)}
    finally:
        net.close()
    iters, chunk = 8000, 50
    hc, _, bc = W.run_batch(solver, test, iters, chunk=chunk)
    hw, _, bw = W.run_batch(solver, test, iters, chunk=chunk, warm=warm)
    level = hc[0] * 1e-6
    ic, iw = W.first_below(hc, level, chunk), W.first_below(hw, level, chunk)
    print("iterations to 1e-6 of the cold start's residual: cold", ic, "warm", iw)
    print("iteration-1 residual cold", hc[0], "warm", hw[0])
    assert np.all(ic > 0) and np.all(iw > 0) and iw.sum() < ic.sum()
    for i, (c, h, m) in enumerate(test):
        fc = W.wall_force(solver, W.member(bc, i, c.cfg))
        fw = W.wall_force(solver, W.member(bw, i, c.cfg))
        rel = np.abs(fw - fc)[[0, 1, 2, 6, 7]] / np.abs(fc)[[0, 1, 2, 6, 7]]
        print("member", i, "cold", fc[[0, 1, 2, 6, 7]], "rel diff", rel)
        assert rel.max() < 1e-3


def test_warm_start_on_the_naca_sa_family(solver):
    """The NACA 4-digit / SA family (config 5's parameter ranges, 4-block
    O-grids of 4 x 65 x 33 x 3): 16 members run 1500 iterations as one
    batch give the training fields, the network predicts 4 held-out
    members, and the held-out batch runs 1500 iterations from the freestream
    and from the prediction.  Every member runs without a failure; the
    prediction starts every held-out member at under 0.8 of its cold
    iteration-1 residual, and no member takes more iterations to fall to
    1e-2 of it warm than cold, fewer in total."""
    from aerocfd_b200 import grids, warmstart as W
    fam = W.naca_family(20, seed=21, ni=65, nj=33)
    train, test = fam[:16], fam[16:]
    _, _, batch, st = W.run_family_batch(solver, train, 1500, chunk=50)
    assert np.all(st == 0), st
    cases = [c for c, _ in train]
    X = np.concatenate([W.naca_features(*m) for m in train])
    T = np.concatenate([W.naca_targets(grids.unbatch(batch, cases, i)) for i in range(len(train))])
    net = W.Network(n_in=W.NACA_IN, n_out=W.NACA_OUT, width=256, depth=8, batch=8192, seed=3)
    try:
        loss = net.train(X, T, steps=2000, lr=1e-3)
        assert loss[-20:].mean() < 0.1 * loss[:5].mean()
        warm = {i: net.predict(W.naca_features(c, p)) for i, (c, p) in enumerate(test)}
    finally:
        net.close()
    hc, _, _, stc = W.run_family_batch(solver, test, 1500, chunk=50)
    hw, _, _, stw = W.run_family_batch(solver, test, 1500, chunk=50, warm=warm)
    assert np.all(stc == 0) and np.all(stw == 0), (stc, stw)
    ratio = hw[0] / hc[0]
    ic, iw = W.first_below(hc, hc[0] * 1e-2, 50), W.first_below(hw, hc[0] * 1e-2, 50)
    print("iteration-1 residual warm / cold", ratio, "iterations to 1e-2: cold", ic, "warm", iw)
    assert np.all(ratio < 0.8)
    assert np.all(ic > 0) and np.all(iw > 0) and np.all(iw <= ic) and iw.sum() < ic.sum()
