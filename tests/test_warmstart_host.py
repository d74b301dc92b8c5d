"""Host side of the NACA/SA warm start (no GPU): the family draws its
parameters inside config 5's ranges, features are finite and O(1), and a
predicted field written by naca_set_state reads back through the primitive
variables as the targets it came from."""
import numpy as np

from aerocfd_b200 import grids, warmstart as W


def test_family_ranges_and_features():
    fam = W.naca_family(6, seed=3, ni=17, nj=9)
    for case, p in fam:
        assert 0.08 <= p["t"] <= 0.15 and 0.0 <= p["m"] <= 0.04 and 0.2 <= p["p"] <= 0.6
        assert -2.0 <= p["aoa_deg"] <= 6.0 and 0.3 <= p["ma"] <= 0.7 and 1e6 <= p["re"] <= 1e7
        assert case.cfg.turbulence == 2 and len(case.blocks) == 4
        f = W.naca_features(case, p)
        assert f.shape == (4 * 17 * 9, W.NACA_IN) and np.all(np.isfinite(f)) and np.abs(f).max() < 5.0


def test_set_state_round_trips_through_the_targets():
    case, p = W.naca_family(1, seed=4, ni=17, nj=9)[0]
    rng = np.random.default_rng(0)
    n = 4 * 17 * 9
    pred = (0.05 * rng.standard_normal((n, W.NACA_OUT))).astype(np.float32)
    W.naca_set_state(case.cfg, case.blocks, pred)
    # primitive variables of the first k-plane, as get_primitivevariables forms them
    for b in case.blocks:
        q = b.fields["q"]
        d = q[..., 0]
        u, v, w = q[..., 1] / d, q[..., 2] / d, q[..., 3] / d
        pr = (q[..., 4] - 0.5 * d * (u * u + v * v + w * w)) * 0.4
        pri = b.fields["pri_v"]
        pri[..., 0], pri[..., 1], pri[..., 2], pri[..., 3], pri[..., 4] = d, u, v, w, pr
    back = W.naca_targets(case)
    assert np.allclose(back, pred, atol=1e-5)


def test_batch_members_and_unbatch():
    cases = [c for c, _ in W.naca_family(3, seed=5, ni=9, nj=5)]
    batch, params = grids.batch_case(cases)
    assert grids.batch_members(cases) == [(0, 4), (4, 8), (8, 12)]
    assert sorted(params) == list(range(1, 13))
    for i, c in enumerate(cases):
        u = grids.unbatch(batch, cases, i)
        assert [b.m for b in u.blocks] == [1, 2, 3, 4]
        for b0, b1 in zip(c.blocks, u.blocks):
            assert [s.blk_t for s in b0.subfaces] == [s.blk_t for s in b1.subfaces]
            assert np.array_equal(b0.fields["x"], b1.fields["x"])
