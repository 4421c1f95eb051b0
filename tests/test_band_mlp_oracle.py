"""The band MLP objective's CPU restatement: its analytical gradient against
central finite differences (FP64, no rounding), and its BF16 rounding."""
import numpy as np

from oracle import band_mlp as M


def _case(seed=3, n=24):
    rng = np.random.default_rng(seed)
    w = M.init_weights(seed, out_scale=1.0).astype(np.float64)
    x = rng.uniform(0, 1, (n, M.FEAT))
    t = rng.normal(0, 3, (n, 2))
    return w, x, t


def test_gradient_matches_finite_differences():
    w, x, t = _case()
    _, _, g = M.objective(w, x, t, alpha=8.0, rounding=False)
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(M.N_PARAMS, 60, replace=False), np.arange(M.N_PARAMS - 258, M.N_PARAMS)])
    h = 1e-6
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (M.objective(wp, x, t, 8.0, False)[1] - M.objective(wm, x, t, 8.0, False)[1]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)), (k, fd, g[k])


def test_asymmetric_weighting():
    w, x, t = _case(n=8)
    o, loss, _ = M.objective(w, x, t, alpha=1.0, rounding=False)
    e = o - t
    assert np.isclose(loss, np.sum(e * e) / 8)
    o8, loss8, _ = M.objective(w, x, t, alpha=8.0, rounding=False)
    under = np.where(e[:, 0] > 0, 8, 1) * e[:, 0] ** 2 + np.where(e[:, 1] < 0, 8, 1) * e[:, 1] ** 2
    assert np.isclose(loss8, under.sum() / 8)


def test_bf16_round():
    v = np.array([1.0, 1.00390625, 1.005859375, 3.1415927, -2.5e-3, 0.0], np.float32)
    r = M.bf16_round(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to the even mantissa (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] - 3.140625) < 1e-12
    assert np.all(np.abs(r - v) <= np.abs(v) * 2.0 ** -8)
