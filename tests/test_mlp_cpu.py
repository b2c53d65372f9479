"""The cost-model oracle on the CPU: its back-propagated gradient against
central finite differences (FP64), which pins it for the GPU gradient check,
and the feature / fallback logic that needs no GPU."""
import numpy as np

from fmm2d_b200 import costmodel as cm
from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin, h1, h2, B = 5, 7, 6, 23
    n = h1 * nin + h1 + h2 * h1 + h2 + h2 + 1
    p = rng.normal(size=n) * 0.5
    X = rng.normal(size=(B, nin))
    T = rng.normal(size=B)
    g = M.gradient(X, T, p, nin, h1, h2)
    fd = np.zeros(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = 1e-6
        fd[i] = (M.loss(X, T, p + e, nin, h1, h2) - M.loss(X, T, p - e, nin, h1, h2)) / 2e-6
    assert np.max(np.abs(g - fd)) < 1e-7 * max(1.0, np.max(np.abs(fd)))


def test_table_fallback_is_lndiv2d():
    assert [cm.table_ndiv(e) for e in (1e-3, 1e-6, 1e-9, 1e-12)] == [10, 15, 20, 25]


def test_features_describe_clustering():
    uni = np.ones((128, 128))
    clu = np.zeros((128, 128))
    clu[60:64, 60:64] = 1000.0
    fu = cm.features_from_hist(uni, 1e-6)
    fc = cm.features_from_hist(clu, 1e-6)
    assert fu.shape == (8,) and np.all(np.isfinite(fu)) and np.all(np.isfinite(fc))
    assert abs(fu[5] - 1.0) < 1e-6 and abs(fu[6] - 1.0) < 1e-6  # full occupancy, max entropy
    assert fc[5] < 0.3 and fc[6] < 0.3                           # compact cluster
