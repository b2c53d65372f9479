"""The device tree equals the oracle's restatement of the reference tree,
array for array (box numbering, centres bit for bit, colleagues, point ranges
and lists 1-4); points inside a leaf are compared as sets."""
import numpy as np
import pytest

from gpu_util import device_tree

pytestmark = pytest.mark.gpu


def _clouds(kind, rng, n):
    if kind == "uniform":
        return rng.uniform(0, 1, (2, n))
    if kind == "gauss16":
        c = rng.uniform(0, 1, (2, 16))
        sig = 10 ** rng.uniform(-4, -1, 16)
        k = rng.integers(0, 16, n)
        return c[:, k] + sig[k] * rng.normal(size=(2, n))
    if kind == "curve":
        th = rng.uniform(0, 2 * np.pi, n)
        r = 0.3 * (1 + 0.2 * np.cos(5 * th))
        return np.stack([0.5 + r * np.cos(th), 0.5 + r * np.sin(th)])
    if kind == "dup":
        x = rng.uniform(0, 1, (2, n // 4))
        return np.concatenate([x, x, x, x], 1)
    if kind == "line":
        x = rng.uniform(-3, 7, n)
        return np.stack([x, 2.5 * np.ones(n)])
    raise ValueError(kind)


CASES = [("uniform", 3000, 0, 15, False), ("gauss16", 20000, 0, 15, False),
         ("curve", 8000, 0, 20, True), ("gauss16", 6000, 2, 10, True),
         ("dup", 400, 0, 3, False), ("line", 2000, 1, 8, True), ("uniform", 7, 0, 3, False),
         ("gauss16", 50000, 0, 20, True)]


@pytest.mark.parametrize("kind,n,idiv,ndiv,with_t", CASES)
def test_tree_matches_oracle(gpu, oracle, kind, n, idiv, ndiv, with_t):
    rng = np.random.default_rng(n + ndiv)
    src = _clouds(kind, rng, n)
    trg = rng.uniform(src.min(), src.max(), (2, n // 2 + 1)) if with_t else None
    a = oracle.tree(src, trg, idiv, ndiv)
    b = device_tree(src, trg, idiv, ndiv)
    assert a["nlevels"] == b["nlevels"] and a["nboxes"] == b["nboxes"]
    for k in ["laddr", "ilevel", "iparent", "nchild", "ichild", "ncoll", "coll", "isrcse",
              "nlist1", "list1", "nlist2", "list2", "nlist3", "list3", "nlist4", "list4"]:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["centers"].view(np.int64), b["centers"].view(np.int64))
    assert np.array_equal(a["boxsize"], b["boxsize"])
    if with_t:
        assert np.array_equal(a["itargse"], b["itargse"])
    leaves = np.nonzero(a["nchild"] == 0)[0]
    for key, se in (("isrc", "isrcse"), ("itarg", "itargse")):
        if key == "itarg" and not with_t:
            continue
        for lb in leaves:
            s, e = a[se][lb]
            assert np.array_equal(np.sort(a[key][s:e]), np.sort(b[key][s:e]))
