"""Device tree and interaction lists vs the oracle: bit-exact box membership
(same box set with bit-identical FP64 centres, same non-leaf flags, same
stable point permutations) and identical list 1 / PW lists as sets."""
import numpy as np
import pytest

import treecmp
from fgt_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(7)
    return [
        ("3d_uniform", 3, 1e-3, 1e-6, 0, W.uniform(rng, 5000, 3), W.uniform(rng, 3000, 3)),
        ("3d_clusters", 3, 1e-5, 1e-9, 0, W.gaussian_clusters(rng, 20000, 3),
         W.uniform(rng, 5000, 3)),
        ("3d_sphere", 3, 1e-4, 1e-6, 0, W.sphere_with_background(rng, 30000), np.zeros((0, 3))),
        ("3d_sphere_deep", 3, 1e-6, 1e-6, 0, W.sphere_with_background(rng, 60000),
         np.zeros((0, 3))),
        ("2d_periodic", 2, 1e-5, 1e-6, 1, W.uniform(rng, 20000, 2), W.uniform(rng, 2000, 2)),
        ("2d_periodic_clusters", 2, 1e-6, 1e-6, 1, W.gaussian_clusters(rng, 30000, 2),
         np.zeros((0, 2))),
        ("2d_wiggly", 2, 1e-4, 1e-9, 0, W.wiggly_curve(rng, 20000, 2),
         W.uniform(rng, 2000, 2) + 0.5),
        ("1d", 1, 1e-6, 1e-6, 0, W.uniform(rng, 5000, 1), np.zeros((0, 1))),
        ("root_only", 3, 10.0, 1e-6, 0, W.uniform(rng, 300, 3), np.zeros((0, 3))),
        ("tiny", 2, 1e-3, 1e-6, 0, W.uniform(rng, 3, 2), np.zeros((0, 2))),
    ]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_tree_matches_oracle(fgt, oracle, case):
    name, dim, delta, eps, per, src, trg = case
    g = fgt.debug_tree(dim, delta, eps, per, src, trg, bs0=1.0, cen0=[0.0] * dim)
    o = oracle.tree(dim, delta, eps, per, src, trg, bs0=1.0, cen0=[0.0] * dim)
    bad = treecmp.compare(g, o, nlevend=g["nlevend"])
    assert not bad, bad
