"""The level-symmetric sets against the reference generator's own output and the
moment conditions (tests/verify_quadraturek.kokkos.cxx:9-30 of the reference)."""
import json
import os

import numpy as np
import pytest

from ubolt_b200 import problem as P
from ubolt_b200._lib import UboltError

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "lqn_reference.json")


@pytest.mark.parametrize("sn", list(range(2, 20, 2)))
def test_octant_matches_reference_generator(sn):
    ref = json.load(open(GOLDEN))["orders"][str(sn)]
    mu, pts, wt = P.lqn_octant(sn)
    rp = np.array([p[:3] for p in ref["points"]])
    rw = np.array([p[3] for p in ref["points"]])
    assert (pts == rp).all(), "octant points out of lexicographic triple order"
    if sn <= 12:
        # Unique sets: the same doubles to within an ulp
        assert np.all(np.abs(mu - ref["mu"]) <= np.spacing(np.asarray(ref["mu"])))
        assert np.all(np.abs(wt - rw) <= np.spacing(rw))
    else:
        # Least-squares members (weight freedom 1-2): long double vs 60 digits
        assert np.max(np.abs(mu - ref["mu"]) / ref["mu"]) < 1e-13
        assert np.max(np.abs(wt - rw) / rw) < 1e-10


@pytest.mark.parametrize("dim,sn", [(2, 2), (2, 4), (2, 8), (2, 12), (3, 2), (3, 4), (3, 8), (3, 16)])
def test_ordinate_set(dim, sn):
    q = P.lqn(dim, sn)
    A = q.n_angles
    assert A == (sn * (sn + 2) // 2 if dim == 2 else sn * (sn + 2))
    assert abs(q.w.sum() - 4 * np.pi) < 1e-13 * 4 * np.pi
    assert q.sum_weights == 4 * np.pi
    # Unit directions (3D); the 2D set drops xi
    if dim == 3:
        assert np.allclose(np.sum(q.omega ** 2, axis=1), 1.0, atol=1e-14)
    else:
        assert np.all(q.omega[:, 2] == 0.0)
    # Odd moments vanish; even axis moments are the sphere's through order N
    for d in range(dim):
        assert abs(np.sum(q.w * q.omega[:, d])) < 1e-13
        for m in range(0, sn // 2 + 1):
            got = np.sum(q.w * q.omega[:, d] ** (2 * m)) / (4 * np.pi)
            assert abs(got - 1.0 / (2 * m + 1)) < 1e-12
    # Reflection maps: negate exactly one cosine, keep the weight, involutive
    for d in range(dim):
        r = q.reflect[d]
        want = q.omega.copy()
        want[:, d] *= -1
        assert np.array_equal(q.omega[r], want)
        assert np.array_equal(q.w[r], q.w)
        assert np.array_equal(r[r], np.arange(A))
    assert np.all(q.reflect[dim:] == -1)


def test_2d_is_the_fold_of_3d():
    """verify_quadraturek: the 2D set is the xi > 0 half of the 3D one, doubled."""
    q2, q3 = P.lqn(2, 8), P.lqn(3, 8)
    upper = q3.omega[:, 2] > 0
    assert np.allclose(np.sort(q2.w), np.sort(2 * q3.w[upper]))
    s2 = sorted(map(tuple, np.round(q2.omega[:, :2], 15)))
    s3 = sorted(map(tuple, np.round(q3.omega[upper][:, :2], 15)))
    assert s2 == s3


@pytest.mark.parametrize("bad", [0, 3, 20, -2])
def test_bad_order_is_rejected(bad):
    with pytest.raises(UboltError) as e:
        P.lqn(2, bad)
    assert "UBOLT_ERR_ARG" in str(e.value)
