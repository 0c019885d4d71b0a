"""The oracle's level-symmetric ordinate sets - TEST INFRASTRUCTURE ONLY.

Built from tests/golden/lqn_reference.json, the octant tables that the
reference's own generator (src/sn_lqn_table.py of stevendargaville/UBOLT)
produced, assembled into the full set as SNQuadrature2D::create and
SNQuadrature3D::create do (src/sn_quadraturek.kokkos.cxx:289-379): per
octant point, every sign combination with the x sign fastest, weights the
table's sphere fractions times 4 pi (doubled in 2D for the folded xi < 0
half), and the reflection maps by search (set_directions, :78-111).
"""
import json
import os
from types import SimpleNamespace

import numpy as np

FIXTURE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                       "lqn_reference.json")
_TABLES = None


def _tables():
    global _TABLES
    if _TABLES is None:
        with open(FIXTURE) as fh:
            _TABLES = json.load(fh)["orders"]
    return _TABLES


def lqn(dim, sn):
    """omega (A, 3), w (A,), reflect (3, A) (-1 past dim), sum_weights 4 pi."""
    t = _tables()[str(sn)]
    mu = t["mu"]
    omega, w = [], []
    four_pi = 4.0 * np.pi
    for i, j, k, frac in t["points"]:
        base = (mu[i - 1], mu[j - 1], mu[k - 1])
        if dim == 2:
            for sy in (-1, 1):
                for sx in (-1, 1):
                    omega.append((sx * base[0], sy * base[1], 0.0))
                    w.append(2.0 * frac * four_pi)
        else:
            for sz in (-1, 1):
                for sy in (-1, 1):
                    for sx in (-1, 1):
                        omega.append((sx * base[0], sy * base[1], sz * base[2]))
                        w.append(frac * four_pi)
    omega = np.array(omega)
    w = np.array(w)
    A = len(w)
    reflect = np.full((3, A), -1, dtype=np.int32)
    for d in range(dim):
        for a in range(A):
            want = omega[a].copy()
            want[d] = -want[d]
            hit = np.nonzero(np.all(omega == want, axis=1))[0]
            assert len(hit) == 1 and w[hit[0]] == w[a]
            reflect[d, a] = hit[0]
    return SimpleNamespace(dim=dim, sn=sn, omega=omega, w=w, reflect=reflect, sum_weights=four_pi, n_angles=A)
