"""Solution-level known answers on the oracle (the reference's own checks):
DG1 second-order convergence on a pure absorber (verify_plexk check 9,
docs/dev/verification.md:415-424) and the infinite medium
(transportk.kokkos.cxx:43-133)."""
import numpy as np
import pytest

import oracle as O
from ubolt_b200 import problem as P


def absorber_error(mesh_fn, n):
    """sigma = 1 on [0,1]^2, inflow 1 (angle-integrated) on the left, reflective
    bottom and top, cold right: the exact scalar flux is
    sum_{mu > 0} w (1/W) exp(-x / mu). Volume-weighted RMS of cell averages
    against it at the centroids."""
    mesh = mesh_fn(n)
    g = P.build_geometry(mesh, 1, side_bc=[0, 0, 1, 1])
    q = P.lqn(2, 4)
    nc = g.n_cells
    op = O.Operator(g, q, np.ones(nc), np.zeros(nc))
    b = O.rhs(g, q, np.zeros(nc), [1.0, 0.0, 0.0, 0.0])
    x, it, res = op.solve(b, rtol=1e-13, max_it=2000)
    assert res <= 1.01e-13
    phi = O.angular_integral(x, nc * 3, q).reshape(nc, 3)[:, 0]
    cx = g.centroid.reshape(nc, 3)[:, 0]
    mu, w = q.omega[:, 0], q.w
    pos = mu > 0
    exact = (w[pos][None, :] / q.sum_weights * np.exp(-cx[:, None] / mu[pos][None, :])).sum(axis=1)
    return np.sqrt(np.sum(g.volume * (phi - exact) ** 2) / g.volume.sum())


@pytest.mark.parametrize("shape,published", [("quad", (3.5e-3, 8.6e-4, 2.1e-4)), ("tri", (2.4e-3, 6.1e-4, 1.5e-4))])
def test_dg1_is_second_order(shape, published):
    if shape == "quad":
        fn = lambda n: P.box_quads(n, n)
    else:
        fn = lambda n: P.box_tris(n, n, diagonals="uniform")
    errs = [absorber_error(fn, n) for n in (4, 8, 16)]
    order = np.log2(errs[1] / errs[2])
    assert order >= 1.8, (errs, order)
    # The reference's published errors for the same measure: on quads the mesh
    # is the same, so they agree to the two digits published; on triangles the
    # diagonal direction is a mesh choice, so allow 10%
    tol = 0.03 if shape == "quad" else 0.10
    for e, p in zip(errs, published):
        assert abs(e - p) <= tol * p + 0.5e-4 * (p / published[0]), (errs, published)


@pytest.mark.parametrize("dim,sn", [(2, 4), (3, 2)])
def test_oracle_infinite_medium(dim, sn):
    rng = np.random.default_rng(3)
    mesh = P.box_tris(4, 4, jitter=0.2, rng=rng) if dim == 2 else P.box_tets(2, 2, 2, jitter=0.1, rng=rng)
    g = P.build_geometry(mesh, 1, side_bc=[1] * (2 * dim))
    q = P.lqn(dim, sn)
    nc = g.n_cells
    op = O.Operator(g, q, np.full(nc, 2.0), np.full(nc, 1.5))
    b = O.rhs(g, q, np.full(nc, 3.0))
    x, it, res = op.solve(b, rtol=1e-13, max_it=3000)
    want = 3.0 / (q.sum_weights * 0.5)
    xx = x.reshape(nc, g.n_basis, q.n_angles)
    assert np.abs(xx[:, 0] - want).max() <= 1e-9 * want
    assert np.abs(xx[:, 1:]).max() <= 1e-9 * want
