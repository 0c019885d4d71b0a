"""Geometry invariants and the reference's known-answer identities on the
assembled operator (tests/verify_plexk.kokkos.cxx checks 4, 7, 8 and 1 of
the reference; docs/dev/verification.md:300-437)."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from ubolt_b200 import problem as P
from ubolt_b200._lib import UboltError

from _cases import CASES, build, case_ids


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_layout_and_geometry_invariants(case):
    mesh, g, q, st, ss = build(case)
    dim, F, nc = g.dim, g.faces_per_cell, g.n_cells
    assert g.n_basis == (1 if case[3] == 0 else dim + 1)
    assert abs(g.volume.sum() - 1.0) < 1e-12
    nA = g.face_nA.reshape(nc, F, 3)
    assert np.abs(nA.sum(axis=1)).max() < 1e-12, "outward normals of a cell do not close"
    nbr = g.face_neighbour.reshape(nc, F)
    for c in range(nc):
        for f in range(F):
            n = nbr[c, f]
            if n >= 0:
                assert c in nbr[n], "neighbour relation not symmetric"
    assert np.all(g.face_distance.reshape(-1, 2)[:, 0] > 0)
    interior = g.face_neighbour >= 0
    assert np.all(g.face_bc[interior] == -1) and np.all(g.face_bc[~interior] >= 0)
    if g.n_basis > 1:
        # (1/(V A)) int_f phi_i phi_j is symmetric in i, j
        own = g.face_own.reshape(nc, F, g.n_basis, g.n_basis)
        assert np.allclose(own, np.swapaxes(own, 2, 3), atol=1e-12), "face_own not symmetric"


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_volume_weighted_opposite_ordinate_symmetry(case):
    """(V A)^T = P (V A) P on streaming + heterogeneous removal, reflective
    couplings included (verify_plexk checks 7a and 8b)."""
    mesh, g, q, st, ss = build(case)
    op = O.Operator(g, q, st, np.zeros_like(st))
    A = q.n_angles
    V = np.repeat(g.volume, g.n_basis * A)
    VA = sp.diags(V) @ op.L
    perm = np.arange(op.n).reshape(-1, A)[:, q.opposite()].ravel()
    d = VA.T - VA[perm][:, perm]
    rel = sp.linalg.norm(d) / sp.linalg.norm(VA)
    assert rel < 1e-12, rel


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_transpose_as_reversed_angle_operator_with_row_weighted_scatter(case):
    """The form the transpose kernel computes: (L - S)^T x = P V L (P V^{-1} x)
    - S^T x with (S^T x)(c, i, a) = sigma_s / W w_a sum_b x(c, i, b). The
    scatter is not P-symmetric once the weights differ (S8 here): its weight
    sits on the column, so its transpose carries it on the row."""
    mesh, g, q, st, ss = build(case)
    op = O.Operator(g, q, st, ss)
    M = op.matrix()
    L = O.Operator(g, q, st, np.zeros_like(st)).L
    nc, nb, A = g.n_cells, g.n_basis, q.n_angles
    V = np.repeat(g.volume, nb * A)
    perm = np.arange(op.n).reshape(-1, A)[:, q.opposite()].ravel()
    x = np.random.default_rng(8).standard_normal(op.n)
    st_x = (ss[:, None, None] / q.sum_weights) * q.w[None, None, :] * x.reshape(nc, nb, A).sum(axis=2)[:, :, None]
    y = (V * (L @ (x / V)[perm]))[perm] - st_x.ravel()
    ref = M.T @ x
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()
    if len(set(q.w.tolist())) > 1:
        # The whole operator, scatter included, is not P-symmetric
        VA = sp.diags(V) @ M
        assert sp.linalg.norm(VA.T - VA[perm][:, perm]) > 1e-6 * sp.linalg.norm(VA)


def test_unweighted_symmetry_fails_on_irregular_mesh(rng):
    """On a mesh with varying cell areas the identity needs the volume weight:
    the unweighted A^T = P A P is off by far more than rounding."""
    mesh = P.box_tris(4, 4, jitter=0.2, rng=rng)
    g = P.build_geometry(mesh, 0)
    q = P.lqn(2, 6)
    op = O.Operator(g, q, rng.uniform(0.5, 2.0, g.n_cells), np.zeros(g.n_cells))
    A = q.n_angles
    perm = np.arange(op.n).reshape(-1, A)[:, q.opposite()].ravel()
    rel = sp.linalg.norm(op.L.T - op.L[perm][:, perm]) / sp.linalg.norm(op.L)
    assert rel > 1e-3


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_constant_inflow_is_exact(case):
    """Inflow psi_in on every vacuum face and source sigma_t psi_in: psi = psi_in
    on basis 0, zero slope (verify_plexk checks 7b and 8c)."""
    mesh, g, q, st, ss = build(case)
    op = O.Operator(g, q, st, np.zeros_like(st))
    psi_in = 0.37
    W = q.sum_weights
    b = O.rhs(g, q, st * psi_in * W, np.full(2 * g.dim, psi_in * W))
    x = np.zeros(op.n)
    x.reshape(g.n_cells, g.n_basis, q.n_angles)[:, 0, :] = psi_in
    assert np.abs(b - op.L @ x).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("case", [c for c in CASES if c[3] == 1], ids=[c[0] for c in CASES if c[3] == 1])
def test_linear_field_through_streaming(case):
    """The modal projection of alpha + b . x, the same in every direction,
    through streaming alone gives Omega . b on basis 0 and zero on the slopes
    in every cell with no boundary face (verify_plexk check 8d)."""
    mesh, g, q, st, ss = build(case)
    dim, nb, nc, F, A = g.dim, g.n_basis, g.n_cells, g.faces_per_cell, q.n_angles
    op = O.Operator(g, q, np.zeros(nc), np.zeros(nc))
    alpha, bvec = 0.3, np.array([0.7, -1.1, 0.45])[:dim]
    cen = g.centroid.reshape(nc, 3)[:, :dim]
    beta = g.basis_grad.reshape(nc, nb, 3)[:, 1:, :dim]
    coef = np.zeros((nc, nb))
    coef[:, 0] = alpha + cen @ bvec
    coef[:, 1:] = np.linalg.solve(np.swapaxes(beta, 1, 2), np.broadcast_to(bvec, (nc, dim))[:, :, None])[:, :, 0]
    x = np.repeat(coef[:, :, None], A, axis=2).ravel()
    y = (op.L @ x).reshape(nc, nb, A)
    inner = np.all(g.face_neighbour.reshape(nc, F) >= 0, axis=1)
    want = q.omega[:, :dim] @ bvec
    scale = np.abs(want).max()
    assert inner.sum() > 0
    assert np.abs(y[inner, 0, :] - want[None, :]).max() < 1e-11 * scale
    assert np.abs(y[inner, 1:, :]).max() < 1e-11 * scale


def test_dg0_quad_box_is_the_fd_twin():
    """DG0 upwind on a uniform quad box is the structured FD stencil to
    rounding (verify_plexk check 1a), reflective sides included."""
    nx, ny = 6, 5
    mesh = P.box_quads(nx, ny, tile=4)
    for sbc in ([0, 0, 0, 0], [1, 0, 1, 0], [0, 1, 0, 1]):
        g = P.build_geometry(mesh, 0, side_bc=sbc)
        q = P.lqn(2, 4)
        A = q.n_angles
        rng = np.random.default_rng(3)
        cen = g.centroid.reshape(-1, 3)
        ij = np.floor(cen[:, :2] * [nx, ny]).astype(int)
        natural = ij[:, 1] * nx + ij[:, 0]
        st_nat = rng.uniform(0.5, 2.0, nx * ny)
        op = O.Operator(g, q, st_nat[natural], np.zeros(g.n_cells))
        fd = O.fd2d(nx, ny, q, st_nat, side_bc=sbc)
        rows = (natural[:, None] * A + np.arange(A)[None, :]).ravel()
        Pm = sp.csr_matrix((np.ones(op.n), (np.arange(op.n), rows)), shape=(op.n, op.n))
        d = op.L - Pm @ fd @ Pm.T
        assert abs(d).max() <= 1e-12 * abs(fd).max()


def test_reflective_face_must_be_axis_aligned():
    """A reflective side whose faces are not axis-aligned is rejected (the
    reference's CheckBoundaryFaceBC); a jittered boundary is still a box side."""
    rng = np.random.default_rng(1)
    mesh = P.box_tris(4, 4, jitter=0.2, rng=rng)
    mesh.vertices[:, 0] += 0.05 * mesh.vertices[:, 1]  # shear: the x sides lean
    with pytest.raises(UboltError):
        P.build_geometry(mesh, 1, side_bc=[1, 0, 0, 0])


def test_bad_meshes_are_rejected():
    mesh = P.box_tris(3, 3)
    bad = P.Mesh(2, mesh.cell_type, mesh.vertices, mesh.cells.copy())
    bad.cells[0, 0] = 10_000
    with pytest.raises(UboltError):
        P.build_geometry(bad, 1)
    with pytest.raises(UboltError):
        P.build_geometry(mesh, 2)
    with pytest.raises(UboltError):
        P.build_geometry(P.Mesh(3, mesh.cell_type, mesh.vertices, mesh.cells), 0)


GEOM_FIELDS = ["volume", "centroid", "face_nA", "face_centroid", "face_distance", "face_own", "face_up",
               "basis_grad", "face_neighbour_grad", "face_basis_value"]


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_library_geometry_matches_the_oracles_own(case):
    """The library's geometry (fan moments and the centroid-plus-second-moment
    face matrices, as the reference computes them) against the oracle's own
    (closed-form simplex moments and Gauss quadrature on the faces): every
    field to rounding, the topology and boundary labels exactly. The parity
    tests rest on the oracle's geometry, never the library's."""
    mesh, g, q, st, ss = build(case)
    og = O.own_geometry(g)
    assert og is not g and not hasattr(og, "arrays")
    for name in ("face_neighbour", "face_bc", "face_side"):
        assert np.array_equal(getattr(g, name), getattr(og, name)), name
    boundary = g.face_neighbour < 0
    assert np.array_equal(g.face_axis[boundary], og.face_axis[boundary])
    for name in GEOM_FIELDS:
        if not hasattr(og, name) or name not in g.arrays:
            continue
        a, b = getattr(g, name), getattr(og, name)
        assert a.shape == b.shape, name
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max(), name


@pytest.mark.parametrize("dim", [2, 3])
def test_library_ordinates_match_the_reference_tables(dim):
    """The library's LQn sets against the oracle's, assembled from the
    reference generator's own octant tables: S2-S10 bit for bit, the
    higher orders (where the library's long-double solve and the
    generator's 60-digit one round differently) to 1e-13."""
    for sn in range(2, 20, 2):
        a, b = P.lqn(dim, sn), O.lqn(dim, sn)
        tol = 0.0 if sn <= 10 else 1e-13
        assert a.n_angles == b.n_angles and a.sum_weights == b.sum_weights
        assert np.abs(a.omega - b.omega).max() <= tol
        assert np.abs(a.w - b.w).max() <= tol * b.w.max()
        assert np.array_equal(a.reflect[:dim], b.reflect[:dim])
