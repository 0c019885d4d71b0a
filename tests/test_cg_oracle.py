"""The CG-SUPG oracle (oracle/cg.py) pinned by the reference's own known
answers (tests/verify_cgk.kokkos.cxx checks 1-3b and 8): the element tables'
identities, the infinite medium's constant reproduced exactly through the
operator and the right-hand side, the global balance that fixes the weak
boundary terms' scale, and the DSA matrix as the transport operator
restricted onto an isotropic flux."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import cg as OC
import oracle as O
from ubolt_b200 import problem as P


def meshes(jitter):
    rng = np.random.default_rng(11)
    j = 0.2 if jitter else 0.0
    return [
        ("quads", P.box_quads(6, 6, 1.0, 0.7, jitter=j, rng=rng), (1.0, 0.7)),
        ("tris", P.box_tris(6, 6, 1.0, 0.7, jitter=j, rng=rng), (1.0, 0.7)),
        ("hexes", P.box_hexes(3, 3, 3, 1.0, 1.2, 1.4, jitter=j, rng=rng), (1.0, 1.2, 1.4)),
        ("tets", P.box_tets(3, 3, 3, jitter=j, rng=rng), (1.0, 1.0, 1.0)),
    ]


ALL = [(n + ("_jit" if jit else ""), m, L) for jit in (False, True) for n, m, L in meshes(jit)]


@pytest.mark.parametrize("name,mesh,L", ALL, ids=[a[0] for a in ALL])
def test_element_tables_identities(name, mesh, L):
    """Partition of unity, zero row sums of G and K, linear exactness
    sum_j G^d_ij x^d'_j = delta_dd' int phi_i, and lumped masses summing to
    the domain volume (verify_cgk check 1 and 2, tol 1e-12)."""
    T = OC.Tables(mesh)
    dim = mesh.dim
    assert np.abs(T.mass.sum(axis=(1, 2)) - T.volume).max() <= 1e-12 * T.volume.max()
    assert np.abs(T.grad.sum(axis=2)).max() <= 1e-12 * np.abs(T.grad).max()
    assert np.abs(T.stiff.sum(axis=2)).max() <= 1e-12 * np.abs(T.stiff).max()
    xj = T.vertices[T.cells]  # (ne, nv, 3)
    lin = np.einsum("eijd,ejf->eidf", T.grad, xj)
    want = np.einsum("ei,df->eidf", T.mass.sum(axis=2), np.eye(3))
    want[:, :, dim:, :] = 0.0
    want[:, :, :, dim:] = 0.0
    lin[:, :, :, dim:] = 0.0
    assert np.abs(lin - want).max() <= 1e-12 * np.abs(want).max()
    assert abs(T.lumped.sum() - np.prod(L)) <= 1e-12 * np.prod(L)


def paint_void(T, box):
    """Elements whose centroid lies in the box (x0, x1, y0, y1[, z0, z1])."""
    c = T.centroid
    inside = np.ones(len(c), dtype=bool)
    for d in range(c.shape[1]):
        inside &= (c[:, d] >= box[2 * d]) & (c[:, d] <= box[2 * d + 1])
    return inside


VOID_2D = (0.3, 0.7, 0.2, 0.5)
VOID_3D = (0.3, 0.8, 0.3, 0.9, 0.5, 1.5)


def constant_problem(mesh, zeta):
    dim = mesh.dim
    quad = O.lqn(dim, 4)
    T = OC.Tables(mesh)
    void = paint_void(T, VOID_2D if dim == 2 else VOID_3D)
    assert void.any() and not void.all()
    st = np.where(void, 0.0, 1.5)
    ss = np.where(void, 0.0, 0.7)
    q = np.where(void, 0.0, 1.0)
    # Reflective low faces, vacuum high faces fed the medium's flux
    sbc = [1, 0] * dim
    pr = OC.Problem(mesh, quad, st, ss, zeta=zeta, side_bc=sbc)
    inflow = 1.0 / (1.5 - 0.7)
    side_in = [0.0 if sbc[s] else inflow for s in range(2 * dim)]
    b = pr.source(q) + pr.ghost_inflow(side_in)
    return pr, b, inflow / pr.W


@pytest.mark.parametrize("zeta", [0.5, 2.0])
@pytest.mark.parametrize("name,mesh,L", ALL, ids=[a[0] for a in ALL])
def test_constant_is_the_infinite_medium_solution(name, mesh, L, zeta):
    """A constant is the exact discrete solution with a void painted in,
    reflective and matching-inflow vacuum faces (verify_cgk check 3)."""
    pr, b, c = constant_problem(mesh, zeta)
    r = pr.matrix() @ np.full(pr.n, c) - b
    assert np.abs(r).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("name,mesh,L", ALL[:4], ids=[a[0] for a in ALL[:4]])
def test_global_balance_of_a_linear_flux(name, mesh, L):
    """Pure streaming, psi = 1 + c . x on every ordinate, vacuum faces fed
    q_in: per ordinate the lumped-mass sum of A psi - b is the outflow of psi
    minus the inflow q_in / W (verify_cgk check 3b)."""
    dim = mesh.dim
    quad = O.lqn(dim, 4)
    ne = len(mesh.cells)
    q_in, c = 0.7, np.array([0.3, -0.45, 0.2])
    pr = OC.Problem(mesh, quad, np.zeros(ne), np.zeros(ne), zeta=0.5, side_bc=[0] * (2 * dim))
    b = pr.ghost_inflow([q_in] * (2 * dim))
    v = 1.0 + pr.T.vertices[:, :dim] @ c[:dim]
    psi = np.repeat(v, pr.A)
    y = (pr.matrix() @ psi - b).reshape(-1, pr.A)
    sums = (pr.T.lumped[:, None] * y).sum(axis=0)
    expect = np.zeros(pr.A)
    for a in range(pr.A):
        om = pr.omega[a]
        for d in range(dim):
            area = np.prod([L[e] for e in range(dim) if e != d])
            rest = 1.0 + sum(c[e] * 0.5 * L[e] for e in range(dim) if e != d)
            for side in (0, 1):
                on = om[d] if side else -om[d]
                face_psi = rest + (c[d] * L[d] if side else 0.0)
                expect[a] += on * area * face_psi if on > 0 else -(-on) * area * q_in / pr.W
    assert np.abs(sums - expect).max() <= 1e-12 * np.abs(expect).max()


@pytest.mark.parametrize("name,mesh,L", ALL, ids=[a[0] for a in ALL])
def test_dsa_matrix_is_the_restricted_transport_operator(name, mesh, L):
    """Thick material and an unbridged void: D phi = m R A P phi to rounding
    (verify_cgk check 8)."""
    dim = mesh.dim
    quad = O.lqn(dim, 4)
    T = OC.Tables(mesh)
    void = paint_void(T, VOID_2D if dim == 2 else VOID_3D)
    st = np.where(void, 0.0, 50.0)
    ss = np.where(void, 0.0, 30.0)
    pr = OC.Problem(mesh, quad, st, ss, zeta=0.5, side_bc=[1, 0] * dim)
    D, info = pr.dsa_matrix(bridge=False)
    assert info["is_void"].any() and not info["bridged"]
    phi = np.random.default_rng(3).uniform(0.5, 1.5, pr.n_vertices)
    lhs = D @ phi
    rhs = pr.dsa_restrict(pr.matrix() @ pr.dsa_prolong(phi))
    assert np.abs(lhs - rhs).max() <= 1e-12 * np.abs(lhs).max()


def test_void_chord_and_singular_guard():
    """The bridged voids' mean chord 4 V / S on a painted block of a box with
    a reflective low x face and vacuum elsewhere: a face on the reflective
    side is not in S, one on a vacuum side is. All-reflective with no
    absorption is refused."""
    mesh = P.box_quads(8, 8)
    quad = O.lqn(2, 4)
    T = OC.Tables(mesh)
    # The void: x < 0.25 (two columns of cells), touching the left (reflective),
    # bottom and top (vacuum) sides
    void = T.centroid[:, 0] < 0.25
    st = np.where(void, 0.0, 1.0)
    pr = OC.Problem(mesh, quad, st, 0.5 * st, side_bc=[1, 0, 0, 0])
    _, bridged, chord, _ = pr.void_policy()
    V, S = 0.25 * 1.0, 1.0 + 0.25 + 0.25
    assert bridged and abs(chord - 4 * V / S) <= 1e-13
    pr = OC.Problem(mesh, quad, np.ones(len(st)), np.ones(len(st)), side_bc=[1, 1, 1, 1])
    with pytest.raises(ValueError):
        pr.void_policy()


def test_oracle_solves_the_absorber_with_inflow():
    """Sanity of the assembled system: a direct solve of a pure absorber with
    unit inflow on the left decays into the slab and stays positive."""
    mesh = P.box_quads(12, 4, 1.0, 0.4)
    quad = O.lqn(2, 4)
    ne = len(mesh.cells)
    pr = OC.Problem(mesh, quad, np.full(ne, 2.0), np.zeros(ne), side_bc=[0, 0, 1, 1])
    b = pr.ghost_inflow([1.0, 0.0, 0.0, 0.0])
    psi = spla.spsolve(pr.matrix().tocsc(), b)
    phi = pr.integral() @ psi
    x = pr.T.vertices[:, 0]
    left, right = phi[np.isclose(x, 0.0)].mean(), phi[np.isclose(x, 1.0)].mean()
    assert phi.min() > 0 and right < 0.5 * left
