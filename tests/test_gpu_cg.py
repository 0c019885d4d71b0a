"""The CG-SUPG backend on the GPU against its CPU oracle (oracle/cg.py),
through the C ABI: the operator (L - S and L, FP64 and FP32), its diagonal,
point Jacobi, the SUPG-weighted source and transfer, the weak inflow, the
CG DSA, and solves with and without the DSA stage. FP64 to 1e-13 of the
result's max norm, FP32 to 2e-5. The oracle computes its own tables from the
same mesh and its own ordinate set in the library's ordinate order."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import cg as OC
import oracle as O
from ubolt_b200 import _lib
from ubolt_b200 import problem as P
from ubolt_b200 import transport as T

from test_cg_oracle import VOID_2D, VOID_3D, paint_void

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 2e-5


def rel(a, b):
    a = a.detach().cpu().double().numpy() if torch.is_tensor(a) else a
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def meshes():
    rng = np.random.default_rng(5)
    return [
        ("quads", P.box_quads(7, 6, 1.0, 0.7), 4),
        ("quads_jit", P.box_quads(6, 6, jitter=0.2, rng=rng), 4),
        ("tris_jit", P.box_tris(7, 6, 1.0, 0.7, jitter=0.2, rng=rng), 6),
        ("hexes", P.box_hexes(3, 3, 3, 1.0, 1.2, 1.4), 4),
        ("hexes_jit", P.box_hexes(3, 3, 2, jitter=0.15, rng=rng), 2),
        ("tets_jit", P.box_tets(3, 3, 3, jitter=0.2, rng=rng), 4),
    ]


MESHES = meshes()


class Case:
    """One group on a mesh: reflective low sides, vacuum high sides, random
    cross sections with a void box painted in, zeta."""

    def __init__(self, mesh, sn, zeta=0.5, seed=3, void=True):
        dim = mesh.dim
        self.sbc = [1, 0] * dim
        self.g = P.build_cg_geometry(mesh, side_bc=self.sbc)
        self.q = P.lqn(dim, sn)
        self.oq = O.own_quadrature(self.q)
        rng = np.random.default_rng(seed)
        ne = self.g.n_elements
        T_ = OC.Tables(mesh)
        is_void = paint_void(T_, VOID_2D if dim == 2 else VOID_3D) if void else np.zeros(ne, dtype=bool)
        self.st = np.where(is_void, 0.0, rng.uniform(0.5, 3.0, ne))
        self.ss = self.st * rng.uniform(0.1, 0.9, ne)
        self.ctx = T.Context(self.g, self.q, zeta=zeta)
        self.keep = (dev(self.st), dev(self.ss))
        self.ctx.set_group(*self.keep)
        self.pr = OC.Problem(mesh, self.oq, self.st, self.ss, zeta=zeta, side_bc=self.sbc)
        self.rng = rng

    def close(self):
        self.ctx.close()


@pytest.fixture(params=[(m, z) for m in MESHES for z in (0.5, 2.0)],
                ids=[f"{m[0]}-zeta{z}" for m in MESHES for z in (0.5, 2.0)])
def case(request):
    (name, mesh, sn), zeta = request.param
    c = Case(mesh, sn, zeta)
    yield c
    c.close()


def test_cg_apply_matches_oracle(case):
    A = T.TransportOperator(case.ctx)
    x = case.rng.standard_normal(case.pr.n)
    xd = dev(x)
    assert case.ctx.is_cg and case.ctx.n_rows == case.pr.n and case.ctx.n_nodes == case.pr.n_vertices
    assert rel(A.mult(xd), case.pr.matrix() @ x) < TOL64
    assert rel(A.mult_unscattered(xd), case.pr.supg_matrix() @ x) < TOL64
    assert rel(A.diagonal(), case.pr.supg_matrix().diagonal()) < TOL64


def test_cg_apply_f32_matches_oracle(case):
    A = T.TransportOperator(case.ctx)
    xs = dev(case.rng.standard_normal(case.pr.n), torch.float32)
    x32 = xs.double().cpu().numpy()
    assert rel(A.mult(xs), case.pr.matrix() @ x32) < TOL32
    assert rel(A.mult_unscattered(xs), case.pr.supg_matrix() @ x32) < TOL32


def test_cg_jacobi_is_the_inverse_diagonal(case):
    B = T.ElementBlockInverse(case.ctx)
    assert B.setup() == 0
    x = case.rng.standard_normal(case.pr.n)
    d = case.pr.supg_matrix().diagonal()
    assert rel(B.apply(dev(x)), x / d) < TOL64
    assert rel(B.apply(dev(x, torch.float32)), x / d) < TOL32


def test_cg_rhs_fills_match_oracle(case):
    ctx, pr = case.ctx, case.pr
    q = case.rng.uniform(0.0, 2.0, pr.T.cells.shape[0])
    b = ctx.vector(fill=0.0)
    lib, check = _lib.lib, _lib.check
    check(lib.ubolt_add_source(ctx.handle, T._p(dev(q)), T._p(b), T._stream()))
    assert rel(b, pr.source(q)) < TOL64
    phi = case.rng.uniform(0.0, 1.0, pr.n_vertices)
    sig = case.rng.uniform(0.0, 0.5, pr.T.cells.shape[0])
    b.zero_()
    # Both inputs stay referenced until the launch: a temporary freed after
    # its pointer is taken can hand its block to the next allocation
    phi_t, sig_t = dev(phi), dev(sig)
    check(lib.ubolt_add_transfer(ctx.handle, T._p(phi_t), T._p(sig_t), T._p(b), T._stream()))
    assert rel(b, pr.transfer(phi, sig)) < TOL64
    side_in = np.arange(1, 2 * pr.dim + 1, dtype=float) * 0.7
    b.zero_()
    T.fill_inflow(ctx, side_in, b)
    assert rel(b, pr.ghost_inflow(side_in)) < TOL64
    phi_d = T.angular_integral(ctx, dev(np.repeat(phi, pr.A)))
    assert rel(phi_d, phi * pr.W) < TOL64


@pytest.mark.parametrize("zeta", [0.5, 2.0])
@pytest.mark.parametrize("mesh_case", MESHES, ids=[m[0] for m in MESHES])
def test_cg_constant_is_reproduced_through_the_library(mesh_case, zeta):
    """The infinite medium's constant, a void box painted in, reflective and
    matching-inflow vacuum faces: A c - b vanishes through the library's own
    operator and right-hand side (verify_cgk check 3)."""
    name, mesh, sn = mesh_case
    dim = mesh.dim
    g = P.build_cg_geometry(mesh, side_bc=[1, 0] * dim)
    q = P.lqn(dim, 4)
    T_ = OC.Tables(mesh)
    void = paint_void(T_, VOID_2D if dim == 2 else VOID_3D)
    st, ss, src = np.where(void, 0.0, 1.5), np.where(void, 0.0, 0.7), np.where(void, 0.0, 1.0)
    ctx = T.Context(g, q, zeta=zeta)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    inflow = 1.0 / (1.5 - 0.7)
    b = ctx.vector(fill=0.0)
    T.fill_inflow(ctx, [0.0 if (s % 2 == 0) else inflow for s in range(2 * dim)], b)
    _lib.check(_lib.lib.ubolt_add_source(ctx.handle, T._p(dev(src)), T._p(b), T._stream()))
    c = ctx.vector(fill=inflow / q.sum_weights)
    r = T.TransportOperator(ctx).mult(c) - b
    assert r.abs().max().item() <= 1e-12 * b.abs().max().item()
    ctx.close()


@pytest.mark.parametrize("bridge", [False, True])
@pytest.mark.parametrize("mesh_case", MESHES, ids=[m[0] for m in MESHES])
def test_cg_dsa_matches_oracle(mesh_case, bridge):
    """The vertex diffusion operator (SpMV against the oracle's CSR), and
    with an unbridged void in a thick medium D phi = m R A P phi through the
    library's own operator, restriction and prolongation."""
    name, mesh, sn = mesh_case
    c = Case(mesh, sn)
    try:
        ds = T.DSAPrecon(c.ctx, void_bridge=bridge)
        ds.set_group()
        D, info = c.pr.dsa_matrix(bridge=bridge)
        n_void, bridged, chord = ds.void_info()
        assert n_void == int(info["is_void"].sum()) and bridged == info["bridged"]
        assert abs(chord - info["chord"]) <= 1e-13 * max(info["chord"], 1.0)
        u = c.rng.uniform(0.5, 1.5, c.pr.n_vertices)
        assert rel(ds.spmv(dev(u)), D @ u) < TOL64
        x = c.rng.standard_normal(c.pr.n)
        assert rel(ds.restrict(dev(x)), c.pr.dsa_restrict(x)) < TOL64
        assert rel(ds.prolong(dev(u)), c.pr.dsa_prolong(u)) < TOL64
    finally:
        c.close()
    # The restriction identity in a thick medium with an unbridged void
    dim = mesh.dim
    g = P.build_cg_geometry(mesh, side_bc=[1, 0] * dim)
    q = P.lqn(dim, 4)
    void = paint_void(OC.Tables(mesh), VOID_2D if dim == 2 else VOID_3D)
    st, ss = np.where(void, 0.0, 50.0), np.where(void, 0.0, 30.0)
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    ds = T.DSAPrecon(ctx, void_bridge=False)
    ds.set_group()
    phi = dev(np.random.default_rng(3).uniform(0.5, 1.5, ctx.n_nodes))
    lhs = ds.spmv(phi)
    rhs = ds.restrict(T.TransportOperator(ctx).mult(ds.prolong(phi)))
    assert ((lhs - rhs).abs().max() / lhs.abs().max()).item() <= 1e-12
    ctx.close()


@pytest.mark.parametrize("pc", ["block", "block+dsa"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mesh_case", [MESHES[1], MESHES[2], MESHES[5]], ids=["quads_jit", "tris_jit", "tets_jit"])
def test_cg_solve_matches_oracle(mesh_case, pc, precision):
    """GMRES on the CG-SUPG system with point Jacobi, alone or with the DSA
    stage, FP64 or mixed: the scalar flux against the oracle's direct solve."""
    name, mesh, sn = mesh_case
    c = Case(mesh, sn, seed=9)
    try:
        pr = c.pr
        qe = c.rng.uniform(0.0, 2.0, pr.T.cells.shape[0])
        side_in = [0.0, 0.6] * pr.dim
        b = pr.source(qe) + pr.ghost_inflow(side_in)
        psi_ref = spla.spsolve(pr.matrix().tocsc(), b)
        if pc == "block+dsa":
            ds = T.DSAPrecon(c.ctx, inner_iterations=40)
            ds.set_group()
        S = T.TransportSolver(c.ctx, rtol=1e-10, precision=precision, pc=pc, restart=60, max_it=2000)
        x, st = S.solve(dev(b))
        assert st["converged"] and st["residual"] <= 1e-10
        phi_ref = pr.integral() @ psi_ref
        phi = T.angular_integral(c.ctx, x)
        assert rel(phi, phi_ref) < 1e-8
    finally:
        c.close()


def test_cg_dsa_cuts_the_iterations_in_a_diffusive_medium():
    """Scattering ratio 0.99 in an optically thick box: the DSA stage takes
    GMRES from many iterations to a handful (the reference's cg_box_diffusive
    pins: 38 without, 6 with)."""
    mesh = P.box_quads(16, 16, 10.0, 10.0)
    g = P.build_cg_geometry(mesh)
    q = P.lqn(2, 4)
    ne = g.n_elements
    st = np.full(ne, 10.0)
    ss = 0.99 * st
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    b = ctx.vector(fill=0.0)
    _lib.check(_lib.lib.ubolt_add_source(ctx.handle, T._p(dev(np.ones(ne))), T._p(b), T._stream()))
    its = {}
    for pc in ("block", "block+dsa"):
        if pc == "block+dsa":
            ds = T.DSAPrecon(ctx, inner_iterations=60)
            ds.set_group()
        S = T.TransportSolver(ctx, rtol=1e-8, pc=pc, restart=200, max_it=3000)
        x, st_ = S.solve(b)
        assert st_["converged"]
        its[pc] = st_["iterations"]
    assert its["block+dsa"] * 3 <= its["block"], its
    ctx.close()


def test_cg_refuses_what_it_does_not_define():
    mesh = P.box_quads(4, 4)
    g = P.build_cg_geometry(mesh)
    q = P.lqn(2, 2)
    ctx = T.Context(g, q)
    keep = (dev(np.ones(g.n_elements)), dev(np.zeros(g.n_elements)))
    ctx.set_group(*keep)
    x = ctx.vector(fill=1.0)
    A = T.TransportOperator(ctx)
    for call in (lambda: A.mult_transpose(x),
                 lambda: _lib.check(_lib.lib.ubolt_sweep_setup(ctx.handle, 0)),
                 lambda: T.TransportSolver(ctx, pc="sweep")):
        with pytest.raises(_lib.UboltError) as e:
            call()
        assert e.value.status == 4
    dg = P.build_geometry(mesh, 0)
    o = _lib.DsaOptions()
    _lib.lib.ubolt_dsa_defaults(C.byref(o))
    gs = dg.struct()
    with pytest.raises(_lib.UboltError) as e:
        _lib.check(_lib.lib.ubolt_dsa_setup(ctx.handle, C.byref(gs), C.byref(o)))
    assert e.value.status == 1
    ctx.close()
