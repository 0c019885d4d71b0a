"""Parity of the CUDA operator kernels with the CPU oracle, through the C ABI.

Every kernel is compared on the same seeded inputs: FP64 to 1e-13 of the
result's max norm (summation order is the only difference), FP32 to 2e-5.
Full-size cases use size-independent properties instead (linearity, the
adjoint identity <A x, y> = <x, A^T y>, FP32 against FP64)."""
import numpy as np
import pytest
import torch

import oracle as O
from ubolt_b200 import problem as P
from ubolt_b200 import transport as T

from _cases import CASES, build, case_ids

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 2e-5


def rel(a, b):
    a = a.detach().cpu().double().numpy() if torch.is_tensor(a) else a
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.fixture(params=CASES, ids=case_ids())
def setup(request):
    mesh, g, q, st, ss = build(request.param)
    ctx = T.Context(g, q)
    st_d, ss_d = dev(st), dev(ss)
    ctx.set_group(st_d, ss_d)
    op = O.Operator(g, q, st, ss)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(op.n)
    yield ctx, op, g, q, st, ss, x, (st_d, ss_d)
    ctx.close()


def test_apply_matches_oracle(setup):
    ctx, op, g, q, st, ss, x, _ = setup
    A = T.TransportOperator(ctx)
    xd = dev(x)
    assert rel(A.mult(xd), op.apply(x)) < TOL64
    assert rel(A.mult_unscattered(xd), op.apply(x, scatter=False)) < TOL64
    assert rel(A.mult_transpose(xd), op.matrix().T @ x) < TOL64
    assert rel(A.diagonal(), op.L.diagonal()) < TOL64


def test_apply_f32_matches_oracle(setup):
    ctx, op, g, q, st, ss, x, _ = setup
    A = T.TransportOperator(ctx)
    xs = dev(x, torch.float32)
    x32 = xs.double().cpu().numpy()
    assert rel(A.mult(xs), op.apply(x32)) < TOL32
    assert rel(A.mult_unscattered(xs), op.apply(x32, scatter=False)) < TOL32
    assert rel(A.mult_transpose(xs), op.matrix().T @ x32) < TOL32


def test_block_inverse_matches_oracle(setup):
    ctx, op, g, q, st, ss, x, _ = setup
    D = T.ElementBlockInverse(ctx)
    assert D.setup() == 0
    inv_ref, n_sing = op.block_inverse()
    assert n_sing == 0
    assert rel(D.inverse(), inv_ref) < 1e-12
    y_ref = op.block_apply(inv_ref, x)
    assert rel(D.apply(dev(x)), y_ref) < 1e-12
    assert rel(D.apply(dev(x, torch.float32)), y_ref) < 1e-4
    # Transpose: <D^{-1} u, v> = <u, D^{-T} v>
    v = np.random.default_rng(5).standard_normal(op.n)
    lhs = float(np.dot(y_ref, v))
    rhs = float(torch.dot(dev(x), D.apply_transpose(dev(v))))
    assert abs(lhs - rhs) <= 1e-12 * np.abs(y_ref).sum() * np.abs(v).max()


def test_moments_and_rhs_match_oracle(setup):
    ctx, op, g, q, st, ss, x, _ = setup
    nodes = g.n_cells * g.n_basis
    assert rel(T.angular_integral(ctx, dev(x)), O.angular_integral(x, nodes, q)) < TOL64
    rng = np.random.default_rng(9)
    src = rng.uniform(0, 2, g.n_cells)
    side = rng.uniform(0.5, 1.5, 2 * g.dim)
    b_ref = O.rhs(g, q, src, side)
    b = ctx.vector(fill=0.0)
    T.fill_inflow(ctx, side, b)
    gt = T.GroupTransfer(ctx, [[dev(ss)]], [dev(src)])
    gt.add_external(0, b)
    assert rel(b, b_ref) < TOL64
    # transfer: b += sigma_s phi / W from a cached flux
    gt.set_scalar_flux(0, dev(x))
    phi = O.angular_integral(x, nodes, q)
    b2 = O.add_transfer(b_ref.copy(), phi, ss, g.n_cells, g.n_basis, q)
    gt.add_transfer(0, 0, b)
    assert rel(b, b2) < TOL64


def test_full_size_operator_properties():
    """The 256 x 256 DG1 S8 triangle workload: linearity, the adjoint identity
    and FP32 against FP64 (no oracle at this size)."""
    from ubolt_b200 import problem as P
    prob = P.config_tri256()
    ctx = T.Context(prob.geometry, prob.quad)
    st, ss = dev(prob.sigma_t[0]), dev(prob.sigma_s[0, 0])
    ctx.set_group(st, ss)
    A = T.TransportOperator(ctx)
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(ctx.n_rows, dtype=torch.float64, device="cuda", generator=gen)
    y = torch.randn(ctx.n_rows, dtype=torch.float64, device="cuda", generator=gen)
    ax, ay = A.mult(x), A.mult(y)
    lin = A.mult(2.0 * x - 3.0 * y)
    assert (lin - (2.0 * ax - 3.0 * ay)).abs().max() <= 1e-13 * ax.abs().max() * 5
    aty = A.mult_transpose(y)
    lhs, rhs_ = torch.dot(ax, y).item(), torch.dot(x, aty).item()
    assert abs(lhs - rhs_) <= 1e-11 * (ax.abs() * y.abs()).sum().item()
    a32 = A.mult(x.float()).double()
    assert (a32 - ax).abs().max() <= 2e-5 * ax.abs().max()
    ctx.close()


def test_apply_with_few_ordinates_and_large_cells():
    """DG1 hexes at S2 (8 ordinates): 32 cells to a block, whose staged shape
    data and flux need more than 48 KB of shared memory."""
    from ubolt_b200 import problem as P
    rng = np.random.default_rng(5)
    g = P.build_geometry(P.box_hexes(4, 4, 3), 1)
    q = P.lqn(3, 2)
    st = rng.uniform(0.5, 2.0, g.n_cells)
    ss = st * rng.uniform(0.1, 0.9, g.n_cells)
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    op = O.Operator(g, q, st, ss)
    x = rng.standard_normal(op.n)
    A = T.TransportOperator(ctx)
    assert rel(A.mult(dev(x)), op.apply(x)) < TOL64
    assert rel(A.mult_unscattered(dev(x)), op.apply(x, scatter=False)) < TOL64
    assert rel(A.mult(dev(x, torch.float32)), op.apply(dev(x, torch.float32).double().cpu().numpy())) < TOL32
    ctx.close()


def test_apply_with_unaligned_vectors():
    """Vectors that do not start on a 16-byte boundary take the one-ordinate
    thread path; it must agree with the oracle as well."""
    mesh, g, q, st, ss = build(CASES[1])
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    op = O.Operator(g, q, st, ss)
    x = np.random.default_rng(4).standard_normal(op.n)
    A = T.TransportOperator(ctx)
    for dtype, tol in ((torch.float64, TOL64), (torch.float32, TOL32)):
        xb = torch.zeros(op.n + 1, dtype=dtype, device="cuda")
        yb = torch.zeros(op.n + 1, dtype=dtype, device="cuda")
        xs, ys = xb[1:], yb[1:]
        xs.copy_(dev(x, dtype))
        xr = xs.double().cpu().numpy()
        assert rel(A.mult(xs, ys), op.apply(xr)) < tol
        assert rel(A.mult_unscattered(xs, ys), op.apply(xr, scatter=False)) < tol
    ctx.close()


@pytest.mark.parametrize("case", [c for c in CASES if c[0] in ("tri_dg1_refl", "hex_dg1_refl", "tet_dg0_vac")],
                         ids=["tri_dg1_refl", "hex_dg1_refl", "tet_dg0_vac"])
def test_transpose_with_shuffled_ordinates_matches_oracle(case):
    """The transpose through both of its kernels: the LQn order, where every
    aligned run of ordinates maps to a reversed run under the opposite (the
    reversed-angle form of the forward kernel), and the same set shuffled,
    where it does not (the column kernel). Both against the oracle's
    assembled A^T, FP64 and FP32."""
    mesh, g, q, st, ss = build(case)
    perm = np.random.default_rng(5).permutation(q.n_angles)
    inv = np.argsort(perm)
    refl = np.full_like(q.reflect, -1)
    refl[:q.dim] = inv[q.reflect[:q.dim][:, perm]]
    shuffled = P.Ordinates(q.dim, q.sn, np.ascontiguousarray(q.omega[perm]), np.ascontiguousarray(q.w[perm]),
                           np.ascontiguousarray(refl.astype(np.int32)), q.sum_weights)
    for quad in (q, shuffled):
        op = O.Operator(g, quad, st, ss)
        ctx = T.Context(g, quad)
        keep = (dev(st), dev(ss))
        ctx.set_group(*keep)
        x = np.random.default_rng(6).standard_normal(op.n)
        ref = op.matrix().T @ x
        A = T.TransportOperator(ctx)
        got = A.mult_transpose(dev(x)).cpu().numpy()
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
        got32 = A.mult_transpose(dev(x, torch.float32)).double().cpu().numpy()
        assert np.abs(got32 - ref).max() <= 2e-5 * np.abs(ref).max()
        ctx.close()
