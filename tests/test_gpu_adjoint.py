"""The adjoint: the transpose solve against a direct solve of A^T on the
oracle's matrix, the gradient against central finite differences of forward
solves, and the torch.autograd.Function against the direct gradient."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import oracle as O
from ubolt_b200 import problem as P
from ubolt_b200 import transport as T

from _cases import CASES, build, case_ids

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("case", CASES, ids=case_ids())
@pytest.mark.parametrize("pc", ["sweep", "block"])
def test_adjoint_solve_matches_direct_transpose_solve(case, pc):
    mesh, g, q, st, ss = build(case)
    op = O.Operator(g, q, st, ss)
    rhs = np.random.default_rng(3).standard_normal(op.n)
    ref = spla.spsolve(op.matrix().T.tocsc(), rhs)
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    lam, stats = T.TransportSolver(ctx, rtol=1e-12, pc=pc, max_it=3000, restart=60).solve_adjoint(dev(rhs))
    assert stats["converged"]
    assert np.abs(lam.cpu().numpy() - ref).max() <= 1e-9 * np.abs(ref).max()
    ctx.close()


def small_response_problem(n=10, sn=4):
    rng = np.random.default_rng(12)
    mesh = P.box_tris(n, n, jitter=0.2, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, sn)
    nc = g.n_cells
    st = rng.lognormal(0.0, 0.5, nc)
    ss = st * rng.uniform(0.3, 0.99, nc)
    src = (np.linalg.norm(g.centroid.reshape(nc, 3)[:, :2] - 0.4, axis=1) < 0.25).astype(float)
    cen = g.centroid.reshape(nc, 3)
    det = ((cen[:, 0] > 0.6) & (cen[:, 1] > 0.55) & (cen[:, 0] < 0.9) & (cen[:, 1] < 0.85)).astype(float)
    return g, q, st, ss, src, det


def test_gradient_matches_central_differences():
    g, q, st, ss, src, det = small_response_problem()
    ctx = T.Context(g, q)
    model = T.DetectorResponse(ctx, src, det, rtol=1e-13, max_it=2000)
    sigma_t = dev(st).requires_grad_(True)
    sigma_s = dev(ss).requires_grad_(True)
    J = model(sigma_t, sigma_s)
    gt, gs = torch.autograd.grad(J, (sigma_t, sigma_s))
    rng = np.random.default_rng(5)
    for _ in range(4):
        dt = rng.standard_normal(g.n_cells)
        ds = rng.standard_normal(g.n_cells)
        dt /= np.linalg.norm(dt)
        ds /= np.linalg.norm(ds)
        h = 1e-6
        with torch.no_grad():
            jp = model(dev(st * (1 + h * dt)), dev(ss * (1 + h * ds))).item()
            jm = model(dev(st * (1 - h * dt)), dev(ss * (1 - h * ds))).item()
        fd = (jp - jm) / (2 * h)
        ad = float(torch.dot(gt, dev(st * dt)) + torch.dot(gs, dev(ss * ds)))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)
    ctx.close()


def test_gradient_matches_oracle_adjoint():
    """The gradient contraction against the same contraction of the oracle's
    forward and direct-transpose solutions."""
    g, q, st, ss, src, det = small_response_problem(n=8)
    op = O.Operator(g, q, st, ss)
    b = O.rhs(g, q, src)
    A = op.matrix().tocsc()
    psi = spla.spsolve(A, b)
    nc, nb, na = g.n_cells, g.n_basis, q.n_angles
    gvec = np.zeros(op.n)
    gvec.reshape(nc, nb, na)[:, 0, :] = (det * g.volume)[:, None] * q.w[None, :]
    lam = spla.spsolve(A.T.tocsc(), gvec)
    L, Ps = lam.reshape(nc, nb, na), psi.reshape(nc, nb, na)
    want_t = -(L * Ps).sum(axis=(1, 2))
    want_s = (L.sum(axis=2) * (Ps @ q.w)).sum(axis=1) / q.sum_weights
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    gt, gs = T.gradient(ctx, dev(psi), dev(lam))
    assert np.abs(gt.cpu().numpy() - want_t).max() <= 1e-12 * np.abs(want_t).max()
    assert np.abs(gs.cpu().numpy() - want_s).max() <= 1e-12 * np.abs(want_s).max()
    gg = T.response_source(ctx, dev(det))
    assert np.abs(gg.cpu().numpy() - gvec).max() <= 1e-14 * np.abs(gvec).max()
    ctx.close()
