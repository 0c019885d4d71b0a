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


def test_named_adjoint_workload_gradient_matches_central_differences():
    """The adjoint workload at its full size: 256 x 256 jittered quads split
    into 131,072 triangles, DG1, S8, the detector response over a seeded
    16 x 16-cell patch; the adjoint gradient with respect to every cell's
    sigma_t and sigma_s (262,144 parameters) against central differences
    (J(s + h d) - J(s - h d)) / 2h, step h = 1e-6 relative to sigma, along 32
    seeded random unit directions: agreement to 1e-5 relative along each.

    Along a random unit direction in 262,144 dimensions the difference
    J(s + h d) - J(s - h d) is ~1e-9 of J, below what two independently
    rounded FP64 solves resolve (each J to ~1e-12). So the numerator is taken
    as g . (psi+ - psi-), the difference of the two forward solutions solved
    as one system: A+ (psi+ - psi-) = (A- - A+) psi-, exact algebra since
    A+ psi+ = A- psi- = b. Only removal and scattering depend on sigma, so
    (A- - A+) x = ds_t x - ds_s / W sum_b w_b x_b with ds = sigma- - sigma+
    (an exact FP64 difference of two nearby values): formed this way it
    carries no cancellation, where two full applies agree to ~1e-9 of their
    size. It is checked against those two applies, and J+ from the direct
    solve against J- + g . (psi+ - psi-)."""
    prob = P.config_tri256()
    g, q = prob.geometry, prob.quad
    st, ss = prob.sigma_t[0], prob.sigma_s[0, 0]
    det = P.detector_patch(prob).astype(np.float64)
    ctx = T.Context(g, q)
    model = T.DetectorResponse(ctx, prob.source[0], det, rtol=1e-12, max_it=2000)
    sigma_t = dev(st).requires_grad_(True)
    sigma_s = dev(ss).requires_grad_(True)
    J = model(sigma_t, sigma_s)
    # The adjoint source sits on 0.2% of the cells, so its right-hand side is
    # small against A lambda and its rounding floor is higher: 1e-11 there
    # bounds the gradient's error far below the 1e-5 asked of it
    model.solver.opts.rtol = 1e-11
    gt, gs = torch.autograd.grad(J, (sigma_t, sigma_s))
    model.solver.opts.rtol = 1e-12
    op = T.TransportOperator(ctx)
    diff = T.TransportSolver(ctx, rtol=1e-10, max_it=2000)
    nc, nb, na = g.n_cells, g.n_basis, q.n_angles
    w = dev(q.w)

    def sigma_difference(ds_t, ds_s, x):
        """(A- - A+) x from the removal and scattering terms alone."""
        xv = x.view(nc, nb, na)
        mom = (xv @ w) / q.sum_weights
        return (ds_t[:, None, None] * xv - (ds_s[:, None] * mom)[:, :, None]).reshape(-1)

    rng = np.random.Generator(np.random.PCG64(P.SEED_BASE + 3))
    worst = worst_j = worst_r = 0.0
    for _ in range(32):
        d = rng.standard_normal(2 * g.n_cells)
        d /= np.linalg.norm(d)
        dt, ds = d[:g.n_cells], d[g.n_cells:]
        h = 1e-6
        plus = (dev(st * (1 + h * dt)), dev(ss * (1 + h * ds)))
        minus = (dev(st * (1 - h * dt)), dev(ss * (1 - h * ds)))
        with torch.no_grad():
            jp = model(*plus).item()
            ctx.set_group(*minus)
            psi_m, _ = model.solver.solve(model.b)
            jm = float(torch.dot(model.g, psi_m))
            r_apply = op.mult(psi_m)
            ctx.set_group(*plus)
            r_apply -= op.mult(psi_m)
            r = sigma_difference(minus[0] - plus[0], minus[1] - plus[1], psi_m)
            worst_r = max(worst_r, float(torch.linalg.norm(r - r_apply) / torch.linalg.norm(r)))
            dpsi, stats = diff.solve(r)
            assert stats["converged"], stats
            dj = float(torch.dot(model.g, dpsi))
        fd = dj / (2 * h)
        ad = float(torch.dot(gt, dev(st * dt)) + torch.dot(gs, dev(ss * ds)))
        worst = max(worst, abs(fd - ad) / abs(ad))
        worst_j = max(worst_j, abs(jp - (jm + dj)) / abs(jp))
    assert worst <= 1e-5, worst
    assert worst_j <= 1e-10, worst_j
    # Two full applies agree to ~1e-9 of their size, so their difference
    # carries ~1e-5 of itself in rounding: the reason it is not used above
    assert worst_r <= 1e-4, worst_r
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


def test_mixed_gradient_on_jittered_tets_matches_central_differences():
    """The combined workload's shape, small: jittered Kuhn tetrahedra, DG1,
    S4, lognormal(0, 1) sigma_t, c ~ U(0.5, 0.999), a central source box and
    a corner detector box; the gradient of the mixed FP32 + FP64-refinement
    solve with respect to every cell's sigma_t against central differences
    of FP64 forward solves along seeded directions."""
    rng = np.random.default_rng(44)
    mesh = P.box_tets(4, 4, 4, jitter=0.2, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(3, 4)
    nc = g.n_cells
    st = rng.lognormal(0.0, 1.0, nc)
    ss = st * rng.uniform(0.5, 0.999, nc)
    cen = g.centroid.reshape(nc, 3)
    src = np.all((cen > 0.25) & (cen < 0.75), axis=1).astype(float)
    det = np.all(cen > 0.55, axis=1).astype(float)
    ctx = T.Context(g, q)
    mixed = T.DetectorResponse(ctx, src, det, rtol=1e-12, max_it=3000, precision="mixed")
    plain = T.DetectorResponse(ctx, src, det, rtol=1e-13, max_it=3000)
    sigma_t = dev(st).requires_grad_(True)
    J = mixed(sigma_t, dev(ss))
    (gt,) = torch.autograd.grad(J, (sigma_t,))
    for _ in range(3):
        d = rng.standard_normal(nc)
        d /= np.linalg.norm(d)
        h = 1e-6
        with torch.no_grad():
            jp = plain(dev(st * (1 + h * d)), dev(ss)).item()
            jm = plain(dev(st * (1 - h * d)), dev(ss)).item()
        fd = (jp - jm) / (2 * h)
        ad = float(torch.dot(gt, dev(st * d)))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)
    ctx.close()
