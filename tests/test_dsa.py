"""The DSA diffusion operators: the oracle's restatement against the
reference's own checks (verify_plexk check 11: the MIP matrix is symmetric
and maps a linear field to V sigma_a u on every cell with no boundary face),
and the CUDA path against the oracle through the C ABI (-m gpu)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle as O
from ubolt_b200 import problem as P

from _cases import CASES, build, case_ids


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_diffusion_matrix_is_symmetric(case):
    mesh, g, q, st, ss = build(case)
    D = O.dsa_matrix(g, q, st, ss)
    assert abs(D - D.T).max() <= 1e-12 * abs(D).max()
    # SPD: the smallest eigenvalue of a small case is positive
    if D.shape[0] < 2000:
        assert np.linalg.eigvalsh(D.toarray()).min() > 0


@pytest.mark.parametrize("case", [c for c in CASES if c[3] == 1], ids=[c[0] for c in CASES if c[3] == 1])
def test_mip_maps_a_linear_field_to_absorption(case):
    """One material: a linear u in each cell's modal basis, no jumps and a
    constant flux, so the face terms cancel the volume diffusion term and
    D u = V sigma_a u on every row of every cell with no boundary face."""
    mesh, g, q, st, ss = build(case)
    nc, nb, F, dim = g.n_cells, g.n_basis, g.faces_per_cell, g.dim
    st1, ss1 = np.full(nc, 1.7), np.full(nc, 0.9)
    D = O.dsa_matrix(g, q, st1, ss1)
    bvec = np.array([0.6, -0.35, 0.8])[:dim]
    cen = g.centroid.reshape(nc, 3)[:, :dim]
    beta = g.basis_grad.reshape(nc, nb, 3)[:, 1:, :dim]
    u = np.zeros((nc, nb))
    u[:, 0] = 0.4 + cen @ bvec
    u[:, 1:] = np.linalg.solve(np.swapaxes(beta, 1, 2), np.broadcast_to(bvec, (nc, dim))[:, :, None])[:, :, 0]
    Du = (D @ u.ravel()).reshape(nc, nb)
    inner = np.all(g.face_neighbour.reshape(nc, F) >= 0, axis=1)
    want = (g.volume * (1.7 - 0.9))[:, None] * u
    assert inner.sum() > 0
    assert np.abs(Du[inner] - want[inner]).max() <= 1e-12 * np.abs(Du).max()


def test_dg0_two_point_flux_of_a_constant_is_absorption():
    mesh = P.box_tris(6, 5, jitter=0.2, rng=np.random.default_rng(1))
    g = P.build_geometry(mesh, 0)
    q = P.lqn(2, 4)
    st, ss = np.random.default_rng(2).uniform(0.5, 2, g.n_cells), np.zeros(g.n_cells)
    ss[:] = 0.3 * st
    D = O.dsa_matrix(g, q, st, ss)
    Du = D @ np.ones(g.n_cells)
    inner = np.all(g.face_neighbour.reshape(g.n_cells, 3) >= 0, axis=1)
    assert np.abs(Du[inner] - (g.volume * (st - ss))[inner]).max() <= 1e-12 * np.abs(Du).max()


@pytest.mark.parametrize("consistent", [True, False])
def test_structured_dsa_is_the_dg0_two_point_dsa_on_a_uniform_box(consistent):
    """The structured backend's DSA star (the reference's config-0 DSA,
    dsa_structuredk.kokkos.cxx:183-288: harmonic face D, Marshak vacuum sides,
    the consistent-D blend) restated in the oracle, against the DG0
    two-point-flux DSA on the same uniform quad box: the same operator, the
    plex rows carrying the cell volume. This is what links config 0's DSA to
    the DG0 kernels the GPU path runs."""
    nx, ny = 9, 7
    mesh = P.box_quads(nx, ny)
    g = P.build_geometry(mesh, 0)
    q = P.lqn(2, 4)
    rng = np.random.default_rng(12)
    st = rng.uniform(0.5, 3.0, g.n_cells)
    ss = st * rng.uniform(0.2, 0.95, g.n_cells)
    Dp = O.dsa_matrix(g, q, st, ss, consistent=consistent).toarray()
    og = O.own_geometry(g)
    c = og.centroid.reshape(-1, 3)
    ij = np.floor(c[:, 0] * nx).astype(int) + nx * np.floor(c[:, 1] * ny).astype(int)
    order = np.empty(g.n_cells, dtype=int)
    order[ij] = np.arange(g.n_cells)      # structured index -> plex cell
    Ds = O.dsa_structured(nx, ny, 1.0 / nx, 1.0 / ny, q, st[order], ss[order], consistent=consistent).toarray()
    V = og.volume[order]
    got = Dp[np.ix_(order, order)]
    assert np.abs(got - V[:, None] * Ds).max() <= 1e-12 * np.abs(got).max()


def test_restrict_prolong_round_trip():
    """P D^{-1} R hands back u / W from the x that restricts to D u
    (verify_plexk check 11, the apply round trip)."""
    mesh, g, q, st, ss = build(CASES[0])
    D = O.dsa_matrix(g, q, st, ss).tocsc()
    u = np.random.default_rng(4).standard_normal(g.n_cells * g.n_basis)
    Du = D @ u
    nb, A = g.n_basis, q.n_angles
    x = np.repeat((Du / (np.repeat(g.volume, nb) * q.sum_weights))[:, None], A, axis=1).ravel()
    rhs = O.dsa_restrict(x, g, q)
    y = O.dsa_prolong(spla.spsolve(D, rhs), g, q)
    assert np.abs(y - np.repeat(u / q.sum_weights, A)).max() <= 1e-9 * np.abs(u / q.sum_weights).max()


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# The CUDA path
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

def _gpu(case, inner=30):
    import torch
    from ubolt_b200 import transport as T
    mesh, g, q, st, ss = build(case)
    ctx = T.Context(g, q)
    keep = (torch.tensor(st, device="cuda"), torch.tensor(ss, device="cuda"))
    ctx.set_group(*keep)
    dsa = T.DSAPrecon(ctx, inner_iterations=inner)
    dsa.set_group()
    return ctx, keep, dsa, g, q, st, ss


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_gpu_dsa_matrix_and_spmv_match_oracle(case):
    import torch
    ctx, keep, dsa, g, q, st, ss = _gpu(case)
    D = O.dsa_matrix(g, q, st, ss)
    Dg = dsa.matrix()
    assert abs(Dg - D).max() <= 1e-13 * abs(D).max()
    u = np.random.default_rng(3).standard_normal(D.shape[0])
    v = dsa.spmv(torch.tensor(u, device="cuda")).cpu().numpy()
    assert np.abs(v - D @ u).max() <= 1e-13 * np.abs(D @ u).max()
    x = np.random.default_rng(5).standard_normal(g.n_cells * g.n_basis * q.n_angles)
    rhs = dsa.restrict(torch.tensor(x, device="cuda")).cpu().numpy()
    assert np.abs(rhs - O.dsa_restrict(x, g, q)).max() <= 1e-13 * np.abs(rhs).max()
    y = dsa.prolong(torch.tensor(u, device="cuda")).cpu().numpy()
    assert np.abs(y - O.dsa_prolong(u, g, q)).max() <= 1e-15 * np.abs(y).max()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES[:4], ids=case_ids()[:4])
def test_gpu_dsa_apply_with_a_converged_inner_solve(case):
    import torch
    ctx, keep, dsa, g, q, st, ss = _gpu(case, inner=3000)
    D = O.dsa_matrix(g, q, st, ss).tocsc()
    x = np.random.default_rng(7).standard_normal(g.n_cells * g.n_basis * q.n_angles)
    ref = O.dsa_prolong(spla.spsolve(D, O.dsa_restrict(x, g, q)), g, q)
    y = dsa.apply(torch.tensor(x, device="cuda")).cpu().numpy()
    assert np.abs(y - ref).max() <= 1e-8 * np.abs(ref).max()
    ctx.close()


@pytest.mark.gpu
def test_gpu_sweep_dsa_solve_is_the_same_answer_in_fewer_iterations():
    """A thick, highly scattering problem: DSA does not change the answer and
    cuts the iterations (the reference's plex_box_diffusive_dg1: 7 with, 34
    without, under PCAIR)."""
    import torch
    from ubolt_b200 import transport as T
    rng = np.random.default_rng(3)
    mesh = P.box_tris(16, 16, jitter=0.2, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, 4)
    nc = g.n_cells
    st = np.full(nc, 100.0)
    ss = 0.99 * st
    ctx = T.Context(g, q)
    keep = (torch.tensor(st, device="cuda"), torch.tensor(ss, device="cuda"))
    ctx.set_group(*keep)
    b = ctx.vector(fill=0.0)
    T.GroupTransfer(ctx, [[keep[1]]], [torch.ones(nc, dtype=torch.float64, device="cuda")]).add_external(0, b)
    x0, s0 = T.TransportSolver(ctx, rtol=1e-10, pc="sweep", max_it=3000).solve(b)
    dsa = T.DSAPrecon(ctx, inner_iterations=60)
    dsa.set_group()
    x1, s1 = T.TransportSolver(ctx, rtol=1e-10, pc="sweep+dsa", max_it=3000).solve(b)
    assert s1["converged"] and s0["converged"]
    assert (x1 - x0).abs().max().item() <= 1e-7 * x0.abs().max().item()
    assert s1["iterations"] < s0["iterations"], (s0["iterations"], s1["iterations"])
    ctx.close()


@pytest.mark.gpu
def test_gpu_dsa_apply_is_deterministic():
    """The inner PCG's dot products are fixed-order grid sums: two applies of
    the same input agree bit for bit."""
    import torch
    ctx, keep, dsa, g, q, st, ss = _gpu(CASES[0])
    x = torch.tensor(np.random.default_rng(11).standard_normal(g.n_cells * g.n_basis * q.n_angles), device="cuda")
    y1 = dsa.apply(x).clone()
    for _ in range(3):
        assert torch.equal(dsa.apply(x), y1)
    ctx.close()
