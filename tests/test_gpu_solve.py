"""The GPU sweep and the GPU solve against the oracle, through the C ABI.

Sweep: on meshes with acyclic upwind graphs the plan is exact, so the GPU
sweep is L^{-1} and matches the oracle's sweep to rounding (reflective
inflow is lagged to zero by both). Solve: FP64 to a tight tolerance
against the oracle's own FP64 GMRES solve, scalar flux within 1e-10; the
mixed form to a 1e-8 true residual with scalar flux within 1e-7 of FP64;
the known answers of the reference (infinite medium, constant inflow)."""
import numpy as np
import pytest
import torch

import oracle as O
from ubolt_b200 import problem as P
from ubolt_b200 import transport as T

from _cases import CASES, build, case_ids

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def ctx_for(g, q, st, ss):
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    return ctx, keep


ACYCLIC = [c for c in CASES if c[1] == 2 or c[0].startswith("hex")]


@pytest.mark.parametrize("case", ACYCLIC, ids=[c[0] for c in ACYCLIC])
@pytest.mark.parametrize("patch", [0, 16, 100])
def test_sweep_matches_oracle(case, patch):
    """Task kernel: both ways to the factors - the per-group store and the
    in-sweep computation - give the oracle's sweep, and each other's bit for
    bit. Wave kernel (one block per ordinate): the oracle's sweep too, the
    same bits on every run, and the task kernel's result to rounding."""
    from ubolt_b200 import _lib
    mesh, g, q, st, ss = build(case)
    ctx, keep = ctx_for(g, q, st, ss)
    sw = T.Sweep(ctx, patch)
    sw.set_kernel("tasks")
    op = O.Operator(g, q, st, ss)
    qv = np.random.default_rng(1).standard_normal(op.n)
    ref = op.sweep(qv)
    runs = [sw.apply(dev(qv)) for _ in range(3)]  # the sentinel fill makes each launch independent
    psi = runs[-1]
    assert all(torch.equal(r, psi) for r in runs)  # and the result does not depend on timing
    info = sw.status()
    assert info["timeouts"] == 0 and info["n_lagged"] == 0 and info["factor_bytes"] > 0
    assert info["kernel"] == _lib.SWEEP_TASKS
    assert np.abs(psi.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    psi32 = sw.apply(dev(qv, torch.float32))
    assert np.abs(psi32.double().cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    sw.set_factor_limit(0)
    assert sw.status()["factor_bytes"] == 0
    assert torch.equal(sw.apply(dev(qv)), psi)
    assert torch.equal(sw.apply(dev(qv, torch.float32)), psi32)

    sw.set_factor_limit(-1)
    sw.set_kernel("wave")
    waves = [sw.apply(dev(qv)) for _ in range(3)]
    info = sw.status()
    assert info["kernel"] == _lib.SWEEP_WAVE and info["timeouts"] == 0 and info["factor_bytes"] > 0
    assert all(torch.equal(r, waves[0]) for r in waves)
    assert np.abs(waves[0].cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    assert float((waves[0] - psi).abs().max()) <= 1e-13 * float(psi.abs().max())
    wave32 = sw.apply(dev(qv, torch.float32))
    assert np.abs(wave32.double().cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    ctx.close()


def test_named_triangle_mesh_sweep_kernels_agree():
    """256 x 256 jittered quads split into triangles, DG1, S8 (the plain FP64
    workload): the wave kernel and the task kernel give the same sweep to
    rounding, in FP64 and in FP32. Its 40 ordinates do not fill the device,
    so the automatic choice is the task kernel."""
    from ubolt_b200 import _lib
    prob = P.config_tri256()
    g, q = prob.geometry, prob.quad
    ctx, keep = ctx_for(g, q, prob.sigma_t[0], prob.sigma_s[0, 0])
    sw = T.Sweep(ctx)
    assert sw.status()["kernel"] == _lib.SWEEP_TASKS
    sw.set_kernel("wave")
    assert sw.status()["kernel"] == _lib.SWEEP_WAVE
    qv = dev(np.random.default_rng(12).uniform(0.0, 1.0, ctx.n_rows))
    wave64 = sw.apply(qv)
    wave32 = sw.apply(qv.float())
    assert sw.status()["timeouts"] == 0
    sw.set_kernel("tasks")
    task64 = sw.apply(qv)
    task32 = sw.apply(qv.float())
    scale = float(task64.abs().max())
    assert float((wave64 - task64).abs().max()) <= 1e-13 * scale
    assert float((wave32 - task32).abs().max()) <= 1e-5 * scale
    assert float((wave32.double() - wave64).abs().max()) <= 1e-5 * scale
    ctx.close()


def test_sweep_factor_store_follows_the_group():
    """set_group with new cross sections: the stored factors are rebuilt."""
    mesh, g, q, st, ss = build(CASES[0])
    ctx, keep = ctx_for(g, q, st, ss)
    sw = T.Sweep(ctx, 0)
    qv = np.random.default_rng(2).standard_normal(g.n_cells * g.n_basis * q.n_angles)
    sw.apply(dev(qv))
    st2 = st * 1.7
    keep2 = (dev(st2), dev(ss))
    ctx.set_group(*keep2)
    psi = sw.apply(dev(qv)).cpu().numpy()
    ref = O.Operator(g, q, st2, ss).sweep(qv)
    assert np.abs(psi - ref).max() <= 1e-12 * np.abs(ref).max()
    ctx.close()


def test_sweep_and_solve_allocate_nothing_once_set_up():
    """Once the solver and the sweep plan are set up (the factor stores are
    reserved then), a new group, its sweeps and its solves allocate no device
    memory: the stores are rebuilt by a kernel, the workspace is reused
    (the reference's rule for the group sweep, AGENTS.md:46-47)."""
    mesh, g, q, st, ss = build(CASES[0])
    ctx, keep = ctx_for(g, q, st, ss)
    solver = T.TransportSolver(ctx, rtol=1e-10, pc="sweep")
    sw = T.Sweep.__new__(T.Sweep)
    sw.ctx = ctx
    assert sw.status()["factor_bytes"] > 0
    rng = np.random.default_rng(9)
    b = dev(rng.uniform(0.1, 1.0, ctx.n_rows))
    x = ctx.vector(fill=0.0)
    qv, psi = dev(rng.standard_normal(ctx.n_rows)), ctx.vector()
    keep2 = (dev(st * 1.3), dev(ss * 0.7))
    solver.solve(b, x)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    ctx.set_group(*keep2)
    sw.apply(qv, psi)
    x, stats = solver.solve(b, x)
    torch.cuda.synchronize()
    assert stats["converged"]
    assert torch.cuda.mem_get_info()[0] == free0
    ctx.close()


def test_sweep_on_tets_inverts_what_it_does_not_lag():
    rng = np.random.default_rng(4)
    mesh = P.box_tets(3, 3, 3, jitter=0.25, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(3, 4)
    st = rng.uniform(0.5, 2.0, g.n_cells)
    ctx, keep = ctx_for(g, q, st, np.zeros(g.n_cells))
    sw = T.Sweep(ctx, 24)
    op = O.Operator(g, q, st, np.zeros(g.n_cells))
    qv = rng.standard_normal(op.n)
    psi = sw.apply(dev(qv)).cpu().numpy()
    info = sw.status()
    res = np.abs(op.L @ psi - qv).reshape(g.n_cells, g.n_basis, q.n_angles).max(axis=1)
    assert (res > 1e-11 * np.abs(qv).max()).sum() <= info["n_lagged"]
    ctx.close()


def oracle_solution(g, q, st, ss, src, side=None, rtol=1e-13):
    op = O.Operator(g, q, st, ss)
    b = O.rhs(g, q, src, side)
    x, it, res = op.solve(b, rtol=rtol, max_it=3000, restart=40)
    assert it > 0 and res <= rtol * 1.01, (it, res)
    return op, b, x


def scalar_flux(x, g, q):
    return O.angular_integral(x, g.n_cells * g.n_basis, q)


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_fp64_solve_matches_oracle(case):
    mesh, g, q, st, ss = build(case)
    src = np.random.default_rng(6).uniform(0.0, 1.0, g.n_cells)
    op, b, xr = oracle_solution(g, q, st, ss, src)
    ctx, keep = ctx_for(g, q, st, ss)
    solver = T.TransportSolver(ctx, rtol=1e-13, precision="fp64", pc="sweep", max_it=2000)
    x, stats = solver.solve(dev(b))
    assert stats["converged"] and stats["residual"] <= 1.01e-13
    phi, phi_r = scalar_flux(x.cpu().numpy(), g, q), scalar_flux(xr, g, q)
    assert np.linalg.norm(phi - phi_r) <= 1e-10 * np.linalg.norm(phi_r)
    ctx.close()


@pytest.mark.parametrize("case", CASES[:6], ids=case_ids()[:6])
def test_mixed_solve_reaches_fp64_accuracy(case):
    mesh, g, q, st, ss = build(case)
    src = np.random.default_rng(6).uniform(0.0, 1.0, g.n_cells)
    op, b, xr = oracle_solution(g, q, st, ss, src)
    ctx, keep = ctx_for(g, q, st, ss)
    solver = T.TransportSolver(ctx, rtol=1e-8, precision="mixed", pc="sweep", max_it=2000)
    x, stats = solver.solve(dev(b))
    assert stats["converged"] and stats["residual"] <= 1.01e-8
    phi, phi_r = scalar_flux(x.cpu().numpy(), g, q), scalar_flux(xr, g, q)
    assert np.linalg.norm(phi - phi_r) <= 1e-7 * np.linalg.norm(phi_r)
    ctx.close()


@pytest.mark.parametrize("pc", ["block", "none"])
def test_other_preconditioners_converge_to_the_same_answer(pc):
    mesh, g, q, st, ss = build(CASES[0])
    src = np.ones(g.n_cells)
    op, b, xr = oracle_solution(g, q, st, ss, src)
    ctx, keep = ctx_for(g, q, st, ss)
    x, stats = T.TransportSolver(ctx, rtol=1e-12, pc=pc, max_it=3000, restart=60).solve(dev(b))
    assert stats["converged"]
    assert np.abs(x.cpu().numpy() - xr).max() <= 1e-9 * np.abs(xr).max()
    ctx.close()


@pytest.mark.parametrize("shape", ["tri", "hex", "tet"])
def test_infinite_medium(shape):
    """Every face reflective: psi = q / (W (sigma_t - sigma_s)), flat
    (transportk.kokkos.cxx:43-133; verify_plexk check 3a)."""
    rng = np.random.default_rng(8)
    if shape == "tri":
        mesh, dim = P.box_tris(5, 4, jitter=0.2, rng=rng), 2
    elif shape == "hex":
        mesh, dim = P.box_hexes(3, 3, 2), 3
    else:
        mesh, dim = P.box_tets(2, 2, 2, jitter=0.15, rng=rng), 3
    g = P.build_geometry(mesh, 1, side_bc=[1] * (2 * dim))
    q = P.lqn(dim, 4)
    nc = g.n_cells
    st, ss, src = np.full(nc, 2.0), np.full(nc, 1.5), np.full(nc, 3.0)
    ctx, keep = ctx_for(g, q, st, ss)
    b = torch.zeros(nc * g.n_basis * q.n_angles, dtype=torch.float64, device="cuda")
    T.GroupTransfer(ctx, [[keep[1]]], [dev(src)]).add_external(0, b)
    x, stats = T.TransportSolver(ctx, rtol=1e-12, max_it=3000).solve(b)
    want = 3.0 / (q.sum_weights * (2.0 - 1.5))
    xx = x.cpu().numpy().reshape(nc, g.n_basis, q.n_angles)
    assert np.abs(xx[:, 0, :] - want).max() <= 1e-9 * want
    assert np.abs(xx[:, 1:, :]).max() <= 1e-9 * want
    ctx.close()


def test_constant_inflow_solve():
    """Inflow psi_in on every face and source sigma_t psi_in with scattering:
    psi = psi_in (verify_plexk check 8c, solved rather than applied)."""
    rng = np.random.default_rng(9)
    mesh = P.box_tris(6, 6, jitter=0.2, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, 4)
    nc = g.n_cells
    st = rng.uniform(0.5, 2.0, nc)
    ss = st * rng.uniform(0.2, 0.9, nc)
    psi_in = 0.8
    W = q.sum_weights
    ctx, keep = ctx_for(g, q, st, ss)
    b = torch.zeros(nc * 3 * q.n_angles, dtype=torch.float64, device="cuda")
    T.fill_inflow(ctx, [psi_in * W] * 4, b)
    T.GroupTransfer(ctx, [[keep[1]]], [dev((st - ss) * psi_in * W)]).add_external(0, b)
    x, stats = T.TransportSolver(ctx, rtol=1e-12).solve(b)
    xx = x.cpu().numpy().reshape(nc, 3, q.n_angles)
    assert np.abs(xx[:, 0, :] - psi_in).max() <= 1e-9
    assert np.abs(xx[:, 1:, :]).max() <= 1e-9
    ctx.close()


def test_multigroup_downscatter_sweep_matches_oracle():
    """Four groups, lower-triangular transfer (the 128^3 hex workload's
    construction on an 8^3 box): per group the GPU solve against the oracle's,
    with the transfer source built from the previous groups' scalar fluxes."""
    prob = P.config_hex128(scale=1.0 / 16.0, sn=4)
    g, q = prob.geometry, prob.quad
    ctx = T.Context(g, q)
    phis, stats = T.solve_groups(ctx, prob.sigma_t, prob.sigma_s, prob.source, rtol=1e-12, max_it=2000)
    nodes = g.n_cells * g.n_basis
    phi_ref = []
    for gg in range(prob.n_groups):
        op = O.Operator(g, q, prob.sigma_t[gg], prob.sigma_s[gg, gg])
        b = O.rhs(g, q, prob.source[gg])
        for h in range(gg):
            if np.any(prob.sigma_s[h, gg]):
                O.add_transfer(b, phi_ref[h], prob.sigma_s[h, gg], g.n_cells, g.n_basis, q)
        x, it, res = op.solve(b, rtol=1e-12, max_it=2000)
        phi_ref.append(O.angular_integral(x, nodes, q))
    for gg in range(prob.n_groups):
        assert stats[gg]["converged"]
        got = phis[gg].cpu().numpy()
        assert np.linalg.norm(got - phi_ref[gg]) <= 1e-10 * np.linalg.norm(phi_ref[gg]), gg
    ctx.close()


def test_plain_cpu_workload_sweep_dsa_solve_matches_the_fd_oracle():
    """The reference's plain CPU case at its full size: 64 x 64 unit-square
    cells, S4, sigma_t 1, sigma_s 0.5, unit source in the central 16 x 16
    cells, vacuum, rtol 1e-10 - on the GPU as DG0 on the uniform quad box
    (the structured FD stencil's twin) with the sweep + DSA preconditioner,
    against the oracle's structured FD operator solved directly."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    prob = P.config_fd64()
    g, q = prob.geometry, prob.quad
    n = prob.meta["n"]
    A = q.n_angles
    st, ss, src = prob.sigma_t[0], prob.sigma_s[0, 0], prob.source[0]
    og = O.own_geometry(g)
    cen = og.centroid.reshape(-1, 3)
    natural = (np.floor(cen[:, 1] * n).astype(int) * n + np.floor(cen[:, 0] * n).astype(int))
    inv = np.empty_like(natural)
    inv[natural] = np.arange(g.n_cells)
    L = O.fd2d(n, n, q, st[inv])
    oq = O.own_quadrature(q)
    S = sp.kron(sp.diags(ss[inv]), np.outer(np.ones(A), oq.w / oq.sum_weights), format="csr")
    b_nat = np.repeat(src[inv] / oq.sum_weights, A)
    x_nat = spla.spsolve((L - S).tocsc(), b_nat)
    phi_ref = (x_nat.reshape(-1, A) @ oq.w)[natural]
    ctx, keep = ctx_for(g, q, st, ss)
    dsa = T.DSAPrecon(ctx)
    dsa.set_group()
    b = ctx.vector(fill=0.0)
    T.GroupTransfer(ctx, [[keep[1]]], [dev(src)]).add_external(0, b)
    x, stats = T.TransportSolver(ctx, rtol=prob.rtol, pc="sweep+dsa", max_it=500).solve(b)
    assert stats["converged"] and stats["residual"] <= prob.rtol * 1.01
    phi = T.angular_integral(ctx, x).cpu().numpy()
    assert np.linalg.norm(phi - phi_ref) <= 1e-9 * np.linalg.norm(phi_ref)
    ctx.close()


@pytest.mark.parametrize("kernel", ["tasks", "wave"])
def test_sweep_wait_that_runs_out_is_reported_and_recovers(kernel):
    """A sweep whose one wait can never be met, with a short limit - the task
    kernel polls a value nothing stores, the wave kernel waits for a level's
    copy that is never issued: the sweep still completes, the host reads
    UBOLT_ERR_TIMEOUT, and the next sweep on the same context is exact again."""
    from ubolt_b200 import _lib
    mesh, g, q, st, ss = build(CASES[0])
    ctx, keep = ctx_for(g, q, st, ss)
    sw = T.Sweep(ctx, 16)
    sw.set_kernel(kernel)
    op = O.Operator(g, q, st, ss)
    qv = np.random.default_rng(1).standard_normal(op.n)
    _lib.check(_lib.lib.ubolt_sweep_test_wait(ctx.handle, 2000, 1))
    sw.apply(dev(qv))
    with pytest.raises(_lib.UboltError) as e:
        sw.status()
    assert e.value.status == 6  # UBOLT_ERR_TIMEOUT
    _lib.check(_lib.lib.ubolt_sweep_test_wait(ctx.handle, 1 << 22, 0))
    psi = sw.apply(dev(qv)).cpu().numpy()
    assert sw.status()["timeouts"] == 0
    ref = op.sweep(qv)
    assert np.abs(psi - ref).max() <= 1e-12 * np.abs(ref).max()
    ctx.close()


VACUUM = [c for c in CASES if c[0].endswith("_vac") and not c[0].startswith("tet")]


@pytest.mark.parametrize("case", VACUUM, ids=[c[0] for c in VACUUM])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kernel", ["auto", "tasks"])
def test_compressed_krylov_matches_full_basis(case, precision, kernel):
    """Exact sweep, no reflective side: the compressed basis (node-space
    vectors plus one scalar each) gives the plain form's answer, in about
    the same iterations, for the forward and the adjoint system (an
    anisotropic and an isotropic adjoint source). With the task kernel the
    kept sweep outputs are ordinate-major (the scatter, the update and the
    adjoint's permutation on that layout); these small meshes otherwise
    take the wave kernel and the row layout."""
    mesh, g, q, st, ss = build(case)
    rng = np.random.default_rng(11)
    src = rng.uniform(0.0, 1.0, g.n_cells)
    op, b, xr = oracle_solution(g, q, st, ss, src)
    ctx, keep = ctx_for(g, q, st, ss)
    if kernel == "tasks":
        T.Sweep(ctx, 0).set_kernel("tasks")
    rtol = 1e-11 if precision == "fp64" else 1e-8
    auto = T.TransportSolver(ctx, rtol=rtol, precision=precision, pc="sweep", max_it=2000)
    x1, s1 = auto.solve(dev(b))
    full = T.TransportSolver(ctx, rtol=rtol, precision=precision, pc="sweep", max_it=2000, krylov="full")
    x2, s2 = full.solve(dev(b))
    assert s1["krylov"] == 2 and s2["krylov"] == 1
    assert s1["converged"] and s2["converged"] and s1["residual"] <= rtol * 1.01
    assert abs(s1["iterations"] - s2["iterations"]) <= 1 + s2["iterations"] // 10
    phi1, phi_r = scalar_flux(x1.cpu().numpy(), g, q), scalar_flux(xr, g, q)
    assert np.linalg.norm(phi1 - phi_r) <= 10 * rtol * np.linalg.norm(phi_r)
    # the adjoint: anisotropic source, the weighted isotropic subspace
    gsrc = rng.standard_normal(op.n)
    l1, a1 = auto.solve_adjoint(dev(gsrc))
    l2, a2 = full.solve_adjoint(dev(gsrc))
    assert a1["krylov"] == 2 and a1["converged"] and a2["converged"]
    lam1, lam2 = l1.cpu().numpy(), l2.cpu().numpy()
    assert np.linalg.norm(lam1 - lam2) <= 20 * rtol * np.linalg.norm(lam2)
    assert np.linalg.norm(op.matrix().T @ lam1 - gsrc) <= 1.01 * rtol * np.linalg.norm(gsrc)
    nn = g.n_cells * g.n_basis
    giso = np.repeat(rng.standard_normal(nn), q.n_angles) * np.tile(q.w, nn)
    l3, a3 = auto.solve_adjoint(dev(giso))
    l4, a4 = full.solve_adjoint(dev(giso))
    assert a3["krylov"] == 2 and a3["converged"] and a4["converged"]
    lam3, lam4 = l3.cpu().numpy(), l4.cpu().numpy()
    assert np.linalg.norm(lam3 - lam4) <= 20 * rtol * np.linalg.norm(lam4)
    assert np.linalg.norm(op.matrix().T @ lam3 - giso) <= 1.01 * rtol * np.linalg.norm(giso)
    ctx.close()


def test_compressed_krylov_is_not_used_where_the_sweep_lags():
    case = [c for c in CASES if c[0] == "tri_dg1_refl"][0]
    mesh, g, q, st, ss = build(case)
    src = np.random.default_rng(6).uniform(0.0, 1.0, g.n_cells)
    op, b, xr = oracle_solution(g, q, st, ss, src)
    ctx, keep = ctx_for(g, q, st, ss)
    x, stats = T.TransportSolver(ctx, rtol=1e-10, pc="sweep").solve(dev(b))
    assert stats["krylov"] == 1 and stats["converged"]
    ctx.close()


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_host_batch_matches_device_solves(pinned):
    """ubolt_solve_host_batch: right-hand sides in host memory, copies on
    their own streams around the solves; each x is the device solve's."""
    mesh, g, q, st, ss = build(CASES[0])
    ctx, keep = ctx_for(g, q, st, ss)
    rng = np.random.default_rng(8)
    bs = [torch.tensor(rng.uniform(0.1, 1.0, ctx.n_rows)) for _ in range(5)]
    if pinned:
        bs = [b.pin_memory() for b in bs]
    xs = [torch.zeros(ctx.n_rows, dtype=torch.float64) for _ in range(5)]
    if pinned:
        xs = [x.pin_memory() for x in xs]
    solver = T.TransportSolver(ctx, rtol=1e-10)
    stats = solver.solve_host_batch(bs, xs)
    torch.cuda.current_stream().synchronize()
    assert len(stats) == 5 and all(s["converged"] for s in stats)
    for b, x in zip(bs, xs):
        ref, _ = solver.solve(b.cuda())
        assert (x - ref.cpu()).abs().max().item() <= 1e-13 * ref.abs().max().item()
    ctx.close()


def test_upscatter_outer_iteration_matches_the_coupled_solve():
    """Three groups on jittered triangles, DG1, S4, with upscatter 2 -> 1 (a
    thermal block of groups 1 and 2): the outer iteration of the reference's
    group loop (block Gauss-Seidel, warm starts, adaptive inner tolerance,
    stop on the error estimate) against a direct solve of the fully coupled
    system A_g psi_g - sum_{h != g} T_{h->g} psi_h = b_g assembled on the CPU
    from the oracle's operators."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    rng = np.random.default_rng(21)
    mesh = P.box_tris(6, 5, jitter=0.2, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, 4)
    nc, nb, na = g.n_cells, g.n_basis, q.n_angles
    G = 3
    st = rng.uniform(0.8, 2.0, (G, nc))
    ss = np.zeros((G, G, nc))
    for gg in range(G):
        ss[gg, gg] = 0.5 * st[gg]
    ss[0, 1], ss[0, 2], ss[1, 2] = 0.2 * st[0], 0.1 * st[0], 0.25 * st[1]
    ss[2, 1] = 0.3 * st[2]  # upscatter
    src = np.zeros((G, nc))
    src[0] = rng.uniform(0.5, 1.0, nc)
    src[2] = 0.2

    n = nc * nb * na
    E = sp.kron(sp.identity(nc * nb), np.ones((na, 1)))          # node -> every angle
    Rw = sp.kron(sp.identity(nc * nb), q.w.reshape(1, na))       # angles -> weighted node sum
    blocks = [[None] * G for _ in range(G)]
    bs = []
    for gg in range(G):
        blocks[gg][gg] = O.Operator(g, q, st[gg], ss[gg, gg]).matrix()
        bs.append(O.rhs(g, q, src[gg]))
        for h in range(G):
            if h != gg and np.any(ss[h, gg]):
                scale = sp.diags(np.repeat(ss[h, gg], nb) / q.sum_weights)
                blocks[gg][h] = -(E @ scale @ Rw)
    M = sp.bmat(blocks, format="csc")
    psi_ref = spla.spsolve(M, np.concatenate(bs)).reshape(G, n)
    phi_ref = [O.angular_integral(psi_ref[gg], nc * nb, q) for gg in range(G)]

    ctx = T.Context(g, q)
    # The angular store, and the moments store with and without the
    # reconstruction steps: the same coupled solution
    for store, recon in (("angular", "tol"), ("moments", "tol"), ("moments", "none")):
        info = {}
        phis, stats = T.solve_groups(ctx, st, ss, src, rtol=1e-12, max_it=2000, outer_rtol=1e-10,
                                     outer_store=store, outer_recon=recon, outer_info=info)
        assert info["upscatter"] and info["g_up"] == 1 and info["converged"] and info["outer_iterations"] >= 3
        assert info["error_estimate"] < 1e-10
        if store == "moments":
            assert info["reconstructed_solves"] > 0
            assert (info["reconstruction_steps"] > 0) == (recon == "tol")
        for gg in range(G):
            err = np.linalg.norm(phis[gg].cpu().numpy() - phi_ref[gg]) / np.linalg.norm(phi_ref[gg])
            assert err <= 1e-9, (store, recon, gg, err)
    # An outer tolerance below the inner one is refused, as the reference does
    with pytest.raises(Exception):
        T.solve_groups(ctx, st, ss, src, rtol=1e-8, outer_rtol=1e-10)
    ctx.close()


@pytest.mark.parametrize("case", [c for c in CASES if c[0] in ("tri_dg1_refl", "hex_dg1_refl")],
                         ids=["tri_dg1_refl", "hex_dg1_refl"])
def test_current_and_p1_expansion_round_trip(case):
    """A P1 field psi = phi / W + Omega . c: its scalar flux and current are
    phi and T c (T = sum_a w_a Omega_a Omega_a^T), and the expansion of those
    moments gives psi back; the current of any psi matches its definition."""
    mesh, g, q, st, ss = build(case)
    ctx, keep = ctx_for(g, q, st, ss)
    nn, A, D = g.n_cells * g.n_basis, q.n_angles, g.dim
    rng = np.random.default_rng(13)
    phi = rng.uniform(0.5, 1.5, nn)
    c = rng.standard_normal((nn, D))
    om = q.omega[:, :D]
    psi = phi[:, None] / q.sum_weights + c @ om.T                 # (nn, A)
    Tm = (q.w[:, None, None] * om[:, :, None] * om[:, None, :]).sum(axis=0)
    J = T.current(ctx, dev(psi.ravel()))
    assert np.abs(J.cpu().numpy() - c @ Tm.T).max() <= 1e-12 * np.abs(c @ Tm.T).max()
    back = T.expand_p1(ctx, dev(phi), J)
    assert np.abs(back.cpu().numpy() - psi.ravel()).max() <= 1e-12 * np.abs(psi).max()
    x = rng.standard_normal(nn * A)
    Jx = T.current(ctx, dev(x)).cpu().numpy()
    assert np.abs(Jx - (x.reshape(nn, A) * q.w) @ om).max() <= 1e-12 * np.abs(x).max() * q.sum_weights
    ctx.close()


def test_sweep_kernel_choice_is_checked():
    """An unknown kernel id is an argument error; the wave kernel where an
    ordinate's upwind graph has a cycle (jittered tets) is a state error, and
    the task kernel keeps running there."""
    from ubolt_b200 import _lib
    rng = np.random.default_rng(4)
    mesh = P.box_tets(3, 3, 3, jitter=0.25, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(3, 4)
    st = rng.uniform(0.5, 2.0, g.n_cells)
    ctx, keep = ctx_for(g, q, st, np.zeros(g.n_cells))
    sw = T.Sweep(ctx)
    with pytest.raises(_lib.UboltError) as e:
        _lib.check(_lib.lib.ubolt_sweep_set_kernel(ctx.handle, 7))
    assert e.value.status == 1
    if not _lib.wave_plan(g, q)["acyclic"]:
        with pytest.raises(_lib.UboltError) as e:
            sw.set_kernel("wave")
        assert e.value.status == 4
    sw.set_kernel("tasks")
    psi = sw.apply(dev(rng.standard_normal(ctx.n_rows)))
    assert torch.isfinite(psi).all() and sw.status()["kernel"] == _lib.SWEEP_TASKS
    ctx.close()


@pytest.mark.parametrize("case", [c for c in ACYCLIC if c[0].startswith(("tri", "hex"))][:4],
                         ids=[c[0] for c in ACYCLIC if c[0].startswith(("tri", "hex"))][:4])
def test_isotropic_sweep_in_both_layouts(case):
    """ubolt_sweep_iso: L^{-1} of an isotropic source u_a phi(node) is the
    sweep of the expanded source, in UBOLT's row layout and ordinate-major
    (the layout the compressed GMRES keeps), FP64 bit for bit, FP32 to its
    rounding; the oracle's sweep of the same source to 1e-12."""
    mesh, g, q, st, ss = build(case)
    ctx, keep = ctx_for(g, q, st, ss)
    try:
        sw = T.Sweep(ctx, 0)
        sw.set_kernel("tasks")
        nn, A, nc, nb = ctx.n_nodes, q.n_angles, g.n_cells, g.n_basis
        rng = np.random.default_rng(5)
        phi = rng.standard_normal(nn)
        u = rng.uniform(0.5, 1.5, A)
        full = (phi[:, None] * u[None, :]).ravel()
        ref = O.Operator(g, q, st, ss).sweep(full)
        plain = sw.apply(dev(full))
        row = sw.apply_iso(dev(phi), torch.empty_like(plain), u=dev(u))
        om = sw.apply_iso(dev(phi), torch.empty_like(plain), u=dev(u), ordinate_major=True)
        assert torch.equal(row, plain)
        assert torch.equal(om.view(A, nc, nb).permute(1, 2, 0).reshape(-1), plain)
        assert np.abs(plain.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
        om32 = sw.apply_iso(dev(phi), torch.empty(ctx.n_rows, dtype=torch.float32, device="cuda"),
                            u=dev(u, torch.float32), ordinate_major=True)
        r32 = om32.view(A, nc, nb).permute(1, 2, 0).reshape(-1).double().cpu().numpy()
        assert np.abs(r32 - ref).max() <= 1e-4 * np.abs(ref).max()
        assert sw.status()["timeouts"] == 0
    finally:
        ctx.close()
