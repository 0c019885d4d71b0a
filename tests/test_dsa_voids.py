"""The DSA's void policy (DSAPrecon::assemble, src/dsak.kokkos.cxx:233-345).

The oracle is held to the reference's own checks 12 and 13
(tests/verify_plexk.kokkos.cxx:68-83):
- a masked void box against the box cut off at the void;
- a void slab that is bridged: its chord, a symmetric positive definite
  matrix, constants mapped to V sigma_a, and coupling through the void.

Then the CUDA path is held to the oracle through the C ABI (-m gpu): the
matrix, the policy's outcome, R and P with the mask, the converged apply and
a solve through a void."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle as O
from ubolt_b200 import problem as P

from _cases import CASES


def _xs(g, void_x=None, void_band=None):
    """Smooth cross sections by position; cells whose centroid x is past
    void_x, or inside void_band = (x0, x1), are void (sigma_t = sigma_s = 0)."""
    cen = g.centroid.reshape(g.n_cells, 3)
    st = 1.0 + 0.5 * np.sin(3.0 * cen[:, 0] + 2.0 * cen[:, 1] + cen[:, 2])
    ss = st * (0.5 + 0.3 * np.cos(2.0 * cen[:, 0] - cen[:, 1]))
    void = np.zeros(g.n_cells, dtype=bool)
    if void_x is not None:
        void |= cen[:, 0] > void_x
    if void_band is not None:
        void |= (cen[:, 0] > void_band[0]) & (cen[:, 0] < void_band[1])
    st[void], ss[void] = 0.0, 0.0
    return st, ss, void


def _keys(g, h):
    """Per cell its (i, j, k) position on a box of spacing h."""
    cen = g.centroid.reshape(g.n_cells, 3)
    return [tuple(int(v) for v in np.floor(c[:g.dim] / h)) for c in cen]


def _box(dim, order, n, h, side_bc=None):
    if dim == 2:
        mesh = P.box_quads(n[0], n[1], lx=n[0] * h, ly=n[1] * h)
    else:
        mesh = P.box_hexes(n[0], n[1], n[2], lx=n[0] * h, ly=n[1] * h, lz=n[2] * h)
    return P.build_geometry(mesh, order, side_bc=side_bc), P.lqn(dim, 4)


@pytest.mark.parametrize("dim,order", [(2, 0), (2, 1), (3, 0), (3, 1)])
def test_masked_void_is_the_box_cut_off_at_the_void(dim, order):
    """Check 12: with bridging off, the rows of the non-void cells are the
    cut box's (a face into the void is a vacuum face), the void rows are V
    times the identity, and P D^-1 R agrees on the non-void nodes and is zero
    on the void."""
    h = 0.125
    n_full = [8, 4, 3][:dim]
    n_cut = [5, 4, 3][:dim]
    gf, q = _box(dim, order, n_full, h)
    gc, _ = _box(dim, order, n_cut, h)
    stf, ssf, void = _xs(gf, void_x=n_cut[0] * h)
    stc, ssc, _ = _xs(gc)
    pol = O.VoidPolicy(gf, stf, ssf, bridge=False)
    assert pol.n_void == void.sum() and not pol.bridged and np.array_equal(pol.masked.astype(bool), void)
    Df = O.dsa_matrix(gf, q, stf, ssf, policy=pol).toarray()
    Dc = O.dsa_matrix(gc, q, stc, ssc).toarray()
    nb = gf.n_basis
    kf, kc = _keys(gf, h), _keys(gc, h)
    where = {k: c for c, k in enumerate(kf)}
    f_of_c = np.array([where[k] for k in kc])
    nodes_f = (f_of_c[:, None] * nb + np.arange(nb)).ravel()
    scale = np.abs(Dc).max()
    assert np.abs(Df[np.ix_(nodes_f, nodes_f)] - Dc).max() <= 1e-13 * scale
    rest = np.setdiff1d(np.arange(Df.shape[0]), nodes_f)
    assert np.abs(Df[np.ix_(nodes_f, rest)]).max() == 0.0
    void_nodes = (np.flatnonzero(void)[:, None] * nb + np.arange(nb)).ravel()
    want = np.diag(np.repeat(O.own_geometry(gf).volume[void], nb))
    assert np.array_equal(Df[np.ix_(void_nodes, void_nodes)], want)
    # P D^-1 R: x a smooth function of (position, ordinate), the same on both boxes
    A = q.n_angles

    def x_of(g, keys):
        key = np.array([sum(v * 100 ** i for i, v in enumerate(k)) for k in keys], dtype=float)
        node = (np.repeat(key, g.n_basis) * 7 + np.tile(np.arange(g.n_basis), g.n_cells))
        return (1.0 + 0.5 * np.sin(0.37 * node[:, None] + 1.3 * np.arange(A)[None, :])).ravel()

    def pdr(g, D, st, ss, x, masked):
        rhs = O.dsa_restrict(x, g, q, masked=masked)
        return O.dsa_prolong(spla.spsolve(D.tocsc() if hasattr(D, "tocsc") else D, rhs), g, q, masked=masked)

    import scipy.sparse as sp
    yf = pdr(gf, sp.csc_matrix(Df), stf, ssf, x_of(gf, kf), pol.masked).reshape(gf.n_cells, nb * A)
    yc = pdr(gc, sp.csc_matrix(Dc), stc, ssc, x_of(gc, kc), None).reshape(gc.n_cells, nb * A)
    assert np.abs(yf[f_of_c] - yc).max() <= 1e-10 * np.abs(yc).max()
    assert np.abs(yf[void]).max() == 0.0


@pytest.mark.parametrize("dim,order", [(2, 0), (2, 1), (3, 0), (3, 1)])
def test_bridged_void_slab(dim, order):
    """Check 13: a void slab across the box is bridged, counted, and its mean
    chord is 4 V / S of the slab (S: its two faces onto the material and its
    vacuum sides). The matrix is symmetric positive definite, maps a
    constant to V sigma_a on every cell off the vacuum boundary, and carries
    a residual on one side through the void to the far side (where the mask
    leaves zero)."""
    h = 0.125
    n = [9, 4, 3][:dim]
    g, q = _box(dim, order, n, h)
    st, ss, void = _xs(g, void_band=(3 * h, 6 * h))
    pol = O.VoidPolicy(g, st, ss)
    assert pol.bridged and pol.n_void == void.sum() == 3 * int(np.prod(n[1:]))
    w, H = 3 * h, n[1] * h
    if dim == 2:
        V, S = w * H, 2 * H + 2 * w
    else:
        Z = n[2] * h
        V, S = w * H * Z, 2 * H * Z + 2 * w * Z + 2 * w * H
    assert abs(pol.chord - 4 * V / S) <= 1e-12 * pol.chord
    assert np.allclose(pol.d[void], 1.0 / (3.0 / pol.chord), rtol=1e-14)
    D = O.dsa_matrix(g, q, st, ss, policy=pol)
    Dd = D.toarray()
    assert np.abs(Dd - Dd.T).max() <= 1e-12 * np.abs(Dd).max()
    assert np.linalg.eigvalsh(Dd).min() > 0
    nb = g.n_basis
    u = np.zeros((g.n_cells, nb))
    u[:, 0] = 1.0
    Du = (D @ u.ravel()).reshape(g.n_cells, nb)
    inner = np.all(g.face_neighbour.reshape(g.n_cells, -1) >= 0, axis=1)
    want = (g.volume * (st - ss))[:, None] * u
    assert inner.sum() > 0
    assert np.abs(Du[inner] - want[inner]).max() <= 1e-12 * np.abs(Du).max()
    # A residual on the low-x side only
    cen = g.centroid.reshape(g.n_cells, 3)
    rhs = np.zeros((g.n_cells, nb))
    rhs[cen[:, 0] < 3 * h, 0] = 1.0
    far = cen[:, 0] > 6 * h
    ub = spla.spsolve(D.tocsc(), rhs.ravel()).reshape(g.n_cells, nb)
    assert np.abs(ub[far]).max() > 1e-6 * np.abs(ub).max()
    polm = O.VoidPolicy(g, st, ss, bridge=False)
    Dm = O.dsa_matrix(g, q, st, ss, policy=polm)
    um = spla.spsolve(Dm.tocsc(), rhs.ravel()).reshape(g.n_cells, nb)
    assert np.abs(um[far]).max() == 0.0


def test_fixed_void_d_and_threshold():
    """-dsa_void_d fixes D in a bridged void; -dsa_void_sigma_t raises the
    threshold, so thin cells count as void."""
    g, q = _box(2, 1, [9, 4], 0.125)
    st, ss, void = _xs(g, void_band=(0.375, 0.75))
    pol = O.VoidPolicy(g, st, ss, void_d=0.7)
    assert pol.bridged and np.all(pol.d[void] == 0.7)
    thin = st < 1.2
    pol2 = O.VoidPolicy(g, st, ss, void_sigma_t=1.2)
    assert pol2.n_void == int((thin | void).sum())


def test_all_reflective_without_absorption_is_singular():
    g, q = _box(2, 0, [4, 4], 0.25, side_bc=[1, 1, 1, 1])
    st = np.full(g.n_cells, 2.0)
    assert O.VoidPolicy(g, st, st).singular
    assert not O.VoidPolicy(g, st, 0.9 * st).singular
    # A masked void is as good as a vacuum face
    st2, ss2 = st.copy(), st.copy()
    st2[0] = ss2[0] = 0.0
    assert not O.VoidPolicy(g, st2, ss2, bridge=False).singular


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# The CUDA path
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

GPU_CASES = [CASES[0], CASES[3], CASES[5], CASES[8]]


def _gpu(case, bridge, inner=30):
    import torch
    from ubolt_b200 import transport as T
    from _cases import build
    mesh, g, q, _, _ = build(case)
    lo = g.centroid.reshape(g.n_cells, 3)[:, 0].min()
    hi = g.centroid.reshape(g.n_cells, 3)[:, 0].max()
    st, ss, void = _xs(g, void_band=(lo + 0.4 * (hi - lo), lo + 0.7 * (hi - lo)))
    ctx = T.Context(g, q)
    keep = (torch.tensor(st, device="cuda"), torch.tensor(ss, device="cuda"))
    ctx.set_group(*keep)
    dsa = T.DSAPrecon(ctx, inner_iterations=inner, void_bridge=bridge)
    dsa.set_group()
    pol = O.VoidPolicy(g, st, ss, bridge=bridge)
    return ctx, keep, dsa, g, q, st, ss, void, pol


@pytest.mark.gpu
@pytest.mark.parametrize("bridge", [True, False], ids=["bridged", "masked"])
@pytest.mark.parametrize("case", GPU_CASES, ids=[c[0] for c in GPU_CASES])
def test_gpu_void_policy_matches_oracle(case, bridge):
    import torch
    ctx, keep, dsa, g, q, st, ss, void, pol = _gpu(case, bridge)
    assert void.sum() > 0
    n_void, bridged, chord = dsa.void_info()
    assert n_void == pol.n_void and bridged == pol.bridged
    assert abs(chord - pol.chord) <= 1e-14 * max(pol.chord, 1.0)
    D = O.dsa_matrix(g, q, st, ss, policy=pol)
    assert abs(dsa.matrix() - D).max() <= 1e-13 * abs(D).max()
    x = np.random.default_rng(5).standard_normal(g.n_cells * g.n_basis * q.n_angles)
    rhs = dsa.restrict(torch.tensor(x, device="cuda")).cpu().numpy()
    want = O.dsa_restrict(x, g, q, masked=pol.masked)
    assert np.abs(rhs - want).max() <= 1e-13 * np.abs(want).max()
    u = np.random.default_rng(3).standard_normal(D.shape[0])
    y = dsa.prolong(torch.tensor(u, device="cuda")).cpu().numpy()
    assert np.abs(y - O.dsa_prolong(u, g, q, masked=pol.masked)).max() <= 1e-15 * np.abs(y).max()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("bridge", [True, False], ids=["bridged", "masked"])
def test_gpu_void_apply_with_a_converged_inner_solve(bridge):
    import torch
    ctx, keep, dsa, g, q, st, ss, void, pol = _gpu(CASES[0], bridge, inner=3000)
    D = O.dsa_matrix(g, q, st, ss, policy=pol).tocsc()
    x = np.random.default_rng(7).standard_normal(g.n_cells * g.n_basis * q.n_angles)
    ref = O.dsa_prolong(spla.spsolve(D, O.dsa_restrict(x, g, q, masked=pol.masked)), g, q, masked=pol.masked)
    y = dsa.apply(torch.tensor(x, device="cuda")).cpu().numpy()
    assert np.abs(y - ref).max() <= 1e-8 * np.abs(ref).max()
    ctx.close()


@pytest.mark.gpu
def test_gpu_singular_group_is_refused():
    import torch
    from ubolt_b200 import transport as T
    from ubolt_b200._lib import UboltError
    g, q = _box(2, 0, [4, 4], 0.25, side_bc=[1, 1, 1, 1])
    st = torch.full((g.n_cells,), 2.0, dtype=torch.float64, device="cuda")
    ctx = T.Context(g, q)
    ctx.set_group(st, st)
    dsa = T.DSAPrecon(ctx)
    with pytest.raises(UboltError, match="singular"):
        dsa.set_group()
    ctx.close()


@pytest.mark.gpu
def test_gpu_solve_through_a_void_with_dsa():
    """A scattering box with a void band: the sweep + DSA solve (bridged and
    masked voids) gives the sweep-only answer."""
    import torch
    from ubolt_b200 import transport as T
    g, q = _box(2, 1, [16, 8], 1.0 / 16)
    st, ss, void = _xs(g, void_band=(0.4, 0.6))
    st[~void] *= 20.0
    ss[~void] = 0.95 * st[~void]
    ctx = T.Context(g, q)
    keep = (torch.tensor(st, device="cuda"), torch.tensor(ss, device="cuda"))
    ctx.set_group(*keep)
    src = torch.tensor((~void).astype(float), device="cuda")
    b = ctx.vector(fill=0.0)
    T.GroupTransfer(ctx, [[keep[1]]], [src]).add_external(0, b)
    x0, s0 = T.TransportSolver(ctx, rtol=1e-10, pc="sweep", max_it=2000).solve(b)
    assert s0["converged"]
    for bridge in (True, False):
        dsa = T.DSAPrecon(ctx, void_bridge=bridge)
        dsa.set_group()
        x1, s1 = T.TransportSolver(ctx, rtol=1e-10, pc="sweep+dsa", max_it=2000).solve(b)
        assert s1["converged"]
        assert (x1 - x0).abs().max().item() <= 1e-7 * x0.abs().max().item()
    ctx.close()


def test_all_void_is_masked_not_bridged():
    """Every cell void: nothing to bridge to, so the voids are masked and the
    operator is V times the identity."""
    g, q = _box(2, 1, [4, 3], 0.25)
    z = np.zeros(g.n_cells)
    pol = O.VoidPolicy(g, z, z)
    assert pol.n_void == g.n_cells and not pol.bridged and pol.masked.all() and not pol.singular
    D = O.dsa_matrix(g, q, z, z, policy=pol).toarray()
    assert np.array_equal(D, np.diag(np.repeat(g.volume, g.n_basis)))
