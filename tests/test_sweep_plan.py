"""The sweep plan, on the CPU: every task's cells belong to its patch and come
in level order, every gathered upwind value comes from an earlier level of
the same task or from a lower-numbered upstream task (which is what makes
the persistent GPU sweep deadlock-free), every cell is solved exactly once
per ordinate, and executing the plan in task order is the exact upwind sweep
L^{-1} wherever the upwind graph is acyclic."""
import numpy as np
import pytest

import oracle as O
from ubolt_b200 import _lib
from ubolt_b200 import problem as P

from _cases import CASES, build, case_ids


def check_plan_invariants(plan, g, q):
    nc, F, A = g.n_cells, g.faces_per_cell, q.n_angles
    Pz = plan["patch_size"]
    nbr = g.face_neighbour.reshape(nc, F)
    nA = g.face_nA.reshape(nc, F, 3)
    solved_by = np.full((A, nc), -1, dtype=np.int64)
    level_of = np.full((A, nc), -1, dtype=np.int64)
    for t in range(plan["n_tasks"]):
        p, a = divmod(int(plan["task_pa"][t]), A)
        base = p * Pz
        c0, c1 = plan["cell_ptr"][t], plan["cell_ptr"][t + 1]
        cells = base + plan["tcell"][c0:c1].astype(np.int64)
        assert np.all(cells < min(nc, base + Pz))
        assert np.all(solved_by[a, cells] == -1), "a cell solved twice for one ordinate"
        solved_by[a, cells] = t
        ends = plan["lvl"][plan["lvl_ptr"][t]:plan["lvl_ptr"][t + 1]]
        assert ends[-1] == c1 - c0 and np.all(np.diff(ends) > 0)
        lo = 0
        for l, hi in enumerate(ends):
            level_of[a, cells[lo:hi]] = l
            lo = hi
        deps = plan["deps"][plan["dep_ptr"][t]:plan["dep_ptr"][t + 1]]
        assert np.all(deps < t), "an upstream task is numbered after its consumer"
        depset = set(deps.tolist())
        for i, c in enumerate(cells):
            m = int(plan["tmask"][c0 + i])
            for f in range(F):
                here, earlier = (m >> f) & 1, (m >> (8 + f)) & 1
                o, n = q.omega[a], nA[c, f]
                s = float(o[0]) * float(n[0]) + float(o[1]) * float(n[1]) + float(o[2]) * float(n[2])
                if nbr[c, f] >= 0 and s < 0:
                    assert here or earlier or plan["n_lagged"] > 0, "an upwind coupling dropped"
                if not (here or earlier):
                    continue
                up = nbr[c, f]
                assert up >= 0 and s < 0
                if here:
                    assert solved_by[a, up] == t and level_of[a, up] < level_of[a, c]
                else:
                    assert solved_by[a, up] in depset
    assert np.all(solved_by >= 0), "a cell never solved"


def simulate(plan, op, g, q_vec, A):
    """Execute the plan on the CPU in task order, each (cell, ordinate)
    block solved from the assembled CSR with the gathered upwind values."""
    nc, nb, F = g.n_cells, g.n_basis, g.faces_per_cell
    L = op.L
    psi = np.zeros(op.n)
    Pz = plan["patch_size"]
    nbr = g.face_neighbour.reshape(nc, F)
    for t in range(plan["n_tasks"]):
        p, a = divmod(int(plan["task_pa"][t]), A)
        base = p * Pz
        for i in range(plan["cell_ptr"][t], plan["cell_ptr"][t + 1]):
            c = base + int(plan["tcell"][i])
            m = int(plan["tmask"][i])
            ups = {nbr[c, f] for f in range(F) if ((m >> f) | (m >> (8 + f))) & 1}
            rows = [(c * nb + ii) * A + a for ii in range(nb)]
            B = np.zeros((nb, nb))
            r = q_vec[rows].copy()
            for k, row in enumerate(rows):
                cols = L.indices[L.indptr[row]:L.indptr[row + 1]]
                vals = L.data[L.indptr[row]:L.indptr[row + 1]]
                for col, v in zip(cols, vals):
                    cc, rem = divmod(int(col), nb * A)
                    jj, aa = divmod(rem, A)
                    if cc == c and aa == a:
                        B[k, jj] = v
                    elif aa == a and cc in ups:
                        r[k] -= v * psi[col]
            psi[rows] = np.linalg.solve(B, r)
    return psi


@pytest.mark.parametrize("case", CASES, ids=case_ids())
def test_plan_invariants(case):
    mesh, g, q, st, ss = build(case)
    for P_ in (0, 7, 32):
        plan = _lib.sweep_plan(g, q, P_)
        check_plan_invariants(plan, g, q)


@pytest.mark.parametrize("case", [c for c in CASES if c[1] == 2 or c[0].startswith("hex")],
                         ids=[c[0] for c in CASES if c[1] == 2 or c[0].startswith("hex")])
def test_plan_executes_the_exact_sweep(case):
    """2D and hex meshes have acyclic upwind graphs: nothing is lagged, and with
    vacuum faces the plan's sweep is L^{-1} - the oracle's sweep, to rounding;
    with reflective faces both lag the mirrored inflow to zero."""
    mesh, g, q, st, ss = build(case)
    op = O.Operator(g, q, st, ss)
    for P_ in (16, 0):
        plan = _lib.sweep_plan(g, q, P_)
        assert plan["n_lagged"] == 0
        rng = np.random.default_rng(2)
        qv = rng.standard_normal(op.n)
        psi = simulate(plan, op, g, qv, q.n_angles)
        ref = op.sweep(qv)
        assert np.abs(psi - ref).max() <= 1e-12 * np.abs(ref).max()
        if not np.any(g.face_bc == _lib.BC_REFLECT):
            assert np.abs(op.L @ psi - qv).max() <= 1e-11 * np.abs(qv).max()


def test_tet_plan_lags_only_what_cycles():
    """Jittered tets can have upwind cycles; whatever the plan lags, L psi = q
    holds on every row except those of cells that lag a coupling."""
    rng = np.random.default_rng(4)
    mesh = P.box_tets(3, 3, 3, jitter=0.25, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(3, 4)
    st = rng.uniform(0.5, 2.0, g.n_cells)
    op = O.Operator(g, q, st, np.zeros(g.n_cells))
    plan = _lib.sweep_plan(g, q, 24)
    check_plan_invariants(plan, g, q)
    qv = rng.standard_normal(op.n)
    psi = simulate(plan, op, g, qv, q.n_angles)
    res = np.abs(op.L @ psi - qv).reshape(g.n_cells, g.n_basis, q.n_angles)
    bad = (res.max(axis=1) > 1e-11 * np.abs(qv).max()).sum()
    assert bad <= plan["n_lagged"]
