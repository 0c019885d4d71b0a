"""The wave plan, on the CPU: per ordinate every cell is placed once, each
level reads only cells of earlier levels, every front slot a position reads
still holds the upwind cell it wants (no later value overwrote it), and
executing the positions in order is the exact upwind sweep L^{-1} - the
oracle's - wherever the plan exists (acyclic upwind graphs)."""
import numpy as np
import pytest

import oracle as O
from ubolt_b200 import _lib
from ubolt_b200 import problem as P

from _cases import CASES, build, case_ids

NONE = 0xFFFF


def unpack(m):
    cell = int(m[0])
    out = int(m[1]) & 0xFFFF
    mask = (int(m[1]) >> 16) & 0xFFFF
    ins = [int(m[2]) & 0xFFFF, (int(m[2]) >> 16) & 0xFFFF, int(m[3]) & 0xFFFF, (int(m[3]) >> 16) & 0xFFFF]
    return cell, out, mask, ins


def check_wave_invariants(plan, g, q):
    nc, F, A = g.n_cells, g.faces_per_cell, q.n_angles
    nbr = g.face_neighbour.reshape(nc, F)
    nA = g.face_nA.reshape(nc, F, 3)
    assert plan["acyclic"]
    widths = []
    for a in range(A):
        l0, l1 = plan["lvl_base"][a], plan["lvl_base"][a + 1]
        lp = plan["lvl_pos"][l0 + a:l1 + a + 1]
        assert lp[0] == 0 and lp[-1] == nc and np.all(np.diff(lp) > 0)
        widths.append(np.diff(lp).max())
        meta = plan["meta"][a]
        cells = meta[:, 0]
        assert np.array_equal(np.sort(cells), np.arange(nc)), "a cell placed twice or never"
        level = np.empty(nc, dtype=np.int64)
        for l in range(len(lp) - 1):
            level[cells[lp[l]:lp[l + 1]]] = l
        front = {}  # slot -> cell whose psi it holds
        for l in range(len(lp) - 1):
            writes = {}
            for p in range(lp[l], lp[l + 1]):
                c, out, mask, ins = unpack(meta[p])
                k = 0
                for f in range(F):
                    o, n = q.omega[a], nA[c, f]
                    s = float(o[0]) * float(n[0]) + float(o[1]) * float(n[1]) + float(o[2]) * float(n[2])
                    want = nbr[c, f] >= 0 and s < 0
                    assert bool((mask >> f) & 1) == want, "gathered-face mask"
                    if not want:
                        continue
                    up = nbr[c, f]
                    assert level[up] < l, "an upwind cell in the same or a later level"
                    assert ins[k] != NONE and front.get(ins[k]) == up, "front slot does not hold the upwind cell"
                    k += 1
                assert all(v == NONE for v in ins[k:])
                assert k <= plan["slots"]
                if out != NONE:
                    assert out < plan["n_front"] and out not in writes
                    writes[out] = c
            front.update(writes)  # written during level l, read from level l + 1 on
    assert max(widths) == plan["max_width"]


def simulate_wave(plan, op, g, q_vec, A):
    nc, nb, F = g.n_cells, g.n_basis, g.faces_per_cell
    L = op.L
    psi = np.zeros(op.n)
    nbr = g.face_neighbour.reshape(nc, F)
    for a in range(A):
        for p in range(nc):
            c, out, mask, ins = unpack(plan["meta"][a, p])
            ups = {nbr[c, f] for f in range(F) if (mask >> f) & 1}
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


ACYCLIC = [c for c in CASES if c[1] == 2 or c[0].startswith("hex")]


@pytest.mark.parametrize("case", ACYCLIC, ids=[c[0] for c in ACYCLIC])
def test_wave_plan_invariants_and_exact_sweep(case):
    mesh, g, q, st, ss = build(case)
    plan = _lib.wave_plan(g, q)
    check_wave_invariants(plan, g, q)
    op = O.Operator(g, q, st, ss)
    qv = np.random.default_rng(3).standard_normal(op.n)
    psi = simulate_wave(plan, op, g, qv, q.n_angles)
    ref = op.sweep(qv)
    assert np.abs(psi - ref).max() <= 1e-12 * np.abs(ref).max()


def test_wave_plan_reports_cycles():
    """Jittered tets whose upwind graph has a cycle get no wave plan (the task sweep serves them)."""
    rng = np.random.default_rng(4)
    mesh = P.box_tets(3, 3, 3, jitter=0.25, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(3, 4)
    tasks = _lib.sweep_plan(g, q, 24)
    plan = _lib.wave_plan(g, q)
    assert plan["acyclic"] == (tasks["n_lagged"] == 0)


def test_wave_plan_of_the_named_triangle_mesh_fits_one_block():
    """256 x 256 jittered quads split into triangles, S8: about a thousand
    levels an ordinate, no level wider than one 256-thread block, and a
    front of a few hundred slots."""
    prob = P.config_tri256()
    plan = _lib.wave_plan(prob.geometry, prob.quad)
    assert plan["acyclic"] and plan["slots"] == 2
    assert plan["max_width"] <= 256 and plan["n_front"] <= 1024
    assert 900 <= plan["max_levels"] <= 1400


# The wave kernel's shared memory, as it addresses it: the mbarriers and a
# flag, then three level tables of max_levels + 1 int32 each
WAVE_STAGES, WAVE_HEADER = 32, 32 * 8 + 128


def chunk_bytes(width, R, elem):
    return (width * R * elem + 15) // 16 * 16


def replay_wave_copies(plan, lay, nb, elem):
    """Replay, per ordinate, the kernel's copy schedule: thread 0 issues
    level `next` while the span from the oldest unconsumed level's chunk to
    the end of `next`'s fits the ring and an mbarrier is free. Check that the
    level a block waits for was issued, that every chunk in flight lies inside
    the ring, 16-byte aligned, disjoint from the others in flight, and that
    every copy's source lies inside the store."""
    A = len(plan["lvl_base"]) - 1
    R = nb * nb * (1 + max(1, plan["slots"]))
    cap = lay["cap"]
    assert cap % 16 == 0 and lay["ring_base"] % 16 == 0
    assert WAVE_HEADER + 3 * 4 * (plan["max_levels"] + 1) <= lay["front_off"]
    assert lay["front_off"] + plan["n_front"] * nb * elem <= lay["ring_base"]
    assert lay["ring_base"] + cap == lay["smem"] <= _lib.B200_MAX_SHARED_PER_BLOCK
    max_ahead = 0
    for a in range(A):
        b0 = plan["lvl_base"][a] + a
        nlev = plan["lvl_base"][a + 1] - plan["lvl_base"][a]
        lp = plan["lvl_pos"][b0:b0 + nlev + 1]
        co = lay["chunk_rel"][b0:b0 + nlev + 1].astype(np.int64)
        ro = lay["ring_off"][b0:b0 + nlev + 1].astype(np.int64)
        region = int(lay["region"][a])
        assert region % 16 == 0
        nbytes = [chunk_bytes(int(lp[l + 1] - lp[l]), R, elem) for l in range(nlev)]
        nxt = 0

        def issue_upto(cur):
            nonlocal nxt
            while nxt < nlev and nxt - cur < WAVE_STAGES and co[nxt] + nbytes[nxt] - co[cur] <= cap:
                assert co[nxt] % 16 == 0 and ro[nxt] % 16 == 0
                assert 0 <= ro[nxt] and ro[nxt] + nbytes[nxt] <= cap, "a chunk crosses the ring's end"
                assert ro[nxt] == co[nxt] % cap
                assert region + co[nxt] + nbytes[nxt] <= lay["store_bytes"]
                nxt += 1

        issue_upto(0)
        for l in range(nlev):
            assert nxt > l, "a level waited for before its copy was issued"
            spans = sorted((int(ro[k]), int(ro[k] + nbytes[k])) for k in range(l, nxt))
            assert all(e0 <= s1 for (s0, e0), (s1, e1) in zip(spans, spans[1:])), "chunks in flight overlap"
            max_ahead = max(max_ahead, nxt - l)
            issue_upto(l + 1)
        assert nxt == nlev
    return max_ahead


@pytest.mark.parametrize("case", ACYCLIC, ids=[c[0] for c in ACYCLIC])
def test_wave_layout_replays_in_bounds(case):
    mesh, g, q, st, ss = build(case)
    nb = g.n_basis
    keys = [(nb, 8, _lib.B200_MAX_SHARED_PER_BLOCK), (nb, 4, _lib.B200_MAX_SHARED_PER_BLOCK)]
    plan = _lib.wave_plan(g, q, layouts=keys)
    for key in keys:
        replay_wave_copies(plan, plan["layout"][key], nb, key[1])
    # A small ring still works, one level at a time at worst
    R = nb * nb * (1 + max(1, plan["slots"]))
    elem = 8
    need = WAVE_HEADER + 3 * 4 * (plan["max_levels"] + 1) + plan["n_front"] * nb * elem + 256
    tight = _lib.wave_plan(g, q, layouts=[(nb, elem, need + chunk_bytes(plan["max_width"], R, elem))])
    replay_wave_copies(tight, tight["layout"][(nb, elem, need + chunk_bytes(plan["max_width"], R, elem))], nb, elem)


def test_named_triangle_mesh_wave_layout_replays_in_bounds():
    """The plain FP64 workload's store and ring, both precisions: every copy
    in bounds and disjoint, several levels in flight."""
    prob = P.config_tri256()
    keys = [(3, 8, _lib.B200_MAX_SHARED_PER_BLOCK), (3, 4, _lib.B200_MAX_SHARED_PER_BLOCK)]
    plan = _lib.wave_plan(prob.geometry, prob.quad, layouts=keys)
    ahead64 = replay_wave_copies(plan, plan["layout"][keys[0]], 3, 8)
    ahead32 = replay_wave_copies(plan, plan["layout"][keys[1]], 3, 4)
    assert ahead64 >= 3 and ahead32 >= 6
    # The stores: 27 values per cell-ordinate, plus the gaps that keep every
    # chunk from crossing the ring's end (memory only: gaps are never copied)
    n = prob.geometry.n_cells * prob.quad.n_angles * 27
    assert n * 8 <= plan["layout"][keys[0]]["store_bytes"] <= 1.12 * n * 8
    assert n * 4 <= plan["layout"][keys[1]]["store_bytes"] <= 1.12 * n * 4
