"""Edge cases of the CUDA path against the oracle, through the C ABI.

The cases are:
- a single cell and a cell count that fills no block;
- the fewest ordinates (2D S2, one FP32 thread per cell);
- a zero right-hand side;
- host batches of zero and one solve."""
import numpy as np
import pytest
import torch

import oracle as O
from ubolt_b200 import problem as P
from ubolt_b200 import transport as T

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def rel(a, b):
    a = a.detach().cpu().double().numpy() if torch.is_tensor(a) else a
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


SMALL = [
    ("one_quad_dg1", lambda: P.box_quads(1, 1), 1, 4),
    ("one_quad_dg0", lambda: P.box_quads(1, 1), 0, 4),
    ("one_hex_dg1", lambda: P.box_hexes(1, 1, 1), 1, 2),
    ("seven_quads_dg1", lambda: P.box_quads(7, 1), 1, 8),
    ("two_tris_dg1_s2", lambda: P.box_tris(1, 1), 1, 2),
    ("quads_dg0_s2", lambda: P.box_quads(5, 3), 0, 2),
]


@pytest.mark.parametrize("name,mk,order,sn", SMALL, ids=[c[0] for c in SMALL])
def test_small_meshes_match_oracle(name, mk, order, sn):
    mesh = mk()
    g = P.build_geometry(mesh, order)
    q = P.lqn(g.dim, sn)
    rng = np.random.default_rng(2)
    st = rng.uniform(0.5, 2.0, g.n_cells)
    ss = st * rng.uniform(0.2, 0.8, g.n_cells)
    ctx = T.Context(g, q)
    keep = (dev(st), dev(ss))
    ctx.set_group(*keep)
    op = O.Operator(g, q, st, ss)
    x = rng.standard_normal(op.n)
    A = T.TransportOperator(ctx)
    assert rel(A.mult(dev(x)), op.apply(x)) < 1e-13
    assert rel(A.mult_unscattered(dev(x)), op.apply(x, scatter=False)) < 1e-13
    assert rel(A.mult_transpose(dev(x)), op.matrix().T @ x) < 1e-13
    x32 = dev(x, torch.float32)
    assert rel(A.mult(x32), op.apply(x32.double().cpu().numpy())) < 2e-5
    # The solve, against the oracle's direct solve
    b = rng.uniform(0.1, 1.0, op.n)
    ref = np.linalg.solve(op.matrix().toarray(), b)
    xs, st_ = T.TransportSolver(ctx, rtol=1e-12).solve(dev(b))
    assert st_["converged"]
    assert rel(xs, ref) < 1e-9
    ctx.close()


def test_zero_right_hand_side_returns_zero():
    mesh = P.box_tris(4, 4, jitter=0.2, rng=np.random.default_rng(1))
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, 4)
    ctx = T.Context(g, q)
    keep = (dev(np.full(g.n_cells, 1.0)), dev(np.full(g.n_cells, 0.5)))
    ctx.set_group(*keep)
    for precision in ("fp64", "mixed"):
        x = ctx.vector(fill=3.0)
        x, st = T.TransportSolver(ctx, precision=precision).solve(ctx.vector(fill=0.0), x)
        assert st["converged"] and st["iterations"] == 0
        assert x.abs().max().item() == 0.0
    ctx.close()


def test_host_batch_of_zero_and_one():
    mesh = P.box_quads(4, 3)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, 4)
    ctx = T.Context(g, q)
    keep = (dev(np.full(g.n_cells, 1.0)), dev(np.full(g.n_cells, 0.4)))
    ctx.set_group(*keep)
    solver = T.TransportSolver(ctx, rtol=1e-10)
    assert solver.solve_host_batch([], []) == []
    b = torch.rand(ctx.n_rows, dtype=torch.float64)
    x = torch.zeros_like(b)
    (st,) = solver.solve_host_batch([b], [x])
    torch.cuda.current_stream().synchronize()
    ref, _ = solver.solve(b.cuda())
    assert st["converged"] and (x - ref.cpu()).abs().max().item() <= 1e-13 * ref.abs().max().item()
    ctx.close()
