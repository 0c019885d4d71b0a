"""The DSA apply whose inner-solve scratch is a fixed array inside the
library (ubolt_dsa_apply_static), for callers that cannot let the library
allocate device memory while they solve - typically because their own memory
pool has already reserved the device. It must give what the workspace path
gives, call after call: the array keeps the previous call's values, so a
second call checks that everything the solve reads is rewritten first.

Named to run last: a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_scratch_dsa_apply_matches_workspace_apply():
    import torch
    from ubolt_b200 import _lib
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T

    rng = np.random.default_rng(17)
    mesh = P.box_tris(24, 20, jitter=0.2, rng=rng)
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, 4)
    nc = g.n_cells
    st = rng.lognormal(0.0, 0.5, nc)
    ss = st * rng.uniform(0.3, 0.99, nc)
    ctx = T.Context(g, q)
    keep = (torch.tensor(st, device="cuda"), torch.tensor(ss, device="cuda"))
    ctx.set_group(*keep)
    dsa = T.DSAPrecon(ctx, inner_iterations=40)
    dsa.set_group()
    for call in range(2):
        x = torch.tensor(rng.standard_normal(ctx.n_rows), device="cuda")
        ref = dsa.apply(x)
        y = torch.full_like(x, np.nan)
        _lib.check(_lib.lib.ubolt_dsa_apply_static(ctx.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        torch.cuda.synchronize()
        err = (y - ref).abs().max().item() / ref.abs().max().item()
        assert err <= 1e-13, (call, err)
    ctx.close()


def test_static_scratch_rejects_a_problem_over_its_limit():
    import torch
    from ubolt_b200 import _lib
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T

    mesh = P.box_quads(260, 260)            # 67600 cells x 3 modes = 202800 nodes: fits
    big = P.box_tris(300, 300)              # 180000 cells x 3 = 540000 nodes: over 262144
    for m, fits in ((mesh, True), (big, False)):
        g = P.build_geometry(m, 1)
        q = P.lqn(2, 2)
        ctx = T.Context(g, q)
        keep = (torch.ones(g.n_cells, dtype=torch.float64, device="cuda"),
                torch.full((g.n_cells,), 0.5, dtype=torch.float64, device="cuda"))
        ctx.set_group(*keep)
        dsa = T.DSAPrecon(ctx, inner_iterations=2)
        dsa.set_group()
        x = torch.ones(ctx.n_rows, dtype=torch.float64, device="cuda")
        x += torch.rand(ctx.n_rows, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
        y = torch.empty_like(x)
        rc = _lib.lib.ubolt_dsa_apply_static(ctx.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        if fits:
            # Close to the limit, where the grid fills most of the partial
            # slots, the fixed array still gives the workspace path's answer
            assert rc == 0, _lib.lib.ubolt_last_error()
            ref = dsa.apply(x)
            torch.cuda.synchronize()
            err = (y - ref).abs().max().item() / ref.abs().max().item()
            assert err <= 1e-13, err
        else:
            assert rc == 1 and b"exceed the fixed scratch" in _lib.lib.ubolt_last_error()
        ctx.close()
