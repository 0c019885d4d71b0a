"""The C ABI without a GPU: the library loads, exports every symbol its header
declares, and its argument checks fail cleanly with a status and a message."""
import ctypes as C

import numpy as np
import pytest

from ubolt_b200 import _lib
from ubolt_b200._lib import lib


def test_every_declared_symbol_is_exported():
    names = _lib.declared_symbols()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in include/ubolt_b200.h but not exported: {missing}"


def test_version_and_error_string():
    assert b"sm_100a" in lib.ubolt_version()
    rc = lib.ubolt_ctx_create(None, None, None)
    assert rc == 1  # UBOLT_ERR_ARG
    assert b"NULL" in lib.ubolt_last_error()


def test_null_context_is_rejected_by_every_apply():
    for name in ("ubolt_apply", "ubolt_apply_f32", "ubolt_apply_unscattered", "ubolt_apply_adjoint",
                 "ubolt_block_apply", "ubolt_scalar_flux"):
        assert getattr(lib, name)(None, None, None, None) == 1, name
    assert lib.ubolt_set_group(None, None, None, None) == 1
    assert lib.ubolt_ctx_destroy(None) == 0


def test_geometry_build_rejects_bad_input():
    v = np.zeros((3, 2))
    cells = np.array([[0, 1, 2]], dtype=np.int64)
    sbc = np.zeros(4, dtype=np.int32)
    h = _lib.vp()
    rc = lib.ubolt_geometry_build(2, _lib.HEX, 3, v.ctypes.data_as(_lib.dp), 1, cells.ctypes.data_as(_lib.i64p), 1,
                                  sbc.ctypes.data_as(_lib.i32p), C.byref(h))
    assert rc == 1 and b"not a 2D shape" in lib.ubolt_last_error()
    # Degenerate (zero-area) triangle
    rc = lib.ubolt_geometry_build(2, _lib.TRI, 3, v.ctypes.data_as(_lib.dp), 1, cells.ctypes.data_as(_lib.i64p), 0,
                                  sbc.ctypes.data_as(_lib.i32p), C.byref(h))
    assert rc == 1


@pytest.mark.parametrize("order", [0, 1])
def test_geometry_view_roundtrip(order):
    from ubolt_b200 import problem as P
    m = P.box_quads(3, 2)
    g = P.build_geometry(m, order)
    assert g.n_cells == 6 and g.faces_per_cell == 4
    assert ("face_own" in g.arrays) == (order == 1)


def test_option_defaults_and_struct_sizes():
    """The ctypes mirrors of the option structs match the header's defaults,
    and the new entry points reject a NULL context."""
    o = _lib.DsaOptions()
    lib.ubolt_dsa_defaults(C.byref(o))
    assert (o.penalty, o.consistent_power, o.consistent_d, o.inner_iterations) == (4.0, 1.5, 1, 30)
    assert (o.void_sigma_t, o.void_d, o.void_bridge) == (0.0, 0.0, 1)
    assert C.sizeof(_lib.DsaOptions) == 48
    s = _lib.SolveOptions()
    lib.ubolt_solve_defaults(C.byref(s))
    assert (s.rtol, s.max_it, s.restart, s.x_zero) == (1e-8, 500, 30, 1)
    n, br, ch = C.c_int64(0), C.c_int32(0), C.c_double(0.0)
    assert lib.ubolt_dsa_void_info(None, C.byref(n), C.byref(br), C.byref(ch)) == 1
    assert lib.ubolt_solve_host_batch(None, 0, None, None, None, None, None) == 1
