"""Python face of the CPU oracle - TEST INFRASTRUCTURE ONLY.

Loads oracle/_build/liboracle.so (built by `make -C oracle`), the plain-C
restatement of UBOLT's assembled operator in oracle/ubolt_oracle.c, and
returns SciPy CSR matrices and NumPy vectors. It computes with its own
geometry (oracle/geometry.py) and the reference's own ordinate tables
(oracle/quadrature.py), never with the library's: handed a geometry or an
ordinate set the library built, it builds its own from the same mesh and
order. Only tests/, the smoke check and bench.py's CPU baseline use this
module; the library never does.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
from types import SimpleNamespace
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
sys.path.insert(0, HERE)
import geometry as _geometry  # noqa: E402  (the oracle's own geometry)
import quadrature as _quadrature  # noqa: E402  (the reference's ordinate sets)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


if not os.path.exists(LIB):
    build()
_lib = C.CDLL(LIB)

dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _sig(name, restype, *args):
    f = getattr(_lib, name)
    f.restype = restype
    f.argtypes = list(args)
    return f


_sig("oracle_dg_nnz_bound", C.c_int64, C.c_int, C.c_int, C.c_int64, C.c_int)
_sig("oracle_assemble_dg", C.c_int64, C.c_int, C.c_int, C.c_int64, C.c_int, dp, i64p, i32p, i32p, dp, C.c_void_p,
     C.c_void_p, C.c_void_p, dp, i32p, dp, i64p, i64p, dp)
_sig("oracle_assemble_fd2d", C.c_int64, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, dp, dp, i32p, i32p, dp,
     i64p, i64p, dp)
_sig("oracle_spmv", None, C.c_int64, i64p, i64p, dp, dp, dp)
_sig("oracle_angular_integral", None, C.c_int64, C.c_int, dp, dp, dp)
_sig("oracle_scatter_add", None, C.c_int64, C.c_int, C.c_int, dp, C.c_double, dp, dp, dp)
_sig("oracle_add_source", None, C.c_int64, C.c_int, C.c_int, C.c_double, dp, dp)
_sig("oracle_add_transfer", None, C.c_int64, C.c_int, C.c_int, C.c_double, dp, dp, dp)
_sig("oracle_ghost_inflow", None, C.c_int, C.c_int, C.c_int64, C.c_int, dp, i64p, i32p, i32p, dp, C.c_void_p, dp,
     C.c_double, dp, dp)
_sig("oracle_block_inverse", C.c_int64, C.c_int64, C.c_int, C.c_int, i64p, i64p, dp, dp)
_sig("oracle_block_apply", None, C.c_int64, C.c_int, C.c_int, dp, dp, dp)
_sig("oracle_solve", C.c_int, C.c_int64, C.c_int, C.c_int, i64p, i64p, dp, dp, C.c_double, dp, dp, dp, C.c_double,
     C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double))
_sig("oracle_sweep", None, C.c_int64, C.c_int, C.c_int, i64p, i64p, dp, dp, dp)
_sig("oracle_threads", C.c_int)

PC_NONE, PC_BLOCK, PC_SWEEP = 0, 1, 2


def geometry_from_mesh(mesh, order, side_bc=None):
    """The oracle's own geometry of a mesh (oracle/geometry.py)."""
    return _geometry.build(mesh.dim, mesh.cell_type, mesh.vertices, mesh.cells, order, side_bc)


def lqn(dim, sn):
    """The reference's level-symmetric set, from its own generator's tables."""
    return _quadrature.lqn(dim, sn)


def own_geometry(g):
    """The oracle never computes with the library's geometry: a geometry the
    library built carries the mesh it came from, and the oracle builds its
    own from that (once per object). An oracle geometry passes through."""
    if not hasattr(g, "arrays"):
        return g
    cached = g.__dict__.get("_oracle_geometry")
    if cached is None:
        mesh, order, side_bc = g.__dict__["source"]
        cached = geometry_from_mesh(mesh, order, side_bc)
        g.__dict__["_oracle_geometry"] = cached
    return cached


def own_quadrature(q):
    """Likewise the ordinates: the reference's set of the same order, its
    ordinates listed in the caller's order (each of the caller's matched to
    one of the oracle's by direction, to 1e-12)."""
    if not hasattr(q, "struct"):
        return q
    cached = q.__dict__.get("_oracle_quadrature")
    if cached is None:
        own = lqn(q.dim, q.sn)
        A = own.n_angles
        given = np.asarray(q.omega, dtype=np.float64).reshape(-1, 3)
        assert len(given) == A, "a quadrature of another size than the LQn set of its order"
        dist = np.abs(given[:, None, :] - own.omega[None, :, :]).max(axis=2)
        perm = dist.argmin(axis=1)
        assert dist[np.arange(A), perm].max() <= 1e-12 and len(set(perm.tolist())) == A, \
            "the ordinates are not the LQn set of their order"
        if np.array_equal(perm, np.arange(A)):
            cached = own
        else:
            inv = np.argsort(perm)
            refl = np.full_like(own.reflect, -1)
            refl[:own.dim] = inv[own.reflect[:own.dim][:, perm]]
            cached = SimpleNamespace(dim=own.dim, sn=own.sn, omega=own.omega[perm], w=own.w[perm], reflect=refl,
                                     sum_weights=own.sum_weights, n_angles=A)
        q.__dict__["_oracle_quadrature"] = cached
    return cached


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Operator:
    """The assembled streaming + removal CSR of one group plus the matrix-free
    scatter: the reference's TransportOperator shell, on the CPU."""

    def __init__(self, geometry, quad, sigma_t, sigma_s):
        g = own_geometry(geometry)
        quad = own_quadrature(quad)
        self.nb, self.F, self.nc, self.A = g.n_basis, g.faces_per_cell, g.n_cells, quad.n_angles
        self.n = self.nc * self.nb * self.A
        self.quad = quad
        self.sigma_t = np.ascontiguousarray(sigma_t, dtype=np.float64)
        self.sigma_s = np.ascontiguousarray(sigma_s, dtype=np.float64)
        cap = _lib.oracle_dg_nnz_bound(self.nb, self.F, self.nc, self.A)
        row_ptr = np.zeros(self.n + 1, dtype=np.int64)
        col = np.zeros(cap, dtype=np.int64)
        val = np.zeros(cap)
        dg1 = self.nb > 1
        nnz = _lib.oracle_assemble_dg(self.nb, self.F, self.nc, self.A, g.face_nA, g.face_neighbour, g.face_bc,
                                      g.face_axis, g.volume, _ptr(g.face_own) if dg1 else None,
                                      _ptr(g.face_up) if dg1 else None, _ptr(g.basis_grad) if dg1 else None,
                                      quad.omega.ravel(), quad.reflect.ravel(), self.sigma_t, row_ptr, col, val)
        if nnz < 0:
            raise MemoryError("oracle_assemble_dg")
        self.L = sp.csr_matrix((val[:nnz], col[:nnz], row_ptr), shape=(self.n, self.n))
        self.L.has_sorted_indices = True

    def apply(self, x, scatter=True):
        """y = (L - S) x, or L x."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        _lib.oracle_spmv(self.n, self.L.indptr.astype(np.int64), self.L.indices.astype(np.int64), self.L.data, x, y)
        if scatter:
            _lib.oracle_scatter_add(self.nc, self.nb, self.A, self.quad.w, self.quad.sum_weights, self.sigma_s, x, y)
        return y

    def scatter_matrix(self):
        """S as a sparse matrix: S[(node, a), (node, b)] = sigma_s w_b / W."""
        nn = self.nc * self.nb
        w = self.quad.w / self.quad.sum_weights
        blocks = np.repeat(self.sigma_s, self.nb)
        rows = (np.arange(nn)[:, None, None] * self.A + np.arange(self.A)[None, :, None]).repeat(self.A, axis=2)
        cols = (np.arange(nn)[:, None, None] * self.A + np.arange(self.A)[None, None, :]).repeat(self.A, axis=1)
        vals = blocks[:, None, None] * np.broadcast_to(w[None, None, :], (nn, self.A, self.A))
        return sp.csr_matrix((vals.ravel(), (rows.ravel(), cols.ravel())), shape=(self.n, self.n))

    def matrix(self):
        return (self.L - self.scatter_matrix()).tocsr()

    def block_inverse(self):
        inv = np.zeros(self.nc * self.A * self.nb * self.nb)
        n_sing = _lib.oracle_block_inverse(self.nc, self.nb, self.A, self.L.indptr.astype(np.int64),
                                           self.L.indices.astype(np.int64), self.L.data, inv)
        return inv, n_sing

    def block_apply(self, inv, x):
        y = np.empty(self.n)
        _lib.oracle_block_apply(self.nc, self.nb, self.A, inv, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def sweep(self, q):
        psi = np.empty(self.n)
        _lib.oracle_sweep(self.nc, self.nb, self.A, self.L.indptr.astype(np.int64), self.L.indices.astype(np.int64),
                          self.L.data, np.ascontiguousarray(q, dtype=np.float64), psi)
        return psi

    def solve(self, b, rtol=1e-12, max_it=2000, restart=30, pc=PC_SWEEP, x0=None):
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        res = C.c_double()
        it = _lib.oracle_solve(self.nc, self.nb, self.A, self.L.indptr.astype(np.int64),
                               self.L.indices.astype(np.int64), self.L.data, self.quad.w, self.quad.sum_weights,
                               self.sigma_s, np.ascontiguousarray(b, dtype=np.float64), x, rtol, max_it, restart, pc,
                               C.byref(res))
        return x, it, res.value


def angular_integral(psi, n_nodes, quad):
    quad = own_quadrature(quad)
    phi = np.empty(n_nodes)
    _lib.oracle_angular_integral(n_nodes, quad.n_angles, quad.w, np.ascontiguousarray(psi, dtype=np.float64), phi)
    return phi


def rhs(geometry, quad, source_cell, side_inflow=None):
    """b = ghost inflow + isotropic source, added onto zero as the driver does."""
    g = own_geometry(geometry)
    quad = own_quadrature(quad)
    n = g.n_cells * g.n_basis * quad.n_angles
    b = np.zeros(n)
    if side_inflow is not None and np.any(np.asarray(side_inflow) != 0.0):
        inflow = np.zeros(6)
        inflow[:len(side_inflow)] = side_inflow
        _lib.oracle_ghost_inflow(g.n_basis, g.faces_per_cell, g.n_cells, quad.n_angles, g.face_nA, g.face_neighbour,
                                 g.face_bc, g.face_side, g.volume,
                                 _ptr(g.face_basis_value) if g.n_basis > 1 else None, quad.omega.ravel(),
                                 quad.sum_weights, inflow, b)
    _lib.oracle_add_source(g.n_cells, g.n_basis, quad.n_angles, quad.sum_weights,
                           np.ascontiguousarray(source_cell, dtype=np.float64), b)
    return b


def add_transfer(b, phi, sigma_s, n_cells, nb, quad):
    quad = own_quadrature(quad)
    _lib.oracle_add_transfer(n_cells, nb, quad.n_angles, quad.sum_weights, np.ascontiguousarray(phi),
                             np.ascontiguousarray(sigma_s, dtype=np.float64), b)
    return b


def fd2d(nx, ny, quad, sigma_t, side_bc=(0, 0, 0, 0), lx=1.0, ly=1.0):
    """Streaming + removal of the structured 2D FD backend (ghost-flux rows)."""
    quad = own_quadrature(quad)
    A = quad.n_angles
    n = nx * ny * A
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    col = np.zeros(3 * n, dtype=np.int64)
    val = np.zeros(3 * n)
    nnz = _lib.oracle_assemble_fd2d(nx, ny, lx / nx, ly / ny, A, np.ascontiguousarray(quad.omega[:, 0]),
                                    np.ascontiguousarray(quad.omega[:, 1]), quad.reflect.ravel(),
                                    np.asarray(side_bc, dtype=np.int32), np.ascontiguousarray(sigma_t, dtype=np.float64),
                                    row_ptr, col, val)
    return sp.csr_matrix((val[:nnz], col[:nnz], row_ptr), shape=(n, n))


def threads():
    return _lib.oracle_threads()


u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_sig("oracle_dsa_void_policy", C.c_int, C.c_int, C.c_int64, dp, i64p, i32p, dp, dp, dp, C.c_double, C.c_int,
     C.c_double, u8p, u8p, dp, dp)
_sig("oracle_dsa_mip", C.c_int64, C.c_int, C.c_int, C.c_int64, dp, i64p, i32p, dp, dp, dp, dp, dp, dp, dp, dp,
     C.c_double, dp, u8p, u8p, C.c_int, i64p, i64p, dp)
_sig("oracle_dsa_dg0", C.c_int64, C.c_int, C.c_int64, C.c_int, dp, i64p, i32p, dp, dp, dp, dp, C.c_double, dp, dp,
     C.c_int, C.c_double, dp, u8p, i64p, i64p, dp)
_sig("oracle_dsa_restrict", None, C.c_int64, C.c_int, C.c_int, dp, dp, dp, C.c_void_p, dp)
_sig("oracle_dsa_prolong", None, C.c_int64, C.c_int, C.c_int, C.c_double, dp, C.c_void_p, dp)


class VoidPolicy:
    """The DSA void policy for one group (DSAPrecon::assemble,
    src/dsak.kokkos.cxx:233-345): per cell is_void, masked and D, the bridge
    decision, the voids' mean chord and their count; singular is True where
    the diffusion operator would be singular."""

    def __init__(self, geometry, sigma_t, sigma_s, void_sigma_t=0.0, bridge=True, void_d=0.0):
        g = own_geometry(geometry)
        nc = g.n_cells
        self.is_void = np.zeros(nc, dtype=np.uint8)
        self.masked = np.zeros(nc, dtype=np.uint8)
        self.d = np.zeros(nc)
        out = np.zeros(3)
        st = np.ascontiguousarray(sigma_t, dtype=np.float64)
        ss = np.ascontiguousarray(sigma_s, dtype=np.float64)
        self.singular = bool(_lib.oracle_dsa_void_policy(g.faces_per_cell, nc, g.face_nA, g.face_neighbour,
                                                         g.face_bc, g.volume, st, ss, void_sigma_t, int(bridge),
                                                         void_d, self.is_void, self.masked, self.d, out))
        self.bridged = bool(out[0])
        self.chord = float(out[1])
        self.n_void = int(out[2])


def dsa_matrix(geometry, quad, sigma_t, sigma_s, penalty=4.0, consistent=True, power=1.5, policy=None):
    """The DSA diffusion matrix (MIP at DG1, two-point flux at DG0) as SciPy
    CSR, with D and the masks of `policy` (default: the void policy's defaults)."""
    g = own_geometry(geometry)
    quad = own_quadrature(quad)
    nc, F, nb = g.n_cells, g.faces_per_cell, g.n_basis
    cap = nc * (F + 1) * nb * nb
    ri, ci, v = np.zeros(cap, dtype=np.int64), np.zeros(cap, dtype=np.int64), np.zeros(cap)
    st = np.ascontiguousarray(sigma_t, dtype=np.float64)
    ss = np.ascontiguousarray(sigma_s, dtype=np.float64)
    pol = policy if policy is not None else VoidPolicy(g, st, ss)
    if nb > 1:
        e = _lib.oracle_dsa_mip(nb, F, nc, g.face_nA, g.face_neighbour, g.face_bc, g.face_distance, g.volume,
                                g.face_own, g.face_up, g.basis_grad, g.face_neighbour_grad, st, ss, penalty,
                                pol.d, pol.is_void, pol.masked, int(pol.bridged), ri, ci, v)
    else:
        e = _lib.oracle_dsa_dg0(F, nc, quad.n_angles, g.face_nA, g.face_neighbour, g.face_bc, g.face_distance,
                                g.volume, quad.omega.ravel(), quad.w, quad.sum_weights, st, ss, int(consistent), power,
                                pol.d, pol.masked, ri, ci, v)
    return sp.csr_matrix((v[:e], (ri[:e], ci[:e])), shape=(nc * nb, nc * nb))


def dsa_restrict(x, geometry, quad, masked=None):
    g = own_geometry(geometry)
    quad = own_quadrature(quad)
    rhs = np.empty(g.n_cells * g.n_basis)
    m = None if masked is None else np.ascontiguousarray(masked, dtype=np.uint8)
    _lib.oracle_dsa_restrict(g.n_cells, g.n_basis, quad.n_angles, quad.w, g.volume,
                             np.ascontiguousarray(x, dtype=np.float64), None if m is None else m.ctypes.data, rhs)
    return rhs


def dsa_prolong(u, geometry, quad, masked=None):
    g = own_geometry(geometry)
    quad = own_quadrature(quad)
    y = np.empty(g.n_cells * g.n_basis * quad.n_angles)
    m = None if masked is None else np.ascontiguousarray(masked, dtype=np.uint8)
    _lib.oracle_dsa_prolong(g.n_cells, g.n_basis, quad.n_angles, quad.sum_weights,
                            np.ascontiguousarray(u, dtype=np.float64), None if m is None else m.ctypes.data, y)
    return y


def dsa_structured(nx, ny, hx, hy, quad, sigma_t, sigma_s, vacuum=(True, True, True, True), consistent=True,
                   power=1.5):
    """The structured backend's DSA matrix, cell-centred 5-point star per unit
    volume (DSAStructured::assemble, src/dsa_structuredk.kokkos.cxx:183-288):
    diagonal sigma_a + sum of the face terms; an interior face the harmonic
    mean of the two D = 1/(3 sigma_t), blended with the axis's half-range
    current times h when `consistent` (BlendD, dsa_operatork.hpp:122-126);
    a vacuum side the Marshak term 1 / (h (2 + h / (2 D_b))), D_b the cell's
    D blended the same way. Cells x-fastest; vacuum = (x lo, x hi, y lo, y hi)."""
    quad = own_quadrature(quad)
    st = np.asarray(sigma_t, dtype=np.float64)
    ss = np.asarray(sigma_s, dtype=np.float64)
    d = 1.0 / (3.0 * st)
    h = (hx, hy)
    half = [float(np.sum(np.where(quad.omega[:, ax] > 0.0, quad.w * quad.omega[:, ax], 0.0)) / quad.sum_weights)
            for ax in range(2)]

    def blend(v, m):
        if not consistent:
            return v
        return v + m if power == 1.0 else (v ** power + m ** power) ** (1.0 / power)

    n = nx * ny
    rows, cols, vals = [], [], []
    for j in range(ny):
        for i in range(nx):
            c = j * nx + i
            diag = st[c] - ss[c]
            for ax in range(2):
                hd = h[ax]
                for side in (-1, 1):
                    ni, nj = (i + side, j) if ax == 0 else (i, j + side)
                    inside = 0 <= ni < nx and 0 <= nj < ny
                    if inside:
                        cn = nj * nx + ni
                        df = blend(2.0 * d[c] * d[cn] / (d[c] + d[cn]), half[ax] * hd)
                        rows.append(c)
                        cols.append(cn)
                        vals.append(-df / (hd * hd))
                        diag += df / (hd * hd)
                    elif vacuum[2 * ax + (0 if side < 0 else 1)]:
                        db = blend(d[c], half[ax] * hd)
                        diag += 1.0 / (hd * (2.0 + hd / (2.0 * db)))
            rows.append(c)
            cols.append(c)
            vals.append(diag)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
