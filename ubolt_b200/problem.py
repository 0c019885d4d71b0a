"""Meshes, ordinates, cross sections and sources: the host-side problem set-up.

The mesh builders make conforming box meshes (quads, triangles, hexes, Kuhn
tets) with optional jitter of the interior vertices, numbering cells tile by
tile so a tile's cells - and so each angular-flux node run - sit together in
HBM. Geometry comes from the library (ubolt_geometry_build); everything here
is NumPy.

The named workloads are seeded: numpy Generator(PCG64(20261203 + i)) with
independent spawned streams for the mesh, the cross sections and the source.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

SEED_BASE = 20261203
# Cell shapes (UBOLT_TRI, ... of the C ABI)
TRI, QUAD, TET, HEX = 3, 4, 10, 12


def _native():
    """The library's binding, loaded on first use: the mesh builders and the
    named workloads' seeded data need no native code, so a CPU-only caller
    (the oracle's baseline) can build them without loading the library."""
    from . import _lib
    return _lib, _lib.lib, _lib.check


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# Ordinates
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

@dataclass
class Ordinates:
    dim: int
    sn: int
    omega: np.ndarray      # (A, 3)
    w: np.ndarray          # (A,)
    reflect: np.ndarray    # (3, A) int32, -1 past dim
    sum_weights: float

    @property
    def n_angles(self):
        return len(self.w)

    def struct(self):
        _lib, _, _ = _native()
        q = _lib.Quadrature()
        q.dim, q.n_angles, q.sum_weights = self.dim, self.n_angles, self.sum_weights
        q.omega = self.omega.ctypes.data_as(_lib.dp)
        q.w = self.w.ctypes.data_as(_lib.dp)
        q.reflect = self.reflect.ctypes.data_as(_lib.i32p)
        return q

    def opposite(self):
        """Index of -Omega_a for every a (the P of (V A)^T = P (V A) P)."""
        out = np.empty(self.n_angles, dtype=np.int64)
        for a in range(self.n_angles):
            hit = np.nonzero(np.all(self.omega == -self.omega[a], axis=1))[0]
            out[a] = hit[0]
        return out


def lqn(dim, sn):
    """The level-symmetric S_N set in 2D (XY) or 3D."""
    _lib, lib, check = _native()
    na, sw = C.c_int32(), C.c_double()
    check(lib.ubolt_quadrature_lqn(dim, sn, None, None, None, C.byref(na), C.byref(sw)))
    A = na.value
    omega = np.zeros((A, 3))
    w = np.zeros(A)
    refl = np.full((3, A), -1, dtype=np.int32)
    check(lib.ubolt_quadrature_lqn(dim, sn, omega.ctypes.data_as(_lib.dp), w.ctypes.data_as(_lib.dp),
                                   refl.ctypes.data_as(_lib.i32p), None, None))
    refl[dim:] = -1
    return Ordinates(dim, sn, omega, w, refl, sw.value)


def lqn_octant(sn):
    """(mu levels, 1-based level triples, whole-sphere weight fractions) of one octant."""
    _lib, lib, check = _native()
    nl, npnt = C.c_int32(), C.c_int32()
    check(lib.ubolt_lqn_octant(sn, None, None, None, C.byref(nl), C.byref(npnt)))
    mu = np.zeros(nl.value)
    pts = np.zeros((npnt.value, 3), dtype=np.int32)
    wt = np.zeros(npnt.value)
    check(lib.ubolt_lqn_octant(sn, mu.ctypes.data_as(_lib.dp), pts.ctypes.data_as(_lib.i32p),
                               wt.ctypes.data_as(_lib.dp), None, None))
    return mu, pts, wt


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# Meshes
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

@dataclass
class Mesh:
    dim: int
    cell_type: int
    vertices: np.ndarray   # (nv, dim)
    cells: np.ndarray      # (nc, verts per cell) int64
    shape: tuple = ()      # structured extent the mesh was built on

    @property
    def n_cells(self):
        return len(self.cells)


def _tile_order(shape, tile):
    """Structured cell indices (row-major, x fastest) listed tile by tile."""
    idx = np.indices(shape[::-1]).reshape(len(shape), -1)[::-1].T  # (n, dim) with x fastest
    t = tuple(max(1, tile) for _ in shape)
    key = []
    for d in reversed(range(len(shape))):
        key.append(idx[:, d] // t[d])
    for d in reversed(range(len(shape))):
        key.append(idx[:, d] % t[d])
    order = np.lexsort(tuple(reversed(key)))
    return idx[order]


def _jitter(v, n, h, amount, rng):
    if amount == 0.0 or rng is None:
        return v
    on_boundary = np.zeros(len(v), dtype=bool)
    for d in range(v.shape[1]):
        on_boundary |= np.isclose(v[:, d], 0.0) | np.isclose(v[:, d], h[d] * n[d])
    dv = rng.uniform(-amount, amount, size=v.shape) * np.asarray(h)
    dv[on_boundary] = 0.0
    return v + dv


def box_quads(nx, ny, lx=1.0, ly=1.0, jitter=0.0, rng=None, tile=8):
    h = (lx / nx, ly / ny)
    gx, gy = np.meshgrid(np.arange(nx + 1) * h[0], np.arange(ny + 1) * h[1], indexing="xy")
    v = np.stack([gx.ravel(), gy.ravel()], axis=1)
    v = _jitter(v, (nx, ny), h, jitter, rng)
    ij = _tile_order((nx, ny), tile)
    i, j = ij[:, 0], ij[:, 1]
    vid = lambda a, b: b * (nx + 1) + a
    cells = np.stack([vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)], axis=1)
    return Mesh(2, QUAD, v, cells.astype(np.int64), (nx, ny))


def box_tris(nx, ny, lx=1.0, ly=1.0, jitter=0.0, rng=None, tile=8, diagonals="random"):
    """Quads split into two triangles; the diagonal of each quad is drawn from
    rng ("random"), alternates in a checkerboard ("alternate") or is always
    the lower-left to upper-right one ("uniform")."""
    q = box_quads(nx, ny, lx, ly, jitter, rng, tile)
    ij = _tile_order((nx, ny), tile)
    if diagonals == "random" and rng is not None:
        flip = rng.integers(0, 2, size=len(ij)).astype(bool)
    elif diagonals == "alternate":
        flip = ((ij[:, 0] + ij[:, 1]) % 2).astype(bool)
    else:
        flip = np.zeros(len(ij), dtype=bool)
    c = q.cells
    t0 = np.where(flip[:, None], c[:, [0, 1, 3]], c[:, [0, 1, 2]])
    t1 = np.where(flip[:, None], c[:, [1, 2, 3]], c[:, [0, 2, 3]])
    cells = np.stack([t0, t1], axis=1).reshape(-1, 3)
    return Mesh(2, TRI, q.vertices, cells, (nx, ny))


def box_hexes(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0, jitter=0.0, rng=None, tile=4):
    h = (lx / nx, ly / ny, lz / nz)
    gx, gy, gz = np.meshgrid(np.arange(nx + 1) * h[0], np.arange(ny + 1) * h[1], np.arange(nz + 1) * h[2],
                             indexing="ij")
    v = np.stack([gx.transpose(2, 1, 0).ravel(), gy.transpose(2, 1, 0).ravel(), gz.transpose(2, 1, 0).ravel()],
                 axis=1)
    v = _jitter(v, (nx, ny, nz), h, jitter, rng)
    ijk = _tile_order((nx, ny, nz), tile)
    i, j, k = ijk[:, 0], ijk[:, 1], ijk[:, 2]
    vid = lambda a, b, c: (c * (ny + 1) + b) * (nx + 1) + a
    cells = np.stack([vid(i, j, k), vid(i + 1, j, k), vid(i + 1, j + 1, k), vid(i, j + 1, k),
                      vid(i, j, k + 1), vid(i + 1, j, k + 1), vid(i + 1, j + 1, k + 1), vid(i, j + 1, k + 1)],
                     axis=1)
    return Mesh(3, HEX, v, cells.astype(np.int64), (nx, ny, nz))


# Kuhn's six tetrahedra of a cube, all sharing the diagonal from vertex 0 to
# vertex 6: one per ordering of the axes walked from corner to corner
_KUHN = [(0, 1, 2, 6), (0, 1, 5, 6), (0, 3, 2, 6), (0, 3, 7, 6), (0, 4, 5, 6), (0, 4, 7, 6)]


def box_tets(nx, ny, nz, jitter=0.0, rng=None, tile=4, lx=1.0, ly=1.0, lz=1.0):
    hx = box_hexes(nx, ny, nz, lx, ly, lz, jitter=jitter, rng=rng, tile=tile)
    cells = np.concatenate([hx.cells[:, list(t)][:, None, :] for t in _KUHN], axis=1).reshape(-1, 4)
    return Mesh(3, TET, hx.vertices, cells, (nx, ny, nz))


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# Geometry
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

_GEOM_ARRAYS = [("volume", np.float64, 1), ("centroid", np.float64, 3), ("face_nA", np.float64, "F3"),
                ("face_neighbour", np.int64, "F"), ("face_bc", np.int32, "F"), ("face_side", np.int32, "F"),
                ("face_axis", np.int32, "F"), ("face_centroid", np.float64, "F3"),
                ("face_distance", np.float64, "F2")]
_DG1_ARRAYS = [("face_own", np.float64, "Fbb"), ("face_up", np.float64, "Fbb"), ("basis_grad", np.float64, "b3"),
               ("face_neighbour_grad", np.float64, "Fb3"), ("face_basis_value", np.float64, "Fb")]


@dataclass
class Geometry:
    """The DG geometry, NumPy-owned, in the C ABI's flat per-(cell, slot) layout."""
    dim: int
    n_basis: int
    faces_per_cell: int
    n_cells: int
    arrays: dict = field(default_factory=dict)

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays", {})
        if name in arrays:
            return arrays[name]
        raise AttributeError(name)

    def struct(self):
        _lib, _, _ = _native()
        g = _lib.DGGeometry()
        g.dim, g.n_basis, g.faces_per_cell, g.n_cells = self.dim, self.n_basis, self.faces_per_cell, self.n_cells
        for name, dt, _ in _GEOM_ARRAYS + _DG1_ARRAYS:
            if name in self.arrays:
                ptr_t = {np.float64: _lib.dp, np.int64: _lib.i64p, np.int32: _lib.i32p}[dt]
                setattr(g, name, self.arrays[name].ctypes.data_as(ptr_t))
        return g


def build_geometry(mesh, order, side_bc=None):
    """ubolt_geometry_build on a Mesh; side_bc[2 * dim] are UBOLT_BC_* (default vacuum).
    The result remembers what it was built from (`source`), so a checker can
    build its own geometry from the same mesh."""
    _lib, lib, check = _native()
    dim = mesh.dim
    sbc = np.zeros(2 * dim, dtype=np.int32) if side_bc is None else np.asarray(side_bc, dtype=np.int32)
    v = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int64)
    h = _lib.vp()
    check(lib.ubolt_geometry_build(dim, mesh.cell_type, len(v), v.ctypes.data_as(_lib.dp), len(cells),
                                   cells.ctypes.data_as(_lib.i64p), order, sbc.ctypes.data_as(_lib.i32p),
                                   C.byref(h)))
    try:
        view = _lib.DGGeometry()
        check(lib.ubolt_geometry_view(h, C.byref(view)))
        nc, F, nb = view.n_cells, view.faces_per_cell, view.n_basis
        sizes = {1: nc, 3: 3 * nc, "F": nc * F, "F3": 3 * nc * F, "F2": 2 * nc * F, "Fbb": nc * F * nb * nb,
                 "b3": nc * nb * 3, "Fb3": nc * F * nb * 3, "Fb": nc * F * nb}
        arrays = {}
        for name, dt, sz in _GEOM_ARRAYS + (_DG1_ARRAYS if nb > 1 else []):
            ptr = getattr(view, name)
            n = sizes[sz]
            arrays[name] = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)
        geo = Geometry(view.dim, nb, F, nc, arrays)
        geo.source = (mesh, order, sbc.copy())
        return geo
    finally:
        lib.ubolt_geometry_free(h)


_CG_ARRAYS = [("elem_vertex", np.int64, "env"), ("mass", np.float64, "enn"), ("grad", np.float64, "enn3"),
              ("stiff", np.float64, "enn9"), ("centre_grad", np.float64, "en3"), ("volume", np.float64, "e"),
              ("centroid", np.float64, "e3"), ("lumped_mass", np.float64, "v"), ("vertex_coord", np.float64, "v3"),
              ("star_offset", np.int64, "v1"), ("star_elem", np.int64, "s"), ("star_li", np.int32, "s"),
              ("bface_offset", np.int64, "v1"), ("bface_nA", np.float64, "b3"), ("bface_mass", np.float64, "b"),
              ("bface_side", np.int32, "b"), ("bface_bc", np.int32, "b"),
              ("elem_face_neighbour", np.int64, "eF"), ("elem_face_area", np.float64, "eF"),
              ("elem_face_bc", np.int32, "eF")]


@dataclass
class CGGeometry:
    """The CG-SUPG tables (ubolt_cg_geometry_build), NumPy-owned, in the C
    ABI's flat layouts: per element the mass, gradient and stiffness matrices
    of the degree-1 Lagrange basis; per vertex its star, lumped mass and
    boundary faces."""
    dim: int
    n_element_vertices: int
    faces_per_element: int
    n_vertices: int
    n_elements: int
    arrays: dict = field(default_factory=dict)

    @property
    def n_cells(self):
        return self.n_elements

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays", {})
        if name in arrays:
            return arrays[name]
        raise AttributeError(name)

    def struct(self):
        _lib, _, _ = _native()
        g = _lib.CGGeometry()
        g.dim, g.n_element_vertices, g.faces_per_element = self.dim, self.n_element_vertices, self.faces_per_element
        g.n_vertices, g.n_elements = self.n_vertices, self.n_elements
        g.n_star, g.n_bfaces = len(self.arrays["star_elem"]), len(self.arrays["bface_mass"])
        for name, dt, _ in _CG_ARRAYS:
            ptr_t = {np.float64: _lib.dp, np.int64: _lib.i64p, np.int32: _lib.i32p}[dt]
            setattr(g, name, self.arrays[name].ctypes.data_as(ptr_t))
        return g


def build_cg_geometry(mesh, side_bc=None):
    """ubolt_cg_geometry_build on a Mesh; side_bc[2 * dim] are UBOLT_BC_* (default vacuum)."""
    _lib, lib, check = _native()
    dim = mesh.dim
    sbc = np.zeros(2 * dim, dtype=np.int32) if side_bc is None else np.asarray(side_bc, dtype=np.int32)
    v = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int64)
    h = _lib.vp()
    check(lib.ubolt_cg_geometry_build(dim, mesh.cell_type, len(v), v.ctypes.data_as(_lib.dp), len(cells),
                                      cells.ctypes.data_as(_lib.i64p), sbc.ctypes.data_as(_lib.i32p), C.byref(h)))
    try:
        view = _lib.CGGeometry()
        check(lib.ubolt_cg_geometry_view(h, C.byref(view)))
        ne, nvx, nv, F = view.n_elements, view.n_vertices, view.n_element_vertices, view.faces_per_element
        sizes = {"env": ne * nv, "enn": ne * nv * nv, "enn3": ne * nv * nv * 3, "enn9": ne * nv * nv * 9,
                 "en3": ne * nv * 3, "e": ne, "e3": ne * 3, "v": nvx, "v3": nvx * 3, "v1": nvx + 1,
                 "s": view.n_star, "b": view.n_bfaces, "b3": view.n_bfaces * 3, "eF": ne * F}
        arrays = {}
        for name, dt, sz in _CG_ARRAYS:
            n = sizes[sz]
            arrays[name] = (np.ctypeslib.as_array(getattr(view, name), shape=(n,)).astype(dt, copy=True) if n
                            else np.zeros(0, dtype=dt))
        geo = CGGeometry(view.dim, nv, F, nvx, ne, arrays)
        geo.source = (mesh, sbc.copy())
        return geo
    finally:
        lib.ubolt_cg_geometry_free(h)


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# Problems
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

@dataclass
class Problem:
    """A fixed-source problem: geometry, ordinates and per-group data.

    sigma_t[g] and source[g] are per cell; sigma_s[g_from][g_to] per cell
    (zero where there is no transfer). Groups run high energy to low, so
    g_from < g_to is downscatter (include/ubolt/multigroup.hpp:15).
    """
    name: str
    mesh: Mesh
    geometry: Geometry
    quad: Ordinates
    sigma_t: np.ndarray          # (G, n_cells)
    sigma_s: np.ndarray          # (G, G, n_cells)
    source: np.ndarray           # (G, n_cells), angle-integrated
    side_inflow: np.ndarray = None   # (2 * dim,) angle-integrated vacuum inflow per side
    side_bc: np.ndarray = None
    rtol: float = 1e-8
    meta: dict = field(default_factory=dict)

    @property
    def n_groups(self):
        return self.sigma_t.shape[0]

    @property
    def n_rows(self):
        return self.geometry.n_cells * self.geometry.n_basis * self.quad.n_angles


def _streams(i, n=4):
    return [np.random.Generator(np.random.PCG64(s)) for s in np.random.SeedSequence(SEED_BASE + i).spawn(n)]


def config_fd64(scale=1.0, geometry=None, quadrature=None):
    """64 x 64 unit-square cells, S4, one group, sigma_t 1, sigma_s 0.5, unit
    source in the central 16 x 16 cells, vacuum - the reference's plain CPU
    case. As DG0 on a uniform quad box, the structured upwind FD stencil's twin."""
    n = max(4, int(round(64 * scale)))
    mesh = box_quads(n, n, tile=8)
    geom = (geometry or build_geometry)(mesh, 0)
    quad = (quadrature or lqn)(2, 4)
    c = geom.centroid.reshape(-1, 3)
    lo, hi = 0.5 - 8.0 / 64.0, 0.5 + 8.0 / 64.0
    inside = (c[:, 0] > lo) & (c[:, 0] < hi) & (c[:, 1] > lo) & (c[:, 1] < hi)
    nc = geom.n_cells
    return Problem("fd64_s4_dg0", mesh, geom, quad, np.ones((1, nc)), np.full((1, 1, nc), 0.5),
                   inside.astype(np.float64)[None, :], np.zeros(4), np.zeros(4, dtype=np.int32), rtol=1e-10,
                   meta={"n": n})


def config_tri256(scale=1.0, order=1, sn=8, geometry=None, quadrature=None):
    """DG1 on a jittered 256 x 256 quad grid split into triangles, S8, one group:
    sigma_t lognormal(0, 0.5), c ~ U(0.3, 0.99), source 1.0 in a disk of 20%
    area with a seeded centre, cold vacuum."""
    n = max(4, int(round(256 * scale)))
    s_mesh, s_xs, s_src, _ = _streams(1)
    mesh = box_tris(n, n, jitter=0.2, rng=s_mesh, tile=8, diagonals="random")
    geom = (geometry or build_geometry)(mesh, order)
    quad = (quadrature or lqn)(2, sn)
    nc = geom.n_cells
    sigma_t = s_xs.lognormal(0.0, 0.5, size=nc)
    ratio = s_xs.uniform(0.3, 0.99, size=nc)
    r = np.sqrt(0.2 / np.pi)
    centre = s_src.uniform(r, 1.0 - r, size=2)
    c = geom.centroid.reshape(-1, 3)[:, :2]
    q = (np.sum((c - centre) ** 2, axis=1) <= r * r).astype(np.float64)
    return Problem(f"tri{n}_s{sn}_dg{order}", mesh, geom, quad, sigma_t[None, :], (ratio * sigma_t)[None, None, :],
                   q[None, :], np.zeros(4), np.zeros(4, dtype=np.int32), rtol=1e-8,
                   meta={"n": n, "disk_centre": centre.tolist(), "disk_radius": r})


def config_hex128(scale=1.0, order=1, sn=8, n_groups=4, geometry=None, quadrature=None):
    """128^3 hex box, S8 (80 angles), 4 groups, downscatter only: sigma_t per
    (8^3 block, group) = 10^U(-1, 1); per (block, group) a total scattering
    fraction f = U(0.5, 0.9) of sigma_t, of which U(0.5, 0.9) stays in group
    and the rest is split equally over the lower groups (the last group keeps
    all of it); source 1.0 in group 0 everywhere; cold vacuum."""
    n = max(8, int(round(128 * scale)))
    _, s_xs, _, _ = _streams(2)
    mesh = box_hexes(n, n, n, tile=4)
    geom = (geometry or build_geometry)(mesh, order)
    quad = (quadrature or lqn)(3, sn)
    nc = geom.n_cells
    nb_blocks = max(1, n // 8)
    c = geom.centroid.reshape(-1, 3)
    blk = np.minimum((c * nb_blocks).astype(np.int64), nb_blocks - 1)
    bid = (blk[:, 2] * nb_blocks + blk[:, 1]) * nb_blocks + blk[:, 0]
    G = n_groups
    nblk = nb_blocks ** 3
    st_blk = 10.0 ** s_xs.uniform(-1.0, 1.0, size=(G, nblk))
    frac = s_xs.uniform(0.5, 0.9, size=(G, nblk))
    within = s_xs.uniform(0.5, 0.9, size=(G, nblk))
    ss_blk = np.zeros((G, G, nblk))
    for g in range(G):
        total = frac[g] * st_blk[g]
        if g == G - 1:
            ss_blk[g, g] = total
        else:
            ss_blk[g, g] = within[g] * total
            rest = (1.0 - within[g]) * total / (G - 1 - g)
            for gp in range(g + 1, G):
                ss_blk[g, gp] = rest
    sigma_t = st_blk[:, bid]
    sigma_s = ss_blk[:, :, bid]
    src = np.zeros((G, nc))
    src[0] = 1.0
    return Problem(f"hex{n}_s{sn}_g{G}_dg{order}", mesh, geom, quad, sigma_t, sigma_s, src, np.zeros(6),
                   np.zeros(6, dtype=np.int32), rtol=1e-8, meta={"n": n})


def config_tet44(scale=1.0, order=1, sn=8, geometry=None, quadrature=None):
    """Jittered Kuhn tets of a 44^3 cube grid (511,104 tets), S8 3D, one group:
    sigma_t lognormal(0, 1), c ~ U(0.5, 0.999), source 1.0 in [0.25, 0.75]^3."""
    n = max(2, int(round(44 * scale)))
    s_mesh, s_xs, _, _ = _streams(4)
    mesh = box_tets(n, n, n, jitter=0.2, rng=s_mesh, tile=4)
    geom = (geometry or build_geometry)(mesh, order)
    quad = (quadrature or lqn)(3, sn)
    nc = geom.n_cells
    sigma_t = s_xs.lognormal(0.0, 1.0, size=nc)
    ratio = s_xs.uniform(0.5, 0.999, size=nc)
    c = geom.centroid.reshape(-1, 3)
    q = np.all((c > 0.25) & (c < 0.75), axis=1).astype(np.float64)
    return Problem(f"tet{n}_s{sn}_dg{order}", mesh, geom, quad, sigma_t[None, :], (ratio * sigma_t)[None, None, :],
                   q[None, :], np.zeros(6), np.zeros(6, dtype=np.int32), rtol=1e-8, meta={"n": n})


def detector_patch(problem, cells_per_side=16, seed_index=3):
    """The detector of the adjoint workload: the cells whose centroids fall in
    a seeded square (cube in 3D) of cells_per_side * h, h the grid spacing."""
    _, _, _, s_det = _streams(seed_index)
    n = problem.meta["n"]
    h = 1.0 / n
    side = cells_per_side * h
    dim = problem.geometry.dim
    lo = s_det.uniform(0.0, 1.0 - side, size=dim)
    c = problem.geometry.centroid.reshape(-1, 3)[:, :dim]
    return np.all((c >= lo) & (c <= lo + side), axis=1)


CONFIGS = {"fd64": config_fd64, "tri256": config_tri256, "hex128": config_hex128, "tet44": config_tet44}
