"""CPU restatement of UBOLT's CG-SUPG backend - TEST INFRASTRUCTURE ONLY.

Continuous P1 (triangles, tetrahedra) / Q1 (quadrilaterals, hexahedra)
Galerkin with consistent SUPG, one unknown per (vertex, ordinate), angle
fastest: row = vertex * A + a. Written from the reference's
include/ubolt/unstructured_cg.hpp:11-88 (the scheme), src/unstructured_cgk.
kokkos.cxx:52-255 (element tables), :276-561 (stars, lumped masses, weak
boundary faces, the ghost inflow) and :676-757 (the weighted load),
src/terms_cgk.kokkos.cxx:41-101 (SUPGFillKernel, the assembled term and its
diagonal) and :203-221 / :325-356 (the scatter and the source), and
src/dsa_cgk.kokkos.cxx:60-84, 114-203 and 247-281 (the CG DSA).

Everything is computed here from the mesh's vertices and cells alone, with
NumPy: its own quadrature (Gauss-Legendre collapsed onto the simplex by the
Duffy map, tensor Gauss-Legendre on the box - four points a direction, the
rule a degree-1 Lagrange element of quadrature order 3 carries), its own face
matching and its own sparse assembly. It returns SciPy CSR matrices; only
tests/, the smoke check and the bench's CPU legs use it.
"""
import numpy as np
import scipy.sparse as sp

TRI, QUAD, TET, HEX = 3, 4, 10, 12  # the VTK cell type numbers the mesh carries
BC_VACUUM, BC_REFLECT = 0, 1

# Corner of each Q1 basis function in the unit box, in the mesh's vertex order
# (counter-clockwise; bottom face then top face)
_QUAD_CORNERS = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=float)
_HEX_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=float)

# Element faces as vertex lists of the element
_FACES = {
    TRI: [(0, 1), (1, 2), (2, 0)],
    QUAD: [(0, 1), (1, 2), (2, 3), (3, 0)],
    TET: [(1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)],
    HEX: [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)],
}


def _gauss01(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (x + 1.0), 0.5 * w


def reference_rule(cell_type):
    """Quadrature points and weights on the reference cell, the basis values
    (nq, nv) and reference gradients (nq, nv, dim) there, and the reference
    centroid."""
    g, gw = _gauss01(4)
    if cell_type in (QUAD, HEX):
        corners = _QUAD_CORNERS if cell_type == QUAD else _HEX_CORNERS
        dim = corners.shape[1]
        grids = np.meshgrid(*([g] * dim), indexing="ij")
        pts = np.stack([t.ravel() for t in grids], axis=1)
        wts = np.prod(np.stack(np.meshgrid(*([gw] * dim), indexing="ij"), axis=0).reshape(dim, -1), axis=0)
        centre = np.full(dim, 0.5)
        phi, dphi = _q1(pts, corners)
        return pts, wts, phi, dphi, centre
    dim = 2 if cell_type == TRI else 3
    uu = np.meshgrid(*([g] * dim), indexing="ij")
    ww = np.meshgrid(*([gw] * dim), indexing="ij")
    u = [t.ravel() for t in uu]
    w = np.prod(np.stack([t.ravel() for t in ww]), axis=0)
    if dim == 2:
        pts = np.stack([u[0], u[1] * (1 - u[0])], axis=1)
        w = w * (1 - u[0])
    else:
        pts = np.stack([u[0], u[1] * (1 - u[0]), u[2] * (1 - u[0]) * (1 - u[1])], axis=1)
        w = w * (1 - u[0]) ** 2 * (1 - u[1])
    phi = np.concatenate([1.0 - pts.sum(axis=1, keepdims=True), pts], axis=1)
    dphi = np.zeros((len(pts), dim + 1, dim))
    dphi[:, 0, :] = -1.0
    for k in range(dim):
        dphi[:, k + 1, k] = 1.0
    return pts, w, phi, dphi, np.full(dim, 1.0 / (dim + 1))


def _q1(pts, corners):
    nq, dim = pts.shape
    nv = len(corners)
    f = np.where(corners[None, :, :] == 1, pts[:, None, :], 1.0 - pts[:, None, :])  # (nq, nv, dim)
    df = np.where(corners[None, :, :] == 1, 1.0, -1.0) * np.ones((nq, nv, dim))
    phi = np.prod(f, axis=2)
    dphi = np.empty((nq, nv, dim))
    for k in range(dim):
        others = np.prod(np.delete(f, k, axis=2), axis=2) if dim > 1 else 1.0
        dphi[:, :, k] = df[:, :, k] * others
    return phi, dphi


class Tables:
    """Per element: M_ij, G^d_ij = int phi_i d_d phi_j, K^{dd'}_ij = int d_d phi_i
    d_d' phi_j (d, d' < 3, zero past dim), the gradients at the reference
    centroid, the volume and the centroid; per vertex the lumped mass."""

    def __init__(self, mesh):
        self.dim = mesh.dim
        self.cell_type = mesh.cell_type
        X = np.asarray(mesh.vertices, dtype=float)[np.asarray(mesh.cells)]  # (ne, nv, dim)
        ne, nv, dim = X.shape
        pts, w, phi, dphi, centre = reference_rule(mesh.cell_type)
        J = np.einsum("ejd,qjk->eqdk", X, dphi)                 # dx_d / dxi_k
        det = np.linalg.det(J)
        if np.any(det == 0):
            raise ValueError("a degenerate element")
        invJ = np.linalg.inv(J)                                  # dxi_k / dx_d
        gphi = np.einsum("qjk,eqkd->eqjd", dphi, invJ)          # d phi_j / dx_d
        wq = w[None, :] * np.abs(det)                           # (ne, nq)
        self.volume = wq.sum(axis=1)
        xq = np.einsum("qj,ejd->eqd", phi, X)
        self.centroid = np.einsum("eq,eqd->ed", wq, xq) / self.volume[:, None]
        g3 = np.zeros((ne, len(w), nv, 3))
        g3[..., :dim] = gphi
        self.mass = np.einsum("eq,qi,qj->eij", wq, phi, phi)
        self.grad = np.einsum("eq,qi,eqjd->eijd", wq, phi, g3)
        self.stiff = np.einsum("eq,eqid,eqjf->eijdf", wq, g3, g3)
        # Gradients at the reference centroid
        if mesh.cell_type in (QUAD, HEX):
            corners = _QUAD_CORNERS if mesh.cell_type == QUAD else _HEX_CORNERS
            _, dc = _q1(centre[None, :], corners)
        else:
            dc = dphi[:1]
        Jc = np.einsum("ejd,jk->edk", X, dc[0])
        gc = np.einsum("jk,ekd->ejd", dc[0], np.linalg.inv(Jc))
        self.centre_grad = np.zeros((ne, nv, 3))
        self.centre_grad[..., :dim] = gc
        self.cells = np.asarray(mesh.cells, dtype=np.int64)
        self.n_vertices = len(mesh.vertices)
        self.vertices = np.zeros((self.n_vertices, 3))
        self.vertices[:, :dim] = mesh.vertices
        self.lumped = np.bincount(self.cells.ravel(), weights=self.mass.sum(axis=2).ravel(),
                                  minlength=self.n_vertices)


class BoundaryFaces:
    """The domain's boundary faces (one element), each with its vertices, the
    outward area-weighted normal, the area and the box side it lies on
    (2 * axis + (0 low | 1 high), by its normal's dominant axis); and every
    element's faces - the element across each (-1 on the boundary), the area
    and the boundary family."""

    def __init__(self, mesh, tables, side_bc):
        faces = _FACES[mesh.cell_type]
        cells = tables.cells
        ne = len(cells)
        F = len(faces)
        key = {}
        for e in range(ne):
            for f, fv in enumerate(faces):
                k = tuple(sorted(int(cells[e, i]) for i in fv))
                key.setdefault(k, []).append((e, f))
        self.elem_nbr = -np.ones((ne, F), dtype=np.int64)
        self.elem_area = np.zeros((ne, F))
        self.elem_bc = -np.ones((ne, F), dtype=np.int64)
        verts, nA, side = [], [], []
        for k, users in key.items():
            e, f = users[0]
            fv = [int(cells[e, i]) for i in faces[f]]
            P = tables.vertices[fv]
            if mesh.dim == 2:
                t = P[1] - P[0]
                n = np.array([t[1], -t[0], 0.0])
            elif len(fv) == 3:
                n = 0.5 * np.cross(P[1] - P[0], P[2] - P[0])
            else:
                n = 0.5 * np.cross(P[2] - P[0], P[3] - P[1])
            c3 = np.zeros(3)
            c3[:mesh.dim] = tables.centroid[e]
            if np.dot(n, P.mean(axis=0) - c3) < 0:
                n = -n
            area = float(np.linalg.norm(n))
            if len(users) == 2:
                (e0, f0), (e1, f1) = users
                self.elem_nbr[e0, f0], self.elem_nbr[e1, f1] = e1, e0
                self.elem_area[e0, f0] = self.elem_area[e1, f1] = area
                continue
            axis = int(np.argmax(np.abs(n[:mesh.dim])))
            s = 2 * axis + (1 if n[axis] > 0 else 0)
            self.elem_area[e, f] = area
            self.elem_bc[e, f] = side_bc[s]
            verts.append(fv)
            nA.append(n)
            side.append(s)
        self.verts = verts
        self.nA = np.array(nA).reshape(-1, 3)
        self.side = np.array(side, dtype=np.int64)


class Problem:
    """One group of the CG-SUPG system on a mesh: sigma_t, sigma_s per
    element, the quadrature (omega, w, reflect, sum_weights), zeta, and the
    box sides' families (UBOLT_BC_*)."""

    def __init__(self, mesh, quad, sigma_t, sigma_s, zeta=0.5, side_bc=None):
        self.mesh = mesh
        self.dim = mesh.dim
        self.T = Tables(mesh)
        self.side_bc = np.zeros(2 * mesh.dim, dtype=np.int64) if side_bc is None else np.asarray(side_bc)
        self.B = BoundaryFaces(mesh, self.T, self.side_bc)
        self.omega = np.asarray(quad.omega, dtype=float).reshape(-1, 3)
        self.w = np.asarray(quad.w, dtype=float)
        self.reflect = np.asarray(quad.reflect).reshape(3, -1)
        self.W = float(quad.sum_weights)
        self.A = len(self.w)
        self.zeta = float(zeta)
        self.sigma_t = np.asarray(sigma_t, dtype=float)
        self.sigma_s = np.asarray(sigma_s, dtype=float)
        self.nv = self.T.cells.shape[1]
        self.n_vertices = self.T.n_vertices
        self.n = self.n_vertices * self.A
        # The reflective faces must be axis-aligned (unstructured_cg.hpp:69-71)
        for n, s in zip(self.B.nA, self.B.side):
            if self.side_bc[s] == BC_REFLECT:
                off = np.abs(np.delete(n[:self.dim], s // 2)).max() if self.dim > 1 else 0.0
                if off > 1e-12 * np.linalg.norm(n):
                    raise ValueError("a reflective face that is not axis-aligned")

    def tau(self, sigma_t=None):
        """tau[e, a] = min(1 / sigma_t, 2 / (zeta sum_j |Omega_a . grad phi_j(x_c)|)),
        the second alone where sigma_t <= 0 (UboltSUPGTau, unstructured_cg.hpp:239-258)."""
        st = self.sigma_t if sigma_t is None else np.asarray(sigma_t, dtype=float)
        s = np.abs(np.einsum("ad,ejd->eaj", self.omega, self.T.centre_grad)).sum(axis=2)
        thin = 2.0 / (self.zeta * s)
        thick = np.where(st > 0, 1.0 / np.where(st > 0, st, 1.0), np.inf)
        return np.minimum(thick[:, None], thin)

    def _rows_cols(self):
        cells = self.T.cells
        ne, nv, A = len(cells), self.nv, self.A
        vi = np.broadcast_to(cells[:, :, None, None], (ne, nv, nv, A))
        vj = np.broadcast_to(cells[:, None, :, None], (ne, nv, nv, A))
        a = np.broadcast_to(np.arange(A)[None, None, None, :], (ne, nv, nv, A))
        return vi, vj, a

    def supg_matrix(self):
        """Streaming + SUPG streaming + removal + the weak boundary terms
        (SUPGFillKernel): row (i, a), per element of i's star and vertex j,
        (Omega.G_ij + tau Omega Omega : K_ij + sigma_t (M_ij + tau Omega.G_ji)) / m_i;
        per inflow boundary face |s| m^f_i / m_i on the diagonal, its negative
        at the mirrored ordinate on a reflective face."""
        T, om = self.T, self.omega
        tau = self.tau()
        og_ij = np.einsum("eijd,ad->eija", T.grad, om)
        og_ji = np.einsum("ejid,ad->eija", T.grad, om)
        oko = np.einsum("eijdf,ad,af->eija", T.stiff, om, om)
        coef = og_ij + tau[:, None, None, :] * oko + self.sigma_t[:, None, None, None] * (
            T.mass[:, :, :, None] + tau[:, None, None, :] * og_ji)
        vi, vj, a = self._rows_cols()
        coef = coef / T.lumped[vi]
        rows = [(vi * self.A + a).ravel()]
        cols = [(vj * self.A + a).ravel()]
        vals = [coef.ravel()]
        br, bc, bv = self._boundary_entries()
        rows.append(br)
        cols.append(bc)
        vals.append(bv)
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(self.n, self.n))

    def _boundary_entries(self):
        rows, cols, vals = [], [], []
        A = self.A
        for fv, n, s in zip(self.B.verts, self.B.nA, self.B.side):
            flux = self.omega @ n
            inflow = np.nonzero(flux < 0)[0]
            for v in fv:
                c = -flux[inflow] / (self.T.lumped[v] * len(fv))
                rows.append(v * A + inflow)
                cols.append(v * A + inflow)
                vals.append(c)
                if self.side_bc[s] == BC_REFLECT:
                    rows.append(v * A + inflow)
                    cols.append(v * A + self.reflect[s // 2][inflow])
                    vals.append(-c)
        if not rows:
            return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0)
        return np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)

    def weighted_load(self, coeff, sigma_t=None):
        """WL (n_rows x n_vertices): row (i, a), column j,
        1 / m_i sum_{e in star(i) with j} coeff_e (M_ij + tau_{e,a} Omega_a . G_ji)
        (WeightedLoadKernel, unstructured_cgk.kokkos.cxx:676-709)."""
        T = self.T
        tau = self.tau(sigma_t)
        og_ji = np.einsum("ejid,ad->eija", T.grad, self.omega)
        wgt = np.asarray(coeff, dtype=float)[:, None, None, None] * (
            T.mass[:, :, :, None] + tau[:, None, None, :] * og_ji)
        vi, vj, a = self._rows_cols()
        wgt = wgt / T.lumped[vi]
        return sp.csr_matrix((wgt.ravel(), ((vi * self.A + a).ravel(), vj.ravel())),
                             shape=(self.n, self.n_vertices))

    def integral(self):
        """Q (n_vertices x n_rows): phi(v) = sum_a w_a psi(v, a)."""
        nvx, A = self.n_vertices, self.A
        r = np.repeat(np.arange(nvx), A)
        c = np.arange(nvx * A)
        return sp.csr_matrix((np.tile(self.w, nvx), (r, c)), shape=(nvx, nvx * A))

    def scatter_matrix(self):
        """S = (1 / W) WL(sigma_s) Q (ScatteringTermCG::apply_add, terms_cgk.kokkos.cxx:203-221)."""
        return (self.weighted_load(self.sigma_s) @ self.integral()) / self.W

    def matrix(self):
        return (self.supg_matrix() - self.scatter_matrix()).tocsr()

    def source(self, q_elem):
        """b += (1 / W) WL(q) 1 (UboltFillSourceCG, terms_cgk.kokkos.cxx:340-356)."""
        return self.weighted_load(q_elem) @ np.ones(self.n_vertices) / self.W

    def transfer(self, phi_from, sigma_s_from_to):
        """b += (1 / W) WL(sigma_s(g' -> g)) phi(g'), tau of this group (GroupTransferCG::add_transfer)."""
        return self.weighted_load(sigma_s_from_to) @ np.asarray(phi_from, dtype=float) / self.W

    def ghost_inflow(self, side_inflow):
        """The weak vacuum inflow: per inflow face of a vacuum side,
        |s| m^f_i / m_i * inflow / W (unstructured_cgk.kokkos.cxx:508-520)."""
        b = np.zeros(self.n)
        for fv, n, s in zip(self.B.verts, self.B.nA, self.B.side):
            if self.side_bc[s] != BC_VACUUM or side_inflow[s] == 0.0:
                continue
            flux = self.omega @ n
            inflow = np.nonzero(flux < 0)[0]
            for v in fv:
                b[v * self.A + inflow] += -flux[inflow] / (self.T.lumped[v] * len(fv)) * side_inflow[s] / self.W
        return b

    # ~~~ The CG DSA (dsa_cgk.kokkos.cxx)

    def supg_d(self):
        """The SUPG operator's own diffusion tensor per element,
        (1 / W) sum_a w_a tau_a Omega_a Omega_a^T (CGSupgDKernel, :66-84)."""
        tau = self.tau()
        return np.einsum("a,ea,ad,af->edf", self.w, tau, self.omega, self.omega) / self.W

    def void_policy(self, void_sigma_t=0.0, bridge=True, void_d=0.0):
        """DSAPrecon::assemble on a backend that cannot mask (dsak.kokkos.cxx:
        233-345): the census, the singular guard, the bridge and the voids'
        mean chord 4 V / S (DSACG::void_volume_surface, dsa_cgk.kokkos.cxx:
        227-243), and D per element (zero in an unbridged void)."""
        st, ss = self.sigma_t, self.sigma_s
        is_void = st <= void_sigma_t
        any_vac = bool(np.any(self.side_bc[self.B.side] == BC_VACUUM)) if len(self.B.side) else False
        if not (any_vac or np.max(st - ss) > 0.0):
            raise ValueError("the DSA diffusion operator is singular")
        bridged, chord = False, 0.0
        if bridge and is_void.any():
            vol = self.T.volume[is_void].sum()
            nbr = self.B.elem_nbr[is_void]
            area = self.B.elem_area[is_void]
            bc = self.B.elem_bc[is_void]
            into = np.where(nbr >= 0, ~is_void[np.maximum(nbr, 0)], bc == BC_VACUUM)
            surf = area[into].sum()
            chord = 4.0 * vol / surf if surf > 0 else 0.0
            bridged = chord > 0
        d = np.zeros(len(st))
        d[~is_void] = 1.0 / (3.0 * st[~is_void])
        if bridged:
            d[is_void] = void_d if void_d > 0 else 1.0 / (3.0 * (np.maximum(st[is_void], 0.0) + 1.0 / chord))
        return is_void, bridged, chord, d

    def dsa_matrix(self, void_sigma_t=0.0, bridge=True, void_d=0.0):
        """D (n_vertices x n_vertices): sum_e (sigma_t - sigma_s) M_ij + D_e : K_ij,
        D_e isotropic from the void policy, the SUPG tensor in an unbridged
        void; plus per vertex its vacuum faces' half-range current times
        A_f / n_face_vertices (DSACG::create/assemble, dsa_cgk.kokkos.cxx:
        114-203, 247-281)."""
        T = self.T
        is_void, bridged, chord, d = self.void_policy(void_sigma_t, bridge, void_d)
        De = np.einsum("e,df->edf", d, np.eye(3))
        if is_void.any() and not bridged:
            De[is_void] = self.supg_d()[is_void]
        vals = (self.sigma_t - self.sigma_s)[:, None, None] * T.mass + np.einsum("edf,eijdf->eij", De, T.stiff)
        cells = T.cells
        nv = self.nv
        r = np.broadcast_to(cells[:, :, None], (len(cells), nv, nv)).ravel()
        c = np.broadcast_to(cells[:, None, :], (len(cells), nv, nv)).ravel()
        diag = np.zeros(self.n_vertices)
        for fv, n, s in zip(self.B.verts, self.B.nA, self.B.side):
            if self.side_bc[s] != BC_VACUUM:
                continue
            area = np.linalg.norm(n)
            cosv = -(self.omega @ n) / area
            m = np.sum(np.where(cosv > 0, self.w * cosv, 0.0)) / self.W
            for v in fv:
                diag[v] += m * area / len(fv)
        D = sp.csr_matrix((vals.ravel(), (r, c)), shape=(self.n_vertices, self.n_vertices))
        return (D + sp.diags(diag)).tocsr(), dict(is_void=is_void, bridged=bridged, chord=chord, d=d)

    def dsa_restrict(self, x):
        """rhs(i) = m_i sum_a w_a x(i, a): the transport rows are per unit
        volume, the diffusion rows the weak form (dsa_cgk.kokkos.cxx:190-200)."""
        return self.T.lumped * (self.integral() @ x)

    def dsa_prolong(self, u):
        return np.repeat(np.asarray(u) / self.W, self.A)
