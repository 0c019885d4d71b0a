"""The oracle's own DG0/DG1 geometry - TEST INFRASTRUCTURE ONLY.

An independent NumPy restatement of what UnstructuredDG::create and
UnstructuredDG::build_dg1_geometry compute (src/unstructured_dgk.kokkos.cxx
of stevendargaville/UBOLT), so that the parity tests compare the library's
kernels against geometry the library did not compute:

* cell and face moments (unstructured_dgk.kokkos.cxx:27-182) - here from a
  different exact decomposition: closed-form simplex moments, quads split
  into two triangles, hexes into six tets about a main diagonal (exact for
  planar faces, which every mesh the tests build has);
* the orthonormal modal P1 basis (:184-218) - here by Gram-Schmidt of the
  coordinate directions in the inner product (1/V) int f g, which gives the
  same basis as the reference's Cholesky of the normalised central moment;
* outward area normals (src/plex_commonk.hpp:291-307), the dominant axis
  (:282-289) and the centroid-to-face distances (:363-371);
* the face matrices face_own / face_up (unstructured_dgk.kokkos.cxx:
  747-821), here int_f phi_i phi_j by Gauss quadrature exact for quadratics
  (two points on a segment, the edge midpoints on a triangle) rather than
  the reference's centroid-value-plus-second-moment formula.

Faces are matched by their vertex sets; a cell's face slots follow the same
per-shape local face order as the library (the order is a layout convention
both sides must share for face-indexed arrays to line up).
"""
from types import SimpleNamespace

import numpy as np

TRI, QUAD, TET, HEX = 3, 4, 10, 12
VACUUM, REFLECT = 0, 1

# Local faces, as vertex indices into the cell's vertex list
FACES = {
    TRI: [(0, 1), (1, 2), (2, 0)],
    QUAD: [(0, 1), (1, 2), (2, 3), (3, 0)],
    TET: [(1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)],
    HEX: [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)],
}
DIM = {TRI: 2, QUAD: 2, TET: 3, HEX: 3}
# Exact simplex decompositions of a cell
CELL_SIMPLICES = {
    TRI: [(0, 1, 2)],
    QUAD: [(0, 1, 2), (0, 2, 3)],
    TET: [(0, 1, 2, 3)],
    HEX: [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)],
}


def _simplex_moments(pts, measure):
    """Measure-weighted centroid and central second moment of simplices:
    int (x - c)(x - c)^T = m / ((d + 1)(d + 2)) sum_i (v_i - c)(v_i - c)^T."""
    k = pts.shape[1]  # vertices per simplex, d + 1
    c = pts.mean(axis=1)
    y = pts - c[:, None, :]
    central = np.einsum("nki,nkj->nij", y, y) * (measure / (k * (k + 1)))[:, None, None]
    return c, central


def _combine(parts):
    """Moments of a union from its parts' (measure, centroid, central)."""
    m = sum(p[0] for p in parts)
    c = sum(p[0][:, None] * p[1] for p in parts) / m[:, None]
    central = np.zeros((len(m), 3, 3))
    for mi, ci, Ci in parts:
        d = ci - c
        central += Ci + mi[:, None, None] * np.einsum("ni,nj->nij", d, d)
    return m, c, central


def _triangle_measure(p):
    return 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)


def _cell_moments(ctype, X):
    parts = []
    for simp in CELL_SIMPLICES[ctype]:
        p = X[:, list(simp)]
        if DIM[ctype] == 2:
            m = _triangle_measure(p)
        else:
            m = np.abs(np.einsum("ni,ni->n", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))) / 6.0
        c, C = _simplex_moments(p, m)
        parts.append((m, c, C))
    return _combine(parts)


def _face_moments_and_rule(dim, P):
    """Area, centroid, unit normal (vertex-cycle orientation) and a quadrature
    rule exact for quadratics (points (n, q, 3), weights (n, q))."""
    if dim == 2:
        e = P[:, 1] - P[:, 0]
        L = np.linalg.norm(e, axis=1)
        c = 0.5 * (P[:, 0] + P[:, 1])
        normal = np.stack([e[:, 1], -e[:, 0], np.zeros(len(e))], axis=1) / L[:, None]
        g = 0.5 / np.sqrt(3.0)
        pts = np.stack([c - g * e, c + g * e], axis=1)
        wts = np.stack([0.5 * L, 0.5 * L], axis=1)
        return L, c, normal, pts, wts
    tris = [(0, 1, 2)] if P.shape[1] == 3 else [(0, 1, 2), (0, 2, 3)]
    area = np.zeros(len(P))
    first = np.zeros((len(P), 3))
    vec = np.zeros((len(P), 3))
    pts, wts = [], []
    for t in tris:
        p = P[:, list(t)]
        cr = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        a = 0.5 * np.linalg.norm(cr, axis=1)
        vec += 0.5 * cr
        area += a
        first += a[:, None] * p.mean(axis=1)
        for (i, j) in ((0, 1), (1, 2), (2, 0)):
            pts.append(0.5 * (p[:, i] + p[:, j]))
            wts.append(a / 3.0)
    c = first / area[:, None]
    normal = vec / np.linalg.norm(vec, axis=1)[:, None]
    return area, c, normal, np.stack(pts, axis=1), np.stack(wts, axis=1)


def _basis(dim, V, central):
    """Gradients beta[n, i, :] of the modes phi_{i+1} = beta_i . (x - centroid):
    Gram-Schmidt of the coordinate directions in <a, b> = a^T (M / V) b."""
    M = central / V[:, None, None]
    beta = np.zeros((len(V), 3, 3))
    for i in range(dim):
        a = np.zeros((len(V), 3))
        a[:, i] = 1.0
        for k in range(i):
            proj = np.einsum("ni,nij,nj->n", a, M, beta[:, k])
            a = a - proj[:, None] * beta[:, k]
        nrm = np.sqrt(np.einsum("ni,nij,nj->n", a, M, a))
        beta[:, i] = a / nrm[:, None]
    return beta


def build(dim, cell_type, vertices, cells, order, side_bc=None):
    """The geometry arrays, in the library's flat per-(cell, slot) layout."""
    assert DIM[cell_type] == dim and order in (0, 1)
    faces = FACES[cell_type]
    F = len(faces)
    nc = len(cells)
    nb = 1 if order == 0 else dim + 1
    sbc = np.zeros(2 * dim, dtype=np.int32) if side_bc is None else np.asarray(side_bc, dtype=np.int32)
    V3 = np.zeros((len(vertices), 3))
    V3[:, :dim] = vertices
    X = V3[np.asarray(cells)]                                   # (nc, nvc, 3)
    vol, cen, central = _cell_moments(cell_type, X)
    lo, hi = V3.min(axis=0), V3.max(axis=0)

    # Faces: moments, outward normals, neighbours by vertex set
    area = np.zeros((nc, F))
    fcen = np.zeros((nc, F, 3))
    nA = np.zeros((nc, F, 3))
    rules = []
    key_of = {}
    nbr = np.full((nc, F), -1, dtype=np.int64)
    cells_a = np.asarray(cells)
    for f, fv in enumerate(faces):
        a, c, n, qp, qw = _face_moments_and_rule(dim, X[:, list(fv)])
        outward = np.einsum("ni,ni->n", n, c - cen)
        n = np.where(outward[:, None] < 0.0, -n, n)
        area[:, f], fcen[:, f], nA[:, f] = a, c, a[:, None] * n
        rules.append((qp, qw))
        for cell in range(nc):
            key = tuple(sorted(cells_a[cell, list(fv)]))
            other = key_of.pop(key, None)
            if other is None:
                key_of[key] = (cell, f)
            else:
                nbr[cell, f] = other[0]
                nbr[other] = cell
    axis = np.argmax(np.abs(nA[:, :, :dim]), axis=2)  # lowest axis on a tie
    unit = nA / area[:, :, None]
    dist = np.zeros((nc, F, 2))
    dist[:, :, 0] = np.einsum("nfi,nfi->nf", unit, fcen - cen[:, None, :])
    inner = nbr >= 0
    dist[:, :, 1] = np.where(inner, np.einsum("nfi,nfi->nf", unit, cen[np.maximum(nbr, 0)] - fcen), 0.0)
    side = np.where(inner, -1, 2 * axis + (np.take_along_axis(nA, axis[:, :, None], 2)[:, :, 0] > 0))
    bc = np.where(inner, -1, sbc[np.maximum(side, 0)]).astype(np.int32)
    # Boundary faces lie on the side of the box they are labelled by
    on = np.where(side >= 0, np.take_along_axis(fcen, axis[:, :, None], 2)[:, :, 0], 0.0)
    plane = np.where(side % 2 == 1, hi[axis], lo[axis])
    assert np.all(np.abs(on - plane)[~inner] <= 1e-9 * np.max(hi - lo)), "a boundary face off the box"

    out = dict(volume=vol, centroid=cen.ravel(), face_nA=nA.ravel(), face_neighbour=nbr.ravel(),
               face_bc=bc.ravel(), face_side=side.astype(np.int32).ravel(), face_axis=axis.astype(np.int32).ravel(),
               face_centroid=fcen.ravel(), face_distance=dist.ravel())
    if order == 1:
        beta = _basis(dim, vol, central)

        def phi(cell_idx, x):
            """All nb mode values of cells cell_idx at points x (n, q, 3) -> (n, q, nb)."""
            y = x - cen[cell_idx][:, None, :]
            lin = np.einsum("nqd,nid->nqi", y, beta[cell_idx][:, :dim])
            return np.concatenate([np.ones(lin.shape[:2] + (1,)), lin], axis=2)

        own = np.zeros((nc, F, nb, nb))
        up = np.zeros((nc, F, nb, nb))
        fbv = np.zeros((nc, F, nb))
        nbgrad = np.zeros((nc, F, nb, 3))
        idx = np.arange(nc)
        for f in range(F):
            qp, qw = rules[f]
            pc = phi(idx, qp)
            scale = 1.0 / (vol * area[:, f])
            own[:, f] = np.einsum("nq,nqi,nqj->nij", qw, pc, pc) * scale[:, None, None]
            other = np.where(inner[:, f], nbr[:, f], np.where(bc[:, f] == REFLECT, idx, -1))
            has = other >= 0
            po = phi(np.maximum(other, 0), qp)
            up[:, f] = np.where(has[:, None, None], np.einsum("nq,nqi,nqj->nij", qw, pc, po) * scale[:, None, None],
                                0.0)
            fbv[:, f] = phi(idx, fcen[:, f][:, None, :])[:, 0]
            g_nb = np.zeros((nc, nb, 3))
            g_nb[:, 1:, :] = beta[np.maximum(nbr[:, f], 0)][:, :dim]
            nbgrad[:, f] = np.where(inner[:, f][:, None, None], g_nb, 0.0)
        grad = np.zeros((nc, nb, 3))
        grad[:, 1:, :] = beta[:, :dim]
        out.update(face_own=own.ravel(), face_up=up.ravel(), basis_grad=grad.ravel(), face_neighbour_grad=nbgrad.ravel(),
                   face_basis_value=fbv.ravel())
    return SimpleNamespace(dim=dim, n_basis=nb, faces_per_cell=F, n_cells=nc, **out)
