"""The library's CG-SUPG host tables (ubolt_cg_geometry_build) against the
oracle's own (oracle/cg.py), computed independently from the same vertices
and cells: element matrices, centroid gradients, volumes, lumped masses,
the boundary faces each vertex sees and every element's faces."""
import numpy as np
import pytest

import cg as OC
from ubolt_b200 import _lib
from ubolt_b200 import problem as P

from test_cg_oracle import ALL


def close(a, b, tol=1e-13):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(np.asarray(a) - np.asarray(b)).max() <= tol * scale


@pytest.mark.parametrize("name,mesh,L", ALL, ids=[a[0] for a in ALL])
def test_cg_tables_match_the_oracle(name, mesh, L):
    sbc = [1, 0] * mesh.dim
    g = P.build_cg_geometry(mesh, side_bc=sbc)
    T = OC.Tables(mesh)
    ne, nv = T.cells.shape
    assert g.n_elements == ne and g.n_element_vertices == nv and g.n_vertices == T.n_vertices
    assert np.array_equal(g.elem_vertex.reshape(ne, nv), T.cells)
    assert close(g.mass.reshape(ne, nv, nv), T.mass)
    assert close(g.grad.reshape(ne, nv, nv, 3), T.grad)
    assert close(g.stiff.reshape(ne, nv, nv, 3, 3), T.stiff)
    assert close(g.centre_grad.reshape(ne, nv, 3), T.centre_grad)
    assert close(g.volume, T.volume)
    assert close(g.centroid.reshape(ne, 3)[:, :mesh.dim], T.centroid)
    assert close(g.lumped_mass, T.lumped)
    # Stars: every (element, basis index) once, under its vertex
    so, se, sl = g.star_offset, g.star_elem, g.star_li
    got = sorted((int(v), int(se[s]), int(sl[s])) for v in range(g.n_vertices) for s in range(so[v], so[v + 1]))
    want = sorted((int(T.cells[e, li]), e, li) for e in range(ne) for li in range(nv))
    assert got == want


@pytest.mark.parametrize("name,mesh,L", ALL, ids=[a[0] for a in ALL])
def test_cg_boundary_faces_match_the_oracle(name, mesh, L):
    sbc = [1, 0] * mesh.dim
    g = P.build_cg_geometry(mesh, side_bc=sbc)
    pr_T = OC.Tables(mesh)
    B = OC.BoundaryFaces(mesh, pr_T, np.asarray(sbc))
    bo = g.bface_offset
    got = sorted((int(v), int(g.bface_side[f]), int(g.bface_bc[f]), *np.round(g.bface_nA[3 * f:3 * f + 3], 12),
                  round(float(g.bface_mass[f]), 12))
                 for v in range(g.n_vertices) for f in range(bo[v], bo[v + 1]))
    want = sorted((v, int(s), int(sbc[s]), *np.round(n, 12), round(1.0 / (pr_T.lumped[v] * len(fv)), 12))
                  for fv, n, s in zip(B.verts, B.nA, B.side) for v in fv)
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert a[:3] == b[:3] and np.allclose(a[3:], b[3:], rtol=0, atol=1e-11)
    F = g.faces_per_element
    assert np.array_equal(g.elem_face_neighbour.reshape(-1, F), B.elem_nbr)
    assert close(g.elem_face_area.reshape(-1, F), B.elem_area)
    assert np.array_equal(g.elem_face_bc.reshape(-1, F), B.elem_bc)


def test_cg_reflective_face_must_be_axis_aligned():
    """A slanted reflective face is refused (UnstructuredCG's PETSC_ERR_SUP,
    unstructured_cg.hpp:69-71); the same mesh with that side vacuum builds."""
    mesh = P.Mesh(2, P.TRI, np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]], dtype=np.int64))
    # The hypotenuse's normal (1, 1) ties between the axes: its side is high x
    with pytest.raises(_lib.UboltError) as e:
        P.build_cg_geometry(mesh, side_bc=[0, 1, 0, 0])
    assert e.value.status == 1
    g = P.build_cg_geometry(mesh, side_bc=[0, 0, 1, 0])
    assert g.n_vertices == 3 and abs(g.lumped_mass.sum() - 0.5) < 1e-15
