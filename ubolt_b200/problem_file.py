"""UBOLT's JSON problem files and Gmsh 2.2 meshes, read into a Problem.

A problem file (docs/problem_files.md, parsed by the reference's ProblemSpec,
include/ubolt/problem_spec.hpp) names everything physical about a fixed-source
solve: dimension, mesh, S_N order, materials, painted regions and boundary
conditions. load() reads one into this library's Problem, on the backends
this library runs:

- structured 2D/3D boxes run as their DG0 twin on the uniform quad/hex box
  (the same stencil to rounding, docs/problem_files.md "Unstructured meshes");
- unstructured boxes (quads/hexes, or with "simplex" every quad split into two
  triangles along one diagonal, every hex into Kuhn's six tetrahedra) and
  Gmsh 2.2 file meshes, at DG0, DG1 or CG-SUPG.

The file is STRICT as in the reference: an unknown key is an error. What the
schema allows but this library does not run raises Unsupported, naming it:
1D slabs (no 1D backend), "dirichlet_cell" vacuum faces, inflow windows, and
boundary faces off the mesh's bounding box. "output" is accepted and not
written (this library writes no VTK files).
"""
import json
import os

import numpy as np

from . import problem as P

BC_VACUUM, BC_REFLECT = 0, 1


class Unsupported(ValueError):
    """A schema feature this library does not run."""


class SpecError(ValueError):
    """A malformed problem file."""


_TOP = {"_comment", "dimension", "mesh", "sn_order", "materials", "regions", "boundary_conditions",
        "vacuum_treatment", "output"}
_MESH = {"_comment", "type", "n_cells", "lengths", "order", "discretisation", "supg_zeta", "simplex", "file"}
_REGIONS = {"_comment", "background", "paint", "cell_sets"}
_FACE = {"_comment", "type", "inflow", "window"}
# Face names -> this library's side (2 axis + high): the reference's face names
# (x faces left/right everywhere; y faces bottom/top in 2D, front/back in 3D;
# z faces bottom/top in 3D)
_SIDES = {2: {"left": 0, "right": 1, "bottom": 2, "top": 3},
          3: {"left": 0, "right": 1, "front": 2, "back": 3, "bottom": 4, "top": 5}}
# PETSc box meshes' "Face Sets" ids -> side (docs/problem_files.md, "Unstructured meshes")
_BOX_FACE_SETS = {2: {1: 2, 2: 1, 3: 3, 4: 0}, 3: {1: 4, 2: 5, 3: 2, 4: 3, 5: 1, 6: 0}}


def _check_keys(obj, allowed, where):
    if not isinstance(obj, dict):
        raise SpecError(f"{where}: an object is required")
    extra = sorted(set(obj) - allowed)
    if extra:
        raise SpecError(f"{where}: unknown key(s) {extra}")


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# Gmsh 2.2 (ASCII)
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

# Gmsh element type -> (dimension, vertices, this library's cell shape or None)
_GMSH_TYPES = {1: (1, 2, None), 2: (2, 3, P.TRI), 3: (2, 4, P.QUAD), 4: (3, 4, P.TET), 5: (3, 8, P.HEX),
               15: (0, 1, None)}


def read_gmsh(path, dim):
    """A Gmsh 2.2 ASCII mesh: (Mesh, cell_sets, face_sets). The cells are the
    elements of dimension `dim` (one shape), cell_sets[c] their first
    (physical) tag; face_sets maps each boundary element of dimension dim - 1,
    as the sorted tuple of its vertex indices, to its physical tag - the
    reference's "Cell Sets" and "Face Sets" labels."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    i = 0
    nodes, elems = {}, []
    while i < len(lines):
        tag = lines[i]
        if tag == "$MeshFormat":
            ver = lines[i + 1].split()
            if not ver[0].startswith("2.") or ver[1] != "0":
                raise Unsupported(f"{path}: Gmsh format {ver[0]} (file type {ver[1]}); 2.x ASCII is read")
        elif tag == "$Nodes":
            n = int(lines[i + 1])
            for ln in lines[i + 2:i + 2 + n]:
                t = ln.split()
                nodes[int(t[0])] = [float(v) for v in t[1:4]]
            i += n + 1
        elif tag == "$Elements":
            n = int(lines[i + 1])
            for ln in lines[i + 2:i + 2 + n]:
                t = [int(v) for v in ln.split()]
                et, ntag = t[1], t[2]
                if et not in _GMSH_TYPES:
                    raise Unsupported(f"{path}: Gmsh element type {et}")
                phys = t[3] if ntag > 0 else -1
                elems.append((et, phys, t[3 + ntag:]))
            i += n + 1
        i += 1
    ids = sorted(nodes)
    index = {k: j for j, k in enumerate(ids)}
    verts = np.array([nodes[k][:dim] for k in ids], dtype=np.float64)
    cells = [(et, phys, vs) for et, phys, vs in elems if _GMSH_TYPES[et][0] == dim]
    shapes = {_GMSH_TYPES[et][2] for et, _, _ in cells}
    if len(shapes) != 1:
        raise Unsupported(f"{path}: {len(shapes)} cell shapes of dimension {dim}; one shape per mesh is run")
    cv = np.array([[index[v] for v in vs] for _, _, vs in cells], dtype=np.int64)
    cell_sets = np.array([phys for _, phys, _ in cells], dtype=np.int64)
    face_sets = {}
    for et, phys, vs in elems:
        if _GMSH_TYPES[et][0] == dim - 1:
            face_sets[tuple(sorted(index[v] for v in vs))] = phys
    return P.Mesh(dim, shapes.pop(), verts, cv, ()), cell_sets, face_sets


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# Materials
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

def read_materials(spec, base_dir):
    """The multigroup materials table (docs/problem_files.md, "The materials
    schema"; TOLERANT of unknown keys): (n_groups, [{name, sigma_t[G],
    sigma_s[G][G] (from, to), source[G]}] indexed by the dense ids)."""
    if isinstance(spec, str):
        with open(os.path.join(base_dir, spec)) as f:
            spec = json.load(f)
    if not isinstance(spec, dict):
        raise SpecError("materials: a path or an object is required")
    if spec.get("representation", "multigroup") != "multigroup":
        raise Unsupported(f"materials representation {spec['representation']!r}")
    G = spec.get("n_groups")
    if not isinstance(G, int) or G < 1:
        raise SpecError("materials.n_groups must be a positive integer")
    mats = spec.get("materials")
    if not isinstance(mats, list) or not mats:
        raise SpecError("materials.materials must be a non-empty array")
    out = [None] * len(mats)
    for m in mats:
        mid = m.get("id")
        if not isinstance(mid, int) or not 0 <= mid < len(mats) or out[mid] is not None:
            raise SpecError(f"material ids must be dense 0..{len(mats) - 1} (got {mid!r})")
        st = np.asarray(m["Sigma_t"], dtype=np.float64)
        ss = np.asarray(m["Sigma_s"], dtype=np.float64)
        src = np.asarray(m.get("Source", [0.0] * G), dtype=np.float64)
        if st.shape != (G,) or ss.shape != (G, G) or src.shape != (G,):
            raise SpecError(f"material {mid}: Sigma_t [G], Sigma_s [G][G] and Source [G] are required, G = {G}")
        out[mid] = {"name": m.get("name"), "sigma_t": st, "sigma_s": ss, "source": src}
    return G, out


def _material_index(ref, mats, where):
    if isinstance(ref, int) and 0 <= ref < len(mats):
        return ref
    for i, m in enumerate(mats):
        if m["name"] is not None and m["name"] == ref:
            return i
    raise SpecError(f"{where}: no material {ref!r}")


# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
# The problem
# ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

def _box_mesh(dim, n, lengths, shape):
    if dim == 2:
        if shape == "simplex":
            return P.box_tris(n[0], n[1], lengths[0], lengths[1], diagonals="uniform")
        return P.box_quads(n[0], n[1], lengths[0], lengths[1])
    if shape == "simplex":
        return P.box_tets(n[0], n[1], n[2], lx=lengths[0], ly=lengths[1], lz=lengths[2])
    return P.box_hexes(n[0], n[1], n[2], lengths[0], lengths[1], lengths[2])


def _face_side_of_set(mesh, faces, tag):
    """The bounding-box side every face of a "Face Sets" value lies on."""
    lo, hi = mesh.vertices.min(axis=0), mesh.vertices.max(axis=0)
    sides = set()
    for vs in faces:
        pts = mesh.vertices[list(vs)]
        found = None
        for d in range(mesh.dim):
            for high, plane in ((0, lo[d]), (1, hi[d])):
                if np.all(np.abs(pts[:, d] - plane) <= 1e-9 * max(1.0, hi[d] - lo[d])):
                    found = 2 * d + high
        if found is None:
            raise Unsupported(f"Face Sets value {tag}: a face off the mesh's bounding box (only box-side "
                              "boundaries are run)")
        sides.add(found)
    if len(sides) != 1:
        raise Unsupported(f"Face Sets value {tag} spans {len(sides)} sides of the box; one side per value is run")
    return sides.pop()


def load(path, order=None):
    """Read a problem file into a Problem (meta carries the problem's name,
    backend, mesh source and zeta). `order` overrides mesh.order."""
    base_dir = os.path.dirname(os.path.abspath(path))
    with open(path) as f:
        spec = json.load(f)
    return from_spec(spec, base_dir, name=os.path.splitext(os.path.basename(path))[0], order=order)


def from_spec(spec, base_dir=".", name="problem", order=None):
    _check_keys(spec, _TOP, "problem")
    dim = spec.get("dimension")
    if dim not in (1, 2, 3):
        raise SpecError("dimension must be 1, 2 or 3")
    if dim == 1:
        raise Unsupported("1D slab problems: this library has no 1D backend")
    mesh_spec = spec.get("mesh", {})
    _check_keys(mesh_spec, _MESH, "mesh")
    mtype = mesh_spec.get("type", "structured")
    if mtype not in ("structured", "unstructured"):
        raise SpecError(f"mesh.type {mtype!r}")
    disc = mesh_spec.get("discretisation", "dg")
    if disc not in ("dg", "cg_supg"):
        raise SpecError(f"mesh.discretisation {disc!r}")
    if mtype == "structured" and any(k in mesh_spec for k in ("order", "discretisation", "simplex", "file")):
        raise SpecError("mesh.order, discretisation, simplex and file are unstructured only")
    dg_order = order if order is not None else int(mesh_spec.get("order", 0 if disc == "dg" else 1))
    if disc == "cg_supg" and dg_order != 1:
        raise SpecError("a cg_supg mesh is linear: order 1 or left out")
    if dg_order not in (0, 1):
        raise SpecError("mesh.order must be 0 or 1")
    vt = spec.get("vacuum_treatment", "ghost_flux")
    if vt == "dirichlet_cell":
        raise Unsupported("vacuum_treatment dirichlet_cell (this library runs ghost-flux faces)")
    if vt != "ghost_flux":
        raise SpecError(f"vacuum_treatment {vt!r}")

    cell_sets = face_sets = None
    if "file" in mesh_spec:
        if any(k in mesh_spec for k in ("n_cells", "lengths", "simplex")):
            raise SpecError("mesh.n_cells, lengths and simplex are errors beside mesh.file")
        mesh, cell_sets, face_sets = read_gmsh(os.path.join(base_dir, mesh_spec["file"]), dim)
        source = mesh_spec["file"]
    else:
        n, lengths = mesh_spec.get("n_cells"), mesh_spec.get("lengths")
        if (not isinstance(n, list) or len(n) != dim or not all(isinstance(v, int) and v > 0 for v in n) or
                not isinstance(lengths, list) or len(lengths) != dim or not all(v > 0 for v in lengths)):
            raise SpecError(f"mesh.n_cells and mesh.lengths need {dim} positive entries")
        mesh = _box_mesh(dim, n, [float(v) for v in lengths], "simplex" if mesh_spec.get("simplex") else "box")
        source = f"box {n} x {lengths}" + (" simplex" if mesh_spec.get("simplex") else "")

    # Boundary conditions per side
    side_bc = np.zeros(2 * dim, dtype=np.int32)
    side_in = np.zeros(2 * dim)
    named = {}
    for key, val in (spec.get("boundary_conditions") or {}).items():
        if key == "_comment":
            continue
        if key in _SIDES[dim]:
            side = _SIDES[dim][key]
        elif key.isdigit():
            if mtype == "structured":
                raise SpecError(f"boundary_conditions: a Face Sets key {key!r} on a structured mesh")
            tag = int(key)
            if face_sets is None:
                if tag not in _BOX_FACE_SETS[dim]:
                    raise SpecError(f"boundary_conditions: no box face carries Face Sets value {tag}")
                side = _BOX_FACE_SETS[dim][tag]
            else:
                faces = [vs for vs, t in face_sets.items() if t == tag]
                if not faces:
                    raise SpecError(f"boundary_conditions: no boundary face carries Face Sets value {tag}")
                side = _face_side_of_set(mesh, faces, tag)
        else:
            raise SpecError(f"boundary_conditions: unknown face {key!r}")
        if side in named:
            raise SpecError(f"boundary_conditions: {key!r} and {named[side]!r} name the same face")
        named[side] = key
        if isinstance(val, str):
            val = {"type": val}
        _check_keys(val, _FACE, f"boundary_conditions.{key}")
        fam = val.get("type")
        if fam not in ("vacuum", "reflect"):
            raise SpecError(f"boundary_conditions.{key}: type must be vacuum or reflect")
        if fam == "reflect" and ("inflow" in val or "window" in val):
            raise SpecError(f"boundary_conditions.{key}: inflow and window are vacuum-only")
        if "window" in val:
            raise Unsupported(f"boundary_conditions.{key}: inflow windows (the library's inflow is per side)")
        side_bc[side] = BC_REFLECT if fam == "reflect" else BC_VACUUM
        side_in[side] = float(val.get("inflow", 0.0))

    if disc == "cg_supg":
        geom = P.build_cg_geometry(mesh, side_bc=side_bc)
        centroids = geom.centroid.reshape(-1, 3)
    else:
        geom = P.build_geometry(mesh, dg_order, side_bc=side_bc)
        centroids = geom.centroid.reshape(-1, 3)
    nc = geom.n_cells
    sn = spec.get("sn_order")
    if not isinstance(sn, int) or sn < 2 or sn % 2 or sn > 18:
        raise SpecError("sn_order must be an even integer 2..18 in 2D and 3D")
    quad = P.lqn(dim, sn)

    # Materials painted: background, then Cell Sets, then paint boxes by centroid
    if "materials" not in spec:
        raise SpecError("materials is required")
    G, mats = read_materials(spec["materials"], base_dir)
    regions = spec.get("regions") or {}
    _check_keys(regions, _REGIONS, "regions")
    mat = np.full(nc, _material_index(regions.get("background", 0), mats, "regions.background"), dtype=np.int64)
    if "cell_sets" in regions:
        if mtype == "structured":
            raise SpecError("regions.cell_sets on a structured mesh")
        labels = cell_sets if cell_sets is not None else np.full(nc, -1)
        for key, ref in regions["cell_sets"].items():
            if key == "_comment":
                continue
            mat[labels == int(key)] = _material_index(ref, mats, f"regions.cell_sets.{key}")
    for k, entry in enumerate(regions.get("paint", [])):
        box = np.asarray(entry.get("box"), dtype=np.float64)
        if box.shape != (2 * dim,) or np.any(box[0::2] > box[1::2]):
            raise SpecError(f"regions.paint[{k}]: box needs {2 * dim} numbers, lo <= hi per axis")
        inside = np.ones(nc, dtype=bool)
        for d in range(dim):
            inside &= (centroids[:, d] >= box[2 * d]) & (centroids[:, d] <= box[2 * d + 1])
        mat[inside] = _material_index(entry.get("material"), mats, f"regions.paint[{k}]")

    sigma_t = np.stack([np.array([mats[m]["sigma_t"][g] for m in mat]) for g in range(G)])
    sigma_s = np.zeros((G, G, nc))
    for gf in range(G):
        for gt in range(G):
            sigma_s[gf, gt] = np.array([mats[m]["sigma_s"][gf, gt] for m in mat])
    src = np.stack([np.array([mats[m]["source"][g] for m in mat]) for g in range(G)])
    backend = "cg_supg" if disc == "cg_supg" else f"dg{dg_order}"
    meta = {"file": name, "backend": backend, "mesh": source, "materials": mat,
            "zeta": float(mesh_spec.get("supg_zeta", 0.5)), "structured_twin": mtype == "structured",
            "output_not_written": "output" in spec}
    return P.Problem(name, mesh, geom, quad, sigma_t, sigma_s, src, side_in, side_bc, meta=meta)


def solve(problem, precision="fp64", pc=None, rtol=1e-10, restart=30, max_it=2000, outer_rtol=None, **opts):
    """Solve a loaded problem on the current CUDA device, group by group (the
    reference driver's group loop, with its outer iteration where anything
    upscatters): (scalar flux per group as NumPy arrays, the stats of each
    group's last solve). pc: the exact sweep on a DG backend, point Jacobi
    on CG-SUPG (which has no sweep)."""
    from . import transport as T
    g = problem.geometry
    ctx = T.Context(g, problem.quad, zeta=problem.meta.get("zeta", 0.5))
    try:
        if pc is None:
            pc = "block" if ctx.is_cg else "sweep"
        solver = T.TransportSolver(ctx, rtol=rtol, precision=precision, pc=pc, restart=restart, max_it=max_it)
        extra = {} if outer_rtol is None else {"outer_rtol": outer_rtol}
        inflow = problem.side_inflow if problem.side_inflow is not None and np.any(problem.side_inflow) else None
        phis, stats = T.solve_groups(ctx, problem.sigma_t, problem.sigma_s, problem.source, side_inflow=inflow,
                                     solver=solver, **extra, **opts)
        return [p.double().cpu().numpy() for p in phis], stats
    finally:
        ctx.close()
