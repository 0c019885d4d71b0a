"""The JSON problem files and Gmsh 2.2 meshes (docs/problem_files.md of the
reference), on the CPU: this repository's fixtures load into the problems
they describe, strict keys and the unsupported features are refused by name,
and - where the reference tree is present - every one of the reference's own
problem files either loads or is refused for a named feature this library
does not run (1D slabs, dirichlet-cell vacuum faces, inflow windows)."""
import glob
import json
import os

import numpy as np
import pytest

from ubolt_b200 import problem_file as PF

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "problems")
# The reference source tree, where it is checked out beside this repository
# (or named by UBOLT_REFERENCE_TREE); the test that reads it is skipped otherwise
REF = os.environ.get("UBOLT_REFERENCE_TREE", os.path.join(os.path.dirname(HERE), "..", "reference"))


def test_gmsh_reader_reads_cells_and_sets():
    mesh, cell_sets, face_sets = PF.read_gmsh(os.path.join(FIX, "square_quads.msh"), 2)
    assert mesh.cells.shape == (6, 4) and mesh.vertices.shape == (12, 2)
    assert sorted(cell_sets.tolist()) == [1, 1, 2, 2, 2, 2]
    assert sorted(set(face_sets.values())) == [10, 11, 12, 13] and len(face_sets) == 10
    # the left column is set 1
    left = mesh.vertices[mesh.cells].mean(axis=1)[:, 0] < 1.0 / 3.0
    assert np.all(cell_sets[left] == 1) and np.all(cell_sets[~left] == 2)


def test_fixture_problems_load():
    pr = PF.load(os.path.join(FIX, "inf_medium_box.json"))
    assert pr.meta["backend"] == "dg0" and pr.meta["structured_twin"]
    assert pr.geometry.n_cells == 120 and pr.quad.n_angles == 12 and pr.n_groups == 1
    assert np.all(pr.side_bc == PF.BC_REFLECT)
    pr = PF.load(os.path.join(FIX, "inf_medium_up2_dg1.json"))
    assert pr.meta["backend"] == "dg1" and pr.geometry.n_cells == 60 and pr.n_groups == 2
    assert pr.sigma_s[1, 0, 0] == 0.2 and pr.sigma_s[0, 1, 0] == 0.5  # [from][to]
    pr = PF.load(os.path.join(FIX, "inf_medium_cg.json"))
    assert pr.meta["backend"] == "cg_supg" and pr.meta["zeta"] == 2.0
    pr = PF.load(os.path.join(FIX, "two_materials_gmsh.json"))
    mat = pr.meta["materials"]
    c = pr.geometry.centroid.reshape(-1, 3)
    painted = (c[:, 0] >= 0.6) & (c[:, 0] <= 0.9) & (c[:, 1] >= 0.6) & (c[:, 1] <= 0.9)
    column = c[:, 0] < 1.0 / 3.0
    assert np.all(mat[column | painted] == 0) and np.all(mat[~column & ~painted] == 1)
    assert pr.side_inflow.tolist() == [1.0, 0.0, 0.0, 0.0]
    assert pr.side_bc.tolist() == [0, 0, 1, 0]
    assert np.all(pr.source[0][mat == 1] == 0.0) and np.all(pr.source[0][mat == 0] == 1.0)


def _spec(**over):
    with open(os.path.join(FIX, "inf_medium_box.json")) as f:
        spec = json.load(f)
    spec.update(over)
    return spec


def test_strict_keys_and_named_refusals():
    with pytest.raises(PF.SpecError, match="unknown key"):
        PF.from_spec(_spec(inflow=1.0))
    with pytest.raises(PF.SpecError, match="unknown key"):
        PF.from_spec(_spec(mesh={"n_cells": [4, 4], "lengths": [1, 1], "cells": 3}))
    with pytest.raises(PF.Unsupported, match="1D"):
        PF.from_spec(_spec(dimension=1, mesh={"n_cells": [8], "lengths": [1.0]}))
    with pytest.raises(PF.Unsupported, match="dirichlet_cell"):
        PF.from_spec(_spec(vacuum_treatment="dirichlet_cell"))
    with pytest.raises(PF.Unsupported, match="window"):
        PF.from_spec(_spec(boundary_conditions={"left": {"type": "vacuum", "inflow": 1.0, "window": [0.2, 0.4]}}))
    with pytest.raises(PF.SpecError, match="vacuum-only"):
        PF.from_spec(_spec(boundary_conditions={"left": {"type": "reflect", "inflow": 1.0}}))
    with pytest.raises(PF.SpecError, match="Face Sets"):
        PF.from_spec(_spec(boundary_conditions={"4": "reflect"}))  # an integer key on a structured mesh
    with pytest.raises(PF.SpecError, match="same face"):
        PF.from_spec(_spec(mesh={"type": "unstructured", "n_cells": [4, 4], "lengths": [1, 1]},
                           boundary_conditions={"left": "reflect", "4": "vacuum"}))
    with pytest.raises(PF.SpecError, match="sn_order"):
        PF.from_spec(_spec(sn_order=5))


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "tests", "problems")), reason="no reference tree here")
def test_every_reference_problem_file_loads_or_is_refused_by_name():
    loaded, refused = [], {}
    for path in sorted(glob.glob(os.path.join(REF, "tests", "problems", "*.json"))):
        try:
            PF.load(path)
            loaded.append(os.path.basename(path))
        except PF.Unsupported as e:
            refused[os.path.basename(path)] = str(e)
    for name, why in refused.items():
        assert any(k in why for k in ("1D slab", "dirichlet_cell", "window")), (name, why)
    assert len(loaded) >= 90, f"{len(loaded)} loaded; refused: {refused}"
