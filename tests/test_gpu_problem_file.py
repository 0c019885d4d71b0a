"""Problem files solved end to end on the GPU: the infinite-medium known
answers (the reference's -check_inf_medium: the discrete solution of a box
with every face reflective is the constant that balances the source, per
group) on the structured twin in 2D and 3D, on DG1 triangles with upscatter
and on CG-SUPG; and a Gmsh file mesh with two painted materials, an inflow
face set and a reflective one against the oracle's own solve."""
import os

import numpy as np
import pytest
import torch

import oracle as O
from ubolt_b200 import problem_file as PF

pytestmark = pytest.mark.gpu
FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "problems")


def _inf_medium(pr):
    """phi_g of the infinite medium: sigma_t,g phi_g - sum_h sigma_s[h][g] phi_h = source_g (cell 0's material)."""
    M = np.diag(pr.sigma_t[:, 0]) - pr.sigma_s[:, :, 0].T
    return np.linalg.solve(M, pr.source[:, 0])


@pytest.mark.parametrize("name", ["inf_medium_box", "inf_medium_cube", "inf_medium_up2_dg1", "inf_medium_cg"])
def test_infinite_medium_problem_files(name):
    torch.cuda.set_device(0)
    pr = PF.load(os.path.join(FIX, name + ".json"))
    exact = _inf_medium(pr)
    phis, stats = PF.solve(pr, rtol=1e-11, outer_rtol=1e-10)
    nb = getattr(pr.geometry, "n_basis", 1)
    for g, phi in enumerate(phis):
        # phi = sum_a w_a psi; at DG1 the cell average is the first (constant)
        # modal coefficient and the slopes vanish
        avg = phi.reshape(-1, nb)[:, 0] if nb > 1 else phi
        assert np.abs(avg - exact[g]).max() <= 1e-8 * abs(exact[g]), (name, g, avg[:3], exact[g])
        if nb > 1:
            assert np.abs(phi.reshape(-1, nb)[:, 1:]).max() <= 1e-8 * abs(exact[g])


def test_gmsh_problem_file_matches_the_oracle():
    torch.cuda.set_device(0)
    pr = PF.load(os.path.join(FIX, "two_materials_gmsh.json"))
    phis, stats = PF.solve(pr, rtol=1e-12)
    g, q = pr.geometry, pr.quad
    op = O.Operator(g, q, pr.sigma_t[0], pr.sigma_s[0, 0])
    b = O.rhs(g, q, pr.source[0], pr.side_inflow)
    x, it, res = op.solve(b, rtol=1e-13, max_it=3000, restart=40)
    ref = O.angular_integral(x, g.n_cells * g.n_basis, q)
    assert np.linalg.norm(phis[0] - ref) <= 1e-10 * np.linalg.norm(ref)
