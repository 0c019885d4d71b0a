"""Small seeded problems over every cell shape and order, shared by the tests."""
import numpy as np

from ubolt_b200 import problem as P

# name, dim, builder(rng), order, sn, side_bc (reflective low faces where 1)
CASES = [
    ("tri_dg1_vac", 2, lambda r: P.box_tris(8, 7, jitter=0.2, rng=r), 1, 4, [0, 0, 0, 0]),
    ("tri_dg1_refl", 2, lambda r: P.box_tris(7, 6, jitter=0.2, rng=r), 1, 4, [1, 0, 1, 0]),
    ("tri_dg0_refl", 2, lambda r: P.box_tris(7, 6, jitter=0.2, rng=r), 0, 4, [1, 0, 1, 0]),
    ("quad_dg0_vac", 2, lambda r: P.box_quads(6, 5), 0, 4, [0, 0, 0, 0]),
    ("quad_dg1_refl", 2, lambda r: P.box_quads(5, 6, jitter=0.15, rng=r), 1, 8, [1, 0, 1, 0]),
    ("hex_dg1_refl", 3, lambda r: P.box_hexes(4, 3, 3), 1, 4, [1, 0, 1, 0, 1, 0]),
    ("hex_dg0_vac", 3, lambda r: P.box_hexes(4, 3, 3), 0, 4, [0, 0, 0, 0, 0, 0]),
    ("tet_dg1_refl", 3, lambda r: P.box_tets(3, 3, 3, jitter=0.2, rng=r), 1, 4, [1, 0, 1, 0, 0, 0]),
    ("tet_dg0_vac", 3, lambda r: P.box_tets(3, 3, 2, jitter=0.2, rng=r), 0, 2, [0, 0, 0, 0, 0, 0]),
]


def build(case, seed=7):
    name, dim, mk, order, sn, sbc = case
    rng = np.random.default_rng(seed)
    mesh = mk(rng)
    geom = P.build_geometry(mesh, order, side_bc=sbc)
    quad = P.lqn(dim, sn)
    nc = geom.n_cells
    sigma_t = rng.uniform(0.3, 3.0, nc)
    sigma_s = sigma_t * rng.uniform(0.1, 0.95, nc)
    return mesh, geom, quad, sigma_t, sigma_s


def case_ids():
    return [c[0] for c in CASES]
