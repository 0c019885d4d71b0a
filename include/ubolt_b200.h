/*
 * libubolt_b200 - the B200 (sm_100a) fixed-source discrete-ordinates solve of
 * UBOLT behind a C ABI.
 *
 * Every entry point returns an int status: UBOLT_OK (0) or a UBOLT_ERR_*
 * code, with a message from ubolt_last_error() (thread-local). No entry point
 * throws across the boundary.
 *
 * Vectors over the phase space are caller-owned DEVICE memory in UBOLT's row
 * layout, row = (cell * n_basis + basis) * n_angles + angle, angle fastest
 * (include/ubolt/phase_space.hpp:20-28). A (cell, basis) pair is a node and
 * owns a contiguous run of n_angles rows. Every kernel runs on the stream the
 * caller passes (a cudaStream_t as void *; NULL is the legacy default stream);
 * nothing is synchronised unless the entry point says so, and no apply, block
 * apply, rhs fill or sweep allocates device memory or copies host<->device
 * (AGENTS.md:44-47 of the reference states the same contract).
 *
 * Each declaration cites the reference interface it replaces, as
 * path:line within stevendargaville/UBOLT.
 */
#ifndef UBOLT_B200_H
#define UBOLT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
   UBOLT_OK = 0,
   UBOLT_ERR_ARG = 1,           /* bad argument / size mismatch (PETSC_ERR_ARG_*) */
   UBOLT_ERR_CUDA = 2,          /* a CUDA runtime call failed */
   UBOLT_ERR_SINGULAR = 3,      /* singular element block (PETSC_ERR_MAT_LU_ZRPVT) */
   UBOLT_ERR_STATE = 4,         /* called out of order (PETSC_ERR_ARG_WRONGSTATE) */
   UBOLT_ERR_NOT_CONVERGED = 5, /* the solve hit its iteration limit */
   UBOLT_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up */
   UBOLT_ERR_NOMEM = 7,         /* device allocation failed at set-up */
   UBOLT_ERR_BREAKDOWN = 8,     /* Krylov breakdown */
   UBOLT_ERR_NONFINITE = 9      /* NaN / Inf met in a residual */
};

/* Cell shapes a mesh may hold (one shape per mesh). */
enum { UBOLT_TRI = 3, UBOLT_QUAD = 4, UBOLT_TET = 10, UBOLT_HEX = 12 };

/* Boundary families per box side (bc_spec.hpp:11-40): vacuum (ghost-flux
 * inflow) or reflective (must be axis-aligned). */
enum { UBOLT_BC_VACUUM = 0, UBOLT_BC_REFLECT = 1 };

const char *ubolt_last_error(void);
const char *ubolt_version(void);
/* Kernels this library has launched in this process (all contexts). */
uint64_t ubolt_launch_count(void);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * Angular quadrature (host)
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

/* One octant of the level-symmetric set of order S2..S18: level cosines
 * (n_levels), the lexicographic level triples (3 * n_points, 1-based) and
 * each point's weight as a fraction of the whole sphere. Any output may be
 * NULL. Replaces the generated table src/sn_lqn_table.hpp:55-368. */
int ubolt_lqn_octant(int sn_order, double *mu, int *points, double *weight, int *n_levels, int *n_points);

/* The 2D (XY, xi > 0 half, doubled weights) or 3D LQn ordinate set:
 * omega (3 * A, xi = 0 in 2D), w (A), reflect (3 * A: the partner with cosine
 * d negated, -1 past dim). Call with all three NULL to size A. sum_weights is
 * the exact 4 pi. Replaces SNQuadrature2D/3D::create
 * (src/sn_quadraturek.kokkos.cxx:309-427, include/ubolt/sn_quadrature.hpp:93-159). */
int ubolt_quadrature_lqn(int dim, int sn_order, double *omega, double *w, int *reflect, int *n_angles,
                         double *sum_weights);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * DG geometry (host). The data UnstructuredDG::create builds
 * (include/ubolt/unstructured_dg.hpp:73-128), flat and per (cell, face slot)
 * with every cell owning exactly faces_per_cell slots.
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */
typedef struct {
   int32_t dim;            /* 2 or 3 */
   int32_t n_basis;        /* 1 (DG0) or dim + 1 (DG1, orthonormal modal P1) */
   int32_t faces_per_cell; /* F */
   int32_t pad_;
   int64_t n_cells;
   const double *volume;         /* [n_cells] (fan volume at DG1) */
   const double *centroid;       /* [n_cells * 3] */
   const double *face_nA;        /* [n_cells * F * 3] outward area-weighted normal, z = 0 in 2D */
   const int64_t *face_neighbour;/* [n_cells * F] neighbour cell, -1 on the boundary */
   const int32_t *face_bc;       /* [n_cells * F] -1 interior, else UBOLT_BC_* of its side */
   const int32_t *face_side;     /* [n_cells * F] boundary side 2 * axis + (0 low | 1 high), -1 interior */
   const int32_t *face_axis;     /* [n_cells * F] dominant axis of the normal */
   const double *face_centroid;  /* [n_cells * F * 3] */
   const double *face_distance;  /* [n_cells * F * 2] centroid-to-face (own, neighbour) */
   /* DG1 only, NULL at DG0 */
   const double *face_own;       /* [n_cells * F * nb * nb] (1/(V A)) int_f phi_i phi_j, own basis */
   const double *face_up;        /* [n_cells * F * nb * nb] the same against the upwind basis, 0 on vacuum */
   const double *basis_grad;     /* [n_cells * nb * 3] grad phi_i (0 for i = 0) */
   const double *face_neighbour_grad; /* [n_cells * F * nb * 3] the neighbour's grad phi_j, 0 on the boundary */
   const double *face_basis_value;    /* [n_cells * F * nb] phi_i at the face centroid */
} ubolt_dg_geometry;

typedef struct ubolt_geometry_owned ubolt_geometry_owned;

/* Build the DG0/DG1 geometry of a conforming mesh of one cell shape
 * (UBOLT_TRI/QUAD in 2D, UBOLT_TET/HEX in 3D): vertices [n_vertices * dim],
 * cell_vertices [n_cells * verts_per_cell] (tri/quad/hex in the usual
 * counter-clockwise / bottom-then-top order, any tet orientation).
 * side_bc[2 * dim] gives each box side's family, the box being the vertices'
 * bounding box. Restates UnstructuredDG::create and build_dg1_geometry
 * (src/unstructured_dgk.kokkos.cxx:27-218, 224-411, 706-821) with this
 * library's own face enumeration in place of DMPlex cones. */
int ubolt_geometry_build(int dim, int cell_type, int64_t n_vertices, const double *vertices, int64_t n_cells,
                         const int64_t *cell_vertices, int order, const int32_t *side_bc,
                         ubolt_geometry_owned **out);
int ubolt_geometry_view(const ubolt_geometry_owned *g, ubolt_dg_geometry *view);
void ubolt_geometry_free(ubolt_geometry_owned *g);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * Device context: the geometry and ordinates uploaded once
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */
typedef struct {
   int32_t dim;
   int32_t n_angles;
   double sum_weights;    /* W: 4 pi for the LQn sets */
   const double *omega;   /* [A * 3] */
   const double *w;       /* [A] */
   const int32_t *reflect;/* [3 * A] */
} ubolt_quadrature;

typedef struct ubolt_ctx ubolt_ctx;

/* Upload geometry and ordinates to the current CUDA device (FP64 and FP32
 * copies) and allocate the per-group FP32 cross-section slots. Replaces the
 * device copies of UnstructuredDG::create (src/unstructured_dgk.kokkos.cxx:
 * 585-661) and the term creates (src/termsk.kokkos.cxx:276-312, 541-572). */
int ubolt_ctx_create(const ubolt_dg_geometry *geom, const ubolt_quadrature *quad, ubolt_ctx **ctx);
int ubolt_ctx_destroy(ubolt_ctx *ctx);
/* Rows, nodes and cells of the phase space (phase_space.hpp:44-50). */
int ubolt_ctx_sizes(const ubolt_ctx *ctx, int64_t *rows, int64_t *nodes, int64_t *cells, int32_t *n_basis,
                    int32_t *n_angles);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * The CG-SUPG backend (include/ubolt/unstructured_cg.hpp:11-263): continuous
 * P1 (triangles, tetrahedra) or Q1 (quadrilaterals, hexahedra) Galerkin with
 * consistent SUPG, one unknown per (VERTEX, ordinate). A context created by
 * ubolt_ctx_create_cg has n_basis 1, nodes = the mesh's vertices (rows =
 * vertex * n_angles + angle) and cells = the mesh's ELEMENTS, the unit cross
 * sections, sources and materials are given on. Its row (i, a) is divided by
 * the lumped mass m_i and reads
 *   1/m_i sum_{e in star(i)} sum_j [Omega.G_ij + tau Omega Omega : K_ij
 *                                   + sigma_t (M_ij + tau Omega.G_ji)] psi(j, a)
 *   + per inflow boundary face |Omega . nA_f| / (m_i n_face_vertices) psi(i, a)
 *     (minus the same at the mirrored ordinate on a reflective face)
 *   - 1/m_i sum_e sigma_s / W sum_j (M_ij + tau Omega.G_ji) phi(j),
 * tau = min(1 / sigma_t, 2 / (zeta sum_j |Omega . grad phi_j(x_c)|)) per
 * (element, ordinate). On such a context:
 *   ubolt_set_group        sigma_t, sigma_s per element
 *   ubolt_apply[_f32], ubolt_apply_unscattered[_f32], ubolt_diagonal
 *                          the operator above (SUPGTermCG + ScatteringTermCG,
 *                          src/terms_cgk.kokkos.cxx:41-101, 203-221)
 *   ubolt_block_setup / ubolt_block_apply[_f32]
 *                          point Jacobi, the element-block inverse at one dof
 *                          per vertex
 *   ubolt_add_source       q per element, SUPG-weighted (UboltFillSourceCG)
 *   ubolt_add_transfer     phi_from per vertex, sigma_s(g'->g) per element,
 *                          tau of the current group (GroupTransferCG)
 *   ubolt_add_ghost_inflow the weak vacuum inflow (unstructured_cgk:508-520)
 *   ubolt_scalar_flux, ubolt_current, ubolt_expand_p1   per vertex
 *   ubolt_dsa_setup(ctx, NULL, opts) and the DSA calls: the CG weak
 *                          diffusion operator on the vertices (DSACG,
 *                          src/dsa_cgk.kokkos.cxx)
 *   ubolt_solve            with UBOLT_PC_NONE, UBOLT_PC_BLOCK or
 *                          UBOLT_PC_BLOCK_DSA
 * The sweep, the transpose and the gradient give UBOLT_ERR_STATE: the SUPG
 * operator is neither block lower-triangular in any ordering nor
 * adjoint-consistent (unstructured_cg.hpp:73-74).
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */
typedef struct {
   int32_t dim;                    /* 2 or 3 */
   int32_t n_element_vertices;     /* nv: 3 / 4 (tri / quad), 4 / 8 (tet / hex) */
   int32_t faces_per_element;      /* F */
   int32_t pad_;
   int64_t n_vertices, n_elements, n_star, n_bfaces;
   const int64_t *elem_vertex;     /* [n_elements * nv] the vertex of each basis function */
   const double *mass;             /* [n_elements * nv * nv] M_ij = int phi_i phi_j */
   const double *grad;             /* [n_elements * nv * nv * 3] G^d_ij = int phi_i d_d phi_j */
   const double *stiff;            /* [n_elements * nv * nv * 9] K^{dd'}_ij = int d_d phi_i d_d' phi_j */
   const double *centre_grad;      /* [n_elements * nv * 3] grad phi_j at the reference centroid */
   const double *volume;           /* [n_elements] */
   const double *centroid;         /* [n_elements * 3] */
   const double *lumped_mass;      /* [n_vertices] m_i = sum_e sum_j M_ij */
   const double *vertex_coord;     /* [n_vertices * 3] */
   const int64_t *star_offset;     /* [n_vertices + 1] CSR over each vertex's elements */
   const int64_t *star_elem;       /* [n_star] */
   const int32_t *star_li;         /* [n_star] the vertex's basis index in that element */
   const int64_t *bface_offset;    /* [n_vertices + 1] CSR over each vertex's boundary faces */
   const double *bface_nA;         /* [n_bfaces * 3] outward area-weighted normal */
   const double *bface_mass;       /* [n_bfaces] 1 / (m_i n_face_vertices) */
   const int32_t *bface_side;      /* [n_bfaces] box side 2 * axis + (0 low | 1 high) */
   const int32_t *bface_bc;        /* [n_bfaces] UBOLT_BC_* of that side */
   const int64_t *elem_face_neighbour; /* [n_elements * F] the element across, -1 on the boundary */
   const double *elem_face_area;   /* [n_elements * F] */
   const int32_t *elem_face_bc;    /* [n_elements * F] UBOLT_BC_* on the boundary, -1 inside */
} ubolt_cg_geometry;

typedef struct ubolt_cg_geometry_owned ubolt_cg_geometry_owned;

/* The CG-SUPG tables of a conforming one-shape mesh (the same vertex and cell
 * layouts as ubolt_geometry_build; the basis functions follow the cell's
 * vertex order). Simplices are integrated in closed form (affine: every
 * table is a polynomial), quads and hexes by the tensor 4-point
 * Gauss-Legendre rule. Reflective sides must be axis-aligned. Restates
 * UnstructuredCG::build_element_tables and ::create
 * (src/unstructured_cgk.kokkos.cxx:52-255, 276-561) with this library's own
 * face matching in place of DMPlex. */
int ubolt_cg_geometry_build(int dim, int cell_type, int64_t n_vertices, const double *vertices, int64_t n_elements,
                            const int64_t *cell_vertices, const int32_t *side_bc, ubolt_cg_geometry_owned **out);
int ubolt_cg_geometry_view(const ubolt_cg_geometry_owned *g, ubolt_cg_geometry *view);
void ubolt_cg_geometry_free(ubolt_cg_geometry_owned *g);

/* Upload the CG tables and ordinates; zeta > 0 is the thin-cell SUPG
 * parameter (0.5 in the reference). Replaces the device half of
 * UnstructuredCG::create (src/unstructured_cgk.kokkos.cxx:592-616) and the
 * CG term creates (src/terms_cgk.kokkos.cxx:8-27, 157-183). */
int ubolt_ctx_create_cg(const ubolt_cg_geometry *geom, const ubolt_quadrature *quad, double zeta, ubolt_ctx **ctx);

/* 1 for a CG-SUPG context, 0 for a DG one. */
int ubolt_ctx_is_cg(const ubolt_ctx *ctx);

/* Point the operator at a group's cross sections: DEVICE arrays of n_cells
 * doubles, not owned, which must outlive their use (RemovalTerm::set_group /
 * ScatteringTerm::set_group, src/termsk.kokkos.cxx:437-443, 574-579;
 * DSAPrecon::set_group, dsa.hpp:92-93). Refreshes the FP32 copies on
 * `stream` - no allocation. */
int ubolt_set_group(ubolt_ctx *ctx, const double *sigma_t, const double *sigma_s_within, void *stream);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * Operator applies (the MatShell MULT). One fused pass: streaming + removal -
 * scatter, matrix-free. y and x must not alias.
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

/* y = (L - S) x. ShellMatMultApply, src/transport_operatork.kokkos.cxx:49-61
 * (assembled StreamingTermDG0/DG1 + RemovalTerm, termsk.kokkos.cxx:170-539,
 * plus ScatteringTerm::apply_add, termsk.kokkos.cxx:584-649). */
int ubolt_apply(ubolt_ctx *ctx, const double *x, double *y, void *stream);
int ubolt_apply_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream);
/* y = L x, no scatter. UnscatteredMatMultApply, transport_operatork.kokkos.cxx:66-78. */
int ubolt_apply_unscattered(ubolt_ctx *ctx, const double *x, double *y, void *stream);
int ubolt_apply_unscattered_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream);
/* y = (L - S)^T x, the reversed-angle (downwind-gather) operator. No
 * reference counterpart: the reference has no transpose apply
 * (docs/architecture.md:493-494); its (V A)^T = P (V A) P identity
 * (docs/architecture.md:284-304) is what the tests hold it to. */
int ubolt_apply_adjoint(ubolt_ctx *ctx, const double *x, double *y, void *stream);
int ubolt_apply_adjoint_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream);

/* d = the streaming + removal diagonal, bitwise the composition of
 * DG0OutflowDiagonal / DG1OutflowDiagonal + sigma_t.
 * TransportOperator::diagonal, transport_operatork.kokkos.cxx:240-256. */
int ubolt_diagonal(ubolt_ctx *ctx, double *d, void *stream);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * Element blocks: the nb x nb (cell, angle) blocks of streaming + removal,
 * rebuilt on the fly from geometry and sigma_t and inverted by Gauss-Jordan
 * with partial pivoting per (cell, angle) - nothing is stored.
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

/* Count singular blocks of the current group (ElementBlockInverse::setup,
 * src/block_inversek.kokkos.cxx:249-299). Synchronises `stream`. Returns
 * UBOLT_ERR_SINGULAR with the count when any is singular. */
int ubolt_block_setup(ubolt_ctx *ctx, int64_t *n_singular, void *stream);
/* y = D^{-1} x (RemovalPCApply -> ElementBlockInverse::apply,
 * transport_solverk.kokkos.cxx:84-94, block_inversek.kokkos.cxx:206-222). */
int ubolt_block_apply(ubolt_ctx *ctx, const double *x, double *y, void *stream);
int ubolt_block_apply_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream);
/* y = D^{-T} x, the adjoint solve's removal stage (no reference counterpart). */
int ubolt_block_apply_transpose(ubolt_ctx *ctx, const double *x, double *y, void *stream);
/* The inverted blocks, ((c * A + a) * nb + i) * nb + j, into a device array
 * of n_cells * A * nb * nb doubles (ElementBlockInverse::inverse_d, for tests:
 * block_inverse.hpp:71-73). */
int ubolt_block_inverse(ubolt_ctx *ctx, double *inv, void *stream);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * Angular moment and right-hand sides. Every rhs fill ADDS to b.
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

/* phi(node) = sum_a w_a psi(node, a). UboltAngularIntegral,
 * sn_quadrature.hpp:163-171, src/sn_quadraturek.kokkos.cxx:400-427. */
int ubolt_scalar_flux(ubolt_ctx *ctx, const double *psi, double *phi, void *stream);
int ubolt_scalar_flux_f32(ubolt_ctx *ctx, const float *psi, float *phi, void *stream);
/* The current J(node, d) = sum_a w_a Omega_a,d psi(node, a), d < dim, into
 * current[node * dim + d] (n_nodes dim values). IntegrateCurrent, under
 * GroupTransfer::set_scalar_flux, src/multigroupk.kokkos.cxx:275-279. */
int ubolt_current(ubolt_ctx *ctx, const double *psi, double *current, void *stream);
/* psi(node, a) = phi(node) / W + sum_d p1(a, d) J(node, d), the P1
 * expansion of a scalar flux and current, p1(a) = T^{-1} Omega_a with
 * T = sum_a w_a Omega_a Omega_a^T (the inverse of the moments of a P1
 * field). The moments store's starting psi: GroupTransfer::enable_current
 * and expand_p1, src/multigroupk.kokkos.cxx:373-499. UBOLT_ERR_ARG where the
 * ordinates' weighted directions do not sum to zero. */
int ubolt_expand_p1(ubolt_ctx *ctx, const double *phi, const double *current, double *psi, void *stream);
/* b(cell, basis 0, a) += q(cell) / W, q the angle-integrated isotropic
 * source per cell (device, n_cells). MaterialSourceTable::add_isotropic,
 * src/material_speck.kokkos.cxx:164-213. */
int ubolt_add_source(ubolt_ctx *ctx, const double *q_cell, double *b, void *stream);
/* b(node, a) += sigma_s(g' -> g)(cell) phi_g'(node) / W on every angle.
 * GroupTransfer::add_transfer, src/multigroupk.kokkos.cxx:306-365. */
int ubolt_add_transfer(ubolt_ctx *ctx, const double *phi_from, const double *sigma_s_from_to, double *b,
                       void *stream);
/* b(c, i, a) += -(s / V) phi_i(x_f) inflow[side] / W over every vacuum face
 * the ordinate enters through, s = Omega_a . nA_f < 0; side_inflow[2 * dim]
 * is each side's angle-integrated inflow (HOST array). The ghost-flux rhs of
 * UboltFillInflow, src/discretisationk.kokkos.cxx:173-210, with the per-row
 * values of src/unstructured_dgk.kokkos.cxx:476-494 built on the fly. */
int ubolt_add_ghost_inflow(ubolt_ctx *ctx, const double *side_inflow, double *b, void *stream);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * The streaming stage: psi = L^{-1} q by an upwind sweep of every ordinate
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */
typedef struct {
   int32_t patch_size;    /* cells per patch */
   int32_t n_patches;
   int64_t n_tasks;       /* patch pieces x ordinates */
   int64_t n_lagged;      /* interior couplings lagged to break cycles */
   int64_t n_split;       /* extra tasks where a patch is solved in pieces */
   int32_t max_levels;    /* most levels in one patch-ordinate task */
   int32_t grid;          /* blocks of the last launch */
   int64_t total_levels;
   uint32_t timeouts;     /* bounded waits that gave up since the last status */
   int32_t kernel;        /* UBOLT_SWEEP_TASKS or UBOLT_SWEEP_WAVE: what ubolt_sweep (FP64) runs now */
   int64_t factor_bytes;  /* device bytes held by the factor stores (FP64 + FP32) */
   int64_t factor_bytes_fp64;  /* of which the FP64 store (what one FP64 sweep reads) */
} ubolt_sweep_info;

/* The two sweep kernels. TASKS: persistent warps over (patch, ordinate)
 * tasks that wait on each other's values through L2 - any mesh, cycles
 * included. WAVE: one block per ordinate walks that ordinate's levels with a
 * barrier between them, its upwind front in shared memory and its factors
 * streamed in by bulk copies - meshes whose every ordinate's upwind graph is
 * acyclic (2D, hexahedra), with a reserved factor store, no wait on another
 * block. One block per ordinate leaves most SMs idle and pays for every
 * scattered psi word on one SM, so AUTO picks WAVE only where it applies
 * and the problem is small (n_cells A <= 2^17, where it measured faster),
 * TASKS otherwise. */
enum { UBOLT_SWEEP_AUTO = 0, UBOLT_SWEEP_TASKS = 1, UBOLT_SWEEP_WAVE = 2 };

/* Build the sweep plan: patches of patch_size consecutive cells (0 picks 64,
 * or 24 on tetrahedra;
 * at most 256), per-ordinate upwind orders, task list; then reserve the
 * factor stores (see ubolt_sweep_set_factor_limit). Host work, one upload
 * and the sweep's only device allocations; independent of the group.
 * Called by the first sweep if not before. The streaming stage of the preconditioner, in place of
 * PCAIR (src/transport_solverk.kokkos.cxx:238-260, composite index 1). */
int ubolt_sweep_setup(ubolt_ctx *ctx, int patch_size);
/* Choose the sweep kernel (UBOLT_SWEEP_*; AUTO by default). WAVE where it
 * does not apply gives UBOLT_ERR_STATE. Both give L^{-1} q to rounding. A
 * set-up call: the factor stores are reserved again in the chosen kernel's
 * order (and rebuilt by the next sweep). */
int ubolt_sweep_set_kernel(ubolt_ctx *ctx, int kernel);
/* psi = L^{-1} q for every ordinate: exact where the per-ordinate upwind
 * graph is acyclic; reflective inflow and cycle-breaking couplings are lagged
 * to zero. psi is first filled with all-ones bytes on `stream` (the kernel's
 * "not yet stored" sentinel), then every value is overwritten. Every wait is
 * bounded; check ubolt_sweep_status. */
int ubolt_sweep(ubolt_ctx *ctx, const double *q, double *psi, void *stream);
int ubolt_sweep_f32(ubolt_ctx *ctx, const float *q, float *psi, void *stream);
/* psi = L^{-1} (u_a phi(node)) for every ordinate: the streaming stage on an
 * isotropic source (u = NULL: u_a = 1), the form the compressed GMRES
 * applies at every iteration (no reference counterpart: PCAIR is applied to
 * whole vectors). phi is FP64 per node (n_cells n_basis); u and psi in the
 * call's precision. ordinate_major: psi[(a n_cells + c) n_basis + i], each
 * ordinate's values contiguous (the task kernel; where the wave kernel runs
 * it gives UBOLT_ERR_STATE), else UBOLT's row layout. As ubolt_sweep
 * otherwise. */
int ubolt_sweep_iso(ubolt_ctx *ctx, const double *phi, const double *u, double *psi, int ordinate_major,
                    void *stream);
int ubolt_sweep_iso_f32(ubolt_ctx *ctx, const double *phi, const float *u, float *psi, int ordinate_major,
                        void *stream);
/* The factor stores: each cell-ordinate's B^{-1} and upwind couplings
 * G_f = B^{-1} s_f face_up_f, which depend on geometry and sigma_t but not on
 * q, rebuilt by one kernel launch on the first sweep after ubolt_set_group
 * and read by every sweep instead of being recomputed: n_cells A nb^2 (1 +
 * slots) values per precision, in task order. Reserved when the plan is
 * built, or now by this call - never inside a sweep. bytes < 0 (the
 * default): each store that fits half the free device memory at that
 * moment (at most 96 GiB), FP32 first; 0: none; otherwise the byte limit
 * for both together. Either way the result is the same, bit for bit. */
int ubolt_sweep_set_factor_limit(ubolt_ctx *ctx, int64_t bytes);
/* Plan statistics and the sticky timeout flag (synchronises `stream`):
 * returns UBOLT_ERR_TIMEOUT, and clears the flag, if a wait gave up. */
int ubolt_sweep_status(ubolt_ctx *ctx, ubolt_sweep_info *info, void *stream);
/* Failure-path check of the sweep's bounded waits (no reference
 * counterpart): set the wait limit in polls (default 2^22), and with
 * make_one_wait_unmet make one task of the NEXT sweep poll, for its first
 * upwind value, a word nothing writes, so that wait runs out: that sweep
 * completes, its result is invalid, ubolt_sweep_status reports
 * UBOLT_ERR_TIMEOUT, and later sweeps are normal again. */
int ubolt_sweep_test_wait(ubolt_ctx *ctx, uint32_t spin_limit, int make_one_wait_unmet);

/* The plan on the host alone, for inspection. Tasks are numbered in launch
 * order; task t solves cells of patch p for ordinate a, task_pa[t] = p * A + a,
 * after its upstream tasks (all numbered below t). Arrays are owned by the
 * returned handle. */
typedef struct ubolt_sweep_plan_host ubolt_sweep_plan_host;
typedef struct {
   int32_t patch_size, n_patches;
   int64_t n_tasks;
   int64_t n_lagged;         /* couplings lagged to break upwind cycles */
   int64_t n_split;          /* extra tasks where a patch is solved in pieces */
   const int32_t *task_pa;   /* [n_tasks] */
   const int32_t *dep_ptr;   /* [n_tasks + 1] */
   const int32_t *deps;
   const int64_t *cell_ptr;  /* [n_tasks + 1] */
   const uint8_t *tcell;     /* local cell index, patch p covering cells [p P, p P + P) */
   const uint16_t *tmask;    /* bit f: face f's upwind cell is in the same task; bit 8 + f: in an earlier task */
   const int32_t *lvl_ptr;   /* [n_tasks + 1] */
   const uint16_t *lvl;      /* level end positions within a task's cells */
} ubolt_sweep_plan_view;
int ubolt_sweep_plan_build(const ubolt_dg_geometry *geom, const ubolt_quadrature *quad, int patch_size,
                           ubolt_sweep_plan_host **out, ubolt_sweep_plan_view *view);
void ubolt_sweep_plan_free(ubolt_sweep_plan_host *plan);

/* The wave plan on the host alone, for inspection: per ordinate, the cells
 * in level order (positions) and the front slot of shared memory each
 * solved value lives in while later levels read it. */
typedef struct ubolt_wave_plan_host ubolt_wave_plan_host;
typedef struct {
   int32_t acyclic;          /* 0: some ordinate's upwind graph has a cycle; the arrays below are NULL */
   int32_t slots;            /* most gathered upwind faces of one position */
   int32_t n_front;          /* front slots the busiest ordinate needs */
   int32_t max_width;        /* most positions in one level */
   int32_t max_levels;       /* most levels of one ordinate */
   int32_t pad_;
   int64_t total_levels;     /* summed over the ordinates */
   const int32_t *lvl_base;  /* [A + 1]: ordinate a's levels are lvl_base[a] .. lvl_base[a + 1] - 1 */
   const int32_t *lvl_pos;   /* [total_levels + A]: level l of ordinate a starts at position
                                lvl_pos[lvl_base[a] + a + l]; one end entry per ordinate */
   const int32_t *meta;      /* [A][n_cells][4] per position: cell; front slot | gathered-face mask << 16
                                (slot 0xffff: no later level reads it); the upwind cells' slots in face
                                order, two 16-bit slots per word */
} ubolt_wave_plan_view;
int ubolt_wave_plan_build(const ubolt_dg_geometry *geom, const ubolt_quadrature *quad, ubolt_wave_plan_host **out,
                          ubolt_wave_plan_view *view);
/* One precision's layout of the wave sweep, for a block with at most
 * max_shared_bytes of shared memory: the block's shared memory (mbarriers,
 * level tables, the front at front_off, the ring of `cap` bytes at
 * ring_base) and the factor store (ordinate a's region at byte region[a];
 * level chunks at region-relative chunk_rel[.], indexed as lvl_pos, landing
 * in the ring at ring_off[.]). Arrays are owned by the plan handle and
 * replaced by the next call. UBOLT_ERR_STATE where a level does not fit. */
typedef struct {
   int32_t front_off, ring_base, cap, smem;
   int64_t store_bytes;
   const int64_t *region;
   const int32_t *chunk_rel;
   const int32_t *ring_off;
} ubolt_wave_layout_view;
int ubolt_wave_plan_layout(ubolt_wave_plan_host *plan, int n_basis, int elem_bytes, int max_shared_bytes,
                           ubolt_wave_layout_view *view);
void ubolt_wave_plan_free(ubolt_wave_plan_host *plan);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * DSA: the diffusion correction y = P D^{-1} R x (DSAPrecon, include/ubolt/dsa.hpp)
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */
typedef struct {
   double penalty;           /* MIP penalty C (-dsa_mip_penalty, default 4) */
   double consistent_power;  /* DG0 consistent-D blend power p (default 1.5) */
   int32_t consistent_d;     /* DG0: blend the upwind numerical diffusion in (default 1) */
   int32_t inner_iterations; /* block-Jacobi PCG iterations of the inner solve (default 30) */
   double void_sigma_t;      /* a cell with sigma_t <= this is void (-dsa_void_sigma_t, default 0) */
   double void_d;            /* D in a bridged void; 0: from the voids' mean chord (-dsa_void_d, default 0) */
   int32_t void_bridge;      /* bridge the voids where the operator allows (-dsa_void_bridge, default 1) */
   int32_t pad_;
} ubolt_dsa_options;

void ubolt_dsa_defaults(ubolt_dsa_options *opts);
/* Keep the host geometry the diffusion operator is built from and allocate
 * its device storage (DSAPrecon::create on an UnstructuredDG,
 * src/dsak.kokkos.cxx:113-121, src/dsa_plexk.kokkos.cxx:68-209). The
 * geometry must be the context's. On a CG-SUPG context pass NULL: the
 * context holds the tables, and the operator is DSACG's weak form on the
 * vertices (src/dsa_cgk.kokkos.cxx:114-203), R scaled by the lumped mass,
 * no masking (an unbridged void keeps the SUPG operator's own tensor D). */
int ubolt_dsa_setup(ubolt_ctx *ctx, const ubolt_dg_geometry *geom, const ubolt_dsa_options *opts);
/* Refill the diffusion matrix for the context's current group - host
 * assembly, then upload (DSAPrecon::set_group, src/dsak.kokkos.cxx:216-226:
 * MIP at DG1, dsa_plexk.kokkos.cxx:365-475; two-point flux with the
 * consistent-D blend at DG0, :288-348), after the void policy
 * (DSAPrecon::assemble, src/dsak.kokkos.cxx:233-345): void cells are bridged
 * (D from their mean chord, or the fixed void D) or, where bridging is off or
 * would leave the operator singular, masked (V times the identity, no
 * coupling, vacuum faces onto them, R and P skip them). UBOLT_ERR_ARG where
 * the operator is singular (every face reflective, no void, no absorption).
 * Synchronises `stream`. */
int ubolt_dsa_set_group(ubolt_ctx *ctx, void *stream);
/* The void policy's outcome for the current group: the number of void cells,
 * whether they are bridged, and their mean chord 4 V / S (0 unless bridged)
 * (DSAPrecon::assemble, src/dsak.kokkos.cxx:255-296). Any pointer may be NULL. */
int ubolt_dsa_void_info(ubolt_ctx *ctx, int64_t *n_void, int32_t *bridged, double *chord);
/* y = P D^{-1} R x (DSAPrecon::apply, src/dsak.kokkos.cxx:350-391), the
 * inner solve a fixed count of FP64 block-Jacobi PCG iterations on device. */
int ubolt_dsa_apply(ubolt_ctx *ctx, const double *x, double *y, void *stream);
/* v = D u over the nodes (n_cells * n_basis): the diffusion SpMV. */
int ubolt_dsa_spmv(ubolt_ctx *ctx, const double *u, double *v, void *stream);
/* rhs(node) = V_c sum_a w_a x(node, a) (RestrictKernel, src/dsak.kokkos.cxx:20-44);
 * zero on a masked void's nodes once a group is filled. */
int ubolt_dsa_restrict(ubolt_ctx *ctx, const double *x, double *rhs, void *stream);
/* y(node, a) = u(node) / W (ProlongKernel, src/dsak.kokkos.cxx:51-62); zero
 * on a masked void's rows once a group is filled. */
int ubolt_dsa_prolong(ubolt_ctx *ctx, const double *u, double *y, void *stream);
/* y = P D^{-1} R x exactly as ubolt_dsa_apply computes it, but with every
 * scratch vector of the inner solve in one fixed device array built into
 * the library rather than in memory the library allocates. No counterpart in
 * the reference. It is for callers that cannot let this library allocate
 * device memory while they solve: an application whose own memory pool (a
 * PETSc/Kokkos or framework allocator) has already reserved the device, where
 * a cudaMalloc from a library underneath would fail or upset the pool.
 * Limit: at most 262144 nodes (n_cells * n_basis); larger problems get
 * UBOLT_ERR_ARG and should use ubolt_dsa_apply. The array (12.6 MB) is held
 * by every GPU that loads the library until the process exits. The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress)
 * with that device current; make that first call before any stream capture.
 * The address is kept for the life of the process: after a cudaDeviceReset
 * on that device the library must be reloaded before this call is used again.
 * Every call, from any context on the device, shares the one array and
 * leaves the last call's values in it: calls that overlap on the GPU race.
 * ubolt_dsa_setup and ubolt_dsa_set_group must have run; the call itself
 * allocates nothing. */
int ubolt_dsa_apply_static(ubolt_ctx *ctx, const double *x, double *y, void *stream);
/* The assembled blocks, host array [n_cells][F + 1][nb][nb]: per cell its
 * neighbour blocks in face-slot order (zero without a neighbour), then its
 * own block. */
int ubolt_dsa_matrix(ubolt_ctx *ctx, double *blocks);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * The solve
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */
/* UBOLT_PC_BLOCK_DSA: the element-block inverse, then the multiplicative
 * DSA stage (the preconditioner of a backend without a sweep: CG-SUPG). */
enum { UBOLT_PC_NONE = 0, UBOLT_PC_BLOCK = 1, UBOLT_PC_SWEEP = 2, UBOLT_PC_SWEEP_DSA = 3, UBOLT_PC_BLOCK_DSA = 4 };
enum { UBOLT_PRECISION_FP64 = 0, UBOLT_PRECISION_MIXED = 1 };
/* UBOLT_KRYLOV_AUTO: with the sweep preconditioner and an exact sweep (no
 * reflective side, no lagged coupling), A M^{-1} = I - S L^{-1}, and every
 * basis vector but the residual's own anisotropic part lies in the
 * isotropic (scattering) subspace: the basis is kept as one n_nodes vector
 * and a scalar per vector, with no operator apply inside the Arnoldi loop -
 * the same iterates in exact arithmetic. Otherwise, or with
 * UBOLT_KRYLOV_FULL, every basis vector has n_rows entries. */
enum { UBOLT_KRYLOV_AUTO = 0, UBOLT_KRYLOV_FULL = 1, UBOLT_KRYLOV_COMPRESSED = 2 };

typedef struct {
   double rtol;        /* stop at ||b - A x|| <= rtol ||b|| (true residual, FP64) */
   double inner_rtol;  /* mixed: each FP32 correction solve's relative tolerance */
   int32_t max_it;     /* GMRES iterations in total */
   int32_t restart;    /* GMRES(m) */
   int32_t precision;  /* UBOLT_PRECISION_* */
   int32_t pc;         /* UBOLT_PC_* */
   int32_t max_outer;  /* mixed: refinement steps */
   int32_t x_zero;     /* 1: start from zero, 0: from the x passed in */
   int32_t krylov;     /* UBOLT_KRYLOV_*: how the GMRES basis is held */
   int32_t pad_;
} ubolt_solve_options;

typedef struct {
   int32_t iterations; /* GMRES iterations (all refinement steps) */
   int32_t outer;      /* refinement steps (1 for FP64) */
   int32_t converged;
   int32_t krylov;     /* the form the basis was held in: UBOLT_KRYLOV_FULL, or 2 for the compressed form */
   double residual;    /* ||b - A x|| / ||b|| of the returned x, FP64 */
   double rnorm0;      /* ||b|| */
   double seconds;     /* host wall time of the call */
} ubolt_solve_stats;

/* rtol 1e-8, inner_rtol 1e-5, max_it 500, restart 30, FP64, sweep preconditioner. */
void ubolt_solve_defaults(ubolt_solve_options *opts);
/* Allocate the solver's workspace ((restart + 1) Krylov vectors, FP64, or
 * FP32 in the mixed form) and the sweep plan its preconditioner needs.
 * ubolt_solve calls it when the workspace is missing or of another shape. */
int ubolt_solver_setup(ubolt_ctx *ctx, const ubolt_solve_options *opts);
/* Solve (L - S) x = b for the current group. Right-preconditioned GMRES
 * (KSPGMRES + PC_RIGHT, src/transport_solverk.kokkos.cxx:196-318; the solve
 * TransportSolver::solve runs, :334-343), stopping on the true residual.
 * Mixed form: FP32 operator, sweep and Krylov storage (FP64 accumulation)
 * inside FP64 iterative refinement r = b - A x. Synchronises `stream`.
 * Returns UBOLT_ERR_NOT_CONVERGED, with x and stats filled, at max_it. */
int ubolt_solve(ubolt_ctx *ctx, const double *b, double *x, const ubolt_solve_options *opts,
                ubolt_solve_stats *stats, void *stream);
/* n solves of right-hand sides held in HOST memory, x_host[i] = A^{-1}
 * b_host[i], each as ubolt_solve. The upload of b_host[i + 1] and the
 * download of x_host[i - 1] run on two copy streams of the context while
 * solve i runs, through two device buffers each for b and x kept in the
 * solver's workspace (4 n_rows doubles). The copies overlap the solves
 * only from page-locked host memory. The first upload waits for the work
 * already on `stream`; on return `stream` waits for the last download, so
 * x_host is complete once `stream` is synchronised. stats (n entries, may be
 * NULL) per solve; every solve starts from zero. Stops at the first solve
 * that fails, returning its status. The batched form of
 * TransportSolver::solve (src/transport_solverk.kokkos.cxx:334-343) for
 * right-hand sides in host Vecs. */
int ubolt_solve_host_batch(ubolt_ctx *ctx, int n, const double *const *b_host, double *const *x_host,
                           const ubolt_solve_options *opts, ubolt_solve_stats *stats, void *stream);

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * Adjoint and gradients. No reference counterpart (the reference has no
 * adjoint, docs/architecture.md:493-494; it tests the identity the adjoint
 * rests on, (V A)^T = P (V A) P, docs/architecture.md:284-304).
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

/* Solve (L - S)^T lambda = g: GMRES on ubolt_apply_adjoint, preconditioned
 * with the transposed stage - the sweep of the reversed ordinates,
 * L^{-T} = V P L^{-1} P V^{-1} (P swaps each ordinate with its opposite, V is
 * the cell volume per row), or the transposed element blocks. Options and
 * returns as ubolt_solve. */
int ubolt_solve_adjoint(ubolt_ctx *ctx, const double *g, double *lambda, const ubolt_solve_options *opts,
                        ubolt_solve_stats *stats, void *stream);
/* g(c, 0, a) += detector(c) V_c w_a: the adjoint source of the response
 * J = sum_c detector(c) V_c phi(c, 0) = g^T psi (detector: device, n_cells). */
int ubolt_add_response_source(ubolt_ctx *ctx, const double *detector, double *g, void *stream);
/* dJ/dsigma_t(c) = -sum_{rows of c} lambda psi and
 * dJ/dsigma_s(c) = sum_i (sum_a lambda(c,i,a)) (sum_b w_b psi(c,i,b)) / W,
 * for J = g^T psi with A psi = b and A^T lambda = g (device, n_cells each;
 * either output may be NULL). */
int ubolt_gradient(ubolt_ctx *ctx, const double *psi, const double *lambda, double *grad_sigma_t,
                   double *grad_sigma_s, void *stream);

#ifdef __cplusplus
}
#endif

#endif
