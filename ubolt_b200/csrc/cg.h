// The CG-SUPG backend behind a ubolt_ctx created by ubolt_ctx_create_cg: its
// device tables and the launchers the shared entry points dispatch to.
#pragma once

#include "ctx.h"

#include <vector>

namespace ubolt {

// One precision's device view. Star entries are vertex-major: vertex i's
// entries are [star_off[i], star_off[i + 1]), each one (element e, i's basis
// index li in e) with its row record - per column j of e, P values:
//   M_ij, G_ij (dim), G_ji (dim), the symmetric part of K_ij summed over
//   (d, d') and (d', d): xx, yy (, zz), xy (, xz, yz)
// - and the vertex of each column.
template <typename T>
struct CgDev {
   int32_t dim, nv, P, A;
   int64_t n_vertices, n_rows;
   T zeta, inv_sum_weights;
   const int32_t *star_off;   // [n_vertices + 1]
   const int32_t *star_elem;  // [n_star]
   const int8_t *star_li;     // [n_star]
   const int32_t *cols;       // [n_star][nv]
   const T *rec;              // [n_star][nv][P]
   const T *cgrad;            // [n_elements][nv][dim] gradients at the reference centroid
   const T *inv_m;            // [n_vertices] 1 / lumped mass
   const int32_t *bf_off;     // [n_vertices + 1]
   const T *bf;               // [n_bfaces][4] outward nA (3), 1 / (m_i n_fv)
   const int8_t *bf_side;     // [n_bfaces]
   int32_t side_bc[6];
   const T *omega;            // [A][3]
   const int32_t *refl;       // [3][A]
   const T *sigma_t, *sigma_s;  // [n_elements] the group's
   const T *tau;                // [n_elements][A] the group's SUPG tau (the apply's; built per group)
};

}  // namespace ubolt

struct ubolt_cg {
   int dim = 0, nv = 0, F = 0, P = 0;
   int64_t n_vertices = 0, n_elements = 0, n_star = 0;
   double zeta = 0.5;
   ubolt::CgDev<double> d64{};
   ubolt::CgDev<float> d32{};
   // Scratch owned by the context: the scalar flux the scatter weighs, and
   // the Jacobi inverse diagonal of the current group (rows)
   double *phi64 = nullptr;
   float *phi32 = nullptr;
   double *jinv64 = nullptr;
   float *jinv32 = nullptr;
   uint64_t jacobi_epoch = 0;  // the group epoch jinv was built for (0: never)
   // tau per (element, ordinate) of the current group, both precisions: it
   // depends on the group's sigma_t, not on the vector, and each of an
   // element's vertices would recompute it per row
   double *tau64 = nullptr;
   float *tau32 = nullptr;
   uint64_t tau_epoch = 0;
   // Host copies the DSA assembles from
   std::vector<int64_t> elem_vertex, elem_face_neighbour, bface_offset;
   std::vector<int32_t> elem_face_bc, bface_bc;
   std::vector<double> mass, stiff, centre_grad, volume, lumped, elem_face_area, bface_nA, bface_mass;
};

namespace ubolt {

template <typename T>
int CgApply(ubolt_ctx *ctx, const T *x, T *y, bool scatter, void *stream);
int CgDiagonal(ubolt_ctx *ctx, double *d, void *stream);
// Point Jacobi: y = D^{-1} x, the inverse diagonal rebuilt first when the group changed
template <typename T>
int CgJacobiApply(ubolt_ctx *ctx, const T *x, T *y, void *stream);
int CgJacobiSetup(ubolt_ctx *ctx, int64_t *n_zero, void *stream);
int CgAddSource(ubolt_ctx *ctx, const double *q_elem, double *b, void *stream);
int CgAddTransfer(ubolt_ctx *ctx, const double *phi_from, const double *sigma_s_from_to, double *b, void *stream);
int CgGhostInflow(ubolt_ctx *ctx, const double *side_inflow, double *b, void *stream);

}  // namespace ubolt
