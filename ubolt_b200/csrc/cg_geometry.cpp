// The CG-SUPG backend's host tables, once per mesh: per element the mass,
// gradient and stiffness matrices of the degree-1 Lagrange basis, the
// gradients at the reference centroid, the volume and the centroid; per
// vertex its star (elements and its basis index in each), its lumped mass and
// its boundary faces; per element its faces (for the DSA's void chord).
//
// Restates UnstructuredCG::build_element_tables (src/unstructured_cgk.
// kokkos.cxx:52-255) and the star / boundary-face half of ::create (:276-443):
//   * the basis function of a cell vertex is that vertex's (the reference
//     matches PetscFE nodes to vertices by position, :155-189; here the
//     vertex order is the basis order by construction),
//   * simplices are affine, so every table is a polynomial and is written in
//     closed form: M_ij = V (1 + delta_ij) / ((d + 1)(d + 2)),
//     G^d_ij = V / (d + 1) d_d phi_j, K^{dd'}_ij = V d_d phi_i d_d' phi_j,
//   * quads and hexes are mapped bi/trilinearly from the unit box and
//     integrated by the tensor 4-point Gauss-Legendre rule (a degree-1
//     Lagrange element's default quadrature of order 3; the stiffness matrix
//     of a non-affine cell is rational, so the rule is part of the scheme),
//   * a boundary face (one element) carries its outward area-weighted normal
//     and, for each of its vertices, m^f_i / (m_i A_f) = 1 / (m_i n_fv) with
//     the lumped face mass m^f_i = A_f / n_fv (:330-372, 445-455).
// Faces are matched by their sorted vertex ids instead of DMPlex cones.
#include "ubolt_internal.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

struct ubolt_cg_geometry_owned {
   int32_t dim = 0, nv = 0, F = 0;
   int64_t n_vertices = 0, n_elements = 0;
   std::vector<int64_t> elem_vertex, star_offset, star_elem, bface_offset, elem_face_neighbour;
   std::vector<int32_t> star_li, bface_side, bface_bc, elem_face_bc;
   std::vector<double> mass, grad, stiff, centre_grad, volume, centroid, lumped, coord, bface_nA, bface_mass,
      elem_face_area;
};

namespace {

using ubolt::SetError;

// Corner of each Q1 basis function in the unit box, in the cell's vertex
// order (counter-clockwise; bottom face then top face)
const int kQuadCorner[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
const int kHexCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

// Gauss-Legendre, 4 points, on [0, 1]
const double kGaussX[4] = {0.5 - 0.5 * 0.861136311594052575224, 0.5 - 0.5 * 0.339981043584856264803,
                           0.5 + 0.5 * 0.339981043584856264803, 0.5 + 0.5 * 0.861136311594052575224};
const double kGaussW[4] = {0.5 * 0.347854845137453857373, 0.5 * 0.652145154862546142627,
                           0.5 * 0.652145154862546142627, 0.5 * 0.347854845137453857373};

// Inverse and determinant of a d x d matrix (d <= 3), stored row-major in a
// 3 x 3 array (entry (r, c) at 3 r + c)
double Invert(int d, const double m[9], double inv[9])
{
   if (d == 2) {
      const double det = m[0] * m[4] - m[1] * m[3];
      inv[0] = m[4] / det;
      inv[1] = -m[1] / det;
      inv[3] = -m[3] / det;
      inv[4] = m[0] / det;
      return det;
   }
   const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
   const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
   inv[0] = c00 / det;
   inv[1] = (m[2] * m[7] - m[1] * m[8]) / det;
   inv[2] = (m[1] * m[5] - m[2] * m[4]) / det;
   inv[3] = c01 / det;
   inv[4] = (m[0] * m[8] - m[2] * m[6]) / det;
   inv[5] = (m[2] * m[3] - m[0] * m[5]) / det;
   inv[6] = c02 / det;
   inv[7] = (m[1] * m[6] - m[0] * m[7]) / det;
   inv[8] = (m[0] * m[4] - m[1] * m[3]) / det;
   return det;
}

// Q1 value and reference gradient of basis function j at xi
void Q1(int dim, int j, const double *xi, double *phi, double *dphi)
{
   double f[3], df[3];
   for (int k = 0; k < dim; k++) {
      const int c = dim == 2 ? kQuadCorner[j][k] : kHexCorner[j][k];
      f[k] = c ? xi[k] : 1.0 - xi[k];
      df[k] = c ? 1.0 : -1.0;
   }
   *phi = 1.0;
   for (int k = 0; k < dim; k++) *phi *= f[k];
   for (int k = 0; k < dim; k++) {
      double p = df[k];
      for (int l = 0; l < dim; l++)
         if (l != k) p *= f[l];
      dphi[k] = p;
   }
}

// Physical gradients of the Q1 basis at xi (3 per function, zero past dim);
// returns det J
double Q1Gradients(int dim, int nv, const double (*X)[3], const double *xi, double *phi, double (*g)[3])
{
   double dref[8][3], J[9] = {0}, inv[9] = {0};
   for (int j = 0; j < nv; j++) Q1(dim, j, xi, &phi[j], dref[j]);
   for (int c = 0; c < dim; c++)
      for (int k = 0; k < dim; k++) {
         double s = 0.0;
         for (int j = 0; j < nv; j++) s += X[j][c] * dref[j][k];
         J[c * 3 + k] = s;
      }
   const double det = Invert(dim, J, inv);
   for (int j = 0; j < nv; j++) {
      for (int c = 0; c < 3; c++) g[j][c] = 0.0;
      for (int c = 0; c < dim; c++)
         for (int k = 0; k < dim; k++) g[j][c] += dref[j][k] * inv[k * 3 + c];
   }
   return det;
}

}  // namespace

extern "C" int ubolt_cg_geometry_build(int dim, int cell_type, int64_t n_vertices, const double *vertices,
                                       int64_t n_elements, const int64_t *cell_vertices, const int32_t *side_bc,
                                       ubolt_cg_geometry_owned **out)
{
   ubolt::ClearError();
   if (!out || !vertices || !cell_vertices) return SetError(UBOLT_ERR_ARG, "cg_geometry_build: NULL argument");
   *out = nullptr;
   const ubolt::CellShape *shape = ubolt::ShapeOf(cell_type);
   if (!shape || shape->dim != dim) return SetError(UBOLT_ERR_ARG, "cell type %d in %dD", cell_type, dim);
   if (n_vertices <= 0 || n_elements <= 0 || n_vertices >= ((int64_t)1 << 31))
      return SetError(UBOLT_ERR_ARG, "cg_geometry_build: %lld vertices, %lld elements", (long long)n_vertices,
                      (long long)n_elements);
   const int nv = shape->n_vertices, F = shape->n_faces;
   const bool simplex = cell_type == UBOLT_TRI || cell_type == UBOLT_TET;
   auto g = new ubolt_cg_geometry_owned();
   auto fail = [&](int rc) {
      delete g;
      return rc;
   };
   g->dim = dim;
   g->nv = nv;
   g->F = F;
   g->n_vertices = n_vertices;
   g->n_elements = n_elements;
   g->coord.assign(3 * n_vertices, 0.0);
   for (int64_t v = 0; v < n_vertices; v++)
      for (int d = 0; d < dim; d++) g->coord[3 * v + d] = vertices[v * dim + d];
   g->elem_vertex.assign(cell_vertices, cell_vertices + n_elements * nv);
   for (int64_t k = 0; k < n_elements * nv; k++)
      if (g->elem_vertex[k] < 0 || g->elem_vertex[k] >= n_vertices)
         return fail(SetError(UBOLT_ERR_ARG, "element %lld names vertex %lld", (long long)(k / nv),
                              (long long)g->elem_vertex[k]));
   const size_t n2 = (size_t)nv * nv;
   g->mass.assign(n_elements * n2, 0.0);
   g->grad.assign(n_elements * n2 * 3, 0.0);
   g->stiff.assign(n_elements * n2 * 9, 0.0);
   g->centre_grad.assign(n_elements * nv * 3, 0.0);
   g->volume.assign(n_elements, 0.0);
   g->centroid.assign(n_elements * 3, 0.0);

   // ~~~~~ Element tables
   for (int64_t e = 0; e < n_elements; e++) {
      double X[8][3];
      for (int j = 0; j < nv; j++)
         for (int c = 0; c < 3; c++) X[j][c] = g->coord[3 * g->elem_vertex[e * nv + j] + c];
      double *M = &g->mass[e * n2], *G = &g->grad[e * n2 * 3], *K = &g->stiff[e * n2 * 9];
      double *cg = &g->centre_grad[e * nv * 3];
      if (simplex) {
         double E[9] = {0}, inv[9] = {0};
         for (int c = 0; c < dim; c++)
            for (int k = 0; k < dim; k++) E[c * 3 + k] = X[k + 1][c] - X[0][c];
         const double det = Invert(dim, E, inv);
         if (!(std::fabs(det) > 0.0)) return fail(SetError(UBOLT_ERR_ARG, "element %lld is degenerate", (long long)e));
         const double V = std::fabs(det) / (dim == 2 ? 2.0 : 6.0);
         double gr[4][3] = {{0}};
         for (int k = 0; k < dim; k++)
            for (int c = 0; c < dim; c++) {
               gr[k + 1][c] = inv[k * 3 + c];
               gr[0][c] -= inv[k * 3 + c];
            }
         for (int i = 0; i < nv; i++)
            for (int j = 0; j < nv; j++) {
               M[i * nv + j] = V * (i == j ? 2.0 : 1.0) / ((dim + 1) * (dim + 2));
               for (int c = 0; c < 3; c++) {
                  G[(i * nv + j) * 3 + c] = V / (dim + 1) * gr[j][c];
                  for (int c2 = 0; c2 < 3; c2++) K[(i * nv + j) * 9 + 3 * c + c2] = V * gr[i][c] * gr[j][c2];
               }
            }
         for (int j = 0; j < nv; j++)
            for (int c = 0; c < 3; c++) cg[j * 3 + c] = gr[j][c];
         g->volume[e] = V;
         for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (int j = 0; j < nv; j++) s += X[j][c];
            g->centroid[e * 3 + c] = s / nv;
         }
      } else {
         const int nq = dim == 2 ? 16 : 64;
         double V = 0.0, cen[3] = {0, 0, 0};
         for (int q = 0; q < nq; q++) {
            const int qi[3] = {q % 4, (q / 4) % 4, q / 16};
            double xi[3], w = 1.0;
            for (int k = 0; k < dim; k++) {
               xi[k] = kGaussX[qi[k]];
               w *= kGaussW[qi[k]];
            }
            double phi[8], gq[8][3];
            const double det = Q1Gradients(dim, nv, X, xi, phi, gq);
            if (!(std::fabs(det) > 0.0))
               return fail(SetError(UBOLT_ERR_ARG, "element %lld is degenerate", (long long)e));
            const double wq = w * std::fabs(det);
            V += wq;
            for (int c = 0; c < dim; c++) {
               double x = 0.0;
               for (int j = 0; j < nv; j++) x += phi[j] * X[j][c];
               cen[c] += wq * x;
            }
            for (int i = 0; i < nv; i++)
               for (int j = 0; j < nv; j++) {
                  M[i * nv + j] += wq * phi[i] * phi[j];
                  for (int c = 0; c < 3; c++) {
                     G[(i * nv + j) * 3 + c] += wq * phi[i] * gq[j][c];
                     for (int c2 = 0; c2 < 3; c2++) K[(i * nv + j) * 9 + 3 * c + c2] += wq * gq[i][c] * gq[j][c2];
                  }
               }
         }
         g->volume[e] = V;
         for (int c = 0; c < dim; c++) g->centroid[e * 3 + c] = cen[c] / V;
         const double mid[3] = {0.5, 0.5, 0.5};
         double phi[8], gc[8][3];
         Q1Gradients(dim, nv, X, mid, phi, gc);
         for (int j = 0; j < nv; j++)
            for (int c = 0; c < 3; c++) cg[j * 3 + c] = gc[j][c];
      }
   }

   // ~~~~~ Stars and lumped masses (a counting sort by vertex, elements ascending)
   g->star_offset.assign(n_vertices + 1, 0);
   for (int64_t k = 0; k < n_elements * nv; k++) g->star_offset[g->elem_vertex[k] + 1]++;
   for (int64_t v = 0; v < n_vertices; v++) g->star_offset[v + 1] += g->star_offset[v];
   g->star_elem.resize(n_elements * nv);
   g->star_li.resize(n_elements * nv);
   {
      std::vector<int64_t> fill(g->star_offset.begin(), g->star_offset.end() - 1);
      for (int64_t e = 0; e < n_elements; e++)
         for (int li = 0; li < nv; li++) {
            const int64_t p = fill[g->elem_vertex[e * nv + li]]++;
            g->star_elem[p] = e;
            g->star_li[p] = li;
         }
   }
   g->lumped.assign(n_vertices, 0.0);
   for (int64_t v = 0; v < n_vertices; v++) {
      for (int64_t s = g->star_offset[v]; s < g->star_offset[v + 1]; s++) {
         const int64_t e = g->star_elem[s];
         const int li = g->star_li[s];
         for (int j = 0; j < nv; j++) g->lumped[v] += g->mass[e * n2 + li * nv + j];
      }
      if (!(g->lumped[v] > 0.0))
         return fail(SetError(UBOLT_ERR_ARG, "vertex %lld has lumped mass %g (no element?)", (long long)v,
                              g->lumped[v]));
   }

   // ~~~~~ Faces: matched by sorted vertex ids
   const int nfv = shape->verts_per_face;
   std::map<std::vector<int64_t>, std::pair<int64_t, int>> open;
   g->elem_face_neighbour.assign(n_elements * F, -1);
   g->elem_face_area.assign(n_elements * F, 0.0);
   g->elem_face_bc.assign(n_elements * F, -1);
   struct BFace {
      int64_t e;
      int f;
      double nA[3];
      int side;
   };
   std::vector<BFace> bfaces;
   auto face_normal = [&](int64_t e, int f, double nA[3]) {
      double P[4][3];
      for (int k = 0; k < nfv; k++)
         for (int c = 0; c < 3; c++) P[k][c] = g->coord[3 * g->elem_vertex[e * nv + shape->face[f][k]] + c];
      if (dim == 2) {
         nA[0] = P[1][1] - P[0][1];
         nA[1] = -(P[1][0] - P[0][0]);
         nA[2] = 0.0;
      } else {
         // Triangle: half of (P1 - P0) x (P2 - P0); quad: half the cross
         // product of the diagonals, (P2 - P0) x (P3 - P1)
         double u[3], w[3];
         for (int d = 0; d < 3; d++) {
            u[d] = nfv == 3 ? P[1][d] - P[0][d] : P[2][d] - P[0][d];
            w[d] = nfv == 3 ? P[2][d] - P[0][d] : P[3][d] - P[1][d];
         }
         nA[0] = 0.5 * (u[1] * w[2] - u[2] * w[1]);
         nA[1] = 0.5 * (u[2] * w[0] - u[0] * w[2]);
         nA[2] = 0.5 * (u[0] * w[1] - u[1] * w[0]);
      }
      // Outward: away from the element's centroid
      double dot = 0.0;
      for (int d = 0; d < 3; d++) {
         double m = 0.0;
         for (int k = 0; k < nfv; k++) m += P[k][d];
         dot += nA[d] * (m / nfv - g->centroid[e * 3 + d]);
      }
      if (dot < 0.0)
         for (int d = 0; d < 3; d++) nA[d] = -nA[d];
   };
   for (int64_t e = 0; e < n_elements; e++)
      for (int f = 0; f < F; f++) {
         std::vector<int64_t> key(nfv);
         for (int k = 0; k < nfv; k++) key[k] = g->elem_vertex[e * nv + shape->face[f][k]];
         std::sort(key.begin(), key.end());
         auto it = open.find(key);
         if (it == open.end()) {
            open.emplace(std::move(key), std::make_pair(e, f));
            continue;
         }
         const int64_t e2 = it->second.first;
         const int f2 = it->second.second;
         open.erase(it);
         double nA[3];
         face_normal(e, f, nA);
         const double area = std::sqrt(nA[0] * nA[0] + nA[1] * nA[1] + nA[2] * nA[2]);
         g->elem_face_neighbour[e * F + f] = e2;
         g->elem_face_neighbour[e2 * F + f2] = e;
         g->elem_face_area[e * F + f] = g->elem_face_area[e2 * F + f2] = area;
      }
   // What is left open is the boundary, visited in element / face order
   std::vector<std::pair<int64_t, int>> rest;
   for (const auto &kv : open) rest.push_back(kv.second);
   std::sort(rest.begin(), rest.end());
   for (const auto &ef : rest) {
      BFace b;
      b.e = ef.first;
      b.f = ef.second;
      face_normal(b.e, b.f, b.nA);
      int axis = 0;
      for (int d = 1; d < dim; d++)
         if (std::fabs(b.nA[d]) > std::fabs(b.nA[axis])) axis = d;
      b.side = 2 * axis + (b.nA[axis] > 0.0 ? 1 : 0);
      const double area = std::sqrt(b.nA[0] * b.nA[0] + b.nA[1] * b.nA[1] + b.nA[2] * b.nA[2]);
      const int bc = side_bc ? side_bc[b.side] : UBOLT_BC_VACUUM;
      if (bc != UBOLT_BC_VACUUM && bc != UBOLT_BC_REFLECT)
         return fail(SetError(UBOLT_ERR_ARG, "side %d has boundary family %d", b.side, bc));
      if (bc == UBOLT_BC_REFLECT)
         for (int d = 0; d < dim; d++)
            if (d != axis && std::fabs(b.nA[d]) > 1e-12 * area)
               return fail(SetError(UBOLT_ERR_ARG,
                                    "a reflective face of element %lld is not axis-aligned (the mirror is over "
                                    "the face's own axis)",
                                    (long long)b.e));
      g->elem_face_area[b.e * F + b.f] = area;
      g->elem_face_bc[b.e * F + b.f] = bc;
      bfaces.push_back(b);
   }

   // ~~~~~ Boundary faces per vertex
   g->bface_offset.assign(n_vertices + 1, 0);
   for (const auto &b : bfaces)
      for (int k = 0; k < nfv; k++) g->bface_offset[g->elem_vertex[b.e * nv + shape->face[b.f][k]] + 1]++;
   for (int64_t v = 0; v < n_vertices; v++) g->bface_offset[v + 1] += g->bface_offset[v];
   const int64_t nb = g->bface_offset[n_vertices];
   g->bface_nA.assign(3 * nb, 0.0);
   g->bface_mass.assign(nb, 0.0);
   g->bface_side.assign(nb, 0);
   g->bface_bc.assign(nb, 0);
   {
      std::vector<int64_t> fill(g->bface_offset.begin(), g->bface_offset.end() - 1);
      for (const auto &b : bfaces)
         for (int k = 0; k < nfv; k++) {
            const int64_t v = g->elem_vertex[b.e * nv + shape->face[b.f][k]];
            const int64_t p = fill[v]++;
            for (int d = 0; d < 3; d++) g->bface_nA[3 * p + d] = b.nA[d];
            g->bface_mass[p] = 1.0 / (g->lumped[v] * nfv);
            g->bface_side[p] = b.side;
            g->bface_bc[p] = side_bc ? side_bc[b.side] : UBOLT_BC_VACUUM;
         }
   }
   *out = g;
   return UBOLT_OK;
}

extern "C" int ubolt_cg_geometry_view(const ubolt_cg_geometry_owned *g, ubolt_cg_geometry *v)
{
   if (!g || !v) return SetError(UBOLT_ERR_ARG, "cg_geometry_view: NULL argument");
   *v = ubolt_cg_geometry{};
   v->dim = g->dim;
   v->n_element_vertices = g->nv;
   v->faces_per_element = g->F;
   v->n_vertices = g->n_vertices;
   v->n_elements = g->n_elements;
   v->n_star = (int64_t)g->star_elem.size();
   v->n_bfaces = (int64_t)g->bface_mass.size();
   v->elem_vertex = g->elem_vertex.data();
   v->mass = g->mass.data();
   v->grad = g->grad.data();
   v->stiff = g->stiff.data();
   v->centre_grad = g->centre_grad.data();
   v->volume = g->volume.data();
   v->centroid = g->centroid.data();
   v->lumped_mass = g->lumped.data();
   v->vertex_coord = g->coord.data();
   v->star_offset = g->star_offset.data();
   v->star_elem = g->star_elem.data();
   v->star_li = g->star_li.data();
   v->bface_offset = g->bface_offset.data();
   v->bface_nA = g->bface_nA.data();
   v->bface_mass = g->bface_mass.data();
   v->bface_side = g->bface_side.data();
   v->bface_bc = g->bface_bc.data();
   v->elem_face_neighbour = g->elem_face_neighbour.data();
   v->elem_face_area = g->elem_face_area.data();
   v->elem_face_bc = g->elem_face_bc.data();
   return UBOLT_OK;
}

extern "C" void ubolt_cg_geometry_free(ubolt_cg_geometry_owned *g) { delete g; }
