// DG0/DG1 geometry of a conforming single-shape mesh, on the host, once.
//
// Restates the geometry half of UnstructuredDG::create and
// UnstructuredDG::build_dg1_geometry (src/unstructured_dgk.kokkos.cxx):
//   * exact moments of each cell and face as a fan of simplices (:27-182),
//   * the orthonormal modal P1 basis by Cholesky of the normalised central
//     second moment (:184-218),
//   * outward area-weighted face normals (src/plex_commonk.hpp:291-307), the
//     dominant axis (:282-289), centroid-to-face distances (:363-371),
//   * the face matrices face_own / face_up and phi_i at the face centroid
//     (:747-821), int_f phi_i phi_j = A phi_i(x_f) phi_j(x_f) + b_i^T C_f b_j.
// Faces are matched by their sorted vertex ids instead of DMPlex cones; a
// cell's face slots follow this library's fixed per-shape face order.
#include "ubolt_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace ubolt {

const CellShape *ShapeOf(int cell_type)
{
   static const CellShape tri = {2, 3, 3, 2, {{0, 1}, {1, 2}, {2, 0}}};
   static const CellShape quad = {2, 4, 4, 2, {{0, 1}, {1, 2}, {2, 3}, {3, 0}}};
   // Faces opposite vertices 0..3, each a cyclic vertex list
   static const CellShape tet = {3, 4, 4, 3, {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}}};
   // Bottom 0-3 and top 4-7 counter-clockwise: -z, +z, -y, +x, +y, -x
   static const CellShape hex = {3, 8, 6, 4,
                                 {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}}};
   switch (cell_type) {
   case UBOLT_TRI: return &tri;
   case UBOLT_QUAD: return &quad;
   case UBOLT_TET: return &tet;
   case UBOLT_HEX: return &hex;
   default: return nullptr;
   }
}

}  // namespace ubolt

struct ubolt_geometry_owned {
   int32_t dim = 0, nb = 1, F = 0;
   int64_t n_cells = 0;
   std::vector<double> volume, centroid, face_nA, face_centroid, face_distance;
   std::vector<int64_t> face_neighbour;
   std::vector<int32_t> face_bc, face_side, face_axis;
   std::vector<double> face_own, face_up, basis_grad, face_nb_grad, face_basis_value;
};

namespace {

// Zeroth, first and second moments about a reference point (unstructured_dgk
// FanMoments / AddSimplex / Centralise, :27-72).
struct Moments {
   double m0 = 0.0;
   double m1[3] = {0, 0, 0};
   double m2[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
};

void AddSimplex(Moments &m, int d, double measure, const double y[][3])
{
   double sum[3] = {0, 0, 0};
   for (int k = 0; k <= d; k++)
      for (int a = 0; a < 3; a++) sum[a] += y[k][a];
   m.m0 += measure;
   for (int a = 0; a < 3; a++) m.m1[a] += measure * sum[a] / (double)(d + 1);
   const double w = measure / (double)((d + 1) * (d + 2));
   for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
         double outer = sum[a] * sum[b];
         for (int k = 0; k <= d; k++) outer += y[k][a] * y[k][b];
         m.m2[3 * a + b] += w * outer;
      }
}

void Centralise(const Moments &m, const double ref[3], double centroid[3], double central[9])
{
   for (int a = 0; a < 3; a++) centroid[a] = ref[a] + m.m1[a] / m.m0;
   for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) central[3 * a + b] = m.m2[3 * a + b] - m.m1[a] * m.m1[b] / m.m0;
}

inline void Sub3(const double *a, const double *b, double *o)
{
   for (int d = 0; d < 3; d++) o[d] = a[d] - b[d];
}

struct FaceGeom {
   double area;
   double centroid[3];
   double central[9];
   double normal[3];  // unit, orientation of the vertex cycle
};

// A face's area, centroid, central second moment and unit normal. 2D: one
// segment. 3D: a fan of triangles off the vertex average, one per edge
// (FaceMoments, unstructured_dgk.kokkos.cxx:100-141).
void FaceMomentsOf(int dim, int nv, const double (*x)[3], FaceGeom &f)
{
   Moments m;
   double ref[3] = {0, 0, 0};
   for (int v = 0; v < nv; v++)
      for (int d = 0; d < 3; d++) ref[d] += x[v][d] / nv;
   if (dim == 2) {
      double y[2][3], e[3];
      Sub3(x[0], ref, y[0]);
      Sub3(x[1], ref, y[1]);
      Sub3(x[1], x[0], e);
      AddSimplex(m, 1, std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]), y);
      const double len = std::sqrt(e[0] * e[0] + e[1] * e[1]);
      f.normal[0] = e[1] / len;
      f.normal[1] = -e[0] / len;
      f.normal[2] = 0.0;
   } else {
      double va[3] = {0, 0, 0};
      for (int e = 0; e < nv; e++) {
         double y[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
         Sub3(x[e], ref, y[1]);
         Sub3(x[(e + 1) % nv], ref, y[2]);
         const double cr[3] = {y[1][1] * y[2][2] - y[1][2] * y[2][1], y[1][2] * y[2][0] - y[1][0] * y[2][2],
                               y[1][0] * y[2][1] - y[1][1] * y[2][0]};
         for (int d = 0; d < 3; d++) va[d] += 0.5 * cr[d];
         AddSimplex(m, 2, 0.5 * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]), y);
      }
      const double n = std::sqrt(va[0] * va[0] + va[1] * va[1] + va[2] * va[2]);
      for (int d = 0; d < 3; d++) f.normal[d] = va[d] / n;
   }
   f.area = m.m0;
   Centralise(m, ref, f.centroid, f.central);
}

// Cholesky of central / V and the rows of its inverse: the gradients of the
// linear modes (OrthonormalGradients, unstructured_dgk.kokkos.cxx:184-218).
bool OrthonormalGradients(int dim, double volume, const double central[9], double beta[9])
{
   double L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
   for (int a = 0; a < dim; a++)
      for (int b = 0; b <= a; b++) {
         double sum = central[3 * a + b] / volume;
         for (int k = 0; k < b; k++) sum -= L[3 * a + k] * L[3 * b + k];
         if (a == b) {
            if (!(sum > 0.0)) return false;
            L[3 * a + a] = std::sqrt(sum);
         } else
            L[3 * a + b] = sum / L[3 * b + b];
      }
   for (int i = 0; i < 9; i++) beta[i] = 0.0;
   for (int col = 0; col < dim; col++)
      for (int a = col; a < dim; a++) {
         double sum = (a == col) ? 1.0 : 0.0;
         for (int k = col; k < a; k++) sum -= L[3 * a + k] * beta[3 * k + col];
         beta[3 * a + col] = sum / L[3 * a + a];
      }
   return true;
}

struct FaceKey {
   int64_t v[4];
   int64_t slot;
   bool operator<(const FaceKey &o) const
   {
      for (int i = 0; i < 4; i++)
         if (v[i] != o.v[i]) return v[i] < o.v[i];
      return slot < o.slot;
   }
   bool same(const FaceKey &o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2] && v[3] == o.v[3]; }
};

}  // namespace

extern "C" int ubolt_geometry_build(int dim, int cell_type, int64_t n_vertices, const double *vertices,
                                    int64_t n_cells, const int64_t *cell_vertices, int order,
                                    const int32_t *side_bc, ubolt_geometry_owned **out)
{
   using namespace ubolt;
   ClearError();
   if (!out) return SetError(UBOLT_ERR_ARG, "ubolt_geometry_build: out is NULL");
   *out = nullptr;
   const CellShape *shape = ShapeOf(cell_type);
   if (!shape || shape->dim != dim)
      return SetError(UBOLT_ERR_ARG, "cell type %d is not a %dD shape", cell_type, dim);
   if (order != 0 && order != 1)
      return SetError(UBOLT_ERR_ARG, "the unstructured backend is DG0 or DG1, was asked for order %d", order);
   if (n_cells <= 0 || n_vertices <= 0 || !vertices || !cell_vertices || !side_bc)
      return SetError(UBOLT_ERR_ARG, "empty mesh or NULL array");

   auto g = std::make_unique<ubolt_geometry_owned>();
   const int F = shape->n_faces, nvc = shape->n_vertices, nvf = shape->verts_per_face;
   const int nb = (order == 0) ? 1 : dim + 1;
   g->dim = dim;
   g->nb = nb;
   g->F = F;
   g->n_cells = n_cells;

   auto X = [&](int64_t v, double x[3]) {
      for (int d = 0; d < 3; d++) x[d] = (d < dim) ? vertices[v * dim + d] : 0.0;
   };
   for (int64_t i = 0; i < n_cells * nvc; i++)
      if (cell_vertices[i] < 0 || cell_vertices[i] >= n_vertices)
         return SetError(UBOLT_ERR_ARG, "cell %lld names vertex %lld of %lld", (long long)(i / nvc),
                         (long long)cell_vertices[i], (long long)n_vertices);

   // Bounding box: the sides the boundary faces are labelled by
   double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
   for (int d = 0; d < dim; d++) {
      lo[d] = hi[d] = vertices[d];
      for (int64_t v = 0; v < n_vertices; v++) {
         lo[d] = std::min(lo[d], vertices[v * dim + d]);
         hi[d] = std::max(hi[d], vertices[v * dim + d]);
      }
   }

   // ~~~~~ Face matching by sorted vertex ids
   const int64_t n_slots = n_cells * F;
   std::vector<FaceKey> keys(n_slots);
   for (int64_t c = 0; c < n_cells; c++)
      for (int lf = 0; lf < F; lf++) {
         FaceKey &k = keys[c * F + lf];
         for (int i = 0; i < 4; i++) k.v[i] = (i < nvf) ? cell_vertices[c * nvc + shape->face[lf][i]] : -1;
         std::sort(k.v, k.v + nvf);
         k.slot = c * F + lf;
      }
   std::vector<FaceKey> sorted = keys;
   std::sort(sorted.begin(), sorted.end());
   g->face_neighbour.assign(n_slots, -1);
   for (int64_t i = 0; i < n_slots;) {
      int64_t j = i + 1;
      while (j < n_slots && sorted[j].same(sorted[i])) j++;
      if (j - i > 2) return SetError(UBOLT_ERR_ARG, "a face is shared by %lld cells", (long long)(j - i));
      if (j - i == 2) {
         g->face_neighbour[sorted[i].slot] = sorted[i + 1].slot / F;
         g->face_neighbour[sorted[i + 1].slot] = sorted[i].slot / F;
      }
      i = j;
   }

   // ~~~~~ Per cell: fan moments, volume, centroid; per face: area, normal
   g->volume.assign(n_cells, 0.0);
   g->centroid.assign(3 * n_cells, 0.0);
   g->face_nA.assign(3 * n_slots, 0.0);
   g->face_centroid.assign(3 * n_slots, 0.0);
   g->face_distance.assign(2 * n_slots, 0.0);
   g->face_bc.assign(n_slots, -1);
   g->face_side.assign(n_slots, -1);
   g->face_axis.assign(n_slots, 0);
   std::vector<double> face_area(n_slots), face_central(9 * n_slots), central(9 * n_cells);

   int bad = 0;
   char msg[256] = "";
#pragma omp parallel for schedule(static)
   for (int64_t c = 0; c < n_cells; c++) {
      double xv[8][3], cref[3] = {0, 0, 0};
      for (int v = 0; v < nvc; v++) {
         X(cell_vertices[c * nvc + v], xv[v]);
         for (int d = 0; d < 3; d++) cref[d] += xv[v][d] / nvc;
      }
      // Faces first: the 3D cell fan needs the face centroids
      FaceGeom fg[6];
      for (int lf = 0; lf < F; lf++) {
         double xf[4][3];
         for (int i = 0; i < nvf; i++)
            for (int d = 0; d < 3; d++) xf[i][d] = xv[shape->face[lf][i]][d];
         FaceMomentsOf(dim, nvf, xf, fg[lf]);
      }
      Moments m;
      for (int lf = 0; lf < F; lf++) {
         if (dim == 2) {
            double y[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            Sub3(xv[shape->face[lf][0]], cref, y[1]);
            Sub3(xv[shape->face[lf][1]], cref, y[2]);
            AddSimplex(m, 2, 0.5 * std::fabs(y[1][0] * y[2][1] - y[1][1] * y[2][0]), y);
         } else {
            for (int e = 0; e < nvf; e++) {
               double y[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
               Sub3(fg[lf].centroid, cref, y[1]);
               Sub3(xv[shape->face[lf][e]], cref, y[2]);
               Sub3(xv[shape->face[lf][(e + 1) % nvf]], cref, y[3]);
               const double det = y[1][0] * (y[2][1] * y[3][2] - y[2][2] * y[3][1]) -
                                  y[1][1] * (y[2][0] * y[3][2] - y[2][2] * y[3][0]) +
                                  y[1][2] * (y[2][0] * y[3][1] - y[2][1] * y[3][0]);
               AddSimplex(m, 3, std::fabs(det) / 6.0, y);
            }
         }
      }
      double cen[3];
      Centralise(m, cref, cen, &central[9 * c]);
      g->volume[c] = m.m0;
      for (int d = 0; d < 3; d++) g->centroid[3 * c + d] = cen[d];
      if (!(m.m0 > 0.0)) {
#pragma omp critical
         { bad = 1; snprintf(msg, sizeof msg, "cell %lld has non-positive volume", (long long)c); }
      }

      for (int lf = 0; lf < F; lf++) {
         const int64_t k = c * F + lf;
         const FaceGeom &f = fg[lf];
         // Outward by the centroid test (OutwardAreaNormal, plex_commonk.hpp:295-307)
         double outward = 0.0;
         for (int d = 0; d < dim; d++) outward += f.normal[d] * (f.centroid[d] - cen[d]);
         const double sign = (outward < 0.0) ? -1.0 : 1.0;
         double nA[3] = {0, 0, 0};
         for (int d = 0; d < dim; d++) nA[d] = sign * f.area * f.normal[d];
         for (int d = 0; d < 3; d++) {
            g->face_nA[3 * k + d] = nA[d];
            g->face_centroid[3 * k + d] = f.centroid[d];
         }
         face_area[k] = f.area;
         for (int i = 0; i < 9; i++) face_central[9 * k + i] = f.central[i];
         // DominantAxis: the largest |n_d|, lowest axis on a tie (plex_commonk.hpp:282-289)
         int axis = 0;
         for (int d = 1; d < dim; d++)
            if (std::fabs(nA[d]) > std::fabs(nA[axis])) axis = d;
         g->face_axis[k] = axis;
         double dist_own = 0.0;
         for (int d = 0; d < dim; d++) dist_own += nA[d] / f.area * (f.centroid[d] - cen[d]);
         g->face_distance[2 * k] = dist_own;
         if (!(dist_own > 0.0)) {
#pragma omp critical
            { bad = 1; snprintf(msg, sizeof msg, "the centroid of cell %lld is not inside its face %d", (long long)c, lf); }
         }
      }
   }
   if (bad) return SetError(UBOLT_ERR_ARG, "%s", msg);

   // Neighbour distances and boundary sides (needs every centroid)
   for (int64_t k = 0; k < n_slots; k++) {
      const int64_t nbr = g->face_neighbour[k];
      const double *nA = &g->face_nA[3 * k], *fc = &g->face_centroid[3 * k];
      if (nbr >= 0) {
         double dist = 0.0;
         for (int d = 0; d < dim; d++) dist += nA[d] / face_area[k] * (g->centroid[3 * nbr + d] - fc[d]);
         g->face_distance[2 * k + 1] = dist;
         if (!(dist > 0.0))
            return SetError(UBOLT_ERR_ARG, "the centroid of cell %lld is not inside its face", (long long)nbr);
      } else {
         const int axis = g->face_axis[k];
         const int side = 2 * axis + (nA[axis] > 0.0 ? 1 : 0);
         const double plane = (side & 1) ? hi[axis] : lo[axis];
         if (std::fabs(fc[axis] - plane) > 1e-9 * std::max(1.0, hi[axis] - lo[axis]))
            return SetError(UBOLT_ERR_ARG, "boundary face %lld of cell %lld is not on a side of the mesh's box",
                            (long long)(k % F), (long long)(k / F));
         g->face_side[k] = side;
         g->face_bc[k] = side_bc[side];
         if (side_bc[side] != UBOLT_BC_VACUUM && side_bc[side] != UBOLT_BC_REFLECT)
            return SetError(UBOLT_ERR_ARG, "side %d has unknown boundary family %d", side, side_bc[side]);
         // CheckBoundaryFaceBC (plex_commonk.hpp:323-339): reflection needs an axis-aligned face
         if (side_bc[side] == UBOLT_BC_REFLECT && std::fabs(nA[axis]) < (1.0 - 1e-10) * face_area[k])
            return SetError(UBOLT_ERR_ARG, "face %lld of cell %lld is reflective but not axis-aligned",
                            (long long)(k % F), (long long)(k / F));
      }
   }

   if (order == 1) {
      // ~~~~~ DG1: basis and face matrices (build_dg1_geometry, :706-821)
      std::vector<double> beta(9 * n_cells);
      for (int64_t c = 0; c < n_cells; c++)
         if (!OrthonormalGradients(dim, g->volume[c], &central[9 * c], &beta[9 * c]))
            return SetError(UBOLT_ERR_ARG, "cell %lld has a degenerate second moment", (long long)c);
      auto value = [&](int64_t m, int i, const double *x) {
         if (i == 0) return 1.0;
         double v = 0.0;
         for (int d = 0; d < 3; d++) v += beta[9 * m + 3 * (i - 1) + d] * (x[d] - g->centroid[3 * m + d]);
         return v;
      };
      auto grad = [&](int64_t m, int i, int d) { return (i == 0) ? 0.0 : beta[9 * m + 3 * (i - 1) + d]; };

      g->face_own.assign(n_slots * nb * nb, 0.0);
      g->face_up.assign(n_slots * nb * nb, 0.0);
      g->face_basis_value.assign(n_slots * nb, 0.0);
      g->basis_grad.assign(n_cells * nb * 3, 0.0);
      g->face_nb_grad.assign(n_slots * nb * 3, 0.0);
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < n_cells; c++) {
         for (int i = 0; i < nb; i++)
            for (int d = 0; d < 3; d++) g->basis_grad[(c * nb + i) * 3 + d] = grad(c, i, d);
         for (int lf = 0; lf < F; lf++) {
            const int64_t k = c * F + lf;
            const double area = face_area[k], *xf = &g->face_centroid[3 * k], *Cf = &face_central[9 * k];
            int64_t up = -1;
            if (g->face_neighbour[k] >= 0) {
               up = g->face_neighbour[k];
               for (int j = 0; j < nb; j++)
                  for (int d = 0; d < 3; d++) g->face_nb_grad[(k * nb + j) * 3 + d] = grad(up, j, d);
            } else if (g->face_bc[k] == UBOLT_BC_REFLECT)
               up = c;
            const double scale = 1.0 / (g->volume[c] * area);
            for (int i = 0; i < nb; i++) {
               const double vi = value(c, i, xf);
               g->face_basis_value[k * nb + i] = vi;
               for (int j = 0; j < nb; j++) {
                  double own = area * vi * value(c, j, xf);
                  for (int a = 0; a < 3; a++)
                     for (int b = 0; b < 3; b++) own += grad(c, i, a) * Cf[3 * a + b] * grad(c, j, b);
                  g->face_own[(k * nb + i) * nb + j] = own * scale;
                  if (up < 0) continue;
                  double cross = area * vi * value(up, j, xf);
                  for (int a = 0; a < 3; a++)
                     for (int b = 0; b < 3; b++) cross += grad(c, i, a) * Cf[3 * a + b] * grad(up, j, b);
                  g->face_up[(k * nb + i) * nb + j] = cross * scale;
               }
            }
         }
      }
   }

   *out = g.release();
   return UBOLT_OK;
}

extern "C" int ubolt_geometry_view(const ubolt_geometry_owned *g, ubolt_dg_geometry *v)
{
   if (!g || !v) return ubolt::SetError(UBOLT_ERR_ARG, "ubolt_geometry_view: NULL argument");
   std::memset(v, 0, sizeof *v);
   v->dim = g->dim;
   v->n_basis = g->nb;
   v->faces_per_cell = g->F;
   v->n_cells = g->n_cells;
   v->volume = g->volume.data();
   v->centroid = g->centroid.data();
   v->face_nA = g->face_nA.data();
   v->face_neighbour = g->face_neighbour.data();
   v->face_bc = g->face_bc.data();
   v->face_side = g->face_side.data();
   v->face_axis = g->face_axis.data();
   v->face_centroid = g->face_centroid.data();
   v->face_distance = g->face_distance.data();
   if (g->nb > 1) {
      v->face_own = g->face_own.data();
      v->face_up = g->face_up.data();
      v->basis_grad = g->basis_grad.data();
      v->face_neighbour_grad = g->face_nb_grad.data();
      v->face_basis_value = g->face_basis_value.data();
   }
   return UBOLT_OK;
}

extern "C" void ubolt_geometry_free(ubolt_geometry_owned *g) { delete g; }
