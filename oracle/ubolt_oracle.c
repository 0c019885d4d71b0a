/*
 * CPU oracle for the B200 transport path - TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of UBOLT's ASSEMBLED operator and its companions, for
 * tests/, __graft_entry__.smoke() and bench.py's CPU baseline to check the
 * CUDA library against. Nothing in the library links or calls this.
 *
 * What it restates (paths within stevendargaville/UBOLT):
 *   oracle_assemble_dg    StreamingTermDG0/DG1::assemble_add + RemovalTerm::assemble_add
 *                         into the slot pattern of UnstructuredDG::create
 *                         (src/termsk.kokkos.cxx:197-240, 314-389, 451-470;
 *                          src/unstructured_dgk.kokkos.cxx:442-540)
 *   oracle_assemble_fd2d  StructuredStreamingKernel<2> on the ghost-flux rows of
 *                         ClassifyRow / BuildStructuredCOO
 *                         (src/termsk.kokkos.cxx:64-98; src/structured_fd_commonk.hpp:231-400)
 *   oracle_scatter_add    ScatteringTerm::apply_add (src/termsk.kokkos.cxx:584-649)
 *   oracle_block_inverse  InvertBlocksKernel / ApplyKernel (src/block_inversek.kokkos.cxx:83-150, 206-222)
 *   oracle_add_source     AddIsotropicKernel (src/material_speck.kokkos.cxx:164-187)
 *   oracle_add_transfer   GroupTransfer::add_transfer (src/multigroupk.kokkos.cxx:306-365)
 *   oracle_ghost_inflow   the ghost-flux inflow rows (src/unstructured_dgk.kokkos.cxx:476-494)
 *   oracle_angular_integral UboltAngularIntegral (src/sn_quadraturek.kokkos.cxx:400-427)
 *   oracle_solve          right-preconditioned restarted GMRES on the shell operator
 *                         (KSPGMRES with PC_RIGHT, src/transport_solverk.kokkos.cxx:196-318),
 *                         its preconditioner an exact upwind sweep of the assembled
 *                         streaming + removal (the streaming stage PCAIR approximates)
 *                         or the element-block Jacobi of the removal stage.
 *
 * Conventions: row = (cell * nb + i) * A + a (include/ubolt/phase_space.hpp:20-28).
 * CSR columns are sorted per row and duplicate slots summed, as
 * MatSetValuesCOO does. Ghost-flux boundaries only (the only treatment at DG1).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXB 4
#define BC_VACUUM 0
#define BC_REFLECT 1

/* Omega_a . nA_k in FaceFlux's term order (src/plex_commonk.hpp:314-317) */
static inline double face_flux(const double *omega, int a, const double *nA, int64_t k)
{
   return omega[3 * a] * nA[3 * k] + omega[3 * a + 1] * nA[3 * k + 1] + omega[3 * a + 2] * nA[3 * k + 2];
}

typedef struct {
   int64_t col;
   double val;
} entry_t;

static int cmp_entry(const void *a, const void *b)
{
   const int64_t x = ((const entry_t *)a)->col, y = ((const entry_t *)b)->col;
   return (x > y) - (x < y);
}

/* Sort a row's slots by column and sum duplicates; returns the count kept. */
static int finish_row(entry_t *e, int n)
{
   if (n == 0) return 0;
   qsort(e, (size_t)n, sizeof(entry_t), cmp_entry);
   int m = 0;
   for (int s = 1; s < n; s++) {
      if (e[s].col == e[m].col) e[m].val += e[s].val;
      else e[++m] = e[s];
   }
   return m + 1;
}

/* Upper bound of the nonzeros of the DG operator: F nb + nb slots per row. */
int64_t oracle_dg_nnz_bound(int nb, int F, int64_t n_cells, int A)
{
   return n_cells * nb * (int64_t)A * (int64_t)(F * nb + nb);
}

/*
 * Streaming + removal of the unstructured DG backend, order 0 (nb = 1) or 1.
 * face_bc: -1 interior, else the face's BC family; face_axis its dominant axis.
 * reflect: [3][A]. Writes CSR row_ptr (n_rows + 1), col, val; returns nnz or -1.
 */
int64_t oracle_assemble_dg(int nb, int F, int64_t n_cells, int A, const double *face_nA, const int64_t *face_nbr,
                           const int32_t *face_bc, const int32_t *face_axis, const double *volume,
                           const double *face_own, const double *face_up, const double *basis_grad,
                           const double *omega, const int32_t *reflect, const double *sigma_t, int64_t *row_ptr,
                           int64_t *col, double *val)
{
   const int64_t n_rows = n_cells * nb * (int64_t)A;
   const int per_row = F * nb + nb;
   /* Pass 1: every row's slots into a scratch of per_row entries */
   entry_t *scratch = (entry_t *)malloc(sizeof(entry_t) * (size_t)n_rows * per_row);
   int *count = (int *)malloc(sizeof(int) * (size_t)n_rows);
   if (!scratch || !count) { free(scratch); free(count); return -1; }

#pragma omp parallel for schedule(static)
   for (int64_t r = 0; r < n_rows; r++) {
      const int64_t node = r / A;
      const int a = (int)(r % A);
      const int64_t c = node / nb;
      const int i = (int)(node % nb);
      entry_t *e = scratch + r * per_row;
      int n = 0;
      if (nb == 1) {
         /* DG0: faces in cone order, then the diagonal (termsk.kokkos.cxx:197-240) */
         double outflow = 0.0;
         for (int k = 0; k < F; k++) {
            const double s = face_flux(omega, a, face_nA, c * F + k);
            if (s > 0.0) outflow += s;
         }
         const double inv_v = 1.0 / volume[c];
         for (int k = 0; k < F; k++) {
            const int64_t kf = c * F + k;
            const double s = face_flux(omega, a, face_nA, kf);
            const int interior = face_nbr[kf] >= 0;
            const int reflective = !interior && face_bc[kf] == BC_REFLECT;
            if (!(s < 0.0 && (interior || reflective))) continue; /* nulled slot */
            e[n].col = interior ? face_nbr[kf] * A + a : c * A + reflect[face_axis[kf] * A + a];
            e[n].val = 0.0;
            if (!(s > 0.0)) e[n].val += s * inv_v;
            n++;
         }
         e[n].col = r;
         e[n].val = outflow * inv_v; /* DG0OutflowDiagonal */
         e[n].val += sigma_t[c];     /* RemovalTerm on the diagonal slot */
         n++;
      } else {
         /* DG1: nb slots per face in cone order, then this cell's own nb */
         int own_base;
         for (int k = 0; k < F; k++) {
            const int64_t kf = c * F + k;
            const double s = face_flux(omega, a, face_nA, kf);
            const int interior = face_nbr[kf] >= 0;
            const int reflective = !interior && face_bc[kf] == BC_REFLECT;
            const int live = (s < 0.0) && (interior || reflective);
            for (int j = 0; j < nb; j++) {
               if (!live) continue;
               e[n].col = interior ? (face_nbr[kf] * nb + j) * A + a
                                   : (c * nb + j) * A + reflect[face_axis[kf] * A + a];
               e[n].val = 0.0;
               if (!(s > 0.0)) e[n].val += s * face_up[(kf * nb + i) * nb + j];
               n++;
            }
         }
         own_base = n;
         for (int j = 0; j < nb; j++) {
            e[n].col = (c * nb + j) * A + a;
            e[n].val = 0.0;
            n++;
         }
         for (int k = 0; k < F; k++) {
            const int64_t kf = c * F + k;
            const double s = face_flux(omega, a, face_nA, kf);
            if (s > 0.0)
               for (int j = 0; j < nb; j++)
                  if (j != i) e[own_base + j].val += s * face_own[(kf * nb + i) * nb + j];
         }
         if (i > 0) {
            const double *g = basis_grad + (c * nb + i) * 3;
            e[own_base].val -= omega[3 * a] * g[0] + omega[3 * a + 1] * g[1] + omega[3 * a + 2] * g[2];
         }
         {
            double diag = 0.0; /* DG1OutflowDiagonal */
            for (int k = 0; k < F; k++) {
               const int64_t kf = c * F + k;
               const double s = face_flux(omega, a, face_nA, kf);
               if (s > 0.0) diag += s * face_own[(kf * nb + i) * nb + i];
            }
            e[own_base + i].val += diag;
         }
         e[own_base + i].val += sigma_t[c];
      }
      count[r] = finish_row(e, n);
   }
   row_ptr[0] = 0;
   for (int64_t r = 0; r < n_rows; r++) row_ptr[r + 1] = row_ptr[r] + count[r];
#pragma omp parallel for schedule(static)
   for (int64_t r = 0; r < n_rows; r++) {
      const entry_t *e = scratch + r * per_row;
      for (int s = 0; s < count[r]; s++) {
         col[row_ptr[r] + s] = e[s].col;
         val[row_ptr[r] + s] = e[s].val;
      }
   }
   const int64_t nnz = row_ptr[n_rows];
   free(scratch);
   free(count);
   return nnz;
}

/*
 * 2D structured upwind FD, ghost-flux rows (StructuredFD2D): cells natural
 * (x fastest), rows cell * A + a, diagonal sum_d |cos_d| / h_d, upwind slot
 * -|cos_d| / h_d on the in-domain neighbour, a reflective side's slot
 * repointed to the mirrored angle in the cell, a vacuum side's slot nulled.
 * side_bc[4] = x low, x high, y low, y high. Returns nnz.
 */
int64_t oracle_assemble_fd2d(int nx, int ny, double hx, double hy, int A, const double *mu, const double *eta,
                             const int32_t *reflect, const int32_t *side_bc, const double *sigma_t,
                             int64_t *row_ptr, int64_t *col, double *val)
{
   const int64_t n_rows = (int64_t)nx * ny * A;
   int64_t nz = 0;
   row_ptr[0] = 0;
   for (int64_t r = 0; r < n_rows; r++) {
      const int64_t cell = r / A;
      const int a = (int)(r % A);
      const int idx[2] = {(int)(cell % nx), (int)(cell / nx)};
      const int n[2] = {nx, ny};
      const double cosv[2] = {mu[a], eta[a]};
      const double h[2] = {hx, hy};
      entry_t e[3];
      int m = 0;
      double cd[2];
      cd[0] = fabs(cosv[0]) / h[0];
      cd[1] = fabs(cosv[1]) / h[1];
      double diag = cd[0];
      diag += cd[1];
      for (int d = 0; d < 2; d++) {
         if (cosv[d] == 0.0) continue;
         const int up = cosv[d] > 0 ? idx[d] - 1 : idx[d] + 1;
         const int side = 2 * d + (cosv[d] > 0 ? 0 : 1);
         int64_t c;
         if (up >= 0 && up < n[d]) {
            int j[2] = {idx[0], idx[1]};
            j[d] = up;
            c = ((int64_t)j[1] * nx + j[0]) * A + a;
         } else if (side_bc[side] == BC_REFLECT) {
            c = cell * A + reflect[d * A + a];
         } else
            continue;
         e[m].col = c;
         e[m].val = -cd[d];
         m++;
      }
      e[m].col = r;
      e[m].val = diag + sigma_t[cell];
      m++;
      m = finish_row(e, m);
      for (int s = 0; s < m; s++) {
         col[nz] = e[s].col;
         val[nz] = e[s].val;
         nz++;
      }
      row_ptr[r + 1] = nz;
   }
   return nz;
}

/* y = A x over a CSR */
void oracle_spmv(int64_t n_rows, const int64_t *row_ptr, const int64_t *col, const double *val, const double *x,
                 double *y)
{
#pragma omp parallel for schedule(static)
   for (int64_t r = 0; r < n_rows; r++) {
      double s = 0.0;
      for (int64_t p = row_ptr[r]; p < row_ptr[r + 1]; p++) s += val[p] * x[col[p]];
      y[r] = s;
   }
}

/* phi(node) = sum_a w_a psi(node, a) */
void oracle_angular_integral(int64_t n_nodes, int A, const double *w, const double *psi, double *phi)
{
#pragma omp parallel for schedule(static)
   for (int64_t n = 0; n < n_nodes; n++) {
      double s = 0.0;
      for (int a = 0; a < A; a++) s += psi[n * A + a] * w[a];
      phi[n] = s;
   }
}

/* y(node, a) -= sigma_s(cell) / W * sum_b w_b x(node, b): the scatter's apply_add */
void oracle_scatter_add(int64_t n_cells, int nb, int A, const double *w, double sum_weights, const double *sigma_s,
                        const double *x, double *y)
{
#pragma omp parallel for schedule(static)
   for (int64_t n = 0; n < n_cells * nb; n++) {
      double phi = 0.0;
      for (int a = 0; a < A; a++) phi += x[n * A + a] * w[a];
      phi *= sigma_s[n / nb] / sum_weights;
      for (int a = 0; a < A; a++) y[n * A + a] -= phi;
   }
}

/* b(cell, 0, a) += q(cell) / W */
void oracle_add_source(int64_t n_cells, int nb, int A, double sum_weights, const double *q, double *b)
{
   for (int64_t c = 0; c < n_cells; c++) {
      const double v = q[c] / sum_weights;
      for (int a = 0; a < A; a++) b[c * nb * A + a] += v;
   }
}

/* b(node, a) += phi(node) * (sigma_s(cell) / W) */
void oracle_add_transfer(int64_t n_cells, int nb, int A, double sum_weights, const double *phi,
                         const double *sigma_s, double *b)
{
   for (int64_t n = 0; n < n_cells * nb; n++) {
      const double v = phi[n] * (sigma_s[n / nb] / sum_weights);
      for (int a = 0; a < A; a++) b[n * A + a] += v;
   }
}

/* Ghost-flux vacuum inflow rows: b += -(s / V) phi_i(x_f) inflow / W */
void oracle_ghost_inflow(int nb, int F, int64_t n_cells, int A, const double *face_nA, const int64_t *face_nbr,
                         const int32_t *face_bc, const int32_t *face_side, const double *volume,
                         const double *face_basis_value, const double *omega, double sum_weights,
                         const double *side_inflow, double *b)
{
   for (int64_t c = 0; c < n_cells; c++)
      for (int i = 0; i < nb; i++)
         for (int a = 0; a < A; a++) {
            double g = 0.0;
            for (int k = 0; k < F; k++) {
               const int64_t kf = c * F + k;
               if (face_nbr[kf] >= 0 || face_bc[kf] != BC_VACUUM) continue;
               const double s = face_flux(omega, a, face_nA, kf);
               if (!(s < 0.0)) continue;
               const double phi_i = (nb == 1) ? 1.0 : face_basis_value[kf * nb + i];
               g += -s / volume[c] * phi_i * (side_inflow[face_side[kf]] / sum_weights);
            }
            b[(c * nb + i) * A + a] += g;
         }
}

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * Element blocks, read from the CSR (InvertBlocksKernel)
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

static void read_block(int64_t c, int a, int nb, int A, const int64_t *row_ptr, const int64_t *col,
                       const double *val, double m[MAXB][MAXB])
{
   for (int i = 0; i < nb; i++) {
      for (int j = 0; j < nb; j++) m[i][j] = 0.0;
      const int64_t r = (c * nb + i) * A + a;
      for (int64_t p = row_ptr[r]; p < row_ptr[r + 1]; p++) {
         const int64_t cl = col[p];
         if (cl % A != a || cl / ((int64_t)nb * A) != c) continue;
         m[i][(cl / A) % nb] = val[p];
      }
   }
}

/* Gauss-Jordan with partial pivoting; 0 on a singular block */
static int gauss_jordan(int nb, double m[MAXB][MAXB], double w[MAXB][MAXB])
{
   for (int i = 0; i < nb; i++)
      for (int j = 0; j < nb; j++) w[i][j] = (i == j) ? 1.0 : 0.0;
   for (int k = 0; k < nb; k++) {
      int piv = k;
      for (int i = k + 1; i < nb; i++)
         if (fabs(m[i][k]) > fabs(m[piv][k])) piv = i;
      if (fabs(m[piv][k]) == 0.0) return 0;
      if (piv != k)
         for (int j = 0; j < nb; j++) {
            double t = m[k][j]; m[k][j] = m[piv][j]; m[piv][j] = t;
            t = w[k][j]; w[k][j] = w[piv][j]; w[piv][j] = t;
         }
      const double inv = 1.0 / m[k][k];
      for (int j = 0; j < nb; j++) { m[k][j] *= inv; w[k][j] *= inv; }
      for (int i = 0; i < nb; i++) {
         if (i == k) continue;
         const double f = m[i][k];
         if (f == 0.0) continue;
         for (int j = 0; j < nb; j++) { m[i][j] -= f * m[k][j]; w[i][j] -= f * w[k][j]; }
      }
   }
   return 1;
}

/* inv[((c * A + a) * nb + i) * nb + j]; returns the number of singular blocks */
int64_t oracle_block_inverse(int64_t n_cells, int nb, int A, const int64_t *row_ptr, const int64_t *col,
                             const double *val, double *inv)
{
   int64_t n_singular = 0;
#pragma omp parallel for schedule(static) reduction(+ : n_singular)
   for (int64_t b = 0; b < n_cells * A; b++) {
      double m[MAXB][MAXB], w[MAXB][MAXB];
      read_block(b / A, (int)(b % A), nb, A, row_ptr, col, val, m);
      const int ok = gauss_jordan(nb, m, w);
      if (!ok) n_singular++;
      for (int i = 0; i < nb; i++)
         for (int j = 0; j < nb; j++) inv[(b * nb + i) * nb + j] = ok ? w[i][j] : 0.0;
   }
   return n_singular;
}

/* y(r_i) = sum_j inv(i, j) x(r_j) */
void oracle_block_apply(int64_t n_cells, int nb, int A, const double *inv, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
   for (int64_t b = 0; b < n_cells * A; b++) {
      const int64_t c = b / A;
      const int a = (int)(b % A);
      double v[MAXB];
      for (int j = 0; j < nb; j++) v[j] = x[(c * nb + j) * A + a];
      for (int i = 0; i < nb; i++) {
         double s = 0.0;
         for (int j = 0; j < nb; j++) s += inv[(b * nb + i) * nb + j] * v[j];
         y[(c * nb + i) * A + a] = s;
      }
   }
}

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * The solve
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

typedef struct {
   int64_t n_cells;
   int nb, A;
   const int64_t *row_ptr, *col;
   const double *val;
   const double *w;
   double sum_weights;
   const double *sigma_s;
   int pc; /* 0 none, 1 block Jacobi, 2 sweep */
   int64_t *order;      /* [A][n_cells] topological cell order per angle */
   double *inv;         /* block inverses for pc 1 */
} oracle_sys;

static void shell_apply(const oracle_sys *s, const double *x, double *y)
{
   const int64_t n = s->n_cells * s->nb * (int64_t)s->A;
   oracle_spmv(n, s->row_ptr, s->col, s->val, x, y);
   oracle_scatter_add(s->n_cells, s->nb, s->A, s->w, s->sum_weights, s->sigma_s, x, y);
}

/* Per angle, a topological order of the cells over the interior upwind
 * couplings in the CSR (Kahn); a cycle is broken by taking the remaining cell
 * of least in-degree, its unresolved upwind values lagged (read as zero). */
static void sweep_orders(oracle_sys *s)
{
   const int64_t nc = s->n_cells;
   const int nb = s->nb, A = s->A;
   s->order = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc * A));
#pragma omp parallel for schedule(dynamic, 1)
   for (int a = 0; a < A; a++) {
      int64_t *indeg = (int64_t *)calloc((size_t)nc, sizeof(int64_t));
      int64_t *ptr = (int64_t *)calloc((size_t)(nc + 1), sizeof(int64_t));
      int64_t *adj, *queue = s->order + (int64_t)a * nc;
      char *done = (char *)calloc((size_t)nc, 1);
      /* edges up -> c from row (c, 0, a) (every basis row carries the same columns) */
      for (int64_t c = 0; c < nc; c++) {
         const int64_t r = (c * nb) * A + a;
         for (int64_t p = s->row_ptr[r]; p < s->row_ptr[r + 1]; p++) {
            const int64_t cl = s->col[p], up = cl / ((int64_t)nb * A);
            if (up != c && cl % A == a) { ptr[up + 1]++; indeg[c]++; }
         }
      }
      for (int64_t c = 0; c < nc; c++) ptr[c + 1] += ptr[c];
      adj = (int64_t *)malloc(sizeof(int64_t) * (size_t)(ptr[nc] + 1));
      int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)nc);
      memcpy(fill, ptr, sizeof(int64_t) * (size_t)nc);
      for (int64_t c = 0; c < nc; c++) {
         const int64_t r = (c * nb) * A + a;
         for (int64_t p = s->row_ptr[r]; p < s->row_ptr[r + 1]; p++) {
            const int64_t cl = s->col[p], up = cl / ((int64_t)nb * A);
            if (up != c && cl % A == a) adj[fill[up]++] = c;
         }
      }
      int64_t head = 0, tail = 0;
      for (int64_t c = 0; c < nc; c++)
         if (indeg[c] == 0) { queue[tail++] = c; done[c] = 1; }
      while (tail < nc) {
         while (head < tail) {
            const int64_t u = queue[head++];
            for (int64_t p = ptr[u]; p < ptr[u + 1]; p++) {
               const int64_t v = adj[p];
               if (--indeg[v] == 0 && !done[v]) { queue[tail++] = v; done[v] = 1; }
            }
         }
         if (tail < nc) { /* a cycle: force the least-blocked cell */
            int64_t best = -1;
            for (int64_t c = 0; c < nc; c++)
               if (!done[c] && (best < 0 || indeg[c] < indeg[best])) best = c;
            queue[tail++] = best;
            done[best] = 1;
         }
      }
      free(indeg); free(ptr); free(adj); free(fill); free(done);
   }
}

/* psi = L^{-1} q over the assembled streaming + removal; reflective couplings
 * (same cell, another angle) and cycle-breaking couplings are read from psi
 * as it stands - zero-initialised, so they are lagged to zero. */
static void sweep(const oracle_sys *s, const double *q, double *psi)
{
   const int64_t nc = s->n_cells;
   const int nb = s->nb, A = s->A;
   const int64_t n = nc * nb * (int64_t)A;
   memset(psi, 0, sizeof(double) * (size_t)n);
#pragma omp parallel for schedule(dynamic, 1)
   for (int a = 0; a < A; a++) {
      const int64_t *ord = s->order + (int64_t)a * nc;
      for (int64_t t = 0; t < nc; t++) {
         const int64_t c = ord[t];
         double m[MAXB][MAXB], w[MAXB][MAXB], rhs[MAXB];
         for (int i = 0; i < nb; i++) {
            for (int j = 0; j < nb; j++) m[i][j] = 0.0;
            const int64_t r = (c * nb + i) * A + a;
            double v = q[r];
            for (int64_t p = s->row_ptr[r]; p < s->row_ptr[r + 1]; p++) {
               const int64_t cl = s->col[p];
               const int64_t cc = cl / ((int64_t)nb * A);
               if (cc == c && cl % A == a) m[i][(cl / A) % nb] = s->val[p];
               else if (cl % A == a) v -= s->val[p] * psi[cl];
            }
            rhs[i] = v;
         }
         gauss_jordan(nb, m, w);
         for (int i = 0; i < nb; i++) {
            double y = 0.0;
            for (int j = 0; j < nb; j++) y += w[i][j] * rhs[j];
            psi[(c * nb + i) * A + a] = y;
         }
      }
   }
}

static void precondition(const oracle_sys *s, const double *x, double *y)
{
   const int64_t n = s->n_cells * s->nb * (int64_t)s->A;
   if (s->pc == 2) sweep(s, x, y);
   else if (s->pc == 1) oracle_block_apply(s->n_cells, s->nb, s->A, s->inv, x, y);
   else memcpy(y, x, sizeof(double) * (size_t)n);
}

static double dot(int64_t n, const double *a, const double *b)
{
   double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
   for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
   return s;
}

/*
 * Solve (L - S) x = b by right-preconditioned restarted GMRES (modified
 * Gram-Schmidt, Givens rotations), stopping when the true residual estimate
 * falls below rtol ||b||. x holds the initial guess. Returns the iteration
 * count, negative if max_it was reached; final_resid receives ||b - A x|| / ||b||.
 */
int oracle_solve(int64_t n_cells, int nb, int A, const int64_t *row_ptr, const int64_t *col, const double *val,
                 const double *w, double sum_weights, const double *sigma_s, const double *b, double *x,
                 double rtol, int max_it, int restart, int pc, double *final_resid)
{
   oracle_sys s = {n_cells, nb, A, row_ptr, col, val, w, sum_weights, sigma_s, pc, NULL, NULL};
   const int64_t n = n_cells * nb * (int64_t)A;
   const int m = restart;
   if (pc == 2) sweep_orders(&s);
   if (pc == 1) {
      s.inv = (double *)malloc(sizeof(double) * (size_t)(n_cells * A * nb * nb));
      oracle_block_inverse(n_cells, nb, A, row_ptr, col, val, s.inv);
   }
   double *V = (double *)malloc(sizeof(double) * (size_t)n * (m + 1));
   double *z = (double *)malloc(sizeof(double) * (size_t)n);
   double *r = (double *)malloc(sizeof(double) * (size_t)n);
   double *H = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
   double *cs = (double *)malloc(sizeof(double) * m), *sn = (double *)malloc(sizeof(double) * m);
   double *g = (double *)malloc(sizeof(double) * (m + 1)), *yv = (double *)malloc(sizeof(double) * m);
   const double bnorm = sqrt(dot(n, b, b));
   int it = 0, converged = 0;
   if (bnorm == 0.0) {
      memset(x, 0, sizeof(double) * (size_t)n);
      converged = 1;
   }
   while (!converged && it < max_it) {
      shell_apply(&s, x, r);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; i++) r[i] = b[i] - r[i];
      const double beta = sqrt(dot(n, r, r));
      if (beta <= rtol * bnorm) { converged = 1; break; }
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; i++) V[i] = r[i] / beta;
      for (int i = 0; i <= m; i++) g[i] = 0.0;
      g[0] = beta;
      int j = 0;
      for (; j < m && it < max_it; j++, it++) {
         double *vj = V + (int64_t)j * n, *vn = V + (int64_t)(j + 1) * n;
         precondition(&s, vj, z);
         shell_apply(&s, z, vn);
         for (int i = 0; i <= j; i++) {
            const double h = dot(n, vn, V + (int64_t)i * n);
            H[i * m + j] = h;
            const double *vi = V + (int64_t)i * n;
#pragma omp parallel for schedule(static)
            for (int64_t k = 0; k < n; k++) vn[k] -= h * vi[k];
         }
         const double hn = sqrt(dot(n, vn, vn));
         H[(j + 1) * m + j] = hn;
         if (hn > 0.0) {
#pragma omp parallel for schedule(static)
            for (int64_t k = 0; k < n; k++) vn[k] /= hn;
         }
         for (int i = 0; i < j; i++) {
            const double t = cs[i] * H[i * m + j] + sn[i] * H[(i + 1) * m + j];
            H[(i + 1) * m + j] = -sn[i] * H[i * m + j] + cs[i] * H[(i + 1) * m + j];
            H[i * m + j] = t;
         }
         const double d = sqrt(H[j * m + j] * H[j * m + j] + hn * hn);
         cs[j] = H[j * m + j] / d;
         sn[j] = hn / d;
         H[j * m + j] = d;
         g[j + 1] = -sn[j] * g[j];
         g[j] = cs[j] * g[j];
         if (fabs(g[j + 1]) <= rtol * bnorm || hn == 0.0) { j++; it++; break; }
      }
      /* x += M^{-1} V y */
      for (int i = j - 1; i >= 0; i--) {
         double t = g[i];
         for (int k = i + 1; k < j; k++) t -= H[i * m + k] * yv[k];
         yv[i] = t / H[i * m + i];
      }
      memset(r, 0, sizeof(double) * (size_t)n);
      for (int i = 0; i < j; i++) {
         const double *vi = V + (int64_t)i * n;
#pragma omp parallel for schedule(static)
         for (int64_t k = 0; k < n; k++) r[k] += yv[i] * vi[k];
      }
      precondition(&s, r, z);
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < n; k++) x[k] += z[k];
   }
   shell_apply(&s, x, r);
#pragma omp parallel for schedule(static)
   for (int64_t i = 0; i < n; i++) r[i] = b[i] - r[i];
   const double res = (bnorm > 0.0) ? sqrt(dot(n, r, r)) / bnorm : 0.0;
   if (final_resid) *final_resid = res;
   free(V); free(z); free(r); free(H); free(cs); free(sn); free(g); free(yv);
   free(s.order); free(s.inv);
   return (res <= rtol * 1.0000001 || converged) ? it : -it;
}

/* The sweep alone, for tests: psi = L^{-1} q with lagged reflective couplings */
void oracle_sweep(int64_t n_cells, int nb, int A, const int64_t *row_ptr, const int64_t *col, const double *val,
                  const double *q, double *psi)
{
   oracle_sys s = {n_cells, nb, A, row_ptr, col, val, NULL, 0.0, NULL, 2, NULL, NULL};
   sweep_orders(&s);
   sweep(&s, q, psi);
   free(s.order);
}

int oracle_threads(void)
{
#ifdef _OPENMP
   return omp_get_max_threads();
#else
   return 1;
#endif
}

/* ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
 * DSA diffusion operators (DSAPlex, src/dsa_plexk.kokkos.cxx): D per cell
 * from the void policy (1/(3 sigma_t) outside voids), sigma_a = sigma_t -
 * sigma_s, VOLUME-weighted rows. Output as COO (row, col, val) with the
 * reference's entry order per row; a masked void's zeroed couplings are left
 * out.
 * ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~ */

/* The void policy of DSAPrecon::assemble (src/dsak.kokkos.cxx:233-345) with
 * DSAPlex::void_volume_surface (src/dsa_plexk.kokkos.cxx:243-262), one rank,
 * a backend that can mask. A cell is void when sigma_t <= void_sigma_t. With
 * bridging asked for and some void, some non-void, and a vacuum face or some
 * absorption anywhere, the voids are bridged when their mean chord 4 V / S
 * is positive (S: the void cells' faces onto non-void cells or vacuum
 * sides). D = 1/(3 sigma_t) outside voids; in a bridged void void_d if > 0,
 * else 1/(3 (max(sigma_t, 0) + 1/chord)); 0 in an unbridged void, which is
 * masked. Fills is_void, masked, d; out[0] = bridged, out[1] = chord,
 * out[2] = number of void cells. Returns 1 where the operator would be
 * singular (every face reflective, no void and no absorption), else 0. */
int oracle_dsa_void_policy(int F, int64_t n_cells, const double *face_nA, const int64_t *face_nbr,
                           const int32_t *face_bc, const double *volume, const double *sigma_t,
                           const double *sigma_s, double void_sigma_t, int bridge, double void_d,
                           uint8_t *is_void, uint8_t *masked, double *d, double *out)
{
   int64_t n_void = 0;
   double max_sa_all = 0.0, max_sa_solid = 0.0;
   int any_vacuum = 0;
   for (int64_t k = 0; k < n_cells * F; k++)
      if (face_nbr[k] < 0 && face_bc[k] == BC_VACUUM) any_vacuum = 1;
   for (int64_t c = 0; c < n_cells; c++) {
      const double sa = sigma_t[c] - sigma_s[c];
      is_void[c] = sigma_t[c] <= void_sigma_t;
      if (is_void[c]) n_void++;
      else if (sa > max_sa_solid) max_sa_solid = sa;
      if (sa > max_sa_all) max_sa_all = sa;
   }
   int bridged = 0;
   double chord = 0.0;
   if (bridge && n_void > 0 && n_void < n_cells && (any_vacuum || max_sa_all > 0.0)) {
      double vs0 = 0.0, vs1 = 0.0;
      for (int64_t c = 0; c < n_cells; c++) {
         if (!is_void[c]) continue;
         vs0 += volume[c];
         for (int f = 0; f < F; f++) {
            const int64_t k = c * F + f;
            const int64_t n = face_nbr[k];
            if (n >= 0 ? !is_void[n] : face_bc[k] == BC_VACUUM) {
               double area = 0.0;
               for (int dd = 0; dd < 3; dd++) area += face_nA[3 * k + dd] * face_nA[3 * k + dd];
               vs1 += sqrt(area);
            }
         }
      }
      chord = vs1 > 0.0 ? 4.0 * vs0 / vs1 : 0.0;
      bridged = chord > 0.0;
   }
   for (int64_t c = 0; c < n_cells; c++) {
      if (!is_void[c]) d[c] = 1.0 / (3.0 * sigma_t[c]);
      else if (bridged) d[c] = void_d > 0.0 ? void_d : 1.0 / (3.0 * ((sigma_t[c] > 0.0 ? sigma_t[c] : 0.0) + 1.0 / chord));
      else d[c] = 0.0;
      masked[c] = is_void[c] && !bridged;
   }
   out[0] = bridged;
   out[1] = chord;
   out[2] = (double)n_void;
   const double sa = bridged ? max_sa_all : max_sa_solid;
   return (any_vacuum || n_void > 0 || sa > 0.0) ? 0 : 1;
}

/* The MIP interior-penalty form at DG1 (assemble_dg1, :365-475); penalty C.
 * Returns the number of entries written. */
int64_t oracle_dsa_mip(int nb, int F, int64_t n_cells, const double *face_nA, const int64_t *face_nbr,
                       const int32_t *face_bc, const double *face_distance, const double *volume,
                       const double *face_own, const double *face_up, const double *basis_grad,
                       const double *face_nb_grad, const double *sigma_t, const double *sigma_s, double penalty,
                       const double *d_cell, const uint8_t *is_void, const uint8_t *masked, int bridged,
                       int64_t *ri, int64_t *ci, double *v)
{
   int64_t e = 0;
   for (int64_t c = 0; c < n_cells; c++) {
      const double vol = volume[c];
      if (masked[c]) {
         /* A masked void: V times the identity block, every coupling zero */
         for (int i = 0; i < nb; i++)
            for (int j = 0; j < nb; j++) {
               ri[e] = c * nb + i;
               ci[e] = c * nb + j;
               v[e++] = i == j ? vol : 0.0;
            }
         continue;
      }
      const double d_c = d_cell[c];
      const double sigma_a = sigma_t[c] - sigma_s[c];
      double own[MAXB][MAXB];
      for (int i = 0; i < nb; i++)
         for (int j = 0; j < nb; j++) {
            double gd = 0.0;
            for (int d = 0; d < 3; d++) gd += basis_grad[(c * nb + i) * 3 + d] * basis_grad[(c * nb + j) * 3 + d];
            own[i][j] = vol * (d_c * gd + (i == j ? sigma_a : 0.0));
         }
      for (int k = 0; k < F; k++) {
         const int64_t kf = c * F + k;
         /* A face into a masked void is a vacuum face, as if the mesh stopped there */
         const int has_nb = face_nbr[kf] >= 0;
         const int interior = has_nb && !masked[face_nbr[kf]];
         if (!has_nb && face_bc[kf] != BC_VACUUM) continue;
         double area = 0.0, nrm[3];
         for (int d = 0; d < 3; d++) area += face_nA[3 * kf + d] * face_nA[3 * kf + d];
         area = sqrt(area);
         for (int d = 0; d < 3; d++) nrm[d] = face_nA[3 * kf + d] / area;
         const double scale = vol * area;
         const double *fo = face_own + kf * nb * nb, *fu = face_up + kf * nb * nb;
         double gc[MAXB], gn[MAXB];
         for (int j = 0; j < nb; j++) {
            gc[j] = 0.0;
            gn[j] = 0.0;
            for (int d = 0; d < 3; d++) {
               gc[j] += basis_grad[(c * nb + j) * 3 + d] * nrm[d];
               gn[j] += face_nb_grad[(kf * nb + j) * 3 + d] * nrm[d];
            }
         }
         const double h_c = 2.0 * face_distance[2 * kf];
         if (interior) {
            const int64_t n = face_nbr[kf];
            const double h_n = 2.0 * face_distance[2 * kf + 1];
            /* A face touching a bridged void: both sides take the face's harmonic D */
            double dc_f = d_c, dn_f = d_cell[n];
            if (bridged && (is_void[c] || is_void[n])) {
               dc_f = 2.0 * d_c * d_cell[n] / (d_c + d_cell[n]);
               dn_f = dc_f;
            }
            double kappa = 0.5 * penalty * (dc_f / h_c + dn_f / h_n);
            if (kappa < 0.25) kappa = 0.25;
            for (int i = 0; i < nb; i++) {
               const double m_i = scale * fo[i * nb];
               for (int j = 0; j < nb; j++) {
                  own[i][j] += kappa * scale * fo[i * nb + j] - 0.5 * dc_f * gc[j] * m_i - 0.5 * dc_f * gc[i] * scale * fo[j];
                  ri[e] = c * nb + i;
                  ci[e] = n * nb + j;
                  v[e++] = -kappa * scale * fu[i * nb + j] - 0.5 * dn_f * gn[j] * m_i + 0.5 * dc_f * gc[i] * scale * fu[j];
               }
            }
         } else {
            double kappa = penalty * d_c / h_c;
            if (kappa < 0.25) kappa = 0.25;
            for (int i = 0; i < nb; i++) {
               const double m_i = scale * fo[i * nb];
               for (int j = 0; j < nb; j++)
                  own[i][j] += kappa * scale * fo[i * nb + j] - 0.5 * d_c * gc[j] * m_i - 0.5 * d_c * gc[i] * scale * fo[j];
            }
         }
      }
      for (int i = 0; i < nb; i++)
         for (int j = 0; j < nb; j++) {
            ri[e] = c * nb + i;
            ci[e] = c * nb + j;
            v[e++] = own[i][j];
         }
   }
   return e;
}

/* The half-range current of an isotropic unit flux through a face,
 * sum_{Omega . n > 0} w (Omega . n) / W (HalfRangeCurrent, dsa_operatork.hpp:110-118) */
static double half_range(int A, const double *omega, const double *w, double sum_weights, const double *nA, int64_t k,
                         double area)
{
   double s = 0.0;
   for (int a = 0; a < A; a++) {
      double dot = 0.0;
      for (int d = 0; d < 3; d++) dot += omega[3 * a + d] * nA[3 * k + d];
      dot /= area;
      if (dot > 0.0) s += w[a] * dot;
   }
   return s / sum_weights;
}

static double blend_d(double d, double m, double p)
{
   if (p == 1.0) return d + m;
   return pow(pow(d, p) + pow(m, p), 1.0 / p);
}

/* The DG0 two-point flux with the consistent-D blend (assemble_dg0, :288-348;
 * BlendD, dsa_operatork.hpp:122-126); consistent = 0 switches the blend off. */
int64_t oracle_dsa_dg0(int F, int64_t n_cells, int A, const double *face_nA, const int64_t *face_nbr,
                       const int32_t *face_bc, const double *face_distance, const double *volume,
                       const double *omega, const double *w, double sum_weights, const double *sigma_t,
                       const double *sigma_s, int consistent, double power, const double *d_cell,
                       const uint8_t *masked, int64_t *ri, int64_t *ci, double *v)
{
   int64_t e = 0;
   for (int64_t c = 0; c < n_cells; c++) {
      if (masked[c]) {
         /* A masked void: V on the diagonal, couplings zero */
         ri[e] = c;
         ci[e] = c;
         v[e++] = volume[c];
         continue;
      }
      const double d_c = d_cell[c];
      double diag = volume[c] * (sigma_t[c] - sigma_s[c]);
      for (int k = 0; k < F; k++) {
         const int64_t kf = c * F + k;
         double area = 0.0;
         for (int d = 0; d < 3; d++) area += face_nA[3 * kf + d] * face_nA[3 * kf + d];
         area = sqrt(area);
         const double hr = half_range(A, omega, w, sum_weights, face_nA, kf, area);
         const double d_own = face_distance[2 * kf];
         if (face_nbr[kf] >= 0 && masked[face_nbr[kf]]) {
            /* A face into a masked void: no coupling, the vacuum face's Marshak term */
            const double d_b = consistent ? blend_d(d_c, 2.0 * d_own * hr, power) : d_c;
            diag += area / (2.0 + d_own / d_b);
         } else if (face_nbr[kf] >= 0) {
            const int64_t n = face_nbr[kf];
            const double d_n = d_cell[n];
            double t_f = area / (d_own / d_c + face_distance[2 * kf + 1] / d_n);
            if (consistent) {
               const double len = d_own + face_distance[2 * kf + 1];
               t_f = area / len * blend_d(t_f * len / area, hr * len, power);
            }
            ri[e] = c;
            ci[e] = n;
            v[e++] = -t_f;
            diag += t_f;
         } else if (face_bc[kf] == BC_VACUUM) {
            const double d_b = consistent ? blend_d(d_c, 2.0 * d_own * hr, power) : d_c;
            diag += area / (2.0 + d_own / d_b);
         }
      }
      ri[e] = c;
      ci[e] = c;
      v[e++] = diag;
   }
   return e;
}

/* R: rhs(node) = V_c sum_a w_a x(node, a); P: y(node, a) = u(node) / W
 * (RestrictKernel / ProlongKernel, src/dsak.kokkos.cxx:20-62, no BC rows).
 * A masked void's nodes restrict to zero and its rows prolong to zero;
 * masked may be NULL (no voids). */
void oracle_dsa_restrict(int64_t n_cells, int nb, int A, const double *w, const double *volume, const double *x,
                         const uint8_t *masked, double *rhs)
{
   for (int64_t n = 0; n < n_cells * nb; n++) {
      double s = 0.0;
      for (int a = 0; a < A; a++) s += w[a] * x[n * A + a];
      rhs[n] = (masked && masked[n / nb]) ? 0.0 : s * volume[n / nb];
   }
}

void oracle_dsa_prolong(int64_t n_cells, int nb, int A, double sum_weights, const double *u, const uint8_t *masked,
                        double *y)
{
   for (int64_t n = 0; n < n_cells * nb; n++)
      for (int a = 0; a < A; a++) y[n * A + a] = (masked && masked[n / nb]) ? 0.0 : u[n] / sum_weights;
}
