// The CG-SUPG backend on the device: the context, the matrix-free operator
// with its fused SUPG scatter, the diagonal and point Jacobi, and the
// SUPG-weighted right-hand-side fills.
//
// Reference arithmetic (include/ubolt/unstructured_cg.hpp:27-48, 239-258;
// src/terms_cgk.kokkos.cxx:41-101; src/unstructured_cgk.kokkos.cxx:676-709):
//   row (i, a) = 1/m_i sum_{(e, li) in star(i)} sum_j
//                  [Omega.G_ij + tau Omega Omega : K_ij + sigma_t (M_ij + tau Omega.G_ji)] psi(j, a)
//              + sum_{inflow faces f of i} |Omega . nA_f| / (m_i n_fv) (psi(i, a) - [reflective] psi(i, R_f a))
//              - 1/m_i sum_e sigma_s / W sum_j (M_ij + tau Omega.G_ji) phi(j)
//   tau(e, a) = min(1 / sigma_t, 2 / (zeta sum_j |Omega_a . grad phi_j(x_c)|)).
// The reference assembles the first two lines into a matrix per group and
// applies the scatter matrix-free; here one thread per row gathers all three
// from the element tables, so there is no matrix to refill per group.
// A row's (element, column) coefficients are needed by the A threads of its
// vertex at once: the star records are laid out vertex-major, so those
// threads read the same addresses (one L1 line serves the warp).
#include "cg.h"

#include <algorithm>
#include <cmath>
#include <type_traits>

namespace ubolt {

// Values per (star entry, column): M, G_ij, G_ji, the symmetric K sums; 3D
// padded to an even count
__host__ __device__ constexpr int CgRecordSize(int dim) { return dim == 2 ? 8 : 14; }

template <typename T, int DIM, int NV>
__device__ __forceinline__ T SupgTau(const T *__restrict__ cg, const T (&om)[DIM], T sigma_t, T zeta)
{
   T sum = T(0);
#pragma unroll
   for (int j = 0; j < NV; j++) {
      T s = T(0);
#pragma unroll
      for (int c = 0; c < DIM; c++) s += om[c] * cg[j * DIM + c];
      sum += fabs(s);
   }
   const T thin = T(2) / (zeta * sum);
   return sigma_t > T(0) ? fmin(T(1) / sigma_t, thin) : thin;
}

// Omega Omega : K from the symmetric sums
template <typename T, int DIM>
__device__ __forceinline__ T OmegaKOmega(const T *__restrict__ k, const T (&om)[DIM])
{
   if constexpr (DIM == 2) return om[0] * om[0] * k[0] + om[1] * om[1] * k[1] + om[0] * om[1] * k[2];
   else
      return om[0] * om[0] * k[0] + om[1] * om[1] * k[1] + om[2] * om[2] * k[2] + om[0] * om[1] * k[3] +
             om[0] * om[2] * k[4] + om[1] * om[2] * k[5];
}

template <typename T, int DIM>
__device__ __forceinline__ T DotD(const T (&om)[DIM], const T *__restrict__ v)
{
   T s = T(0);
#pragma unroll
   for (int c = 0; c < DIM; c++) s += om[c] * v[c];
   return s;
}

// The weak boundary faces of vertex i at ordinate a: with `x`, their terms
// applied to x (the diagonal and the reflective mirror); without, the
// diagonal part alone
template <typename T, int DIM>
__device__ __forceinline__ T BoundaryTerms(const CgDev<T> &d, int64_t i, int a, const T (&om)[DIM],
                                           const T *__restrict__ x)
{
   T out = T(0);
   const int f1 = d.bf_off[i + 1];
   for (int f = d.bf_off[i]; f < f1; f++) {
      const T *b = d.bf + (int64_t)f * 4;
      const T s = DotD<T, DIM>(om, b);
      if (!(s < T(0))) continue;
      const T c = -s * b[3];
      if (!x) {
         out += c;
         continue;
      }
      out += c * x[i * d.A + a];
      const int side = d.bf_side[f];
      if (d.side_bc[side] == UBOLT_BC_REFLECT) out -= c * x[i * d.A + d.refl[(side >> 1) * d.A + a]];
   }
   return out;
}

// y = (L - S) x (SCATTER) or L x, one thread per row. phi: the scalar flux of x.
template <typename T, int DIM, int NV, bool SCATTER>
__global__ void __launch_bounds__(256) CgApplyKernel(const CgDev<T> d, const T *__restrict__ x,
                                                     const T *__restrict__ phi, T *__restrict__ y)
{
   constexpr int P = CgRecordSize(DIM);
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= d.n_rows) return;
   const int64_t i = r / d.A;
   const int a = (int)(r - i * d.A);
   T om[DIM];
#pragma unroll
   for (int c = 0; c < DIM; c++) om[c] = d.omega[3 * a + c];
   T acc = T(0), sacc = T(0);
   const int s1 = d.star_off[i + 1];
   for (int s = d.star_off[i]; s < s1; s++) {
      const int e = d.star_elem[s];
      const T st = d.sigma_t[e];
      const T tau = d.tau[(int64_t)e * d.A + a];
      const T *rec = d.rec + (int64_t)s * NV * P;
      const int32_t *col = d.cols + (int64_t)s * NV;
      T srow = T(0);
#pragma unroll
      for (int j = 0; j < NV; j++) {
         const T *q = rec + j * P;
         const T w = q[0] + tau * DotD<T, DIM>(om, q + 1 + DIM);
         const T coef = DotD<T, DIM>(om, q + 1) + tau * OmegaKOmega<T, DIM>(q + 1 + 2 * DIM, om) + st * w;
         const int64_t v = col[j];
         acc += coef * x[v * d.A + a];
         if constexpr (SCATTER) srow += w * phi[v];
      }
      if constexpr (SCATTER) sacc += d.sigma_s[e] * srow;
   }
   T out = acc;
   if constexpr (SCATTER) out -= sacc * d.inv_sum_weights;
   y[r] = out * d.inv_m[i] + BoundaryTerms<T, DIM>(d, i, a, om, x);
}

// The diagonal of L (the assembled term's diagonal slot, SUPGTermCG::
// add_diagonal): the star's j = li coefficients and the inflow faces' own
// part. Writes diag, and/or 1 / diag in both precisions; counts zero diagonals.
template <int DIM, int NV>
__global__ void __launch_bounds__(256) CgDiagonalKernel(const CgDev<double> d, double *__restrict__ diag,
                                                        double *__restrict__ inv64, float *__restrict__ inv32,
                                                        unsigned long long *n_zero)
{
   constexpr int P = CgRecordSize(DIM);
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= d.n_rows) return;
   const int64_t i = r / d.A;
   const int a = (int)(r - i * d.A);
   double om[DIM];
#pragma unroll
   for (int c = 0; c < DIM; c++) om[c] = d.omega[3 * a + c];
   double acc = 0.0;
   const int s1 = d.star_off[i + 1];
   for (int s = d.star_off[i]; s < s1; s++) {
      const int e = d.star_elem[s];
      const double st = d.sigma_t[e];
      const double tau = SupgTau<double, DIM, NV>(d.cgrad + (int64_t)e * NV * DIM, om, st, d.zeta);
      const double *q = d.rec + ((int64_t)s * NV + d.star_li[s]) * P;
      const double og = DotD<double, DIM>(om, q + 1);
      acc += og + tau * OmegaKOmega<double, DIM>(q + 1 + 2 * DIM, om) + st * (q[0] + tau * og);
   }
   const double v = acc * d.inv_m[i] + BoundaryTerms<double, DIM>(d, i, a, om, nullptr);
   if (diag) diag[r] = v;
   if (inv64) {
      const double iv = v != 0.0 ? 1.0 / v : 0.0;
      inv64[r] = iv;
      inv32[r] = (float)iv;
   }
   if (n_zero && v == 0.0) atomicAdd(n_zero, 1ull);
}

// b(i, a) += scale / m_i sum_e coeff_e sum_j (M_ij + tau Omega.G_ji) f(j), f = 1 where NULL
// (UnstructuredCG::add_weighted_load's WeightedLoadKernel)
template <int DIM, int NV>
__global__ void __launch_bounds__(256) CgWeightedLoadKernel(const CgDev<double> d, const double *__restrict__ coeff,
                                                            const double *__restrict__ f, double scale,
                                                            double *__restrict__ b)
{
   constexpr int P = CgRecordSize(DIM);
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= d.n_rows) return;
   const int64_t i = r / d.A;
   const int a = (int)(r - i * d.A);
   double om[DIM];
#pragma unroll
   for (int c = 0; c < DIM; c++) om[c] = d.omega[3 * a + c];
   double acc = 0.0;
   const int s1 = d.star_off[i + 1];
   for (int s = d.star_off[i]; s < s1; s++) {
      const int e = d.star_elem[s];
      const double ce = coeff[e];
      if (ce == 0.0) continue;
      const double tau = SupgTau<double, DIM, NV>(d.cgrad + (int64_t)e * NV * DIM, om, d.sigma_t[e], d.zeta);
      const double *rec = d.rec + (int64_t)s * NV * P;
      double srow = 0.0;
#pragma unroll
      for (int j = 0; j < NV; j++) {
         const double *q = rec + j * P;
         const double w = q[0] + tau * DotD<double, DIM>(om, q + 1 + DIM);
         srow += f ? w * f[d.cols[(int64_t)s * NV + j]] : w;
      }
      acc += ce * srow;
   }
   b[r] += scale * d.inv_m[i] * acc;
}

struct SideValues {
   double v[6];
};

// The weak vacuum inflow: b(i, a) += sum over i's inflow faces on a vacuum
// side of |Omega . nA_f| / (m_i n_fv) inflow / W
template <int DIM>
__global__ void __launch_bounds__(256) CgGhostInflowKernel(const CgDev<double> d, SideValues in,
                                                           double *__restrict__ b)
{
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= d.n_rows) return;
   const int64_t i = r / d.A;
   const int a = (int)(r - i * d.A);
   double om[DIM];
#pragma unroll
   for (int c = 0; c < DIM; c++) om[c] = d.omega[3 * a + c];
   double add = 0.0;
   const int f1 = d.bf_off[i + 1];
   for (int f = d.bf_off[i]; f < f1; f++) {
      const int side = d.bf_side[f];
      if (d.side_bc[side] != UBOLT_BC_VACUUM || in.v[side] == 0.0) continue;
      const double *bf = d.bf + (int64_t)f * 4;
      const double s = DotD<double, DIM>(om, bf);
      if (s < 0.0) add += -s * bf[3] * in.v[side] * d.inv_sum_weights;
   }
   if (add != 0.0) b[r] += add;
}

template <typename T>
__global__ void ScaleByKernel(const T *__restrict__ s, const T *__restrict__ x, T *__restrict__ y, int64_t n)
{
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      y[k] = s[k] * x[k];
}

// The kernel families are templated on the dimension and the vertices per
// element; a mesh picks one instantiation at run time
#define UBOLT_CG_DISPATCH(dim_, nv_, ...)                                         \
   do {                                                                          \
      if ((dim_) == 2 && (nv_) == 3) { constexpr int D_ = 2, N_ = 3; __VA_ARGS__; } \
      else if ((dim_) == 2 && (nv_) == 4) { constexpr int D_ = 2, N_ = 4; __VA_ARGS__; } \
      else if ((dim_) == 3 && (nv_) == 4) { constexpr int D_ = 3, N_ = 4; __VA_ARGS__; } \
      else if ((dim_) == 3 && (nv_) == 8) { constexpr int D_ = 3, N_ = 8; __VA_ARGS__; } \
   } while (0)

static int Grid(int64_t n) { return (int)((n + 255) / 256); }

// One precision's view with the current group's cross sections
template <typename T>
static CgDev<T> DevOf(const ubolt_ctx *ctx)
{
   CgDev<T> d;
   if constexpr (std::is_same<T, double>::value) d = ctx->cg->d64;
   else d = ctx->cg->d32;
   d.sigma_t = ctx->geom<T>().sigma_t;
   d.sigma_s = ctx->geom<T>().sigma_s;
   if constexpr (std::is_same<T, double>::value) d.tau = ctx->cg->tau64;
   else d.tau = ctx->cg->tau32;
   return d;
}

// tau[e A + a] of the current group, in FP64 and rounded to FP32
template <int DIM, int NV>
__global__ void __launch_bounds__(256) CgTauKernel(const CgDev<double> d, int64_t n_elements,
                                                   double *__restrict__ tau64, float *__restrict__ tau32)
{
   const int64_t total = n_elements * d.A;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
      const int64_t e = k / d.A;
      const int a = (int)(k - e * d.A);
      double om[DIM];
#pragma unroll
      for (int c = 0; c < DIM; c++) om[c] = d.omega[3 * a + c];
      const double t = SupgTau<double, DIM, NV>(d.cgrad + e * NV * DIM, om, d.sigma_t[e], d.zeta);
      tau64[k] = t;
      tau32[k] = (float)t;
   }
}

// The tau table for the current group (a kernel launch, no allocation)
static int EnsureTau(ubolt_ctx *ctx, cudaStream_t s)
{
   ubolt_cg *cg = ctx->cg;
   if (cg->tau_epoch == ctx->group_epoch) return UBOLT_OK;
   const CgDev<double> d = DevOf<double>(ctx);
   const int64_t total = cg->n_elements * ctx->A;
   const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
   UBOLT_CG_DISPATCH(cg->dim, cg->nv, (CgTauKernel<D_, N_><<<grid, 256, 0, s>>>(d, cg->n_elements, cg->tau64, cg->tau32)));
   const int rc = CheckLaunch("cg tau");
   if (!rc) cg->tau_epoch = ctx->group_epoch;
   return rc;
}

template <typename T>
int CgApply(ubolt_ctx *ctx, const T *x, T *y, bool scatter, void *stream)
{
   ubolt_cg *cg = ctx->cg;
   cudaStream_t s = (cudaStream_t)stream;
   if (int rc = EnsureTau(ctx, s)) return rc;
   const CgDev<T> d = DevOf<T>(ctx);
   T *phi = nullptr;
   if (scatter) {
      int rc = 0;
      if constexpr (std::is_same<T, double>::value) {
         phi = cg->phi64;
         rc = ubolt_scalar_flux(ctx, x, phi, stream);
      } else {
         phi = cg->phi32;
         rc = ubolt_scalar_flux_f32(ctx, x, phi, stream);
      }
      if (rc) return rc;
   }
   UBOLT_CG_DISPATCH(cg->dim, cg->nv, {
      if (scatter) CgApplyKernel<T, D_, N_, true><<<Grid(d.n_rows), 256, 0, s>>>(d, x, phi, y);
      else CgApplyKernel<T, D_, N_, false><<<Grid(d.n_rows), 256, 0, s>>>(d, x, phi, y);
   });
   return CheckLaunch("cg apply");
}
template int CgApply<double>(ubolt_ctx *, const double *, double *, bool, void *);
template int CgApply<float>(ubolt_ctx *, const float *, float *, bool, void *);

int CgDiagonal(ubolt_ctx *ctx, double *diag, void *stream)
{
   const CgDev<double> d = DevOf<double>(ctx);
   UBOLT_CG_DISPATCH(ctx->cg->dim, ctx->cg->nv,
                     (CgDiagonalKernel<D_, N_><<<Grid(d.n_rows), 256, 0, (cudaStream_t)stream>>>(
                        d, diag, nullptr, nullptr, nullptr)));
   return CheckLaunch("cg diagonal");
}

// The inverse diagonal of the current group, launched on `stream` (no wait);
// with n_zero, also counts the zero diagonals there (device counter)
static int JacobiBuild(ubolt_ctx *ctx, unsigned long long *n_zero, cudaStream_t s)
{
   ubolt_cg *cg = ctx->cg;
   const CgDev<double> d = DevOf<double>(ctx);
   UBOLT_CG_DISPATCH(cg->dim, cg->nv,
                     (CgDiagonalKernel<D_, N_><<<Grid(d.n_rows), 256, 0, s>>>(d, nullptr, cg->jinv64, cg->jinv32,
                                                                              n_zero)));
   const int rc = CheckLaunch("cg jacobi");
   if (!rc) cg->jacobi_epoch = ctx->group_epoch;
   return rc;
}

int CgJacobiSetup(ubolt_ctx *ctx, int64_t *n_zero, void *stream)
{
   cudaStream_t s = (cudaStream_t)stream;
   unsigned long long *dz = ctx->d_counters, h = 0;
   cudaMemsetAsync(dz, 0, sizeof *dz, s);
   int rc = JacobiBuild(ctx, dz, s);
   cudaMemcpyAsync(&h, dz, sizeof h, cudaMemcpyDeviceToHost, s);
   if (!rc) rc = CudaCheck(cudaStreamSynchronize(s), "block_setup");
   if (n_zero) *n_zero = (int64_t)h;
   if (rc) return rc;
   if (h) return SetError(UBOLT_ERR_SINGULAR, "%llu of %lld rows have a zero diagonal", h, (long long)ctx->n_rows);
   return UBOLT_OK;
}

template <typename T>
int CgJacobiApply(ubolt_ctx *ctx, const T *x, T *y, void *stream)
{
   ubolt_cg *cg = ctx->cg;
   cudaStream_t s = (cudaStream_t)stream;
   int rc = 0;
   if (cg->jacobi_epoch != ctx->group_epoch && (rc = JacobiBuild(ctx, nullptr, s))) return rc;
   const T *inv;
   if constexpr (std::is_same<T, double>::value) inv = cg->jinv64;
   else inv = cg->jinv32;
   const int64_t n = ctx->n_rows;
   ScaleByKernel<T><<<(int)std::min<int64_t>(Grid(n), 148 * 16), 256, 0, s>>>(inv, x, y, n);
   return CheckLaunch("cg jacobi apply");
}
template int CgJacobiApply<double>(ubolt_ctx *, const double *, double *, void *);
template int CgJacobiApply<float>(ubolt_ctx *, const float *, float *, void *);

int CgAddSource(ubolt_ctx *ctx, const double *q_elem, double *b, void *stream)
{
   const CgDev<double> d = DevOf<double>(ctx);
   UBOLT_CG_DISPATCH(ctx->cg->dim, ctx->cg->nv,
                     (CgWeightedLoadKernel<D_, N_><<<Grid(d.n_rows), 256, 0, (cudaStream_t)stream>>>(
                        d, q_elem, nullptr, 1.0 / ctx->sum_weights, b)));
   return CheckLaunch("cg add_source");
}

int CgAddTransfer(ubolt_ctx *ctx, const double *phi_from, const double *sigma_s_from_to, double *b, void *stream)
{
   const CgDev<double> d = DevOf<double>(ctx);
   UBOLT_CG_DISPATCH(ctx->cg->dim, ctx->cg->nv,
                     (CgWeightedLoadKernel<D_, N_><<<Grid(d.n_rows), 256, 0, (cudaStream_t)stream>>>(
                        d, sigma_s_from_to, phi_from, 1.0 / ctx->sum_weights, b)));
   return CheckLaunch("cg add_transfer");
}

int CgGhostInflow(ubolt_ctx *ctx, const double *side_inflow, double *b, void *stream)
{
   SideValues in{};
   for (int k = 0; k < 2 * ctx->dim; k++) in.v[k] = side_inflow[k];
   const CgDev<double> d = DevOf<double>(ctx);
   if (ctx->dim == 2)
      CgGhostInflowKernel<2><<<Grid(d.n_rows), 256, 0, (cudaStream_t)stream>>>(d, in, b);
   else
      CgGhostInflowKernel<3><<<Grid(d.n_rows), 256, 0, (cudaStream_t)stream>>>(d, in, b);
   return CheckLaunch("cg add_ghost_inflow");
}

template <typename T>
static int UploadVec(ubolt_ctx *ctx, const std::vector<T> &h, const T **d)
{
   void *p = nullptr;
   int rc = CtxAlloc(ctx, h.size() * sizeof(T), &p);
   if (rc) return rc;
   if (!h.empty() && (rc = CudaCheck(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload")))
      return rc;
   *d = static_cast<const T *>(p);
   return UBOLT_OK;
}

template <typename T>
static std::vector<T> Narrow(const std::vector<double> &v)
{
   return std::vector<T>(v.begin(), v.end());
}

}  // namespace ubolt

using namespace ubolt;

void UboltCgFree(ubolt_ctx *ctx)
{
   delete ctx->cg;
   ctx->cg = nullptr;
}

extern "C" int ubolt_ctx_is_cg(const ubolt_ctx *ctx) { return ctx && ctx->cg ? 1 : 0; }

extern "C" int ubolt_ctx_create_cg(const ubolt_cg_geometry *geom, const ubolt_quadrature *quad, double zeta,
                                   ubolt_ctx **out)
{
   ClearError();
   if (!out || !geom || !quad) return SetError(UBOLT_ERR_ARG, "ubolt_ctx_create_cg: NULL argument");
   *out = nullptr;
   const int dim = geom->dim, nv = geom->n_element_vertices, A = quad->n_angles;
   const int64_t nvx = geom->n_vertices, ne = geom->n_elements, ns = geom->n_star, nbf = geom->n_bfaces;
   if (dim != 2 && dim != 3) return SetError(UBOLT_ERR_ARG, "dimension %d", dim);
   if (quad->dim != dim) return SetError(UBOLT_ERR_ARG, "a %dD quadrature was handed to a %dD mesh", quad->dim, dim);
   if (!((dim == 2 && (nv == 3 || nv == 4)) || (dim == 3 && (nv == 4 || nv == 8))))
      return SetError(UBOLT_ERR_ARG, "%d vertices per element in %dD", nv, dim);
   if (A <= 0 || A > 1024) return SetError(UBOLT_ERR_ARG, "n_angles %d (1..1024)", A);
   if (!(zeta > 0.0)) return SetError(UBOLT_ERR_ARG, "the SUPG zeta must be positive, was given %g", zeta);
   if (nvx <= 0 || ne <= 0 || ns != ne * nv || ns >= ((int64_t)1 << 31) || nbf >= ((int64_t)1 << 31) ||
       nvx * (int64_t)A >= ((int64_t)1 << 40))
      return SetError(UBOLT_ERR_ARG, "CG sizes out of range (%lld vertices, %lld elements, %lld star entries)",
                      (long long)nvx, (long long)ne, (long long)ns);
   if (!geom->elem_vertex || !geom->mass || !geom->grad || !geom->stiff || !geom->centre_grad || !geom->volume ||
       !geom->lumped_mass || !geom->star_offset || !geom->star_elem || !geom->star_li || !geom->bface_offset ||
       !geom->bface_nA || !geom->bface_mass || !geom->bface_side || !geom->bface_bc || !geom->elem_face_neighbour ||
       !geom->elem_face_area || !geom->elem_face_bc)
      return SetError(UBOLT_ERR_ARG, "CG geometry arrays missing");
   if (!quad->omega || !quad->w || !quad->reflect) return SetError(UBOLT_ERR_ARG, "quadrature arrays missing");

   auto ctx = new ubolt_ctx();
   auto fail = [&](int rc) {
      ubolt_ctx_destroy(ctx);
      return rc;
   };
   cudaGetDevice(&ctx->device);
   ctx->dim = dim;
   ctx->nb = 1;
   ctx->F = geom->faces_per_element;
   ctx->A = A;
   ctx->n_cells = ne;
   ctx->n_nodes = nvx;
   ctx->n_rows = nvx * A;
   ctx->sum_weights = quad->sum_weights;
   auto cg = new ubolt_cg();
   ctx->cg = cg;
   cg->dim = dim;
   cg->nv = nv;
   cg->F = geom->faces_per_element;
   cg->P = CgRecordSize(dim);
   cg->n_vertices = nvx;
   cg->n_elements = ne;
   cg->n_star = ns;
   cg->zeta = zeta;

   // ~~~~~ Sides: one family each, from the boundary faces
   for (int k = 0; k < 6; k++) ctx->side_bc[k] = UBOLT_BC_VACUUM;
   for (int64_t f = 0; f < nbf; f++) {
      const int side = geom->bface_side[f];
      if (side < 0 || side >= 2 * dim) return fail(SetError(UBOLT_ERR_ARG, "boundary face on side %d", side));
      ctx->side_bc[side] = geom->bface_bc[f];
      if (geom->bface_bc[f] == UBOLT_BC_REFLECT) ctx->has_reflect = true;
   }

   // ~~~~~ The star records, vertex-major
   const int P = cg->P;
   const size_t n2 = (size_t)nv * nv;
   std::vector<int32_t> star_off(nvx + 1), star_elem(ns), cols(ns * nv);
   std::vector<int8_t> star_li(ns);
   std::vector<double> rec((size_t)ns * nv * P, 0.0);
   for (int64_t v = 0; v <= nvx; v++) star_off[v] = (int32_t)geom->star_offset[v];
   if (geom->star_offset[0] != 0 || geom->star_offset[nvx] != ns || geom->bface_offset[0] != 0 ||
       geom->bface_offset[nvx] != nbf)
      return fail(SetError(UBOLT_ERR_ARG, "the star / boundary-face CSR does not cover its entries"));
   for (int64_t v = 0; v < nvx; v++)
      if (geom->star_offset[v + 1] < geom->star_offset[v] || geom->bface_offset[v + 1] < geom->bface_offset[v])
         return fail(SetError(UBOLT_ERR_ARG, "the star / boundary-face offsets of vertex %lld decrease", (long long)v));
   for (int64_t k = 0; k < ne * nv; k++)
      if (geom->elem_vertex[k] < 0 || geom->elem_vertex[k] >= nvx)
         return fail(SetError(UBOLT_ERR_ARG, "element %lld names vertex %lld", (long long)(k / nv),
                              (long long)geom->elem_vertex[k]));
   for (int64_t v = 0; v < nvx; v++)
      if (!(geom->lumped_mass[v] > 0.0))
         return fail(SetError(UBOLT_ERR_ARG, "vertex %lld has lumped mass %g", (long long)v, geom->lumped_mass[v]));
   for (int64_t s = 0; s < ns; s++) {
      const int64_t e = geom->star_elem[s];
      const int li = geom->star_li[s];
      if (e < 0 || e >= ne || li < 0 || li >= nv) return fail(SetError(UBOLT_ERR_ARG, "bad star entry %lld", (long long)s));
      star_elem[s] = (int32_t)e;
      star_li[s] = (int8_t)li;
      for (int j = 0; j < nv; j++) {
         cols[s * nv + j] = (int32_t)geom->elem_vertex[e * nv + j];
         double *q = &rec[((size_t)s * nv + j) * P];
         const size_t ij = e * n2 + (size_t)li * nv + j, ji = e * n2 + (size_t)j * nv + li;
         q[0] = geom->mass[ij];
         for (int c = 0; c < dim; c++) {
            q[1 + c] = geom->grad[ij * 3 + c];
            q[1 + dim + c] = geom->grad[ji * 3 + c];
         }
         const double *K = &geom->stiff[ij * 9];
         double *k = q + 1 + 2 * dim;
         if (dim == 2) {
            k[0] = K[0];
            k[1] = K[4];
            k[2] = K[1] + K[3];
         } else {
            k[0] = K[0];
            k[1] = K[4];
            k[2] = K[8];
            k[3] = K[1] + K[3];
            k[4] = K[2] + K[6];
            k[5] = K[5] + K[7];
         }
      }
   }
   std::vector<double> cgrad((size_t)ne * nv * dim), inv_m(nvx), bf((size_t)nbf * 4);
   for (int64_t e = 0; e < ne; e++)
      for (int j = 0; j < nv; j++)
         for (int c = 0; c < dim; c++) cgrad[((size_t)e * nv + j) * dim + c] = geom->centre_grad[(e * nv + j) * 3 + c];
   for (int64_t v = 0; v < nvx; v++) inv_m[v] = 1.0 / geom->lumped_mass[v];
   std::vector<int32_t> bf_off(nvx + 1);
   std::vector<int8_t> bf_side(nbf);
   for (int64_t v = 0; v <= nvx; v++) bf_off[v] = (int32_t)geom->bface_offset[v];
   for (int64_t f = 0; f < nbf; f++) {
      for (int c = 0; c < 3; c++) bf[f * 4 + c] = geom->bface_nA[f * 3 + c];
      bf[f * 4 + 3] = geom->bface_mass[f];
      bf_side[f] = (int8_t)geom->bface_side[f];
   }

   // ~~~~~ Upload
   int rc = 0;
   DevGeom<double> &g = ctx->g64;
   DevGeom<float> &h = ctx->g32;
   g.dim = h.dim = dim;
   g.nb = h.nb = 1;
   g.F = h.F = 0;
   g.A = h.A = A;
   g.n_cells = h.n_cells = ne;
   g.sum_weights = quad->sum_weights;
   h.sum_weights = (float)quad->sum_weights;
   g.inv_sum_weights = 1.0 / quad->sum_weights;
   h.inv_sum_weights = (float)(1.0 / quad->sum_weights);
   for (int k = 0; k < 6; k++) g.side_bc[k] = h.side_bc[k] = ctx->side_bc[k];
   if ((rc = UploadOrdinates(ctx, quad))) return fail(rc);
   std::vector<double> lumped(geom->lumped_mass, geom->lumped_mass + nvx);
   if ((rc = UploadVec(ctx, lumped, &ctx->d_volume))) return fail(rc);
   CgDev<double> &d = cg->d64;
   CgDev<float> &d32 = cg->d32;
   d.dim = d32.dim = dim;
   d.nv = d32.nv = nv;
   d.P = d32.P = P;
   d.A = d32.A = A;
   d.n_vertices = d32.n_vertices = nvx;
   d.n_rows = d32.n_rows = ctx->n_rows;
   d.zeta = zeta;
   d32.zeta = (float)zeta;
   d.inv_sum_weights = g.inv_sum_weights;
   d32.inv_sum_weights = h.inv_sum_weights;
   for (int k = 0; k < 6; k++) d.side_bc[k] = d32.side_bc[k] = ctx->side_bc[k];
   d.omega = g.omega;
   d32.omega = h.omega;
   d.refl = d32.refl = g.refl;
   if ((rc = UploadVec(ctx, star_off, &d.star_off)) || (rc = UploadVec(ctx, star_elem, &d.star_elem)) ||
       (rc = UploadVec(ctx, star_li, &d.star_li)) || (rc = UploadVec(ctx, cols, &d.cols)) ||
       (rc = UploadVec(ctx, bf_off, &d.bf_off)) || (rc = UploadVec(ctx, bf_side, &d.bf_side)))
      return fail(rc);
   d32.star_off = d.star_off;
   d32.star_elem = d.star_elem;
   d32.star_li = d.star_li;
   d32.cols = d.cols;
   d32.bf_off = d.bf_off;
   d32.bf_side = d.bf_side;
   if ((rc = UploadVec(ctx, rec, &d.rec)) || (rc = UploadVec(ctx, Narrow<float>(rec), &d32.rec)) ||
       (rc = UploadVec(ctx, cgrad, &d.cgrad)) || (rc = UploadVec(ctx, Narrow<float>(cgrad), &d32.cgrad)) ||
       (rc = UploadVec(ctx, inv_m, &d.inv_m)) || (rc = UploadVec(ctx, Narrow<float>(inv_m), &d32.inv_m)) ||
       (rc = UploadVec(ctx, bf, &d.bf)) || (rc = UploadVec(ctx, Narrow<float>(bf), &d32.bf)))
      return fail(rc);
   void *p = nullptr;
   if ((rc = CtxAlloc(ctx, nvx * sizeof(double), &p))) return fail(rc);
   cg->phi64 = static_cast<double *>(p);
   if ((rc = CtxAlloc(ctx, nvx * sizeof(float), &p))) return fail(rc);
   cg->phi32 = static_cast<float *>(p);
   if ((rc = CtxAlloc(ctx, ctx->n_rows * sizeof(double), &p))) return fail(rc);
   cg->jinv64 = static_cast<double *>(p);
   if ((rc = CtxAlloc(ctx, ctx->n_rows * sizeof(float), &p))) return fail(rc);
   cg->jinv32 = static_cast<float *>(p);
   if ((rc = CtxAlloc(ctx, (size_t)ne * ctx->A * sizeof(double), &p))) return fail(rc);
   cg->tau64 = static_cast<double *>(p);
   if ((rc = CtxAlloc(ctx, (size_t)ne * ctx->A * sizeof(float), &p))) return fail(rc);
   cg->tau32 = static_cast<float *>(p);

   // ~~~~~ Host copies for the DSA
   cg->elem_vertex.assign(geom->elem_vertex, geom->elem_vertex + ne * nv);
   cg->mass.assign(geom->mass, geom->mass + ne * n2);
   cg->stiff.assign(geom->stiff, geom->stiff + ne * n2 * 9);
   cg->centre_grad.assign(geom->centre_grad, geom->centre_grad + ne * nv * 3);
   cg->volume.assign(geom->volume, geom->volume + ne);
   cg->lumped = lumped;
   cg->elem_face_neighbour.assign(geom->elem_face_neighbour, geom->elem_face_neighbour + ne * cg->F);
   cg->elem_face_area.assign(geom->elem_face_area, geom->elem_face_area + ne * cg->F);
   cg->elem_face_bc.assign(geom->elem_face_bc, geom->elem_face_bc + ne * cg->F);
   cg->bface_offset.assign(geom->bface_offset, geom->bface_offset + nvx + 1);
   cg->bface_nA.assign(geom->bface_nA, geom->bface_nA + nbf * 3);
   cg->bface_mass.assign(geom->bface_mass, geom->bface_mass + nbf);
   cg->bface_bc.assign(geom->bface_bc, geom->bface_bc + nbf);
   if ((rc = CudaCheck(cudaDeviceSynchronize(), "ctx_create_cg"))) return fail(rc);
   *out = ctx;
   return UBOLT_OK;
}
