// The angular moment and the right-hand-side fills.
#include "cg.h"
#include "ctx.h"

namespace ubolt {

// phi(node) = sum_a w_a psi(node, a) (UboltAngularIntegral's gemm,
// sn_quadraturek.kokkos.cxx:400-427): a node-run kernel, accumulated in FP64
template <typename T>
__global__ void __launch_bounds__(256) ScalarFluxKernel(const T *__restrict__ psi, const T *__restrict__ w,
                                                        T *__restrict__ phi, int64_t n_nodes, int A)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      const bool live = node < n_nodes;
      double sum = 0.0;
      if (live)
         for (int a = sub; a < A; a += kLpn) sum += (double)w[a] * (double)psi[node * A + a];
      sum = GroupSum(sum);
      if (live && sub == 0) phi[node] = (T)sum;
   }
}

// b(cell, basis 0, a) += q(cell) / W (AddIsotropicKernel, material_speck.kokkos.cxx:164-187):
// a run kernel over each cell's basis-0 run
__global__ void __launch_bounds__(256) AddSourceKernel(const DevGeom<double> g, const double *__restrict__ q,
                                                       double *__restrict__ b)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   const int A = g.A;
   for (int64_t c0 = warp * 4; c0 < g.n_cells; c0 += n_warps * 4) {
      const int64_t c = c0 + (lane >> 3);
      if (c >= g.n_cells) continue;
      const double v = q[c] / g.sum_weights;
      double *run = b + c * g.nb * A;
      for (int a = sub; a < A; a += kLpn) run[a] += v;
   }
}

// b(node, a) += phi(node) (sigma_s(cell) / W) (GroupTransfer::add_transfer,
// multigroupk.kokkos.cxx:329-362: scaled into scratch, then added)
__global__ void __launch_bounds__(256) AddTransferKernel(const DevGeom<double> g, const double *__restrict__ phi,
                                                         const double *__restrict__ sigma_s, double *__restrict__ b)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   const int A = g.A;
   const int64_t n_nodes = g.n_cells * g.nb;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      if (node >= n_nodes) continue;
      const double v = phi[node] * (sigma_s[node / g.nb] / g.sum_weights);
      double *run = b + node * A;
      for (int a = sub; a < A; a += kLpn) run[a] += v;
   }
}

// Ghost-flux vacuum inflow, -(s / V) phi_i(x_f) inflow / W per entering face
// (unstructured_dgk.kokkos.cxx:486-494 and 515-522), added per row
// (FillGhostInflowKernel, discretisationk.kokkos.cxx:173-185)
struct Inflow {
   double v[6];
};
__global__ void GhostInflowKernel(const DevGeom<double> g, const double *__restrict__ volume, Inflow in,
                                  double *__restrict__ b)
{
   const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (tid >= g.n_cells * g.A) return;
   const int64_t c = tid / g.A;
   const int a = (int)(tid - c * g.A);
   const int32_t cl = g.cls[c];
   const double om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
   double add[kMaxNb] = {0, 0, 0, 0};
   bool any = false;
   for (int f = 0; f < g.F; f++) {
      const int32_t code = g.code[c * g.F + f];
      if (FaceInterior(code)) continue;
      const int side = FaceSide(code);
      if (g.side_bc[side] != UBOLT_BC_VACUUM || in.v[side] == 0.0) continue;
      const double s = Dot3(om, g.nA + ((int64_t)cl * g.F + f) * 3);
      if (!(s < 0.0)) continue;
      const double inflow = in.v[side] / g.sum_weights;
      for (int i = 0; i < g.nb; i++) {
         const double phi_i = (g.nb == 1) ? 1.0 : g.fbv[((int64_t)cl * g.F + f) * g.nb + i];
         add[i] += -s / volume[c] * phi_i * inflow;
      }
      any = true;
   }
   if (!any) return;
   for (int i = 0; i < g.nb; i++) b[(c * g.nb + i) * g.A + a] += add[i];
}

// J(node, d) = sum_a w_a Omega_a,d psi(node, a): a node-run kernel
__global__ void __launch_bounds__(256) CurrentKernel(const double *__restrict__ psi, const double *__restrict__ w_omega,
                                                     double *__restrict__ cur, int64_t n_nodes, int A, int dim)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      const bool live = node < n_nodes;
      double s[3] = {0.0, 0.0, 0.0};
      if (live)
         for (int a = sub; a < A; a += kLpn) {
            const double v = psi[node * A + a];
            for (int d = 0; d < dim; d++) s[d] += w_omega[a * dim + d] * v;
         }
      for (int d = 0; d < 3; d++) s[d] = GroupSum(s[d]);
      if (live && sub == 0)
         for (int d = 0; d < dim; d++) cur[node * dim + d] = s[d];
   }
}

// psi(node, a) = phi(node) / W + sum_d p1(a, d) J(node, d): a node-run kernel
__global__ void __launch_bounds__(256) ExpandP1Kernel(const double *__restrict__ phi, const double *__restrict__ cur,
                                                      const double *__restrict__ p1, double inv_w,
                                                      double *__restrict__ psi, int64_t n_nodes, int A, int dim)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      if (node >= n_nodes) continue;
      double j[3] = {0.0, 0.0, 0.0};
      for (int d = 0; d < dim; d++) j[d] = cur[node * dim + d];
      const double base = phi[node] * inv_w;
      for (int a = sub; a < A; a += kLpn) {
         double v = base;
         for (int d = 0; d < dim; d++) v += p1[a * dim + d] * j[d];
         psi[node * A + a] = v;
      }
   }
}

template <typename T>
static int ScalarFlux(ubolt_ctx *ctx, const T *psi, T *phi, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!psi || !phi) return SetError(UBOLT_ERR_ARG, "scalar_flux: NULL array");
   ScalarFluxKernel<T><<<RunGrid(ctx->n_nodes), 256, 0, (cudaStream_t)stream>>>(psi, ctx->geom<T>().w, phi,
                                                                                ctx->n_nodes, ctx->A);
   return CheckLaunch("scalar_flux");
}

template <typename T>
void LaunchScalarFlux(const ubolt_ctx *ctx, const T *psi, T *phi, cudaStream_t s)
{
   ScalarFluxKernel<T><<<RunGrid(ctx->n_nodes), 256, 0, s>>>(psi, ctx->geom<T>().w, phi, ctx->n_nodes, ctx->A);
}
template void LaunchScalarFlux<double>(const ubolt_ctx *, const double *, double *, cudaStream_t);
template void LaunchScalarFlux<float>(const ubolt_ctx *, const float *, float *, cudaStream_t);

}  // namespace ubolt

using namespace ubolt;

extern "C" int ubolt_scalar_flux(ubolt_ctx *ctx, const double *psi, double *phi, void *stream)
{
   return ScalarFlux<double>(ctx, psi, phi, stream);
}
extern "C" int ubolt_scalar_flux_f32(ubolt_ctx *ctx, const float *psi, float *phi, void *stream)
{
   return ScalarFlux<float>(ctx, psi, phi, stream);
}

extern "C" int ubolt_current(ubolt_ctx *ctx, const double *psi, double *current, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!psi || !current) return SetError(UBOLT_ERR_ARG, "current: NULL array");
   CurrentKernel<<<RunGrid(ctx->n_nodes), 256, 0, (cudaStream_t)stream>>>(psi, ctx->d_w_omega, current, ctx->n_nodes,
                                                                          ctx->A, ctx->dim);
   return CheckLaunch("current");
}

extern "C" int ubolt_expand_p1(ubolt_ctx *ctx, const double *phi, const double *current, double *psi, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!phi || !current || !psi) return SetError(UBOLT_ERR_ARG, "expand_p1: NULL array");
   if (!ctx->p1_ok)
      return SetError(UBOLT_ERR_ARG, "expand_p1: the ordinates' weighted directions do not sum to zero, or their "
                                     "second moment is singular");
   ExpandP1Kernel<<<RunGrid(ctx->n_nodes), 256, 0, (cudaStream_t)stream>>>(phi, current, ctx->d_p1,
                                                                           1.0 / ctx->sum_weights, psi, ctx->n_nodes,
                                                                           ctx->A, ctx->dim);
   return CheckLaunch("expand_p1");
}

extern "C" int ubolt_add_source(ubolt_ctx *ctx, const double *q_cell, double *b, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!q_cell || !b) return SetError(UBOLT_ERR_ARG, "add_source: NULL array");
   if (ctx->cg) {
      // SUPG-weighted: tau needs the group's sigma_t
      if ((rc = CheckReady(ctx, true))) return rc;
      return CgAddSource(ctx, q_cell, b, stream);
   }
   AddSourceKernel<<<RunGrid(ctx->n_cells), 256, 0, (cudaStream_t)stream>>>(ctx->g64, q_cell, b);
   return CheckLaunch("add_source");
}

extern "C" int ubolt_add_transfer(ubolt_ctx *ctx, const double *phi_from, const double *sigma_s_from_to, double *b,
                                  void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!phi_from || !sigma_s_from_to || !b) return SetError(UBOLT_ERR_ARG, "add_transfer: NULL array");
   if (ctx->cg) {
      if ((rc = CheckReady(ctx, true))) return rc;
      return CgAddTransfer(ctx, phi_from, sigma_s_from_to, b, stream);
   }
   AddTransferKernel<<<RunGrid(ctx->n_nodes), 256, 0, (cudaStream_t)stream>>>(ctx->g64, phi_from, sigma_s_from_to,
                                                                              b);
   return CheckLaunch("add_transfer");
}

extern "C" int ubolt_add_ghost_inflow(ubolt_ctx *ctx, const double *side_inflow, double *b, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!side_inflow || !b) return SetError(UBOLT_ERR_ARG, "add_ghost_inflow: NULL array");
   Inflow in{};
   bool any = false;
   for (int s = 0; s < 2 * ctx->dim; s++) {
      in.v[s] = side_inflow[s];
      if (in.v[s] != 0.0 && ctx->side_bc[s] == UBOLT_BC_VACUUM) any = true;
   }
   if (!any) return UBOLT_OK;
   if (ctx->cg) return CgGhostInflow(ctx, side_inflow, b, stream);
   const int64_t n = ctx->n_cells * ctx->A;
   GhostInflowKernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(ctx->g64, ctx->d_volume, in, b);
   return CheckLaunch("add_ghost_inflow");
}
