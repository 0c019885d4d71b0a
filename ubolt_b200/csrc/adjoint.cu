// Detector response and its gradient with respect to the per-cell cross
// sections. No reference counterpart: UBOLT has no adjoint
// (docs/architecture.md:493-494); the contractions follow from A = L - S with
// removal sigma_t on every row of a cell and S(c,i,a; c,i,b) = sigma_s w_b / W
// (src/termsk.kokkos.cxx:451-539, 584-649): for J = g^T psi, A psi = b,
// A^T lambda = g,
//    dJ/dsigma_t(c) = - sum_{rows of c} lambda psi
//    dJ/dsigma_s(c) = sum_i (sum_a lambda(c,i,a)) (sum_b w_b psi(c,i,b)) / W.
#include "ctx.h"

namespace ubolt {

// g(c, 0, a) += d(c) V_c w_a: the source whose inner product with psi is
// J = sum_c d(c) V_c phi(c, basis 0) - the detector's volume-integrated flux
__global__ void __launch_bounds__(256) ResponseSourceKernel(const DevGeom<double> g, const double *__restrict__ volume,
                                                            const double *__restrict__ d, double *__restrict__ out)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t c0 = warp * 4; c0 < g.n_cells; c0 += n_warps * 4) {
      const int64_t c = c0 + (lane >> 3);
      if (c >= g.n_cells || d[c] == 0.0) continue;
      const double v = d[c] * volume[c];
      double *run = out + c * g.nb * g.A;
      for (int a = sub; a < g.A; a += kLpn) run[a] += v * g.w[a];
   }
}

// A cell-run kernel: 8 lanes per cell (its nb node runs one after another),
// four cells per warp, as the node-run kernels
__global__ void __launch_bounds__(256) GradientKernel(const DevGeom<double> g, const double *__restrict__ psi,
                                                      const double *__restrict__ lam, double *__restrict__ gt,
                                                      double *__restrict__ gs)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   const int A = g.A;
   for (int64_t c0 = warp * 4; c0 < g.n_cells; c0 += n_warps * 4) {
      const int64_t c = c0 + (lane >> 3);
      const bool live = c < g.n_cells;
      double rt = 0.0, rs = 0.0;
      for (int i = 0; i < g.nb; i++) {
         double l_sum = 0.0, phi = 0.0;
         if (live) {
            const int64_t base = (c * g.nb + i) * A;
            for (int a = sub; a < A; a += kLpn) {
               const double l = lam[base + a], p = psi[base + a];
               rt += l * p;
               l_sum += l;
               phi += g.w[a] * p;
            }
         }
         rs += GroupSum(l_sum) * GroupSum(phi);
      }
      rt = GroupSum(rt);
      if (live && sub == 0) {
         if (gt) gt[c] = -rt;
         if (gs) gs[c] = rs * g.inv_sum_weights;
      }
   }
}

}  // namespace ubolt

using namespace ubolt;

extern "C" int ubolt_add_response_source(ubolt_ctx *ctx, const double *detector, double *g, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!detector || !g) return SetError(UBOLT_ERR_ARG, "add_response_source: NULL array");
   if ((rc = RequireDg(ctx, "add_response_source"))) return rc;
   ResponseSourceKernel<<<RunGrid(ctx->n_cells), 256, 0, (cudaStream_t)stream>>>(ctx->g64, ctx->d_volume, detector,
                                                                                 g);
   return CheckLaunch("add_response_source");
}

extern "C" int ubolt_gradient(ubolt_ctx *ctx, const double *psi, const double *lambda, double *grad_sigma_t,
                              double *grad_sigma_s, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!psi || !lambda || (!grad_sigma_t && !grad_sigma_s)) return SetError(UBOLT_ERR_ARG, "gradient: NULL array");
   if ((rc = RequireDg(ctx, "the gradient"))) return rc;
   GradientKernel<<<RunGrid(ctx->n_cells), 256, 0, (cudaStream_t)stream>>>(ctx->g64, psi, lambda, grad_sigma_t,
                                                                            grad_sigma_s);
   return CheckLaunch("gradient");
}
