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
__global__ void ResponseSourceKernel(const DevGeom<double> g, const double *__restrict__ volume,
                                     const double *__restrict__ d, double *__restrict__ out)
{
   const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (tid >= g.n_cells * g.A) return;
   const int64_t c = tid / g.A;
   const int a = (int)(tid - c * g.A);
   if (d[c] != 0.0) out[c * g.nb * g.A + a] += d[c] * volume[c] * g.w[a];
}

// One warp per cell
__global__ void GradientKernel(const DevGeom<double> g, const double *__restrict__ psi,
                               const double *__restrict__ lam, double *__restrict__ gt, double *__restrict__ gs)
{
   const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int lane = threadIdx.x & 31;
   if (c >= g.n_cells) return;
   const int A = g.A;
   double rt = 0.0, rs = 0.0;
   for (int i = 0; i < g.nb; i++) {
      const int64_t base = (c * g.nb + i) * A;
      double l_sum = 0.0, phi = 0.0;
      for (int a = lane; a < A; a += 32) {
         const double l = lam[base + a], p = psi[base + a];
         rt += l * p;
         l_sum += l;
         phi += g.w[a] * p;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
         l_sum += __shfl_xor_sync(0xffffffffu, l_sum, o);
         phi += __shfl_xor_sync(0xffffffffu, phi, o);
      }
      rs += l_sum * phi;
   }
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) rt += __shfl_xor_sync(0xffffffffu, rt, o);
   if (lane == 0) {
      if (gt) gt[c] = -rt;
      if (gs) gs[c] = rs * g.inv_sum_weights;
   }
}

}  // namespace ubolt

using namespace ubolt;

extern "C" int ubolt_add_response_source(ubolt_ctx *ctx, const double *detector, double *g, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!detector || !g) return SetError(UBOLT_ERR_ARG, "add_response_source: NULL array");
   const int64_t n = ctx->n_cells * ctx->A;
   ResponseSourceKernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(ctx->g64, ctx->d_volume, detector, g);
   return CheckLaunch("add_response_source");
}

extern "C" int ubolt_gradient(ubolt_ctx *ctx, const double *psi, const double *lambda, double *grad_sigma_t,
                              double *grad_sigma_s, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!psi || !lambda || (!grad_sigma_t && !grad_sigma_s)) return SetError(UBOLT_ERR_ARG, "gradient: NULL array");
   const int64_t threads = ctx->n_cells * 32;
   GradientKernel<<<(threads + 255) / 256, 256, 0, (cudaStream_t)stream>>>(ctx->g64, psi, lambda, grad_sigma_t,
                                                                            grad_sigma_s);
   return CheckLaunch("gradient");
}
