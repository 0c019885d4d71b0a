// Element blocks of streaming + removal, never stored: each (cell, angle)
// block is rebuilt from the class geometry and sigma_t and solved in
// registers. ElementBlockInverse (src/block_inversek.kokkos.cxx) stores
// n_cells * A * nb^2 inverted blocks instead - 86 GB at 128^3 hexes, S8, FP64 -
// and reads them on every apply.
#include "cg.h"
#include "ctx.h"

namespace ubolt {

template <typename T, int NB, int F, bool TRANS>
__global__ void BlockApplyKernel(const DevGeom<T> g, const T *__restrict__ x, T *__restrict__ y)
{
   const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (tid >= g.n_cells * g.A) return;
   const int64_t c = tid / g.A;
   const int a = (int)(tid - c * g.A);
   const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
   T B[NB][NB], r[NB];
   BuildBlock<T, NB, F>(g, g.cls[c], om, g.sigma_t[c], B);
   if constexpr (TRANS) Transpose<T, NB>(B);
#pragma unroll
   for (int j = 0; j < NB; j++) r[j] = x[(c * NB + j) * g.A + a];
   // A singular block maps to zero, as its zeroed inverse does in the reference
   if (!SolveBlock<T, NB>(B, r))
#pragma unroll
      for (int j = 0; j < NB; j++) r[j] = T(0);
#pragma unroll
   for (int j = 0; j < NB; j++) y[(c * NB + j) * g.A + a] = r[j];
}

// Singular-block census (ElementBlockInverse::setup's check,
// block_inversek.kokkos.cxx:291-296)
template <typename T, int NB, int F>
__global__ void BlockCountKernel(const DevGeom<T> g, unsigned long long *n_singular)
{
   const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   bool bad = false;
   if (tid < g.n_cells * g.A) {
      const int64_t c = tid / g.A;
      const int a = (int)(tid - c * g.A);
      const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
      T B[NB][NB], r[NB];
      BuildBlock<T, NB, F>(g, g.cls[c], om, g.sigma_t[c], B);
#pragma unroll
      for (int j = 0; j < NB; j++) r[j] = T(1);
      bad = !SolveBlock<T, NB>(B, r);
   }
   const unsigned m = __ballot_sync(0xffffffffu, bad);
   if ((threadIdx.x & 31) == 0 && m) atomicAdd(n_singular, (unsigned long long)__popc(m));
}

// The explicit inverse of every (cell, angle) block (InvertBlocksKernel,
// block_inversek.kokkos.cxx:83-150); a singular block is stored as zero.
template <typename T, int NB, int F>
__global__ void BlockInverseKernel(const DevGeom<T> g, T *__restrict__ inv)
{
   const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= g.n_cells * g.A) return;
   const int64_t c = b / g.A;
   const int a = (int)(b - c * g.A);
   const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
   T m[NB][NB], w[NB][NB];
   BuildBlock<T, NB, F>(g, g.cls[c], om, g.sigma_t[c], m);
   const bool ok = InvertBlock<T, NB>(m, w);
#pragma unroll
   for (int i = 0; i < NB; i++)
#pragma unroll
      for (int j = 0; j < NB; j++) inv[(b * NB + i) * NB + j] = ok ? w[i][j] : T(0);
}

template <typename T, int NB, int F>
static int LaunchBlockApply(const DevGeom<T> &g, const T *x, T *y, bool trans, cudaStream_t s)
{
   const int64_t n = g.n_cells * g.A;
   if (trans) BlockApplyKernel<T, NB, F, true><<<(n + 255) / 256, 256, 0, s>>>(g, x, y);
   else BlockApplyKernel<T, NB, F, false><<<(n + 255) / 256, 256, 0, s>>>(g, x, y);
   return CheckLaunch("block_apply");
}

template <typename T>
int BlockApply(ubolt_ctx *ctx, const T *x, T *y, bool trans, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!x || !y || (const void *)x == (const void *)y)
      return SetError(UBOLT_ERR_ARG, "block apply: x and y must be distinct device arrays");
   if (ctx->cg) {
      if (trans) return RequireDg(ctx, "the transposed block apply");
      return CgJacobiApply<T>(ctx, x, y, stream);
   }
   UBOLT_DISPATCH(ctx->nb, ctx->F,
                  return (LaunchBlockApply<T, NB_, F_>(ctx->geom<T>(), x, y, trans, (cudaStream_t)stream)));
   return SetError(UBOLT_ERR_STATE, "no kernel for this shape");
}

template int BlockApply<double>(ubolt_ctx *, const double *, double *, bool, void *);
template int BlockApply<float>(ubolt_ctx *, const float *, float *, bool, void *);

}  // namespace ubolt

using namespace ubolt;

extern "C" int ubolt_block_apply(ubolt_ctx *ctx, const double *x, double *y, void *stream)
{
   return BlockApply<double>(ctx, x, y, false, stream);
}
extern "C" int ubolt_block_apply_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream)
{
   return BlockApply<float>(ctx, x, y, false, stream);
}
extern "C" int ubolt_block_apply_transpose(ubolt_ctx *ctx, const double *x, double *y, void *stream)
{
   return BlockApply<double>(ctx, x, y, true, stream);
}

extern "C" int ubolt_block_setup(ubolt_ctx *ctx, int64_t *n_singular, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (ctx->cg) return CgJacobiSetup(ctx, n_singular, stream);
   unsigned long long *d = ctx->d_counters, h = 0;
   cudaStream_t s = (cudaStream_t)stream;
   cudaMemsetAsync(d, 0, sizeof *d, s);
   const int64_t n = ctx->n_cells * ctx->A;
   UBOLT_DISPATCH(ctx->nb, ctx->F, (BlockCountKernel<double, NB_, F_><<<(n + 255) / 256, 256, 0, s>>>(ctx->g64, d)));
   rc = CheckLaunch("block_setup");
   cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, s);
   if (!rc) rc = CudaCheck(cudaStreamSynchronize(s), "block_setup");
   if (n_singular) *n_singular = (int64_t)h;
   if (rc) return rc;
   if (h) return SetError(UBOLT_ERR_SINGULAR, "%llu of %lld element blocks are singular", h, (long long)n);
   return UBOLT_OK;
}

extern "C" int ubolt_block_inverse(ubolt_ctx *ctx, double *inv, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!inv) return SetError(UBOLT_ERR_ARG, "block_inverse: NULL output");
   if ((rc = RequireDg(ctx, "block_inverse"))) return rc;
   const int64_t n = ctx->n_cells * ctx->A;
   cudaStream_t s = (cudaStream_t)stream;
   UBOLT_DISPATCH(ctx->nb, ctx->F, (BlockInverseKernel<double, NB_, F_><<<(n + 255) / 256, 256, 0, s>>>(ctx->g64, inv)));
   return CheckLaunch("block_inverse");
}
