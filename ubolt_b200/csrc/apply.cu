// The matrix-free transport operator: y = (L - S) x, y = L x and
// y = (L - S)^T x in one pass over the angular flux.
//
// Reference arithmetic (src/termsk.kokkos.cxx):
//   DG0 row (c, a):  (sum_{s>0} s) / V x(c, a) + sum_{s<0, interior} s / V x(up, a)
//                    + sum_{s<0, reflective} s / V x(c, refl(a))          (:170-240)
//   DG1 row (c,i,a): sum_{s>0} s sum_j face_own(i,j) x(c,j,a)
//                    + sum_{s<0} s sum_j face_up(i,j) x(up|c, j, a|refl(a))
//                    - (Omega . grad phi_i) x(c,0,a)  [i > 0]             (:314-389)
//   removal: + sigma_t(c) x(c,i,a)                                         (:451-539)
//   scatter: - sigma_s(c) / W sum_b w_b x(c,i,b)                           (:584-649)
// Vacuum inflow slots are nulled (their value is rhs), s == 0 adds nothing.
//
// One block holds K whole cells, one thread per (cell, angle); a thread
// computes all n_basis rows of its (cell, angle).
//
// Forward (L - S and L): everything a block needs besides its upwind
// neighbours is staged in shared memory by coalesced cooperative loads
// issued together - the cells' angular flux, their shape data (normals,
// face matrices, gradients), face codes and cross sections - so a block
// waits on two rounds of memory latency (class id -> shape data, face code
// -> neighbour flux) instead of a chain of per-face loads. The upwind
// neighbours' values are loaded into registers before the scatter's
// per-node angular moment (a warp-shuffle reduction over the staged flux)
// is formed, so those loads overlap it. A reflective face reads its
// mirrored angle from the staged flux.
//
// Adjoint ((L - S)^T): a column also needs the NEIGHBOUR's shape data (its
// face slot and matrix for the shared face), so that kernel gathers class
// data straight from L1/L2.
#include "ctx.h"

namespace ubolt {

enum { kFull = 0, kUnscattered = 1, kAdjoint = 2 };

template <typename T>
__device__ __forceinline__ T WarpSum(T v)
{
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

// Two 256-thread blocks per SM at most 64 registers; the FP64 4 x 4 block
// needs more and takes them
template <typename T, int NB, int F>
constexpr int ApplyMinBlocks() { return (sizeof(T) == 8 && NB == 4) ? 1 : 2; }

template <typename T, int NB, int F, bool SCATTER>
__global__ void __launch_bounds__(512, ApplyMinBlocks<T, NB, F>()) ApplyKernel(const DevGeom<T> g, const T *__restrict__ x, T *__restrict__ y, int K)
{
   constexpr RecordLayout L(NB, F, (int)sizeof(T));
   constexpr int U = L.size * (int)sizeof(T) / 16;  // 16-byte units per class record
   extern __shared__ __align__(16) unsigned char smem_raw[];
   const int A = g.A;
   T *geo = reinterpret_cast<T *>(smem_raw);                   // [K][L.size]
   T *xs = geo + K * L.size;                                    // [K][NB][A]
   T *mom = xs + K * NB * A;                                    // [K][NB]
   T *sig = mom + K * NB;                                       // [K][2]: sigma_t, sigma_s / W
   int32_t *codes = reinterpret_cast<int32_t *>(sig + 2 * K);  // [K][F]
   const int t = threadIdx.x;
   const int k = t / A;
   const int a = t - k * A;
   const int64_t c0 = (int64_t)blockIdx.x * K;
   const int kc = (int)min((int64_t)K, g.n_cells - c0);  // cells in this block
   const bool live = k < kc;
   const T *xb = x + c0 * NB * A;  // this block's rows, then 32-bit offsets
   T *yb = y + c0 * NB * A;

   // Round 1: own flux, face codes, cross sections; class ids -> shape data
   if (live) {
#pragma unroll
      for (int j = 0; j < NB; j++) xs[(k * NB + j) * A + a] = xb[(k * NB + j) * A + a];
   }
   for (int e = t; e < kc * F; e += blockDim.x) codes[e] = g.code[c0 * F + e];
   for (int e = t; e < kc; e += blockDim.x) {
      sig[2 * e] = g.sigma_t[c0 + e];
      sig[2 * e + 1] = SCATTER ? g.sigma_s[c0 + e] * g.inv_sum_weights : T(0);
   }
   for (int e = t; e < kc * U; e += blockDim.x) {
      const int kk = e / U;
      const int u = e - kk * U;
      const int64_t cl = g.cls[c0 + kk];
      reinterpret_cast<int4 *>(geo)[kk * U + u] = reinterpret_cast<const int4 *>(g.rec)[cl * U + u];
   }
   __syncthreads();

   // Round 2: the upwind neighbours of this (cell, angle), loaded together
   // and folded in at once (inflow faces: the upwind neighbour, or the
   // mirrored angle here), so they hold no registers past this point
   const T *gs = geo + k * L.size;
   T ox = T(0), oy = T(0), oz = T(0);
   T sf[F];
   T acc[NB];
#pragma unroll
   for (int i = 0; i < NB; i++) acc[i] = T(0);
   if (live) {
      ox = g.omega[3 * a];
      oy = g.omega[3 * a + 1];
      oz = g.omega[3 * a + 2];
#pragma unroll
      for (int f = 0; f < F; f++) sf[f] = Dot3(ox, oy, oz, gs + L.nA + 3 * f);
      // Faces in chunks of FC: every load of a chunk is in flight at once
      constexpr int FC = (F * NB <= 9) ? F : (F % 3 == 0 ? 3 : 2);
#pragma unroll
      for (int f0 = 0; f0 < F; f0 += FC) {
      T xn[FC][NB];
#pragma unroll
      for (int ff = 0; ff < FC; ff++) {
         const int32_t code = codes[k * F + f0 + ff];
         const bool up = sf[f0 + ff] < T(0) && FaceInterior(code);
         const T *xu = x + (size_t)(up ? code : 0) * (NB * A) + a;
#pragma unroll
         for (int j = 0; j < NB; j++) xn[ff][j] = up ? xu[j * A] : T(0);
      }
#pragma unroll
      for (int ff = 0; ff < FC; ff++) {
         const int f = f0 + ff;
         if (!(sf[f] < T(0))) continue;
         const int32_t code = codes[k * F + f];
         if (!FaceInterior(code)) {
            const int side = FaceSide(code);
            if (g.side_bc[side] != UBOLT_BC_REFLECT) continue;
            const int ar = g.refl[(side >> 1) * A + a];
#pragma unroll
            for (int j = 0; j < NB; j++) xn[ff][j] = xs[(k * NB + j) * A + ar];
         }
         if constexpr (NB == 1) {
            acc[0] += sf[f] * gs[L.ivol] * xn[ff][0];
         } else {
            const T *M = gs + L.fup + f * NB * NB;
#pragma unroll
            for (int i = 0; i < NB; i++) {
               T u = T(0);
#pragma unroll
               for (int j = 0; j < NB; j++) u += M[i * NB + j] * xn[ff][j];
               acc[i] += sf[f] * u;
            }
         }
      }
      }
   }
   if constexpr (SCATTER) {
      // Per node: sigma_s / W sum_b w_b x(node, b)
      const int warp = t >> 5, lane = t & 31, n_warps = blockDim.x >> 5;
      for (int n = warp; n < kc * NB; n += n_warps) {
         T s = T(0);
         for (int b = lane; b < A; b += 32) s += g.w[b] * xs[n * A + b];
         s = WarpSum(s);
         if (lane == 0) mom[n] = s * sig[2 * (n / NB) + 1];
      }
      __syncthreads();
   }
   if (!live) return;

   // Own block: outflow faces, volume term, removal
   if constexpr (NB == 1) {
      T out = T(0);
#pragma unroll
      for (int f = 0; f < F; f++)
         if (sf[f] > T(0)) out += sf[f];
      acc[0] += (out * gs[L.ivol] + sig[2 * k]) * xs[k * A + a];
   } else {
      T B[NB][NB];
#pragma unroll
      for (int i = 0; i < NB; i++)
#pragma unroll
         for (int j = 0; j < NB; j++) B[i][j] = T(0);
#pragma unroll
      for (int f = 0; f < F; f++) {
         if (sf[f] > T(0)) {
            const T *M = gs + L.fown + f * NB * NB;
#pragma unroll
            for (int i = 0; i < NB; i++)
#pragma unroll
               for (int j = 0; j < NB; j++) B[i][j] += sf[f] * M[i * NB + j];
         }
      }
#pragma unroll
      for (int i = 1; i < NB; i++) B[i][0] -= Dot3(ox, oy, oz, gs + L.bgrad + 3 * i);
#pragma unroll
      for (int i = 0; i < NB; i++) B[i][i] += sig[2 * k];
      T xo[NB];
#pragma unroll
      for (int j = 0; j < NB; j++) xo[j] = xs[(k * NB + j) * A + a];
#pragma unroll
      for (int i = 0; i < NB; i++) {
         T u = T(0);
#pragma unroll
         for (int j = 0; j < NB; j++) u += B[i][j] * xo[j];
         acc[i] += u;
      }
   }
   if constexpr (SCATTER) {
#pragma unroll
      for (int i = 0; i < NB; i++) acc[i] -= mom[k * NB + i];
   }
#pragma unroll
   for (int i = 0; i < NB; i++) yb[(k * NB + i) * A + a] = acc[i];
}

// Column (c, j, a) of L - S: the own block transposed, the scatter's
// column, and every row that reads this cell as its upwind neighbour
template <typename T, int NB, int F>
__global__ void __launch_bounds__(512) AdjointApplyKernel(const DevGeom<T> g, const T *__restrict__ x, T *__restrict__ y,
                                                          int K)
{
   extern __shared__ __align__(16) unsigned char smem_raw[];
   T *xs = reinterpret_cast<T *>(smem_raw);  // [K][NB][A]
   T *mom = xs + K * NB * g.A;                 // [K][NB]
   const int A = g.A;
   const int t = threadIdx.x;
   const int k = t / A;
   const int a = t - k * A;
   const int64_t c = (int64_t)blockIdx.x * K + k;
   const bool live = (k < K) && (c < g.n_cells);

   T xo[NB];
   if (live) {
#pragma unroll
      for (int j = 0; j < NB; j++) {
         xo[j] = x[(c * NB + j) * A + a];
         xs[(k * NB + j) * A + a] = xo[j];
      }
   }
   __syncthreads();
   {
      // Per node: sigma_s / W sum_b x(node, b)
      const int warp = t >> 5, lane = t & 31, n_warps = blockDim.x >> 5;
      for (int n = warp; n < K * NB; n += n_warps) {
         const int64_t cc = (int64_t)blockIdx.x * K + n / NB;
         T s = T(0);
         if (cc < g.n_cells)
            for (int b = lane; b < A; b += 32) s += xs[n * A + b];
         s = WarpSum(s);
         if (lane == 0 && cc < g.n_cells) mom[n] = s * (g.sigma_s[cc] * g.inv_sum_weights);
      }
      __syncthreads();
   }
   if (!live) return;

   const int32_t cl = g.cls[c];
   const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
   T acc[NB];
   T B[NB][NB];
   BuildBlock<T, NB, F>(g, cl, om, g.sigma_t[c], B);
#pragma unroll
   for (int j = 0; j < NB; j++) {
      T s = T(0);
#pragma unroll
      for (int i = 0; i < NB; i++) s += B[i][j] * xo[i];
      acc[j] = s - g.w[a] * mom[k * NB + j];
   }
#pragma unroll
   for (int f = 0; f < F; f++) {
      const int32_t code = g.code[c * F + f];
      if (FaceInterior(code)) {
         // Row (n, i, a) couples to (c, j, a) through n's slot for this face
         const int64_t n = code;
         const int mf = g.mirror[c * F + f];
         const int32_t ncl = g.cls[n];
         const T s = Dot3(om, g.nA + ((int64_t)ncl * F + mf) * 3);
         if (!(s < T(0))) continue;
         T xn[NB];
#pragma unroll
         for (int i = 0; i < NB; i++) xn[i] = x[(n * NB + i) * A + a];
         if constexpr (NB == 1) {
            acc[0] += s * g.inv_vol[ncl] * xn[0];
         } else {
            const T *M = g.fup + ((int64_t)ncl * F + mf) * NB * NB;
#pragma unroll
            for (int j = 0; j < NB; j++) {
               T u = T(0);
#pragma unroll
               for (int i = 0; i < NB; i++) u += M[i * NB + j] * xn[i];
               acc[j] += s * u;
            }
         }
      } else {
         // Row (c, i, refl(a)) reads (c, j, a) through this reflective face
         const int side = FaceSide(code);
         if (g.side_bc[side] != UBOLT_BC_REFLECT) continue;
         const int ar = g.refl[(side >> 1) * A + a];
         const T orr[3] = {g.omega[3 * ar], g.omega[3 * ar + 1], g.omega[3 * ar + 2]};
         const T s = Dot3(orr, g.nA + ((int64_t)cl * F + f) * 3);
         if (!(s < T(0))) continue;
         T xn[NB];
#pragma unroll
         for (int i = 0; i < NB; i++) xn[i] = xs[(k * NB + i) * A + ar];
         if constexpr (NB == 1) {
            acc[0] += s * g.inv_vol[cl] * xn[0];
         } else {
            const T *M = g.fup + ((int64_t)cl * F + f) * NB * NB;
#pragma unroll
            for (int j = 0; j < NB; j++) {
               T u = T(0);
#pragma unroll
               for (int i = 0; i < NB; i++) u += M[i * NB + j] * xn[i];
               acc[j] += s * u;
            }
         }
      }
   }
#pragma unroll
   for (int i = 0; i < NB; i++) y[(c * NB + i) * A + a] = acc[i];
}

// The streaming + removal diagonal, the block's own diagonal entries
// (DG0OutflowDiagonal / DG1OutflowDiagonal + sigma_t, composed as
// TransportOperator::diagonal does, transport_operatork.kokkos.cxx:240-256).
template <typename T, int NB, int F>
__global__ void DiagonalKernel(const DevGeom<T> g, T *__restrict__ d)
{
   const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (tid >= g.n_cells * g.A) return;
   const int64_t c = tid / g.A;
   const int a = (int)(tid - c * g.A);
   const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
   T B[NB][NB];
   BuildBlock<T, NB, F>(g, g.cls[c], om, g.sigma_t[c], B);
#pragma unroll
   for (int i = 0; i < NB; i++) d[(c * NB + i) * g.A + a] = B[i][i];
}

template <typename T, int NB, int F>
int LaunchApply(const ubolt_ctx *ctx, const DevGeom<T> &g, const T *x, T *y, int mode, cudaStream_t s)
{
   const int K = CellsPerBlock(g.A);
   const int threads = ((K * g.A + 31) / 32) * 32;
   const int64_t blocks = (g.n_cells + K - 1) / K;
   if (mode == kAdjoint) {
      const size_t smem = sizeof(T) * (size_t)(K * NB * g.A + K * NB);
      AdjointApplyKernel<T, NB, F><<<blocks, threads, smem, s>>>(g, x, y, K);
   } else {
      const size_t smem = sizeof(T) * (size_t)K * (RecordLayout(NB, F, (int)sizeof(T)).size + NB * g.A + NB + 2) +
                          sizeof(int32_t) * K * F;
      auto kern = mode == kFull ? ApplyKernel<T, NB, F, true> : ApplyKernel<T, NB, F, false>;
      // Few ordinates mean many cells per block (DG1 hexes at S2: 32 cells, 67 KB)
      if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kern<<<blocks, threads, smem, s>>>(g, x, y, K);
   }
   return CheckLaunch("apply");
}

template <typename T, int NB, int F>
int LaunchDiagonal(const DevGeom<T> &g, T *d, cudaStream_t s)
{
   const int64_t n = g.n_cells * g.A;
   DiagonalKernel<T, NB, F><<<(n + 255) / 256, 256, 0, s>>>(g, d);
   return CheckLaunch("diagonal");
}

template <typename T>
static int Apply(ubolt_ctx *ctx, const T *x, T *y, int mode, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!x || !y || (const void *)x == (const void *)y)
      return SetError(UBOLT_ERR_ARG, "apply: x and y must be distinct device arrays");
   const DevGeom<T> &g = ctx->geom<T>();
   cudaStream_t s = (cudaStream_t)stream;
   UBOLT_DISPATCH(ctx->nb, ctx->F, return (LaunchApply<T, NB_, F_>(ctx, g, x, y, mode, s)));
   return SetError(UBOLT_ERR_STATE, "no kernel for n_basis %d with %d faces", ctx->nb, ctx->F);
}

}  // namespace ubolt

using namespace ubolt;

extern "C" int ubolt_apply(ubolt_ctx *ctx, const double *x, double *y, void *stream)
{
   return Apply<double>(ctx, x, y, kFull, stream);
}
extern "C" int ubolt_apply_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream)
{
   return Apply<float>(ctx, x, y, kFull, stream);
}
extern "C" int ubolt_apply_unscattered(ubolt_ctx *ctx, const double *x, double *y, void *stream)
{
   return Apply<double>(ctx, x, y, kUnscattered, stream);
}
extern "C" int ubolt_apply_unscattered_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream)
{
   return Apply<float>(ctx, x, y, kUnscattered, stream);
}
extern "C" int ubolt_apply_adjoint(ubolt_ctx *ctx, const double *x, double *y, void *stream)
{
   return Apply<double>(ctx, x, y, kAdjoint, stream);
}
extern "C" int ubolt_apply_adjoint_f32(ubolt_ctx *ctx, const float *x, float *y, void *stream)
{
   return Apply<float>(ctx, x, y, kAdjoint, stream);
}

extern "C" int ubolt_diagonal(ubolt_ctx *ctx, double *d, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!d) return SetError(UBOLT_ERR_ARG, "diagonal: d is NULL");
   const DevGeom<double> &g = ctx->geom<double>();
   UBOLT_DISPATCH(ctx->nb, ctx->F, return (LaunchDiagonal<double, NB_, F_>(g, d, (cudaStream_t)stream)));
   return SetError(UBOLT_ERR_STATE, "no kernel for n_basis %d with %d faces", ctx->nb, ctx->F);
}
