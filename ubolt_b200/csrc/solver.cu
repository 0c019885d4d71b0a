// The solve: right-preconditioned restarted GMRES on the shell operator,
// in a plain FP64 form and a mixed form (FP32 operator, preconditioner and
// Krylov storage inside FP64 iterative refinement).
//
// Restates the reference's KSP set-up (src/transport_solverk.kokkos.cxx:
// 196-318): GMRES with PC_RIGHT, so the stopping test is the true residual
// ||b - A x|| against rtol ||b||, the preconditioner being the streaming
// stage (here the exact sweep, ubolt_sweep), optionally followed by the DSA
// correction formed on the operator's own residual, or the removal block
// stage alone (ubolt_block_apply). Orthogonalisation is classical
// Gram-Schmidt with one reorthogonalisation (PETSc's GMRES default refines),
// as fused multi-vector dot and update kernels that read each basis vector
// once and accumulate in FP64 whatever the storage precision. The Hessenberg
// least-squares problem and its Givens rotations stay on the host.
#include "ctx.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

namespace ubolt {
template <typename T>
int Sweep(ubolt_ctx *ctx, const T *q, T *psi, void *stream);
template <typename T>
int BlockApply(ubolt_ctx *ctx, const T *x, T *y, bool trans, void *stream);
template <typename T>
int DsaCorrect(ubolt_ctx *ctx, const T *r, T *y, T *tmp, void *stream);
bool SweepIsExact(ubolt_ctx *ctx);
template <typename T>
int SweepAffine(ubolt_ctx *ctx, const T *r0, const double *alpha, const double *phi, const double *rho, const T *u,
                T *psi, void *stream, bool ordinate_major, bool inv_volume);
template <typename T>
int Sweep(ubolt_ctx *ctx, const T *q, T *psi, void *stream, bool ordinate_major);
template <typename T>
bool SweepWritesOrdinateMajor(ubolt_ctx *ctx);
}  // namespace ubolt

struct ubolt_solver {
   int restart = 0;
   int64_t n = 0;
   bool mixed = false;
   // FP64 workspace: residual, preconditioned vector, spare
   double *r = nullptr, *z = nullptr, *t = nullptr;
   double *V = nullptr;  // (restart + 1) x n, plain form
   // FP32 workspace, mixed form: basis, preconditioned vector, rhs, spare, correction
   float *V32 = nullptr, *z32 = nullptr, *b32 = nullptr, *t32 = nullptr, *d32 = nullptr;
   // Flexible GMRES (a preconditioner that varies, the DSA's inner PCG): the
   // preconditioned basis, restart x n, FP64 (Z) or FP32 (Z32)
   bool flexible = false;
   double *Z = nullptr;
   float *Z32 = nullptr;
   // Reductions: partial[red_blocks][restart + 2], h[3 * (restart + 2)]
   double *partial = nullptr, *h = nullptr;
   int red_blocks = 0;
   unsigned *md_count = nullptr;  // the multi-dot's finished-block counter, zero between launches
   // The compressed form (sweep preconditioner, exact sweep): node-space
   // basis (restart + 1) x n_nodes, the residual's isotropic part, the basis
   // scalars alpha[restart + 2] and four reduction slots
   int64_t n_nodes = 0;
   double *Phi = nullptr, *rho = nullptr, *alpha = nullptr, *scal = nullptr;
   // The solver's small host <-> device values (dot products, scalars, the
   // update coefficients) pass through mapped page-locked memory, copied by
   // one-block kernels, not the copy engines: a large host copy on another
   // stream (a host-buffer batch) would hold a small copy up for its whole
   // length. First half device -> host, second half host -> device.
   double *mb_h = nullptr, *mb_d = nullptr;
   int mb_half = 0;
   // Host-buffer batches: two device buffers each for b and x, the upload
   // and download streams, and per buffer the events that order them
   double *hb[2] = {nullptr, nullptr}, *hx[2] = {nullptr, nullptr};
   cudaStream_t up = nullptr, down = nullptr;
   cudaEvent_t entry = nullptr, uploaded[2] = {nullptr, nullptr}, solved[2] = {nullptr, nullptr},
               downloaded[2] = {nullptr, nullptr};
};

namespace ubolt {

constexpr int kRedThreads = 256;
constexpr int kChunk = 8;

// One Gram-Schmidt pass's scalars of the compressed basis, formed by the
// multi-dot's last block once every dot is in (see IsoCombine below)
struct IsoCombineArgs {
   double *alpha = nullptr;
   int j1 = 0, first = 0, on = 0;
   double rp2 = 0.0, kappa = 0.0;
};

// h[i] = alpha[i] alpha_w |r_perp|^2 + kappa d[i] for i < j1 (in place over
// d), then alpha[j1] = alpha_w - sum_i h[i] alpha[i]: one Gram-Schmidt
// pass's scalars. alpha_w is alpha[j1], or on the first pass alpha[j1 - 1]
// (the new vector w = v_j - ... starts with v_j's scalar). One thread.
__device__ __forceinline__ void IsoCombine(double *__restrict__ d, const IsoCombineArgs &c)
{
   double *alpha = c.alpha;
   const int j1 = c.j1;
   const double aw = c.first ? alpha[j1 - 1] : alpha[j1];
   double upd = 0.0;
   for (int i = 0; i < j1; i++) {
      const double h = alpha[i] * aw * c.rp2 + c.kappa * d[i];
      d[i] = h;
      upd += h * alpha[i];
   }
   alpha[j1] = aw - upd;
}

// The new Arnoldi vector's norm from its two parts, hn = sqrt(alpha_w^2
// |r_perp|^2 + kappa |phi_w|^2); where it is positive and finite, alpha[j1]
// = alpha_w / hn and inv[0] = 1 / hn, else inv[0] = 1 (the vector is left as
// it is; the host sees the same hn and stops). The host forms the same hn
// from the same values for the Hessenberg column.
__global__ void IsoNormalizeKernel(const double *__restrict__ phi2, double *__restrict__ alpha, int j1, double rp2,
                                   double kappa, double *__restrict__ inv)
{
   if (threadIdx.x != 0 || blockIdx.x != 0) return;
   const double aw = alpha[j1];
   // Rounded step by step (no fused multiply-add), as the host's expression is
   const double hn = sqrt(__dadd_rn(__dmul_rn(__dmul_rn(aw, aw), rp2), __dmul_rn(kappa, phi2[0])));
   if (hn > 0.0 && isfinite(hn)) {
      alpha[j1] = aw / hn;
      inv[0] = 1.0 / hn;
   } else {
      inv[0] = 1.0;
   }
}

// x *= s[0], s on the device
__global__ void ScaleByDeviceKernel(double *__restrict__ x, const double *__restrict__ sp, int64_t n)
{
   const double sc = sp[0];
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      x[k] = sc * x[k];
}

// h[i0 + i] = V_{i0+i} . w for i < nc: each block's share to
// partial[blk][i0 + i], then the last block to finish (an integer counter,
// reset by that block) adds the shares in a fixed order, one warp per value:
// per-lane strided sums, then a shuffle tree, the same every run. No block
// waits on another. With cmb.on (the last chunk of a compressed-basis pass)
// that block then forms the pass's scalars from all of h.
template <typename S>
__global__ void __launch_bounds__(kRedThreads) MultiDotKernel(const S *__restrict__ V, int64_t n, int i0, int nc,
                                                              const S *__restrict__ w, double *__restrict__ partial,
                                                              int stride, double *__restrict__ h,
                                                              unsigned *__restrict__ count, IsoCombineArgs cmb)
{
   double acc[kChunk];
#pragma unroll
   for (int i = 0; i < kChunk; i++) acc[i] = 0.0;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
      const double wk = (double)w[k];
#pragma unroll
      for (int i = 0; i < kChunk; i++)
         if (i < nc) acc[i] += (double)V[(int64_t)(i0 + i) * n + k] * wk;
   }
   __shared__ double red[kChunk][kRedThreads / 32];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
   for (int i = 0; i < kChunk; i++) {
      double v = acc[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[i][warp] = v;
   }
   __syncthreads();
   if (threadIdx.x < nc) {
      double s = 0.0;
      for (int k = 0; k < kRedThreads / 32; k++) s += red[threadIdx.x][k];
      partial[(int64_t)blockIdx.x * stride + i0 + threadIdx.x] = s;
      __threadfence();
   }
   __shared__ bool last;
   __syncthreads();
   if (threadIdx.x == 0) last = atomicAdd(count, 1u) == gridDim.x - 1;
   __syncthreads();
   if (!last) return;
   __threadfence();
   if (warp < nc) {
      double s = 0.0;
      for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(&partial[(int64_t)b * stride + i0 + warp]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) h[i0 + warp] = s;
   }
   if (threadIdx.x == 0) *count = 0;
   if (cmb.on) {
      __syncthreads();
      if (threadIdx.x == 0) IsoCombine(h, cmb);
   }
}

// out[i] = sum over blocks of partial[blk][i]
__global__ void ReducePartialKernel(const double *__restrict__ partial, int n_blocks, int stride,
                                    double *__restrict__ out)
{
   const int i = blockIdx.x;
   double s = 0.0;
   for (int b = threadIdx.x; b < n_blocks; b += blockDim.x) s += partial[(int64_t)b * stride + i];
   __shared__ double red[32];
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
   if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
   __syncthreads();
   if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < (int)(blockDim.x + 31) / 32; k++) t += red[k];
      out[i] = t;
   }
}

// w = sign * w + sum_i c[i] V_i, c on the device (sign 1: update, 0: assign)
template <typename S>
__global__ void MultiAxpyKernel(const S *__restrict__ V, int64_t n, int nv, const double *__restrict__ c,
                                double scale_c, S *__restrict__ w, int keep_w)
{
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
      double s = keep_w ? (double)w[k] : 0.0;
      for (int i = 0; i < nv; i++) s += scale_c * c[i] * (double)V[(int64_t)i * n + k];
      w[k] = (S)s;
   }
}

// y = alpha * x (in place allowed), any precision pair
template <typename A, typename B>
__global__ void ScaleKernel(const A *__restrict__ x, B *__restrict__ y, double alpha, int64_t n)
{
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      y[k] = (B)(alpha * (double)x[k]);
}

// y += alpha * x
template <typename A, typename B>
__global__ void AxpyKernel(const A *__restrict__ x, B *__restrict__ y, double alpha, int64_t n)
{
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      y[k] = (B)((double)y[k] + alpha * (double)x[k]);
}

// r = b - r
template <typename S>
__global__ void ResidualKernel(const S *__restrict__ b, S *__restrict__ r, int64_t n)
{
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      r[k] = b[k] - r[k];
}

static int GridFor(int64_t n)
{
   int dev = 0, sms = 148;
   cudaGetDevice(&dev);
   cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
   const int64_t want = (n + 255) / 256;
   return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 8));
}

// h[0..nv) = V^T w, computed on the device
template <typename S>
static void MultiDot(const ubolt_solver *ws, const S *V, int nv, const S *w, int64_t n, double *h, cudaStream_t s,
                     IsoCombineArgs cmb = IsoCombineArgs())
{
   const int stride = ws->restart + 2;
   // Four elements per thread: a short (node-space) vector still spreads
   // over a few hundred blocks, and the partials to reduce stay few
   const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(ws->red_blocks, n / (4 * kRedThreads)));
   for (int i0 = 0; i0 < nv; i0 += kChunk) {
      IsoCombineArgs c = cmb;
      c.on = cmb.on && i0 + kChunk >= nv;  // after the last chunk's dots
      MultiDotKernel<S><<<blocks, kRedThreads, 0, s>>>(V, n, i0, std::min(kChunk, nv - i0), w, ws->partial, stride,
                                                       h, ws->md_count, c);
   }
   CountLaunch((nv + kChunk - 1) / kChunk);
}

// y = x on the SMs: a device-to-device cudaMemcpy may go to a copy engine,
// where a large host copy on another stream would hold it up
template <typename T>
__global__ void CopyKernel(const T *__restrict__ x, T *__restrict__ y, int64_t n)
{
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      y[k] = x[k];
}

template <typename T>
static int DeviceCopy(T *y, const T *x, int64_t n, cudaStream_t s, const char *what)
{
   CopyKernel<T><<<GridFor(n), 256, 0, s>>>(x, y, n);
   CountLaunch();
   return CudaCheck(cudaGetLastError(), what);
}

__global__ void MailCopyKernel(const double *__restrict__ src, double *__restrict__ dst, int n)
{
   for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Mailbox offsets (doubles) in each half
constexpr int kMbScalars = 0, kMbH1 = 8;

// n device values to the mailbox at off; read ws->mb_h[off ...] after the stream syncs
static void ToHost(const ubolt_solver *ws, const double *dev, int off, int n, cudaStream_t s)
{
   MailCopyKernel<<<1, 64, 0, s>>>(dev, ws->mb_d + off, n);
   CountLaunch();
}

// Up to three runs of device values to the mailbox in one launch
struct MailRuns {
   const double *src[3];
   int off[3], n[3];
};

__global__ void MailGatherKernel(MailRuns r, double *__restrict__ box)
{
#pragma unroll
   for (int k = 0; k < 3; k++)
      for (int i = threadIdx.x; i < r.n[k]; i += blockDim.x) box[r.off[k] + i] = r.src[k][i];
}

static void ToHost3(const ubolt_solver *ws, const MailRuns &r, cudaStream_t s)
{
   MailGatherKernel<<<1, 64, 0, s>>>(r, ws->mb_d);
   CountLaunch();
}

// n host values to the device through the mailbox at off (the previous
// value at that offset has been consumed: the solver syncs in between)
static void ToDevice(const ubolt_solver *ws, const double *host, double *dev, int off, int n, cudaStream_t s)
{
   double *box = ws->mb_h + ws->mb_half + off;
   for (int i = 0; i < n; i++) box[i] = host[i];
   MailCopyKernel<<<1, 64, 0, s>>>(ws->mb_d + ws->mb_half + off, dev, n);
   CountLaunch();
}

template <typename S>
static double Norm(const ubolt_solver *ws, const S *x, int64_t n, cudaStream_t s, int *rc)
{
   double *slot = ws->h + 3 * (ws->restart + 2) - 1;
   MultiDot<S>(ws, x, 1, x, n, slot, s);
   ToHost(ws, slot, kMbScalars, 1, s);
   *rc = CudaCheck(cudaStreamSynchronize(s), "norm");
   return std::sqrt(ws->mb_h[kMbScalars]);
}

// y(c, i, a) = x(c, i, opp(a)) / V_c: P V^{-1} (P the swap of each ordinate
// with its opposite, V the cell volume). A node-run kernel.
template <typename S>
__global__ void __launch_bounds__(256) OppositeScaleKernel(const S *__restrict__ x, S *__restrict__ y,
                                                           const int32_t *__restrict__ opp,
                                                           const double *__restrict__ volume, int nb, int A,
                                                           int64_t n_nodes)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      if (node >= n_nodes) continue;
      const double iv = 1.0 / volume[node / nb];
      const S *xr = x + node * A;
      S *yr = y + node * A;
      for (int a = sub; a < A; a += kLpn) yr[a] = (S)((double)xr[opp[a]] * iv);
   }
}

// y = V P y in place: each pair (a, opp(a)) swapped and scaled by V_c by the
// lane that owns its lower index (the opposite is an involution). A node-run kernel.
template <typename S>
__global__ void __launch_bounds__(256) OppositeScaleInPlaceKernel(S *__restrict__ y, const int32_t *__restrict__ opp,
                                                                  const double *__restrict__ volume, int nb, int A,
                                                                  int64_t n_nodes)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      if (node >= n_nodes) continue;
      const double v = volume[node / nb];
      S *yr = y + node * A;
      for (int a = sub; a < A; a += kLpn) {
         const int b = opp[a];
         if (b < a) continue;
         const double ya = (double)yr[a], yb = (double)yr[b];
         yr[a] = (S)(yb * v);
         if (b != a) yr[b] = (S)(ya * v);
      }
   }
}

// The same on psi ordinate-major (y[a n_nodes + node]): each ordinate's run
// swapped with its opposite's and scaled by the cell volume, one thread per
// (pair, node), coalesced along the nodes
template <typename S>
__global__ void __launch_bounds__(256) OppositeScaleInPlaceOmKernel(S *__restrict__ y, const int32_t *__restrict__ opp,
                                                                    const double *__restrict__ volume, int nb, int A,
                                                                    int64_t n_nodes)
{
   const int64_t total = (int64_t)A * n_nodes;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
      const int a = (int)(k / n_nodes);
      const int b = opp[a];
      if (b < a) continue;
      const int64_t node = k - (int64_t)a * n_nodes;
      const double v = volume[node / nb];
      S *ya = y + (int64_t)a * n_nodes + node, *yb = y + (int64_t)b * n_nodes + node;
      const double va = (double)*ya, vb = (double)*yb;
      *ya = (S)(vb * v);
      if (b != a) *yb = (S)(va * v);
   }
}

// The system GMRES iterates on: A = L - S, or its transpose for the adjoint
template <typename T>
int OperatorApply(ubolt_ctx *ctx, bool adjoint, const T *x, T *y, void *stream);
template <>
int OperatorApply<double>(ubolt_ctx *ctx, bool adjoint, const double *x, double *y, void *stream)
{
   return adjoint ? ubolt_apply_adjoint(ctx, x, y, stream) : ubolt_apply(ctx, x, y, stream);
}
template <>
int OperatorApply<float>(ubolt_ctx *ctx, bool adjoint, const float *x, float *y, void *stream)
{
   return adjoint ? ubolt_apply_adjoint_f32(ctx, x, y, stream) : ubolt_apply_f32(ctx, x, y, stream);
}

// y = M^{-1} x. tmp is scratch of n values. For the adjoint system the
// transposed preconditioner: the transposed blocks, or the sweep of the
// reversed ordinates, L^{-T} = V P L^{-1} P V^{-1} - from (V L)^T = P (V L) P
// (docs/architecture.md:284-304 of the reference; P swaps each ordinate with
// its opposite, V is the cell volume per row).
template <typename T>
static int Precondition(ubolt_ctx *ctx, int pc, bool adjoint, const T *x, T *y, T *tmp, int64_t n, void *stream)
{
   cudaStream_t s = (cudaStream_t)stream;
   if (adjoint && (pc == UBOLT_PC_SWEEP || pc == UBOLT_PC_SWEEP_DSA)) {
      const int grid = RunGrid(ctx->n_nodes);
      OppositeScaleKernel<T><<<grid, 256, 0, s>>>(x, tmp, ctx->d_opp, ctx->d_volume, ctx->nb, ctx->A, ctx->n_nodes);
      CountLaunch();
      int rc = Sweep<T>(ctx, tmp, y, stream);
      if (rc) return rc;
      OppositeScaleInPlaceKernel<T><<<grid, 256, 0, s>>>(y, ctx->d_opp, ctx->d_volume, ctx->nb, ctx->A, ctx->n_nodes);
      return CheckLaunch("adjoint pc");
   }
   switch (pc) {
   case UBOLT_PC_NONE:
      return DeviceCopy<T>(y, x, n, s, "pc copy");
   case UBOLT_PC_BLOCK: return BlockApply<T>(ctx, x, y, adjoint, stream);
   case UBOLT_PC_SWEEP: return Sweep<T>(ctx, x, y, stream);
   case UBOLT_PC_SWEEP_DSA: {
      int rc = Sweep<T>(ctx, x, y, stream);
      if (rc) return rc;
      return DsaCorrect<T>(ctx, x, y, tmp, stream);
   }
   case UBOLT_PC_BLOCK_DSA: {
      if (adjoint) return SetError(UBOLT_ERR_ARG, "the DSA stage has no transpose here");
      int rc = BlockApply<T>(ctx, x, y, false, stream);
      if (rc) return rc;
      return DsaCorrect<T>(ctx, x, y, tmp, stream);
   }
   default: return SetError(UBOLT_ERR_ARG, "unknown preconditioner %d", pc);
   }
}

struct GmresResult {
   int iterations = 0;
   double estimate = 1.0;  // last residual estimate / ||b||
   bool converged = false;
};

// Right-preconditioned GMRES(m) for A x = b in storage precision S from the
// guess in x (x_zero: it is zero). V: (m + 1) n basis, z, t: n each.
template <typename S>
static int Gmres(ubolt_ctx *ctx, const ubolt_solver *ws, S *V, S *Zb, S *z, S *t, const S *b, S *x, double bnorm,
                 double rtol, int max_it, int pc, bool adjoint, bool x_zero, GmresResult *out, void *stream)
{
   cudaStream_t s = (cudaStream_t)stream;
   const int64_t n = ws->n;
   const int m = ws->restart;
   const int grid = GridFor(n);
   std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), y(m), h1(m + 1), h2(m + 2);
   double *dh1 = ws->h, *dh2 = ws->h + (m + 2), *dy = ws->h + 2 * (m + 2);
   int rc = 0;
   out->iterations = 0;
   out->converged = false;
   while (out->iterations < max_it) {
      if (x_zero) {
         rc = DeviceCopy<S>(V, b, n, s, "gmres");
         x_zero = false;
      } else {
         rc = OperatorApply<S>(ctx, adjoint, x, V, stream);
         ResidualKernel<S><<<grid, 256, 0, s>>>(b, V, n);
         CountLaunch();
      }
      if (rc) return rc;
      const double beta = Norm<S>(ws, V, n, s, &rc);
      if (rc) return rc;
      if (!std::isfinite(beta)) return SetError(UBOLT_ERR_NONFINITE, "GMRES residual is not finite");
      out->estimate = bnorm > 0 ? beta / bnorm : 0.0;
      if (beta <= rtol * bnorm || beta == 0.0) {
         out->converged = true;
         break;
      }
      ScaleKernel<S, S><<<grid, 256, 0, s>>>(V, V, 1.0 / beta, n);
      CountLaunch();
      std::fill(g.begin(), g.end(), 0.0);
      g[0] = beta;
      int j = 0;
      for (; j < m && out->iterations < max_it; j++) {
         S *vj = V + (int64_t)j * n, *vn = V + (int64_t)(j + 1) * n;
         S *zj = Zb ? Zb + (int64_t)j * n : z;
         if ((rc = Precondition<S>(ctx, pc, adjoint, vj, zj, t, n, stream))) return rc;
         if ((rc = OperatorApply<S>(ctx, adjoint, zj, vn, stream))) return rc;
         MultiDot<S>(ws, V, j + 1, vn, n, dh1, s);
         MultiAxpyKernel<S><<<grid, 256, 0, s>>>(V, n, j + 1, dh1, -1.0, vn, 1);
         CountLaunch();
         MultiDot<S>(ws, V, j + 1, vn, n, dh2, s);
         MultiAxpyKernel<S><<<grid, 256, 0, s>>>(V, n, j + 1, dh2, -1.0, vn, 1);
         CountLaunch();
         MultiDot<S>(ws, vn, 1, vn, n, dh2 + j + 1, s);
         ToHost3(ws, MailRuns{{dh1, dh2, dh2}, {kMbH1, kMbH1 + (m + 2), 0}, {j + 1, j + 2, 0}}, s);
         if ((rc = CudaCheck(cudaStreamSynchronize(s), "gmres"))) return rc;
         std::copy(ws->mb_h + kMbH1, ws->mb_h + kMbH1 + j + 1, h1.begin());
         std::copy(ws->mb_h + kMbH1 + (m + 2), ws->mb_h + kMbH1 + (m + 2) + j + 2, h2.begin());
         out->iterations++;
         const double hn = std::sqrt(h2[j + 1]);
         if (!std::isfinite(hn)) return SetError(UBOLT_ERR_NONFINITE, "GMRES Arnoldi vector is not finite");
         for (int i = 0; i <= j; i++) H[i * m + j] = h1[i] + h2[i];
         if (hn > 0.0) {
            ScaleKernel<S, S><<<grid, 256, 0, s>>>(vn, vn, 1.0 / hn, n);
            CountLaunch();
         }
         for (int i = 0; i < j; i++) {
            const double tt = cs[i] * H[i * m + j] + sn[i] * H[(i + 1) * m + j];
            H[(i + 1) * m + j] = -sn[i] * H[i * m + j] + cs[i] * H[(i + 1) * m + j];
            H[i * m + j] = tt;
         }
         const double d = std::hypot(H[j * m + j], hn);
         if (d == 0.0) return SetError(UBOLT_ERR_BREAKDOWN, "GMRES breakdown at iteration %d", out->iterations);
         cs[j] = H[j * m + j] / d;
         sn[j] = hn / d;
         H[j * m + j] = d;
         g[j + 1] = -sn[j] * g[j];
         g[j] = cs[j] * g[j];
         out->estimate = bnorm > 0 ? std::fabs(g[j + 1]) / bnorm : 0.0;
         if (std::fabs(g[j + 1]) <= rtol * bnorm || hn == 0.0) {
            j++;
            out->converged = true;
            break;
         }
      }
      // x += M^{-1} (V y)
      for (int i = j - 1; i >= 0; i--) {
         double tt = g[i];
         for (int k = i + 1; k < j; k++) tt -= H[i * m + k] * y[k];
         y[i] = tt / H[i * m + i];
      }
      ToDevice(ws, y.data(), dy, kMbH1, j, s);
      if (Zb) {
         // Flexible: x += Z y, the preconditioned vectors kept
         MultiAxpyKernel<S><<<grid, 256, 0, s>>>(Zb, n, j, dy, 1.0, x, 1);
         CountLaunch();
      } else {
         // V_m is free scratch here: the next cycle rebuilds the basis
         S *u = V + (int64_t)m * n;
         MultiAxpyKernel<S><<<grid, 256, 0, s>>>(V, n, j, dy, 1.0, u, 0);
         CountLaunch();
         if ((rc = Precondition<S>(ctx, pc, adjoint, u, z, t, n, stream))) return rc;
         AxpyKernel<S, S><<<grid, 256, 0, s>>>(z, x, 1.0, n);
         CountLaunch();
      }
      if (out->converged) break;
   }
   return CheckLaunch("gmres");
}

// ~~~ GMRES on the sweep-preconditioned system in compressed form
//
// With the exact sweep as M^{-1} = L^{-1}: A M^{-1} = (L - S) L^{-1} =
// I - S L^{-1}, and S maps every vector into Iso_u = {u_a phi(node)} - u = 1
// for L - S (S psi = sigma_s / W sum_b w_b psi(node, b), alike for every
// ordinate), u = w for its transpose. Split the cycle's starting residual
// r0 = E_u rho + r_perp, rho = R_u r0 / kappa (R_u r = sum_a u_a r(., a),
// kappa = sum_a u_a^2), so r_perp is orthogonal to Iso_u. Every Arnoldi vector
// is then v = alpha r_perp + E_u phi, with
//    <v_i, v_j> = alpha_i alpha_j |r_perp|^2 + kappa <phi_i, phi_j>,
//    A M^{-1} v = v - E_u m(M^{-1} v),  m = the scattering moment,
// so the basis is n_nodes-long phi plus one scalar each, the Arnoldi step
// needs no operator apply, and Gram-Schmidt runs on n_nodes-long vectors.
// In exact arithmetic these are the plain form's iterates. Used only where
// the sweep inverts L exactly (no lagged coupling: no reflective side, no
// cycle break); the true residual of every cycle is still b - A x.

template <typename T>
__device__ __forceinline__ T WarpSumSolver(T v)
{
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

// The node kernels below are node-run kernels (kLpn lanes per node).

// rho(node) = R_u r0 (node) / kappa, and this block's share of |r0 - E_u rho|^2
template <typename S>
__global__ void __launch_bounds__(256) IsoSplitKernel(const S *__restrict__ r0, const S *__restrict__ u, int A,
                                                      int64_t n_nodes, double inv_kappa, double *__restrict__ rho,
                                                      double *__restrict__ partial)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   double acc = 0.0;
   for (int64_t nb0 = warp * 4; nb0 < n_nodes; nb0 += n_warps * 4) {
      const int64_t node = nb0 + (lane >> 3);
      const bool live = node < n_nodes;
      const S *rn = r0 + node * A;
      double sum = 0.0;
      if (live)
         for (int a = sub; a < A; a += kLpn) sum += (u ? (double)u[a] : 1.0) * (double)rn[a];
      const double rh = GroupSum(sum) * inv_kappa;
      if (live) {
         if (sub == 0) rho[node] = rh;
         for (int a = sub; a < A; a += kLpn) {
            const double d = (double)rn[a] - (u ? (double)u[a] : 1.0) * rh;
            acc += d * d;
         }
      }
   }
   __shared__ double red[8];
   acc = WarpSumSolver(acc);
   if (lane == 0) red[threadIdx.x >> 5] = acc;
   __syncthreads();
   if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
      partial[blockIdx.x] = t;
   }
}

// t(node, a) = alpha r0(node, a) + u_a (phi(node) - alpha rho(node)) = alpha r_perp + E_u phi
template <typename S>
__global__ void __launch_bounds__(256) IsoExpandKernel(const S *__restrict__ r0, const double *__restrict__ alpha_p,
                                                       const double *__restrict__ phi, const double *__restrict__ rho,
                                                       const S *__restrict__ u, int A, int64_t n_nodes,
                                                       S *__restrict__ t, const int32_t *__restrict__ opp,
                                                       const double *__restrict__ volume, int nb)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   const double al = *alpha_p;
   for (int64_t nb0 = warp * 4; nb0 < n_nodes; nb0 += n_warps * 4) {
      const int64_t node = nb0 + (lane >> 3);
      if (node >= n_nodes) continue;
      // With opp: P V^{-1} of the expansion (u is symmetric under the opposite)
      const double sc = opp ? 1.0 / volume[node / nb] : 1.0;
      if (!r0) {  // r0 isotropic: alpha r_perp = 0
         for (int a = sub; a < A; a += kLpn) t[node * A + a] = (S)((u ? (double)u[a] : 1.0) * phi[node] * sc);
         continue;
      }
      const double iso = phi[node] - al * rho[node];
      for (int a = sub; a < A; a += kLpn) {
         const int ar = opp ? opp[a] : a;
         t[node * A + a] = (S)((al * (double)r0[node * A + ar] + (u ? (double)u[a] : 1.0) * iso) * sc);
      }
   }
}

// phi_out(node) = phi_in(node) - sigma_s(c) / W (R_w z)(node) for L - S, or
// - sigma_s(c) / W (R_1 z)(node) for the transpose: v - S z in Iso_u terms
template <typename S>
__global__ void __launch_bounds__(256) IsoScatterKernel(const S *__restrict__ z, const S *__restrict__ w,
                                                        const S *__restrict__ sigma_s, double inv_W, int nb, int A,
                                                        int64_t n_nodes, const double *__restrict__ phi_in,
                                                        double *__restrict__ phi_out)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t nb0 = warp * 4; nb0 < n_nodes; nb0 += n_warps * 4) {
      const int64_t node = nb0 + (lane >> 3);
      const bool live = node < n_nodes;
      double sum = 0.0;
      if (live)
         for (int a = sub; a < A; a += kLpn) sum += (w ? (double)w[a] : 1.0) * (double)z[node * A + a];
      sum = GroupSum(sum);
      if (live && sub == 0) phi_out[node] = phi_in[node] - (double)sigma_s[node / nb] * inv_W * sum;
   }
}

// The same from z ordinate-major (z[a n_nodes + node]): one thread per node,
// each warp's loads of one ordinate coalesced
template <typename S>
__global__ void __launch_bounds__(256) IsoScatterOmKernel(const S *__restrict__ z, const S *__restrict__ w,
                                                          const S *__restrict__ sigma_s, double inv_W, int nb, int A,
                                                          int64_t n_nodes, const double *__restrict__ phi_in,
                                                          double *__restrict__ phi_out)
{
   for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < n_nodes;
        node += (int64_t)gridDim.x * blockDim.x) {
      double sum = 0.0;
      const S *zn = z + node;
      if (w) {
#pragma unroll 8
         for (int a = 0; a < A; a++) sum += (double)w[a] * (double)zn[(int64_t)a * n_nodes];
      } else {
#pragma unroll 8
         for (int a = 0; a < A; a++) sum += (double)zn[(int64_t)a * n_nodes];
      }
      phi_out[node] = phi_in[node] - (double)sigma_s[node / nb] * inv_W * sum;
   }
}

// x(node, a) += sum_i c[i] Z_i(a, node): the update from ordinate-major
// vectors into UBOLT's row layout, through a 32 x 32 shared-memory tile per
// block so that both the reads (nodes fastest) and the writes (ordinates
// fastest) are coalesced
template <typename S>
__global__ void __launch_bounds__(256) MultiAxpyOmKernel(const S *__restrict__ Z, int64_t n, int nv,
                                                         const double *__restrict__ c, int64_t n_nodes, int A,
                                                         S *__restrict__ x)
{
   __shared__ double tile[32][33];
   const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
   const int64_t node0 = (int64_t)blockIdx.x * 32;
   const int a0 = blockIdx.y * 32;
#pragma unroll
   for (int r = 0; r < 4; r++) {
      const int a = a0 + ty + 8 * r;
      const int64_t node = node0 + tx;
      double v = 0.0;
      if (a < A && node < n_nodes)
         for (int i = 0; i < nv; i++) v += c[i] * (double)Z[(int64_t)i * n + (int64_t)a * n_nodes + node];
      tile[ty + 8 * r][tx] = v;
   }
   __syncthreads();
#pragma unroll
   for (int r = 0; r < 4; r++) {
      const int64_t node = node0 + ty + 8 * r;
      const int a = a0 + tx;
      if (a < A && node < n_nodes) {
         const int64_t k = node * A + a;
         x[k] = (S)((double)x[k] + tile[tx][ty + 8 * r]);
      }
   }
}


// z = M^{-1} (alpha r_perp + E_u phi). The forward sweep forms its input as
// it reads it; the adjoint's reversed-ordinate sweep takes it expanded in t.
template <typename S>
static int IsoPrecondition(ubolt_ctx *ctx, bool adjoint, const S *r0, const double *alpha, const double *phi,
                           const double *rho, const S *u, S *t, S *z, S *tmp, int64_t n, int igrid, void *stream,
                           bool ordinate_major)
{
   if (!adjoint) return SweepAffine<S>(ctx, r0, alpha, phi, rho, u, z, stream, ordinate_major, false);
   // L^{-T} = V P L^{-1} P V^{-1}: the expansion and P V^{-1} in one pass
   // (or, for an isotropic source, in the sweep's own read of it: u = w is
   // symmetric under the opposite, so P V^{-1} E_w phi = E_w (phi / V)), the
   // sweep, then V P in place
   int rc = 0;
   if (!r0 && ordinate_major) {
      rc = SweepAffine<S>(ctx, nullptr, alpha, phi, rho, u, z, stream, true, true);
   } else {
      IsoExpandKernel<S><<<igrid, 256, 0, (cudaStream_t)stream>>>(r0, alpha, phi, rho, u, ctx->A, ctx->n_nodes, t,
                                                                  ctx->d_opp, ctx->d_volume, ctx->nb);
      CountLaunch();
      rc = Sweep<S>(ctx, t, z, stream, ordinate_major);
   }
   if (rc) return rc;
   if (ordinate_major)
      OppositeScaleInPlaceOmKernel<S><<<(int)std::min<int64_t>((ctx->n_nodes * ctx->A + 255) / 256, 148 * 16), 256, 0,
                                        (cudaStream_t)stream>>>(z, ctx->d_opp, ctx->d_volume, ctx->nb, ctx->A,
                                                                ctx->n_nodes);
   else
      OppositeScaleInPlaceKernel<S><<<RunGrid(ctx->n_nodes), 256, 0, (cudaStream_t)stream>>>(z, ctx->d_opp,
                                                                                          ctx->d_volume, ctx->nb,
                                                                                          ctx->A, ctx->n_nodes);
   (void)tmp;
   (void)n;
   return CheckLaunch("adjoint pc");
}

static int IsoGrid(int64_t n_nodes)
{
   return (int)std::max<int64_t>(1, std::min<int64_t>((n_nodes + 31) / 32, 148 * 16));
}

template <typename S>
static int GmresIso(ubolt_ctx *ctx, const ubolt_solver *ws, S *work, const S *b, S *x, double bnorm, double rtol,
                    int max_it, bool adjoint, bool x_zero, GmresResult *out, void *stream)
{
   cudaStream_t s = (cudaStream_t)stream;
   const int64_t n = ws->n, nn = ws->n_nodes;
   const int m = ws->restart, A = ctx->A;
   const int grid = GridFor(n), igrid = IsoGrid(nn);
   const DevGeom<S> &g = ctx->geom<S>();
   const S *u = adjoint ? g.w : nullptr;
   const S *wgt = adjoint ? nullptr : g.w;
   const S *sig_s = g.sigma_s;
   double kappa = 0.0;
   if (adjoint)
      for (double wa : ctx->h_w) kappa += wa * wa;
   else
      kappa = (double)A;
   // Full-length vectors live in the (unused) plain basis: r0, t, tmp, then
   // the preconditioned vectors z_j = M^{-1} v_j of the cycle, kept so the
   // update x += sum_j y_j z_j needs no further sweep. The sweep (forward,
   // or the adjoint's reversed-ordinate one) writes them ordinate-major (each
   // task's psi contiguous, whole sectors written), read back by the scatter
   // and the update, wherever the task kernel runs
   const bool om = SweepWritesOrdinateMajor<S>(ctx);
   S *r0 = work, *t = work + n, *tmp = work + 2 * n, *Zb = work + 3 * n;
   double *Phi = ws->Phi, *alpha = ws->alpha, *scal = ws->scal;
   std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), gv(m + 1), y(m), h1(m + 1), h2(m + 2),
       alpha_h(m + 2, 0.0);
   double *dh1 = ws->h, *dh2 = ws->h + (m + 2), *dy = ws->h + 2 * (m + 2);
   int rc = 0;
   out->iterations = 0;
   out->converged = false;
   while (out->iterations < max_it) {
      // The cycle's residual, read-only from here on: b itself from x = 0
      const S *res = r0;
      if (x_zero) {
         res = b;
         x_zero = false;
      } else {
         rc = OperatorApply<S>(ctx, adjoint, x, r0, stream);
         ResidualKernel<S><<<grid, 256, 0, s>>>(b, r0, n);
         CountLaunch();
      }
      if (rc) return rc;
      // r0 = E_u rho + r_perp; beta^2 = |r_perp|^2 + kappa |rho|^2
      IsoSplitKernel<S><<<igrid, 256, 0, s>>>(res, u, A, nn, 1.0 / kappa, ws->rho, ws->partial);
      ReducePartialKernel<<<1, 256, 0, s>>>(ws->partial, igrid, 1, scal);
      CountLaunch(2);
      MultiDot<double>(ws, ws->rho, 1, ws->rho, nn, scal + 1, s);
      ToHost(ws, scal, kMbScalars, 2, s);
      if ((rc = CudaCheck(cudaStreamSynchronize(s), "gmres"))) return rc;
      const double sc[2] = {ws->mb_h[kMbScalars], ws->mb_h[kMbScalars + 1]};
      // A residual isotropic to rounding (r_perp below 1e-14 of it: the first
      // cycle of an isotropic source) is taken as isotropic: r_perp = 0, and
      // the sweep reads the node vector alone, not r0
      double rp2 = sc[0];
      const bool iso_r0 = rp2 <= 1e-28 * (rp2 + kappa * sc[1]);
      if (iso_r0) rp2 = 0.0;
      const S *r0_in = iso_r0 ? nullptr : res;
      const double beta = std::sqrt(rp2 + kappa * sc[1]);
      if (!std::isfinite(beta)) return SetError(UBOLT_ERR_NONFINITE, "GMRES residual is not finite");
      out->estimate = bnorm > 0 ? beta / bnorm : 0.0;
      if (beta <= rtol * bnorm || beta == 0.0) {
         out->converged = true;
         break;
      }
      // v_0 = r0 / beta: alpha_0 = 1 / beta, phi_0 = rho / beta
      alpha_h[0] = 1.0 / beta;
      ToDevice(ws, alpha_h.data(), alpha, kMbScalars, 1, s);
      ScaleKernel<double, double><<<igrid, 256, 0, s>>>(ws->rho, Phi, 1.0 / beta, nn);
      CountLaunch();
      std::fill(gv.begin(), gv.end(), 0.0);
      gv[0] = beta;
      int j = 0;
      for (; j < m && out->iterations < max_it; j++) {
         double *pj = Phi + (int64_t)j * nn, *pn = Phi + (int64_t)(j + 1) * nn;
         S *z = Zb + (int64_t)j * n;
         // w = v_j - E_u m(M^{-1} v_j): alpha_w = alpha_j, phi_w = phi_j - m
         if ((rc = IsoPrecondition<S>(ctx, adjoint, r0_in, alpha + j, pj, ws->rho, u, t, z, tmp, n, igrid, stream,
                                      om)))
            return rc;
         if (om)
            IsoScatterOmKernel<S><<<(int)std::min<int64_t>((nn + 255) / 256, 148 * 16), 256, 0, s>>>(z, wgt, sig_s, 1.0 / ctx->sum_weights, ctx->nb, A, nn,
                                                              pj, pn);
         else
            IsoScatterKernel<S><<<igrid, 256, 0, s>>>(z, wgt, sig_s, 1.0 / ctx->sum_weights, ctx->nb, A, nn, pj, pn);
         CountLaunch();
         // Classical Gram-Schmidt, twice, in the compressed inner product
         for (int pass = 0; pass < 2; pass++) {
            double *dh = pass ? dh2 : dh1;
            IsoCombineArgs cmb;
            cmb.alpha = alpha;
            cmb.j1 = j + 1;
            cmb.first = pass == 0;
            cmb.on = 1;
            cmb.rp2 = rp2;
            cmb.kappa = kappa;
            MultiDot<double>(ws, Phi, j + 1, pn, nn, dh, s, cmb);
            MultiAxpyKernel<double><<<igrid, 256, 0, s>>>(Phi, nn, j + 1, dh, -1.0, pn, 1);
            CountLaunch();
         }
         MultiDot<double>(ws, pn, 1, pn, nn, dh2 + j + 1, s);
         ToHost3(ws, MailRuns{{dh1, dh2, alpha + j + 1}, {kMbH1, kMbH1 + (m + 2), kMbScalars}, {j + 1, j + 2, 1}}, s);
         // The new vector normalised on the device, behind the mailbox
         // copy, so that the next sweep waits on nothing the host sends
         IsoNormalizeKernel<<<1, 32, 0, s>>>(dh2 + j + 1, alpha, j + 1, rp2, kappa, scal + 3);
         ScaleByDeviceKernel<<<igrid, 256, 0, s>>>(pn, scal + 3, nn);
         CountLaunch(2);
         if ((rc = CudaCheck(cudaStreamSynchronize(s), "gmres"))) return rc;
         std::copy(ws->mb_h + kMbH1, ws->mb_h + kMbH1 + j + 1, h1.begin());
         std::copy(ws->mb_h + kMbH1 + (m + 2), ws->mb_h + kMbH1 + (m + 2) + j + 2, h2.begin());
         alpha_h[j + 1] = ws->mb_h[kMbScalars];
         out->iterations++;
         const double aw = alpha_h[j + 1];
         const double hn = std::sqrt(aw * aw * rp2 + kappa * h2[j + 1]);
         if (!std::isfinite(hn)) return SetError(UBOLT_ERR_NONFINITE, "GMRES Arnoldi vector is not finite");
         for (int i = 0; i <= j; i++) H[i * m + j] = h1[i] + h2[i];
         if (hn > 0.0) alpha_h[j + 1] = aw / hn;  // as the device has it
         for (int i = 0; i < j; i++) {
            const double tt = cs[i] * H[i * m + j] + sn[i] * H[(i + 1) * m + j];
            H[(i + 1) * m + j] = -sn[i] * H[i * m + j] + cs[i] * H[(i + 1) * m + j];
            H[i * m + j] = tt;
         }
         const double d = std::hypot(H[j * m + j], hn);
         if (d == 0.0) return SetError(UBOLT_ERR_BREAKDOWN, "GMRES breakdown at iteration %d", out->iterations);
         cs[j] = H[j * m + j] / d;
         sn[j] = hn / d;
         H[j * m + j] = d;
         gv[j + 1] = -sn[j] * gv[j];
         gv[j] = cs[j] * gv[j];
         out->estimate = bnorm > 0 ? std::fabs(gv[j + 1]) / bnorm : 0.0;
         if (std::fabs(gv[j + 1]) <= rtol * bnorm || hn == 0.0) {
            j++;
            out->converged = true;
            break;
         }
      }
      // x += sum_i y_i z_i = M^{-1} (sum_i y_i v_i)
      for (int i = j - 1; i >= 0; i--) {
         double tt = gv[i];
         for (int k = i + 1; k < j; k++) tt -= H[i * m + k] * y[k];
         y[i] = tt / H[i * m + i];
      }
      ToDevice(ws, y.data(), dy, kMbH1, j, s);
      if (om)
         MultiAxpyOmKernel<S><<<dim3((unsigned)((nn + 31) / 32), (unsigned)((A + 31) / 32)), 256, 0, s>>>(Zb, n, j, dy,
                                                                                                         nn, A, x);
      else
         MultiAxpyKernel<S><<<grid, 256, 0, s>>>(Zb, n, j, dy, 1.0, x, 1);
      CountLaunch();
      if (out->converged) break;
   }
   return CheckLaunch("gmres");
}

static void FreeWorkspace(ubolt_ctx *ctx)
{
   ubolt_solver *ws = ctx->solver;
   if (!ws) return;
   cudaDeviceSynchronize();
   for (void *p : {(void *)ws->r, (void *)ws->z, (void *)ws->t, (void *)ws->V, (void *)ws->V32, (void *)ws->z32,
                   (void *)ws->b32, (void *)ws->t32, (void *)ws->d32, (void *)ws->Z, (void *)ws->Z32,
                   (void *)ws->partial, (void *)ws->h, (void *)ws->Phi, (void *)ws->rho,
                   (void *)ws->alpha, (void *)ws->scal, (void *)ws->hb[0], (void *)ws->hb[1], (void *)ws->hx[0],
                   (void *)ws->hx[1], (void *)ws->md_count})
      if (p) cudaFree(p);
   if (ws->mb_h) cudaFreeHost(ws->mb_h);
   for (cudaStream_t st : {ws->up, ws->down})
      if (st) cudaStreamDestroy(st);
   for (cudaEvent_t ev : {ws->entry, ws->uploaded[0], ws->uploaded[1], ws->solved[0], ws->solved[1],
                          ws->downloaded[0], ws->downloaded[1]})
      if (ev) cudaEventDestroy(ev);
   delete ws;
   ctx->solver = nullptr;
}

static int EnsureWorkspace(ubolt_ctx *ctx, const ubolt_solve_options *o)
{
   const bool mixed = o->precision == UBOLT_PRECISION_MIXED;
   // A DSA stage whose inner solve is PCG is not a fixed linear map: flexible GMRES
   const bool flexible = o->pc == UBOLT_PC_SWEEP_DSA || o->pc == UBOLT_PC_BLOCK_DSA;
   const int m = o->restart > 0 ? o->restart : 30;
   ubolt_solver *ws = ctx->solver;
   if (ws && ws->restart == m && ws->mixed == mixed && ws->flexible == flexible) return UBOLT_OK;
   // Workspace is re-made only when its shape changes
   FreeWorkspace(ctx);
   ws = new ubolt_solver();
   ws->restart = m;
   ws->n = ctx->n_rows;
   ws->mixed = mixed;
   ws->flexible = flexible;
   ws->red_blocks = std::min(GridFor(ws->n), 1184);
   const int64_t n = ws->n;
   auto alloc = [&](void **p, size_t bytes) -> int {
      const cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
      if (e != cudaSuccess) {
         cudaGetLastError();
         *p = nullptr;
         return SetError(UBOLT_ERR_NOMEM, "solver workspace: cudaMalloc of %zu bytes: %s", bytes,
                         cudaGetErrorString(e));
      }
      return UBOLT_OK;
   };
   int rc = 0;
   ctx->solver = ws;
   if ((rc = alloc((void **)&ws->r, n * 8)) || (rc = alloc((void **)&ws->z, n * 8)) ||
       (rc = alloc((void **)&ws->t, n * 8)) || (rc = alloc((void **)&ws->partial, (size_t)ws->red_blocks * (m + 2) * 8)) ||
       (rc = alloc((void **)&ws->h, 3 * (size_t)(m + 2) * 8)))
      return rc;
   if ((rc = alloc((void **)&ws->md_count, 16))) return rc;
   if ((rc = CudaCheck(cudaMemset(ws->md_count, 0, 16), "solver workspace"))) return rc;
   ws->mb_half = 16 + 3 * (m + 2);
   if (cudaHostAlloc((void **)&ws->mb_h, 2 * (size_t)ws->mb_half * 8, cudaHostAllocMapped) != cudaSuccess ||
       cudaHostGetDevicePointer((void **)&ws->mb_d, ws->mb_h, 0) != cudaSuccess) {
      cudaGetLastError();
      return SetError(UBOLT_ERR_NOMEM, "solver workspace: mapped host memory");
   }
   ws->n_nodes = ctx->n_nodes;
   if (!flexible && ((rc = alloc((void **)&ws->Phi, (size_t)(m + 1) * ws->n_nodes * 8)) ||
                     (rc = alloc((void **)&ws->rho, ws->n_nodes * 8)) ||
                     (rc = alloc((void **)&ws->alpha, (size_t)(m + 2) * 8)) || (rc = alloc((void **)&ws->scal, 4 * 8))))
      return rc;
   // The plain basis holds m + 1 vectors; the compressed form keeps r0, two
   // scratch vectors and the cycle's m preconditioned vectors in the same space
   const size_t nv = flexible ? (size_t)(m + 1) : (size_t)(m + 3);
   if (!mixed) {
      if ((rc = alloc((void **)&ws->V, nv * n * 8))) return rc;
      if (flexible && (rc = alloc((void **)&ws->Z, (size_t)m * n * 8))) return rc;
   } else {
      if ((rc = alloc((void **)&ws->V32, nv * n * 4)) || (rc = alloc((void **)&ws->z32, n * 4)) ||
          (rc = alloc((void **)&ws->b32, n * 4)) || (rc = alloc((void **)&ws->t32, n * 4)) ||
          (rc = alloc((void **)&ws->d32, n * 4)))
         return rc;
      if (flexible && (rc = alloc((void **)&ws->Z32, (size_t)m * n * 4))) return rc;
   }
   return UBOLT_OK;
}

}  // namespace ubolt

using namespace ubolt;

void UboltSolverFree(ubolt_ctx *ctx) { FreeWorkspace(ctx); }

extern "C" void ubolt_solve_defaults(ubolt_solve_options *o)
{
   if (!o) return;
   o->rtol = 1e-8;
   o->max_it = 500;
   o->restart = 30;
   o->precision = UBOLT_PRECISION_FP64;
   o->pc = UBOLT_PC_SWEEP;
   o->inner_rtol = 1e-5;
   o->max_outer = 10;
   o->x_zero = 1;
   o->krylov = UBOLT_KRYLOV_AUTO;
   o->pad_ = 0;
}

extern "C" int ubolt_solver_setup(ubolt_ctx *ctx, const ubolt_solve_options *opts)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   ubolt_solve_options o;
   ubolt_solve_defaults(&o);
   if (opts) o = *opts;
   if (o.restart < 1 || o.restart > 200) return SetError(UBOLT_ERR_ARG, "restart %d (1..200)", o.restart);
   if (o.pc < UBOLT_PC_NONE || o.pc > UBOLT_PC_BLOCK_DSA) return SetError(UBOLT_ERR_ARG, "preconditioner %d", o.pc);
   if ((rc = EnsureWorkspace(ctx, &o))) return rc;
   if ((o.pc == UBOLT_PC_SWEEP || o.pc == UBOLT_PC_SWEEP_DSA) && !ctx->sweep) return ubolt_sweep_setup(ctx, 0);
   return UBOLT_OK;
}

static int SolveSystem(ubolt_ctx *ctx, bool adjoint, const double *b, double *x, const ubolt_solve_options *opts,
                       ubolt_solve_stats *stats, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!b || !x || (const void *)b == (const void *)x) return SetError(UBOLT_ERR_ARG, "solve: b and x must be distinct");
   ubolt_solve_options o;
   ubolt_solve_defaults(&o);
   if (opts) o = *opts;
   if (!(o.rtol > 0.0) || o.max_it < 1) return SetError(UBOLT_ERR_ARG, "solve: rtol must be > 0 and max_it >= 1");
   if ((rc = ubolt_solver_setup(ctx, &o))) return rc;
   ubolt_solver *ws = ctx->solver;
   cudaStream_t s = (cudaStream_t)stream;
   const int64_t n = ws->n;
   const int grid = GridFor(n);
   const auto t0 = std::chrono::steady_clock::now();
   // The multi-dot's finished-block counter starts every solve at zero,
   // whatever an earlier launch that failed part-way left in it
   if ((rc = CudaCheck(cudaMemsetAsync(ws->md_count, 0, sizeof(unsigned), s), "solve"))) return rc;
   // The compressed form wherever its identity holds: the exact sweep alone
   // as preconditioner, and room for its four full-length vectors
   const bool iso = o.pc == UBOLT_PC_SWEEP && ws->Phi && SweepIsExact(ctx) &&
                    o.krylov == UBOLT_KRYLOV_AUTO;
   if (o.x_zero) cudaMemsetAsync(x, 0, n * sizeof(double), s);
   const double bnorm = Norm<double>(ws, b, n, s, &rc);
   if (rc) return rc;
   if (!std::isfinite(bnorm)) return SetError(UBOLT_ERR_NONFINITE, "the right-hand side is not finite");

   ubolt_solve_stats st{};
   st.krylov = iso ? UBOLT_KRYLOV_COMPRESSED : UBOLT_KRYLOV_FULL;
   bool converged = false;
   bool r_of_x = false;  // ws->r holds b - A x of the x to be returned, st.residual its norm
   if (bnorm == 0.0) {
      cudaMemsetAsync(x, 0, n * sizeof(double), s);
      converged = true;
   } else if (o.precision == UBOLT_PRECISION_FP64) {
      GmresResult res;
      if (iso)
         rc = GmresIso<double>(ctx, ws, ws->V, b, x, bnorm, o.rtol, o.max_it, adjoint, o.x_zero != 0, &res, stream);
      else
         rc = Gmres<double>(ctx, ws, ws->V, ws->Z, ws->z, ws->t, b, x, bnorm, o.rtol, o.max_it, o.pc, adjoint,
                            o.x_zero != 0, &res, stream);
      if (rc) return rc;
      st.iterations = res.iterations;
      st.outer = 1;
      converged = res.converged;
   } else {
      // Iterative refinement: r = b - A x in FP64, A d = r in FP32, x += d.
      // From x = 0 the first residual is b itself, its norm already known
      bool x_zero = o.x_zero != 0;
      for (int outer = 0; outer < o.max_outer; outer++) {
         const double *resid = ws->r;
         double rnorm = bnorm;
         if (x_zero) {
            resid = b;
         } else {
            if ((rc = OperatorApply<double>(ctx, adjoint, x, ws->r, stream))) return rc;
            ResidualKernel<double><<<grid, 256, 0, s>>>(b, ws->r, n);
            CountLaunch();
            rnorm = Norm<double>(ws, ws->r, n, s, &rc);
            if (rc) return rc;
            r_of_x = true;
         }
         if (!std::isfinite(rnorm)) return SetError(UBOLT_ERR_NONFINITE, "refinement residual is not finite");
         st.residual = rnorm / bnorm;
         if (rnorm <= o.rtol * bnorm) {
            converged = true;
            break;
         }
         r_of_x = false;
         st.outer = outer + 1;
         // The correction equation, scaled to unit norm so FP32 has the range
         ScaleKernel<double, float><<<grid, 256, 0, s>>>(resid, ws->b32, 1.0 / rnorm, n);
         CountLaunch();
         cudaMemsetAsync(ws->d32, 0, n * sizeof(float), s);
         GmresResult res;
         const double inner = std::max(o.inner_rtol, 0.5 * o.rtol * bnorm / rnorm);
         if (iso)
            rc = GmresIso<float>(ctx, ws, ws->V32, ws->b32, ws->d32, 1.0, inner, o.max_it - st.iterations, adjoint,
                                 true, &res, stream);
         else
            rc = Gmres<float>(ctx, ws, ws->V32, ws->Z32, ws->z32, ws->t32, ws->b32, ws->d32, 1.0, inner,
                              o.max_it - st.iterations, o.pc, adjoint, true, &res, stream);
         if (rc) return rc;
         st.iterations += res.iterations;
         AxpyKernel<float, double><<<grid, 256, 0, s>>>(ws->d32, x, rnorm, n);
         CountLaunch();
         x_zero = false;
         if (st.iterations >= o.max_it) break;
      }
   }
   // The true residual of what is returned (the refinement's last residual
   // where that was taken of the x returned)
   if (!r_of_x) {
      if ((rc = OperatorApply<double>(ctx, adjoint, x, ws->r, stream))) return rc;
      ResidualKernel<double><<<grid, 256, 0, s>>>(b, ws->r, n);
      CountLaunch();
      const double rn = Norm<double>(ws, ws->r, n, s, &rc);
      if (rc) return rc;
      st.residual = bnorm > 0 ? rn / bnorm : 0.0;
   }
   st.rnorm0 = bnorm;
   st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
   if (ctx->sweep && (o.pc == UBOLT_PC_SWEEP || o.pc == UBOLT_PC_SWEEP_DSA)) {
      ubolt_sweep_info si;
      if ((rc = ubolt_sweep_status(ctx, &si, stream))) return rc;
   }
   converged = converged && st.residual <= o.rtol * 1.01;
   st.converged = converged ? 1 : 0;
   if (stats) *stats = st;
   if (!converged)
      return SetError(UBOLT_ERR_NOT_CONVERGED, "not converged: true residual %.3e after %d iterations", st.residual,
                      st.iterations);
   return UBOLT_OK;
}

extern "C" int ubolt_solve(ubolt_ctx *ctx, const double *b, double *x, const ubolt_solve_options *opts,
                           ubolt_solve_stats *stats, void *stream)
{
   return SolveSystem(ctx, false, b, x, opts, stats, stream);
}

// The batch's device buffers, streams and events, made once per workspace
static int EnsureHostBatch(ubolt_solver *ws)
{
   if (ws->up) return UBOLT_OK;
   const size_t bytes = (size_t)ws->n * sizeof(double);
   for (double **p : {&ws->hb[0], &ws->hb[1], &ws->hx[0], &ws->hx[1]}) {
      if (cudaMalloc((void **)p, bytes) != cudaSuccess) {
         cudaGetLastError();
         *p = nullptr;
         return SetError(UBOLT_ERR_NOMEM, "host batch: cudaMalloc of %zu bytes", bytes);
      }
   }
   int rc = 0;
   if ((rc = CudaCheck(cudaStreamCreateWithFlags(&ws->up, cudaStreamNonBlocking), "host batch stream")) ||
       (rc = CudaCheck(cudaStreamCreateWithFlags(&ws->down, cudaStreamNonBlocking), "host batch stream")))
      return rc;
   for (cudaEvent_t *ev : {&ws->entry, &ws->uploaded[0], &ws->uploaded[1], &ws->solved[0], &ws->solved[1],
                           &ws->downloaded[0], &ws->downloaded[1]})
      if ((rc = CudaCheck(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "host batch event"))) return rc;
   return UBOLT_OK;
}

extern "C" int ubolt_solve_host_batch(ubolt_ctx *ctx, int n, const double *const *b_host, double *const *x_host,
                                      const ubolt_solve_options *opts, ubolt_solve_stats *stats, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (n < 0 || (n > 0 && (!b_host || !x_host))) return SetError(UBOLT_ERR_ARG, "solve_host_batch: bad arguments");
   if (n == 0) return UBOLT_OK;
   for (int i = 0; i < n; i++)
      if (!b_host[i] || !x_host[i]) return SetError(UBOLT_ERR_ARG, "solve_host_batch: NULL buffer %d", i);
   ubolt_solve_options o;
   ubolt_solve_defaults(&o);
   if (opts) o = *opts;
   o.x_zero = 1;  // the device x buffers hold another solve's x
   if ((rc = ubolt_solver_setup(ctx, &o))) return rc;
   ubolt_solver *ws = ctx->solver;
   if ((rc = EnsureHostBatch(ws))) return rc;
   cudaStream_t s = (cudaStream_t)stream;
   const size_t bytes = (size_t)ws->n * sizeof(double);
   // Upload i + 1 while solve i runs; download i while solve i + 1 runs.
   // Buffer i % 2 holds b and x of solve i.
   cudaEventRecord(ws->entry, s);
   cudaStreamWaitEvent(ws->up, ws->entry, 0);
   cudaMemcpyAsync(ws->hb[0], b_host[0], bytes, cudaMemcpyHostToDevice, ws->up);
   cudaEventRecord(ws->uploaded[0], ws->up);
   for (int i = 0; i < n; i++) {
      const int k = i & 1;
      if (i + 1 < n) {
         const int kn = (i + 1) & 1;
         if (i >= 1) cudaStreamWaitEvent(ws->up, ws->solved[kn], 0);  // solve i - 1 has read it
         cudaMemcpyAsync(ws->hb[kn], b_host[i + 1], bytes, cudaMemcpyHostToDevice, ws->up);
         cudaEventRecord(ws->uploaded[kn], ws->up);
      }
      cudaStreamWaitEvent(s, ws->uploaded[k], 0);
      if (i >= 2) cudaStreamWaitEvent(s, ws->downloaded[k], 0);  // x of solve i - 2 is out
      rc = SolveSystem(ctx, false, ws->hb[k], ws->hx[k], &o, stats ? &stats[i] : nullptr, stream);
      if (rc && rc != UBOLT_ERR_NOT_CONVERGED) break;
      cudaEventRecord(ws->solved[k], s);
      cudaStreamWaitEvent(ws->down, ws->solved[k], 0);
      cudaMemcpyAsync(x_host[i], ws->hx[k], bytes, cudaMemcpyDeviceToHost, ws->down);
      cudaEventRecord(ws->downloaded[k], ws->down);
      if (rc) break;
   }
   // The caller's stream orders after every copy this call issued
   cudaEventRecord(ws->entry, ws->up);
   cudaStreamWaitEvent(s, ws->entry, 0);
   cudaEventRecord(ws->entry, ws->down);
   cudaStreamWaitEvent(s, ws->entry, 0);
   const int rc_copy = CudaCheck(cudaGetLastError(), "solve_host_batch");
   return rc ? rc : rc_copy;
}

extern "C" int ubolt_solve_adjoint(ubolt_ctx *ctx, const double *g, double *lambda, const ubolt_solve_options *opts,
                                   ubolt_solve_stats *stats, void *stream)
{
   return SolveSystem(ctx, true, g, lambda, opts, stats, stream);
}
