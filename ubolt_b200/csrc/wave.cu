// The wave sweep: psi = L^{-1} q with one block per ordinate.
//
// The sweep of one ordinate is a chain of levels (the wave plan: a cell's
// level is the length of the longest upwind chain ending in it), each level
// a set of cells that depend only on earlier levels. A block walks its
// ordinate's levels in order, one thread per cell of a level and a block
// barrier between levels, so no block ever waits on another: no flags, no
// polling, no sentinel fill of psi.
//
// Per level a thread solves its cell:
//   psi_c = W_c r_c - sum_s G_{c,s} psi(up_s),
// with W = B^{-1} (the cell-ordinate's streaming + removal block inverted)
// and G_s = W s_f face_up_f for each gathered upwind face, both from the
// factor store, which holds them level by level per ordinate, element-major
// within a level (consecutive threads read consecutive words). The block
// streams its ordinate's chunks through a ring in shared memory with bulk
// copies (cp.async.bulk, one per level, issued by thread 0 as far ahead as
// the ring holds, each completing on its own mbarrier). The upwind values
// come from the front: a cell read by a later level leaves its psi in a
// shared-memory slot the plan assigned. Each thread prefetches, eight and
// four levels ahead, its cell's plan record and its input values into
// registers, so a level's critical path is the ring read, a few dependent
// FMAs and the barrier.
//
// Every wait (on a level's copy) is bounded: on giving up the block records
// a timeout in the sweep's error words, stops walking, waits (bounded again)
// for the copies it issued and returns - the result is then invalid and the
// host reads UBOLT_ERR_TIMEOUT from ubolt_sweep_status.
#include "wave.h"

#include <algorithm>

namespace ubolt {

namespace {

__device__ __forceinline__ uint32_t SmemAddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void MbarInit(uint64_t *bar, uint32_t count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void MbarInitFence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void MbarExpectTx(uint64_t *bar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes) : "memory");
}

// One contiguous global -> shared copy completing on `bar` (both addresses
// 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void BulkLoad(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    SmemAddr(dst)),
                "l"(src), "r"(bytes), "r"(SmemAddr(bar))
                : "memory");
}

__device__ __forceinline__ bool MbarTryWait(uint64_t *bar, uint32_t parity)
{
   uint32_t ok;
   asm volatile(
       "{\n\t.reg .pred p;\n\t"
       "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
       "selp.u32 %0, 1, 0, p;\n\t}"
       : "=r"(ok)
       : "r"(SmemAddr(bar)), "r"(parity)
       : "memory");
   return ok != 0;
}

// At most limit + 1 polls of the phase
__device__ __forceinline__ bool MbarWaitBounded(uint64_t *bar, uint32_t parity, uint32_t limit)
{
   for (uint32_t k = 0; k <= limit; k++)
      if (MbarTryWait(bar, parity)) return true;
   return false;
}

// One level's factor chunk: W, then the S couplings, element-major
template <typename T>
__host__ __device__ __forceinline__ uint32_t ChunkBytes(int width, int R)
{
   return (uint32_t)(((int64_t)width * R * (int64_t)sizeof(T) + 15) / 16 * 16);
}

// The factor store in wave order: one warp per level, a lane per position
template <typename T, int NB, int F>
__global__ void __launch_bounds__(128) WaveFactorKernel(const DevGeom<T> g, const WaveDev w, unsigned char *__restrict__ fac,
                                                        int64_t total_levels)
{
   const int lane = threadIdx.x & 31;
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t L = warp; L < total_levels; L += n_warps) {
      const int a = w.lvl_ord[L];
      const int32_t p0 = w.lvl_pos[L + a], p1 = w.lvl_pos[L + a + 1];
      const int n = p1 - p0;
      T *ck = reinterpret_cast<T *>(fac + w.region[a] + w.chunk_rel[L + a]);
      const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
      for (int i = lane; i < n; i += 32) {
         const int4 m = w.meta[(int64_t)a * w.n_cells + p0 + i];
         const uint32_t mask = ((uint32_t)m.y >> 16) & 0xffu;
         T W[NB][NB];
         CellFactors<T, NB, F>(g, m.x, om, mask, W, ck + (size_t)NB * NB * n + i, (size_t)NB * NB * n, (size_t)n);
#pragma unroll
         for (int ii = 0; ii < NB; ii++)
#pragma unroll
            for (int j = 0; j < NB; j++) ck[(size_t)(ii * NB + j) * n + i] = W[ii][j];
      }
   }
}

// MODE 0: q; 1: u_a phi(node); 2: alpha q + u_a (phi(node) - alpha rho(node)).
// SMAX: the most gathered faces a cell of this shape can have (F - 1); the
// plan's S <= SMAX sets the store's stride.
template <typename T, int NB, int SMAX, int THREADS, int MODE>
__global__ void __launch_bounds__(THREADS, 1) WaveSweepKernel(const WaveDev w, const T *__restrict__ q,
                                                              T *__restrict__ psi, const unsigned char *__restrict__ fac,
                                                              const WaveInput in)
{
   extern __shared__ __align__(128) unsigned char smem[];
   uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
   int *s_abort = reinterpret_cast<int *>(smem + kWaveStages * 8);
   const int a = blockIdx.x, t = threadIdx.x;
   const int A = w.A;
   const int L0 = w.lvl_base[a];
   const int nlev = w.lvl_base[a + 1] - L0;
   int32_t *s_lp = reinterpret_cast<int32_t *>(smem + kWaveHeader);
   int32_t *s_co = s_lp + (w.max_levels + 1);
   int32_t *s_ro = s_co + (w.max_levels + 1);
   T *front = reinterpret_cast<T *>(smem + w.front_off);
   unsigned char *ring = smem + w.ring_base;
   const int S = w.S;
   const int R = NB * NB * (1 + S);

   for (int k = t; k <= nlev; k += THREADS) {
      s_lp[k] = w.lvl_pos[L0 + a + k];
      s_co[k] = w.chunk_rel[L0 + a + k];
      s_ro[k] = w.ring_off[L0 + a + k];
   }
   if (t == 0) {
      for (int k = 0; k < kWaveStages; k++) MbarInit(&bars[k], 1);
      *s_abort = 0;
      MbarInitFence();
   }
   __syncthreads();

   const unsigned char *region = fac + w.region[a];
   // Thread 0 keeps the copies going: level `next` is issued once the span
   // from the oldest unconsumed level's chunk to the end of its own fits the
   // ring (so chunks in flight never overlap) and it has a free mbarrier
   int next = 0;
   auto issue_upto = [&](int cur) {
      while (next < nlev && next - cur < kWaveStages &&
             (int64_t)s_co[next] + ChunkBytes<T>(s_lp[next + 1] - s_lp[next], R) - s_co[cur] <= w.cap) {
         uint64_t *bar = &bars[next % kWaveStages];
         const uint32_t bytes = ChunkBytes<T>(s_lp[next + 1] - s_lp[next], R);
         MbarExpectTx(bar, bytes);
         if ((int64_t)L0 + next != w.unmet_level) BulkLoad(ring + s_ro[next], region + s_co[next], bytes, bar);
         next++;
      }
   };
   if (t == 0) issue_upto(0);

   const T ua = (MODE != 0 && in.u) ? static_cast<const T *>(in.u)[a] : T(1);
   const double al = MODE == 2 ? *in.alpha : 0.0;
   const int4 *meta = w.meta + (int64_t)a * w.n_cells;

   // Register rings: plan records eight levels ahead (slot = level % 8), the
   // input values four levels ahead (slot = level % 4)
   int4 mreg[8];
   T rq[4][NB];
   double rp[4][NB], rr[4][NB];
#pragma unroll
   for (int k = 0; k < 8; k++) {
      mreg[k] = make_int4(-1, 0, 0, 0);
      if (k < nlev && s_lp[k] + t < s_lp[k + 1]) mreg[k] = __ldg(meta + s_lp[k] + t);
   }
#pragma unroll
   for (int k = 0; k < 4; k++) {
      const int64_t c = mreg[k].x;
#pragma unroll
      for (int j = 0; j < NB; j++) {
         rq[k][j] = T(0);
         rp[k][j] = rr[k][j] = 0.0;
         if (c >= 0) {
            if (MODE != 1) rq[k][j] = q[(c * NB + j) * A + a];
            if (MODE >= 1) rp[k][j] = in.phi[c * NB + j];
            if (MODE == 2) rr[k][j] = in.rho[c * NB + j];
         }
      }
   }

   bool aborted = false;
   for (int l0 = 0; l0 < nlev && !aborted; l0 += 8) {
#pragma unroll
      for (int u = 0; u < 8; u++) {
         const int l = l0 + u;
         if (l >= nlev) break;
         if (!MbarWaitBounded(&bars[l % kWaveStages], (uint32_t)(l / kWaveStages) & 1u, w.spin_limit)) {
            if (atomicCAS(s_abort, 0, 1) == 0) {
               atomicOr(&w.ctrl[kSweepCtrlError], 1u);
               atomicAdd(&w.ctrl[kSweepCtrlError + 1], 1u);
            }
         } else if (mreg[u].x >= 0) {
            const int4 m = mreg[u];
            const int n = s_lp[l + 1] - s_lp[l];
            const T *ck = reinterpret_cast<const T *>(ring + s_ro[l]);
            T r[NB];
#pragma unroll
            for (int j = 0; j < NB; j++) {
               if (MODE == 0) r[j] = rq[u & 3][j];
               else if (MODE == 1) r[j] = (T)((double)ua * rp[u & 3][j]);
               else r[j] = (T)(al * (double)rq[u & 3][j] + (double)ua * (rp[u & 3][j] - al * rr[u & 3][j]));
            }
            T y[NB];
#pragma unroll
            for (int ii = 0; ii < NB; ii++) {
               T acc = T(0);
#pragma unroll
               for (int j = 0; j < NB; j++) acc += ck[(ii * NB + j) * n + t] * r[j];
               y[ii] = acc;
            }
            const uint32_t ins[4] = {(uint32_t)m.z & 0xffffu, (uint32_t)m.z >> 16, (uint32_t)m.w & 0xffffu,
                                     (uint32_t)m.w >> 16};
#pragma unroll
            for (int s = 0; s < SMAX; s++) {
               if (s >= S || ins[s] == 0xffffu) continue;
               T x[NB];
#pragma unroll
               for (int j = 0; j < NB; j++) x[j] = front[ins[s] * NB + j];
               const T *G = ck + (size_t)NB * NB * (1 + s) * n + t;
#pragma unroll
               for (int ii = 0; ii < NB; ii++) {
                  T acc = T(0);
#pragma unroll
                  for (int j = 0; j < NB; j++) acc += G[(ii * NB + j) * n] * x[j];
                  y[ii] -= acc;
               }
            }
            const uint32_t out = (uint32_t)m.y & 0xffffu;
            if (out != 0xffffu)
#pragma unroll
               for (int j = 0; j < NB; j++) front[out * NB + j] = y[j];
#pragma unroll
            for (int j = 0; j < NB; j++) psi[((int64_t)m.x * NB + j) * A + a] = y[j];
         }
         // Refill: the input of level l + 4 (its record came four levels
         // ago), then the record of level l + 8
         {
            const int64_t c = mreg[(u + 4) & 7].x;
#pragma unroll
            for (int j = 0; j < NB; j++)
               if (c >= 0) {
                  if (MODE != 1) rq[u & 3][j] = q[(c * NB + j) * A + a];
                  if (MODE >= 1) rp[u & 3][j] = in.phi[c * NB + j];
                  if (MODE == 2) rr[u & 3][j] = in.rho[c * NB + j];
               }
            const int l8 = l + 8;
            mreg[u] = make_int4(-1, 0, 0, 0);
            if (l8 < nlev && s_lp[l8] + t < s_lp[l8 + 1]) mreg[u] = __ldg(meta + s_lp[l8] + t);
         }
         __syncthreads();
         if (*(volatile int *)s_abort) {
            aborted = true;
            break;
         }
         if (t == 0) issue_upto(l + 1);
      }
   }
   if (aborted && t == 0) {
      // Copies issued and not consumed are waited for (bounded) before the
      // block's shared memory goes away; the hook's level never had one
      for (int lv = 0; lv < next; lv++) {
         if ((int64_t)L0 + lv == w.unmet_level) continue;
         MbarWaitBounded(&bars[lv % kWaveStages], (uint32_t)(lv / kWaveStages) & 1u, w.spin_limit);
      }
   }
}

template <typename T, int NB, int SMAX, int THREADS>
int LaunchWaveSweepT(const WaveDev &w, const T *q, T *psi, const void *fac, const WaveInput *in, cudaStream_t st)
{
   WaveInput none;
   const WaveInput &inp = in ? *in : none;
   const int mode = !in ? 0 : (in->iso ? 1 : 2);
   auto kern = mode == 0   ? WaveSweepKernel<T, NB, SMAX, THREADS, 0>
               : mode == 1 ? WaveSweepKernel<T, NB, SMAX, THREADS, 1>
                           : WaveSweepKernel<T, NB, SMAX, THREADS, 2>;
   if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, w.smem) != cudaSuccess)
      return CudaCheck(cudaGetLastError(), "wave sweep shared memory");
   kern<<<w.A, THREADS, w.smem, st>>>(w, q, psi, static_cast<const unsigned char *>(fac), inp);
   return CheckLaunch("wave sweep");
}

}  // namespace

int WaveFactors(ubolt_ctx *ctx, const WaveDev &w, void *fac, int elem, cudaStream_t st, int64_t total_levels)
{
   int n_sm = 0, dev = 0;
   cudaGetDevice(&dev);
   cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
   const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total_levels + 3) / 4, (int64_t)n_sm * 16));
   unsigned char *f = static_cast<unsigned char *>(fac);
   if (elem == 8) {
      UBOLT_DISPATCH(ctx->nb, ctx->F, {
         WaveFactorKernel<double, NB_, F_><<<grid, 128, 0, st>>>(ctx->geom<double>(), w, f, total_levels);
         return CheckLaunch("wave factors");
      });
   } else {
      UBOLT_DISPATCH(ctx->nb, ctx->F, {
         WaveFactorKernel<float, NB_, F_><<<grid, 128, 0, st>>>(ctx->geom<float>(), w, f, total_levels);
         return CheckLaunch("wave factors");
      });
   }
   return SetError(UBOLT_ERR_STATE, "no wave factor kernel for this shape");
}

int WaveSweep(ubolt_ctx *ctx, const WaveDev &w, const void *q, void *psi, const void *fac, int elem,
              const WaveInput *in, int threads, cudaStream_t st)
{
   if (elem == 8) {
      UBOLT_DISPATCH(ctx->nb, ctx->F, {
         const double *qq = static_cast<const double *>(q);
         double *pp = static_cast<double *>(psi);
         return threads <= 256 ? LaunchWaveSweepT<double, NB_, F_ - 1, 256>(w, qq, pp, fac, in, st)
                               : LaunchWaveSweepT<double, NB_, F_ - 1, 512>(w, qq, pp, fac, in, st);
      });
   } else {
      UBOLT_DISPATCH(ctx->nb, ctx->F, {
         const float *qq = static_cast<const float *>(q);
         float *pp = static_cast<float *>(psi);
         return threads <= 256 ? LaunchWaveSweepT<float, NB_, F_ - 1, 256>(w, qq, pp, fac, in, st)
                               : LaunchWaveSweepT<float, NB_, F_ - 1, 512>(w, qq, pp, fac, in, st);
      });
   }
   return SetError(UBOLT_ERR_STATE, "no wave sweep kernel for this shape");
}

}  // namespace ubolt
