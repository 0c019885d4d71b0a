// The streaming stage of the preconditioner: psi = L^{-1} q, L = streaming +
// removal, by an upwind transport sweep of every ordinate at once.
//
// UBOLT preconditions streaming with PCAIR (src/transport_solverk.kokkos.cxx:
// 238-260), an algebraic multigrid approximation of L^{-1}. Here L^{-1} is
// applied exactly wherever the per-ordinate upwind graph is acyclic.
//
// The plan (sweep_plan.cpp, host, once per mesh and ordinate set) cuts each
// ordinate's sweep into tasks - a piece of one patch of consecutive cells,
// its cells in level order - numbered so every task's upstream tasks come
// before it. Reflective inflow couples ordinates and is lagged (read as zero),
// as are the couplings a cycle break releases.
//
// Kernel: persistent, one warp per task, tasks taken in number order. The
// critical path of a sweep is the chain of upwind dependencies, so everything
// off that chain is moved ahead of the wait: in a prologue the lanes build and
// LU-factorise every cell's nb x nb block from geometry and sigma_t, and keep
// y0 = B^{-1} q and G_f = B^{-1} s_f face_up_f (one per gathered face) in the
// warp's shared-memory slice. Then the warp waits, with a bounded spin, on the
// epoch flags of its upstream tasks, folds their values in once
// (y0 -= G_f psi(up), read from L2 with ld.global.cg), and walks its levels
// touching only shared memory: psi_c = y0 - sum G_f psi(up). It publishes its
// flag with a release store after a device-scope fence. Deadlock-free: a task
// waits only on lower-numbered tasks, which were taken by warps already running.
#include "ctx.h"
#include "sweep_plan.h"

#include <algorithm>
#include <vector>

struct ubolt_sweep_plan {
   int32_t P = 0, n_patches = 0, A = 0;
   int64_t n_tasks = 0, n_lagged = 0, n_split = 0, total_levels = 0;
   int32_t max_levels = 0, max_inflow = 0;
   // Device arrays (owned by the context's allocation list)
   const int32_t *task_pa = nullptr;    // [n_tasks] patch * A + ordinate
   const int32_t *dep_ptr = nullptr;    // [n_tasks + 1]
   const int32_t *deps = nullptr;       // upstream task ids
   const int64_t *cell_ptr = nullptr;   // [n_tasks + 1]
   const uint8_t *tcell = nullptr;      // local cell index in the patch, level order
   const uint16_t *tmask = nullptr;     // upwind faces: in task (bit f) / earlier task (bit 8 + f)
   const int32_t *lvl_ptr = nullptr;    // [n_tasks + 1]
   const uint16_t *lvl = nullptr;       // level end positions within the task
   uint32_t *flags = nullptr;           // [n_tasks] epoch of the last completion
   uint32_t *ctrl = nullptr;            // [0] task counter, [1] error flag, [2] timeout count
   uint32_t epoch = 0;
   int grid = 0, warps_per_block = 4;
   uint32_t spin_limit = 1u << 22;
   int64_t unmet_task = -1;  // ubolt_sweep_test_wait: one task waits on a flag nothing sets
};

namespace ubolt {

namespace {

template <typename T>
int UploadVec(ubolt_ctx *ctx, const std::vector<T> &h, const T **d)
{
   void *p = nullptr;
   int rc = CtxAlloc(ctx, std::max<size_t>(h.size(), 1) * sizeof(T), &p);
   if (rc) return rc;
   if (!h.empty()) rc = CudaCheck(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "sweep plan");
   *d = static_cast<const T *>(p);
   return rc;
}

}  // namespace

__device__ __forceinline__ uint32_t LoadAcquire(const uint32_t *p)
{
   uint32_t v;
   asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
   return v;
}

__device__ __forceinline__ void StoreRelease(uint32_t *p, uint32_t v)
{
   asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct SweepDev {
   int32_t P, A;
   int64_t n_tasks;
   const int32_t *task_pa, *dep_ptr, *deps;
   const int64_t *cell_ptr;
   const uint8_t *tcell;
   const uint16_t *tmask;
   const int32_t *lvl_ptr;
   const uint16_t *lvl;
   uint32_t *flags, *ctrl;
   uint32_t epoch;
   uint32_t spin_limit;
   int32_t slots;
   int64_t unmet_task;
};

template <typename T, int NB, int F>
__global__ void __launch_bounds__(128) SweepKernel(const DevGeom<T> g, const SweepDev s, const T *__restrict__ q,
                                                   T *__restrict__ psi)
{
   extern __shared__ __align__(16) unsigned char smem_raw[];
   const int lane = threadIdx.x & 31;
   const int warp = threadIdx.x >> 5;
   const int S = s.slots;  // coupling matrices kept per cell
   // Per warp: loc[P][NB] (the right-hand side, then the solution) and
   // G[P][S][NB][NB], G_f = B^{-1} s_f face_up_f for each gathered face
   T *loc = reinterpret_cast<T *>(smem_raw) + (size_t)warp * s.P * (NB + S * NB * NB);
   T *G = loc + (size_t)s.P * NB;
   const int A = s.A;

   for (;;) {
      int64_t t = 0;
      if (lane == 0) t = (int64_t)atomicAdd(&s.ctrl[0], 1u);
      t = __shfl_sync(0xffffffffu, t, 0);
      if (t >= s.n_tasks) break;
      const int32_t pa = s.task_pa[t];
      const int32_t p = pa / A;
      const int a = pa - p * A;
      const int64_t base = (int64_t)p * s.P;
      const int64_t off = s.cell_ptr[t];
      const int ncell = (int)(s.cell_ptr[t + 1] - off);
      const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};

      // Prologue, before the wait - nothing here depends on upstream values:
      // every cell's block B factorised once, y0 = B^{-1} q into loc, and
      // G_f = B^{-1} (s_f face_up_f) for every gathered face into G
      for (int i = lane; i < ncell; i += 32) {
         const int local = s.tcell[off + i];
         const uint32_t mask = s.tmask[off + i];
         const int64_t c = base + local;
         const int32_t cl = g.cls[c];
         T B[NB][NB];
         int perm[NB];
         BuildBlock<T, NB, F>(g, cl, om, g.sigma_t[c], B);
         const bool ok = LuFactor<T, NB>(B, perm);
         T r[NB];
#pragma unroll
         for (int j = 0; j < NB; j++) r[j] = ok ? q[(c * NB + j) * A + a] : T(0);
         if (ok) LuSolve<T, NB>(B, perm, r);
#pragma unroll
         for (int j = 0; j < NB; j++) loc[local * NB + j] = r[j];
         int slot = 0;
#pragma unroll
         for (int f = 0; f < F; f++) {
            if (!(((mask >> f) | (mask >> (8 + f))) & 1u)) continue;
            const T sf = Dot3(om, g.nA + ((int64_t)cl * F + f) * 3);
            T *Gf = G + ((size_t)local * S + slot) * NB * NB;
            if constexpr (NB == 1) {
               Gf[0] = ok ? sf * g.inv_vol[cl] / B[0][0] : T(0);
            } else {
               const T *M = g.fup + ((int64_t)cl * F + f) * NB * NB;
#pragma unroll
               for (int j = 0; j < NB; j++) {
                  T col[NB];
#pragma unroll
                  for (int ii = 0; ii < NB; ii++) col[ii] = sf * M[ii * NB + j];
                  if (ok) LuSolve<T, NB>(B, perm, col);
#pragma unroll
                  for (int ii = 0; ii < NB; ii++) Gf[ii * NB + j] = ok ? col[ii] : T(0);
               }
            }
            slot++;
         }
      }

      // Wait for the upstream tasks: bounded, and a timeout is reported
      for (int d = s.dep_ptr[t] + lane; d < s.dep_ptr[t + 1]; d += 32) {
         const uint32_t *f = &s.flags[s.deps[d]];
         uint32_t spins = 0;
         const uint32_t want = (t == s.unmet_task) ? s.epoch + 1u : s.epoch;
         while (LoadAcquire(f) != want) {
            if (++spins > s.spin_limit || *(volatile uint32_t *)&s.ctrl[1]) {
               atomicOr(&s.ctrl[1], 1u);
               atomicAdd(&s.ctrl[2], 1u);
               break;
            }
            __nanosleep(spins < 64 ? 32 : 256);
         }
      }
      __syncwarp();
      __threadfence();

      // Fold the upwind values from earlier tasks in: y0 -= G_f psi(up)
      for (int i = lane; i < ncell; i += 32) {
         const uint32_t mask = s.tmask[off + i];
         if (!(mask >> 8)) continue;
         const int local = s.tcell[off + i];
         const int64_t c = base + local;
         T y[NB];
#pragma unroll
         for (int j = 0; j < NB; j++) y[j] = loc[local * NB + j];
         int slot = 0;
#pragma unroll
         for (int f = 0; f < F; f++) {
            const bool here = (mask >> f) & 1u, earlier = (mask >> (8 + f)) & 1u;
            if (!(here || earlier)) continue;
            if (earlier) {
               const int64_t up = g.code[c * F + f];
               const T *Gf = G + ((size_t)local * S + slot) * NB * NB;
               T xn[NB];
#pragma unroll
               for (int j = 0; j < NB; j++) xn[j] = __ldcg(&psi[(up * NB + j) * A + a]);
#pragma unroll
               for (int ii = 0; ii < NB; ii++) {
                  T u = T(0);
#pragma unroll
                  for (int j = 0; j < NB; j++) u += Gf[ii * NB + j] * xn[j];
                  y[ii] -= u;
               }
            }
            slot++;
         }
#pragma unroll
         for (int j = 0; j < NB; j++) loc[local * NB + j] = y[j];
      }
      __syncwarp();

      // Level by level, shared memory only: psi_c = y0 - sum_{in-task f} G_f psi(up)
      int lo = 0;
      for (int l = s.lvl_ptr[t]; l < s.lvl_ptr[t + 1]; l++) {
         const int hi = s.lvl[l];
         for (int i = lo + lane; i < hi; i += 32) {
            const int local = s.tcell[off + i];
            const uint32_t mask = s.tmask[off + i];
            const int64_t c = base + local;
            T y[NB];
#pragma unroll
            for (int j = 0; j < NB; j++) y[j] = loc[local * NB + j];
            if (mask & 0xffu) {
               int slot = 0;
#pragma unroll
               for (int f = 0; f < F; f++) {
                  const bool here = (mask >> f) & 1u, earlier = (mask >> (8 + f)) & 1u;
                  if (!(here || earlier)) continue;
                  if (here) {
                     const int ul = (int)(g.code[c * F + f] - base);
                     const T *Gf = G + ((size_t)local * S + slot) * NB * NB;
#pragma unroll
                     for (int ii = 0; ii < NB; ii++) {
                        T u = T(0);
#pragma unroll
                        for (int j = 0; j < NB; j++) u += Gf[ii * NB + j] * loc[ul * NB + j];
                        y[ii] -= u;
                     }
                  }
                  slot++;
               }
#pragma unroll
               for (int j = 0; j < NB; j++) loc[local * NB + j] = y[j];
            }
#pragma unroll
            for (int j = 0; j < NB; j++) psi[(c * NB + j) * A + a] = y[j];
         }
         lo = hi;
         __syncwarp();
      }
      __threadfence();
      __syncwarp();
      if (lane == 0) StoreRelease(&s.flags[t], s.epoch);
   }
}

// ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

int BuildSweepPlan(ubolt_ctx *ctx, int patch_size)
{
   const int64_t nc = ctx->n_cells;
   int P = patch_size > 0 ? patch_size : 64;
   if (P > 256) P = 256;
   if (P > nc) P = (int)nc;
   if (((nc + P - 1) / P) * (int64_t)ctx->A * 4 >= INT32_MAX) return SetError(UBOLT_ERR_ARG, "too many sweep tasks");
   HostSweepPlan h;
   BuildHostSweepPlan(nc, ctx->F, ctx->A, P, ctx->h_omega.data(), ctx->h_nA.data(), ctx->h_code.data(), h);

   auto plan = new ubolt_sweep_plan();
   plan->P = h.P;
   plan->n_patches = h.n_patches;
   plan->A = h.A;
   plan->n_tasks = h.n_tasks;
   plan->n_lagged = h.n_lagged;
   plan->n_split = h.n_split;
   plan->max_levels = h.max_levels;
   plan->max_inflow = h.max_inflow;
   plan->total_levels = (int64_t)h.lvl.size();
   int rc = 0;
   if ((rc = UploadVec(ctx, h.task_pa, &plan->task_pa)) || (rc = UploadVec(ctx, h.dep_ptr, &plan->dep_ptr)) ||
       (rc = UploadVec(ctx, h.deps, &plan->deps)) || (rc = UploadVec(ctx, h.cell_ptr, &plan->cell_ptr)) ||
       (rc = UploadVec(ctx, h.tcell, &plan->tcell)) || (rc = UploadVec(ctx, h.tmask, &plan->tmask)) ||
       (rc = UploadVec(ctx, h.lvl_ptr, &plan->lvl_ptr)) || (rc = UploadVec(ctx, h.lvl, &plan->lvl))) {
      delete plan;
      return rc;
   }
   void *p = nullptr;
   if ((rc = CtxAlloc(ctx, h.n_tasks * sizeof(uint32_t), &p))) { delete plan; return rc; }
   plan->flags = static_cast<uint32_t *>(p);
   cudaMemset(plan->flags, 0, h.n_tasks * sizeof(uint32_t));
   if ((rc = CtxAlloc(ctx, 4 * sizeof(uint32_t), &p))) { delete plan; return rc; }
   plan->ctrl = static_cast<uint32_t *>(p);
   cudaMemset(plan->ctrl, 0, 4 * sizeof(uint32_t));
   delete ctx->sweep;
   ctx->sweep = plan;
   return CudaCheck(cudaDeviceSynchronize(), "sweep plan");
}

template <typename T, int NB, int F>
static int LaunchSweep(ubolt_ctx *ctx, const T *q, T *psi, cudaStream_t st)
{
   ubolt_sweep_plan *pl = ctx->sweep;
   const int threads = 32 * pl->warps_per_block;
   const int slots = std::max(1, std::min(F - 1, (int)pl->max_inflow));
   const size_t smem = sizeof(T) * (size_t)pl->warps_per_block * pl->P * (NB + slots * NB * NB);
   auto kern = SweepKernel<T, NB, F>;
   if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
   int per_sm = 0, n_sm = 0, dev = 0;
   cudaGetDevice(&dev);
   cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
   const int64_t want = (pl->n_tasks + pl->warps_per_block - 1) / pl->warps_per_block;
   const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::max(per_sm, 1) * n_sm, want));
   pl->grid = grid;
   pl->epoch++;
   if (pl->epoch == 0) pl->epoch = 1;
   SweepDev s;
   s.P = pl->P;
   s.A = pl->A;
   s.n_tasks = pl->n_tasks;
   s.task_pa = pl->task_pa;
   s.dep_ptr = pl->dep_ptr;
   s.deps = pl->deps;
   s.cell_ptr = pl->cell_ptr;
   s.tcell = pl->tcell;
   s.tmask = pl->tmask;
   s.lvl_ptr = pl->lvl_ptr;
   s.lvl = pl->lvl;
   s.flags = pl->flags;
   s.ctrl = pl->ctrl;
   s.epoch = pl->epoch;
   s.spin_limit = pl->spin_limit;
   s.unmet_task = pl->unmet_task;
   pl->unmet_task = -1;
   s.slots = slots;
   cudaMemsetAsync(pl->ctrl, 0, sizeof(uint32_t), st);  // task counter; the error flag stays sticky
   kern<<<grid, threads, smem, st>>>(ctx->geom<T>(), s, q, psi);
   return CheckLaunch("sweep");
}

template <typename T>
int Sweep(ubolt_ctx *ctx, const T *q, T *psi, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!ctx->sweep && (rc = BuildSweepPlan(ctx, 0))) return rc;
   if (!q || !psi || (const void *)q == (const void *)psi)
      return SetError(UBOLT_ERR_ARG, "sweep: q and psi must be distinct device arrays");
   UBOLT_DISPATCH(ctx->nb, ctx->F, return (LaunchSweep<T, NB_, F_>(ctx, q, psi, (cudaStream_t)stream)));
   return SetError(UBOLT_ERR_STATE, "no sweep kernel for this shape");
}

template int Sweep<double>(ubolt_ctx *, const double *, double *, void *);
template int Sweep<float>(ubolt_ctx *, const float *, float *, void *);

}  // namespace ubolt

using namespace ubolt;

void UboltSweepFree(ubolt_ctx *ctx)
{
   delete ctx->sweep;
   ctx->sweep = nullptr;
}

extern "C" int ubolt_sweep_setup(ubolt_ctx *ctx, int patch_size)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (patch_size < 0 || patch_size > 256) return SetError(UBOLT_ERR_ARG, "patch size %d (1..256, 0 = default)", patch_size);
   return BuildSweepPlan(ctx, patch_size);
}

extern "C" int ubolt_sweep(ubolt_ctx *ctx, const double *q, double *psi, void *stream)
{
   return Sweep<double>(ctx, q, psi, stream);
}

extern "C" int ubolt_sweep_f32(ubolt_ctx *ctx, const float *q, float *psi, void *stream)
{
   return Sweep<float>(ctx, q, psi, stream);
}

extern "C" int ubolt_sweep_status(ubolt_ctx *ctx, ubolt_sweep_info *info, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!ctx->sweep) return SetError(UBOLT_ERR_STATE, "no sweep plan");
   ubolt_sweep_plan *pl = ctx->sweep;
   uint32_t h[4] = {0, 0, 0, 0};
   cudaStream_t s = (cudaStream_t)stream;
   cudaMemcpyAsync(h, pl->ctrl, sizeof h, cudaMemcpyDeviceToHost, s);
   if ((rc = CudaCheck(cudaStreamSynchronize(s), "sweep_status"))) return rc;
   if (info) {
      info->patch_size = pl->P;
      info->n_patches = pl->n_patches;
      info->n_tasks = pl->n_tasks;
      info->n_lagged = pl->n_lagged;
      info->n_split = pl->n_split;
      info->max_levels = pl->max_levels;
      info->total_levels = pl->total_levels;
      info->grid = pl->grid;
      info->timeouts = h[2];
   }
   if (h[1]) {
      cudaMemsetAsync(pl->ctrl + 1, 0, 2 * sizeof(uint32_t), s);
      cudaStreamSynchronize(s);
      return SetError(UBOLT_ERR_TIMEOUT, "a sweep wait gave up (%u timeouts); its result is not valid", h[2]);
   }
   return UBOLT_OK;
}

extern "C" int ubolt_sweep_test_wait(ubolt_ctx *ctx, uint32_t spin_limit, int make_one_wait_unmet)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!ctx->sweep && (rc = BuildSweepPlan(ctx, 0))) return rc;
   ubolt_sweep_plan *pl = ctx->sweep;
   if (spin_limit < 16) return SetError(UBOLT_ERR_ARG, "spin limit %u too small", spin_limit);
   pl->spin_limit = spin_limit;
   pl->unmet_task = -1;
   if (make_one_wait_unmet) {
      // The first task that has an upstream task waits for an epoch that no
      // task of this sweep publishes
      std::vector<int32_t> dp(pl->n_tasks + 1);
      cudaMemcpy(dp.data(), pl->dep_ptr, dp.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
      for (int64_t t = 0; t < pl->n_tasks; t++)
         if (dp[t + 1] > dp[t]) { pl->unmet_task = t; break; }
      if (pl->unmet_task < 0) return SetError(UBOLT_ERR_STATE, "no task of this plan waits on another");
   }
   return UBOLT_OK;
}
