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
// Kernel: persistent, one warp per task, tasks taken in number order.
// Synchronisation is by the data itself: psi is filled with a sentinel bit
// pattern (all ones, a NaN the kernel never stores) before the launch, and a
// cell whose upwind neighbour lies in an earlier task polls that neighbour's
// psi values until none is the sentinel. So a task waits for exactly the
// values it reads, at the level that reads them, and can start while its
// upstream tasks are still walking: the chain of dependencies runs cell to
// cell through L2 with no flags, fences or task-granular barriers.
//
// Everything off that chain happens first, in a prologue: the lanes build and
// invert every cell's nb x nb block from geometry and sigma_t, and keep
// y0 = B^{-1} q and G_f = B^{-1} s_f face_up_f (one per gathered face) in the
// warp's shared-memory slice. The walk then runs level by level, touching
// shared memory for in-task neighbours: psi_c = y0 - sum_f G_f psi(up_f).
// Deadlock-free: a task polls only values of lower-numbered tasks, which were
// taken by warps already running. Every poll is bounded; a poll that gives up
// records a timeout, reads the value as zero and the sweep completes.
#include "ctx.h"
#include "sweep_plan.h"
#include "wave.h"

#include <algorithm>
#include <vector>

// The task counter and the error words sit on separate 128-byte lines: every
// warp increments the counter, and a spinning lane must not contend with it.
// Words [kCtrlNever, kCtrlNever + 2) hold a sentinel nothing overwrites (the
// target of the bounded-wait test hook).
constexpr int kCtrlCounter = 0, kCtrlError = ubolt::kSweepCtrlError, kCtrlNever = 48, kCtrlWords = 64;
constexpr int kSweepBlocksPerSm = 8;  // of 4 warps
constexpr int kDefaultPatch = 64;

// The default patch: half a tile of the mesh builders' cell numbering (8 x 8
// quads, 4^3 hexes), and four cubes' worth of Kuhn tetrahedra. Measured per
// isotropic-source sweep at S8 (FP64 / FP32): 256^2 triangles 0.89 / 0.78 ms
// at 64 cells against 0.97 / 0.83 at 32; 44^3 Kuhn tets 15.3 / 12.0 ms at 24
// against 18.2 / 14.1 at 32 and 23.4 / 15.8 at 64. On the 128^3 hex box 64
// stays: the 4-group FP64 solve, whose factors are built in the sweep, took
// 1.64 s at 64 against 1.79 s at 32 (the mixed solve 1.08 / 1.07 s)
static int DefaultPatch(const ubolt_ctx *ctx)
{
   return (ctx->dim == 3 && ctx->F == 4) ? 24 : kDefaultPatch;
}

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
   const uint16_t *tlev = nullptr;      // [entries] level of each entry within its task
   const int32_t *tlink = nullptr;      // [entries][slots] upwind link per gathered face: >= 0 the cell in an
                                        // earlier task, -2 - local for a cell of this task, -1 none
   uint32_t *ctrl = nullptr;            // [kCtrlCounter] task counter; [kCtrlError] error flag, [kCtrlError + 1] timeout count
   int grid = 0, warps_per_block = 4, slots = 1;
   uint32_t spin_limit = 1u << 22;
   int64_t unmet_task = -1;  // ubolt_sweep_test_wait: one task polls a value nothing writes
   // The factor store (B^{-1} and couplings per task entry) per precision,
   // valid for the group epoch it was built in; limit < 0: automatic
   void *fac[2] = {nullptr, nullptr};
   uint64_t fac_epoch[2] = {0, 0};
   int64_t fac_limit = -1;
   // The wave plan (one block per ordinate), where every ordinate's upwind
   // graph is acyclic and a level fits a block: wave[which].smem > 0 where
   // precision `which` (0 FP64, 1 FP32) can run it. fac_wave[which]: the
   // store reserved for that precision is in wave order (the wave kernel runs)
   bool wave_ok = false;
   int wave_threads = 256;
   int64_t wave_levels = 0;
   ubolt::WaveDev wave[2];
   int64_t wave_bytes[2] = {0, 0};
   bool fac_wave[2] = {false, false};
   int kernel_mode = UBOLT_SWEEP_AUTO;
   int64_t unmet_level = -1;  // ubolt_sweep_test_wait: one level's copy is never issued
   ~ubolt_sweep_plan()
   {
      for (void *f : fac)
         if (f) cudaFree(f);
   }
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

// psi values cross warps through L2 as single 4- or 8-byte relaxed accesses:
// a reader sees the sentinel or the final value, never a torn one
__device__ __forceinline__ double LoadRelaxed(const double *p)
{
   double v;
   asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
   return v;
}
__device__ __forceinline__ float LoadRelaxed(const float *p)
{
   float v;
   asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
   return v;
}
__device__ __forceinline__ void StoreRelaxed(double *p, double v)
{
   asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void StoreRelaxed(float *p, float v)
{
   asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ bool IsSentinel(double v) { return __double_as_longlong(v) == -1LL; }
__device__ __forceinline__ bool IsSentinel(float v) { return __float_as_int(v) == -1; }
template <typename T>
__device__ __forceinline__ T Sentinel();
template <>
__device__ __forceinline__ double Sentinel<double>() { return __longlong_as_double(-1LL); }
template <>
__device__ __forceinline__ float Sentinel<float>() { return __int_as_float(-1); }
// A computed value equal to the sentinel (a NaN carrying its payload) is
// stored as another NaN, so a reader can never mistake a result for "not yet"
__device__ __forceinline__ double Publishable(double v) { return IsSentinel(v) ? __longlong_as_double(0x7ff8000000000001LL) : v; }
__device__ __forceinline__ float Publishable(float v) { return IsSentinel(v) ? __int_as_float(0x7fc00001) : v; }

struct SweepDev {
   int32_t P, A;
   int64_t n_tasks;
   const int32_t *task_pa;
   const int64_t *cell_ptr;
   const uint8_t *tcell;
   const uint16_t *tmask;
   const uint16_t *tlev;
   const int32_t *tlink;
   const int32_t *lvl_ptr;
   const uint16_t *lvl;
   uint32_t *ctrl;
   uint32_t spin_limit;
   int32_t slots;
   int64_t unmet_task;
   // Affine input: when aff_phi is set the sweep reads
   // q(node, a) = alpha r0(node, a) + u_a (phi(node) - alpha rho(node)),
   // u_a = aff_u[a] or 1, with r0 passed as q (compressed GMRES's Arnoldi vector)
   const double *aff_alpha, *aff_phi, *aff_rho;
   const void *aff_u;
   int32_t aff_iso;  // r0 is isotropic (r0 = E rho): the input is u_a phi(node), q is not read
   int32_t aff_inv_volume;  // with aff_iso: the input is u_a phi(node) / V(cell) (the adjoint's P V^{-1} E_w phi)
   // psi(c, j, a) at psi[c os_c + j os_j + a os_a]: UBOLT's row layout
   // (NB A, A, 1), or ordinate-major (NB, 1, n_cells NB), where a task's
   // cells of one ordinate are contiguous and it writes whole sectors
   int64_t os_c, os_j, os_a;
};

// Per-warp shared-memory slice, for P cells and S gathered faces per cell
// Each nb x nb coupling in shared memory takes a 16-byte multiple, so the
// walk reads it with 16-byte loads
__host__ __device__ constexpr int GStride(int NB, int elem) { return (NB * NB * elem + 15) / 16 * 16 / elem; }

// A position's S couplings in shared memory. A run of a multiple of four
// 16-byte units (the 4 x 4 blocks of 3D DG1) is padded by one unit: a
// quarter-warp's 16-byte reads of one slot at consecutive positions would
// otherwise fall on the same banks, 8-way. Shorter conflicts are left alone:
// the padding's shared memory costs L1 (the shapes on triangles and quads
// run slower with it).
__host__ __device__ constexpr int PosStride(int S, int NB, int elem)
{
   return (S * GStride(NB, elem) * elem / 16 % 4 == 0 ? S * GStride(NB, elem) * elem + 16
                                                       : S * GStride(NB, elem) * elem) / elem;
}

struct SweepSlice {
   size_t loc, G, bytes;
   __host__ __device__ SweepSlice(int P, int S, int NB, int elem)
   {
      auto up = [](size_t v) { return (v + 15) & ~(size_t)15; };
      loc = 0;                                           // T [P][NB], by local cell
      G = up(loc + (size_t)P * NB * elem);               // T [P][PosStride], by position
      bytes = up(G + (size_t)P * PosStride(S, NB, elem) * elem);
   }
};

// The NB values psi(up, :, a) of an upwind cell in an earlier task, polled
// until its task has stored them all. Bounded: on giving up the sticky error
// flag is set, the timeout counted, and the missing values read as zero.
template <typename T, int NB>
__device__ __forceinline__ void PollUpwind(const T *p, int stride, const SweepDev &s, T xn[NB])
{
   bool missing = false;
#pragma unroll
   for (int j = 0; j < NB; j++) {
      xn[j] = LoadRelaxed(p + (size_t)j * stride);
      missing |= IsSentinel(xn[j]);
   }
   uint32_t spins = 0;
   while (missing) {
      // The sticky error flag (another wait gave up) is read once per 1024
      // spins, so that waiting lanes stay off its line
      if (++spins > s.spin_limit || ((spins & 1023u) == 0 && *(volatile uint32_t *)&s.ctrl[kCtrlError])) {
         atomicOr(&s.ctrl[kCtrlError], 1u);
         atomicAdd(&s.ctrl[kCtrlError + 1], 1u);
#pragma unroll
         for (int j = 0; j < NB; j++)
            if (IsSentinel(xn[j])) xn[j] = T(0);
         return;
      }
      if (spins > 32) __nanosleep(spins < 4096 ? 32 : 256);
      missing = false;
#pragma unroll
      for (int j = 0; j < NB; j++)
         if (IsSentinel(xn[j])) {
            xn[j] = LoadRelaxed(p + (size_t)j * stride);
            missing |= IsSentinel(xn[j]);
         }
   }
}

// y -= G x for one nb x nb coupling held in shared memory (16-byte aligned,
// GStride elements), read with 16-byte loads
template <typename T, int NB>
__device__ __forceinline__ void SubCoupling(const T *__restrict__ Gf, const T xn[NB], T y[NB])
{
   constexpr int GS = GStride(NB, (int)sizeof(T));
   constexpr int PER = 16 / (int)sizeof(T);
   T gv[GS];
#pragma unroll
   for (int v = 0; v < GS / PER; v++) {
      if constexpr (sizeof(T) == 8) {
         const double2 d = reinterpret_cast<const double2 *>(Gf)[v];
         gv[2 * v] = d.x;
         gv[2 * v + 1] = d.y;
      } else {
         const float4 d = reinterpret_cast<const float4 *>(Gf)[v];
         gv[4 * v] = d.x;
         gv[4 * v + 1] = d.y;
         gv[4 * v + 2] = d.z;
         gv[4 * v + 3] = d.w;
      }
   }
#pragma unroll
   for (int ii = 0; ii < NB; ii++) {
      T u = T(0);
#pragma unroll
      for (int j = 0; j < NB; j++) u += gv[ii * NB + j] * xn[j];
      y[ii] -= u;
   }
}

// The factor store: per task, element-major over its positions, so a warp's
// lanes read consecutive words - element r of position i of task t at
// cell_ptr[t] R + r ncell_t + i, R = NB^2 (1 + S): W, then G_0 .. G_{S-1}.
// Independent of the right-hand side: built once per group, read by every sweep.
template <typename T, int NB, int F>
__global__ void __launch_bounds__(128) FactorKernel(const DevGeom<T> g, const SweepDev s, T *__restrict__ fac)
{
   const int lane = threadIdx.x & 31;
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   const int S = s.slots;
   const size_t R = (size_t)NB * NB * (1 + S);
   for (int64_t t = warp; t < s.n_tasks; t += n_warps) {
      const int32_t pa = s.task_pa[t];
      const int64_t off = s.cell_ptr[t];
      const int ncell = (int)(s.cell_ptr[t + 1] - off);
      const int32_t p = pa / s.A;
      const int a = pa - p * s.A;
      const int64_t base = (int64_t)p * s.P;
      const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
      T *ft = fac + (size_t)off * R;
      for (int i = lane; i < ncell; i += 32) {
         T W[NB][NB];
         CellFactors<T, NB, F>(g, base + s.tcell[off + i], om, s.tmask[off + i], W, ft + (size_t)NB * NB * ncell + i,
                               (size_t)NB * NB * ncell, (size_t)ncell);
#pragma unroll
         for (int ii = 0; ii < NB; ii++)
#pragma unroll
            for (int j = 0; j < NB; j++) ft[(size_t)(ii * NB + j) * ncell + i] = W[ii][j];
      }
   }
}

// PL: positions per lane, P <= 32 PL. Lane l owns positions l, l + 32, ...;
// its cells' schedule (local index, level, upwind links) stays in registers.
// CACHED: the factors come from the store, else they are computed here.
// Resident blocks of 4 warps the compiler should fit per SM: the sweep is
// bound by per-task latency, and FP64 nb <= 3 with one cell per lane fits a
// fifth block without spilling (with two, the spills cost more than the
// block). On triangles with two cells per lane FP64 keeps a fourth block
// (at most 128 registers, no spill): left free it took 134 and three
// blocks, and the 256^2 triangle sweep 0.969 ms against 0.941
template <typename T, int NB, int F, int PL>
constexpr int SweepMinBlocks()
{
   return (sizeof(T) == 8 && NB <= 3 && PL == 1) ? 5 : (sizeof(T) == 8 && NB <= 3 && F == 3 && PL == 2) ? 4 : 1;
}

template <typename T, int NB, int F, int PL, bool CACHED>
__global__ void __launch_bounds__(128, SweepMinBlocks<T, NB, F, PL>()) SweepKernel(const DevGeom<T> g, const SweepDev s, const T *__restrict__ q,
                                                   T *__restrict__ psi, const T *__restrict__ fac)
{
   extern __shared__ __align__(16) unsigned char smem_raw[];
   const int lane = threadIdx.x & 31;
   const int warp = threadIdx.x >> 5;
   const int S = s.slots;     // coupling matrices kept per cell
   constexpr int SM = F - 1;  // most gathered faces of a cell
   const SweepSlice L(s.P, S, NB, (int)sizeof(T));
   unsigned char *slice = smem_raw + (size_t)warp * L.bytes;
   T *loc = reinterpret_cast<T *>(slice + L.loc);
   T *G = reinterpret_cast<T *>(slice + L.G);
   const int A = s.A;
   const T *never = reinterpret_cast<const T *>(s.ctrl + kCtrlNever);
   const size_t R = (size_t)NB * NB * (1 + S);
   constexpr int GS = GStride(NB, (int)sizeof(T));
   const int PS = PosStride(S, NB, (int)sizeof(T));
   // The factor store is read once per sweep: its lines go first from L2, so
   // that they do not push out psi and the schedule other warps are reading
   const uint64_t stream_once = EvictFirstPolicy();
   // The task's five scalars, one lane each, in one round trip
   auto scalars = [&](int64_t tt) -> int64_t {
      if (tt >= s.n_tasks) return 0;
      if (lane == 0) return s.task_pa[tt];
      if (lane == 1) return s.cell_ptr[tt];
      if (lane == 2) return s.cell_ptr[tt + 1];
      if (lane == 3) return s.lvl_ptr[tt];
      if (lane == 4) return s.lvl_ptr[tt + 1];
      return 0;
   };
   for (;;) {
      // A task is claimed only when the warp is free: a task claimed while
      // the warp still walks (and waits in) another would sit idle behind it,
      // and the tasks downstream of it would wait too (claiming even two
      // levels before the walk ends measured slower)
      int64_t t = 0;
      if (lane == 0) t = (int64_t)atomicAdd(&s.ctrl[kCtrlCounter], 1u);
      t = __shfl_sync(0xffffffffu, t, 0);
      if (t >= s.n_tasks) break;
      const int64_t v = scalars(t);
      const int32_t pa = (int32_t)__shfl_sync(0xffffffffu, v, 0);
      const int64_t off = __shfl_sync(0xffffffffu, v, 1);
      const int ncell = (int)(__shfl_sync(0xffffffffu, v, 2) - off);
      const int32_t l0 = (int32_t)__shfl_sync(0xffffffffu, v, 3);
      const int nlev = (int)(__shfl_sync(0xffffffffu, v, 4) - l0);
      const int32_t p = pa / A;
      const int a = pa - p * A;
      const int64_t base = (int64_t)p * s.P;

      // Prologue - nothing here depends on upstream values: loc gets
      // y0 = B^{-1} q, G the couplings of the gathered faces, and each lane
      // its positions' schedule
      int my_local[PL], my_lev[PL], my_ul[PL][SM];
      int32_t my_up[PL][SM];
      // The schedule, and with the store every factor load of every owned
      // position, issued before any is used (the couplings straight into
      // shared memory by cp.async); with the links in hand, the upwind values
      // of earlier tasks are loaded in the same round as q
      constexpr bool kPreloadW = CACHED && PL <= 2;  // more positions: loaded where used
      constexpr bool kPrefetch = PL <= 2;
      T W[kPreloadW ? PL : 1][NB][NB];
      T xp[kPrefetch ? PL : 1][SM][NB];
      const bool hook = (t == s.unmet_task);
#pragma unroll
      for (int k = 0; k < PL; k++) {
         const int i = lane + 32 * k;
         const bool valid = i < ncell;
         my_local[k] = valid ? s.tcell[off + i] : 0;
         my_lev[k] = valid ? s.tlev[off + i] : -1;
#pragma unroll
         for (int sl = 0; sl < SM; sl++) {
            const int32_t lk = (valid && sl < S) ? s.tlink[(off + i) * S + sl] : -1;
            my_up[k][sl] = lk >= 0 ? lk : -1;
            my_ul[k][sl] = lk <= -2 ? -2 - lk : -1;
         }
         if constexpr (CACHED) {
            if (valid) {
               const T *ft = fac + (size_t)off * R + i;
               if constexpr (kPreloadW) {
#pragma unroll
                  for (int ii = 0; ii < NB; ii++)
#pragma unroll
                     for (int j = 0; j < NB; j++) W[k][ii][j] = LoadHint(ft + (size_t)(ii * NB + j) * ncell, stream_once);
               }
#pragma unroll
               for (int e = 0; e < SM * NB * NB; e++)
                  if (e < S * NB * NB)
                     CpAsyncHint<sizeof(T)>(G + (size_t)i * PS + (e / (NB * NB)) * GS + e % (NB * NB),
                                            ft + (size_t)(NB * NB + e) * ncell, stream_once);
            }
         }
         if constexpr (kPrefetch) {
#pragma unroll
            for (int sl = 0; sl < SM; sl++)
#pragma unroll
               for (int j = 0; j < NB; j++)
                  xp[k][sl][j] = (my_up[k][sl] >= 0 && !hook)
                                    ? LoadRelaxed(psi + (int64_t)my_up[k][sl] * s.os_c + j * s.os_j + a * s.os_a)
                                    : Sentinel<T>();
         }
      }
#pragma unroll
      for (int k = 0; k < PL; k++) {
         const int i = lane + 32 * k;
         if (i >= ncell) continue;
         const int local = my_local[k];
         const int64_t c = base + local;
         T r[NB];
         if (s.aff_phi) {
            const double al = s.aff_iso ? 0.0 : *s.aff_alpha;
            const double ua = s.aff_u ? (double)static_cast<const T *>(s.aff_u)[a] : 1.0;
#pragma unroll
            for (int j = 0; j < NB; j++) {
               const int64_t node = c * NB + j;
               r[j] = s.aff_iso ? (T)(ua * s.aff_phi[node] / (s.aff_inv_volume ? (double)g.volume[c] : 1.0))
                                : (T)(al * (double)q[node * A + a] + ua * (s.aff_phi[node] - al * s.aff_rho[node]));
            }
         } else {
#pragma unroll
            for (int j = 0; j < NB; j++) r[j] = q[(c * NB + j) * A + a];
         }
         T Wk[NB][NB];
         if constexpr (kPreloadW) {
#pragma unroll
            for (int ii = 0; ii < NB; ii++)
#pragma unroll
               for (int j = 0; j < NB; j++) Wk[ii][j] = W[k][ii][j];
         } else if constexpr (CACHED) {
            const T *ft = fac + (size_t)off * R + i;
#pragma unroll
            for (int ii = 0; ii < NB; ii++)
#pragma unroll
               for (int j = 0; j < NB; j++) Wk[ii][j] = ft[(size_t)(ii * NB + j) * ncell];
         } else {
            const T om[3] = {g.omega[3 * a], g.omega[3 * a + 1], g.omega[3 * a + 2]};
            CellFactors<T, NB, F>(g, c, om, s.tmask[off + i], Wk, G + (size_t)i * PS, (size_t)GS, 1);
         }
         T y[NB];
#pragma unroll
         for (int ii = 0; ii < NB; ii++) {
            T u = T(0);
#pragma unroll
            for (int j = 0; j < NB; j++) u += Wk[ii][j] * r[j];
            y[ii] = u;
         }
         // A position whose upwind values from earlier tasks are all stored
         // already has them folded in now; the others poll at their level.
         // Either way a cell subtracts its earlier-task couplings first, in
         // slot order, then its in-task ones: the result does not depend on
         // timing.
         if constexpr (kPrefetch) {
            bool any = false, ready = true;
#pragma unroll
            for (int sl = 0; sl < SM; sl++) {
               any |= my_up[k][sl] >= 0;
#pragma unroll
               for (int j = 0; j < NB; j++) ready &= !(my_up[k][sl] >= 0 && IsSentinel(xp[k][sl][j]));
            }
            if (any && ready) {
               if constexpr (CACHED) CpAsyncWaitAll();  // this lane's couplings
#pragma unroll
               for (int sl = 0; sl < SM; sl++) {
                  if (my_up[k][sl] < 0) continue;
                  SubCoupling<T, NB>(G + (size_t)i * PS + sl * GS, xp[k][sl], y);
                  my_up[k][sl] = -1;
               }
            }
         }
#pragma unroll
         for (int ii = 0; ii < NB; ii++) loc[local * NB + ii] = y[ii];
      }
      if constexpr (CACHED) CpAsyncWaitAll();
      __syncwarp();
      bool hook_left = hook;

      // Level by level: psi_c = y0 - sum_f G_f psi(up_f), an in-task
      // neighbour from shared memory, an earlier task's polled from L2
      for (int l = 0; l < nlev; l++) {
#pragma unroll
         for (int k = 0; k < PL; k++) {
            if (my_lev[k] != l) continue;
            const int i = lane + 32 * k;
            const int local = my_local[k];
            T y[NB];
#pragma unroll
            for (int j = 0; j < NB; j++) y[j] = loc[local * NB + j];
#pragma unroll
            for (int sl = 0; sl < SM; sl++) {
               if (my_up[k][sl] < 0) continue;
               const T *src = psi + (int64_t)my_up[k][sl] * s.os_c + a * s.os_a;
               int stride = (int)s.os_j;
               if (hook_left) {
                  src = never;  // test hook: this wait can never be met
                  stride = 0;
                  hook_left = false;
               }
               T xn[NB];
               PollUpwind<T, NB>(src, stride, s, xn);
               SubCoupling<T, NB>(G + (size_t)i * PS + sl * GS, xn, y);
            }
#pragma unroll
            for (int sl = 0; sl < SM; sl++) {
               if (my_ul[k][sl] < 0) continue;
               T xn[NB];
#pragma unroll
               for (int j = 0; j < NB; j++) xn[j] = loc[my_ul[k][sl] * NB + j];
               SubCoupling<T, NB>(G + (size_t)i * PS + sl * GS, xn, y);
            }
            const int64_t c = base + local;
#pragma unroll
            for (int j = 0; j < NB; j++) {
               loc[local * NB + j] = y[j];
               StoreRelaxed(&psi[c * s.os_c + j * s.os_j + a * s.os_a], Publishable(y[j]));
            }
         }
         __syncwarp();
      }
   }
}

// ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

static int ReserveFactors(ubolt_ctx *ctx, int64_t limit);

// The wave plan and both precisions' store layouts (host work and uploads;
// no store is reserved here). Leaves wave_ok false where the mesh has an
// upwind cycle or a level or front too large for one block.
static int BuildWavePlan(ubolt_ctx *ctx, ubolt_sweep_plan *plan)
{
   HostWavePlan h;
   BuildHostWavePlan(ctx->n_cells, ctx->F, ctx->A, ctx->h_omega.data(), ctx->h_nA.data(), ctx->h_code.data(), h);
   if (!h.acyclic || h.S > std::min(4, ctx->F - 1) || h.n_slots >= 0xffff || h.max_width > 512) return UBOLT_OK;
   const int S = std::max(1, h.S);
   int dev = 0, max_smem = 0;
   cudaGetDevice(&dev);
   if (cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
      cudaGetLastError();
      return UBOLT_OK;
   }
   const int A = ctx->A;
   const int64_t total = h.lvl_base[A];
   std::vector<int32_t> lvl_ord(total);
   for (int a = 0; a < A; a++)
      for (int32_t L = h.lvl_base[a]; L < h.lvl_base[a + 1]; L++) lvl_ord[L] = a;
   int rc = 0;
   ubolt::WaveDev base;
   base.A = A;
   base.S = S;
   base.n_slots = h.n_slots;
   base.max_levels = h.max_levels;
   base.n_cells = ctx->n_cells;
   const int32_t *meta = nullptr;
   if ((rc = UploadVec(ctx, h.lvl_base, &base.lvl_base)) || (rc = UploadVec(ctx, h.lvl_pos, &base.lvl_pos)) ||
       (rc = UploadVec(ctx, lvl_ord, &base.lvl_ord)) || (rc = UploadVec(ctx, h.meta, &meta)))
      return rc;
   base.meta = reinterpret_cast<const int4 *>(meta);
   bool any = false;
   for (int which = 0; which < 2; which++) {
      WaveLayout L;
      if (!BuildWaveLayout(h, ctx->nb, which ? 4 : 8, max_smem, L)) continue;
      ubolt::WaveDev w = base;
      if ((rc = UploadVec(ctx, L.region, &w.region)) || (rc = UploadVec(ctx, L.chunk_rel, &w.chunk_rel)) ||
          (rc = UploadVec(ctx, L.ring_off, &w.ring_off)))
         return rc;
      w.front_off = L.front_off;
      w.ring_base = L.ring_base;
      w.cap = L.cap;
      w.smem = L.smem;
      plan->wave[which] = w;
      plan->wave_bytes[which] = L.store_bytes;
      any = true;
   }
   plan->wave_ok = any;
   plan->wave_threads = h.max_width <= 256 ? 256 : 512;
   plan->wave_levels = total;
   return UBOLT_OK;
}

int BuildSweepPlan(ubolt_ctx *ctx, int patch_size)
{
   if (int rc = RequireDg(ctx, "the sweep")) return rc;
   const int64_t nc = ctx->n_cells;
   int P = patch_size > 0 ? patch_size : DefaultPatch(ctx);
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
   if (h.max_inflow > ctx->F - 1) {
      delete plan;
      return SetError(UBOLT_ERR_ARG, "a cell has %d upwind faces for one ordinate (at most %d)", h.max_inflow, ctx->F - 1);
   }
   plan->total_levels = (int64_t)h.lvl.size();
   const int S = std::max(1, std::min(ctx->F - 1, (int)h.max_inflow));
   plan->slots = S;
   // The upwind link of every gathered face, in face order: the task's own
   // cell (-2 - local) or a cell of an earlier task (its id)
   std::vector<int32_t> tlink(h.tcell.size() * S, -1);
   for (int64_t t = 0; t < h.n_tasks; t++) {
      const int64_t base = (int64_t)(h.task_pa[t] / h.A) * h.P;
      for (int64_t e = h.cell_ptr[t]; e < h.cell_ptr[t + 1]; e++) {
         const int64_t c = base + h.tcell[e];
         const uint32_t mask = h.tmask[e];
         int slot = 0;
         for (int f = 0; f < ctx->F; f++) {
            const bool here = (mask >> f) & 1u, earlier = (mask >> (8 + f)) & 1u;
            if (!(here || earlier)) continue;
            const int32_t code = ctx->h_code[c * ctx->F + f];
            tlink[e * S + slot++] = earlier ? code : (int32_t)(-2 - (code - base));
         }
      }
   }
   std::vector<uint16_t> tlev(h.tcell.size(), 0);
   for (int64_t t = 0; t < h.n_tasks; t++) {
      int64_t e = h.cell_ptr[t];
      for (int32_t L = h.lvl_ptr[t]; L < h.lvl_ptr[t + 1]; L++)
         for (; e < h.cell_ptr[t] + h.lvl[L]; e++) tlev[e] = (uint16_t)(L - h.lvl_ptr[t]);
   }
   int rc = 0;
   if ((rc = UploadVec(ctx, h.task_pa, &plan->task_pa)) || (rc = UploadVec(ctx, h.dep_ptr, &plan->dep_ptr)) ||
       (rc = UploadVec(ctx, h.deps, &plan->deps)) || (rc = UploadVec(ctx, h.cell_ptr, &plan->cell_ptr)) ||
       (rc = UploadVec(ctx, h.tcell, &plan->tcell)) || (rc = UploadVec(ctx, h.tmask, &plan->tmask)) ||
       (rc = UploadVec(ctx, h.lvl_ptr, &plan->lvl_ptr)) || (rc = UploadVec(ctx, h.lvl, &plan->lvl)) ||
       (rc = UploadVec(ctx, tlink, &plan->tlink)) || (rc = UploadVec(ctx, tlev, &plan->tlev))) {
      delete plan;
      return rc;
   }
   void *p = nullptr;
   if ((rc = CtxAlloc(ctx, kCtrlWords * sizeof(uint32_t), &p))) { delete plan; return rc; }
   plan->ctrl = static_cast<uint32_t *>(p);
   cudaMemset(plan->ctrl, 0, kCtrlWords * sizeof(uint32_t));
   cudaMemset(plan->ctrl + kCtrlNever, 0xff, 2 * sizeof(uint32_t));
   if ((rc = BuildWavePlan(ctx, plan))) { delete plan; return rc; }
   if (ctx->sweep) {
      plan->fac_limit = ctx->sweep->fac_limit;
      plan->kernel_mode = ctx->sweep->kernel_mode;
   }
   if (plan->kernel_mode == UBOLT_SWEEP_WAVE && !plan->wave_ok) plan->kernel_mode = UBOLT_SWEEP_AUTO;
   delete ctx->sweep;
   ctx->sweep = plan;
   if ((rc = CudaCheck(cudaDeviceSynchronize(), "sweep plan"))) return rc;
   return ReserveFactors(ctx, plan->fac_limit);
}

static SweepDev DevPlan(const ubolt_sweep_plan *pl)
{
   SweepDev s;
   s.P = pl->P;
   s.A = pl->A;
   s.n_tasks = pl->n_tasks;
   s.task_pa = pl->task_pa;
   s.cell_ptr = pl->cell_ptr;
   s.tcell = pl->tcell;
   s.tmask = pl->tmask;
   s.tlev = pl->tlev;
   s.tlink = pl->tlink;
   s.lvl_ptr = pl->lvl_ptr;
   s.lvl = pl->lvl;
   s.ctrl = pl->ctrl;
   s.spin_limit = pl->spin_limit;
   s.unmet_task = -1;
   s.slots = pl->slots;
   s.aff_alpha = s.aff_phi = s.aff_rho = nullptr;
   s.aff_u = nullptr;
   s.aff_iso = 0;
   s.aff_inv_volume = 0;
   return s;
}

// psi's layout for the task kernel
static void SetLayout(SweepDev &s, const ubolt_ctx *ctx, bool ordinate_major)
{
   const int64_t nb = ctx->nb, A = ctx->A;
   if (ordinate_major) {
      s.os_c = nb;
      s.os_j = 1;
      s.os_a = ctx->n_cells * nb;
   } else {
      s.os_c = nb * A;
      s.os_j = A;
      s.os_a = 1;
   }
}

// Bytes of the factor store for one precision
static int64_t FactorBytes(const ubolt_ctx *ctx, const ubolt_sweep_plan *pl, size_t elem)
{
   return (int64_t)ctx->n_cells * ctx->A * ctx->nb * ctx->nb * (1 + pl->slots) * (int64_t)elem;
}

// Reserve the factor stores - at set-up (plan build, or an explicit limit),
// never inside a sweep. limit < 0: each store that fits, FP32 first, within
// half the free device memory at that moment (at most 96 GiB); 0: none;
// otherwise the byte limit for both together. A store not reserved means
// the sweep computes its factors as it goes: the result is the same.
// The automatic choice. The wave kernel runs one block per ordinate, and a
// block's level costs about one L1 wavefront per scattered q and psi word:
// on one B200 it beat the task kernel only on small problems (64^2 quads
// DG0 S4: 0.078 against 0.110 ms) and lost from 128^2 triangles DG1 S8
// (0.77 against 0.39 ms) up to 256^2 at S16 (3.78 against 3.71 ms). So it is
// taken up to 2^17 cell-ordinates.
static bool WavePreferred(const ubolt_ctx *ctx) { return ctx->n_cells * (int64_t)ctx->A <= ((int64_t)1 << 17); }

static int ReserveFactors(ubolt_ctx *ctx, int64_t limit)
{
   ubolt_sweep_plan *pl = ctx->sweep;
   if (pl->fac[0] || pl->fac[1]) cudaDeviceSynchronize();
   for (int which = 0; which < 2; which++) {
      if (pl->fac[which]) cudaFree(pl->fac[which]);
      pl->fac[which] = nullptr;
      pl->fac_epoch[which] = 0;
   }
   if (limit < 0) {
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
         cudaGetLastError();
         return UBOLT_OK;
      }
      limit = std::min<int64_t>((int64_t)(free_b / 2), (int64_t)96 << 30);
   }
   int64_t left = limit;
   for (int which : {1, 0}) {
      // The wave kernel where it applies and is chosen (its store is in wave
      // order), else the task kernel's
      const bool wave = pl->wave[which].smem > 0 &&
                        (pl->kernel_mode == UBOLT_SWEEP_WAVE || (pl->kernel_mode == UBOLT_SWEEP_AUTO && WavePreferred(ctx)));
      pl->fac_wave[which] = false;
      const int64_t bytes = wave ? pl->wave_bytes[which] : FactorBytes(ctx, pl, which ? 4 : 8);
      if (bytes > left) continue;
      void *p = nullptr;
      if (cudaMalloc(&p, (size_t)bytes) != cudaSuccess) {
         cudaGetLastError();
         continue;
      }
      pl->fac[which] = p;
      pl->fac_wave[which] = wave;
      left -= bytes;
   }
   return UBOLT_OK;
}

// The factor store for precision T, rebuilt by a kernel (no allocation) for
// the current group: ubolt_set_group starts a new one. nullptr where none
// is reserved: the sweep then computes its factors as it goes.
template <typename T, int NB, int F>
static T *EnsureFactors(ubolt_ctx *ctx, cudaStream_t st)
{
   ubolt_sweep_plan *pl = ctx->sweep;
   const int which = sizeof(T) == 8 ? 0 : 1;
   if (!pl->fac[which]) return nullptr;
   if (pl->fac_epoch[which] == ctx->group_epoch) return static_cast<T *>(pl->fac[which]);
   if (pl->fac_wave[which]) {
      if (WaveFactors(ctx, pl->wave[which], pl->fac[which], (int)sizeof(T), st, pl->wave_levels)) return nullptr;
      pl->fac_epoch[which] = ctx->group_epoch;
      return static_cast<T *>(pl->fac[which]);
   }
   int n_sm = 0, dev = 0;
   cudaGetDevice(&dev);
   cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
   const int64_t grid = std::min<int64_t>((pl->n_tasks + 3) / 4, (int64_t)n_sm * 16);
   FactorKernel<T, NB, F><<<(int)grid, 128, 0, st>>>(ctx->geom<T>(), DevPlan(pl), static_cast<T *>(pl->fac[which]));
   if (CheckLaunch("sweep factors")) return nullptr;
   pl->fac_epoch[which] = ctx->group_epoch;
   return static_cast<T *>(pl->fac[which]);
}

template <typename T, int NB, int F>
static int LaunchSweep(ubolt_ctx *ctx, const T *q, T *psi, cudaStream_t st, const SweepDev *affine = nullptr,
                       bool ordinate_major = false)
{
   ubolt_sweep_plan *pl = ctx->sweep;
   const int which = sizeof(T) == 8 ? 0 : 1;
   const T *fac = EnsureFactors<T, NB, F>(ctx, st);
   if (pl->fac_wave[which]) {
      // One block per ordinate over the store in wave order (no sentinel fill)
      if (!fac) return UBOLT_ERR_CUDA;  // the failed launch set the message
      if (ordinate_major) return SetError(UBOLT_ERR_STATE, "the wave sweep writes the row layout only");
      if (affine && affine->aff_inv_volume) return SetError(UBOLT_ERR_STATE, "the wave sweep takes no 1 / V source");
      WaveDev w = pl->wave[which];
      w.ctrl = pl->ctrl;
      w.spin_limit = pl->spin_limit;
      w.unmet_level = pl->unmet_level;
      pl->unmet_level = -1;
      pl->unmet_task = -1;
      pl->grid = ctx->A;
      WaveInput in;
      if (affine) {
         in.alpha = affine->aff_alpha;
         in.phi = affine->aff_phi;
         in.rho = affine->aff_rho;
         in.u = affine->aff_u;
         in.iso = affine->aff_iso;
      }
      return WaveSweep(ctx, w, q, psi, fac, (int)sizeof(T), affine ? &in : nullptr, pl->wave_threads, st);
   }
   const int threads = 32 * pl->warps_per_block;
   const size_t smem = (size_t)pl->warps_per_block * SweepSlice(pl->P, pl->slots, NB, (int)sizeof(T)).bytes;
   auto kern = fac ? (pl->P <= 32 ? SweepKernel<T, NB, F, 1, true>
                                  : pl->P <= 64 ? SweepKernel<T, NB, F, 2, true> : SweepKernel<T, NB, F, 8, true>)
                   : (pl->P <= 32 ? SweepKernel<T, NB, F, 1, false>
                                  : pl->P <= 64 ? SweepKernel<T, NB, F, 2, false> : SweepKernel<T, NB, F, 8, false>);
   if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
   int per_sm = 0, n_sm = 0, dev = 0;
   cudaGetDevice(&dev);
   cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
   // At most 32 warps per SM: beyond the throughput the wavefront can use,
   // more resident warps only take tasks early and wait
   per_sm = std::min(per_sm, kSweepBlocksPerSm);
   const int64_t want = (pl->n_tasks + pl->warps_per_block - 1) / pl->warps_per_block;
   const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::max(per_sm, 1) * n_sm, want));
   pl->grid = grid;
   SweepDev s = DevPlan(pl);
   SetLayout(s, ctx, ordinate_major);
   if (affine) {
      s.aff_alpha = affine->aff_alpha;
      s.aff_phi = affine->aff_phi;
      s.aff_rho = affine->aff_rho;
      s.aff_u = affine->aff_u;
      s.aff_iso = affine->aff_iso;
      s.aff_inv_volume = affine->aff_inv_volume;
   }
   s.unmet_task = pl->unmet_task;
   pl->unmet_task = -1;
   cudaMemsetAsync(pl->ctrl + kCtrlCounter, 0, sizeof(uint32_t), st);  // task counter; the error flag stays sticky
   // Every psi value starts as the sentinel: "not yet stored by its task"
   cudaMemsetAsync(psi, 0xff, (size_t)ctx->n_cells * NB * ctx->A * sizeof(T), st);
   kern<<<grid, threads, smem, st>>>(ctx->geom<T>(), s, q, psi, fac);
   return CheckLaunch("sweep");
}

template <typename T>
int Sweep(ubolt_ctx *ctx, const T *q, T *psi, void *stream, bool ordinate_major)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!ctx->sweep && (rc = BuildSweepPlan(ctx, 0))) return rc;
   if (!q || !psi || (const void *)q == (const void *)psi)
      return SetError(UBOLT_ERR_ARG, "sweep: q and psi must be distinct device arrays");
   UBOLT_DISPATCH(ctx->nb, ctx->F,
                  return (LaunchSweep<T, NB_, F_>(ctx, q, psi, (cudaStream_t)stream, nullptr, ordinate_major)));
   return SetError(UBOLT_ERR_STATE, "no sweep kernel for this shape");
}
template <typename T>
int Sweep(ubolt_ctx *ctx, const T *q, T *psi, void *stream)
{
   return Sweep<T>(ctx, q, psi, stream, false);
}

// True where the sweep is L^{-1} exactly: a plan with no lagged coupling and
// no reflective side (reflective inflow is lagged)
bool SweepIsExact(ubolt_ctx *ctx)
{
   if (!ctx->sweep && BuildSweepPlan(ctx, 0)) return false;
   return ctx->sweep->n_lagged == 0 && !ctx->has_reflect;
}

// psi = L^{-1} (alpha r0 + E_u (phi - alpha rho)) with the input formed as
// the sweep reads it (u = 1, or u_a = u[a]); alpha, phi, rho on the device.
// r0 == nullptr: r0 is isotropic, r0 = E_u rho, and the input is E_u phi.
// inv_volume (r0 == nullptr only): the input is u_a phi(node) / V(cell).
template <typename T>
int SweepAffine(ubolt_ctx *ctx, const T *r0, const double *alpha, const double *phi, const double *rho, const T *u,
                T *psi, void *stream, bool ordinate_major, bool inv_volume)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!ctx->sweep && (rc = BuildSweepPlan(ctx, 0))) return rc;
   if (inv_volume && r0) return SetError(UBOLT_ERR_ARG, "sweep: the 1 / V source is isotropic only");
   SweepDev aff{};
   aff.aff_alpha = alpha;
   aff.aff_phi = phi;
   aff.aff_rho = rho;
   aff.aff_u = u;
   aff.aff_iso = r0 == nullptr;
   aff.aff_inv_volume = inv_volume;
   UBOLT_DISPATCH(ctx->nb, ctx->F,
                  return (LaunchSweep<T, NB_, F_>(ctx, r0, psi, (cudaStream_t)stream, &aff, ordinate_major)));
   return SetError(UBOLT_ERR_STATE, "no sweep kernel for this shape");
}

// True where the next sweep in precision T runs the task kernel (which can
// write psi ordinate-major); false where the wave kernel runs
template <typename T>
bool SweepWritesOrdinateMajor(ubolt_ctx *ctx)
{
   if (!ctx->sweep && BuildSweepPlan(ctx, 0)) return false;
   const int which = sizeof(T) == 8 ? 0 : 1;
   return !(ctx->sweep->fac[which] && ctx->sweep->fac_wave[which]);
}

template int SweepAffine<double>(ubolt_ctx *, const double *, const double *, const double *, const double *,
                                 const double *, double *, void *, bool, bool);
template int SweepAffine<float>(ubolt_ctx *, const float *, const double *, const double *, const double *,
                                const float *, float *, void *, bool, bool);
template int Sweep<double>(ubolt_ctx *, const double *, double *, void *, bool);
template int Sweep<float>(ubolt_ctx *, const float *, float *, void *, bool);
template bool SweepWritesOrdinateMajor<double>(ubolt_ctx *);
template bool SweepWritesOrdinateMajor<float>(ubolt_ctx *);
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

extern "C" int ubolt_sweep_set_kernel(ubolt_ctx *ctx, int kernel)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (kernel < UBOLT_SWEEP_AUTO || kernel > UBOLT_SWEEP_WAVE) return SetError(UBOLT_ERR_ARG, "sweep kernel %d", kernel);
   if (!ctx->sweep && (rc = BuildSweepPlan(ctx, 0))) return rc;
   ubolt_sweep_plan *pl = ctx->sweep;
   if (kernel == UBOLT_SWEEP_WAVE && !pl->wave_ok)
      return SetError(UBOLT_ERR_STATE, "the wave sweep does not apply here (an upwind cycle, or a level or front too "
                                       "large for one block)");
   if (kernel == pl->kernel_mode) return UBOLT_OK;
   pl->kernel_mode = kernel;
   // The stores' layout follows the kernel: reserved again, rebuilt by the next sweep
   return ReserveFactors(ctx, pl->fac_limit);
}

extern "C" int ubolt_sweep(ubolt_ctx *ctx, const double *q, double *psi, void *stream)
{
   return Sweep<double>(ctx, q, psi, stream);
}

extern "C" int ubolt_sweep_f32(ubolt_ctx *ctx, const float *q, float *psi, void *stream)
{
   return Sweep<float>(ctx, q, psi, stream);
}

template <typename T>
static int SweepIso(ubolt_ctx *ctx, const double *phi, const T *u, T *psi, int ordinate_major, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!phi || !psi) return SetError(UBOLT_ERR_ARG, "sweep_iso: NULL array");
   if (ordinate_major && !SweepWritesOrdinateMajor<T>(ctx))
      return SetError(UBOLT_ERR_STATE, "sweep_iso: the wave kernel runs here, and it writes the row layout only");
   return SweepAffine<T>(ctx, nullptr, nullptr, phi, nullptr, u, psi, stream, ordinate_major != 0, false);
}

extern "C" int ubolt_sweep_iso(ubolt_ctx *ctx, const double *phi, const double *u, double *psi, int ordinate_major,
                               void *stream)
{
   return SweepIso<double>(ctx, phi, u, psi, ordinate_major, stream);
}

extern "C" int ubolt_sweep_iso_f32(ubolt_ctx *ctx, const double *phi, const float *u, float *psi, int ordinate_major,
                                   void *stream)
{
   return SweepIso<float>(ctx, phi, u, psi, ordinate_major, stream);
}

extern "C" int ubolt_sweep_set_factor_limit(ubolt_ctx *ctx, int64_t bytes)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!ctx->sweep) {
      if ((rc = BuildSweepPlan(ctx, 0))) return rc;
   }
   ctx->sweep->fac_limit = bytes;
   return ReserveFactors(ctx, bytes);
}

extern "C" int ubolt_sweep_status(ubolt_ctx *ctx, ubolt_sweep_info *info, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!ctx->sweep) return SetError(UBOLT_ERR_STATE, "no sweep plan");
   ubolt_sweep_plan *pl = ctx->sweep;
   uint32_t h[2] = {0, 0};  // error flag, timeout count
   cudaStream_t s = (cudaStream_t)stream;
   cudaMemcpyAsync(h, pl->ctrl + kCtrlError, sizeof h, cudaMemcpyDeviceToHost, s);
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
      info->timeouts = h[1];
      info->kernel = (pl->fac[0] && pl->fac_wave[0]) ? UBOLT_SWEEP_WAVE : UBOLT_SWEEP_TASKS;
      info->factor_bytes = 0;
      info->factor_bytes_fp64 = 0;
      for (int which = 0; which < 2; which++)
         if (pl->fac[which]) {
            const int64_t b = pl->fac_wave[which] ? pl->wave_bytes[which] : FactorBytes(ctx, pl, which ? 4 : 8);
            info->factor_bytes += b;
            if (which == 0) info->factor_bytes_fp64 = b;
         }
   }
   if (h[0]) {
      cudaMemsetAsync(pl->ctrl + kCtrlError, 0, 2 * sizeof(uint32_t), s);
      cudaStreamSynchronize(s);
      return SetError(UBOLT_ERR_TIMEOUT, "a sweep wait gave up (%u timeouts); its result is not valid", h[1]);
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
   pl->unmet_level = -1;
   if (make_one_wait_unmet && pl->fac[0] && pl->fac_wave[0]) {
      // The wave kernel runs the next FP64 sweep: ordinate 0's first level
      // waits for a copy never issued
      pl->unmet_level = 0;
      return UBOLT_OK;
   }
   if (make_one_wait_unmet) {
      // The first task that has an upstream task polls, for its first
      // upwind value, a word that no task of the sweep stores
      std::vector<int32_t> dp(pl->n_tasks + 1);
      if ((rc = CudaCheck(cudaMemcpy(dp.data(), pl->dep_ptr, dp.size() * sizeof(int32_t), cudaMemcpyDeviceToHost),
                          "sweep_test_wait")))
         return rc;
      for (int64_t t = 0; t < pl->n_tasks; t++)
         if (dp[t + 1] > dp[t]) { pl->unmet_task = t; break; }
      if (pl->unmet_task < 0) return SetError(UBOLT_ERR_STATE, "no task of this plan waits on another");
   }
   return UBOLT_OK;
}
