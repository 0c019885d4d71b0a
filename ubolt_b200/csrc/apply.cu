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
// Forward (L - S and L): a block holds K whole cells, one thread per (cell,
// AP consecutive ordinates), AP = 16 bytes / element (2 in FP64, 4 in FP32)
// where the ordinate count and the vectors' alignment allow, else 1. The
// block first stages in shared memory, with asynchronous copies all in
// flight at once: its cells' rows (one contiguous range of x), each cell's
// class record (per face: normal and both face matrices, 16-byte parts) and
// each thread's upwind runs (the neighbour's rows at its ordinates). After
// one wait everything is read from shared memory, so a block costs two
// rounds of memory latency (face codes and class ids, then the copies). The
// scatter's node moments are summed from the staged rows by four lanes per
// node and two shuffles, in a fixed order. Every face is folded in without a
// branch on the sign of s = Omega . nA: the outflow part max(s, 0) face_own x
// and the inflow part min(s, 0) face_up x_up (x_up the neighbour, the
// mirrored ordinate of this cell on a reflective side, zero on a vacuum side).
//
// Adjoint ((L - S)^T): a column also needs the NEIGHBOUR's shape data (its
// face slot and matrix for the shared face), so that kernel gathers class
// data straight from L1/L2, one thread per (cell, ordinate).
#include "cg.h"
#include "ctx.h"

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

namespace ubolt {

enum { kFull = 0, kUnscattered = 1, kAdjoint = 2 };

template <typename T>
__device__ __forceinline__ T WarpSum(T v)
{
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

// N consecutive values from an address aligned to 16 bytes (N * sizeof(T)
// a multiple of 16), to 8 bytes (8), or element-aligned
template <typename T, int N>
__device__ __forceinline__ void LoadRun(const T *__restrict__ p, T v[N])
{
   constexpr int B = (int)sizeof(T) * N;
   if constexpr (B % 16 == 0) {
#pragma unroll
      for (int u = 0; u < B / 16; u++) {
         const int4 w = __ldg(reinterpret_cast<const int4 *>(p) + u);
         memcpy(&v[u * (16 / (int)sizeof(T))], &w, 16);
      }
   } else if constexpr (B == 8 && sizeof(T) == 4) {
      const int2 w = __ldg(reinterpret_cast<const int2 *>(p));
      memcpy(v, &w, 8);
   } else {
#pragma unroll
      for (int i = 0; i < N; i++) v[i] = __ldg(p + i);
   }
}

template <typename T, int N>
__device__ __forceinline__ void StoreRun(T *__restrict__ p, const T v[N])
{
   constexpr int B = (int)sizeof(T) * N;
   if constexpr (B % 16 == 0) {
#pragma unroll
      for (int u = 0; u < B / 16; u++) {
         int4 w;
         memcpy(&w, &v[u * (16 / (int)sizeof(T))], 16);
         __stcs(reinterpret_cast<int4 *>(p) + u, w);
      }
   } else {
#pragma unroll
      for (int i = 0; i < N; i++) p[i] = v[i];
   }
}

// N consecutive values from shared memory, 16-byte aligned when N *
// sizeof(T) is a multiple of 16
template <typename T, int N>
__device__ __forceinline__ void LoadShared(const T *p, T v[N])
{
   if constexpr ((int)sizeof(T) * N % 16 == 0) {
#pragma unroll
      for (int u = 0; u < (int)sizeof(T) * N / 16; u++) {
         const int4 w = reinterpret_cast<const int4 *>(p)[u];
         memcpy(&v[u * (16 / (int)sizeof(T))], &w, 16);
      }
   } else {
#pragma unroll
      for (int i = 0; i < N; i++) v[i] = p[i];
   }
}

// One run of CU bytes (4, 8, 16 or a multiple of 16), both addresses aligned
// to min(CU, 16)
template <int CU>
__device__ __forceinline__ void CpAsyncRun(void *dst, const void *src)
{
   if constexpr (CU <= 16) {
      CpAsync<CU>(dst, src);
   } else {
#pragma unroll
      for (int u = 0; u < CU / 16; u++)
         CpAsync<16>(static_cast<unsigned char *>(dst) + 16 * u, static_cast<const unsigned char *>(src) + 16 * u);
   }
}

// Upwind runs staged per thread: every face at once where F * NB <= 12,
// else a ring of two faces fetched ahead of the walk over the faces (DG1
// tets and hexes, whose F * NB runs would crowd the SM's shared memory)
template <int NB, int F>
constexpr int UpSlots() { return F * NB > 12 ? 2 : F; }

// Shared memory of one apply block, in elements of T: the cells' class
// records [K][L.size], the threads' upwind runs [slots][NB][threads][AP]
// (thread-fastest, so a warp's 16-byte reads hit distinct banks), the
// cells' own rows [K][NB][A], then for the scatter the node moments
// [K][NB], sigma_s / W per cell [K] and the ordinate weights [A]
template <typename T, int NB, int F, int AP>
__host__ __device__ constexpr size_t ApplySmemElems(int K, int threads, int A, bool rev = false)
{
   return (size_t)K * RecordLayout(NB, F, (int)sizeof(T)).size + (size_t)threads * UpSlots<NB, F>() * NB * AP +
          (size_t)K * NB * A +
          (size_t)K * NB + (size_t)K + (size_t)A + (rev ? (size_t)F * threads : 0);
}

// The register cap, as 256-thread blocks per SM: three (at most 80
// registers, so 768 threads fit whatever block size the launch picks), two
// where the four basis functions' rows of AP > 1 ordinates need more
template <typename T, int NB, int AP>
constexpr int ApplyMinBlocks() { return (NB == 4 && AP > 1) ? 2 : 3; }

// REV: the transpose (L - S)^T = L^T - S^T, L^T as the reversed-angle
// operator. (V L)^T = P (V L) P (V the cell volume on every row, P the swap
// of each ordinate with its opposite) gives L^T x = P V L (P V^{-1} x): the
// thread applies L, as above, to z = P V^{-1} x and writes P V of the
// result. Its own terms take x at the opposite ordinates and need no
// scaling (V_c / V_c); an interior inflow term takes the neighbour's x at
// the opposite ordinates times V_c / V_neighbour. The scatter puts its
// weight on the row: (S^T x)(a) = sigma_s / W w_a sum_b x(b). It needs every
// aligned run of AP ordinates to map to a reversed aligned run under the
// opposite (the launcher checks; the column kernel below serves otherwise).
template <typename T, int NB, int F, int AP, bool SCATTER, bool REV = false>
__global__ void __launch_bounds__(256, ApplyMinBlocks<T, NB, AP>()) ApplyKernel(const DevGeom<T> g, const T *__restrict__ x, T *__restrict__ y, int K)
{
   constexpr RecordLayout L(NB, F, (int)sizeof(T));
   constexpr int CU = AP * (int)sizeof(T);  // bytes of one thread's run of a row
   constexpr int RU = L.size * (int)sizeof(T) / 16;
   constexpr int XS = UpSlots<NB, F>();
   constexpr bool kRing = XS < F;
   extern __shared__ __align__(16) unsigned char smem_raw[];
   const int A = g.A, QA = A / AP;
   T *recs = reinterpret_cast<T *>(smem_raw);
   T *xup = recs + K * L.size;
   T *xs = xup + (size_t)blockDim.x * XS * NB * AP;
   T *mom = xs + K * NB * A;  // scatter: [K][NB] sigma_s / W sum_b w_b x(node, b)
   T *ssw = mom + K * NB;     // scatter: [K] sigma_s / W
   T *ws = ssw + K;           // scatter: [A] the weights
   T *rat = ws + A;           // REV: [F][threads] V_c / V_neighbour per face
   const int t = threadIdx.x;
   const int k = t / QA;
   const int q = t - k * QA;
   const int a0 = q * AP;
   // The run of x read for this cell and its neighbours, and of y written:
   // this thread's ordinates, or (REV) their opposites, the same run reversed
   const int ar0 = REV ? g.opp[a0 + AP - 1] : a0;
   const int64_t c0 = (int64_t)blockIdx.x * K;
   const int64_t c = c0 + k;
   const int kc = (int)min((int64_t)K, g.n_cells - c0);
   const bool live = k < kc;

   // Stage: the block's own rows (one contiguous range), each cell's class
   // record and this thread's upwind runs, all in flight at once (with the
   // ring, the first two faces' runs, each in a commit group of its own).
   // Per face 4 bits of fcode: 8 for an interior face, else the boundary side.
   unsigned fcode = 0;
   {
      const int nu = kc * NB * A * (int)sizeof(T) / CU;
      const unsigned char *src = reinterpret_cast<const unsigned char *>(x + c0 * NB * A);
      for (int u = t; u < nu; u += blockDim.x) CpAsyncRun<CU>(reinterpret_cast<unsigned char *>(xs) + u * CU, src + u * CU);
   }
   if (live) {
      const T *rec = g.rec + (int64_t)g.cls[c] * L.size;
      for (int u = q; u < RU; u += QA) CpAsync<16>(recs + k * L.size + u * (16 / (int)sizeof(T)), rec + u * (16 / (int)sizeof(T)));
      if constexpr (kRing) CpAsyncCommit();
      T vc = T(0);
      if constexpr (REV) vc = g.volume[c];
#pragma unroll
      for (int f = 0; f < F; f++) {
         const int32_t cf = g.code[c * F + f];
         if (FaceInterior(cf)) {
            fcode |= 8u << (4 * f);
            if constexpr (REV) rat[f * (int)blockDim.x + t] = vc * g.inv_vol[g.cls[cf]];
            if (!kRing || f < XS) {
#pragma unroll
               for (int j = 0; j < NB; j++)
                  CpAsyncRun<CU>(xup + ((f * NB + j) * (int)blockDim.x + t) * AP, x + ((int64_t)cf * NB + j) * A + ar0);
            }
         } else {
            fcode |= (unsigned)FaceSide(cf) << (4 * f);
         }
         if (kRing && f < XS) CpAsyncCommit();
      }
   }
   T om[3 * AP];
   T sig_t = T(0);
   if (live) {
      LoadRun<T, 3 * AP>(g.omega + 3 * a0, om);
      sig_t = g.sigma_t[c];
      if (SCATTER && q == 0) ssw[k] = g.sigma_s[c] * g.inv_sum_weights;
   }
   if constexpr (SCATTER)
      for (int b = t; b < A; b += blockDim.x) ws[b] = g.w[b];
   // The shared rows and records are in; with the ring, a live thread's two
   // face groups may still be in flight (a thread without a cell committed
   // no group, so it waits for all of its copies)
   if (kRing && live) CpAsyncWaitGroup<XS>();
   else CpAsyncWaitAll();
   __syncthreads();

   if constexpr (SCATTER) {
      // sigma_s / W sum_b w_b x(node, b) from the staged rows: four lanes
      // per node, each a fixed quarter of the ordinates, then two shuffles.
      // The loop bound is the same for every thread (the shuffles need the
      // whole warp).
      constexpr int G = 4;
      const int nodes = kc * NB;
      for (int base = 0; base < nodes * G; base += blockDim.x) {
         const int idx = base + t;
         const int n = idx / G, part = idx - (idx / G) * G;
         T m = T(0);
         if (n < nodes)
            for (int b = part; b < A; b += G) m += (REV ? T(1) : ws[b]) * xs[n * A + b];
         m += __shfl_xor_sync(0xffffffffu, m, 1);
         m += __shfl_xor_sync(0xffffffffu, m, 2);
         if (part == 0 && n < nodes) mom[n] = m * ssw[n / NB];
      }
   }

   T acc[AP][NB];
   if (live) {
      const T *r = recs + k * L.size;
      const T *xk = xs + k * NB * A;
      constexpr int TS = L.size - L.tail;  // grad phi and 1 / V
      T tl[TS];
      LoadShared<T, TS>(r + L.tail, tl);
      T xo[AP][NB];
#pragma unroll
      for (int j = 0; j < NB; j++) {
         T v[AP];
         LoadShared<T, AP>(xk + j * A + ar0, v);
#pragma unroll
         for (int p = 0; p < AP; p++) xo[p][j] = REV ? v[AP - 1 - p] : v[p];
      }
      // Removal, and the volume term -(Omega . grad phi_i) x(c, 0, a) for i > 0
#pragma unroll
      for (int p = 0; p < AP; p++)
#pragma unroll
         for (int i = 0; i < NB; i++) acc[p][i] = sig_t * xo[p][i];
      if constexpr (NB > 1) {
#pragma unroll
         for (int i = 1; i < NB; i++)
#pragma unroll
            for (int p = 0; p < AP; p++) acc[p][i] -= Dot3(om + 3 * p, tl + 3 * i) * xo[p][0];
      }
      // Each face without a branch on the sign of s = Omega . nA: outflow
      // max(s, 0) face_own x, inflow min(s, 0) face_up x_up, x_up the
      // neighbour, this cell's mirrored ordinate on a reflective side, zero
      // on a vacuum side (DG0: the same with 1 / V for both matrices). The
      // faces one at a time: unrolled, their reads would be hoisted together
      // and spill
#pragma unroll 1
      for (int f = 0; f < F; f++) {
         const unsigned fc = (fcode >> (4 * f)) & 15u;
         T na[4];
         LoadShared<T, 4>(r + L.nA(f), na);
         T xn[AP][NB];
         const int slot = kRing ? (f & 1) : f;
         if constexpr (kRing) {
            // This face's group is in once at most the next face's is pending
            if (f + 1 < F) CpAsyncWaitGroup<1>();
            else CpAsyncWaitGroup<0>();
         }
         if (fc & 8u) {
#pragma unroll
            for (int j = 0; j < NB; j++) {
               T v[AP];
               LoadShared<T, AP>(xup + ((slot * NB + j) * (int)blockDim.x + t) * AP, v);
#pragma unroll
               for (int p = 0; p < AP; p++) xn[p][j] = REV ? v[AP - 1 - p] : v[p];
            }
         } else {
            const int side = (int)fc;
            const bool refl = g.side_bc[side] == UBOLT_BC_REFLECT;
#pragma unroll
            for (int p = 0; p < AP; p++) {
               int ar = refl ? g.refl[(side >> 1) * A + a0 + p] : 0;
               if (REV && refl) ar = g.opp[ar];
#pragma unroll
               for (int j = 0; j < NB; j++) xn[p][j] = refl ? xk[j * A + ar] : T(0);
            }
         }
         T sp[AP], sm[AP];
         const T ratio = (REV && (fc & 8u)) ? rat[f * (int)blockDim.x + t] : T(1);
#pragma unroll
         for (int p = 0; p < AP; p++) {
            const T s = Dot3(om + 3 * p, na);
            sp[p] = fmax(s, T(0));
            sm[p] = fmin(s, T(0));
            if constexpr (REV) sm[p] *= ratio;
         }
         if constexpr (NB == 1) {
#pragma unroll
            for (int p = 0; p < AP; p++) acc[p][0] += (sp[p] * xo[p][0] + sm[p] * xn[p][0]) * tl[0];
         } else {
            {
               T m[L.fm];
               LoadShared<T, L.fm>(r + L.fown(f), m);
#pragma unroll
               for (int p = 0; p < AP; p++)
#pragma unroll
                  for (int i = 0; i < NB; i++) {
                     T u = T(0);
#pragma unroll
                     for (int j = 0; j < NB; j++) u += m[i * NB + j] * xo[p][j];
                     acc[p][i] += sp[p] * u;
                  }
            }
            {
               T m[L.fm];
               LoadShared<T, L.fm>(r + L.fup(f), m);
#pragma unroll
               for (int p = 0; p < AP; p++)
#pragma unroll
                  for (int i = 0; i < NB; i++) {
                     T v = T(0);
#pragma unroll
                     for (int j = 0; j < NB; j++) v += m[i * NB + j] * xn[p][j];
                     acc[p][i] += sm[p] * v;
                  }
            }
         }
         if constexpr (kRing) {
            // This face's runs are used: fetch face f + 2's into the slot
            if (f + XS < F) {
               const int32_t cf = g.code[c * F + f + XS];
               if (FaceInterior(cf)) {
#pragma unroll
                  for (int j = 0; j < NB; j++)
                     CpAsyncRun<CU>(xup + ((slot * NB + j) * (int)blockDim.x + t) * AP, x + ((int64_t)cf * NB + j) * A + ar0);
               }
            }
            CpAsyncCommit();
         }
      }
   }
   if constexpr (SCATTER) {
      __syncthreads();
      if (live) {
#pragma unroll
         for (int p = 0; p < AP; p++) {
            const T wa = REV ? ws[a0 + p] : T(1);  // the transpose: w of the row's own ordinate (w_opp = w)
#pragma unroll
            for (int i = 0; i < NB; i++) acc[p][i] -= wa * mom[k * NB + i];
         }
      }
   }
   if (!live) return;
#pragma unroll
   for (int i = 0; i < NB; i++) {
      T v[AP];
#pragma unroll
      for (int p = 0; p < AP; p++) v[REV ? AP - 1 - p : p] = acc[p][i];
      StoreRun<T, AP>(y + (c * NB + i) * A + ar0, v);
   }
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

// Cells per block for QA threads per cell: the most live threads resident
// per SM for this kernel (registers and shared memory), then the fewest idle
// lanes, then the most blocks per SM (more blocks stage their copies
// independently). Cached per kernel and QA.
template <typename Kern, typename Smem>
static int ApplyCells(Kern kern, int QA, Smem smem_of)
{
   static std::mutex mu;
   static std::map<std::pair<const void *, int>, int> memo;
   const auto key = std::make_pair(reinterpret_cast<const void *>(kern), QA);
   {
      std::lock_guard<std::mutex> lk(mu);
      auto it = memo.find(key);
      if (it != memo.end()) return it->second;
   }
   int dev = 0, smem_max = 48 * 1024;
   cudaGetDevice(&dev);
   cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
   int best = 1, best_blocks = 0;
   long best_live = -1;
   double best_idle = 2.0;
   for (int K = 1; K * QA <= 256; K++) {
      const int thr = (K * QA + 31) / 32 * 32;
      const size_t smem = smem_of(K, thr);
      if (smem > (size_t)smem_max) break;  // grows with K
      int per_sm = 0;
      if (smem > 48 * 1024 &&
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
         cudaGetLastError();
         break;
      }
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, thr, smem) != cudaSuccess) {
         cudaGetLastError();
         per_sm = 0;
      }
      const long live = (long)per_sm * K * QA;
      const double idle = (double)(thr - K * QA) / thr;
      if (live > best_live || (live == best_live && (idle < best_idle - 1e-9 ||
                                                     (idle < best_idle + 1e-9 && per_sm > best_blocks)))) {
         best = K;
         best_live = live;
         best_idle = idle;
         best_blocks = per_sm;
      }
   }
   std::lock_guard<std::mutex> lk(mu);
   memo[key] = best;
   return best;
}

// True where the opposite maps every aligned run of ap ordinates onto an
// aligned run in reverse order (the LQn sets, with the x sign fastest, do)
static bool OppositeRunsReverse(const ubolt_ctx *ctx, int ap)
{
   const int A = ctx->A;
   if ((int)ctx->h_opp.size() != A || A % ap != 0) return false;
   for (int a0 = 0; a0 < A; a0 += ap) {
      const int r0 = ctx->h_opp[a0 + ap - 1];
      if (r0 % ap != 0) return false;
      for (int p = 0; p < ap; p++)
         if (ctx->h_opp[a0 + p] != r0 + (ap - 1 - p)) return false;
   }
   return true;
}

template <typename T, int NB, int F>
int LaunchApply(const ubolt_ctx *ctx, const DevGeom<T> &g, const T *x, T *y, int mode, cudaStream_t s)
{
   const int K = CellsPerBlock(g.A);
   const int threads = ((K * g.A + 31) / 32) * 32;
   const int64_t blocks = (g.n_cells + K - 1) / K;
   // AP ordinates per thread as one 16-byte run where they fit evenly and
   // both vectors are 16-byte aligned
   constexpr int AV = 16 / (int)sizeof(T);
   const bool vec = g.A % AV == 0 && (reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 16 == 0;
   const bool rev = mode == kAdjoint && OppositeRunsReverse(ctx, vec ? AV : 1);
   if (mode == kAdjoint && !rev) {
      const size_t smem = sizeof(T) * (size_t)(K * NB * g.A + K * NB);
      AdjointApplyKernel<T, NB, F><<<blocks, threads, smem, s>>>(g, x, y, K);
   } else {
      const int AP = vec ? AV : 1;
      const int QA = g.A / AP;
      if (QA > 256) return SetError(UBOLT_ERR_ARG, "apply: %d ordinates need 16-byte aligned vectors", g.A);
      auto kern = rev ? (vec ? ApplyKernel<T, NB, F, AV, true, true> : ApplyKernel<T, NB, F, 1, true, true>)
                  : vec ? (mode == kFull ? ApplyKernel<T, NB, F, AV, true> : ApplyKernel<T, NB, F, AV, false>)
                        : (mode == kFull ? ApplyKernel<T, NB, F, 1, true> : ApplyKernel<T, NB, F, 1, false>);
      const int A = g.A;
      auto smem_of = [vec, A, rev](int K, int thr) {
         return sizeof(T) * (vec ? ApplySmemElems<T, NB, F, AV>(K, thr, A, rev)
                                 : ApplySmemElems<T, NB, F, 1>(K, thr, A, rev));
      };
      const int Kt = ApplyCells(kern, QA, smem_of);
      const int64_t nblk = (g.n_cells + Kt - 1) / Kt;
      const int nthr = (Kt * QA + 31) / 32 * 32;
      const size_t smem = smem_of(Kt, nthr);
      if (smem > 48 * 1024) {
         const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
         if (e != cudaSuccess) {
            cudaGetLastError();
            return SetError(UBOLT_ERR_ARG, "apply: %zu bytes of shared memory for %d ordinates: %s", smem, g.A,
                            cudaGetErrorString(e));
         }
      }
      kern<<<nblk, nthr, smem, s>>>(g, x, y, Kt);
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
   if (ctx->cg) {
      if (mode == kAdjoint) return RequireDg(ctx, "the transpose apply");
      return CgApply<T>(ctx, x, y, mode == kFull, stream);
   }
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
   if (ctx->cg) return CgDiagonal(ctx, d, stream);
   const DevGeom<double> &g = ctx->geom<double>();
   UBOLT_DISPATCH(ctx->nb, ctx->F, return (LaunchDiagonal<double, NB_, F_>(g, d, (cudaStream_t)stream)));
   return SetError(UBOLT_ERR_STATE, "no kernel for n_basis %d with %d faces", ctx->nb, ctx->F);
}
