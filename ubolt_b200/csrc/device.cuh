// Device-side data layout and the per-(cell, angle) arithmetic shared by the
// apply, block, sweep and adjoint kernels.
//
// HBM layout. Phase-space vectors keep UBOLT's row order (angle fastest), so
// a cell's n_basis * n_angles values are one contiguous run. Geometry is
// split into a per-CELL part - the face codes (neighbour or boundary side),
// the mirror slot of each interior face, a geometry-class id - and a
// per-CLASS part holding everything derived from shape: outward area
// normals, face matrices, basis gradients, face basis values, volume. Cells
// whose class data are bitwise equal share a class, so a uniform box reads
// a few dozen classes from L1/L2 instead of kilobytes of geometry per cell.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ubolt {

constexpr int kMaxNb = 4;
constexpr int kMaxFaces = 6;

// Face code per (cell, slot): >= 0 the neighbour cell; -1 - side on the
// boundary, side = 2 * axis + (0 low | 1 high).
__host__ __device__ inline bool FaceInterior(int32_t code) { return code >= 0; }
__host__ __device__ inline int FaceSide(int32_t code) { return -1 - code; }

// n elements of `elem` bytes rounded up to a whole number of 16-byte units
__host__ __device__ constexpr int Pad16(int n, int elem) { return (n + 16 / elem - 1) / (16 / elem) * (16 / elem); }

// A geometry class packed as one record of 16-byte units, so a thread reads
// a face's parts with a few vector loads: per face f a slab [nA_f (3, padded
// to 4) | face_own_f (nb x nb) | face_up_f (nb x nb)], then [grad phi (nb x
// 3) | 1 / V] (the matrices and gradients only for nb > 1), each part padded
// to 16 bytes. Offsets in elements of `elem` bytes.
struct RecordLayout {
   int nb, fm, fs, tail, size;
   __host__ __device__ constexpr RecordLayout(int nb_, int F, int elem)
       : nb(nb_), fm(nb_ > 1 ? Pad16(nb_ * nb_, elem) : 0), fs(4 + 2 * (nb_ > 1 ? Pad16(nb_ * nb_, elem) : 0)),
         tail(F * (4 + 2 * (nb_ > 1 ? Pad16(nb_ * nb_, elem) : 0))),
         size(F * (4 + 2 * (nb_ > 1 ? Pad16(nb_ * nb_, elem) : 0)) + Pad16((nb_ > 1 ? 3 * nb_ : 0) + 1, elem))
   {
   }
   __host__ __device__ constexpr int nA(int f) const { return f * fs; }
   __host__ __device__ constexpr int fown(int f) const { return f * fs + 4; }
   __host__ __device__ constexpr int fup(int f) const { return f * fs + 4 + fm; }
   __host__ __device__ constexpr int bgrad() const { return tail; }
   __host__ __device__ constexpr int ivol() const { return tail + (nb > 1 ? 3 * nb : 0); }
};

template <typename T>
struct DevGeom {
   int32_t dim, nb, F, A;
   int64_t n_cells;
   T sum_weights;
   T inv_sum_weights;
   // Per class
   const T *nA;       // [class][F][3]
   const T *fown;     // [class][F][nb][nb]
   const T *fup;      // [class][F][nb][nb]
   const T *bgrad;    // [class][nb][3]
   const T *fbv;      // [class][F][nb]
   const T *inv_vol;  // [class]
   const T *rec;      // [class][RecordLayout(nb, F, sizeof(T)).size]: the same data packed per class
   // Per cell
   const int32_t *cls;     // [cell]
   const int32_t *code;    // [cell][F]
   const int8_t *mirror;   // [cell][F]: the neighbour's slot for the same face, -1 on the boundary
   // Quadrature
   const T *omega;         // [A][3]
   const T *w;             // [A]
   const int32_t *refl;    // [3][A]
   int32_t side_bc[6];     // UBOLT_BC_* per side
   const int32_t *opp;     // [A] the opposite ordinate (every cosine negated)
   const T *volume;        // [cell] cell volume
   // Group cross sections (per cell)
   const T *sigma_t;
   const T *sigma_s;
};

// An asynchronous global -> shared copy of one 4-, 8- or 16-byte word, both
// addresses aligned to its size
template <int BYTES>
__device__ __forceinline__ void CpAsync(void *smem_dst, const void *src)
{
   const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
   asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
}
// An L2 policy that evicts a line first: for data read once per launch
// (streamed through, not to displace what other warps are about to read)
__device__ __forceinline__ uint64_t EvictFirstPolicy()
{
   uint64_t p;
   asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
   return p;
}
// CpAsync with an L2 cache policy
template <int BYTES>
__device__ __forceinline__ void CpAsyncHint(void *smem_dst, const void *src, uint64_t policy)
{
   const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
   asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], %2, %3;" ::"r"(d), "l"(src), "n"(BYTES),
                "l"(policy)
                : "memory");
}
// A load with an L2 cache policy
__device__ __forceinline__ double LoadHint(const double *p, uint64_t policy)
{
   double v;
   asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(policy));
   return v;
}
__device__ __forceinline__ float LoadHint(const float *p, uint64_t policy)
{
   float v;
   asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(policy));
   return v;
}
__device__ __forceinline__ void CpAsyncWaitAll() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void CpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void CpAsyncWaitGroup() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename T>
__device__ __forceinline__ T Dot3(const T *__restrict__ om, const T *__restrict__ n)
{
   // Omega . nA in the reference's term order (FaceFlux, plex_commonk.hpp:314-317)
   return om[0] * n[0] + om[1] * n[1] + om[2] * n[2];
}
template <typename T>
__device__ __forceinline__ T Dot3(T ox, T oy, T oz, const T *__restrict__ n)
{
   return ox * n[0] + oy * n[1] + oz * n[2];
}

// The (cell, angle) element block of streaming + removal:
//   B(i, j) = sum_{f: s_f > 0} s_f face_own_f(i, j) - [j == 0, i > 0] Omega . grad phi_i + sigma_t delta_ij
// DG0: B = (sum_{s > 0} s) / V + sigma_t (DG0OutflowDiagonal then removal,
// termsk.kokkos.cxx:183-196, 451-470). DG1: StreamingTermDG1::assemble_add,
// termsk.kokkos.cxx:314-389.
template <typename T, int NB, int F>
__device__ __forceinline__ void BuildBlock(const DevGeom<T> &g, int32_t cl, const T om[3], T sigma_t, T B[NB][NB])
{
   if constexpr (NB == 1) {
      T outflow = T(0);
#pragma unroll
      for (int f = 0; f < F; f++) {
         const T s = Dot3(om, g.nA + ((int64_t)cl * F + f) * 3);
         if (s > T(0)) outflow += s;
      }
      B[0][0] = outflow * g.inv_vol[cl] + sigma_t;
   } else {
#pragma unroll
      for (int i = 0; i < NB; i++)
#pragma unroll
         for (int j = 0; j < NB; j++) B[i][j] = T(0);
#pragma unroll
      for (int f = 0; f < F; f++) {
         const T s = Dot3(om, g.nA + ((int64_t)cl * F + f) * 3);
         if (s > T(0)) {
            const T *M = g.fown + ((int64_t)cl * F + f) * NB * NB;
#pragma unroll
            for (int i = 0; i < NB; i++)
#pragma unroll
               for (int j = 0; j < NB; j++) B[i][j] += s * M[i * NB + j];
         }
      }
#pragma unroll
      for (int i = 1; i < NB; i++) B[i][0] -= Dot3(om, g.bgrad + ((int64_t)cl * NB + i) * 3);
#pragma unroll
      for (int i = 0; i < NB; i++) B[i][i] += sigma_t;
   }
}

// Solve B y = r in place by Gaussian elimination with partial pivoting.
// Returns false for a singular block (a zero pivot), leaving r unchanged.
template <typename T, int NB>
__device__ __forceinline__ bool SolveBlock(T B[NB][NB], T r[NB])
{
   if constexpr (NB == 1) {
      if (B[0][0] == T(0)) return false;
      r[0] = r[0] / B[0][0];
      return true;
   } else {
#pragma unroll
      for (int k = 0; k < NB; k++) {
         int piv = k;
         T best = fabs(B[k][k]);
#pragma unroll
         for (int i = k + 1; i < NB; i++) {
            const T v = fabs(B[i][k]);
            if (v > best) { best = v; piv = i; }
         }
         if (best == T(0)) return false;
         if (piv != k) {
#pragma unroll
            for (int i = k + 1; i < NB; i++)
               if (i == piv) {
#pragma unroll
                  for (int j = 0; j < NB; j++) { const T t = B[k][j]; B[k][j] = B[i][j]; B[i][j] = t; }
                  const T t = r[k]; r[k] = r[i]; r[i] = t;
               }
         }
         const T inv = T(1) / B[k][k];
#pragma unroll
         for (int i = k + 1; i < NB; i++) {
            const T f = B[i][k] * inv;
#pragma unroll
            for (int j = k + 1; j < NB; j++) B[i][j] -= f * B[k][j];
            r[i] -= f * r[k];
         }
      }
#pragma unroll
      for (int k = NB - 1; k >= 0; k--) {
         T s = r[k];
#pragma unroll
         for (int j = k + 1; j < NB; j++) s -= B[k][j] * r[j];
         r[k] = s / B[k][k];
      }
      return true;
   }
}

// LU factorisation with partial pivoting in place (unit lower L below the
// diagonal, U on and above it); perm records the row swaps. False on a zero pivot.
template <typename T, int NB>
__device__ __forceinline__ bool LuFactor(T B[NB][NB], int perm[NB])
{
#pragma unroll
   for (int k = 0; k < NB; k++) perm[k] = k;
#pragma unroll
   for (int k = 0; k < NB; k++) {
      int piv = k;
      T best = fabs(B[k][k]);
#pragma unroll
      for (int i = k + 1; i < NB; i++) {
         const T v = fabs(B[i][k]);
         if (v > best) { best = v; piv = i; }
      }
      if (best == T(0)) return false;
      if (piv != k) {
#pragma unroll
         for (int i = k + 1; i < NB; i++)
            if (i == piv) {
#pragma unroll
               for (int j = 0; j < NB; j++) { const T t = B[k][j]; B[k][j] = B[i][j]; B[i][j] = t; }
               const int t = perm[k]; perm[k] = perm[i]; perm[i] = t;
            }
      }
      const T inv = T(1) / B[k][k];
#pragma unroll
      for (int i = k + 1; i < NB; i++) {
         B[i][k] *= inv;
#pragma unroll
         for (int j = k + 1; j < NB; j++) B[i][j] -= B[i][k] * B[k][j];
      }
   }
   return true;
}

// x = B^{-1} r from LuFactor's output (r is overwritten with x)
template <typename T, int NB>
__device__ __forceinline__ void LuSolve(const T B[NB][NB], const int perm[NB], T r[NB])
{
   T y[NB];
#pragma unroll
   for (int i = 0; i < NB; i++) {
      T s = T(0);
#pragma unroll
      for (int j = 0; j < NB; j++)
         if (j == perm[i]) s = r[j];
      y[i] = s;
   }
#pragma unroll
   for (int i = 0; i < NB; i++)
#pragma unroll
      for (int j = 0; j < i; j++) y[i] -= B[i][j] * y[j];
#pragma unroll
   for (int i = NB - 1; i >= 0; i--) {
#pragma unroll
      for (int j = i + 1; j < NB; j++) y[i] -= B[i][j] * y[j];
      y[i] /= B[i][i];
   }
#pragma unroll
   for (int i = 0; i < NB; i++) r[i] = y[i];
}

// The explicit inverse by Gauss-Jordan with partial pivoting, [B | I] ->
// [I | B^{-1}], in InvertBlocksKernel's order (block_inversek.kokkos.cxx:83-150).
// B is destroyed. False on a zero pivot, with W left partial.
template <typename T, int NB>
__device__ __forceinline__ bool InvertBlock(T m[NB][NB], T w[NB][NB])
{
#pragma unroll
   for (int i = 0; i < NB; i++)
#pragma unroll
      for (int j = 0; j < NB; j++) w[i][j] = (i == j) ? T(1) : T(0);
#pragma unroll
   for (int k = 0; k < NB; k++) {
      int piv = k;
      T best = fabs(m[k][k]);
#pragma unroll
      for (int i = k + 1; i < NB; i++) {
         const T v = fabs(m[i][k]);
         if (v > best) { best = v; piv = i; }
      }
      if (best == T(0)) return false;
      if (piv != k) {
#pragma unroll
         for (int i = 0; i < NB; i++)
            if (i == piv && i != k) {
#pragma unroll
               for (int j = 0; j < NB; j++) {
                  T t = m[k][j]; m[k][j] = m[i][j]; m[i][j] = t;
                  t = w[k][j]; w[k][j] = w[i][j]; w[i][j] = t;
               }
            }
      }
      const T inv_piv = T(1) / m[k][k];
#pragma unroll
      for (int j = 0; j < NB; j++) { m[k][j] *= inv_piv; w[k][j] *= inv_piv; }
#pragma unroll
      for (int i = 0; i < NB; i++) {
         if (i == k) continue;
         const T f = m[i][k];
         if (f == T(0)) continue;
#pragma unroll
         for (int j = 0; j < NB; j++) { m[i][j] -= f * m[k][j]; w[i][j] -= f * w[k][j]; }
      }
   }
   return true;
}

template <typename T, int NB>
__device__ __forceinline__ void Transpose(T B[NB][NB])
{
#pragma unroll
   for (int i = 0; i < NB; i++)
#pragma unroll
      for (int j = i + 1; j < NB; j++) { const T t = B[i][j]; B[i][j] = B[j][i]; B[j][i] = t; }
}

// Threads per block for the (cell, angle)-flattened kernels: whole cells per
// block, about 256 threads.
__host__ inline int CellsPerBlock(int A)
{
   int k = (256 + A / 2) / A;
   return k < 1 ? 1 : k;
}

// The factors of one (cell, ordinate) for the sweep: W = B^{-1} of its
// streaming + removal block, and G_s = W (s_f face_up_f) for each gathered
// face f in face order (slot s); element (s, ii, j) goes to Gout[s * gs + (ii * NB + j) * ge].
// A singular block gives zero factors. Returns false then.
template <typename T, int NB, int F>
__device__ __forceinline__ bool CellFactors(const DevGeom<T> &g, int64_t c, const T om[3], uint32_t mask, T W[NB][NB],
                                            T *Gout, size_t gs, size_t ge)
{
   const int32_t cl = g.cls[c];
   T B[NB][NB];
   BuildBlock<T, NB, F>(g, cl, om, g.sigma_t[c], B);
   const bool ok = InvertBlock<T, NB>(B, W);
   if (!ok)
#pragma unroll
      for (int ii = 0; ii < NB; ii++)
#pragma unroll
         for (int j = 0; j < NB; j++) W[ii][j] = T(0);
   int slot = 0;
#pragma unroll
   for (int f = 0; f < F; f++) {
      if (!(((mask >> f) | (mask >> (8 + f))) & 1u)) continue;
      const T sf = Dot3(om, g.nA + ((int64_t)cl * F + f) * 3);
      T *Gf = Gout + (size_t)slot * gs;
      if constexpr (NB == 1) {
         Gf[0] = W[0][0] * (sf * g.inv_vol[cl]);
      } else {
         const T *M = g.fup + ((int64_t)cl * F + f) * NB * NB;
         T Ms[NB][NB];
#pragma unroll
         for (int kk = 0; kk < NB; kk++)
#pragma unroll
            for (int j = 0; j < NB; j++) Ms[kk][j] = sf * M[kk * NB + j];
#pragma unroll
         for (int ii = 0; ii < NB; ii++)
#pragma unroll
            for (int j = 0; j < NB; j++) {
               T u = T(0);
#pragma unroll
               for (int kk = 0; kk < NB; kk++) u += W[ii][kk] * Ms[kk][j];
               Gf[(size_t)(ii * NB + j) * ge] = u;
            }
      }
      slot++;
   }
   return ok;
}

// Node-run kernels. A node's A ordinates are one contiguous run of psi. A
// warp takes kLpn = 8 lanes per node, four nodes at a time; lane `sub` of a
// node strides its run by 8, so every load or store of the warp covers four
// runs of 8 consecutive values (whole sectors), and a node's eight partial
// sums meet in 3 shuffle steps. All lanes of a warp run the same iterations.
constexpr int kLpn = 8;

__device__ __forceinline__ double GroupSum(double v)
{
   v += __shfl_xor_sync(0xffffffffu, v, 4);
   v += __shfl_xor_sync(0xffffffffu, v, 2);
   v += __shfl_xor_sync(0xffffffffu, v, 1);
   return v;
}

// Blocks of 256 threads for a grid-stride loop over groups of four runs
__host__ inline int RunGrid(int64_t n_runs)
{
   const int64_t want = (n_runs + 31) / 32;
   return (int)(want < 1 ? 1 : (want > 148 * 16 ? 148 * 16 : want));
}

}  // namespace ubolt
