// Diffusion synthetic acceleration, the scattering half of the preconditioner
// (DSAPrecon, include/ubolt/dsa.hpp; src/dsak.kokkos.cxx, src/dsa_plexk.kokkos.cxx):
//
//    y = P D^{-1} R x,  R: rhs(node) = V_c sum_a w_a x(node, a),
//                       P: y(node, a) = u(node) / W,
//    D the VOLUME-weighted diffusion operator on the cell nodes,
//    D_c = 1 / (3 sigma_t), sigma_a = sigma_t - sigma_s:
//      DG1: the MIP interior-penalty form on the modal basis, penalty C (4),
//           floor 1/4 (DSAPlex::assemble_dg1, dsa_plexk.kokkos.cxx:365-475);
//      DG0: the two-point flux with the consistent-D blend
//           (D^p + (m h)^p)^(1/p), p = 1.5 (assemble_dg0, :288-348).
// Voids follow DSAPrecon::assemble's policy (dsak.kokkos.cxx:233-345), on
// one rank of a backend that can mask: a cell with sigma_t <= void_sigma_t
// is void; the voids are bridged (D = 1/(3 (sigma_t + 1/L)), L their mean
// chord 4 V / S, or a fixed void D) when that is asked for and leaves the
// operator nonsingular, else masked: V times the identity, no coupling, a
// face into one is a vacuum face, and R and P skip its nodes
// (dsa_plexk.kokkos.cxx:288-475, RestrictKernel/ProlongKernel).
//
// As in the reference the matrix is refilled on the host per group (a host
// loop) and uploaded; here into a block-ELL layout - per cell its F neighbour
// blocks (slot order, zero where a face has no neighbour) then its own block,
// nb x nb each - so the SpMV is one gather per face, coalesced over nodes.
// The inner solve replaces the reference's one GAMG V-cycle (PCGAMG,
// dsak.kokkos.cxx:197-212) with a fixed number of block-Jacobi PCG
// iterations run entirely on the device (scalars stay in device memory, no
// host round trip), in FP64 whatever the outer precision.
//
// On a CG-SUPG context the operator is DSACG's (src/dsa_cgk.kokkos.cxx): one
// unknown per vertex, the weak form
//    sum_e int_e D_e grad u . grad v + sigma_a u v + per vacuum face its
//    incoming half-range current times the lumped face mass on the diagonal,
// in CSR; R weighs by the lumped mass instead of the volume, P is the same,
// nothing is masked, and an unbridged void keeps the SUPG operator's own
// tensor D_e = (1/W) sum_a w_a tau_a Omega_a Omega_a^T (CGSupgDKernel, :66-84).
#include "cg.h"
#include "ctx.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

struct ubolt_dsa {
   int nb = 1, F = 0;
   int64_t nc = 0, n_nodes = 0;
   double penalty = 4.0, power = 1.5;
   int consistent = 1, inner_its = 30;
   bool assembled = false;
   // The void policy: options, the boundary's vacuum faces, and this group's outcome
   double void_sigma_t = 0.0, void_d = 0.0;
   int void_bridge = 1;
   bool any_vacuum = false;
   int64_t n_void = 0;
   int bridged = 0;
   double chord = 0.0;
   std::vector<uint8_t> h_void, h_mask;
   std::vector<double> h_d;
   uint8_t *mask = nullptr;  // device, per cell: a masked void
   // Host geometry (the backend data DSAPlex::create keeps)
   std::vector<double> area, nrm, dist, volume, fown, fup, bgrad, nbgrad, half_range;
   std::vector<int64_t> nbr;
   std::vector<int32_t> bc;
   std::vector<double> h_val, h_jinv;
   // CG-SUPG: the vertex CSR, and per (element, li, j) its entry
   bool cg = false;
   std::vector<int64_t> rp, entry;
   std::vector<int32_t> col;
   std::vector<double> vacuum_weight;  // per vertex
   int64_t *d_rp = nullptr;
   int32_t *d_col = nullptr;
   // Device
   double *val = nullptr, *jinv = nullptr;          // [nc][F+1][nb][nb], [nc][nb][nb] (CG: [nnz], [n_nodes])
   double *rhs = nullptr, *u = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
   // [0] rho, [1] rho_new, [2] pq, [3] the grid sums' block counter (an
   // unsigned int in a double's slot), then one partial per block
   double *scal = nullptr;
};

namespace ubolt {

constexpr int kDsaThreads = 256;

// Scalar slots ahead of the per-block partials
constexpr int kDsaScalars = 4;

// Deterministic sum of d over the grid into *out: each block's total goes to
// part[blockIdx.x]; the last block to finish (an integer counter) adds the
// totals in a fixed order - per-lane strided sums, then a shuffle tree, the
// same every run - writes *out and resets the counter. No block waits on
// another. Every thread of the block must call it.
__device__ __forceinline__ void GridSum(double d, double *part, unsigned *count, double *out)
{
   __shared__ double red[kDsaThreads / 32];
   __shared__ bool last;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
   if (lane == 0) red[warp] = d;
   __syncthreads();
   if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < nw; w++) s += red[w];
      part[blockIdx.x] = s;
      __threadfence();
      last = atomicAdd(count, 1u) == gridDim.x - 1;
   }
   __syncthreads();
   if (!last) return;
   __threadfence();
   double s = 0.0;
   for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += __ldcg(&part[b]);
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
   __syncthreads();
   if (lane == 0) red[warp] = s;
   __syncthreads();
   if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nw; w++) t += red[w];
      *out = t;
      *count = 0;
   }
}

__device__ __forceinline__ unsigned *GridCount(double *scal) { return reinterpret_cast<unsigned *>(scal + 3); }

// v = D u over the block-ELL rows, one thread per node
__global__ void DsaSpmvKernel(int64_t n_nodes, int nb, int F, const int32_t *__restrict__ code,
                              const double *__restrict__ val, const double *__restrict__ u, double *__restrict__ v,
                              const double *__restrict__ dotw, double *scal)
{
   const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   double d = 0.0;
   if (node < n_nodes) {
      const int64_t c = node / nb;
      const int i = (int)(node - c * nb);
      const double *blk = val + (c * (F + 1)) * nb * nb;
      double s = 0.0;
      for (int f = 0; f < F; f++) {
         const int32_t n = code[c * F + f];
         if (n < 0) continue;
         for (int j = 0; j < nb; j++) s += blk[(f * nb + i) * nb + j] * u[(int64_t)n * nb + j];
      }
      for (int j = 0; j < nb; j++) s += blk[(F * nb + i) * nb + j] * u[c * nb + j];
      v[node] = s;
      if (dotw) d = dotw[node] * s;
   }
   // scal[2] = (dotw, v), when asked
   if (scal) GridSum(d, scal + kDsaScalars, GridCount(scal), &scal[2]);
}

// v = D u over CSR rows (the CG-SUPG vertices), one thread per row
__global__ void DsaCsrSpmvKernel(int64_t n_nodes, const int64_t *__restrict__ rp, const int32_t *__restrict__ col,
                                 const double *__restrict__ val, const double *__restrict__ u, double *__restrict__ v,
                                 const double *__restrict__ dotw, double *scal)
{
   const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   double d = 0.0;
   if (node < n_nodes) {
      double s = 0.0;
      for (int64_t k = rp[node]; k < rp[node + 1]; k++) s += val[k] * u[col[k]];
      v[node] = s;
      if (dotw) d = dotw[node] * s;
   }
   if (scal) GridSum(d, scal + kDsaScalars, GridCount(scal), &scal[2]);
}

// v = D u in whichever storage the context's DSA has; with scal, also (dotw, v) into scal[2]
static void DsaSpmvLaunch(const ubolt_ctx *ctx, const ubolt_dsa *ds, const double *u, double *v, const double *dotw,
                          double *scal, cudaStream_t s)
{
   const int64_t grid = (ds->n_nodes + kDsaThreads - 1) / kDsaThreads;
   if (ds->cg)
      DsaCsrSpmvKernel<<<grid, kDsaThreads, 0, s>>>(ds->n_nodes, ds->d_rp, ds->d_col, ds->val, u, v, dotw, scal);
   else
      DsaSpmvKernel<<<grid, kDsaThreads, 0, s>>>(ds->n_nodes, ds->nb, ds->F, ctx->g64.code, ds->val, u, v, dotw,
                                                 scal);
}

// rhs(node) = V_c sum_a w_a (x(node, a) - ax(node, a)); ax may be NULL. A
// node-run kernel. A masked void's nodes restrict to zero (mask may be NULL: none).
template <typename T>
__global__ void __launch_bounds__(256) DsaRestrictKernel(int64_t n_nodes, int nb, int A, const double *__restrict__ w,
                                                         const double *__restrict__ volume, const T *__restrict__ x,
                                                         const T *__restrict__ ax, const uint8_t *__restrict__ mask,
                                                         double *__restrict__ rhs)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      const bool live = node < n_nodes;
      double s = 0.0;
      if (live)
         for (int a = sub; a < A; a += kLpn) {
            double v = (double)x[node * A + a];
            if (ax) v -= (double)ax[node * A + a];
            s += w[a] * v;
         }
      s = GroupSum(s);
      if (live && sub == 0) rhs[node] = (mask && mask[node / nb]) ? 0.0 : s * volume[node / nb];
   }
}

// y(node, a) (+)= u(node) / W; a masked void's rows get zero (mask may be NULL)
template <typename T>
__global__ void __launch_bounds__(256) DsaProlongKernel(int64_t n_nodes, int nb, int A, double inv_w,
                                                        const double *__restrict__ u, const uint8_t *__restrict__ mask,
                                                        T *__restrict__ y, int add)
{
   const int lane = threadIdx.x & 31, sub = lane & (kLpn - 1);
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t n0 = warp * 4; n0 < n_nodes; n0 += n_warps * 4) {
      const int64_t node = n0 + (lane >> 3);
      if (node >= n_nodes) continue;
      const double v = (mask && mask[node / nb]) ? 0.0 : u[node] * inv_w;
      T *run = y + node * A;
      for (int a = sub; a < A; a += kLpn) run[a] = add ? (T)((double)run[a] + v) : (T)v;
   }
}

// ~~~ Block-Jacobi PCG on the device, a fixed number of iterations from u = 0

// r = rhs, u = 0, z = J r, p = z, scal[0] = (r, z)
__global__ void CgStartKernel(int64_t n_nodes, int nb, const double *__restrict__ jinv, const double *__restrict__ rhs,
                              double *__restrict__ u, double *__restrict__ r, double *__restrict__ z,
                              double *__restrict__ p, double *scal)
{
   const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   double d = 0.0;
   if (node < n_nodes) {
      const int64_t c = node / nb;
      const int i = (int)(node - c * nb);
      double zz = 0.0;
      for (int j = 0; j < nb; j++) zz += jinv[(c * nb + i) * nb + j] * rhs[c * nb + j];
      r[node] = rhs[node];
      u[node] = 0.0;
      z[node] = zz;
      p[node] = zz;
      d = rhs[node] * zz;
   }
   GridSum(d, scal + kDsaScalars, GridCount(scal), &scal[0]);
}

// alpha = rho / pq; u += alpha p; r -= alpha q
__global__ void CgUpdateKernel(int64_t n_nodes, const double *__restrict__ p, const double *__restrict__ q,
                               double *__restrict__ u, double *__restrict__ r, const double *scal)
{
   const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (node >= n_nodes) return;
   const double pq = scal[2];
   const double alpha = pq != 0.0 ? scal[0] / pq : 0.0;
   u[node] += alpha * p[node];
   r[node] -= alpha * q[node];
}

// z = J r; scal[1] = (r, z)
__global__ void CgPrecondKernel(int64_t n_nodes, int nb, const double *__restrict__ jinv, const double *__restrict__ r,
                                double *__restrict__ z, double *scal)
{
   const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   double d = 0.0;
   if (node < n_nodes) {
      const int64_t c = node / nb;
      const int i = (int)(node - c * nb);
      double zz = 0.0;
      for (int j = 0; j < nb; j++) zz += jinv[(c * nb + i) * nb + j] * r[c * nb + j];
      z[node] = zz;
      d = r[node] * zz;
   }
   GridSum(d, scal + kDsaScalars, GridCount(scal), &scal[1]);
}

// beta = rho_new / rho; p = z + beta p; rho = rho_new; clear rho_new and pq (one thread does the scalars)
__global__ void CgDirectionKernel(int64_t n_nodes, const double *__restrict__ z, double *__restrict__ p, double *scal)
{
   const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   const double rho = scal[0], rho_new = scal[1];
   const double beta = rho != 0.0 ? rho_new / rho : 0.0;
   if (node < n_nodes) p[node] = z[node] + beta * p[node];
}

__global__ void CgRotateScalars(double *scal)
{
   scal[0] = scal[1];
   scal[1] = 0.0;
   scal[2] = 0.0;
}

// ~~~ Host assembly

static void InvertSmall(int nb, const double *m_in, double *inv)
{
   double m[4][4], w[4][4];
   for (int i = 0; i < nb; i++)
      for (int j = 0; j < nb; j++) {
         m[i][j] = m_in[i * nb + j];
         w[i][j] = (i == j) ? 1.0 : 0.0;
      }
   for (int k = 0; k < nb; k++) {
      int piv = k;
      for (int i = k + 1; i < nb; i++)
         if (std::fabs(m[i][k]) > std::fabs(m[piv][k])) piv = i;
      if (m[piv][k] == 0.0) {
         for (int i = 0; i < nb * nb; i++) inv[i] = 0.0;
         return;
      }
      if (piv != k)
         for (int j = 0; j < nb; j++) {
            std::swap(m[k][j], m[piv][j]);
            std::swap(w[k][j], w[piv][j]);
         }
      const double ip = 1.0 / m[k][k];
      for (int j = 0; j < nb; j++) { m[k][j] *= ip; w[k][j] *= ip; }
      for (int i = 0; i < nb; i++) {
         if (i == k) continue;
         const double f = m[i][k];
         for (int j = 0; j < nb; j++) { m[i][j] -= f * m[k][j]; w[i][j] -= f * w[k][j]; }
      }
   }
   for (int i = 0; i < nb; i++)
      for (int j = 0; j < nb; j++) inv[i * nb + j] = w[i][j];
}

static double BlendD(double d, double m, double p)
{
   if (p == 1.0) return d + m;
   return std::pow(std::pow(d, p) + std::pow(m, p), 1.0 / p);
}

// The void policy for one group (DSAPrecon::assemble, dsak.kokkos.cxx:233-345,
// with DSAPlex::void_volume_surface, dsa_plexk.kokkos.cxx:243-262): the
// census, the bridge decision and the voids' mean chord, D per cell and the
// mask, and the guard against a singular operator. A backend that cannot
// mask (CG-SUPG) checks the guard first, without counting on a void, and
// bridges whenever there is a void.
static int VoidPolicy(ubolt_dsa *ds, const double *st, const double *ss, bool can_mask = true)
{
   const int F = ds->F;
   const int64_t nc = ds->nc;
   ds->h_void.assign(nc, 0);
   ds->h_mask.assign(nc, 0);
   ds->h_d.assign(nc, 0.0);
   int64_t n_void = 0;
   // The largest sigma_a anywhere, and outside the voids
   double max_sa_all = 0.0, max_sa_solid = 0.0;
   for (int64_t c = 0; c < nc; c++) {
      const double sa = st[c] - ss[c];
      ds->h_void[c] = st[c] <= ds->void_sigma_t;
      if (ds->h_void[c]) n_void++;
      else max_sa_solid = std::max(max_sa_solid, sa);
      max_sa_all = std::max(max_sa_all, sa);
   }
   if (!can_mask && !(ds->any_vacuum || max_sa_all > 0.0))
      return SetError(UBOLT_ERR_ARG,
                      "the DSA diffusion operator is singular: every face is reflective and sigma_a = sigma_t - "
                      "sigma_s is zero everywhere in this group");
   // Bridge when asked, some cell is void and some is not, and a vacuum face
   // or some absorption holds the bridged operator; bridged iff a face ends
   // a flight through the voids (their chord is positive)
   ds->bridged = 0;
   ds->chord = 0.0;
   if (ds->void_bridge && n_void > 0 &&
       (!can_mask || (n_void < nc && (ds->any_vacuum || max_sa_all > 0.0)))) {
      double vol = 0.0, surf = 0.0;
      for (int64_t c = 0; c < nc; c++) {
         if (!ds->h_void[c]) continue;
         vol += ds->volume[c];
         for (int f = 0; f < F; f++) {
            const int64_t k = c * F + f;
            const int64_t n = ds->nbr[k];
            if (n >= 0 ? !ds->h_void[n] : ds->bc[k] == UBOLT_BC_VACUUM) surf += ds->area[k];
         }
      }
      ds->chord = surf > 0.0 ? 4.0 * vol / surf : 0.0;
      ds->bridged = ds->chord > 0.0;
   }
   // D: 1/(3 sigma_t); in a bridged void 1/3 of the flight 1/(sigma_t + 1/L)
   // unless a void D is fixed; 0 in an unbridged void, which is masked
   for (int64_t c = 0; c < nc; c++) {
      if (!ds->h_void[c]) ds->h_d[c] = 1.0 / (3.0 * st[c]);
      else if (ds->bridged)
         ds->h_d[c] = ds->void_d > 0.0 ? ds->void_d : 1.0 / (3.0 * (std::max(st[c], 0.0) + 1.0 / ds->chord));
      ds->h_mask[c] = can_mask && ds->h_void[c] && !ds->bridged;
   }
   ds->n_void = n_void;
   if (!can_mask) return UBOLT_OK;
   // Every face reflective (pure Neumann): only absorption, or a masked void
   // (whose faces are Marshak faces), keeps the operator nonsingular
   const double sa = ds->bridged ? max_sa_all : max_sa_solid;
   if (!(ds->any_vacuum || n_void > 0 || sa > 0.0))
      return SetError(UBOLT_ERR_ARG,
                      "the DSA diffusion operator is singular: every face is reflective, there is no void, and "
                      "sigma_a = sigma_t - sigma_s is zero everywhere in this group");
   return UBOLT_OK;
}

// Fill the block-ELL values and the block-Jacobi inverses for one group.
static int Assemble(ubolt_dsa *ds, const double *st, const double *ss)
{
   const int nb = ds->nb, F = ds->F;
   const int64_t nc = ds->nc;
   const size_t bs = (size_t)nb * nb;
   int rc = VoidPolicy(ds, st, ss);
   if (rc) return rc;
   ds->h_val.assign(nc * (F + 1) * bs, 0.0);
   ds->h_jinv.assign(nc * bs, 0.0);
   const double *dcell = ds->h_d.data();
   const uint8_t *masked = ds->h_mask.data(), *is_void = ds->h_void.data();
#pragma omp parallel for schedule(static)
   for (int64_t c = 0; c < nc; c++) {
      double *blk = &ds->h_val[c * (F + 1) * bs];
      double *own = blk + F * bs;
      const double vol = ds->volume[c];
      if (masked[c]) {
         // A masked void: V times the identity, every coupling zero
         for (int i = 0; i < nb; i++) own[i * nb + i] = vol;
         InvertSmall(nb, own, &ds->h_jinv[c * bs]);
         continue;
      }
      const double d_c = dcell[c];
      if (nb == 1) {
         double diag = vol * (st[c] - ss[c]);
         for (int f = 0; f < F; f++) {
            const int64_t k = c * F + f;
            const double d_own = ds->dist[2 * k];
            const int64_t n = ds->nbr[k];
            if (n >= 0 && !masked[n]) {
               const double d_n = dcell[n];
               double t_f = ds->area[k] / (d_own / d_c + ds->dist[2 * k + 1] / d_n);
               if (ds->consistent) {
                  const double len = d_own + ds->dist[2 * k + 1];
                  t_f = ds->area[k] / len * BlendD(t_f * len / ds->area[k], ds->half_range[k] * len, ds->power);
               }
               blk[f] = -t_f;
               diag += t_f;
            } else if (n >= 0 || ds->bc[k] == UBOLT_BC_VACUUM) {
               // A vacuum side, or a face into a masked void: Marshak
               const double d_b = ds->consistent ? BlendD(d_c, 2.0 * d_own * ds->half_range[k], ds->power) : d_c;
               diag += ds->area[k] / (2.0 + d_own / d_b);
            }
         }
         own[0] = diag;
      } else {
         const double sigma_a = st[c] - ss[c];
         for (int i = 0; i < nb; i++)
            for (int j = 0; j < nb; j++) {
               double gd = 0.0;
               for (int d = 0; d < 3; d++) gd += ds->bgrad[(c * nb + i) * 3 + d] * ds->bgrad[(c * nb + j) * 3 + d];
               own[i * nb + j] = vol * (d_c * gd + (i == j ? sigma_a : 0.0));
            }
         for (int f = 0; f < F; f++) {
            const int64_t k = c * F + f;
            const int64_t n = ds->nbr[k];
            // A face into a masked void is a vacuum face, as if the mesh stopped there
            const bool interior = n >= 0 && !masked[n];
            if (n < 0 && ds->bc[k] != UBOLT_BC_VACUUM) continue;
            const double scale = vol * ds->area[k];
            const double *fo = &ds->fown[k * bs], *fu = &ds->fup[k * bs];
            double gc[4], gn[4];
            for (int j = 0; j < nb; j++) {
               gc[j] = gn[j] = 0.0;
               for (int d = 0; d < 3; d++) {
                  gc[j] += ds->bgrad[(c * nb + j) * 3 + d] * ds->nrm[3 * k + d];
                  gn[j] += ds->nbgrad[(k * nb + j) * 3 + d] * ds->nrm[3 * k + d];
               }
            }
            const double h_c = 2.0 * ds->dist[2 * k];
            if (interior) {
               const double h_n = 2.0 * ds->dist[2 * k + 1];
               // A face touching a bridged void: both sides take the face's
               // harmonic D, in the averages and in kappa
               double dc_f = d_c, dn_f = dcell[n];
               if (ds->bridged && (is_void[c] || is_void[n])) {
                  dc_f = 2.0 * d_c * dcell[n] / (d_c + dcell[n]);
                  dn_f = dc_f;
               }
               const double kappa = std::max(0.5 * ds->penalty * (dc_f / h_c + dn_f / h_n), 0.25);
               double *nbb = blk + f * bs;
               for (int i = 0; i < nb; i++) {
                  const double m_i = scale * fo[i * nb];
                  for (int j = 0; j < nb; j++) {
                     own[i * nb + j] += kappa * scale * fo[i * nb + j] - 0.5 * dc_f * gc[j] * m_i -
                                        0.5 * dc_f * gc[i] * scale * fo[j];
                     nbb[i * nb + j] = -kappa * scale * fu[i * nb + j] - 0.5 * dn_f * gn[j] * m_i +
                                       0.5 * dc_f * gc[i] * scale * fu[j];
                  }
               }
            } else {
               const double kappa = std::max(ds->penalty * d_c / h_c, 0.25);
               for (int i = 0; i < nb; i++) {
                  const double m_i = scale * fo[i * nb];
                  for (int j = 0; j < nb; j++)
                     own[i * nb + j] += kappa * scale * fo[i * nb + j] - 0.5 * d_c * gc[j] * m_i -
                                        0.5 * d_c * gc[i] * scale * fo[j];
               }
            }
         }
      }
      InvertSmall(nb, own, &ds->h_jinv[c * bs]);
   }
   return UBOLT_OK;
}

// The CG-SUPG vertex operator for one group (DSACG::assemble,
// dsa_cgk.kokkos.cxx:247-281): per element (sigma_t - sigma_s) M_ij + D_e : K_ij
// into its (li, j) entries, D_e isotropic from the void policy or, in an
// unbridged void, the SUPG operator's own tensor; then the vacuum faces on the
// diagonal. Point-Jacobi inverses.
static int AssembleCg(const ubolt_ctx *ctx, ubolt_dsa *ds, const double *st, const double *ss)
{
   const ubolt_cg *cg = ctx->cg;
   int rc = VoidPolicy(ds, st, ss, false);
   if (rc) return rc;
   const int nv = cg->nv, A = ctx->A, dim = ctx->dim;
   const int64_t ne = cg->n_elements;
   const size_t n2 = (size_t)nv * nv;
   ds->h_val.assign(ds->col.size(), 0.0);
   std::vector<double> De(9);
   for (int64_t e = 0; e < ne; e++) {
      for (int k = 0; k < 9; k++) De[k] = (k % 4 == 0) ? ds->h_d[e] : 0.0;
      if (ds->h_void[e] && !ds->bridged) {
         // (1/W) sum_a w_a tau_a Omega_a Omega_a^T with the transport's own tau
         for (int k = 0; k < 9; k++) De[k] = 0.0;
         for (int a = 0; a < A; a++) {
            const double *om = &ctx->h_omega[3 * a];
            double sum = 0.0;
            for (int j = 0; j < nv; j++) {
               double s = 0.0;
               for (int c = 0; c < dim; c++) s += om[c] * cg->centre_grad[(e * nv + j) * 3 + c];
               sum += std::fabs(s);
            }
            const double thin = 2.0 / (cg->zeta * sum);
            const double tau = st[e] > 0.0 ? std::min(1.0 / st[e], thin) : thin;
            const double wt = ctx->h_w[a] * tau / ctx->sum_weights;
            for (int c = 0; c < 3; c++)
               for (int c2 = 0; c2 < 3; c2++) De[3 * c + c2] += wt * om[c] * om[c2];
         }
      }
      const double sa = st[e] - ss[e];
      for (size_t ij = 0; ij < n2; ij++) {
         double v = sa * cg->mass[e * n2 + ij];
         for (int k = 0; k < 9; k++) v += De[k] * cg->stiff[(e * n2 + ij) * 9 + k];
         ds->h_val[ds->entry[e * n2 + ij]] += v;
      }
   }
   ds->h_jinv.assign(ds->n_nodes, 0.0);
   for (int64_t i = 0; i < ds->n_nodes; i++) {
      double diag = 0.0;
      for (int64_t k = ds->rp[i]; k < ds->rp[i + 1]; k++)
         if (ds->col[k] == i) {
            ds->h_val[k] += ds->vacuum_weight[i];
            diag = ds->h_val[k];
         }
      ds->h_jinv[i] = diag != 0.0 ? 1.0 / diag : 0.0;
   }
   return UBOLT_OK;
}

int DsaSolveOnDevice(ubolt_ctx *ctx, cudaStream_t s)
{
   ubolt_dsa *ds = ctx->dsa;
   const int64_t nn = ds->n_nodes;
   const int bl = kDsaThreads;
   const int64_t grid = (nn + bl - 1) / bl;
   cudaMemsetAsync(ds->scal, 0, kDsaScalars * sizeof(double), s);
   CgStartKernel<<<grid, bl, 0, s>>>(nn, ds->nb, ds->jinv, ds->rhs, ds->u, ds->r, ds->z, ds->p, ds->scal);
   CountLaunch();
   for (int it = 0; it < ds->inner_its; it++) {
      DsaSpmvLaunch(ctx, ds, ds->p, ds->q, ds->p, ds->scal, s);
      CgUpdateKernel<<<grid, bl, 0, s>>>(nn, ds->p, ds->q, ds->u, ds->r, ds->scal);
      CgPrecondKernel<<<grid, bl, 0, s>>>(nn, ds->nb, ds->jinv, ds->r, ds->z, ds->scal);
      CgDirectionKernel<<<grid, bl, 0, s>>>(nn, ds->z, ds->p, ds->scal);
      CgRotateScalars<<<1, 1, 0, s>>>(ds->scal);
      CountLaunch(5);
   }
   return CheckLaunch("dsa solve");
}

// The per-cell void mask of the current group, or NULL (no DSA filled, or no masked void)
static const uint8_t *DsaMask(const ubolt_ctx *ctx)
{
   return (ctx->dsa && ctx->dsa->assembled) ? ctx->dsa->mask : nullptr;
}

static int CheckDsa(ubolt_ctx *ctx)
{
   if (!ctx->dsa) return SetError(UBOLT_ERR_STATE, "no DSA - call ubolt_dsa_setup first");
   if (!ctx->dsa->assembled) return SetError(UBOLT_ERR_STATE, "DSA not filled for a group - call ubolt_dsa_set_group");
   return UBOLT_OK;
}

template <typename T>
int OperatorApply(ubolt_ctx *ctx, bool adjoint, const T *x, T *y, void *stream);

// The multiplicative DSA stage after the sweep, its residual formed with the
// operator itself (PCSetUseAmat, transport_solverk.kokkos.cxx:280-289):
// y += P D^{-1} R (r - A y)
template <typename T>
int DsaCorrect(ubolt_ctx *ctx, const T *r, T *y, T *tmp, void *stream)
{
   int rc = CheckDsa(ctx);
   if (rc) return rc;
   cudaStream_t s = (cudaStream_t)stream;
   ubolt_dsa *ds = ctx->dsa;
   if ((rc = OperatorApply<T>(ctx, false, y, tmp, stream))) return rc;
   DsaRestrictKernel<T><<<RunGrid(ds->n_nodes), 256, 0, s>>>(ds->n_nodes, ds->nb, ctx->A, ctx->geom<double>().w, ctx->d_volume,
                                                              r, tmp, ds->mask, ds->rhs);
   CountLaunch();
   if ((rc = DsaSolveOnDevice(ctx, s))) return rc;
   DsaProlongKernel<T><<<RunGrid(ctx->n_nodes), 256, 0, s>>>(ctx->n_nodes, ds->nb, ctx->A, 1.0 / ctx->sum_weights,
                                                                  ds->u, ds->mask, y, 1);
   return CheckLaunch("dsa correct");
}
template int DsaCorrect<double>(ubolt_ctx *, const double *, double *, double *, void *);
template int DsaCorrect<float>(ubolt_ctx *, const float *, float *, float *, void *);

}  // namespace ubolt

using namespace ubolt;

void UboltDsaFree(ubolt_ctx *ctx)
{
   ubolt_dsa *ds = ctx->dsa;
   if (!ds) return;
   for (void *p : {(void *)ds->val, (void *)ds->jinv, (void *)ds->rhs, (void *)ds->u, (void *)ds->r, (void *)ds->z,
                   (void *)ds->p, (void *)ds->q, (void *)ds->scal, (void *)ds->mask, (void *)ds->d_rp,
                   (void *)ds->d_col})
      if (p) cudaFree(p);
   delete ds;
   ctx->dsa = nullptr;
}

extern "C" void ubolt_dsa_defaults(ubolt_dsa_options *o)
{
   if (!o) return;
   o->penalty = 4.0;
   o->consistent_power = 1.5;
   o->consistent_d = 1;
   o->inner_iterations = 30;
   o->void_sigma_t = 0.0;
   o->void_d = 0.0;
   o->void_bridge = 1;
   o->pad_ = 0;
}

// Device storage of one DSA: the operator's values (n_val), the Jacobi
// inverses (n_jinv) and the inner solve's vectors and scalars
static int AllocDsa(ubolt_dsa *ds, size_t n_val, size_t n_jinv)
{
   auto alloc = [&](double **p, size_t n) -> int {
      const cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(double));
      if (e != cudaSuccess) {
         cudaGetLastError();
         return SetError(UBOLT_ERR_NOMEM, "DSA workspace: %s", cudaGetErrorString(e));
      }
      return UBOLT_OK;
   };
   const size_t nn = (size_t)ds->n_nodes;
   int rc = 0;
   if ((rc = alloc(&ds->val, n_val)) || (rc = alloc(&ds->jinv, n_jinv)) || (rc = alloc(&ds->rhs, nn)) ||
       (rc = alloc(&ds->u, nn)) || (rc = alloc(&ds->r, nn)) || (rc = alloc(&ds->z, nn)) || (rc = alloc(&ds->p, nn)) ||
       (rc = alloc(&ds->q, nn)) || (rc = alloc(&ds->scal, kDsaScalars + (nn + kDsaThreads - 1) / kDsaThreads)))
      return rc;
   return UBOLT_OK;
}

// DSACG::create (dsa_cgk.kokkos.cxx:114-203) on the context's CG tables: the
// vertex CSR pattern (each vertex's star vertices, sorted), the entry of
// every (element, li, j), and each vertex's vacuum weight - over its vacuum
// boundary faces, the incoming half-range current times A_f / n_fv
static int CgDsaSetup(ubolt_ctx *ctx, const ubolt_dsa_options &o)
{
   UboltDsaFree(ctx);
   auto ds = new ubolt_dsa();
   ctx->dsa = ds;
   const ubolt_cg *cg = ctx->cg;
   const int nv = cg->nv, F = cg->F, A = ctx->A;
   const int64_t ne = cg->n_elements, nvx = cg->n_vertices;
   const size_t n2 = (size_t)nv * nv;
   ds->cg = true;
   ds->nb = 1;
   ds->F = F;
   ds->nc = ne;
   ds->n_nodes = nvx;
   ds->inner_its = o.inner_iterations;
   ds->void_sigma_t = o.void_sigma_t;
   ds->void_d = o.void_d;
   ds->void_bridge = o.void_bridge != 0;
   ds->volume = cg->volume;
   ds->nbr = cg->elem_face_neighbour;
   ds->bc = cg->elem_face_bc;
   ds->area = cg->elem_face_area;
   for (int64_t k = 0; k < ne * F; k++)
      if (ds->nbr[k] < 0 && ds->bc[k] == UBOLT_BC_VACUUM) ds->any_vacuum = true;
   std::vector<std::vector<int32_t>> cols(nvx);
   for (int64_t e = 0; e < ne; e++)
      for (int li = 0; li < nv; li++)
         for (int j = 0; j < nv; j++) cols[cg->elem_vertex[e * nv + li]].push_back((int32_t)cg->elem_vertex[e * nv + j]);
   ds->rp.assign(nvx + 1, 0);
   for (int64_t i = 0; i < nvx; i++) {
      std::sort(cols[i].begin(), cols[i].end());
      cols[i].erase(std::unique(cols[i].begin(), cols[i].end()), cols[i].end());
      ds->rp[i + 1] = ds->rp[i] + (int64_t)cols[i].size();
   }
   ds->col.resize(ds->rp[nvx]);
   for (int64_t i = 0; i < nvx; i++) std::copy(cols[i].begin(), cols[i].end(), ds->col.begin() + ds->rp[i]);
   ds->entry.resize(ne * n2);
   for (int64_t e = 0; e < ne; e++)
      for (int li = 0; li < nv; li++) {
         const int64_t i = cg->elem_vertex[e * nv + li];
         for (int j = 0; j < nv; j++) {
            const int32_t c = (int32_t)cg->elem_vertex[e * nv + j];
            ds->entry[e * n2 + li * nv + j] = std::lower_bound(cols[i].begin(), cols[i].end(), c) - cols[i].begin() +
                                              ds->rp[i];
         }
      }
   ds->vacuum_weight.assign(nvx, 0.0);
   for (int64_t i = 0; i < nvx; i++)
      for (int64_t f = cg->bface_offset[i]; f < cg->bface_offset[i + 1]; f++) {
         if (cg->bface_bc[f] != UBOLT_BC_VACUUM) continue;
         const double *nA = &cg->bface_nA[3 * f];
         const double area = std::sqrt(nA[0] * nA[0] + nA[1] * nA[1] + nA[2] * nA[2]);
         double m = 0.0;
         for (int a = 0; a < A; a++) {
            const double *om = &ctx->h_omega[3 * a];
            const double cosv = -(om[0] * nA[0] + om[1] * nA[1] + om[2] * nA[2]) / area;
            if (cosv > 0.0) m += ctx->h_w[a] * cosv;
         }
         m /= ctx->sum_weights;
         ds->vacuum_weight[i] += m * cg->bface_mass[f] * cg->lumped[i] * area;
      }
   int rc = AllocDsa(ds, ds->col.size(), (size_t)nvx);
   if (!rc && (cudaMalloc((void **)&ds->d_rp, ds->rp.size() * sizeof(int64_t)) != cudaSuccess ||
               cudaMalloc((void **)&ds->d_col, std::max<size_t>(ds->col.size(), 1) * sizeof(int32_t)) != cudaSuccess)) {
      cudaGetLastError();
      rc = SetError(UBOLT_ERR_NOMEM, "DSA pattern");
   }
   if (!rc)
      rc = CudaCheck(cudaMemcpy(ds->d_rp, ds->rp.data(), ds->rp.size() * sizeof(int64_t), cudaMemcpyHostToDevice),
                     "dsa_setup");
   if (!rc)
      rc = CudaCheck(cudaMemcpy(ds->d_col, ds->col.data(), ds->col.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
                     "dsa_setup");
   if (rc) UboltDsaFree(ctx);
   return rc;
}

static int DsaOptions(const ubolt_dsa_options *opts, ubolt_dsa_options *o)
{
   ubolt_dsa_defaults(o);
   if (opts) *o = *opts;
   if (!(o->penalty > 0.0)) return SetError(UBOLT_ERR_ARG, "dsa penalty must be positive, got %g", o->penalty);
   if (!(o->consistent_power >= 1.0)) return SetError(UBOLT_ERR_ARG, "consistent-D power must be >= 1");
   if (o->inner_iterations < 1 || o->inner_iterations > 10000) return SetError(UBOLT_ERR_ARG, "inner iterations");
   if (!(o->void_d >= 0.0)) return SetError(UBOLT_ERR_ARG, "void D must be >= 0 (0: from the voids' chord)");
   return UBOLT_OK;
}

extern "C" int ubolt_dsa_setup(ubolt_ctx *ctx, const ubolt_dg_geometry *g, const ubolt_dsa_options *opts)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (ctx->cg) {
      if (g) return SetError(UBOLT_ERR_ARG, "dsa_setup: a CG-SUPG context holds its own tables - pass NULL");
      ubolt_dsa_options o;
      if ((rc = DsaOptions(opts, &o))) return rc;
      return CgDsaSetup(ctx, o);
   }
   if (!g) return SetError(UBOLT_ERR_ARG, "dsa_setup: NULL geometry");
   if (g->n_cells != ctx->n_cells || g->n_basis != ctx->nb || g->faces_per_cell != ctx->F)
      return SetError(UBOLT_ERR_ARG, "dsa_setup: the geometry is not the context's");
   if (ctx->nb > 1 && (!g->face_own || !g->face_up || !g->basis_grad || !g->face_neighbour_grad))
      return SetError(UBOLT_ERR_ARG, "dsa_setup: DG1 needs face matrices and basis gradients");
   if (!g->face_distance) return SetError(UBOLT_ERR_ARG, "dsa_setup: face distances missing");
   ubolt_dsa_options o;
   if ((rc = DsaOptions(opts, &o))) return rc;
   UboltDsaFree(ctx);
   auto ds = new ubolt_dsa();
   ctx->dsa = ds;
   const int nb = ctx->nb, F = ctx->F, A = ctx->A;
   const int64_t nc = ctx->n_cells, ns = nc * F;
   ds->nb = nb;
   ds->F = F;
   ds->nc = nc;
   ds->n_nodes = nc * nb;
   ds->penalty = o.penalty;
   ds->consistent = o.consistent_d;
   ds->power = o.consistent_power;
   ds->inner_its = o.inner_iterations;
   ds->void_sigma_t = o.void_sigma_t;
   ds->void_d = o.void_d;
   ds->void_bridge = o.void_bridge != 0;
   ds->volume.assign(g->volume, g->volume + nc);
   ds->nbr.assign(g->face_neighbour, g->face_neighbour + ns);
   ds->bc.assign(g->face_bc, g->face_bc + ns);
   ds->dist.assign(g->face_distance, g->face_distance + 2 * ns);
   for (int64_t k = 0; k < ns; k++)
      if (ds->nbr[k] < 0 && ds->bc[k] == UBOLT_BC_VACUUM) ds->any_vacuum = true;
   ds->area.resize(ns);
   ds->nrm.resize(3 * ns);
   for (int64_t k = 0; k < ns; k++) {
      double a = 0.0;
      for (int d = 0; d < 3; d++) a += g->face_nA[3 * k + d] * g->face_nA[3 * k + d];
      ds->area[k] = std::sqrt(a);
      for (int d = 0; d < 3; d++) ds->nrm[3 * k + d] = g->face_nA[3 * k + d] / ds->area[k];
   }
   if (nb > 1) {
      ds->fown.assign(g->face_own, g->face_own + ns * nb * nb);
      ds->fup.assign(g->face_up, g->face_up + ns * nb * nb);
      ds->bgrad.assign(g->basis_grad, g->basis_grad + nc * nb * 3);
      ds->nbgrad.assign(g->face_neighbour_grad, g->face_neighbour_grad + ns * nb * 3);
   } else {
      // The consistent D's half-range current per face slot, off the same ordinates
      ds->half_range.resize(ns);
      for (int64_t k = 0; k < ns; k++) {
         double sum = 0.0;
         for (int a = 0; a < A; a++) {
            double dot = 0.0;
            for (int d = 0; d < 3; d++) dot += ctx->h_omega[3 * a + d] * g->face_nA[3 * k + d];
            dot /= ds->area[k];
            if (dot > 0.0) sum += ctx->h_w[a] * dot;
         }
         ds->half_range[k] = sum / ctx->sum_weights;
      }
   }
   const size_t bs = (size_t)nb * nb;
   if ((rc = AllocDsa(ds, nc * (F + 1) * bs, nc * bs))) {
      UboltDsaFree(ctx);
      return rc;
   }
   if (cudaMalloc((void **)&ds->mask, std::max<int64_t>(nc, 1)) != cudaSuccess) {
      cudaGetLastError();
      ds->mask = nullptr;
      UboltDsaFree(ctx);
      return SetError(UBOLT_ERR_NOMEM, "DSA void mask");
   }
   return UBOLT_OK;
}

extern "C" int ubolt_dsa_set_group(ubolt_ctx *ctx, void *stream)
{
   int rc = CheckReady(ctx, true);
   if (rc) return rc;
   if (!ctx->dsa) return SetError(UBOLT_ERR_STATE, "no DSA - call ubolt_dsa_setup first");
   ubolt_dsa *ds = ctx->dsa;
   cudaStream_t s = (cudaStream_t)stream;
   // The assembly is a host loop (DSAHostCopy then DSAPlex::assemble in the reference)
   std::vector<double> st(ds->nc), ss(ds->nc);
   cudaMemcpyAsync(st.data(), ctx->g64.sigma_t, ds->nc * 8, cudaMemcpyDeviceToHost, s);
   cudaMemcpyAsync(ss.data(), ctx->g64.sigma_s, ds->nc * 8, cudaMemcpyDeviceToHost, s);
   if ((rc = CudaCheck(cudaStreamSynchronize(s), "dsa_set_group"))) return rc;
   if ((rc = ds->cg ? AssembleCg(ctx, ds, st.data(), ss.data()) : Assemble(ds, st.data(), ss.data()))) return rc;
   cudaMemcpyAsync(ds->val, ds->h_val.data(), ds->h_val.size() * 8, cudaMemcpyHostToDevice, s);
   cudaMemcpyAsync(ds->jinv, ds->h_jinv.data(), ds->h_jinv.size() * 8, cudaMemcpyHostToDevice, s);
   if (ds->mask) cudaMemcpyAsync(ds->mask, ds->h_mask.data(), ds->nc, cudaMemcpyHostToDevice, s);
   if ((rc = CudaCheck(cudaStreamSynchronize(s), "dsa upload"))) return rc;
   ds->assembled = true;
   return UBOLT_OK;
}

extern "C" int ubolt_dsa_void_info(ubolt_ctx *ctx, int64_t *n_void, int32_t *bridged, double *chord)
{
   int rc = CheckReady(ctx, false);
   if (rc || (rc = CheckDsa(ctx))) return rc;
   if (n_void) *n_void = ctx->dsa->n_void;
   if (bridged) *bridged = ctx->dsa->bridged;
   if (chord) *chord = ctx->dsa->chord;
   return UBOLT_OK;
}

extern "C" int ubolt_dsa_spmv(ubolt_ctx *ctx, const double *u, double *v, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc || (rc = CheckDsa(ctx))) return rc;
   if (!u || !v || u == v) return SetError(UBOLT_ERR_ARG, "dsa_spmv: u and v must be distinct device arrays");
   DsaSpmvLaunch(ctx, ctx->dsa, u, v, nullptr, nullptr, (cudaStream_t)stream);
   return CheckLaunch("dsa_spmv");
}

extern "C" int ubolt_dsa_restrict(ubolt_ctx *ctx, const double *x, double *rhs, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!x || !rhs) return SetError(UBOLT_ERR_ARG, "dsa_restrict: NULL array");
   DsaRestrictKernel<double><<<RunGrid(ctx->n_nodes), 256, 0, (cudaStream_t)stream>>>(
      ctx->n_nodes, ctx->nb, ctx->A, ctx->geom<double>().w, ctx->d_volume, x, nullptr, DsaMask(ctx), rhs);
   return CheckLaunch("dsa_restrict");
}

extern "C" int ubolt_dsa_prolong(ubolt_ctx *ctx, const double *u, double *y, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!u || !y) return SetError(UBOLT_ERR_ARG, "dsa_prolong: NULL array");
   DsaProlongKernel<double><<<RunGrid(ctx->n_nodes), 256, 0, (cudaStream_t)stream>>>(
      ctx->n_nodes, ctx->nb, ctx->A, 1.0 / ctx->sum_weights, u, DsaMask(ctx), y, 0);
   return CheckLaunch("dsa_prolong");
}

extern "C" int ubolt_dsa_apply(ubolt_ctx *ctx, const double *x, double *y, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc || (rc = CheckDsa(ctx))) return rc;
   if (!x || !y || x == y) return SetError(UBOLT_ERR_ARG, "dsa_apply: x and y must be distinct device arrays");
   cudaStream_t s = (cudaStream_t)stream;
   ubolt_dsa *ds = ctx->dsa;
   DsaRestrictKernel<double><<<RunGrid(ds->n_nodes), 256, 0, s>>>(ds->n_nodes, ds->nb, ctx->A, ctx->geom<double>().w,
                                                                   ctx->d_volume, x, nullptr, ds->mask, ds->rhs);
   CountLaunch();
   if ((rc = DsaSolveOnDevice(ctx, s))) return rc;
   DsaProlongKernel<double><<<RunGrid(ctx->n_nodes), 256, 0, s>>>(ctx->n_nodes, ds->nb, ctx->A,
                                                                      1.0 / ctx->sum_weights, ds->u, ds->mask, y, 0);
   return CheckLaunch("dsa_apply");
}

extern "C" int ubolt_dsa_matrix(ubolt_ctx *ctx, double *blocks)
{
   int rc = CheckReady(ctx, false);
   if (rc || (rc = CheckDsa(ctx))) return rc;
   if (!blocks) return SetError(UBOLT_ERR_ARG, "dsa_matrix: NULL output");
   if (ctx->dsa->cg) return SetError(UBOLT_ERR_STATE, "dsa_matrix: the CG-SUPG operator is CSR, read it by ubolt_dsa_spmv");
   std::copy(ctx->dsa->h_val.begin(), ctx->dsa->h_val.end(), blocks);
   return UBOLT_OK;
}

// ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
// The DSA apply with its scratch in a fixed device array instead of the
// context's workspace: for a caller that cannot have this library allocate
// device memory while it solves - typically an application whose own memory
// pool (a PETSc/Kokkos or framework allocator) has already reserved the
// device, so a cudaMalloc from a library underneath it would fail or break
// the pool's accounting. The array is part of the loaded library: every GPU
// that loads it holds these 12.6 MB until the process exits.
// ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

namespace {

// Six node vectors (restricted rhs and the PCG's u, r, z, p, q) of at most
// kStaticDsaNodes nodes each, then the scalars and one partial sum per block
constexpr int64_t kStaticDsaNodes = (int64_t)1 << 18;
constexpr int64_t kStaticDsaDoubles = 6 * kStaticDsaNodes + kDsaScalars + kStaticDsaNodes / kDsaThreads;
static __device__ __align__(256) double g_dsa_scratch[kStaticDsaDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_dsa_scratch_mutex;
double *g_dsa_scratch_addr[kMaxDevices] = {};

// The scratch array's device address on the current device. The symbol's
// name in host code is a host-side stand-in, not a device address, so the
// address is fetched once per device with cudaGetSymbolAddress while that
// device is current.
int StaticScratch(int device, double **out)
{
   if (device < 0 || device >= kMaxDevices) return SetError(UBOLT_ERR_ARG, "device %d out of range", device);
   std::lock_guard<std::mutex> lock(g_dsa_scratch_mutex);
   if (!g_dsa_scratch_addr[device]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_dsa_scratch);
      if (e != cudaSuccess) return CudaCheck(e, "cudaGetSymbolAddress(dsa scratch)");
      g_dsa_scratch_addr[device] = static_cast<double *>(p);
   }
   *out = g_dsa_scratch_addr[device];
   return UBOLT_OK;
}

}  // namespace

extern "C" int ubolt_dsa_apply_static(ubolt_ctx *ctx, const double *x, double *y, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc || (rc = CheckDsa(ctx))) return rc;
   if (!x || !y || x == y) return SetError(UBOLT_ERR_ARG, "dsa_apply_static: x and y must be distinct device arrays");
   ubolt_dsa *ds = ctx->dsa;
   if (ds->n_nodes > kStaticDsaNodes)
      return SetError(UBOLT_ERR_ARG,
                      "dsa_apply_static: %lld nodes exceed the fixed scratch of %lld nodes - use ubolt_dsa_apply",
                      (long long)ds->n_nodes, (long long)kStaticDsaNodes);
   double *base = nullptr;
   if ((rc = StaticScratch(ctx->device, &base))) return rc;
   const int64_t nn = kStaticDsaNodes;
   double *rhs = base, *u = base + nn, *r = base + 2 * nn, *z = base + 3 * nn, *p = base + 4 * nn, *q = base + 5 * nn;
   double *scal = base + 6 * nn;
   cudaStream_t s = (cudaStream_t)stream;
   DsaRestrictKernel<double><<<RunGrid(ds->n_nodes), 256, 0, s>>>(ds->n_nodes, ds->nb, ctx->A, ctx->geom<double>().w,
                                                                   ctx->d_volume, x, nullptr, ds->mask, rhs);
   CountLaunch();
   // The same fixed-count block-Jacobi PCG as the workspace path; the
   // scalars are cleared here, every vector is written before it is read
   const int64_t nodes = ds->n_nodes;
   const int64_t grid = (nodes + 255) / 256;
   if ((rc = CudaCheck(cudaMemsetAsync(scal, 0, kDsaScalars * sizeof(double), s), "dsa_apply_static"))) return rc;
   CgStartKernel<<<grid, 256, 0, s>>>(nodes, ds->nb, ds->jinv, rhs, u, r, z, p, scal);
   CountLaunch();
   for (int it = 0; it < ds->inner_its; it++) {
      DsaSpmvLaunch(ctx, ds, p, q, p, scal, s);
      CgUpdateKernel<<<grid, 256, 0, s>>>(nodes, p, q, u, r, scal);
      CgPrecondKernel<<<grid, 256, 0, s>>>(nodes, ds->nb, ds->jinv, r, z, scal);
      CgDirectionKernel<<<grid, 256, 0, s>>>(nodes, z, p, scal);
      CgRotateScalars<<<1, 1, 0, s>>>(scal);
      CountLaunch(5);
   }
   DsaProlongKernel<double><<<RunGrid(ctx->n_nodes), 256, 0, s>>>(ctx->n_nodes, ds->nb, ctx->A,
                                                                      1.0 / ctx->sum_weights, u, ds->mask, y, 0);
   return CheckLaunch("dsa_apply_static");
}
