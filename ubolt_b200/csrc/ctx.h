// The device context behind ubolt_ctx and the launch helpers every CUDA
// translation unit of the library shares.
#pragma once

#include "device.cuh"
#include "ubolt_internal.h"

#include <cuda_runtime.h>

#include <vector>

struct ubolt_sweep_plan;
struct ubolt_dsa;
struct ubolt_solver;
struct ubolt_cg;

struct ubolt_ctx {
   int device = 0;
   int dim = 0, nb = 1, F = 0, A = 0;
   int64_t n_cells = 0, n_rows = 0, n_nodes = 0, n_classes = 0;
   double sum_weights = 0.0;
   int32_t side_bc[6] = {0, 0, 0, 0, 0, 0};
   bool has_reflect = false;

   // Host copies kept for set-up work (sweep plans, DSA assembly)
   std::vector<double> h_omega, h_w, h_volume, h_nA;
   std::vector<int32_t> h_refl, h_code, h_cls;
   std::vector<int8_t> h_mirror;
   std::vector<int32_t> h_opp;  // the opposite ordinate of each ordinate

   // Device allocations (owned)
   std::vector<void *> owned;
   ubolt::DevGeom<double> g64{};
   ubolt::DevGeom<float> g32{};
   float *sigma_t32 = nullptr, *sigma_s32 = nullptr;
   const double *d_volume = nullptr;           // [n_cells] FP64 cell volumes (CG-SUPG: [n_nodes] lumped masses)
   const int32_t *d_opp = nullptr;             // [A] the ordinate opposite each ordinate
   const double *d_p1 = nullptr;               // [A][dim] T^{-1} Omega_a, T = sum_a w_a Omega_a Omega_a^T
   bool p1_ok = false;                         // sum_a w_a Omega_a = 0 and T regular (the P1 expansion exists)
   const double *d_w_omega = nullptr;          // [A][dim] w_a Omega_a
   unsigned long long *d_counters = nullptr;   // 64 counters/flags for set-up calls
   bool group_set = false;
   uint64_t group_epoch = 0;  // bumped by every ubolt_set_group: caches keyed on the cross sections

   ubolt_sweep_plan *sweep = nullptr;
   ubolt_dsa *dsa = nullptr;
   ubolt_solver *solver = nullptr;
   // The CG-SUPG backend's tables, or NULL for a DG context. A CG context's
   // nodes are the mesh's vertices (nb 1) and its cells the elements, the
   // unit cross sections are given on; the DG geometry above is unset.
   ubolt_cg *cg = nullptr;

   template <typename T>
   const ubolt::DevGeom<T> &geom() const;
};

template <>
inline const ubolt::DevGeom<double> &ubolt_ctx::geom<double>() const
{
   return g64;
}
template <>
inline const ubolt::DevGeom<float> &ubolt_ctx::geom<float>() const
{
   return g32;
}

namespace ubolt {

int CheckLaunch(const char *what);
// Count kernels launched by the library (ubolt_launch_count)
void CountLaunch(int n = 1);
int CudaCheck(cudaError_t e, const char *what);
// Context exists (and, with need_group, has cross sections) and its device is current
int CheckReady(const ubolt_ctx *ctx, bool need_group);
// Device allocation owned by the context, freed by ubolt_ctx_destroy
int CtxAlloc(ubolt_ctx *ctx, size_t bytes, void **p);
// The ordinates, the opposite map, the P1 tables, the FP32 cross-section
// slots (ctx->n_cells each) and the counters; ctx->dim, n_cells and
// sum_weights set first
int UploadOrdinates(ubolt_ctx *ctx, const ubolt_quadrature *quad);
// A context of the DG backend: UBOLT_ERR_STATE naming `what` on a CG-SUPG one
int RequireDg(const ubolt_ctx *ctx, const char *what);

}  // namespace ubolt

// The kernel families are templated on the basis count and the faces per
// cell; a mesh picks one instantiation at run time.
#define UBOLT_DISPATCH(nb_, f_, ...)                                                      \
   do {                                                                                   \
      if ((nb_) == 1 && (f_) == 3) { constexpr int NB_ = 1, F_ = 3; __VA_ARGS__; }        \
      else if ((nb_) == 1 && (f_) == 4) { constexpr int NB_ = 1, F_ = 4; __VA_ARGS__; }   \
      else if ((nb_) == 1 && (f_) == 6) { constexpr int NB_ = 1, F_ = 6; __VA_ARGS__; }   \
      else if ((nb_) == 3 && (f_) == 3) { constexpr int NB_ = 3, F_ = 3; __VA_ARGS__; }   \
      else if ((nb_) == 3 && (f_) == 4) { constexpr int NB_ = 3, F_ = 4; __VA_ARGS__; }   \
      else if ((nb_) == 4 && (f_) == 4) { constexpr int NB_ = 4, F_ = 4; __VA_ARGS__; }   \
      else if ((nb_) == 4 && (f_) == 6) { constexpr int NB_ = 4, F_ = 6; __VA_ARGS__; }   \
   } while (0)
