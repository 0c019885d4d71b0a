// ubolt_ctx: geometry and ordinates uploaded once, geometry classes, the
// FP32 mirror, and the per-group cross-section pointers.
#include "ctx.h"

#include <cmath>

#include <atomic>
#include <cstring>
#include <unordered_map>

namespace ubolt {

int CudaCheck(cudaError_t e, const char *what)
{
   if (e == cudaSuccess) return UBOLT_OK;
   return SetError(UBOLT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

static std::atomic<uint64_t> g_launches{0};

void CountLaunch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

// Every launch wrapper calls this once per kernel it launched
int CheckLaunch(const char *what)
{
   CountLaunch(1);
   return CudaCheck(cudaGetLastError(), what);
}

int CheckReady(const ubolt_ctx *ctx, bool need_group)
{
   if (!ctx) return SetError(UBOLT_ERR_ARG, "NULL context");
   if (need_group && !ctx->group_set)
      return SetError(UBOLT_ERR_STATE, "no group cross sections - call ubolt_set_group first");
   int dev = -1;
   if (cudaGetDevice(&dev) != cudaSuccess || dev != ctx->device) {
      const cudaError_t e = cudaSetDevice(ctx->device);
      if (e != cudaSuccess) return CudaCheck(e, "cudaSetDevice");
   }
   return UBOLT_OK;
}

int RequireDg(const ubolt_ctx *ctx, const char *what)
{
   if (ctx && ctx->cg)
      return SetError(UBOLT_ERR_STATE, "%s is not defined on the CG-SUPG backend (no upwind sweep, no transpose)",
                      what);
   return UBOLT_OK;
}

int CtxAlloc(ubolt_ctx *ctx, size_t bytes, void **p)
{
   *p = nullptr;
   if (bytes == 0) bytes = 16;
   const cudaError_t e = cudaMalloc(p, bytes);
   if (e != cudaSuccess) {
      cudaGetLastError();
      return SetError(UBOLT_ERR_NOMEM, "cudaMalloc of %zu bytes: %s", bytes, cudaGetErrorString(e));
   }
   ctx->owned.push_back(*p);
   return UBOLT_OK;
}

template <typename T>
static int Upload(ubolt_ctx *ctx, const std::vector<T> &h, const T **d)
{
   void *p = nullptr;
   int rc = CtxAlloc(ctx, h.size() * sizeof(T), &p);
   if (rc) return rc;
   if (!h.empty()) {
      rc = CudaCheck(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
      if (rc) return rc;
   }
   *d = static_cast<const T *>(p);
   return UBOLT_OK;
}

static std::vector<float> ToF32(const std::vector<double> &v)
{
   std::vector<float> o(v.size());
   for (size_t i = 0; i < v.size(); i++) o[i] = (float)v[i];
   return o;
}

// 64-bit FNV-1a over a byte range
static uint64_t Fnv(const void *p, size_t n, uint64_t h)
{
   const unsigned char *b = static_cast<const unsigned char *>(p);
   for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
   return h;
}

template <typename T>
__global__ void ToFloatKernel(const T *__restrict__ in, float *__restrict__ out, int64_t n)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i < n) out[i] = (float)in[i];
}

// The ordinates in both precisions (omega, w, the reflection maps), the
// opposite of each ordinate, the P1 expansion's tables, the per-group FP32
// cross-section slots (n_cells each) and the set-up counters: what every
// context holds whatever its discretisation.
int UploadOrdinates(ubolt_ctx *ctx, const ubolt_quadrature *quad)
{
   const int A = quad->n_angles, dim = ctx->dim;
   int rc = 0;
   DevGeom<double> &g = ctx->g64;
   DevGeom<float> &h = ctx->g32;
   ctx->h_omega.assign(quad->omega, quad->omega + 3 * A);
   ctx->h_w.assign(quad->w, quad->w + A);
   ctx->h_refl.assign(3 * A, 0);
   for (int d = 0; d < 3 * A; d++) ctx->h_refl[d] = (d < dim * A) ? quad->reflect[d] : 0;
   for (int d = 0; d < dim * A; d++)
      if (ctx->h_refl[d] < 0 || ctx->h_refl[d] >= A) return SetError(UBOLT_ERR_ARG, "bad reflection map");
   if ((rc = Upload(ctx, ctx->h_omega, &g.omega)) || (rc = Upload(ctx, ToF32(ctx->h_omega), &h.omega))) return rc;
   if ((rc = Upload(ctx, ctx->h_w, &g.w)) || (rc = Upload(ctx, ToF32(ctx->h_w), &h.w))) return rc;
   if ((rc = Upload(ctx, ctx->h_refl, &g.refl))) return rc;
   h.refl = g.refl;
   void *p = nullptr;
   if ((rc = CtxAlloc(ctx, ctx->n_cells * sizeof(float), &p))) return rc;
   ctx->sigma_t32 = static_cast<float *>(p);
   if ((rc = CtxAlloc(ctx, ctx->n_cells * sizeof(float), &p))) return rc;
   ctx->sigma_s32 = static_cast<float *>(p);
   h.sigma_t = ctx->sigma_t32;
   h.sigma_s = ctx->sigma_s32;
   {
      // The opposite ordinate (every cosine negated), by exact search
      std::vector<int32_t> opp(A, -1);
      for (int a = 0; a < A; a++)
         for (int b = 0; b < A; b++)
            if (ctx->h_omega[3 * b] == -ctx->h_omega[3 * a] && ctx->h_omega[3 * b + 1] == -ctx->h_omega[3 * a + 1] &&
                ctx->h_omega[3 * b + 2] == -ctx->h_omega[3 * a + 2]) {
               opp[a] = b;
               break;
            }
      for (int a = 0; a < A; a++)
         if (opp[a] < 0 || ctx->h_w[opp[a]] != ctx->h_w[a])
            return SetError(UBOLT_ERR_ARG, "ordinate %d has no opposite of equal weight", a);
      if ((rc = Upload(ctx, opp, &ctx->d_opp))) return rc;
      g.opp = h.opp = ctx->d_opp;
      ctx->h_opp = opp;
   }
   {
      // The P1 expansion's tables: w_a Omega_a, and p1(a) = T^{-1} Omega_a
      // with T = sum_a w_a Omega_a Omega_a^T, inverted by Gauss-Jordan
      // (dim <= 3); usable where sum_a w_a Omega_a vanishes
      const int D = ctx->dim;
      double t[3][3] = {}, first[3] = {}, inv[3][3] = {};
      for (int a = 0; a < A; a++)
         for (int d = 0; d < D; d++) {
            first[d] += ctx->h_w[a] * ctx->h_omega[3 * a + d];
            for (int e = 0; e < D; e++) t[d][e] += ctx->h_w[a] * ctx->h_omega[3 * a + d] * ctx->h_omega[3 * a + e];
         }
      bool ok = true;
      for (int d = 0; d < D; d++) ok &= std::fabs(first[d]) <= 1e-12 * std::fabs(ctx->sum_weights);
      for (int d = 0; d < D; d++) inv[d][d] = 1.0;
      for (int k = 0; k < D && ok; k++) {
         int piv = k;
         for (int i = k + 1; i < D; i++)
            if (std::fabs(t[i][k]) > std::fabs(t[piv][k])) piv = i;
         if (!(std::fabs(t[piv][k]) > 0.0)) {
            ok = false;
            break;
         }
         for (int j = 0; j < 3; j++) {
            std::swap(t[k][j], t[piv][j]);
            std::swap(inv[k][j], inv[piv][j]);
         }
         const double r = 1.0 / t[k][k];
         for (int j = 0; j < D; j++) {
            t[k][j] *= r;
            inv[k][j] *= r;
         }
         for (int i = 0; i < D; i++) {
            if (i == k) continue;
            const double f = t[i][k];
            for (int j = 0; j < D; j++) {
               t[i][j] -= f * t[k][j];
               inv[i][j] -= f * inv[k][j];
            }
         }
      }
      std::vector<double> p1((size_t)A * D, 0.0), wom((size_t)A * D, 0.0);
      for (int a = 0; a < A; a++)
         for (int d = 0; d < D; d++) {
            wom[(size_t)a * D + d] = ctx->h_w[a] * ctx->h_omega[3 * a + d];
            double sum = 0.0;
            for (int e = 0; e < D; e++) sum += inv[d][e] * ctx->h_omega[3 * a + e];
            p1[(size_t)a * D + d] = sum;
         }
      if ((rc = Upload(ctx, p1, &ctx->d_p1)) || (rc = Upload(ctx, wom, &ctx->d_w_omega))) return rc;
      ctx->p1_ok = ok;
   }
   if ((rc = CtxAlloc(ctx, 64 * sizeof(unsigned long long), &p))) return rc;
   ctx->d_counters = static_cast<unsigned long long *>(p);
   return UBOLT_OK;
}

}  // namespace ubolt

using namespace ubolt;

extern "C" int ubolt_ctx_create(const ubolt_dg_geometry *geom, const ubolt_quadrature *quad, ubolt_ctx **out)
{
   ClearError();
   if (!out || !geom || !quad) return SetError(UBOLT_ERR_ARG, "ubolt_ctx_create: NULL argument");
   *out = nullptr;
   const int dim = geom->dim, nb = geom->n_basis, F = geom->faces_per_cell, A = quad->n_angles;
   const int64_t nc = geom->n_cells;
   if (dim != 2 && dim != 3) return SetError(UBOLT_ERR_ARG, "dimension %d", dim);
   if (quad->dim != dim) return SetError(UBOLT_ERR_ARG, "a %dD quadrature was handed to a %dD mesh", quad->dim, dim);
   if (nb != 1 && nb != dim + 1) return SetError(UBOLT_ERR_ARG, "n_basis %d is neither DG0 nor DG1", nb);
   if (F < 3 || F > kMaxFaces) return SetError(UBOLT_ERR_ARG, "faces per cell %d", F);
   if (A <= 0 || A > 1024) return SetError(UBOLT_ERR_ARG, "n_angles %d (1..1024)", A);
   if (nc <= 0 || nc * nb * (int64_t)A >= ((int64_t)1 << 31) * 8)
      return SetError(UBOLT_ERR_ARG, "n_cells %lld out of range", (long long)nc);
   if (!geom->face_nA || !geom->face_neighbour || !geom->face_bc || !geom->face_side || !geom->volume)
      return SetError(UBOLT_ERR_ARG, "geometry arrays missing");
   if (nb > 1 && (!geom->face_own || !geom->face_up || !geom->basis_grad || !geom->face_basis_value))
      return SetError(UBOLT_ERR_ARG, "DG1 geometry needs face_own, face_up, basis_grad and face_basis_value");
   if (!quad->omega || !quad->w || !quad->reflect) return SetError(UBOLT_ERR_ARG, "quadrature arrays missing");
   {
      bool found = false;
      UBOLT_DISPATCH(nb, F, found = true);
      if (!found) return SetError(UBOLT_ERR_ARG, "no kernels for n_basis %d with %d faces per cell", nb, F);
   }

   auto ctx = new ubolt_ctx();
   auto fail = [&](int rc) {
      ubolt_ctx_destroy(ctx);
      return rc;
   };
   cudaGetDevice(&ctx->device);
   ctx->dim = dim;
   ctx->nb = nb;
   ctx->F = F;
   ctx->A = A;
   ctx->n_cells = nc;
   ctx->n_rows = nc * nb * A;
   ctx->n_nodes = nc * nb;
   ctx->sum_weights = quad->sum_weights;

   // ~~~~~ Per-cell face codes, mirror slots, the sides' families
   const int64_t ns = nc * F;
   ctx->h_code.resize(ns);
   ctx->h_mirror.assign(ns, -1);
   for (int i = 0; i < 6; i++) ctx->side_bc[i] = UBOLT_BC_VACUUM;
   for (int64_t k = 0; k < ns; k++) {
      const int64_t n = geom->face_neighbour[k];
      if (n >= 0) {
         if (n >= nc) return fail(SetError(UBOLT_ERR_ARG, "face %lld names cell %lld", (long long)k, (long long)n));
         ctx->h_code[k] = (int32_t)n;
      } else {
         const int side = geom->face_side[k];
         if (side < 0 || side >= 2 * dim)
            return fail(SetError(UBOLT_ERR_ARG, "boundary face %lld has side %d", (long long)k, side));
         ctx->h_code[k] = -1 - side;
         ctx->side_bc[side] = geom->face_bc[k];
         if (geom->face_bc[k] == UBOLT_BC_REFLECT) ctx->has_reflect = true;
      }
   }
   for (int64_t k = 0; k < ns; k++) {
      const int64_t n = geom->face_neighbour[k];
      if (n < 0) continue;
      const int64_t c = k / F;
      for (int f = 0; f < F; f++)
         if (geom->face_neighbour[n * F + f] == c) { ctx->h_mirror[k] = (int8_t)f; break; }
      if (ctx->h_mirror[k] < 0)
         return fail(SetError(UBOLT_ERR_ARG, "cell %lld is not a neighbour of its neighbour %lld", (long long)c,
                              (long long)n));
   }

   // ~~~~~ Geometry classes: cells whose shape data are bitwise equal
   const size_t s_nA = (size_t)F * 3, s_m = (size_t)F * nb * nb, s_g = (size_t)nb * 3, s_v = (size_t)F * nb;
   auto same = [&](int64_t a, int64_t b) {
      if (std::memcmp(&geom->face_nA[a * s_nA], &geom->face_nA[b * s_nA], s_nA * 8)) return false;
      if (geom->volume[a] != geom->volume[b]) return false;
      if (nb > 1) {
         if (std::memcmp(&geom->face_own[a * s_m], &geom->face_own[b * s_m], s_m * 8)) return false;
         if (std::memcmp(&geom->face_up[a * s_m], &geom->face_up[b * s_m], s_m * 8)) return false;
         if (std::memcmp(&geom->basis_grad[a * s_g], &geom->basis_grad[b * s_g], s_g * 8)) return false;
         if (std::memcmp(&geom->face_basis_value[a * s_v], &geom->face_basis_value[b * s_v], s_v * 8)) return false;
      }
      return true;
   };
   std::unordered_map<uint64_t, std::vector<int64_t>> buckets;
   std::vector<int64_t> rep;  // class -> representative cell
   ctx->h_cls.resize(nc);
   for (int64_t c = 0; c < nc; c++) {
      uint64_t h = 1469598103934665603ull;
      h = Fnv(&geom->face_nA[c * s_nA], s_nA * 8, h);
      h = Fnv(&geom->volume[c], 8, h);
      if (nb > 1) {
         h = Fnv(&geom->face_own[c * s_m], s_m * 8, h);
         h = Fnv(&geom->face_up[c * s_m], s_m * 8, h);
      }
      auto &bucket = buckets[h];
      int64_t cls = -1;
      for (int64_t cand : bucket)
         if (same(rep[cand], c)) { cls = cand; break; }
      if (cls < 0) {
         cls = (int64_t)rep.size();
         rep.push_back(c);
         bucket.push_back(cls);
      }
      ctx->h_cls[c] = (int32_t)cls;
   }
   const int64_t ncls = (int64_t)rep.size();
   ctx->n_classes = ncls;
   std::vector<double> nA(ncls * s_nA), fown, fup, bgrad, fbv, inv_vol(ncls);
   if (nb > 1) {
      fown.resize(ncls * s_m);
      fup.resize(ncls * s_m);
      bgrad.resize(ncls * s_g);
      fbv.resize(ncls * s_v);
   }
   for (int64_t q = 0; q < ncls; q++) {
      const int64_t c = rep[q];
      std::memcpy(&nA[q * s_nA], &geom->face_nA[c * s_nA], s_nA * 8);
      inv_vol[q] = 1.0 / geom->volume[c];
      if (nb > 1) {
         std::memcpy(&fown[q * s_m], &geom->face_own[c * s_m], s_m * 8);
         std::memcpy(&fup[q * s_m], &geom->face_up[c * s_m], s_m * 8);
         std::memcpy(&bgrad[q * s_g], &geom->basis_grad[c * s_g], s_g * 8);
         std::memcpy(&fbv[q * s_v], &geom->face_basis_value[c * s_v], s_v * 8);
      }
   }
   ctx->h_volume.assign(geom->volume, geom->volume + nc);
   ctx->h_nA.assign(geom->face_nA, geom->face_nA + nc * s_nA);

   // ~~~~~ Upload, FP64 and FP32
   int rc = 0;
   DevGeom<double> &g = ctx->g64;
   DevGeom<float> &h = ctx->g32;
   g.dim = h.dim = dim;
   g.nb = h.nb = nb;
   g.F = h.F = F;
   g.A = h.A = A;
   g.n_cells = h.n_cells = nc;
   g.sum_weights = quad->sum_weights;
   h.sum_weights = (float)quad->sum_weights;
   g.inv_sum_weights = 1.0 / quad->sum_weights;
   h.inv_sum_weights = (float)(1.0 / quad->sum_weights);
   for (int i = 0; i < 6; i++) g.side_bc[i] = h.side_bc[i] = ctx->side_bc[i];
   if ((rc = Upload(ctx, nA, &g.nA)) || (rc = Upload(ctx, ToF32(nA), &h.nA))) return fail(rc);
   if ((rc = Upload(ctx, inv_vol, &g.inv_vol)) || (rc = Upload(ctx, ToF32(inv_vol), &h.inv_vol))) return fail(rc);
   if (nb > 1) {
      if ((rc = Upload(ctx, fown, &g.fown)) || (rc = Upload(ctx, ToF32(fown), &h.fown))) return fail(rc);
      if ((rc = Upload(ctx, fup, &g.fup)) || (rc = Upload(ctx, ToF32(fup), &h.fup))) return fail(rc);
      if ((rc = Upload(ctx, bgrad, &g.bgrad)) || (rc = Upload(ctx, ToF32(bgrad), &h.bgrad))) return fail(rc);
      if ((rc = Upload(ctx, fbv, &g.fbv)) || (rc = Upload(ctx, ToF32(fbv), &h.fbv))) return fail(rc);
   }
   {
      // Packed records, one per class, for kernels that read a cell's shape data whole
      const RecordLayout L64(nb, F, 8), L32(nb, F, 4);
      std::vector<double> r64((size_t)ncls * L64.size, 0.0);
      std::vector<float> r32((size_t)ncls * L32.size, 0.0f);
      for (int64_t q = 0; q < ncls; q++) {
         double *d64 = &r64[(size_t)q * L64.size];
         float *d32 = &r32[(size_t)q * L32.size];
         // Offsets differ between the two: each part is padded to 16 bytes
         auto put = [&](int o64, int o32, double v) {
            d64[o64] = v;
            d32[o32] = (float)v;
         };
         for (int f = 0; f < F; f++) {
            for (int d = 0; d < 3; d++) put(L64.nA(f) + d, L32.nA(f) + d, nA[q * s_nA + f * 3 + d]);
            if (nb > 1)
               for (int k = 0; k < nb * nb; k++) {
                  put(L64.fown(f) + k, L32.fown(f) + k, fown[q * s_m + f * nb * nb + k]);
                  put(L64.fup(f) + k, L32.fup(f) + k, fup[q * s_m + f * nb * nb + k]);
               }
         }
         if (nb > 1)
            for (int k = 0; k < (int)s_g; k++) put(L64.bgrad() + k, L32.bgrad() + k, bgrad[q * s_g + k]);
         put(L64.ivol(), L32.ivol(), inv_vol[q]);
      }
      if ((rc = Upload(ctx, r64, &g.rec)) || (rc = Upload(ctx, r32, &h.rec))) return fail(rc);
   }
   if ((rc = Upload(ctx, ctx->h_cls, &g.cls))) return fail(rc);
   if ((rc = Upload(ctx, ctx->h_code, &g.code))) return fail(rc);
   if ((rc = Upload(ctx, ctx->h_mirror, &g.mirror))) return fail(rc);
   h.cls = g.cls;
   h.code = g.code;
   h.mirror = g.mirror;
   if ((rc = UploadOrdinates(ctx, quad))) return fail(rc);
   if ((rc = Upload(ctx, ctx->h_volume, &ctx->d_volume))) return fail(rc);
   g.volume = ctx->d_volume;
   if ((rc = Upload(ctx, ToF32(ctx->h_volume), &h.volume))) return fail(rc);
   if ((rc = CudaCheck(cudaDeviceSynchronize(), "ctx_create"))) return fail(rc);
   *out = ctx;
   return UBOLT_OK;
}

void UboltSweepFree(ubolt_ctx *ctx);
void UboltDsaFree(ubolt_ctx *ctx);
void UboltSolverFree(ubolt_ctx *ctx);
void UboltCgFree(ubolt_ctx *ctx);

extern "C" uint64_t ubolt_launch_count(void) { return g_launches.load(); }

extern "C" int ubolt_ctx_destroy(ubolt_ctx *ctx)
{
   if (!ctx) return UBOLT_OK;
   cudaSetDevice(ctx->device);
   cudaDeviceSynchronize();
   UboltSolverFree(ctx);
   UboltDsaFree(ctx);
   UboltSweepFree(ctx);
   UboltCgFree(ctx);
   for (void *p : ctx->owned) cudaFree(p);
   delete ctx;
   return UBOLT_OK;
}

extern "C" int ubolt_ctx_sizes(const ubolt_ctx *ctx, int64_t *rows, int64_t *nodes, int64_t *cells, int32_t *n_basis,
                               int32_t *n_angles)
{
   if (!ctx) return SetError(UBOLT_ERR_ARG, "NULL context");
   if (rows) *rows = ctx->n_rows;
   if (nodes) *nodes = ctx->n_nodes;
   if (cells) *cells = ctx->n_cells;
   if (n_basis) *n_basis = ctx->nb;
   if (n_angles) *n_angles = ctx->A;
   return UBOLT_OK;
}

extern "C" int ubolt_set_group(ubolt_ctx *ctx, const double *sigma_t, const double *sigma_s_within, void *stream)
{
   int rc = CheckReady(ctx, false);
   if (rc) return rc;
   if (!sigma_t || !sigma_s_within) return SetError(UBOLT_ERR_ARG, "set_group: NULL cross sections");
   ctx->g64.sigma_t = sigma_t;
   ctx->g64.sigma_s = sigma_s_within;
   const int64_t n = ctx->n_cells;
   cudaStream_t s = (cudaStream_t)stream;
   ToFloatKernel<double><<<(n + 255) / 256, 256, 0, s>>>(sigma_t, ctx->sigma_t32, n);
   ToFloatKernel<double><<<(n + 255) / 256, 256, 0, s>>>(sigma_s_within, ctx->sigma_s32, n);
   CountLaunch(1);
   rc = CheckLaunch("set_group");
   if (rc) return rc;
   ctx->group_set = true;
   ctx->group_epoch++;
   return UBOLT_OK;
}
