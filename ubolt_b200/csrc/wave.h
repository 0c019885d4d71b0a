// The wave sweep: one block per ordinate (see wave.cu). Internal interface
// between the sweep plan (sweep.cu) and the kernels.
#pragma once

#include "ctx.h"
#include "sweep_plan.h"

#include <cstdint>

namespace ubolt {

// The sweep's control words (shared by both kernels): [kSweepCtrlError] the
// sticky error flag, [kSweepCtrlError + 1] the count of waits that gave up
constexpr int kSweepCtrlError = 32;

// Device view of the wave plan and of one precision's factor store layout
struct WaveDev {
   int32_t A = 0, S = 0, n_slots = 0, max_levels = 0;
   int64_t n_cells = 0;
   const int32_t *lvl_base = nullptr;   // [A + 1]
   const int32_t *lvl_pos = nullptr;    // [total + A]
   const int32_t *lvl_ord = nullptr;    // [total] ordinate of each level
   const int4 *meta = nullptr;          // [A][n_cells]
   // One precision's store: ordinate a's region at byte region[a]; level
   // chunks at region-relative chunk_rel[.] (same indexing as lvl_pos), each
   // landing in the ring at ring_off[.]
   const int64_t *region = nullptr;     // [A]
   const int32_t *chunk_rel = nullptr;  // [total + A]
   const int32_t *ring_off = nullptr;   // [total + A]
   int32_t cap = 0;                     // ring bytes
   int32_t front_off = 0, ring_base = 0;  // byte offsets of the front and the ring in shared memory
   int32_t smem = 0;                    // dynamic shared memory of a block
   uint32_t *ctrl = nullptr;            // the sweep's error flag and timeout count
   uint32_t spin_limit = 1u << 22;
   int64_t unmet_level = -1;            // test hook: this level's copy is never issued
};

// The input of one sweep: q itself (in == nullptr), or the affine form the
// compressed GMRES passes, q(node, a) = alpha r0(node, a) + u_a (phi(node) -
// alpha rho(node)), or u_a phi(node) alone when iso (r0 isotropic).
struct WaveInput {
   const double *alpha = nullptr, *phi = nullptr, *rho = nullptr;
   const void *u = nullptr;
   int iso = 0;
};

// Fill the store for the current group (one kernel launch)
int WaveFactors(ubolt_ctx *ctx, const WaveDev &w, void *fac, int elem, cudaStream_t st, int64_t total_levels);
// psi = L^{-1} q for every ordinate, one block per ordinate
int WaveSweep(ubolt_ctx *ctx, const WaveDev &w, const void *q, void *psi, const void *fac, int elem,
              const WaveInput *in, int threads, cudaStream_t st);

}  // namespace ubolt
