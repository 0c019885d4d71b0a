// The wave plan on the host: each ordinate's whole sweep as one sequence of
// levels, for the kernel that sweeps one ordinate per block.
//
// Per ordinate, Kahn's algorithm over the cell upwind graph (interior faces
// with Omega . nA < 0, the same test and arithmetic as the task plan) gives
// every cell its level, the length of the longest upwind chain ending there.
// Cells are then laid out level by level (by cell id within a level): the
// positions. A cell read by a later level keeps its psi in a front slot of
// shared memory from the level that solves it to the last level that reads
// it; the slots are handed out by level, a freed slot going to a later level
// only (the block barrier between levels separates the last read of a slot
// from its next write).
//
// A cycle (possible on tetrahedra) leaves cells unreached: the plan is then
// marked cyclic and the task sweep serves that mesh.
#include "sweep_plan.h"

#include "ubolt_internal.h"

#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>

namespace ubolt {

void BuildHostWavePlan(int64_t nc, int F, int A, const double *om, const double *nA, const int32_t *code,
                       HostWavePlan &plan)
{
   plan = HostWavePlan();
   plan.A = A;
   plan.n_cells = nc;
   std::vector<std::vector<int32_t>> lvl_pos(A);
   std::vector<int32_t> n_slots(A, 0), max_width(A, 0), max_in(A, 0);
   std::vector<char> cyclic(A, 0);
   plan.meta.assign((size_t)A * nc * 4, 0);

#pragma omp parallel for schedule(dynamic, 1)
   for (int a = 0; a < A; a++) {
      std::vector<uint8_t> upmask(nc, 0);
      std::vector<int32_t> indeg(nc, 0);
      std::vector<int64_t> optr(nc + 1, 0);
      for (int64_t c = 0; c < nc; c++)
         for (int f = 0; f < F; f++) {
            const int64_t k = c * F + f;
            if (code[k] < 0) continue;
            const double s = om[3 * a] * nA[3 * k] + om[3 * a + 1] * nA[3 * k + 1] + om[3 * a + 2] * nA[3 * k + 2];
            if (s < 0.0) {
               upmask[c] |= (uint8_t)(1u << f);
               indeg[c]++;
               optr[code[k] + 1]++;
            }
         }
      for (int64_t c = 0; c < nc; c++) optr[c + 1] += optr[c];
      std::vector<int32_t> oadj(optr[nc]);
      {
         std::vector<int64_t> fill(optr.begin(), optr.end() - 1);
         for (int64_t c = 0; c < nc; c++)
            for (int f = 0; f < F; f++)
               if ((upmask[c] >> f) & 1) oadj[fill[code[c * F + f]]++] = (int32_t)c;
      }
      // Levels, front by front
      std::vector<int32_t> level(nc, -1), front, next;
      for (int64_t c = 0; c < nc; c++)
         if (indeg[c] == 0) front.push_back((int32_t)c);
      int64_t placed = 0;
      std::vector<int32_t> &lp = lvl_pos[a];
      std::vector<int32_t> order;
      order.reserve(nc);
      for (int32_t l = 0; !front.empty(); l++) {
         std::sort(front.begin(), front.end());
         lp.push_back((int32_t)placed);
         max_width[a] = std::max(max_width[a], (int32_t)front.size());
         next.clear();
         for (const int32_t c : front) {
            level[c] = l;
            order.push_back(c);
            for (int64_t e = optr[c]; e < optr[c + 1]; e++)
               if (--indeg[oadj[e]] == 0) next.push_back(oadj[e]);
         }
         placed += (int64_t)front.size();
         front.swap(next);
      }
      lp.push_back((int32_t)placed);
      if (placed != nc) {
         cyclic[a] = 1;
         continue;
      }
      // Last level reading each cell, then the front slots by level
      std::vector<int32_t> last(nc, -1);
      for (int64_t c = 0; c < nc; c++)
         for (int64_t e = optr[c]; e < optr[c + 1]; e++) last[c] = std::max(last[c], level[oadj[e]]);
      const int32_t nlev = (int32_t)lp.size() - 1;
      std::vector<std::vector<int32_t>> release(nlev + 1);
      std::vector<int32_t> free_slots, slot(nc, -1);
      int32_t used = 0;
      for (int32_t l = 0; l < nlev; l++) {
         for (const int32_t sl : release[l]) free_slots.push_back(sl);
         for (int32_t p = lp[l]; p < lp[l + 1]; p++) {
            const int32_t c = order[p];
            if (last[c] < 0) continue;
            int32_t sl;
            if (!free_slots.empty()) {
               sl = free_slots.back();
               free_slots.pop_back();
            } else {
               sl = used++;
            }
            slot[c] = sl;
            release[last[c] + 1].push_back(sl);
         }
      }
      n_slots[a] = used;
      // Per position: cell, out slot | gathered-face mask << 16, then the
      // upwind cells' slots in face order, two per word
      int32_t *m = plan.meta.data() + (size_t)a * nc * 4;
      for (int64_t p = 0; p < nc; p++) {
         const int32_t c = order[p];
         const uint32_t out = slot[c] < 0 ? 0xffffu : (uint32_t)slot[c];
         uint32_t ins[4] = {0xffffu, 0xffffu, 0xffffu, 0xffffu};
         int n_in = 0;
         for (int f = 0; f < F; f++)
            if ((upmask[c] >> f) & 1) {
               if (n_in < 4) ins[n_in] = (uint32_t)slot[code[c * F + f]];
               n_in++;
            }
         max_in[a] = std::max(max_in[a], n_in);
         m[4 * p] = c;
         m[4 * p + 1] = (int32_t)(out | ((uint32_t)upmask[c] << 16));
         m[4 * p + 2] = (int32_t)(ins[0] | (ins[1] << 16));
         m[4 * p + 3] = (int32_t)(ins[2] | (ins[3] << 16));
      }
   }

   plan.acyclic = true;
   plan.lvl_base.assign(A + 1, 0);
   for (int a = 0; a < A; a++) {
      if (cyclic[a]) plan.acyclic = false;
      plan.lvl_base[a + 1] = plan.lvl_base[a] + (int32_t)lvl_pos[a].size() - 1;
      plan.n_slots = std::max(plan.n_slots, n_slots[a]);
      plan.max_width = std::max(plan.max_width, max_width[a]);
      plan.max_levels = std::max(plan.max_levels, (int32_t)lvl_pos[a].size() - 1);
      plan.S = std::max(plan.S, max_in[a]);
   }
   if (!plan.acyclic) {
      plan.meta.clear();
      return;
   }
   plan.lvl_pos.reserve((size_t)plan.lvl_base[A] + A);
   for (int a = 0; a < A; a++) plan.lvl_pos.insert(plan.lvl_pos.end(), lvl_pos[a].begin(), lvl_pos[a].end());
}

void WaveChunkOffsets(const HostWavePlan &plan, int64_t elems_per_position, int elem, int64_t cap,
                      std::vector<int64_t> &off)
{
   const int A = plan.A;
   off.assign((size_t)plan.lvl_base[A] + A, 0);
   int64_t cursor = 0;
   for (int a = 0; a < A; a++) {
      const int64_t base = cursor;  // the ordinate's region starts on a ring boundary
      const int32_t nlev = plan.lvl_base[a + 1] - plan.lvl_base[a];
      const int32_t *lp = plan.lvl_pos.data() + plan.lvl_base[a] + a;
      int64_t *o = off.data() + plan.lvl_base[a] + a;
      for (int32_t l = 0; l < nlev; l++) {
         const int64_t bytes = WaveChunkBytes(lp[l + 1] - lp[l], elems_per_position, elem);
         // A chunk never straddles a ring boundary: the copy into the ring is
         // one contiguous piece
         const int64_t in_ring = (cursor - base) % cap;
         if (in_ring + bytes > cap) cursor += cap - in_ring;
         o[l] = cursor;
         cursor += bytes;
      }
      o[nlev] = cursor;
      cursor = base + (cursor - base + cap - 1) / cap * cap;
   }
}

bool BuildWaveLayout(const HostWavePlan &plan, int nb, int elem, int max_smem, WaveLayout &out)
{
   out = WaveLayout();
   if (!plan.acyclic) return false;
   const int A = plan.A;
   const int64_t R = (int64_t)nb * nb * (1 + std::max(1, plan.S));
   out.front_off = (kWaveHeader + 3 * 4 * (plan.max_levels + 1) + 15) / 16 * 16;
   const int64_t front_bytes = ((int64_t)plan.n_slots * nb * elem + 15) / 16 * 16;
   out.ring_base = (int32_t)((out.front_off + front_bytes + 127) / 128 * 128);
   const int64_t cap = ((int64_t)max_smem - out.ring_base) / 16 * 16;
   if (cap < WaveChunkBytes(plan.max_width, R, elem)) return false;
   std::vector<int64_t> off;
   WaveChunkOffsets(plan, R, elem, cap, off);
   out.region.assign(A, 0);
   out.chunk_rel.assign(off.size(), 0);
   out.ring_off.assign(off.size(), 0);
   for (int a = 0; a < A; a++) {
      const int64_t b0 = plan.lvl_base[a] + a, b1 = plan.lvl_base[a + 1] + a;
      out.region[a] = off[b0];
      for (int64_t k = b0; k <= b1; k++) {
         const int64_t r = off[k] - out.region[a];
         if (r >= INT32_MAX) return false;
         out.chunk_rel[k] = (int32_t)r;
         out.ring_off[k] = (int32_t)(r % cap);
      }
      out.store_bytes = std::max(out.store_bytes, off[b1]);
   }
   out.cap = (int32_t)cap;
   out.smem = (int32_t)(out.ring_base + cap);
   return true;
}

}  // namespace ubolt

// ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

struct ubolt_wave_plan_host {
   ubolt::HostWavePlan plan;
   ubolt::WaveLayout layout;
};

extern "C" int ubolt_wave_plan_build(const ubolt_dg_geometry *g, const ubolt_quadrature *q, ubolt_wave_plan_host **out,
                                     ubolt_wave_plan_view *view)
{
   using namespace ubolt;
   if (!g || !q || !out || !view) return SetError(UBOLT_ERR_ARG, "wave_plan_build: NULL argument");
   const int F = g->faces_per_cell, A = q->n_angles;
   const int64_t nc = g->n_cells;
   if (F > 8) return SetError(UBOLT_ERR_ARG, "at most 8 faces per cell");
   std::vector<int32_t> code(nc * F);
   for (int64_t k = 0; k < nc * F; k++)
      code[k] = g->face_neighbour[k] >= 0 ? (int32_t)g->face_neighbour[k] : -1 - std::max(0, g->face_side[k]);
   auto h = std::make_unique<ubolt_wave_plan_host>();
   BuildHostWavePlan(nc, F, A, q->omega, g->face_nA, code.data(), h->plan);
   const HostWavePlan &p = h->plan;
   std::memset(view, 0, sizeof *view);
   view->acyclic = p.acyclic ? 1 : 0;
   view->slots = p.S;
   view->n_front = p.n_slots;
   view->max_width = p.max_width;
   view->max_levels = p.max_levels;
   view->total_levels = p.lvl_base.empty() ? 0 : p.lvl_base[A];
   view->lvl_base = p.lvl_base.data();
   view->lvl_pos = p.acyclic ? p.lvl_pos.data() : nullptr;
   view->meta = p.acyclic ? p.meta.data() : nullptr;
   *out = h.release();
   return UBOLT_OK;
}

extern "C" void ubolt_wave_plan_free(ubolt_wave_plan_host *p) { delete p; }

extern "C" int ubolt_wave_plan_layout(ubolt_wave_plan_host *p, int n_basis, int elem_bytes, int max_shared_bytes,
                                      ubolt_wave_layout_view *view)
{
   using namespace ubolt;
   if (!p || !view) return SetError(UBOLT_ERR_ARG, "wave_plan_layout: NULL argument");
   if (n_basis < 1 || n_basis > 4 || (elem_bytes != 4 && elem_bytes != 8) || max_shared_bytes < 1)
      return SetError(UBOLT_ERR_ARG, "wave_plan_layout: n_basis 1..4, 4- or 8-byte elements");
   std::memset(view, 0, sizeof *view);
   if (!BuildWaveLayout(p->plan, n_basis, elem_bytes, max_shared_bytes, p->layout))
      return SetError(UBOLT_ERR_STATE, "no wave layout: a cycle, or a level too large for the ring");
   const WaveLayout &L = p->layout;
   view->front_off = L.front_off;
   view->ring_base = L.ring_base;
   view->cap = L.cap;
   view->smem = L.smem;
   view->store_bytes = L.store_bytes;
   view->region = L.region.data();
   view->chunk_rel = L.chunk_rel.data();
   view->ring_off = L.ring_off.data();
   return UBOLT_OK;
}
