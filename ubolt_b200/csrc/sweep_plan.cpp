// The sweep plan on the host.
//
// Per ordinate, Kahn's algorithm over the cell upwind graph (interior faces
// with Omega . nA < 0, each cell's own normal deciding its own inflow), run
// with patch affinity: a patch with ready cells becomes a task holding the
// closure of its cells that can be solved from what is already done - cells
// become ready inside the task as their in-patch upwind neighbours are solved.
// Cells still waiting on another patch are picked up by a later task of the
// same patch. The tasks of an ordinate come out in a topological order, and
// no coupling is dropped: the sweep is exact wherever the graph is acyclic.
// A cycle (possible on tetrahedra) is broken by releasing the waiting cell
// with the fewest unresolved inputs; those inputs are lagged (read as zero).
//
// All ordinates' tasks are merged by a modelled pickup time that is
// topological for every ordinate (see kLevelCost), and renumbered in that order.
#include "sweep_plan.h"

#include "ubolt_internal.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>

namespace ubolt {

namespace {

struct AngleTask {
   int32_t patch;
   std::vector<uint8_t> cells;   // local indices, level order
   std::vector<uint16_t> mask;
   std::vector<uint16_t> lvl;    // level ends
   std::vector<int32_t> deps;    // angle-local task ids
   double start = 0.0;           // modelled pickup time (see below)
};

// Launch order. The kernel walks a task level by level and each level waits
// for its earlier-task inputs, so a task taken too early holds a warp while
// it waits, and one taken too late delays everything downstream. Model the
// walk at level granularity: a level takes kLevelCost, an input crossing
// from another task kHopCost (both in level units); a task's pickup time is
// the latest time at which none of its levels would wait. Tasks are numbered
// by that time, raised above every upstream task's so the order stays
// topological.
constexpr double kLevelCost = 1.0, kHopCost = 4.0;

}  // namespace

void BuildHostSweepPlan(int64_t nc, int F, int A, int P, const double *om, const double *nA, const int32_t *code,
                        HostSweepPlan &plan)
{
   const int32_t np = (int32_t)((nc + P - 1) / P);
   plan.P = P;
   plan.n_patches = np;
   plan.A = A;
   std::vector<std::vector<AngleTask>> per_angle(A);
   std::vector<int64_t> lagged(A, 0), split(A, 0);

#pragma omp parallel for schedule(dynamic, 1)
   for (int a = 0; a < A; a++) {
      // Upwind faces per cell, and the downwind lists built from them
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
      std::vector<int32_t> task_of(nc, -1), level(nc, 0);
      std::vector<char> released(nc, 0);
      std::vector<std::vector<int32_t>> ready(np);
      std::vector<char> queued(np, 0);
      std::vector<int32_t> fifo;
      size_t head = 0;
      auto release = [&](int64_t c) {
         released[c] = 1;
         const int32_t p = (int32_t)(c / P);
         ready[p].push_back((int32_t)c);
         if (!queued[p]) { queued[p] = 1; fifo.push_back(p); }
      };
      for (int64_t c = 0; c < nc; c++)
         if (indeg[c] == 0) release(c);
      int64_t done = 0;
      auto &tasks = per_angle[a];
      std::vector<int32_t> stack, members;
      while (done < nc) {
         while (head < fifo.size()) {
            const int32_t p = fifo[head++];
            queued[p] = 0;
            if (ready[p].empty()) continue;
            const int32_t t = (int32_t)tasks.size();
            tasks.emplace_back();
            AngleTask &T = tasks.back();
            T.patch = p;
            stack.swap(ready[p]);
            ready[p].clear();
            members.clear();
            const int64_t base = (int64_t)p * P;
            while (!stack.empty()) {
               const int32_t c = stack.back();
               stack.pop_back();
               task_of[c] = t;
               members.push_back(c);
               done++;
               int lv = 0;
               for (int f = 0; f < F; f++)
                  if ((upmask[c] >> f) & 1) {
                     const int32_t u = code[(int64_t)c * F + f];
                     if (task_of[u] == t) lv = std::max(lv, level[u] + 1);
                  }
               level[c] = lv;
               for (int64_t e = optr[c]; e < optr[c + 1]; e++) {
                  const int32_t d = oadj[e];
                  if (released[d]) continue;
                  if (--indeg[d] == 0) {
                     if (d / P == p) { released[d] = 1; stack.push_back(d); }
                     else release(d);
                  }
               }
            }
            // Cells in level order; masks and upstream tasks
            std::stable_sort(members.begin(), members.end(), [&](int32_t x, int32_t y) { return level[x] < level[y]; });
            T.cells.resize(members.size());
            T.mask.resize(members.size());
            for (size_t i = 0; i < members.size(); i++) {
               const int32_t c = members[i];
               T.cells[i] = (uint8_t)(c - base);
               uint16_t m = 0;
               for (int f = 0; f < F; f++)
                  if ((upmask[c] >> f) & 1) {
                     const int32_t u = code[(int64_t)c * F + f];
                     if (task_of[u] == t) m |= (uint16_t)(1u << f);
                     else if (task_of[u] >= 0) { m |= (uint16_t)(1u << (8 + f)); T.deps.push_back(task_of[u]); }
                     else lagged[a]++;  // released by a cycle break: lagged to zero
                  }
               T.mask[i] = m;
               if (i + 1 == members.size() || level[members[i + 1]] != level[c]) T.lvl.push_back((uint16_t)(i + 1));
            }
            std::sort(T.deps.begin(), T.deps.end());
            T.deps.erase(std::unique(T.deps.begin(), T.deps.end()), T.deps.end());
         }
         if (done < nc) {
            // A cycle: release the waiting cell with the fewest unresolved inputs
            int64_t best = -1;
            for (int64_t c = 0; c < nc; c++)
               if (!released[c] && (best < 0 || indeg[c] < indeg[best])) best = c;
            release(best);
         }
      }
      // Levels by modelled finish time. A task's walk is level-synchronous,
      // so a cell whose earlier-task input is late holds up every later
      // level. Model each cell's finish: an in-task upwind input adds
      // kLevelCost, an earlier-task one kHopCost; then order each task's
      // cells by that time (ties keep the upwind level order) and start a
      // new level wherever it changes. An in-task upwind cell finishes
      // strictly earlier, so it still sits at a lower level.
      {
         std::vector<double> cf(nc, 0.0), tcf;
         std::vector<int32_t> idx;
         std::vector<uint8_t> cells;
         std::vector<uint16_t> mask;
         for (auto &T : tasks) {
            const int64_t base = (int64_t)T.patch * P;
            const size_t n = T.cells.size();
            tcf.assign(n, 0.0);
            for (size_t i = 0; i < n; i++) {
               const int64_t c = base + T.cells[i];
               double r = kLevelCost;
               for (int f = 0; f < F; f++) {
                  if ((T.mask[i] >> f) & 1u) r = std::max(r, cf[code[c * F + f]] + kLevelCost);
                  else if ((T.mask[i] >> (8 + f)) & 1u) r = std::max(r, cf[code[c * F + f]] + kHopCost);
               }
               cf[c] = r;
               tcf[i] = r;
            }
            idx.resize(n);
            std::iota(idx.begin(), idx.end(), 0);
            std::stable_sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) { return tcf[x] < tcf[y]; });
            cells.resize(n);
            mask.resize(n);
            T.lvl.clear();
            for (size_t i = 0; i < n; i++) {
               cells[i] = T.cells[idx[i]];
               mask[i] = T.mask[idx[i]];
               if (i + 1 == n || tcf[idx[i + 1]] != tcf[idx[i]]) T.lvl.push_back((uint16_t)(i + 1));
            }
            T.cells.swap(cells);
            T.mask.swap(mask);
         }
      }
      // Modelled pickup times, tasks in (topological) creation order
      {
         std::vector<double> cfin(nc, 0.0);
         for (auto &T : tasks) {
            const int64_t base = (int64_t)T.patch * P;
            double prev = 0.0, start = -1e300;
            size_t lo = 0;
            for (size_t L = 0; L < T.lvl.size(); L++) {
               const size_t hi = T.lvl[L];
               double ready = -1e300;
               for (size_t i = lo; i < hi; i++) {
                  const int64_t c = base + T.cells[i];
                  for (int f = 0; f < F; f++)
                     if ((T.mask[i] >> (8 + f)) & 1u) ready = std::max(ready, cfin[code[c * F + f]] + kHopCost);
               }
               start = std::max(start, ready - (double)L * kLevelCost);
               const double end = std::max(prev, ready) + kLevelCost;
               for (size_t i = lo; i < hi; i++) cfin[base + T.cells[i]] = end;
               prev = end;
               lo = hi;
            }
            start = std::max(start, 0.0);
            for (int32_t d : T.deps) start = std::max(start, tasks[d].start + 1e-6);
            T.start = start;
         }
      }
      // Patches solved in more than one task for this ordinate
      std::vector<int32_t> count(np, 0);
      for (const auto &T : tasks) count[T.patch]++;
      for (int32_t p = 0; p < np; p++) split[a] += std::max(0, count[p] - 1);
   }

   // ~~~ Merge the ordinates by depth and renumber in launch order
   std::vector<std::pair<int32_t, int32_t>> all;  // (angle, angle-local id)
   for (int a = 0; a < A; a++)
      for (int32_t t = 0; t < (int32_t)per_angle[a].size(); t++) all.emplace_back(a, t);
   // By modelled pickup time; ties (the same time) by patch, so warps taking
   // consecutive tasks read that patch's data while it is in L2
   std::stable_sort(all.begin(), all.end(), [&](const auto &x, const auto &y) {
      const AngleTask &tx = per_angle[x.first][x.second], &ty = per_angle[y.first][y.second];
      if (tx.start != ty.start) return tx.start < ty.start;
      if (tx.patch != ty.patch) return tx.patch < ty.patch;
      return x.first < y.first;
   });
   std::vector<std::vector<int32_t>> gid(A);
   for (int a = 0; a < A; a++) gid[a].resize(per_angle[a].size());
   for (size_t i = 0; i < all.size(); i++) gid[all[i].first][all[i].second] = (int32_t)i;

   const int64_t nt = (int64_t)all.size();
   plan.n_tasks = nt;
   plan.task_pa.resize(nt);
   plan.dep_ptr.assign(nt + 1, 0);
   plan.cell_ptr.assign(nt + 1, 0);
   plan.lvl_ptr.assign(nt + 1, 0);
   plan.deps.clear();
   plan.tcell.clear();
   plan.tmask.clear();
   plan.lvl.clear();
   plan.tcell.reserve(nc * A);
   plan.tmask.reserve(nc * A);
   plan.max_levels = 0;
   for (int64_t i = 0; i < nt; i++) {
      const int a = all[i].first;
      const AngleTask &T = per_angle[a][all[i].second];
      plan.task_pa[i] = (int32_t)((int64_t)T.patch * A + a);
      for (int32_t d : T.deps) plan.deps.push_back(gid[a][d]);
      plan.dep_ptr[i + 1] = (int32_t)plan.deps.size();
      plan.tcell.insert(plan.tcell.end(), T.cells.begin(), T.cells.end());
      plan.tmask.insert(plan.tmask.end(), T.mask.begin(), T.mask.end());
      plan.cell_ptr[i + 1] = (int64_t)plan.tcell.size();
      plan.lvl.insert(plan.lvl.end(), T.lvl.begin(), T.lvl.end());
      plan.lvl_ptr[i + 1] = (int32_t)plan.lvl.size();
      plan.max_levels = std::max<int32_t>(plan.max_levels, (int32_t)T.lvl.size());
   }
   plan.max_inflow = 0;
   for (const uint16_t m : plan.tmask)
      plan.max_inflow = std::max(plan.max_inflow, __builtin_popcount((unsigned)(m & 0xff) | (unsigned)(m >> 8)));
   plan.n_lagged = 0;
   plan.n_split = 0;
   for (int a = 0; a < A; a++) {
      plan.n_lagged += lagged[a];
      plan.n_split += split[a];
   }
}

}  // namespace ubolt

// ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

struct ubolt_sweep_plan_host {
   ubolt::HostSweepPlan plan;
};

extern "C" int ubolt_sweep_plan_build(const ubolt_dg_geometry *g, const ubolt_quadrature *q, int patch_size,
                                      ubolt_sweep_plan_host **out, ubolt_sweep_plan_view *view)
{
   using namespace ubolt;
   if (!g || !q || !out || !view) return SetError(UBOLT_ERR_ARG, "sweep_plan_build: NULL argument");
   const int F = g->faces_per_cell, A = q->n_angles;
   const int64_t nc = g->n_cells;
   if (patch_size < 0 || patch_size > 256) return SetError(UBOLT_ERR_ARG, "patch size %d (0..256)", patch_size);
   if (F > 8) return SetError(UBOLT_ERR_ARG, "at most 8 faces per cell");
   int P = patch_size > 0 ? patch_size : 64;
   if (P > nc) P = (int)nc;
   std::vector<int32_t> code(nc * F);
   for (int64_t k = 0; k < nc * F; k++)
      code[k] = g->face_neighbour[k] >= 0 ? (int32_t)g->face_neighbour[k] : -1 - std::max(0, g->face_side[k]);
   auto h = std::make_unique<ubolt_sweep_plan_host>();
   BuildHostSweepPlan(nc, F, A, P, q->omega, g->face_nA, code.data(), h->plan);
   const HostSweepPlan &p = h->plan;
   std::memset(view, 0, sizeof *view);
   view->patch_size = p.P;
   view->n_patches = p.n_patches;
   view->n_tasks = p.n_tasks;
   view->n_lagged = p.n_lagged;
   view->n_split = p.n_split;
   view->task_pa = p.task_pa.data();
   view->dep_ptr = p.dep_ptr.data();
   view->deps = p.deps.data();
   view->cell_ptr = p.cell_ptr.data();
   view->tcell = p.tcell.data();
   view->tmask = p.tmask.data();
   view->lvl_ptr = p.lvl_ptr.data();
   view->lvl = p.lvl.data();
   *out = h.release();
   return UBOLT_OK;
}

extern "C" void ubolt_sweep_plan_free(ubolt_sweep_plan_host *p) { delete p; }
