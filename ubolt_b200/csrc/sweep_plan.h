// Host half of the sweep: per-ordinate upwind orders as tasks over patches.
#pragma once

#include <cstdint>
#include <vector>

namespace ubolt {

// Tasks are numbered in launch order. Task t covers cells of one patch p
// (cells [p P, p P + P)) for one ordinate a: task_pa[t] = p * A + a.
struct HostSweepPlan {
   int32_t P = 0, n_patches = 0, A = 0;
   int64_t n_tasks = 0, n_lagged = 0, n_split = 0;
   int32_t max_levels = 0;
   int32_t max_inflow = 0;          // most gathered upwind faces of one (cell, ordinate)
   std::vector<int32_t> task_pa;    // [n_tasks]
   std::vector<int32_t> dep_ptr;    // [n_tasks + 1]
   std::vector<int32_t> deps;       // upstream task ids, all < t
   std::vector<int64_t> cell_ptr;   // [n_tasks + 1]
   std::vector<uint8_t> tcell;      // local cell index in the patch, level order
   std::vector<uint16_t> tmask;     // bit f: upwind through face f is in this task (shared memory);
                                    // bit 8 + f: in an earlier task (global memory)
   std::vector<int32_t> lvl_ptr;    // [n_tasks + 1]
   std::vector<uint16_t> lvl;       // level end positions within the task
};

// code[c * F + f]: neighbour cell (>= 0) or a boundary code (< 0); nA and
// omega as the context holds them. 1 <= P <= 256.
void BuildHostSweepPlan(int64_t n_cells, int F, int A, int P, const double *omega, const double *nA,
                        const int32_t *code, HostSweepPlan &plan);

}  // namespace ubolt
