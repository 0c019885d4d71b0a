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

// The wave plan: every ordinate's sweep as one sequence of levels (one block
// per ordinate walks them with a barrier between levels). Positions number an
// ordinate's cells level by level; ordinate a's level l covers positions
// [lvl_pos[lvl_base[a] + a + l], lvl_pos[lvl_base[a] + a + l + 1]).
struct HostWavePlan {
   int32_t A = 0;
   int64_t n_cells = 0;
   bool acyclic = false;            // false: some ordinate's upwind graph has a cycle (no wave plan)
   int32_t S = 0;                   // most gathered upwind faces of one position
   int32_t n_slots = 0;             // front slots the busiest ordinate needs
   int32_t max_width = 0;           // most positions in one level
   int32_t max_levels = 0;
   std::vector<int32_t> lvl_base;   // [A + 1]
   std::vector<int32_t> lvl_pos;    // [lvl_base[A] + A]
   std::vector<int32_t> meta;       // [A][n_cells][4]: cell; out slot | gathered-face mask << 16;
                                    // the upwind cells' slots in face order, two per word (0xffff: none)
};

void BuildHostWavePlan(int64_t n_cells, int F, int A, const double *omega, const double *nA, const int32_t *code,
                       HostWavePlan &plan);

// Bytes of one level's factor chunk: elems_per_position values of `elem`
// bytes per position, element-major, padded to 16 bytes
inline int64_t WaveChunkBytes(int64_t width, int64_t elems_per_position, int elem)
{
   return (width * elems_per_position * elem + 15) / 16 * 16;
}

// Byte offsets of every level's chunk in the wave factor store (same indexing
// as lvl_pos; entry nlev of an ordinate is the end of its last chunk). Each
// ordinate's region starts on a multiple of cap, and no chunk crosses one, so
// a chunk lands in a ring of cap bytes at (offset - region start) % cap in
// one piece.
void WaveChunkOffsets(const HostWavePlan &plan, int64_t elems_per_position, int elem, int64_t cap,
                      std::vector<int64_t> &off);

// Shared memory ahead of a wave block's staged level tables (the mbarriers
// and a flag), and the number of mbarriers (levels whose copies may be in
// flight at once)
constexpr int kWaveStages = 32;
constexpr int kWaveHeader = kWaveStages * 8 + 128;

// One precision's layout: the block's shared memory - header, level starts,
// chunk offsets and ring offsets [max_levels + 1] each, the front, the ring -
// and the store - ordinate a's region at byte region[a], its level chunks at
// region-relative chunk_rel[.] (lvl_pos indexing), each landing in the ring at
// ring_off[.]
struct WaveLayout {
   int32_t front_off = 0, ring_base = 0, cap = 0, smem = 0;
   int64_t store_bytes = 0;
   std::vector<int64_t> region;
   std::vector<int32_t> chunk_rel, ring_off;
};

// False where a level's chunk does not fit the ring left by max_smem bytes,
// or an ordinate's region exceeds 2^31 bytes
bool BuildWaveLayout(const HostWavePlan &plan, int nb, int elem, int max_smem, WaveLayout &out);

}  // namespace ubolt
