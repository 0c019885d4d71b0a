// Internal declarations shared by the host C++ and the CUDA translation units
// of libubolt_b200. Never installed: the public surface is include/ubolt_b200.h.
#pragma once

#include "ubolt_b200.h"

#include <array>
#include <cstdarg>
#include <cstdint>
#include <string>
#include <vector>

namespace ubolt {

// Record a failure for ubolt_last_error() and return its status, so a call
// site reads `return SetError(UBOLT_ERR_ARG, "...", ...)`.
int SetError(int status, const char *fmt, ...);
void ClearError();

int LqnOctant(int sn_order, std::vector<double> &mu, std::vector<std::array<int, 3>> &points,
              std::vector<double> &weight);

// Local faces of each cell shape, as vertex indices into the cell's own list.
// The order is this library's cone order: the slot order of a row's faces.
struct CellShape {
   int dim;
   int n_vertices;
   int n_faces;
   int verts_per_face;
   int face[6][4];
};
const CellShape *ShapeOf(int cell_type);

}  // namespace ubolt
