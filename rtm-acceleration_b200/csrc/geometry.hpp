// geometry.hpp -- source/receiver positions to extended-grid cells, and the
// per-column receiver lists the fused step kernel walks.
#pragma once
#include <vector>

#include "internal.hpp"

namespace rtmb {

struct ShotGeometry {
    int src_x = 0, src_z = 0;          // extended coordinates of the source
    std::vector<int> col_start;        // nxe+1 offsets into pts
    std::vector<PointEntry> pts;       // receiver cells sorted by (x, z)
    std::vector<int> ir;               // receivers of each cell, ascending
    std::vector<int> rec_col;          // nxe+1 offsets into ir: receivers of the columns before x
    std::vector<int> rec_z;            // extended row of each receiver, in ir order
    int nclamped = 0;                  // positions clamped onto the model edge
};

// Nearest grid point (lround of the float quotient), clamped to the interior,
// as extended coordinates (reference src/rtm/rtm_cpu.cpp:99-123).  nx is the
// width of the domain the shot is migrated on (its aperture window) and ox the
// x origin of that domain.
void grid_cell(float x, float z, int nx, int nz, float dx, float dz, float ox, float oz, int nb,
               int* ixe, int* ize, bool* clamped);

ShotGeometry build_geometry(float sx, float sz, int nrec, const float* rx, const float* rz, int nx,
                            int nz, float dx, float dz, float ox, float oz, int nb);

}  // namespace rtmb
