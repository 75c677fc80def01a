// geometry.cpp -- see geometry.hpp.
#include "geometry.hpp"

#include <algorithm>
#include <cmath>

namespace rtmb {

void grid_cell(float x, float z, int nx, int nz, float dx, float dz, float ox, float oz, int nb,
               int* ixe, int* ize, bool* clamped) {
    const int ix0 = (int)std::lround((x - ox) / dx);
    const int iz0 = (int)std::lround((z - oz) / dz);
    const int ix = std::min(std::max(ix0, 0), nx - 1);
    const int iz = std::min(std::max(iz0, 0), nz - 1);
    *clamped = (ix != ix0) || (iz != iz0);
    *ixe = ix + nb;
    *ize = iz + nb;
}

ShotGeometry build_geometry(float sx, float sz, int nrec, const float* rx, const float* rz, int nx,
                            int nz, float dx, float dz, float ox, float oz, int nb) {
    ShotGeometry g;
    bool cl = false;
    grid_cell(sx, sz, nx, nz, dx, dz, ox, oz, nb, &g.src_x, &g.src_z, &cl);
    g.nclamped += cl ? 1 : 0;

    struct Rec { int x, z, ir; };
    std::vector<Rec> recs((size_t)std::max(nrec, 0));
    for (int ir = 0; ir < nrec; ++ir) {
        grid_cell(rx[ir], rz[ir], nx, nz, dx, dz, ox, oz, nb, &recs[ir].x, &recs[ir].z, &cl);
        recs[ir].ir = ir;
        g.nclamped += cl ? 1 : 0;
    }
    // Stable: receivers that share a cell keep ascending ir order, so the
    // kernel adds their samples in the reference's sequential order.
    std::stable_sort(recs.begin(), recs.end(),
                     [](const Rec& a, const Rec& b) { return a.x != b.x ? a.x < b.x : a.z < b.z; });
    const int nxe = nx + 2 * nb;
    g.col_start.assign((size_t)nxe + 1, 0);
    g.ir.reserve(recs.size());
    for (size_t i = 0; i < recs.size();) {
        size_t j = i;
        PointEntry e{recs[i].z, (int)g.ir.size(), 0, 0};
        while (j < recs.size() && recs[j].x == recs[i].x && recs[j].z == recs[i].z) {
            g.ir.push_back(recs[j].ir);
            ++j;
        }
        e.ir_count = (int)(j - i);
        g.pts.push_back(e);
        g.col_start[(size_t)recs[i].x + 1] += 1;
        i = j;
    }
    for (int x = 0; x < nxe; ++x) g.col_start[(size_t)x + 1] += g.col_start[(size_t)x];
    // Per-receiver view of the same order (the kernel stages a tile's receivers
    // from it): row of each receiver and receiver offsets per column.
    g.rec_col.assign((size_t)nxe + 1, 0);
    g.rec_z.reserve(g.ir.size());
    for (int x = 0; x < nxe; ++x) {
        int n = 0;
        for (int j = g.col_start[(size_t)x]; j < g.col_start[(size_t)x + 1]; ++j) {
            for (int r = 0; r < g.pts[(size_t)j].ir_count; ++r) g.rec_z.push_back(g.pts[(size_t)j].z);
            n += g.pts[(size_t)j].ir_count;
        }
        g.rec_col[(size_t)x + 1] = g.rec_col[(size_t)x] + n;
    }
    return g;
}

}  // namespace rtmb
