// Interface between the host ghost-grid builder (ghostgrid.cpp) and the GPU
// least-squares table build (lsbuild.cu). Private to the library.
#pragma once
#include <cstdint>

namespace rh3t {

// Offsets of the per-order blocks inside one ghost's tables (bc1.rs:45-47):
// E_r stencil nodes, S_r (m x m, m = (r+1)^2) and w_r ((r+1) x m).
constexpr int LS_STENCIL = 55, LS_S = 979, LS_W = 225;
// quadratic forms M_1..M_4 of one grid, row-major n x n (n = (r+1)(r+2)/2)
constexpr int LS_M = 9 + 36 + 100 + 225;

// One geometry: node placement (field1.rs:6-15 x = x0 + i dx), the r = 0
// smoothness entry 2 h^2 (bc1.rs:167-168) and M_r (bc1.rs:62-85).
struct LsGrid {
    double x0, y0, dx, dy;
    int64_t ny;
    double s0;
    double M[LS_M];
};

// One Wall / Outflow / FarField ghost: its final projection (P0, outward
// normal) and where its tables go (grid index, heavy slot).
struct LsJob {
    double p0x, p0y, nx, ny;
    int32_t grid, slot;
};

// Computes S_0..S_4 and w_0..w_4 of every job on `device` from the jobs'
// E_r stencils (stencils[55 * job], linear node indices i * ny + j) and
// writes them to s_out[grid] + 979 * slot and w_out[grid] + 225 * slot
// (host memory). The arithmetic is the host build's, operation for
// operation. Returns 0, or a CUDA error code with a message in err.
int ls_tables_device(int device, int n_grids, const LsGrid* grids, long long n_jobs, const LsJob* jobs,
                     const uint32_t* stencils, double* const* s_out, double* const* w_out, char* err, int err_len);

} // namespace rh3t
