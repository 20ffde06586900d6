// Device data layout of the rh3t solver (shared by host and device code).
//
// A context holds one or more independent instances (a batch); every kernel
// launch covers a contiguous range of them through per-instance Inst records.
// HBM layout of one solver instance:
//   state buffers U, A, B: 6 component planes each, padded node grid
//     (nx + 2*PAD) x nyp with nyp = round_up(ny + 2*PAD, 8); node (i, j)
//     lives at (i + PAD) * nyp + (j + PAD), j fastest (the reference's i*ny+j
//     order, padded). Ghost values are written into their own node position,
//     so every stencil read is a direct load (the reference goes through the
//     per-cell access table of ghost.rs:71-107 instead).
//   x faces fx: 6 planes of (nx+1)*ny, face (i, j) = interface i-1/2 of row j
//     at i*ny + j; y faces fy: 6 planes of nx*(ny+1), face (i, j) =
//     interface j-1/2 of column i at i*(ny+1) + j (main.rs:45-67 keeps y
//     faces as [j][i]; j fastest here for coalescing).
//   diffusion faces dfx/dfy: 3 planes (ee, ei, er) of the same shapes.
#pragma once
#include <stdint.h>

#define RH3T_PAD 4

namespace rh3t {

struct DevParams {
    double gamma_e, gamma_i, gamma_r;
    double cve, cvi, a_rad;
    double kappa_e, kappa_i, kappa_r;
    double omega_ei, omega_er;
    double lambda, weno_q, eps;
    double periodic_ly;
};

struct DevBC {
    int32_t kind;
    int32_t reserved;
    double state[6];
    double p_inf, sigma, l_domain;
    double td_x0, td_speed;
    double td_left[6], td_right[6];
};

enum BCKind {
    BC_REFLECTIVE_WALL = 0, BC_WALL = 1, BC_PERIODIC = 2, BC_CONSTANT = 3,
    BC_TIME_DEPENDENT = 4, BC_OUTFLOW = 5, BC_ZEROTH_ORDER = 6, BC_FAR_FIELD = 7
};

// one ghost node (ghost.rs:18-27 GhostInfo, with the static parts of the
// cheap BCs resolved at set-up: the mirror / wrap source node)
struct GhostRec {
    int32_t inst;     // instance id
    int32_t bc;       // index into the instance's BC table (outer sides, then inner)
    int32_t kind;     // BC kind of that side
    int32_t node;     // padded node index of the ghost (write target)
    int32_t src;      // padded node index of the source node (cheap kinds) or nearest node (heavy)
    int32_t heavy;    // slot in the heavy tables or -1
    int32_t gid;      // ghost id within its instance
    int32_t pad_;
    double p0x, p0y, nx, ny, dist;
    double pad2_[3];
};

// per-instance scalars kept on the device (one 128-byte line)
struct DevScalars {
    unsigned long long dt_cfl_bits; // running min of local dt (bit pattern of a positive double)
    unsigned int counter;           // blocks finished in the dt reduction
    unsigned int pad_;
    double dt;                      // dt of the current step
    double t;                       // time at the start of the current step
    double t_stage[3];              // ghost times of the three stages (main.rs:362, 366)
    double t_after;                 // time after the current step
    double cfl_factor, t_final;
    double coef[3];                 // stage rhs coefficients dt, dt/4, 2dt/3
    double dt_cfl;                  // last reduced dt_cfl (calc_global_dt)
    long long step;                 // index of the current step (error keys)
    long long steps_started;
};

// error record: one 64-bit key, min over all reports (the earliest failure):
// key = step << 40 | phase << 37 | code << 32 | index, phase = 2*stage (+1
// for the stage update, 0 for the ghost update of that stage; 7 = dt).
struct DevError {
    unsigned long long key;         // ~0ull when clear
};

struct Inst {
    int32_t nx, ny, nyp, n_tiles_dt;
    long long plane;                // (nx + 2*PAD) * nyp
    long long cell_off;             // sum of nx*ny over the instances before this one
    long long aoff;                 // sum of 6*plane before this one: offset in batch-wide plane sets
    double dx, dy;
    DevParams P;
    int32_t diffusion, source;
    double* U;
    double* A;
    double* B;
    const uint8_t* mask;            // padded fluid mask, 1 = fluid
    double* fx;
    double* fy;
    double* dfx;
    double* dfy;
    const DevBC* bcs;
    DevScalars* sc;
    DevError* err;
};

// work tile. Cell (dt) tiles: CELL_TILE consecutive j at one i. Face and
// RHS tiles: a (64 >> lg) x (1 << lg) block of x faces, y faces (64 faces,
// i x j) or a (256 >> lg) x (1 << lg) block of cells (RHS), starting at
// (i, j0). The shape is chosen per tile, so one launch can mix instances
// tuned to different shapes.
struct Tile {
    int32_t inst, i, j0, lg;
};

// Heavy-ghost record (one per GhostBC slot, bc1.rs:50-57), repacked at set-up
// so one 16-byte-aligned bulk copy brings a ghost's data to shared memory:
// S (979 doubles, offsets of bc1.rs:45-47, each S_r stored transposed) |
// w (225) | d (5) | pad (1) | E_r stencil as 55 padded node indices (int32,
// + 1 pad) | per stage: L (6x6, row-major), R (6x6, by column), lambda (6),
// pad (2), written by the ghost preparation kernel.
constexpr int GH_S = 0, GH_W = 979, GH_D = 1204, GH_ST = 1210;
constexpr int GH_L = 1238, GH_R = 1274, GH_LAM = 1310;
constexpr int GH_LR = 80;                        // doubles of the per-stage part at GH_L
constexpr int GH_REC = 1318;                     // doubles per record (10544 bytes)

constexpr int CELL_TILE = 128;
constexpr int FLUX_FACES = 64;                   // faces per flux block
constexpr int FLUX_THREADS = 192;                // 6 warps: one per characteristic field
constexpr int RHS_THREADS = 256;                 // cells per RHS block
// admissible shapes (log2 of the j extent)
constexpr int FX_LG_MIN = 2, FX_LG_MAX = 4;      // x faces 16x4, 8x8, 4x16
constexpr int FY_LG_MIN = 4, FY_LG_MAX = 6;      // y faces 4x16, 2x32, 1x64
constexpr int RHS_LG_MIN = 4, RHS_LG_MAX = 6;    // cells 16x16, 8x32, 4x64
constexpr int FX_LG_DEF = 3, FY_LG_DEF = 6, RHS_LG_DEF = 5;
// staged points per flux block: max over shapes of (TI + 5) * TJ (x) and
// TI * (TJ + 5) (y)
constexpr int FLUX_NPT = 144;
// RHS halo points: max over shapes of (TI + 8) * (TJ + 8)
constexpr int RHS_NPT = 864;

} // namespace rh3t
