// Launchers of the rh3t device kernels (kernels.cu, ghosts.cu, flux.cu, rhs.cu).
#pragma once
#include <cuda_runtime.h>
#include "rh3t_dev.h"

namespace rh3t {
// heavy: Wall / Outflow / FarField records; cheap: all other kinds (ghosts.cu)
// hrec: heavy records (GH_REC doubles per GhostBC slot; the per-stage L, R,
// lambda part is written by the launch). Two kernels: ghost_launches() of them.
void launch_ghosts(cudaStream_t s, const Inst* insts, const GhostRec* heavy, int nh, const GhostRec* cheap, int nc,
                   double* hrec, int stage);
int ghost_launches(int nh, int nc);
void launch_flux(cudaStream_t s, const Inst* insts, const Tile* tx, int ntx, const Tile* ty, int nty, int stage);
void launch_rhs_stage(cudaStream_t s, const Inst* insts, const Tile* tc, int nt, int stage, int mode, double* rhs);
void launch_dt(cudaStream_t s, const Inst* insts, const Tile* tc, int nt, int mode);
void launch_set_dt(cudaStream_t s, const Inst* insts, int n_inst, double dt);
void launch_scatter(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, const double* aos,
                    const double* times);
void launch_gather(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, double* aos);
void launch_set_step(cudaStream_t s, const Inst* insts, int k0, int n, double cfl, double t_final);
void launch_planes_to_aos(cudaStream_t s, const double* planes, long long n, double* aos);
void launch_ghost_values(cudaStream_t s, const Inst* insts, const GhostRec* recs, int n, double* out);
void launch_dfma(cudaStream_t s, int blocks, double* out, int iters);
void launch_math_check(cudaStream_t s, const double* x, int n, double q, double* out);
} // namespace rh3t
