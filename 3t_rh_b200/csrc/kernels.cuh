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
// x faces, then y faces: flux_launches() kernels
void launch_flux(cudaStream_t s, const Inst* insts, const Tile* tx, int ntx, const Tile* ty, int nty, int stage);
int flux_launches(int ntx, int nty);
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
// adjoint (adjoint.cu): plane sets are batch-wide arrays of 6 padded planes
// per instance at Inst::aoff
// tx, ty, tr: the face and RHS tiles of instances [k0, k0 + n); slots:
// AG_SLOT doubles of scratch per heavy ghost
constexpr int AG_SLOT = 120;
void launch_adj_l(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, const Tile* tx, int ntx,
                  const Tile* ty, int nty, const Tile* tr, int ntr, const GhostRec* heavy, int nh,
                  const GhostRec* cheap, int nc, const double* hrec, const double* X, const double* rbar, double* W,
                  double* Ub, double* pbar, double* slots, int wall_outflow);
int adj_l_launches(int nh, int nc, int wall_outflow);
void launch_adj_copy(cudaStream_t s, const Inst* insts, int k0, int n, long long max_plane, int which, double* set,
                     int dir);
void launch_adj_aos(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, double* aos, double* set,
                    int dir);
void launch_adj_stage(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, int stage,
                      const double* Y, double* U0, double* Uin, double* rbar, const double* R, const DevScalars* sc,
                      double* dtbar);
void launch_adj_dt(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, const double* X,
                   const DevScalars* sc, const double* dtbar, unsigned long long* argmin, double* U0, double* pbar);
void launch_math_check(cudaStream_t s, const double* x, int n, double q, double* out);
} // namespace rh3t
