// Host-side state of an rh3t context (include/rh3t.h rh3t_ctx): one or more
// independent solver instances resident on one GPU, advanced together by one
// launch per kernel phase. Private to the library (context.cu, tune.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/rh3t.h"
#include "rh3t_dev.h"

namespace rh3t {

struct Shape {
    int lgx = FX_LG_DEF, lgy = FY_LG_DEF, lgr = RHS_LG_DEF;
};

struct HostInst {
    rh3t_grid grid{};
    long nx = 0, ny = 0, nyp = 0;
    long long plane = 0, cell_off = 0;
    std::vector<uint8_t> fluid;    // nx*ny (tile lists are rebuilt from it)
    std::vector<int32_t> ghost_ij; // (i, j) per ghost, for error records
    int n_ghosts = 0, ghost_off = 0;
    int gh0 = 0, ngh = 0, gc0 = 0, ngc = 0; // heavy / cheap segments of d_gpart
    int tx0 = 0, ntx = 0, ty0 = 0, nty = 0, tc0 = 0, ntc = 0, tr0 = 0, ntr = 0;
    int diffusion = 0;
    int n_wall_outflow = 0;        // heavy ghosts of kind Wall or Outflow
    Shape shape;
};

// a contiguous range of instances [k0, k1)
struct Span {
    int k0, k1;
};

} // namespace rh3t

struct rh3t_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_inst = 0;
    std::vector<rh3t::Inst> h;
    std::vector<rh3t::HostInst> hi;
    rh3t::Inst* d_inst = nullptr;
    double* d_state = nullptr;   // per instance: 3 buffers x 6 planes
    uint8_t* d_mask = nullptr;
    double* d_faces = nullptr;   // per instance: fx, fy (6 planes each) + dfx, dfy (3 planes each)
    rh3t::DevBC* d_bcs = nullptr;
    rh3t::DevScalars* d_sc = nullptr;
    rh3t::DevError* d_err = nullptr;
    double* d_times = nullptr;   // upload times, one per instance
    rh3t::GhostRec* d_ghosts = nullptr; // table order (instance-major, gid within)
    rh3t::GhostRec* d_gpart = nullptr;  // heavy ghosts by heavy slot, then the cheap ones
    double* d_hrec = nullptr;           // heavy records (GH_REC doubles each)
    rh3t::Tile* d_tx = nullptr;
    rh3t::Tile* d_ty = nullptr;
    rh3t::Tile* d_tc = nullptr;
    rh3t::Tile* d_tr = nullptr;
    int ntx = 0, nty = 0, ntc = 0, ntr = 0;
    double* d_io = nullptr;      // total_cells*6: AoS staging of all instances
    double* d_io2 = nullptr;     // total_cells*6 rhs planes + max_ghosts*6 ghost values
    long long total_cells = 0, max_cells = 0;
    long long total_planes = 0;   // sum of 6*plane: size of a batch-wide plane set
    long long max_faces = 0;      // max over instances of max((nx+1)*ny, nx*(ny+1))
    struct AdjBuffers* adj = nullptr;
    struct rh3t_io* io = nullptr; // snapshot and diagnostic buffers (io.cu)
    int n_ghosts = 0, n_heavy = 0, n_gheavy = 0, n_gcheap = 0, max_ghosts = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t xfer[2] = {nullptr, nullptr};  // host-copy streams of rh3t_step_host_batch (in, out)
    rh3t::DevScalars* h_sc = nullptr;            // pinned: the instances' scalars read back by it
    long long launches = 0;
    rh3t_error last{};
    std::vector<int32_t> inst_status;
};

namespace rh3t {
int set_error(rh3t_ctx* c, int code, const char* what);
int cuda_check(rh3t_ctx* c, cudaError_t e, const char* where);
// rebuild and upload every tile list from the instances' shapes (drops the graph)
int make_tiles(rh3t_ctx* c);
// x-face, y-face and RHS tiles of one instance for a given shape
void instance_tiles(const HostInst& H, const Shape& sh, int inst, std::vector<Tile>* tx, std::vector<Tile>* ty,
                    std::vector<Tile>* tr);
// returns the number of kernels launched (x and y faces: flux_launches)
int enqueue_flux(rh3t_ctx* c, cudaStream_t s, int stage, Span r);
void enqueue_rhs(rh3t_ctx* c, cudaStream_t s, int stage, int mode, double* rhs, Span r);
void adj_free(rh3t_ctx* c);
void io_free(rh3t_ctx* c);
} // namespace rh3t

#define CK(ctx, call)                                                  \
    do {                                                               \
        int _rc = rh3t::cuda_check((ctx), (call), #call);              \
        if (_rc) return _rc;                                           \
    } while (0)
