// C ABI of the rh3t device solver (include/rh3t.h): context set-up from a
// Field + GhostGrid handed over by the host, state transfer, l(), rk3_ssp,
// calc_global_dt and the device-resident time loop (CUDA-graph replay).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rh3t.h"
#include "kernels.cuh"
#include "rh3t_dev.h"

using namespace rh3t;

namespace {

constexpr int TILE = CELL_TILE;

template <class T> cudaError_t dalloc(T** p, size_t n) { return cudaMalloc((void**)p, n * sizeof(T) + 16); }

} // namespace

struct rh3t_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    Inst h{};
    Inst* d_inst = nullptr;
    // device allocations
    double* d_state = nullptr;   // 3 buffers x 6 planes
    uint8_t* d_mask = nullptr;
    double* d_faces = nullptr;   // fx, fy (6 planes each) + dfx, dfy (3 planes each)
    DevBC* d_bcs = nullptr;
    DevScalars* d_sc = nullptr;
    DevError* d_err = nullptr;
    GhostRec* d_ghosts = nullptr;
    int32_t* d_hst = nullptr;
    double* d_hs = nullptr;
    double* d_hw = nullptr;
    double* d_hd = nullptr;
    Tile* d_tx = nullptr;
    Tile* d_ty = nullptr;
    Tile* d_tc = nullptr;
    Tile* d_tr = nullptr;
    double* d_io = nullptr;      // nx*ny*6 staging for AoS transfers / rhs planes
    double* d_io2 = nullptr;
    int n_ghosts = 0, n_heavy = 0, ntx = 0, nty = 0, ntc = 0, ntr = 0;
    std::vector<int32_t> ghost_ij; // for error reports
    cudaGraphExec_t graph = nullptr;
    double graph_cfl = -1.0, graph_tfinal = 0.0;
    long long launches = 0;
    rh3t_error last{};
    std::string msg;
};

static int set_error(rh3t_ctx* c, int code, const char* what) {
    if (c) {
        c->last = rh3t_error{};
        c->last.code = code;
        c->last.ghost = -1;
        std::snprintf(c->last.message, sizeof(c->last.message), "%s", what);
    }
    return code;
}

static int cuda_check(rh3t_ctx* c, cudaError_t e, const char* where) {
    if (e == cudaSuccess) return RH3T_OK;
    char buf[160];
    std::snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    return set_error(c, RH3T_ERR_CUDA, buf);
}

#define CK(ctx, call)                                                  \
    do {                                                               \
        int _rc = cuda_check((ctx), (call), #call);                    \
        if (_rc) return _rc;                                           \
    } while (0)

extern "C" void rh3t_default_params(rh3t_params* p) {
    *p = rh3t_params{1.4, 1.4, 1.4, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.5, 10.0, 1e-12, 0.5};
}

// bc1.rs:930-1037 / 471-545: nearest fluid node to the mirror point 2 P0 - Pg
// among the 9 candidates around coord2idx (field1.rs:68-72). Grid nodes
// outside [0,nx) x [0,ny) count as non-fluid (the reference evaluates its
// polygons there, which for a grid that covers the fluid domain is false).
static bool mirror_source(const rh3t_grid& G, const uint8_t* fluid, long gi, long gj, double p0x, double p0y,
                          long& oi, long& oj) {
    double pgx = G.x0 + (double)gi * G.dx, pgy = G.y0 + (double)gj * G.dy;
    double pix = 2.0 * p0x - pgx, piy = 2.0 * p0y - pgy;
    long ic = (long)std::round((pix - G.x0) / G.dx), jc = (long)std::round((piy - G.y0) / G.dy);
    const long cand[9][2] = {{ic, jc}, {ic - 1, jc}, {ic + 1, jc}, {ic, jc - 1}, {ic, jc + 1},
                             {ic - 1, jc - 1}, {ic - 1, jc + 1}, {ic + 1, jc - 1}, {ic + 1, jc + 1}};
    bool found = false;
    double best = INFINITY;
    for (int k = 0; k < 9; ++k) {
        long a = cand[k][0], b = cand[k][1];
        if (a < 0 || a >= G.nx || b < 0 || b >= G.ny || !fluid[(size_t)a * G.ny + b]) continue;
        double xq = G.x0 + (double)a * G.dx, yq = G.y0 + (double)b * G.dy;
        double d2 = (xq - pix) * (xq - pix) + (yq - piy) * (yq - piy);
        if (d2 < best) { best = d2; oi = a; oj = b; found = true; }
    }
    return found;
}

static DevBC to_dev(const rh3t_bc& b) {
    DevBC d;
    std::memcpy(&d, &b, sizeof(DevBC));
    return d;
}

static_assert(sizeof(DevBC) == sizeof(rh3t_bc), "DevBC mirrors rh3t_bc");
static_assert(sizeof(DevParams) == sizeof(rh3t_params), "DevParams mirrors rh3t_params");

extern "C" int rh3t_create(const rh3t_grid* grid, const rh3t_params* params, const uint8_t* fluid,
                           int32_t n_outer_bc, const rh3t_bc* outer_bcs, int32_t n_inner_bc,
                           const rh3t_bc* inner_bcs, const rh3t_ghost_table* gt, int32_t device, rh3t_ctx** out) {
    if (!out) return RH3T_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!grid || !params || !fluid || !gt || grid->nx <= 0 || grid->ny <= 0 || !(grid->dx > 0) || !(grid->dy > 0) ||
        n_outer_bc < 0 || n_inner_bc < 0 || (n_outer_bc && !outer_bcs) || (n_inner_bc && !inner_bcs))
        return RH3T_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device) return RH3T_ERR_NO_DEVICE;
    rh3t_ctx* c = new rh3t_ctx();
    c->device = device;
    auto fail = [&](int code, const char* m) {
        set_error(c, code, m);
        std::fprintf(stderr, "rh3t_create: %s\n", m);
        rh3t_destroy(c);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(RH3T_ERR_CUDA, "cudaSetDevice failed");
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(RH3T_ERR_CUDA, "stream create failed");

    const long nx = grid->nx, ny = grid->ny;
    const long nxp = nx + 2 * RH3T_PAD;
    const long nyp = ((ny + 2 * RH3T_PAD) + 7) / 8 * 8;
    const long long plane = (long long)nxp * nyp;
    Inst& I = c->h;
    I.nx = (int)nx; I.ny = (int)ny; I.nyp = (int)nyp; I.plane = plane;
    I.dx = grid->dx; I.dy = grid->dy;
    std::memcpy(&I.P, params, sizeof(DevParams));
    I.diffusion = (params->kappa_e != 0.0 || params->kappa_i != 0.0 || params->kappa_r != 0.0) ? 1 : 0;
    I.source = (params->omega_ei != 0.0 || params->omega_er != 0.0) ? 1 : 0;

    // ---- padded mask
    std::vector<uint8_t> mask((size_t)plane, 0);
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j)
            mask[(size_t)(i + RH3T_PAD) * nyp + (j + RH3T_PAD)] = fluid[(size_t)i * ny + j] ? 1 : 0;

    // ---- BC table: outer sides then inner sides
    std::vector<DevBC> bcs;
    for (int k = 0; k < n_outer_bc; ++k) bcs.push_back(to_dev(outer_bcs[k]));
    for (int k = 0; k < n_inner_bc; ++k) bcs.push_back(to_dev(inner_bcs[k]));
    if (bcs.empty()) bcs.push_back(DevBC{});

    // ---- ghost records
    const int ng = gt->n_ghosts, nh = gt->n_heavy;
    if (ng < 0 || nh < 0 || (ng && (!gt->idx || !gt->boundary || !gt->side || !gt->proj || !gt->pre)) ||
        (nh && (!gt->nearest || !gt->stencil || !gt->s || !gt->w || !gt->d)))
        return fail(RH3T_ERR_INVALID_ARGUMENT, "incomplete ghost table");
    std::vector<GhostRec> recs((size_t)ng);
    std::vector<int32_t> hst((size_t)nh * 55);
    auto node = [&](long i, long j) { return (int32_t)((i + RH3T_PAD) * nyp + (j + RH3T_PAD)); };
    c->ghost_ij.assign(gt->idx, gt->idx + 2 * (size_t)ng);
    for (int g = 0; g < ng; ++g) {
        long i = gt->idx[2 * g], j = gt->idx[2 * g + 1];
        if (i < -RH3T_PAD || i >= nx + RH3T_PAD || j < -RH3T_PAD || j >= ny + RH3T_PAD)
            return fail(RH3T_ERR_GEOMETRY, "ghost index outside the radius-4 band of the grid");
        if (i >= 0 && i < nx && j >= 0 && j < ny && fluid[(size_t)i * ny + j])
            return fail(RH3T_ERR_GEOMETRY, "ghost index is a fluid node");
        int side = gt->side[g];
        int bidx = gt->boundary[g] == 0 ? side : n_outer_bc + side;
        if (side < 0 || (gt->boundary[g] == 0 && side >= n_outer_bc) || (gt->boundary[g] != 0 && side >= n_inner_bc))
            return fail(RH3T_ERR_INVALID_ARGUMENT, "ghost side out of range");
        GhostRec& R = recs[g];
        std::memset(&R, 0, sizeof(R));
        R.inst = 0; R.bc = bidx; R.kind = bcs[bidx].kind; R.node = node(i, j); R.gid = g;
        R.p0x = gt->proj[5 * g]; R.p0y = gt->proj[5 * g + 1]; R.nx = gt->proj[5 * g + 2];
        R.ny = gt->proj[5 * g + 3]; R.dist = gt->proj[5 * g + 4];
        R.heavy = -1;
        const int kind = R.kind;
        if (kind == BC_WALL || kind == BC_OUTFLOW || kind == BC_FAR_FIELD) {
            int k = gt->pre[g];
            if (k < 0 || k >= nh) return fail(RH3T_ERR_INVALID_ARGUMENT, "heavy ghost without GhostBC data");
            R.heavy = k;
            long ni = gt->nearest[2 * k], nj = gt->nearest[2 * k + 1];
            if (ni < 0 || ni >= nx || nj < 0 || nj >= ny) return fail(RH3T_ERR_GEOMETRY, "nearest node outside grid");
            R.src = node(ni, nj);
        } else if (kind == BC_REFLECTIVE_WALL || kind == BC_ZEROTH_ORDER) {
            long oi = 0, oj = 0;
            if (!mirror_source(*grid, fluid, i, j, R.p0x, R.p0y, oi, oj))
                return fail(RH3T_ERR_GEOMETRY, "cannot find reflected interior point for ghost");
            R.src = node(oi, oj);
        } else if (kind == BC_PERIODIC) {
            // bc1.rs:547-607 (ly a parameter instead of the hardcoded 0.5)
            long np = (long)std::round(params->periodic_ly / grid->dy);
            if (np <= 0) return fail(RH3T_ERR_PERIODIC_WRAP, "periodic wrap length is zero");
            long jw = ((j % np) + np) % np;
            if (!(i >= 0 && i < nx && jw >= 0 && jw < ny && fluid[(size_t)i * ny + jw]))
                return fail(RH3T_ERR_PERIODIC_WRAP, "periodic wrapped point is not fluid");
            R.src = node(i, jw);
        } else {
            R.src = R.node;
        }
    }
    for (long k = 0; k < (long)nh * 55; ++k) {
        uint32_t l = gt->stencil[k];
        long i = (long)(l / (uint32_t)ny), j = (long)(l % (uint32_t)ny);
        if (i >= nx || !fluid[l]) return fail(RH3T_ERR_GEOMETRY, "E_r stencil node is not fluid");
        hst[k] = node(i, j);
    }

    // ---- tiles
    std::vector<Tile> tx, ty, tc, tr;
    auto isf = [&](long i, long j) { return i >= 0 && i < nx && j >= 0 && j < ny && fluid[(size_t)i * ny + j]; };
    // x faces (i - 1/2, j), i in [0, nx]: tiles of FX_TI x FX_TJ faces
    for (long i0 = 0; i0 <= nx; i0 += FX_TI)
        for (long j0 = 0; j0 < ny; j0 += FX_TJ) {
            bool any = false;
            for (long i = i0; i < std::min(nx + 1, i0 + FX_TI) && !any; ++i)
                for (long j = j0; j < std::min(ny, j0 + FX_TJ) && !any; ++j) any = isf(i, j) || isf(i - 1, j);
            if (any) tx.push_back({0, (int)i0, (int)j0, 0});
        }
    // y faces (i, j - 1/2), j in [0, ny]: tiles of FY_TJ faces along j
    for (long i = 0; i < nx; ++i)
        for (long j0 = 0; j0 <= ny; j0 += FY_TJ) {
            bool any = false;
            for (long j = j0; j <= std::min(ny, j0 + FY_TJ - 1) && !any; ++j) any = isf(i, j) || isf(i, j - 1);
            if (any) ty.push_back({0, (int)i, (int)j0, 0});
        }
    for (long i = 0; i < nx; ++i)
        for (long j0 = 0; j0 < ny; j0 += TILE) {
            bool any = false;
            for (long j = j0; j < std::min(ny, j0 + TILE) && !any; ++j) any = isf(i, j);
            if (any) tc.push_back({0, (int)i, (int)j0, 0});
        }
    // RHS / stage-update tiles: RHS_TI x RHS_TJ cells
    for (long i0 = 0; i0 < nx; i0 += RHS_TI)
        for (long j0 = 0; j0 < ny; j0 += RHS_TJ) {
            bool any = false;
            for (long i = i0; i < std::min(nx, i0 + RHS_TI) && !any; ++i)
                for (long j = j0; j < std::min(ny, j0 + RHS_TJ) && !any; ++j) any = isf(i, j);
            if (any) tr.push_back({0, (int)i0, (int)j0, 0});
        }
    c->ntx = (int)tx.size(); c->nty = (int)ty.size(); c->ntc = (int)tc.size(); c->ntr = (int)tr.size();
    I.n_tiles_dt = c->ntc;
    c->n_ghosts = ng; c->n_heavy = nh;

    // ---- device allocations
    const long long nfx = (long long)(nx + 1) * ny, nfy = (long long)nx * (ny + 1);
    cudaError_t e = cudaSuccess;
#define DA(ptr, n) do { e = dalloc(&(ptr), (size_t)(n)); if (e != cudaSuccess) return fail(RH3T_ERR_CUDA, "cudaMalloc failed: " #ptr); } while (0)
    DA(c->d_state, 3 * 6 * plane);
    DA(c->d_mask, plane);
    const long long nfaces = 6 * (nfx + nfy) + (I.diffusion ? 3 * (nfx + nfy) : 0);
    DA(c->d_faces, nfaces);
    DA(c->d_bcs, bcs.size());
    DA(c->d_sc, 1);
    DA(c->d_err, 1);
    DA(c->d_inst, 1);
    DA(c->d_ghosts, std::max(ng, 1));
    DA(c->d_hst, std::max((long long)nh * 55, 1LL));
    DA(c->d_hs, std::max((long long)nh * 979, 1LL));
    DA(c->d_hw, std::max((long long)nh * 225, 1LL));
    DA(c->d_hd, std::max((long long)nh * 5, 1LL));
    DA(c->d_tx, std::max(c->ntx, 1));
    DA(c->d_ty, std::max(c->nty, 1));
    DA(c->d_tc, std::max(c->ntc, 1));
    DA(c->d_tr, std::max(c->ntr, 1));
    DA(c->d_io, nx * ny * 6);
    DA(c->d_io2, std::max((long long)nx * ny, (long long)ng) * 6); // rhs planes or ghost values
#undef DA
    I.U = c->d_state; I.A = c->d_state + 6 * plane; I.B = c->d_state + 12 * plane;
    I.mask = c->d_mask;
    I.fx = c->d_faces; I.fy = c->d_faces + 6 * nfx;
    I.dfx = I.diffusion ? c->d_faces + 6 * (nfx + nfy) : nullptr;
    I.dfy = I.diffusion ? I.dfx + 3 * nfx : nullptr;
    I.bcs = c->d_bcs; I.sc = c->d_sc; I.err = c->d_err;

    DevScalars sc{};
    sc.dt_cfl_bits = 0ull;
    {
        // orderable key of +inf (see kernels.cu dkey)
        double inf = INFINITY;
        unsigned long long b;
        std::memcpy(&b, &inf, 8);
        sc.dt_cfl_bits = b | 0x8000000000000000ull;
    }
    sc.cfl_factor = 0.05; sc.t_final = INFINITY;
    DevError er{~0ull};
    cudaStream_t s = c->stream;
#define CP(dst, src, n) do { e = cudaMemcpyAsync((dst), (src), (size_t)(n), cudaMemcpyHostToDevice, s); if (e != cudaSuccess) return fail(RH3T_ERR_CUDA, "upload failed"); } while (0)
    if (cudaMemsetAsync(c->d_state, 0, (size_t)3 * 6 * plane * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(c->d_faces, 0, (size_t)nfaces * sizeof(double), s) != cudaSuccess)
        return fail(RH3T_ERR_CUDA, "memset failed");
    CP(c->d_mask, mask.data(), plane);
    CP(c->d_bcs, bcs.data(), bcs.size() * sizeof(DevBC));
    CP(c->d_sc, &sc, sizeof(sc));
    CP(c->d_err, &er, sizeof(er));
    CP(c->d_inst, &I, sizeof(Inst));
    if (ng) CP(c->d_ghosts, recs.data(), (size_t)ng * sizeof(GhostRec));
    if (nh) {
        CP(c->d_hst, hst.data(), hst.size() * sizeof(int32_t));
        CP(c->d_hs, gt->s, (size_t)nh * 979 * sizeof(double));
        CP(c->d_hw, gt->w, (size_t)nh * 225 * sizeof(double));
        CP(c->d_hd, gt->d, (size_t)nh * 5 * sizeof(double));
    }
    if (c->ntx) CP(c->d_tx, tx.data(), tx.size() * sizeof(Tile));
    if (c->nty) CP(c->d_ty, ty.data(), ty.size() * sizeof(Tile));
    if (c->ntc) CP(c->d_tc, tc.data(), tc.size() * sizeof(Tile));
    if (c->ntr) CP(c->d_tr, tr.data(), tr.size() * sizeof(Tile));
#undef CP
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail(RH3T_ERR_CUDA, "set-up synchronize failed");
    *out = c;
    return RH3T_OK;
}

extern "C" void rh3t_destroy(rh3t_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    void* ptrs[] = {c->d_state, c->d_mask, c->d_faces, c->d_bcs, c->d_sc, c->d_err, c->d_inst, c->d_ghosts,
                    c->d_hst, c->d_hs, c->d_hw, c->d_hd, c->d_tx, c->d_ty, c->d_tc, c->d_tr, c->d_io, c->d_io2};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

// decode the device error key into rh3t_error (see rh3t_dev.h DevError)
static int fetch_error(rh3t_ctx* c) {
    DevError er;
    CK(c, cudaMemcpyAsync(&er, c->d_err, sizeof(er), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    if (er.key == ~0ull) return RH3T_OK;
    rh3t_error& L = c->last;
    L = rh3t_error{};
    unsigned long long k = er.key;
    int phase = (int)((k >> 37) & 7ull);
    L.code = (int)((k >> 32) & 31ull);
    L.step = (int64_t)(k >> 40);
    unsigned idx = (unsigned)(k & 0xffffffffull);
    L.ghost = -1;
    if (phase == 0) {
        L.stage = 0;
        std::snprintf(L.message, sizeof(L.message), "non-positive dt");
    } else if (phase % 2 == 1) {
        L.stage = (phase + 1) / 2;
        L.ghost = (int)idx;
        if ((int)idx < c->n_ghosts) { L.i = c->ghost_ij[2 * idx]; L.j = c->ghost_ij[2 * idx + 1]; }
        std::snprintf(L.message, sizeof(L.message), L.code == RH3T_ERR_SINGULAR_ILW
                          ? "singular ILW/extrapolation system at boundary"
                          : "NON-FINITE GHOST STATE");
    } else {
        L.stage = phase / 2;
        L.i = (int)(idx / (unsigned)c->h.ny);
        L.j = (int)(idx % (unsigned)c->h.ny);
        std::snprintf(L.message, sizeof(L.message), "non-physical state at (%d, %d) in RK%d state", L.i, L.j,
                      L.stage);
    }
    return L.code;
}

static void enqueue_stage(rh3t_ctx* c, int stage) {
    cudaStream_t s = c->stream;
    launch_ghosts(s, c->d_inst, c->d_ghosts, c->n_ghosts, c->d_hst, c->d_hs, c->d_hw, c->d_hd, stage);
    launch_flux(s, c->d_inst, c->d_tx, c->ntx, c->d_ty, c->nty, stage);
    launch_rhs_stage(s, c->d_inst, c->d_tr, c->ntr, stage, 1, nullptr);
    c->launches += (c->n_ghosts > 0) + 2;
}

static void enqueue_step(rh3t_ctx* c) {
    launch_dt(c->stream, c->d_inst, c->d_tc, c->ntc, 1);
    c->launches += 1;
    for (int st = 0; st < 3; ++st) enqueue_stage(c, st);
}

static int set_step_params(rh3t_ctx* c, double cfl, double t_final) {
    // patch cfl_factor / t_final in the device scalars (two doubles)
    size_t off = offsetof(DevScalars, cfl_factor);
    double v[2] = {cfl, t_final};
    CK(c, cudaMemcpyAsync((char*)c->d_sc + off, v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
    return RH3T_OK;
}

extern "C" int rh3t_upload_state(rh3t_ctx* c, const double* value, double time) {
    if (!c || !value) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    long long n = (long long)c->h.nx * c->h.ny;
    CK(c, cudaMemcpyAsync(c->d_io, value, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_scatter(c->stream, c->d_inst, 0, n, c->d_io, time);
    c->launches += 1;
    CK(c, cudaGetLastError());
    CK(c, cudaStreamSynchronize(c->stream));
    return RH3T_OK;
}

extern "C" int rh3t_download_state(rh3t_ctx* c, double* value, double* time) {
    if (!c || !value) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    long long n = (long long)c->h.nx * c->h.ny;
    launch_gather(c->stream, c->d_inst, 0, n, c->d_io);
    c->launches += 1;
    CK(c, cudaGetLastError());
    CK(c, cudaMemcpyAsync(value, c->d_io, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (time) CK(c, cudaMemcpyAsync(time, (char*)c->d_sc + offsetof(DevScalars, t_after), sizeof(double),
                                    cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return RH3T_OK;
}

extern "C" int rh3t_l(rh3t_ctx* c, double* rhs, double* ghost_values) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    long long n = (long long)c->h.nx * c->h.ny;
    // ghost time of a standalone l(): the field time (Field::time)
    size_t off_t = offsetof(DevScalars, t_after), off_ts = offsetof(DevScalars, t_stage);
    CK(c, cudaMemcpyAsync((char*)c->d_sc + off_ts, (char*)c->d_sc + off_t, sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
    launch_ghosts(s, c->d_inst, c->d_ghosts, c->n_ghosts, c->d_hst, c->d_hs, c->d_hw, c->d_hd, 0);
    launch_flux(s, c->d_inst, c->d_tx, c->ntx, c->d_ty, c->nty, 0);
    CK(c, cudaMemsetAsync(c->d_io2, 0, (size_t)n * 6 * sizeof(double), s));
    launch_rhs_stage(s, c->d_inst, c->d_tr, c->ntr, 0, 0, c->d_io2);
    c->launches += 3;
    if (rhs) {
        launch_planes_to_aos(s, c->d_io2, n, c->d_io);
        c->launches += 1;
        CK(c, cudaMemcpyAsync(rhs, c->d_io, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (ghost_values && c->n_ghosts) {
        launch_ghost_values(s, c->d_inst, c->d_ghosts, c->n_ghosts, c->d_io2);
        c->launches += 1;
        CK(c, cudaMemcpyAsync(ghost_values, c->d_io2, (size_t)c->n_ghosts * 6 * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    }
    CK(c, cudaGetLastError());
    return fetch_error(c);
}

extern "C" int rh3t_calc_global_dt(rh3t_ctx* c, double* dt_cfl) {
    if (!c || !dt_cfl) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    launch_dt(c->stream, c->d_inst, c->d_tc, c->ntc, 0);
    c->launches += 1;
    CK(c, cudaGetLastError());
    CK(c, cudaMemcpyAsync(dt_cfl, (char*)c->d_sc + offsetof(DevScalars, dt_cfl), sizeof(double),
                          cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return RH3T_OK;
}

extern "C" int rh3t_rk3_ssp(rh3t_ctx* c, double dt) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    launch_set_dt(c->stream, c->d_inst, 1, dt);
    c->launches += 1;
    for (int st = 0; st < 3; ++st) enqueue_stage(c, st);
    CK(c, cudaGetLastError());
    return fetch_error(c);
}

static int ensure_graph(rh3t_ctx* c) {
    if (c->graph) return RH3T_OK;
    cudaGraph_t g;
    long long before = c->launches;
    CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->launches = before; // captured launches are counted at replay
    CK(c, e);
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    CK(c, e);
    return RH3T_OK;
}

static long long launches_per_step(const rh3t_ctx* c) { return 1 + 3 * ((c->n_ghosts > 0) + 2); }

extern "C" int rh3t_advance(rh3t_ctx* c, int32_t nsteps, double cfl_factor, double t_final, int32_t use_graph) {
    if (!c || nsteps < 0) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    int rc = set_step_params(c, cfl_factor, t_final);
    if (rc) return rc;
    if (use_graph) {
        rc = ensure_graph(c);
        if (rc) return rc;
        for (int n = 0; n < nsteps; ++n) CK(c, cudaGraphLaunch(c->graph, c->stream));
        c->launches += (long long)nsteps * launches_per_step(c);
    } else {
        for (int n = 0; n < nsteps; ++n) enqueue_step(c);
    }
    CK(c, cudaGetLastError());
    return fetch_error(c);
}

extern "C" int rh3t_step_host(rh3t_ctx* c, double* value, double* time, double cfl_factor, double* dt_out) {
    if (!c || !value || !time) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    long long n = (long long)c->h.nx * c->h.ny;
    int rc = set_step_params(c, cfl_factor, INFINITY);
    if (rc) return rc;
    rc = ensure_graph(c);
    if (rc) return rc;
    CK(c, cudaMemcpyAsync(c->d_io, value, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_scatter(s, c->d_inst, 0, n, c->d_io, *time);
    CK(c, cudaGraphLaunch(c->graph, s));
    launch_gather(s, c->d_inst, 0, n, c->d_io);
    c->launches += 2 + launches_per_step(c);
    CK(c, cudaMemcpyAsync(value, c->d_io, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(c, cudaMemcpyAsync(time, (char*)c->d_sc + offsetof(DevScalars, t_after), sizeof(double),
                          cudaMemcpyDeviceToHost, s));
    if (dt_out)
        CK(c, cudaMemcpyAsync(dt_out, (char*)c->d_sc + offsetof(DevScalars, dt), sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    CK(c, cudaGetLastError());
    return fetch_error(c);
}

extern "C" int rh3t_profile_steps(rh3t_ctx* c, int32_t nsteps, double cfl_factor, double* ms_out,
                                  int64_t* launches_out) {
    if (!c || !ms_out || nsteps < 0) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    int rc = set_step_params(c, cfl_factor, INFINITY);
    if (rc) return rc;
    cudaStream_t s = c->stream;
    std::vector<cudaEvent_t> ev;
    std::vector<int> cls;
    auto mark = [&](int k) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        ev.push_back(e);
        cls.push_back(k);
    };
    for (int n = 0; n < nsteps; ++n) {
        mark(-1);
        launch_dt(s, c->d_inst, c->d_tc, c->ntc, 1);
        mark(3);
        for (int st = 0; st < 3; ++st) {
            launch_ghosts(s, c->d_inst, c->d_ghosts, c->n_ghosts, c->d_hst, c->d_hs, c->d_hw, c->d_hd, st);
            mark(0);
            launch_flux(s, c->d_inst, c->d_tx, c->ntx, c->d_ty, c->nty, st);
            mark(1);
            launch_rhs_stage(s, c->d_inst, c->d_tr, c->ntr, st, 1, nullptr);
            mark(2);
        }
    }
    c->launches += (long long)nsteps * launches_per_step(c);
    CK(c, cudaGetLastError());
    CK(c, cudaStreamSynchronize(s));
    double acc[4] = {0, 0, 0, 0};
    int64_t cnt[4] = {0, 0, 0, 0};
    for (size_t k = 1; k < ev.size(); ++k) {
        if (cls[k] < 0) continue;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[k - 1], ev[k]);
        acc[cls[k]] += ms;
        cnt[cls[k]] += 1;
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 4; ++k) ms_out[k] = acc[k];
    if (launches_out)
        for (int k = 0; k < 4; ++k) launches_out[k] = cnt[k];
    return fetch_error(c);
}

extern "C" int rh3t_fp64_peak(int32_t device, double* tflops) {
    if (!tflops) return RH3T_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return RH3T_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return RH3T_ERR_CUDA;
    double* out = nullptr;
    int blocks = prop.multiProcessorCount * 8;
    if (cudaMalloc(&out, blocks * sizeof(double)) != cudaSuccess) return RH3T_ERR_CUDA;
    cudaStream_t s;
    cudaStreamCreate(&s);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int iters = 1 << 16;
    launch_dfma(s, blocks, out, iters / 16); // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a, s);
        launch_dfma(s, blocks, out, iters);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        double flops = 2.0 * 8.0 * (double)iters * (double)blocks * 256.0;
        if (ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaStreamDestroy(s);
    cudaFree(out);
    if (e != cudaSuccess) return RH3T_ERR_CUDA;
    *tflops = best;
    return RH3T_OK;
}

extern "C" int rh3t_math_check(int32_t device, const double* x, int32_t n, double q, double* out) {
    if (!x || !out || n < 0) return RH3T_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return RH3T_ERR_NO_DEVICE;
    double *dx = nullptr, *dout = nullptr;
    if (cudaMalloc(&dx, (size_t)std::max(n, 1) * sizeof(double)) != cudaSuccess) return RH3T_ERR_CUDA;
    if (cudaMalloc(&dout, (size_t)std::max(n, 1) * 3 * sizeof(double)) != cudaSuccess) {
        cudaFree(dx);
        return RH3T_ERR_CUDA;
    }
    cudaError_t e = cudaMemcpy(dx, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) {
        launch_math_check(0, dx, n, q, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dout);
    return e == cudaSuccess ? RH3T_OK : RH3T_ERR_CUDA;
}

extern "C" int rh3t_last_dt(rh3t_ctx* c, double* dt) {
    if (!c || !dt) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaMemcpyAsync(dt, (char*)c->d_sc + offsetof(DevScalars, dt), sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return RH3T_OK;
}

extern "C" int rh3t_synchronize(rh3t_ctx* c) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaStreamSynchronize(c->stream));
    return fetch_error(c);
}

extern "C" int rh3t_last_error(const rh3t_ctx* c, rh3t_error* out) {
    if (!c || !out) return RH3T_ERR_INVALID_ARGUMENT;
    *out = c->last;
    return c->last.code;
}

extern "C" int64_t rh3t_kernel_launches(const rh3t_ctx* c) { return c ? c->launches : 0; }
extern "C" void* rh3t_stream(const rh3t_ctx* c) { return c ? (void*)c->stream : nullptr; }
