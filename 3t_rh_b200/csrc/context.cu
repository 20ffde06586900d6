// C ABI of the rh3t device solver (include/rh3t.h): context set-up from one
// or more Field + GhostGrid pairs handed over by the host (a batch of
// independent instances; the plain solver is a batch of one), state
// transfer, l(), rk3_ssp, calc_global_dt and the device-resident time loop
// (CUDA-graph replay of one step of every instance).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.cuh"

using namespace rh3t;

namespace {

template <class T> cudaError_t dalloc(T** p, size_t n) { return cudaMalloc((void**)p, n * sizeof(T) + 16); }

template <class T> void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

Span all(const rh3t_ctx* c) { return Span{0, c->n_inst}; }

} // namespace

namespace rh3t {

int set_error(rh3t_ctx* c, int code, const char* what) {
    if (c) {
        c->last = rh3t_error{};
        c->last.code = code;
        c->last.ghost = -1;
        c->last.instance = -1;
        std::snprintf(c->last.message, sizeof(c->last.message), "%s", what);
    }
    return code;
}

int cuda_check(rh3t_ctx* c, cudaError_t e, const char* where) {
    if (e == cudaSuccess) return RH3T_OK;
    char buf[160];
    std::snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    return set_error(c, RH3T_ERR_CUDA, buf);
}

void instance_tiles(const HostInst& H, const Shape& sh, int inst, std::vector<Tile>* tx, std::vector<Tile>* ty,
                    std::vector<Tile>* tr) {
    const long nx = H.nx, ny = H.ny;
    const uint8_t* fl = H.fluid.data();
    auto isf = [&](long i, long j) { return i >= 0 && i < nx && j >= 0 && j < ny && fl[(size_t)i * ny + j]; };
    if (tx) { // x faces (i - 1/2, j), i in [0, nx]
        const long rows = FLUX_FACES >> sh.lgx, cols = 1L << sh.lgx;
        for (long i0 = 0; i0 <= nx; i0 += rows)
            for (long j0 = 0; j0 < ny; j0 += cols) {
                bool any = false;
                for (long i = i0; i < std::min(nx + 1, i0 + rows) && !any; ++i)
                    for (long j = j0; j < std::min(ny, j0 + cols) && !any; ++j) any = isf(i, j) || isf(i - 1, j);
                if (any) tx->push_back({inst, (int)i0, (int)j0, sh.lgx});
            }
    }
    if (ty) { // y faces (i, j - 1/2), j in [0, ny]
        const long rows = FLUX_FACES >> sh.lgy, cols = 1L << sh.lgy;
        for (long i0 = 0; i0 < nx; i0 += rows)
            for (long j0 = 0; j0 <= ny; j0 += cols) {
                bool any = false;
                for (long i = i0; i < std::min(nx, i0 + rows) && !any; ++i)
                    for (long j = j0; j < std::min(ny + 1, j0 + cols) && !any; ++j) any = isf(i, j) || isf(i, j - 1);
                if (any) ty->push_back({inst, (int)i0, (int)j0, sh.lgy});
            }
    }
    if (tr) { // RHS / stage-update cells
        const long rows = RHS_THREADS >> sh.lgr, cols = 1L << sh.lgr;
        for (long i0 = 0; i0 < nx; i0 += rows)
            for (long j0 = 0; j0 < ny; j0 += cols) {
                bool any = false;
                for (long i = i0; i < std::min(nx, i0 + rows) && !any; ++i)
                    for (long j = j0; j < std::min(ny, j0 + cols) && !any; ++j) any = isf(i, j);
                if (any) tr->push_back({inst, (int)i0, (int)j0, sh.lgr});
            }
    }
}

int make_tiles(rh3t_ctx* c) {
    std::vector<Tile> tx, ty, tc, tr;
    for (int k = 0; k < c->n_inst; ++k) {
        HostInst& H = c->hi[k];
        H.tx0 = (int)tx.size(); H.ty0 = (int)ty.size(); H.tc0 = (int)tc.size(); H.tr0 = (int)tr.size();
        instance_tiles(H, H.shape, k, &tx, &ty, &tr);
        const long nx = H.nx, ny = H.ny;
        for (long i = 0; i < nx; ++i)
            for (long j0 = 0; j0 < ny; j0 += CELL_TILE) {
                bool any = false;
                for (long j = j0; j < std::min(ny, j0 + (long)CELL_TILE) && !any; ++j)
                    any = H.fluid[(size_t)i * ny + j] != 0;
                if (any) tc.push_back({k, (int)i, (int)j0, 0});
            }
        H.ntx = (int)tx.size() - H.tx0; H.nty = (int)ty.size() - H.ty0;
        H.ntc = (int)tc.size() - H.tc0; H.ntr = (int)tr.size() - H.tr0;
        c->h[k].n_tiles_dt = H.ntc;
    }
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    CK(c, cudaStreamSynchronize(c->stream));
    dfree(c->d_tx); dfree(c->d_ty); dfree(c->d_tc); dfree(c->d_tr);
    CK(c, dalloc(&c->d_tx, std::max<size_t>(tx.size(), 1)));
    CK(c, dalloc(&c->d_ty, std::max<size_t>(ty.size(), 1)));
    CK(c, dalloc(&c->d_tc, std::max<size_t>(tc.size(), 1)));
    CK(c, dalloc(&c->d_tr, std::max<size_t>(tr.size(), 1)));
    c->ntx = (int)tx.size(); c->nty = (int)ty.size(); c->ntc = (int)tc.size(); c->ntr = (int)tr.size();
    cudaStream_t s = c->stream;
    if (c->ntx) CK(c, cudaMemcpyAsync(c->d_tx, tx.data(), tx.size() * sizeof(Tile), cudaMemcpyHostToDevice, s));
    if (c->nty) CK(c, cudaMemcpyAsync(c->d_ty, ty.data(), ty.size() * sizeof(Tile), cudaMemcpyHostToDevice, s));
    if (c->ntc) CK(c, cudaMemcpyAsync(c->d_tc, tc.data(), tc.size() * sizeof(Tile), cudaMemcpyHostToDevice, s));
    if (c->ntr) CK(c, cudaMemcpyAsync(c->d_tr, tr.data(), tr.size() * sizeof(Tile), cudaMemcpyHostToDevice, s));
    CK(c, cudaMemcpyAsync(c->d_inst, c->h.data(), c->h.size() * sizeof(Inst), cudaMemcpyHostToDevice, s));
    CK(c, cudaStreamSynchronize(s));
    return RH3T_OK;
}

// returns the number of kernels launched
int enqueue_flux(rh3t_ctx* c, cudaStream_t s, int stage, Span r) {
    const HostInst &a = c->hi[r.k0], &b = c->hi[r.k1 - 1];
    const int ntx = b.tx0 + b.ntx - a.tx0, nty = b.ty0 + b.nty - a.ty0;
    launch_flux(s, c->d_inst, c->d_tx + a.tx0, ntx, c->d_ty + a.ty0, nty, stage);
    return flux_launches(ntx, nty);
}

void enqueue_rhs(rh3t_ctx* c, cudaStream_t s, int stage, int mode, double* rhs, Span r) {
    const HostInst &a = c->hi[r.k0], &b = c->hi[r.k1 - 1];
    launch_rhs_stage(s, c->d_inst, c->d_tr + a.tr0, b.tr0 + b.ntr - a.tr0, stage, mode, rhs);
}

} // namespace rh3t

namespace {

// heavy and cheap ghost counts of an instance range
void ghost_counts(const rh3t_ctx* c, Span r, int& nh, int& nc) {
    const HostInst &a = c->hi[r.k0], &b = c->hi[r.k1 - 1];
    nh = b.gh0 + b.ngh - a.gh0;
    nc = b.gc0 + b.ngc - a.gc0;
}

// returns the number of kernels launched
int enqueue_ghosts(rh3t_ctx* c, cudaStream_t s, int stage, Span r) {
    const HostInst& a = c->hi[r.k0];
    int nh, nc;
    ghost_counts(c, r, nh, nc);
    launch_ghosts(s, c->d_inst, c->d_gpart + a.gh0, nh, c->d_gpart + c->n_gheavy + a.gc0, nc, c->d_hrec, stage);
    return ghost_launches(nh, nc);
}

void enqueue_dt(rh3t_ctx* c, cudaStream_t s, int mode, Span r) {
    const HostInst &a = c->hi[r.k0], &b = c->hi[r.k1 - 1];
    launch_dt(s, c->d_inst, c->d_tc + a.tc0, b.tc0 + b.ntc - a.tc0, mode);
}

void enqueue_stage(rh3t_ctx* c, int stage, Span r) {
    cudaStream_t s = c->stream;
    const int ng = enqueue_ghosts(c, s, stage, r);
    const int nf = enqueue_flux(c, s, stage, r);
    enqueue_rhs(c, s, stage, 1, nullptr, r);
    c->launches += ng + nf + 1;
}

void enqueue_step(rh3t_ctx* c, Span r) {
    enqueue_dt(c, c->stream, 1, r);
    c->launches += 1;
    for (int st = 0; st < 3; ++st) enqueue_stage(c, st, r);
}

long long launches_per_step(const rh3t_ctx* c) {
    int nh, nc;
    ghost_counts(c, all(c), nh, nc);
    const HostInst &a = c->hi[0], &b = c->hi[c->n_inst - 1];
    const int nf = flux_launches(b.tx0 + b.ntx - a.tx0, b.ty0 + b.nty - a.ty0);
    return 1 + 3 * (ghost_launches(nh, nc) + nf + 1);
}

// bc1.rs:930-1037 / 471-545: nearest fluid node to the mirror point 2 P0 - Pg
// among the 9 candidates around coord2idx (field1.rs:68-72). Grid nodes
// outside [0,nx) x [0,ny) count as non-fluid (the reference evaluates its
// polygons there, which for a grid that covers the fluid domain is false).
bool mirror_source(const rh3t_grid& G, const uint8_t* fluid, long gi, long gj, double p0x, double p0y, long& oi,
                   long& oj) {
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

DevBC to_dev(const rh3t_bc& b) {
    DevBC d;
    std::memcpy(&d, &b, sizeof(DevBC));
    return d;
}

static_assert(sizeof(DevBC) == sizeof(rh3t_bc), "DevBC mirrors rh3t_bc");
static_assert(sizeof(DevParams) == sizeof(rh3t_params), "DevParams mirrors rh3t_params");

// host arrays of one instance, before concatenation
struct Built {
    std::vector<uint8_t> mask; // padded
    std::vector<DevBC> bcs;
    std::vector<GhostRec> recs; // table order
    std::vector<double> hrec;   // n_heavy * GH_REC
    int n_heavy = 0;
};

// Validates one instance description and resolves its ghost records
// (ghost.rs:18-46, bc1.rs:50-57 and the static parts of the cheap BCs).
int build_instance(const rh3t_instance& d, int inst, HostInst& H, Inst& I, Built& B, std::string& err) {
    const rh3t_grid* grid = d.grid;
    const rh3t_params* params = d.params;
    const rh3t_ghost_table* gt = d.ghosts;
    if (!grid || !params || !d.fluid || !gt || grid->nx <= 0 || grid->ny <= 0 || !(grid->dx > 0) ||
        !(grid->dy > 0) || d.n_outer_bc < 0 || d.n_inner_bc < 0 || (d.n_outer_bc && !d.outer_bcs) ||
        (d.n_inner_bc && !d.inner_bcs)) {
        err = "invalid instance description";
        return RH3T_ERR_INVALID_ARGUMENT;
    }
    const long nx = grid->nx, ny = grid->ny;
    const long nxp = nx + 2 * RH3T_PAD;
    const long nyp = ((ny + 2 * RH3T_PAD) + 7) / 8 * 8;
    const long long plane = (long long)nxp * nyp;
    H.grid = *grid;
    H.nx = nx; H.ny = ny; H.nyp = nyp; H.plane = plane;
    H.fluid.assign(d.fluid, d.fluid + (size_t)nx * ny);
    const uint8_t* fluid = H.fluid.data();
    I = Inst{};
    I.nx = (int)nx; I.ny = (int)ny; I.nyp = (int)nyp; I.plane = plane;
    I.dx = grid->dx; I.dy = grid->dy;
    std::memcpy(&I.P, params, sizeof(DevParams));
    I.diffusion = (params->kappa_e != 0.0 || params->kappa_i != 0.0 || params->kappa_r != 0.0) ? 1 : 0;
    I.source = (params->omega_ei != 0.0 || params->omega_er != 0.0) ? 1 : 0;
    H.diffusion = I.diffusion;

    B.mask.assign((size_t)plane, 0);
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j)
            B.mask[(size_t)(i + RH3T_PAD) * nyp + (j + RH3T_PAD)] = fluid[(size_t)i * ny + j] ? 1 : 0;
    // BC table: outer sides then inner sides
    for (int k = 0; k < d.n_outer_bc; ++k) B.bcs.push_back(to_dev(d.outer_bcs[k]));
    for (int k = 0; k < d.n_inner_bc; ++k) B.bcs.push_back(to_dev(d.inner_bcs[k]));
    if (B.bcs.empty()) B.bcs.push_back(DevBC{});

    const int ng = gt->n_ghosts, nh = gt->n_heavy;
    if (ng < 0 || nh < 0 || (ng && (!gt->idx || !gt->boundary || !gt->side || !gt->proj || !gt->pre)) ||
        (nh && (!gt->nearest || !gt->stencil || !gt->s || !gt->w || !gt->d))) {
        err = "incomplete ghost table";
        return RH3T_ERR_INVALID_ARGUMENT;
    }
    auto node = [&](long i, long j) { return (int32_t)((i + RH3T_PAD) * nyp + (j + RH3T_PAD)); };
    H.n_ghosts = ng;
    H.ghost_ij.assign(gt->idx, gt->idx + 2 * (size_t)ng);
    B.recs.resize((size_t)ng);
    B.n_heavy = nh;
    for (int g = 0; g < ng; ++g) {
        long i = gt->idx[2 * g], j = gt->idx[2 * g + 1];
        if (i < -RH3T_PAD || i >= nx + RH3T_PAD || j < -RH3T_PAD || j >= ny + RH3T_PAD) {
            err = "ghost index outside the radius-4 band of the grid";
            return RH3T_ERR_GEOMETRY;
        }
        if (i >= 0 && i < nx && j >= 0 && j < ny && fluid[(size_t)i * ny + j]) {
            err = "ghost index is a fluid node";
            return RH3T_ERR_GEOMETRY;
        }
        int side = gt->side[g];
        int bidx = gt->boundary[g] == 0 ? side : d.n_outer_bc + side;
        if (side < 0 || (gt->boundary[g] == 0 && side >= d.n_outer_bc) ||
            (gt->boundary[g] != 0 && side >= d.n_inner_bc)) {
            err = "ghost side out of range";
            return RH3T_ERR_INVALID_ARGUMENT;
        }
        GhostRec& R = B.recs[g];
        std::memset(&R, 0, sizeof(R));
        R.inst = inst; R.bc = bidx; R.kind = B.bcs[bidx].kind; R.node = node(i, j); R.gid = g;
        R.p0x = gt->proj[5 * g]; R.p0y = gt->proj[5 * g + 1]; R.nx = gt->proj[5 * g + 2];
        R.ny = gt->proj[5 * g + 3]; R.dist = gt->proj[5 * g + 4];
        R.heavy = -1;
        const int kind = R.kind;
        if (kind == BC_WALL || kind == BC_OUTFLOW) ++H.n_wall_outflow;
        if (kind == BC_WALL || kind == BC_OUTFLOW || kind == BC_FAR_FIELD) {
            int k = gt->pre[g];
            if (k < 0 || k >= nh) {
                err = "heavy ghost without GhostBC data";
                return RH3T_ERR_INVALID_ARGUMENT;
            }
            R.heavy = k; // made global at concatenation
            long ni = gt->nearest[2 * k], nj = gt->nearest[2 * k + 1];
            if (ni < 0 || ni >= nx || nj < 0 || nj >= ny) {
                err = "nearest node outside grid";
                return RH3T_ERR_GEOMETRY;
            }
            R.src = node(ni, nj);
        } else if (kind == BC_REFLECTIVE_WALL || kind == BC_ZEROTH_ORDER) {
            long oi = 0, oj = 0;
            if (!mirror_source(*grid, fluid, i, j, R.p0x, R.p0y, oi, oj)) {
                err = "cannot find reflected interior point for ghost";
                return RH3T_ERR_GEOMETRY;
            }
            R.src = node(oi, oj);
        } else if (kind == BC_PERIODIC) {
            // bc1.rs:547-607 (ly a parameter instead of the hardcoded 0.5)
            long np = (long)std::round(params->periodic_ly / grid->dy);
            if (np <= 0) {
                err = "periodic wrap length is zero";
                return RH3T_ERR_PERIODIC_WRAP;
            }
            long jw = ((j % np) + np) % np;
            if (!(i >= 0 && i < nx && jw >= 0 && jw < ny && fluid[(size_t)i * ny + jw])) {
                err = "periodic wrapped point is not fluid";
                return RH3T_ERR_PERIODIC_WRAP;
            }
            R.src = node(i, jw);
        } else {
            R.src = R.node;
        }
    }
    // heavy records: S | w | d | pad | stencil nodes
    B.hrec.assign((size_t)nh * GH_REC, 0.0);
    for (int k = 0; k < nh; ++k) {
        double* r = B.hrec.data() + (size_t)k * GH_REC;
        // S_r transposed per order (the kernel reads column b of all rows a)
        static const int soff[5] = {0, 1, 17, 98, 354};
        const double* S = gt->s + (size_t)k * 979;
        for (int q = 0; q < 5; ++q) {
            const int m = (q + 1) * (q + 1);
            for (int a = 0; a < m; ++a)
                for (int b = 0; b < m; ++b) r[GH_S + soff[q] + b * m + a] = S[soff[q] + a * m + b];
        }
        std::memcpy(r + GH_W, gt->w + (size_t)k * 225, 225 * sizeof(double));
        std::memcpy(r + GH_D, gt->d + (size_t)k * 5, 5 * sizeof(double));
        int32_t st[56] = {0};
        for (int a = 0; a < 55; ++a) {
            uint32_t l = gt->stencil[(size_t)k * 55 + a];
            long i = (long)(l / (uint32_t)ny), j = (long)(l % (uint32_t)ny);
            if (i >= nx || !fluid[l]) {
                err = "E_r stencil node is not fluid";
                return RH3T_ERR_GEOMETRY;
            }
            st[a] = node(i, j);
        }
        std::memcpy(r + GH_ST, st, sizeof(st));
    }
    return RH3T_OK;
}

// decode the device error keys of instances [k0, k1) into c->last (first
// failing instance) and c->inst_status
int fetch_error(rh3t_ctx* c, Span r) {
    const int n = r.k1 - r.k0;
    std::vector<DevError> er((size_t)n);
    CK(c, cudaMemcpyAsync(er.data(), c->d_err + r.k0, (size_t)n * sizeof(DevError), cudaMemcpyDeviceToHost,
                          c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    int first = -1;
    for (int q = 0; q < n; ++q) {
        const int k = r.k0 + q;
        if (er[q].key == ~0ull) {
            c->inst_status[k] = RH3T_OK;
            continue;
        }
        c->inst_status[k] = (int)((er[q].key >> 32) & 31ull);
        if (first < 0) first = q;
    }
    if (first < 0) return RH3T_OK;
    const int k = r.k0 + first;
    const HostInst& H = c->hi[k];
    rh3t_error& L = c->last;
    L = rh3t_error{};
    unsigned long long key = er[first].key;
    int phase = (int)((key >> 37) & 7ull);
    L.code = (int)((key >> 32) & 31ull);
    L.step = (int64_t)(key >> 40);
    L.instance = k;
    unsigned idx = (unsigned)(key & 0xffffffffull);
    L.ghost = -1;
    if (phase == 0) {
        L.stage = 0;
        std::snprintf(L.message, sizeof(L.message), "non-positive dt");
    } else if (phase % 2 == 1) {
        L.stage = (phase + 1) / 2;
        L.ghost = (int)idx;
        if ((int)idx < H.n_ghosts) { L.i = H.ghost_ij[2 * idx]; L.j = H.ghost_ij[2 * idx + 1]; }
        std::snprintf(L.message, sizeof(L.message), "%s",
                      L.code == RH3T_ERR_SINGULAR_ILW ? "singular ILW/extrapolation system at boundary"
                      : L.code == RH3T_ERR_DEVICE_TIMEOUT ? "device wait timed out in the ghost update"
                                                          : "NON-FINITE GHOST STATE");
    } else {
        L.stage = phase / 2;
        L.i = (int)(idx / (unsigned)H.ny);
        L.j = (int)(idx % (unsigned)H.ny);
        std::snprintf(L.message, sizeof(L.message), "non-physical state at (%d, %d) in RK%d state", L.i, L.j,
                      L.stage);
    }
    return L.code;
}

int set_step_params(rh3t_ctx* c, double cfl, double t_final, Span r) {
    launch_set_step(c->stream, c->d_inst, r.k0, r.k1 - r.k0, cfl, t_final);
    c->launches += 1;
    CK(c, cudaGetLastError());
    return RH3T_OK;
}

int check_instance(rh3t_ctx* c, int k) {
    if (k < 0 || k >= c->n_inst) return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "instance index out of range");
    return RH3T_OK;
}

int ensure_graph(rh3t_ctx* c) {
    if (c->graph) return RH3T_OK;
    cudaGraph_t g;
    long long before = c->launches;
    CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c, all(c));
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->launches = before; // captured launches are counted at replay
    CK(c, e);
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    CK(c, e);
    return RH3T_OK;
}

long long range_cells(const rh3t_ctx* c, Span r, long long* max_cells) {
    const HostInst &a = c->hi[r.k0], &b = c->hi[r.k1 - 1];
    long long m = 0;
    for (int k = r.k0; k < r.k1; ++k) m = std::max(m, (long long)c->hi[k].nx * c->hi[k].ny);
    *max_cells = m;
    return b.cell_off + b.nx * b.ny - a.cell_off;
}

int upload_range(rh3t_ctx* c, Span r, const double* values, const double* times) {
    long long maxc = 0;
    const long long cells = range_cells(c, r, &maxc);
    cudaStream_t s = c->stream;
    CK(c, cudaMemcpyAsync(c->d_io + 6 * c->hi[r.k0].cell_off, values, (size_t)cells * 6 * sizeof(double),
                          cudaMemcpyHostToDevice, s));
    CK(c, cudaMemcpyAsync(c->d_times + r.k0, times, (size_t)(r.k1 - r.k0) * sizeof(double), cudaMemcpyHostToDevice,
                          s));
    launch_scatter(s, c->d_inst, r.k0, r.k1 - r.k0, maxc, c->d_io, c->d_times);
    c->launches += 1;
    CK(c, cudaGetLastError());
    CK(c, cudaStreamSynchronize(s));
    return RH3T_OK;
}

int download_range(rh3t_ctx* c, Span r, double* values, double* times) {
    long long maxc = 0;
    const long long cells = range_cells(c, r, &maxc);
    cudaStream_t s = c->stream;
    launch_gather(s, c->d_inst, r.k0, r.k1 - r.k0, maxc, c->d_io);
    c->launches += 1;
    CK(c, cudaGetLastError());
    CK(c, cudaMemcpyAsync(values, c->d_io + 6 * c->hi[r.k0].cell_off, (size_t)cells * 6 * sizeof(double),
                          cudaMemcpyDeviceToHost, s));
    std::vector<DevScalars> sc;
    if (times) {
        sc.resize((size_t)(r.k1 - r.k0));
        CK(c, cudaMemcpyAsync(sc.data(), c->d_sc + r.k0, sc.size() * sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
    }
    CK(c, cudaStreamSynchronize(s));
    for (size_t q = 0; q < sc.size(); ++q) times[q] = sc[q].t_after;
    return RH3T_OK;
}

int l_instance(rh3t_ctx* c, int k, double* rhs, double* ghost_values) {
    cudaStream_t s = c->stream;
    const Span r{k, k + 1};
    const HostInst& H = c->hi[k];
    const long long n = H.nx * H.ny;
    // ghost time of a standalone l(): the field time (Field::time)
    DevScalars* sc = c->d_sc + k;
    CK(c, cudaMemcpyAsync(&sc->t_stage[0], &sc->t_after, sizeof(double), cudaMemcpyDeviceToDevice, s));
    const int ng = enqueue_ghosts(c, s, 0, r);
    const int nf = enqueue_flux(c, s, 0, r);
    double* planes = c->d_io2 + 6 * H.cell_off;
    CK(c, cudaMemsetAsync(planes, 0, (size_t)n * 6 * sizeof(double), s));
    enqueue_rhs(c, s, 0, 0, c->d_io2, r);
    c->launches += ng + nf + 1;
    if (rhs) {
        double* aos = c->d_io + 6 * H.cell_off;
        launch_planes_to_aos(s, planes, n, aos);
        c->launches += 1;
        CK(c, cudaMemcpyAsync(rhs, aos, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (ghost_values && H.n_ghosts) {
        double* gv = c->d_io2 + 6 * c->total_cells;
        launch_ghost_values(s, c->d_inst, c->d_ghosts + H.ghost_off, H.n_ghosts, gv);
        c->launches += 1;
        CK(c, cudaMemcpyAsync(ghost_values, gv, (size_t)H.n_ghosts * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CK(c, cudaGetLastError());
    return fetch_error(c, r);
}

} // namespace

extern "C" void rh3t_default_params(rh3t_params* p) {
    *p = rh3t_params{1.4, 1.4, 1.4, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.5, 10.0, 1e-12, 0.5};
}

// the failure of the last rh3t_batch_create / rh3t_create on this thread (the
// context it would have returned no longer exists to carry it)
static thread_local int g_create_code = 0;
static thread_local char g_create_msg[192] = {0};

static void set_create_error(int code, const char* m) {
    g_create_code = code;
    std::snprintf(g_create_msg, sizeof(g_create_msg), "%s", m ? m : "");
}

extern "C" int rh3t_create_error(char* message, int32_t len) {
    if (message && len > 0) std::snprintf(message, (size_t)len, "%s", g_create_msg);
    return g_create_code;
}

extern "C" int rh3t_batch_create(int32_t n, const rh3t_instance* desc, int32_t device, rh3t_ctx** out) {
    set_create_error(0, "");
    if (!out) return RH3T_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (n <= 0 || !desc) return RH3T_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < n; ++k) { // argument checks come before any device call
        const rh3t_instance& d = desc[k];
        if (!d.grid || !d.params || !d.fluid || !d.ghosts || d.grid->nx <= 0 || d.grid->ny <= 0 ||
            d.n_outer_bc < 0 || d.n_inner_bc < 0 || (d.n_outer_bc && !d.outer_bcs) || (d.n_inner_bc && !d.inner_bcs)) {
            char m[96];
            std::snprintf(m, sizeof(m), "instance %d: missing or malformed description", k);
            set_create_error(RH3T_ERR_INVALID_ARGUMENT, m);
            return RH3T_ERR_INVALID_ARGUMENT;
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || ndev <= device) {
        set_create_error(RH3T_ERR_NO_DEVICE, "no such CUDA device");
        return RH3T_ERR_NO_DEVICE;
    }
    rh3t_ctx* c = new rh3t_ctx();
    c->device = device;
    auto fail = [&](int code, const char* m) {
        set_error(c, code, m);
        set_create_error(code, m);
        std::fprintf(stderr, "rh3t_batch_create: %s\n", m);
        rh3t_destroy(c);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(RH3T_ERR_CUDA, "cudaSetDevice failed");
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(RH3T_ERR_CUDA, "stream create failed");

    c->n_inst = n;
    c->h.resize((size_t)n);
    c->hi.resize((size_t)n);
    c->inst_status.assign((size_t)n, 0);
    std::vector<Built> B((size_t)n);
    for (int k = 0; k < n; ++k) {
        std::string err;
        int rc = build_instance(desc[k], k, c->hi[k], c->h[k], B[k], err);
        if (rc) {
            char m[160];
            std::snprintf(m, sizeof(m), "instance %d: %.120s", k, err.c_str());
            return fail(rc, m);
        }
    }
    // ---- offsets of every instance in the concatenated arrays
    long long n_state = 0, n_mask = 0, n_faces = 0;
    size_t n_bcs = 0;
    std::vector<long long> off_state(n), off_mask(n), off_faces(n);
    std::vector<size_t> off_bcs(n);
    int heavy_base = 0, ghost_base = 0;
    for (int k = 0; k < n; ++k) {
        HostInst& H = c->hi[k];
        Inst& I = c->h[k];
        const long long nfx = (long long)(H.nx + 1) * H.ny, nfy = (long long)H.nx * (H.ny + 1);
        off_state[k] = n_state; n_state += 3 * 6 * H.plane;
        off_mask[k] = n_mask; n_mask += (H.plane + 15) / 16 * 16;
        off_faces[k] = n_faces; n_faces += 6 * (nfx + nfy) + (I.diffusion ? 3 * (nfx + nfy) : 0);
        off_bcs[k] = n_bcs; n_bcs += B[k].bcs.size();
        H.cell_off = c->total_cells;
        I.cell_off = H.cell_off;
        I.aoff = c->total_planes;
        c->total_planes += 6 * H.plane;
        c->max_faces = std::max(c->max_faces, std::max((long long)(H.nx + 1) * H.ny, (long long)H.nx * (H.ny + 1)));
        c->total_cells += H.nx * H.ny;
        c->max_cells = std::max(c->max_cells, (long long)H.nx * H.ny);
        H.ghost_off = ghost_base;
        for (GhostRec& R : B[k].recs)
            if (R.heavy >= 0) R.heavy += heavy_base;
        heavy_base += B[k].n_heavy;
        ghost_base += H.n_ghosts;
        c->max_ghosts = std::max(c->max_ghosts, H.n_ghosts);
    }
    c->n_ghosts = ghost_base;
    c->n_heavy = heavy_base;
    // ghost partition: heavy records by heavy slot, then the cheap ones; both
    // instance-major, so every instance range maps to two contiguous segments
    std::vector<GhostRec> recs, part;
    recs.reserve((size_t)c->n_ghosts);
    part.reserve((size_t)c->n_ghosts);
    for (int k = 0; k < n; ++k) recs.insert(recs.end(), B[k].recs.begin(), B[k].recs.end());
    for (int k = 0; k < n; ++k) {
        HostInst& H = c->hi[k];
        H.gh0 = (int)part.size();
        std::vector<GhostRec> hv;
        for (const GhostRec& R : B[k].recs)
            if (R.heavy >= 0) hv.push_back(R);
        std::stable_sort(hv.begin(), hv.end(), [](const GhostRec& a, const GhostRec& b) { return a.heavy < b.heavy; });
        part.insert(part.end(), hv.begin(), hv.end());
        H.ngh = (int)hv.size();
    }
    c->n_gheavy = (int)part.size();
    for (int k = 0; k < n; ++k) {
        HostInst& H = c->hi[k];
        H.gc0 = (int)part.size() - c->n_gheavy;
        for (const GhostRec& R : B[k].recs)
            if (R.heavy < 0) part.push_back(R);
        H.ngc = (int)part.size() - c->n_gheavy - H.gc0;
    }
    c->n_gcheap = (int)part.size() - c->n_gheavy;

    // ---- device allocations
    cudaError_t e = cudaSuccess;
#define DA(ptr, cnt) do { e = dalloc(&(ptr), (size_t)(cnt)); if (e != cudaSuccess) return fail(RH3T_ERR_CUDA, "cudaMalloc failed: " #ptr); } while (0)
    DA(c->d_state, n_state);
    DA(c->d_mask, n_mask);
    DA(c->d_faces, std::max(n_faces, 1LL));
    DA(c->d_bcs, n_bcs);
    DA(c->d_sc, n);
    DA(c->d_err, n);
    DA(c->d_times, n);
    DA(c->d_inst, n);
    DA(c->d_ghosts, std::max(c->n_ghosts, 1));
    DA(c->d_gpart, std::max(c->n_ghosts, 1));
    DA(c->d_hrec, std::max((long long)c->n_heavy * GH_REC, 1LL));
    DA(c->d_io, c->total_cells * 6);
    DA(c->d_io2, (c->total_cells + c->max_ghosts) * 6); // rhs planes, then ghost values
#undef DA
    for (int k = 0; k < n; ++k) {
        Inst& I = c->h[k];
        const HostInst& H = c->hi[k];
        const long long nfx = (long long)(H.nx + 1) * H.ny, nfy = (long long)H.nx * (H.ny + 1);
        I.U = c->d_state + off_state[k];
        I.A = I.U + 6 * H.plane;
        I.B = I.U + 12 * H.plane;
        I.mask = c->d_mask + off_mask[k];
        I.fx = c->d_faces + off_faces[k];
        I.fy = I.fx + 6 * nfx;
        I.dfx = I.diffusion ? I.fx + 6 * (nfx + nfy) : nullptr;
        I.dfy = I.diffusion ? I.dfx + 3 * nfx : nullptr;
        I.bcs = c->d_bcs + off_bcs[k];
        I.sc = c->d_sc + k;
        I.err = c->d_err + k;
    }

    DevScalars sc{};
    {
        // orderable key of +inf (see kernels.cu dkey)
        double inf = INFINITY;
        unsigned long long b;
        std::memcpy(&b, &inf, 8);
        sc.dt_cfl_bits = b | 0x8000000000000000ull;
    }
    sc.cfl_factor = 0.05;
    sc.t_final = INFINITY;
    std::vector<DevScalars> scs((size_t)n, sc);
    std::vector<DevError> ers((size_t)n, DevError{~0ull});
    cudaStream_t s = c->stream;
#define CP(dst, src, bytes) do { e = cudaMemcpyAsync((dst), (src), (size_t)(bytes), cudaMemcpyHostToDevice, s); if (e != cudaSuccess) return fail(RH3T_ERR_CUDA, "upload failed"); } while (0)
    if (cudaMemsetAsync(c->d_state, 0, (size_t)n_state * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(c->d_faces, 0, (size_t)std::max(n_faces, 1LL) * sizeof(double), s) != cudaSuccess)
        return fail(RH3T_ERR_CUDA, "memset failed");
    for (int k = 0; k < n; ++k) {
        CP(c->d_mask + off_mask[k], B[k].mask.data(), B[k].mask.size());
        CP(c->d_bcs + off_bcs[k], B[k].bcs.data(), B[k].bcs.size() * sizeof(DevBC));
    }
    CP(c->d_sc, scs.data(), scs.size() * sizeof(DevScalars));
    CP(c->d_err, ers.data(), ers.size() * sizeof(DevError));
    if (c->n_ghosts) {
        CP(c->d_ghosts, recs.data(), recs.size() * sizeof(GhostRec));
        CP(c->d_gpart, part.data(), part.size() * sizeof(GhostRec));
    }
    {
        size_t off = 0;
        for (int k = 0; k < n; ++k) {
            if (!B[k].hrec.empty()) CP(c->d_hrec + off, B[k].hrec.data(), B[k].hrec.size() * sizeof(double));
            off += B[k].hrec.size();
        }
    }
#undef CP
    // the host arrays above must outlive the copies
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail(RH3T_ERR_CUDA, "set-up synchronize failed");
    int rc = make_tiles(c); // also uploads the Inst records
    if (rc) return fail(rc, "tile upload failed");
    *out = c;
    return RH3T_OK;
}

extern "C" int rh3t_create(const rh3t_grid* grid, const rh3t_params* params, const uint8_t* fluid,
                           int32_t n_outer_bc, const rh3t_bc* outer_bcs, int32_t n_inner_bc,
                           const rh3t_bc* inner_bcs, const rh3t_ghost_table* gt, int32_t device, rh3t_ctx** out) {
    rh3t_instance d{grid, params, fluid, n_outer_bc, outer_bcs, n_inner_bc, inner_bcs, gt};
    return rh3t_batch_create(1, &d, device, out);
}

extern "C" void rh3t_destroy(rh3t_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    io_free(c);
    adj_free(c);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (cudaStream_t x : c->xfer)
        if (x) cudaStreamDestroy(x);
    if (c->h_sc) cudaFreeHost(c->h_sc);
    dfree(c->d_state); dfree(c->d_mask); dfree(c->d_faces); dfree(c->d_bcs); dfree(c->d_sc); dfree(c->d_err);
    dfree(c->d_times); dfree(c->d_inst); dfree(c->d_ghosts); dfree(c->d_gpart); dfree(c->d_hrec);
    dfree(c->d_tx); dfree(c->d_ty); dfree(c->d_tc); dfree(c->d_tr); dfree(c->d_io); dfree(c->d_io2);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int32_t rh3t_instance_count(const rh3t_ctx* c) { return c ? c->n_inst : 0; }

extern "C" int rh3t_upload_instance(rh3t_ctx* c, int32_t k, const double* value, double time) {
    if (!c || !value) return RH3T_ERR_INVALID_ARGUMENT;
    if (int rc = check_instance(c, k)) return rc;
    CK(c, cudaSetDevice(c->device));
    return upload_range(c, Span{k, k + 1}, value, &time);
}

extern "C" int rh3t_download_instance(rh3t_ctx* c, int32_t k, double* value, double* time) {
    if (!c || !value) return RH3T_ERR_INVALID_ARGUMENT;
    if (int rc = check_instance(c, k)) return rc;
    CK(c, cudaSetDevice(c->device));
    return download_range(c, Span{k, k + 1}, value, time);
}

extern "C" int rh3t_upload_state(rh3t_ctx* c, const double* value, double time) {
    return rh3t_upload_instance(c, 0, value, time);
}

extern "C" int rh3t_download_state(rh3t_ctx* c, double* value, double* time) {
    return rh3t_download_instance(c, 0, value, time);
}

extern "C" int rh3t_upload_batch(rh3t_ctx* c, const double* values, const double* times) {
    if (!c || !values || !times) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    return upload_range(c, all(c), values, times);
}

extern "C" int rh3t_download_batch(rh3t_ctx* c, double* values, double* times) {
    if (!c || !values) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    return download_range(c, all(c), values, times);
}

extern "C" int rh3t_l_instance(rh3t_ctx* c, int32_t k, double* rhs, double* ghost_values) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    if (int rc = check_instance(c, k)) return rc;
    CK(c, cudaSetDevice(c->device));
    return l_instance(c, k, rhs, ghost_values);
}

extern "C" int rh3t_l(rh3t_ctx* c, double* rhs, double* ghost_values) {
    return rh3t_l_instance(c, 0, rhs, ghost_values);
}

extern "C" int rh3t_calc_global_dt(rh3t_ctx* c, double* dt_cfl) {
    if (!c || !dt_cfl) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    enqueue_dt(c, c->stream, 0, Span{0, 1});
    c->launches += 1;
    CK(c, cudaGetLastError());
    CK(c, cudaMemcpyAsync(dt_cfl, (char*)c->d_sc + offsetof(DevScalars, dt_cfl), sizeof(double),
                          cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return RH3T_OK;
}

extern "C" int rh3t_calc_global_dt_batch(rh3t_ctx* c, double* dt_cfl) {
    if (!c || !dt_cfl) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    enqueue_dt(c, c->stream, 0, all(c));
    c->launches += 1;
    CK(c, cudaGetLastError());
    std::vector<DevScalars> sc((size_t)c->n_inst);
    CK(c, cudaMemcpyAsync(sc.data(), c->d_sc, sc.size() * sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < c->n_inst; ++k) dt_cfl[k] = sc[k].dt_cfl;
    return RH3T_OK;
}

extern "C" int rh3t_rk3_ssp(rh3t_ctx* c, double dt) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    launch_set_dt(c->stream, c->d_inst, c->n_inst, dt);
    c->launches += 1;
    for (int st = 0; st < 3; ++st) enqueue_stage(c, st, all(c));
    CK(c, cudaGetLastError());
    return fetch_error(c, all(c));
}

extern "C" int rh3t_advance(rh3t_ctx* c, int32_t nsteps, double cfl_factor, double t_final, int32_t use_graph) {
    if (!c || nsteps < 0) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    int rc = set_step_params(c, cfl_factor, t_final, all(c));
    if (rc) return rc;
    if (use_graph) {
        rc = ensure_graph(c);
        if (rc) return rc;
        for (int n = 0; n < nsteps; ++n) CK(c, cudaGraphLaunch(c->graph, c->stream));
        c->launches += (long long)nsteps * launches_per_step(c);
    } else {
        for (int n = 0; n < nsteps; ++n) enqueue_step(c, all(c));
    }
    CK(c, cudaGetLastError());
    return fetch_error(c, all(c));
}

extern "C" int rh3t_step_host(rh3t_ctx* c, double* value, double* time, double cfl_factor, double* dt_out) {
    if (!c || !value || !time) return RH3T_ERR_INVALID_ARGUMENT;
    if (c->n_inst != 1)
        return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "rh3t_step_host needs a one-instance context");
    CK(c, cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const long long n = c->total_cells;
    int rc = set_step_params(c, cfl_factor, INFINITY, all(c));
    if (rc) return rc;
    rc = ensure_graph(c);
    if (rc) return rc;
    CK(c, cudaMemcpyAsync(c->d_io, value, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(c, cudaMemcpyAsync(c->d_times, time, sizeof(double), cudaMemcpyHostToDevice, s));
    launch_scatter(s, c->d_inst, 0, 1, n, c->d_io, c->d_times);
    CK(c, cudaGraphLaunch(c->graph, s));
    launch_gather(s, c->d_inst, 0, 1, n, c->d_io);
    c->launches += 2 + launches_per_step(c);
    CK(c, cudaMemcpyAsync(value, c->d_io, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(c, cudaMemcpyAsync(time, (char*)c->d_sc + offsetof(DevScalars, t_after), sizeof(double),
                          cudaMemcpyDeviceToHost, s));
    if (dt_out)
        CK(c, cudaMemcpyAsync(dt_out, (char*)c->d_sc + offsetof(DevScalars, dt), sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    CK(c, cudaGetLastError());
    return fetch_error(c, all(c));
}

// Host value arrays in, one step, host value arrays out, with the copies of
// one group of instances overlapping the step of another: instance groups of
// about equal cell counts go host -> device on one copy stream, take their
// step on the context's stream (eager launches over the group's instance
// range) and return on a second copy stream.
extern "C" int rh3t_step_host_batch(rh3t_ctx* c, double* values, double* times, double cfl_factor,
                                    int32_t n_groups) {
    if (!c || !values || !times) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    for (cudaStream_t& x : c->xfer)
        if (!x) CK(c, cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    if (!c->h_sc) CK(c, cudaMallocHost((void**)&c->h_sc, (size_t)c->n_inst * sizeof(DevScalars)));
    const int groups = std::max(1, std::min(n_groups > 0 ? n_groups : 8, c->n_inst));
    std::vector<Span> gr;
    {
        const long long total = c->total_cells;
        int k0 = 0;
        for (int g = 0; g < groups && k0 < c->n_inst; ++g) {
            const long long target = total * (g + 1) / groups;
            int k1 = k0 + 1;
            while (k1 < c->n_inst && c->hi[k1].cell_off + c->hi[k1].nx * c->hi[k1].ny <= target) ++k1;
            if (g == groups - 1) k1 = c->n_inst;
            gr.push_back(Span{k0, k1});
            k0 = k1;
        }
        if (k0 < c->n_inst) gr.back().k1 = c->n_inst;
    }
    const int G = (int)gr.size();
    cudaStream_t sc = c->stream, su = c->xfer[0], sd = c->xfer[1];
    int rc = set_step_params(c, cfl_factor, INFINITY, all(c));
    if (rc) return rc;
    std::vector<cudaEvent_t> ev((size_t)(2 * G + 2), nullptr);
    auto release = [&]() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    };
    for (cudaEvent_t& e : ev) {
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            release();
            return set_error(c, RH3T_ERR_CUDA, "event create failed");
        }
    }
    auto ck = [&](cudaError_t e, const char* where) {
        if (e == cudaSuccess) return 0;
        release();
        return cuda_check(c, e, where);
    };
#define CKE(call) do { if (int _rc = ck((call), #call)) return _rc; } while (0)
    CKE(cudaEventRecord(ev[0], sc)); // the step parameters are set
    CKE(cudaStreamWaitEvent(su, ev[0], 0));
    CKE(cudaMemcpyAsync(c->d_times, times, (size_t)c->n_inst * sizeof(double), cudaMemcpyHostToDevice, su));
    for (int g = 0; g < G; ++g) {
        long long maxc = 0;
        const long long cells = range_cells(c, gr[g], &maxc);
        const long long o = 6 * c->hi[gr[g].k0].cell_off;
        CKE(cudaMemcpyAsync(c->d_io + o, values + o, (size_t)cells * 6 * sizeof(double), cudaMemcpyHostToDevice, su));
        launch_scatter(su, c->d_inst, gr[g].k0, gr[g].k1 - gr[g].k0, maxc, c->d_io, c->d_times);
        CKE(cudaEventRecord(ev[1 + g], su));
    }
    for (int g = 0; g < G; ++g) {
        long long maxc = 0;
        const long long cells = range_cells(c, gr[g], &maxc);
        const long long o = 6 * c->hi[gr[g].k0].cell_off;
        CKE(cudaStreamWaitEvent(sc, ev[1 + g], 0));
        enqueue_step(c, gr[g]);
        CKE(cudaEventRecord(ev[1 + G + g], sc));
        CKE(cudaStreamWaitEvent(sd, ev[1 + G + g], 0));
        launch_gather(sd, c->d_inst, gr[g].k0, gr[g].k1 - gr[g].k0, maxc, c->d_io);
        CKE(cudaMemcpyAsync(values + o, c->d_io + o, (size_t)cells * 6 * sizeof(double), cudaMemcpyDeviceToHost, sd));
        CKE(cudaMemcpyAsync(c->h_sc + gr[g].k0, c->d_sc + gr[g].k0, (size_t)(gr[g].k1 - gr[g].k0) * sizeof(DevScalars),
                            cudaMemcpyDeviceToHost, sd));
    }
    CKE(cudaEventRecord(ev[1 + 2 * G], sd));
    CKE(cudaStreamWaitEvent(sc, ev[1 + 2 * G], 0));
    c->launches += 2 * G;
    CKE(cudaGetLastError());
#undef CKE
    rc = fetch_error(c, all(c)); // synchronises the context's stream, and so both copy streams
    release();
    for (int k = 0; k < c->n_inst; ++k) times[k] = c->h_sc[k].t_after;
    return rc;
}

extern "C" int rh3t_profile_steps(rh3t_ctx* c, int32_t nsteps, double cfl_factor, double* ms_out,
                                  int64_t* launches_out) {
    if (!c || !ms_out || nsteps < 0) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    int rc = set_step_params(c, cfl_factor, INFINITY, all(c));
    if (rc) return rc;
    cudaStream_t s = c->stream;
    std::vector<cudaEvent_t> ev;
    std::vector<int> cls, kn; // class and kernel count of the interval ending at each event
    auto mark = [&](int k, int n_kernels) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        ev.push_back(e);
        cls.push_back(k);
        kn.push_back(n_kernels);
    };
    const Span r = all(c);
    for (int n = 0; n < nsteps; ++n) {
        mark(-1, 0);
        enqueue_dt(c, s, 1, r);
        mark(3, 1);
        for (int st = 0; st < 3; ++st) {
            const int ng = enqueue_ghosts(c, s, st, r);
            mark(0, ng);
            const int nf = enqueue_flux(c, s, st, r);
            mark(1, nf);
            enqueue_rhs(c, s, st, 1, nullptr, r);
            mark(2, 1);
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
        cnt[cls[k]] += kn[k];
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 4; ++k) ms_out[k] = acc[k];
    if (launches_out)
        for (int k = 0; k < 4; ++k) launches_out[k] = cnt[k];
    return fetch_error(c, r);
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

extern "C" int rh3t_instance_times(rh3t_ctx* c, double* t, double* dt, int64_t* steps) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    std::vector<DevScalars> sc((size_t)c->n_inst);
    CK(c, cudaMemcpyAsync(sc.data(), c->d_sc, sc.size() * sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < c->n_inst; ++k) {
        if (t) t[k] = sc[k].t_after;
        if (dt) dt[k] = sc[k].dt;
        if (steps) steps[k] = sc[k].steps_started;
    }
    return RH3T_OK;
}

extern "C" int rh3t_instance_status(const rh3t_ctx* c, int32_t* codes) {
    if (!c || !codes) return RH3T_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < c->n_inst; ++k) codes[k] = c->inst_status[k];
    return RH3T_OK;
}

extern "C" int rh3t_synchronize(rh3t_ctx* c) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaStreamSynchronize(c->stream));
    return fetch_error(c, all(c));
}

extern "C" int rh3t_last_error(const rh3t_ctx* c, rh3t_error* out) {
    if (!c || !out) return RH3T_ERR_INVALID_ARGUMENT;
    *out = c->last;
    return c->last.code;
}

extern "C" int64_t rh3t_kernel_launches(const rh3t_ctx* c) { return c ? c->launches : 0; }
extern "C" void* rh3t_stream(const rh3t_ctx* c) { return c ? (void*)c->stream : nullptr; }
