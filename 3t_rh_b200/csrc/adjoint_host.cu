// Host side of the adjoint (include/rh3t.h rh3t_l_vjp, rh3t_adjoint_forward,
// rh3t_adjoint_backward): checkpointed reverse sweep of the SSP-RK3 time
// loop over every instance of a context.
//
// Forward: the state of every instance is saved every `ckpt_every` steps.
// Backward, segment by segment from the last: the segment is recomputed from
// its checkpoint with every stage state (ghost nodes included), every stage
// rhs and every step's scalars kept; then its steps are reversed:
//   Y = cotangent of u3;
//   stage 2: U0 = Y/3, U2 = 2Y/3 + vjp_l(u2)^T (2dt/3 Y);
//   stage 1: U0 += 3 U2/4, U1 = U2/4 + vjp_l(u1)^T (dt/4 U2);
//   stage 0: U0 += U1 + vjp_l(u0)^T (dt U1);
//   dt = cfl dt_cfl(u0): U0 += cfl dtbar d(local dt)/du at the minimising cell,
//   with dtbar = <r2, 2Y/3> + <r1, U2/4> + <r0, U1>;
// and U0 is the next Y. Memory: (n_steps / ckpt_every) states plus
// n_rec x ckpt_every x (3 stage states + 3 rhs) plane sets. The forward run
// records its last n_rec segments as it goes, so the reverse sweep starts
// with n_rec segments it does not recompute: n_rec is as many records as fit
// in a quarter of the device memory free at allocation (at least one, at most
// the number of segments).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"
#include "kernels.cuh"

using namespace rh3t;

struct AdjBuffers {
    int ckpt_every = 0, nsteps = 0, n_ckpt = 0;
    bool last_recorded = false; // seg holds the forward run's last segment
    double cfl = 0.05;
    double* ckpt = nullptr;     // n_ckpt plane sets (state U at segment starts)
    DevScalars* ckpt_sc = nullptr; // n_ckpt x n_inst scalars at segment starts
    int n_rec = 0;              // segment records allocated
    int max_rec = 0;            // cap on n_rec (0: the memory budget alone)
    double* seg = nullptr;      // n_rec x ckpt_every x 6 plane sets: U0 U1 U2 R0 R1 R2 per step
    DevScalars* seg_sc = nullptr; // n_rec x ckpt_every x n_inst scalars (after the step's dt)
    double *Y = nullptr, *U0 = nullptr, *U1 = nullptr, *U2 = nullptr, *W = nullptr, *rbar = nullptr;
    double* pbar = nullptr;     // n_inst x 8
    double* dtbar = nullptr;    // n_inst
    unsigned long long* argmin = nullptr; // n_inst: the dt-minimising cell
    double* gslots = nullptr;   // AG_SLOT doubles per heavy ghost (ghost vjp scratch)
    double* final_state = nullptr; // the forward run's end state, restored after the sweep
};

namespace rh3t {
void adj_free(rh3t_ctx* c) {
    AdjBuffers* a = c->adj;
    if (!a) return;
    void* ptrs[] = {a->ckpt, a->ckpt_sc, a->seg,   a->seg_sc, a->Y,      a->U0,     a->U1,
                    a->U2,   a->W,       a->rbar,  a->pbar,   a->dtbar, a->argmin, a->gslots, a->final_state};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete a;
    c->adj = nullptr;
}
} // namespace rh3t

namespace {

Span all_of(const rh3t_ctx* c) { return Span{0, c->n_inst}; }

long long max_plane(const rh3t_ctx* c) {
    long long m = 0;
    for (const HostInst& H : c->hi) m = std::max(m, H.plane);
    return m;
}

// the work buffers every vjp needs (Y, U0, U1, U2, W, rbar, pbar, dtbar)
int ensure_work(rh3t_ctx* c) {
    if (!c->adj) c->adj = new AdjBuffers();
    AdjBuffers* a = c->adj;
    if (a->Y) return RH3T_OK;
    const size_t np = (size_t)c->total_planes;
    double** bufs[] = {&a->Y, &a->U0, &a->U1, &a->U2, &a->W, &a->rbar};
    for (double** b : bufs) {
        CK(c, cudaMalloc(b, np * sizeof(double)));
        CK(c, cudaMemsetAsync(*b, 0, np * sizeof(double), c->stream));
    }
    CK(c, cudaMalloc(&a->pbar, (size_t)c->n_inst * 8 * sizeof(double)));
    CK(c, cudaMalloc(&a->dtbar, (size_t)c->n_inst * sizeof(double)));
    CK(c, cudaMalloc(&a->argmin, (size_t)c->n_inst * sizeof(unsigned long long)));
    CK(c, cudaMalloc(&a->gslots, (size_t)std::max(c->n_gheavy, 1) * AG_SLOT * sizeof(double)));
    CK(c, cudaMalloc(&a->final_state, np * sizeof(double)));
    return RH3T_OK;
}

void ghost_ranges(const rh3t_ctx* c, int& nh, int& nc) {
    const HostInst &a = c->hi[0], &b = c->hi[c->n_inst - 1];
    nh = b.gh0 + b.ngh - a.gh0;
    nc = b.gc0 + b.ngc - a.gc0;
}

// Ub += vjp_l(X)^T rbar for every instance (W zeroed first)
void enqueue_vjp_l(rh3t_ctx* c, const double* X, const double* rbar, double* Ub) {
    AdjBuffers* a = c->adj;
    cudaMemsetAsync(a->W, 0, (size_t)c->total_planes * sizeof(double), c->stream);
    int nh, nc;
    ghost_ranges(c, nh, nc);
    int wo = 0;
    for (const HostInst& H : c->hi) wo |= H.n_wall_outflow > 0;
    launch_adj_l(c->stream, c->d_inst, 0, c->n_inst, c->max_cells, c->d_tx, c->ntx, c->d_ty, c->nty, c->d_tr, c->ntr,
                 c->d_gpart, nh, c->d_gpart + c->n_gheavy, nc, c->d_hrec, X, rbar, a->W, Ub, a->pbar, a->gslots, wo);
    c->launches += adj_l_launches(nh, nc, wo);
}

// forward stage with the adjoint's record (stage state with ghosts, rhs)
void enqueue_recorded_step(rh3t_ctx* c, double* rec) {
    cudaStream_t s = c->stream;
    const long long np = c->total_planes;
    const Span r = all_of(c);
    const HostInst &h0 = c->hi[0], &h1 = c->hi[c->n_inst - 1];
    const long long mp = max_plane(c);
    launch_dt(s, c->d_inst, c->d_tc + h0.tc0, h1.tc0 + h1.ntc - h0.tc0, 1);
    int nh, nc;
    ghost_ranges(c, nh, nc);
    for (int st = 0; st < 3; ++st) {
        launch_ghosts(s, c->d_inst, c->d_gpart, nh, c->d_gpart + c->n_gheavy, nc, c->d_hrec, st);
        launch_adj_copy(s, c->d_inst, 0, c->n_inst, mp, st, rec + st * np, 0);
        const int nf = enqueue_flux(c, s, st, r);
        enqueue_rhs(c, s, st, 2, rec + (3 + st) * np, r);
        c->launches += ghost_launches(nh, nc) + nf + 2;
    }
    c->launches += 1;
}

int fetch_status(rh3t_ctx* c) { return rh3t_synchronize(c); }

} // namespace

extern "C" int rh3t_l_vjp(rh3t_ctx* c, int32_t k, const double* rbar, double* ubar, double* pbar8) {
    if (!c || !rbar || !ubar) return RH3T_ERR_INVALID_ARGUMENT;
    if (k < 0 || k >= c->n_inst) return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "instance index out of range");
    CK(c, cudaSetDevice(c->device));
    if (int rc = ensure_work(c)) return rc;
    AdjBuffers* a = c->adj;
    cudaStream_t s = c->stream;
    const HostInst& H = c->hi[k];
    const long long n = H.nx * H.ny;
    const size_t np = (size_t)c->total_planes;
    // ghost nodes of the resident state at the field time (stage 0 buffer)
    DevScalars* sc = c->d_sc + k;
    CK(c, cudaMemcpyAsync(&sc->t_stage[0], &sc->t_after, sizeof(double), cudaMemcpyDeviceToDevice, s));
    int nh, nc;
    ghost_ranges(c, nh, nc);
    launch_ghosts(s, c->d_inst, c->d_gpart, nh, c->d_gpart + c->n_gheavy, nc, c->d_hrec, 0);
    launch_adj_copy(s, c->d_inst, 0, c->n_inst, max_plane(c), 0, a->U2, 0); // X = U2 as scratch
    CK(c, cudaMemsetAsync(a->rbar, 0, np * sizeof(double), s));
    CK(c, cudaMemsetAsync(a->U0, 0, np * sizeof(double), s));
    CK(c, cudaMemsetAsync(a->pbar, 0, (size_t)c->n_inst * 8 * sizeof(double), s));
    CK(c, cudaMemcpyAsync(c->d_io + 6 * H.cell_off, rbar, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_adj_aos(s, c->d_inst, k, 1, n, c->d_io, a->rbar, 0);
    enqueue_vjp_l(c, a->U2, a->rbar, a->U0);
    launch_adj_aos(s, c->d_inst, k, 1, n, c->d_io, a->U0, 1);
    c->launches += ghost_launches(nh, nc) + 3;
    CK(c, cudaMemcpyAsync(ubar, c->d_io + 6 * H.cell_off, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (pbar8) CK(c, cudaMemcpyAsync(pbar8, a->pbar + 8 * k, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(c, cudaGetLastError());
    return fetch_status(c);
}

extern "C" int32_t rh3t_adjoint_records(const rh3t_ctx* c) { return c && c->adj ? c->adj->n_rec : 0; }

extern "C" int rh3t_adjoint_max_records(rh3t_ctx* c, int32_t n) {
    if (!c || n < 0) return RH3T_ERR_INVALID_ARGUMENT;
    if (!c->adj) c->adj = new AdjBuffers();
    c->adj->max_rec = n;
    c->adj->n_ckpt = 0; // the next rh3t_adjoint_forward allocates again
    c->adj->last_recorded = false;
    return RH3T_OK;
}

extern "C" int rh3t_adjoint_forward(rh3t_ctx* c, int32_t nsteps, double cfl_factor, int32_t ckpt_every) {
    if (!c || nsteps <= 0 || ckpt_every <= 0) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    if (int rc = ensure_work(c)) return rc;
    AdjBuffers* a = c->adj;
    cudaStream_t s = c->stream;
    const size_t np = (size_t)c->total_planes, ni = (size_t)c->n_inst;
    const int n_ckpt = (nsteps + ckpt_every - 1) / ckpt_every;
    if (a->n_ckpt < n_ckpt || a->ckpt_every < ckpt_every) {
        if (a->ckpt) cudaFree(a->ckpt);
        if (a->ckpt_sc) cudaFree(a->ckpt_sc);
        if (a->seg) cudaFree(a->seg);
        if (a->seg_sc) cudaFree(a->seg_sc);
        a->ckpt = nullptr; a->ckpt_sc = nullptr; a->seg = nullptr; a->seg_sc = nullptr;
        CK(c, cudaMalloc(&a->ckpt, (size_t)n_ckpt * np * sizeof(double)));
        CK(c, cudaMalloc(&a->ckpt_sc, (size_t)n_ckpt * ni * sizeof(DevScalars)));
        // as many segment records as fit in a quarter of the free memory
        const size_t rec_bytes = (size_t)ckpt_every * 6 * np * sizeof(double);
        size_t free_b = 0, total_b = 0;
        CK(c, cudaMemGetInfo(&free_b, &total_b));
        int n_rec = (int)std::min<size_t>((size_t)n_ckpt, std::max<size_t>(1, free_b / 4 / rec_bytes));
        if (a->max_rec > 0) n_rec = std::min(n_rec, a->max_rec);
        while (n_rec > 1 && cudaMalloc(&a->seg, (size_t)n_rec * rec_bytes) != cudaSuccess) {
            cudaGetLastError(); // an out-of-memory here only means fewer records
            --n_rec;
        }
        if (n_rec == 1) CK(c, cudaMalloc(&a->seg, rec_bytes));
        a->n_rec = n_rec;
        CK(c, cudaMalloc(&a->seg_sc, (size_t)n_rec * ckpt_every * ni * sizeof(DevScalars)));
    }
    a->last_recorded = false;
    const int n_rec = std::min(a->n_rec, n_ckpt);
    a->n_ckpt = n_ckpt;
    a->ckpt_every = ckpt_every;
    a->nsteps = nsteps;
    a->cfl = cfl_factor;
    // cfl_factor and t_final (none) of every instance
    int rc = rh3t_advance(c, 0, cfl_factor, INFINITY, 0);
    if (rc) return rc;
    const long long mp = max_plane(c);
    int done = 0;
    for (int q = 0; q < n_ckpt; ++q) {
        launch_adj_copy(s, c->d_inst, 0, c->n_inst, mp, 0, a->ckpt + (size_t)q * np, 0);
        CK(c, cudaMemcpyAsync(a->ckpt_sc + (size_t)q * ni, c->d_sc, ni * sizeof(DevScalars), cudaMemcpyDeviceToDevice,
                              s));
        c->launches += 1;
        const int len = std::min(ckpt_every, nsteps - done);
        if (q < n_ckpt - n_rec) {
            rc = rh3t_advance(c, len, cfl_factor, INFINITY, 1);
            if (rc) return rc;
        } else {
            // one of the last n_rec segments, with its record (stage states, rhs, scalars)
            const size_t r = (size_t)(q - (n_ckpt - n_rec)) * ckpt_every;
            for (int j = 0; j < len; ++j) {
                enqueue_recorded_step(c, a->seg + (r + j) * 6 * np);
                CK(c, cudaMemcpyAsync(a->seg_sc + (r + j) * ni, c->d_sc, ni * sizeof(DevScalars),
                                      cudaMemcpyDeviceToDevice, s));
            }
            CK(c, cudaGetLastError());
            rc = fetch_status(c);
            if (rc) return rc;
        }
        done += len;
    }
    a->last_recorded = true;
    return RH3T_OK;
}

extern "C" int rh3t_adjoint_backward(rh3t_ctx* c, const double* dJ_du, double* dJ_du0, double* dJ_dparams) {
    if (!c || !dJ_du || !dJ_du0) return RH3T_ERR_INVALID_ARGUMENT;
    AdjBuffers* a = c->adj;
    if (!a || a->nsteps <= 0) return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "rh3t_adjoint_forward must run first");
    CK(c, cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const size_t np = (size_t)c->total_planes, ni = (size_t)c->n_inst;
    const long long mp = max_plane(c);
    // Y = dJ/du of the final state
    CK(c, cudaMemcpyAsync(c->d_io, dJ_du, (size_t)c->total_cells * 6 * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_adj_aos(s, c->d_inst, 0, c->n_inst, c->max_cells, c->d_io, a->Y, 0);
    CK(c, cudaMemsetAsync(a->pbar, 0, ni * 8 * sizeof(double), s));
    c->launches += 1;
    // the state at the end of the forward run, restored after the sweep
    std::vector<DevScalars> end_sc(ni);
    CK(c, cudaMemcpyAsync(end_sc.data(), c->d_sc, ni * sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
    CK(c, cudaStreamSynchronize(s));
    double* final_state = a->final_state;
    launch_adj_copy(s, c->d_inst, 0, c->n_inst, mp, 0, final_state, 0);
    const int n_rec = std::min(a->n_rec, a->n_ckpt);
    const bool recorded = a->last_recorded;
    a->last_recorded = false;
    for (int q = a->n_ckpt - 1; q >= 0; --q) {
        const int len = std::min(a->ckpt_every, a->nsteps - q * a->ckpt_every);
        // the last n_rec segments were recorded by the forward run; the others
        // are recomputed into the first record
        const bool have = recorded && q >= a->n_ckpt - n_rec;
        const size_t r0 = have ? (size_t)(q - (a->n_ckpt - n_rec)) * a->ckpt_every : 0;
        if (!have) {
            launch_adj_copy(s, c->d_inst, 0, c->n_inst, mp, 0, a->ckpt + (size_t)q * np, 1);
            CK(c, cudaMemcpyAsync(c->d_sc, a->ckpt_sc + (size_t)q * ni, ni * sizeof(DevScalars),
                                  cudaMemcpyDeviceToDevice, s));
            c->launches += 1;
        }
        for (int j = 0; j < len && !have; ++j) {
            double* rec = a->seg + (size_t)j * 6 * np;
            // the step's scalars are those after its dt: record them after the step
            enqueue_recorded_step(c, rec);
            CK(c, cudaMemcpyAsync(a->seg_sc + (size_t)j * ni, c->d_sc, ni * sizeof(DevScalars),
                                  cudaMemcpyDeviceToDevice, s));
        }
        for (int j = len - 1; j >= 0; --j) {
            double* rec = a->seg + (r0 + j) * 6 * np;
            const DevScalars* sc = a->seg_sc + (r0 + j) * ni;
            CK(c, cudaMemsetAsync(a->dtbar, 0, ni * sizeof(double), s));
            launch_adj_stage(s, c->d_inst, 0, c->n_inst, c->max_cells, 2, a->Y, a->U0, a->U2, a->rbar,
                             rec + 5 * np, sc, a->dtbar);
            enqueue_vjp_l(c, rec + 2 * np, a->rbar, a->U2);
            launch_adj_stage(s, c->d_inst, 0, c->n_inst, c->max_cells, 1, a->U2, a->U0, a->U1, a->rbar,
                             rec + 4 * np, sc, a->dtbar);
            enqueue_vjp_l(c, rec + 1 * np, a->rbar, a->U1);
            launch_adj_stage(s, c->d_inst, 0, c->n_inst, c->max_cells, 0, a->U1, a->U0, nullptr, a->rbar,
                             rec + 3 * np, sc, a->dtbar);
            enqueue_vjp_l(c, rec, a->rbar, a->U0);
            launch_adj_dt(s, c->d_inst, 0, c->n_inst, c->max_cells, rec, sc, a->dtbar, a->argmin, a->U0, a->pbar);
            c->launches += 5;
            std::swap(a->Y, a->U0);
        }
        CK(c, cudaGetLastError());
    }
    // dJ/du0 and the parameter cotangents
    launch_adj_aos(s, c->d_inst, 0, c->n_inst, c->max_cells, c->d_io, a->Y, 1);
    c->launches += 1;
    CK(c, cudaMemcpyAsync(dJ_du0, c->d_io, (size_t)c->total_cells * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (dJ_dparams)
        CK(c, cudaMemcpyAsync(dJ_dparams, a->pbar, ni * 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
    // restore the end state of the forward run
    launch_adj_copy(s, c->d_inst, 0, c->n_inst, mp, 0, final_state, 1);
    CK(c, cudaMemcpyAsync(c->d_sc, end_sc.data(), ni * sizeof(DevScalars), cudaMemcpyHostToDevice, s));
    c->launches += 1;
    CK(c, cudaStreamSynchronize(s));
    CK(c, cudaGetLastError());
    return fetch_status(c);
}
