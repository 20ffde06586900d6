// Work-tile shapes and their autotuner (include/rh3t.h rh3t_set_tile_shapes,
// rh3t_autotune). A shape is per instance and travels in every Tile record,
// so one launch mixes instances tuned to different shapes; the arithmetic of
// a face or a cell does not depend on the shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "context.h"
#include "kernels.cuh"

using namespace rh3t;

namespace {

struct ClassKey {
    int nx, ny, diffusion;
    bool operator<(const ClassKey& o) const {
        return std::tie(nx, ny, diffusion) < std::tie(o.nx, o.ny, o.diffusion);
    }
};

std::mutex g_mu;
std::map<ClassKey, Shape> g_cache; // process-wide tuning results

bool shape_ok(int lgx, int lgy, int lgr) {
    return lgx >= FX_LG_MIN && lgx <= FX_LG_MAX && lgy >= FY_LG_MIN && lgy <= FY_LG_MAX && lgr >= RHS_LG_MIN &&
           lgr <= RHS_LG_MAX;
}

// cache file: one "nx ny diffusion lg_fx lg_fy lg_rhs" line per class
void load_cache(const char* path) {
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    int nx, ny, df, a, b, r;
    while (std::fscanf(f, "%d %d %d %d %d %d", &nx, &ny, &df, &a, &b, &r) == 6)
        if (shape_ok(a, b, r)) g_cache[ClassKey{nx, ny, df}] = Shape{a, b, r};
    std::fclose(f);
}

bool save_cache(const char* path) {
    std::string tmp = std::string(path) + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return false;
    for (const auto& kv : g_cache)
        std::fprintf(f, "%d %d %d %d %d %d\n", kv.first.nx, kv.first.ny, kv.first.diffusion, kv.second.lgx,
                     kv.second.lgy, kv.second.lgr);
    bool ok = std::fclose(f) == 0;
    return ok && std::rename(tmp.c_str(), path) == 0;
}

enum Kind { KX = 0, KY = 1, KR = 2 };

// minimum over `reps` launches of one tile kind over the class's tiles (ms)
int time_kind(rh3t_ctx* c, Kind kind, const std::vector<Tile>& tiles, int reps, double* ms_out) {
    *ms_out = 0.0;
    if (tiles.empty()) return RH3T_OK;
    cudaStream_t s = c->stream;
    Tile* d = nullptr;
    CK(c, cudaMalloc(&d, tiles.size() * sizeof(Tile)));
    cudaError_t e = cudaMemcpyAsync(d, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, s);
    cudaEvent_t a = nullptr, b = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const int n = (int)tiles.size();
    auto launch = [&]() {
        if (kind == KX) launch_flux(s, c->d_inst, d, n, nullptr, 0, 0);
        else if (kind == KY) launch_flux(s, c->d_inst, nullptr, 0, d, n, 0);
        else launch_rhs_stage(s, c->d_inst, d, n, 0, 0, c->d_io2);
        c->launches += 1;
    };
    double best = 1e30;
    if (e == cudaSuccess) {
        launch(); // warm-up
        for (int r = 0; r < reps && e == cudaSuccess; ++r) {
            cudaEventRecord(a, s);
            launch();
            cudaEventRecord(b, s);
            e = cudaEventSynchronize(b);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
            best = std::min(best, (double)ms);
        }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaStreamSynchronize(s);
    cudaFree(d);
    CK(c, e);
    *ms_out = best;
    return RH3T_OK;
}

} // namespace

extern "C" int rh3t_set_tile_shapes(rh3t_ctx* c, int32_t k, int32_t lg_fx, int32_t lg_fy, int32_t lg_rhs) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    if (k < -1 || k >= c->n_inst || !shape_ok(lg_fx, lg_fy, lg_rhs))
        return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "tile shape or instance out of range");
    CK(c, cudaSetDevice(c->device));
    for (int q = 0; q < c->n_inst; ++q)
        if (k < 0 || q == k) c->hi[q].shape = Shape{lg_fx, lg_fy, lg_rhs};
    return make_tiles(c);
}

extern "C" int rh3t_get_tile_shapes(const rh3t_ctx* c, int32_t k, int32_t* lg3) {
    if (!c || !lg3 || k < 0 || k >= c->n_inst) return RH3T_ERR_INVALID_ARGUMENT;
    const Shape& s = c->hi[k].shape;
    lg3[0] = s.lgx;
    lg3[1] = s.lgy;
    lg3[2] = s.lgr;
    return RH3T_OK;
}

extern "C" int rh3t_autotune(rh3t_ctx* c, const char* cache_path, int32_t reps, rh3t_tune_entry* out,
                             int32_t max_out, int32_t* n_out) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    reps = std::max(1, std::min(reps, 100));
    std::lock_guard<std::mutex> lock(g_mu);
    if (cache_path) load_cache(cache_path);
    std::map<ClassKey, std::vector<int>> classes;
    for (int k = 0; k < c->n_inst; ++k)
        classes[ClassKey{(int)c->hi[k].nx, (int)c->hi[k].ny, c->hi[k].diffusion}].push_back(k);
    std::vector<rh3t_tune_entry> entries;
    for (const auto& kv : classes) {
        rh3t_tune_entry E{};
        E.nx = kv.first.nx;
        E.ny = kv.first.ny;
        E.diffusion = kv.first.diffusion;
        E.n_instances = (int)kv.second.size();
        Shape best;
        auto hit = g_cache.find(kv.first);
        if (hit != g_cache.end()) {
            best = hit->second;
            E.from_cache = 1;
        } else {
            const int lo[3] = {FX_LG_MIN, FY_LG_MIN, RHS_LG_MIN}, hi[3] = {FX_LG_MAX, FY_LG_MAX, RHS_LG_MAX};
            double* ms[3] = {E.ms_fx, E.ms_fy, E.ms_rhs};
            int pick[3] = {FX_LG_DEF, FY_LG_DEF, RHS_LG_DEF};
            for (int kind = 0; kind < 3; ++kind) {
                double tbest = 1e30;
                for (int lg = lo[kind]; lg <= hi[kind]; ++lg) {
                    Shape sh;
                    sh.lgx = kind == KX ? lg : FX_LG_DEF;
                    sh.lgy = kind == KY ? lg : FY_LG_DEF;
                    sh.lgr = kind == KR ? lg : RHS_LG_DEF;
                    std::vector<Tile> tiles;
                    for (int k : kv.second)
                        instance_tiles(c->hi[k], sh, k, kind == KX ? &tiles : nullptr,
                                       kind == KY ? &tiles : nullptr, kind == KR ? &tiles : nullptr);
                    double t = 0.0;
                    int rc = time_kind(c, (Kind)kind, tiles, reps, &t);
                    if (rc) return rc;
                    ms[kind][lg - lo[kind]] = t;
                    if (t < tbest) { tbest = t; pick[kind] = lg; }
                }
            }
            best = Shape{pick[0], pick[1], pick[2]};
            g_cache[kv.first] = best;
        }
        E.lg_fx = best.lgx;
        E.lg_fy = best.lgy;
        E.lg_rhs = best.lgr;
        for (int k : kv.second) c->hi[k].shape = best;
        entries.push_back(E);
    }
    int rc = make_tiles(c);
    if (rc) return rc;
    if (cache_path && !save_cache(cache_path))
        return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "cannot write the tuning cache file");
    if (out)
        for (int q = 0; q < (int)entries.size() && q < max_out; ++q) out[q] = entries[q];
    if (n_out) *n_out = (int)entries.size();
    return RH3T_OK;
}
