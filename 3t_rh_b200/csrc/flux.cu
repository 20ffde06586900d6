// Interface fluxes (main.rs:165-246: weno.rs:685-802 reconstruction_fast per
// x and y face, plus diffusion.rs:27-50 when diffusion is on).
//
// Work split: six lanes per face, lane c owning characteristic field c
// (5 faces per warp, lanes 30-31 only help staging). Lane c forms row c of L,
// projects the six stencil points, runs the two WENO5 reconstructions of f+
// and f- and obtains g_c; the six g are exchanged by warp shuffles and lane c
// returns component c of R.g with the reference's summation order
// (weno.rs:793, 834-843).
//
// Staging: a block covers 40 faces. The stencil points of the tile (x: 10x8,
// y: 45) are loaded once into shared memory together with their physical flux
// and the Roe inputs, instead of once per face (six times per point).
//
// RH3T_EXACT selects the reference's expressions; otherwise the fastm forms
// (shared reciprocals, one division per WENO5) are used.
#include "common.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace rh3t {

#ifdef RH3T_EXACT
constexpr bool kExact = true;
#else
constexpr bool kExact = false;
#endif

__device__ __forceinline__ double weno5_any(double a, double b, double c, double d, double e, double eps) {
    if (kExact) return weno5(a, b, c, d, e, eps);
    return fastm::weno5(a, b, c, d, e, eps);
}

template <int DIR>
__device__ __forceinline__ void flux_tile(const Inst& I, const Tile& t, int stage, double (*sU)[FLUX_NPT],
                                          double (*sF)[FLUX_NPT], double (*sR)[FLUX_NPT], double (*sT)[FLUX_NPT]) {
    const DevParams& P = I.P;
    const double* __restrict__ buf = stage_src(I, stage);
    const long long plane = I.plane;
    const int nx = I.nx, ny = I.ny;
    const int np = DIR == 0 ? (FX_TI + 5) * FX_TJ : FY_TJ + 5;
    const bool diff = I.diffusion != 0;
    // ---- stage the tile's stencil points
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        int pi, pj;
        if (DIR == 0) { pi = t.i - 3 + p / FX_TJ; pj = t.j0 + p % FX_TJ; }
        else { pi = t.i; pj = t.j0 - 3 + p; }
        double s[6] = {1.0, 0.0, 0.0, 1.0, 1.0, 1.0};
        if (pi >= -RH3T_PAD && pi < nx + RH3T_PAD && pj >= -RH3T_PAD && pj < ny + RH3T_PAD)
            load6(buf, plane, node_of(I, pi, pj), s);
        Prim d = kExact ? prim_from_state(s, P) : fastm::prim(s, P);
        double f[6];
        phys_flux<DIR>(s, d, f);
#pragma unroll
        for (int k = 0; k < 6; ++k) { sU[k][p] = s[k]; sF[k][p] = f[k]; }
        sR[0][p] = sqrt(s[0]); sR[1][p] = d.u; sR[2][p] = d.v;
        sR[3][p] = d.e_e; sR[4][p] = d.e_i; sR[5][p] = d.e_r;
        if (diff) {
            double te, ti, tr;
            temps_from_state(s, P, te, ti, tr);
            sT[0][p] = te; sT[1][p] = ti; sT[2][p] = tr;
        }
    }
    __syncthreads();
    // ---- one face per 6 lanes
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int fw = lane < 30 ? lane / 6 : 4;
    const int c = lane - 6 * fw;
    const int f = warp * 5 + fw;
    int i, j, p0, ps;
    if (DIR == 0) { i = t.i + f / FX_TJ; j = t.j0 + f % FX_TJ; p0 = (f / FX_TJ) * FX_TJ + f % FX_TJ; ps = FX_TJ; }
    else { i = t.i; j = t.j0 + f; p0 = f; ps = 1; }
    bool active = lane < 30 && f < FLUX_FACES;
    if (DIR == 0) active = active && i <= nx && j < ny;
    else active = active && j <= ny;
    if (active) {
        const uint8_t m0 = I.mask[node_of(I, i, j)];
        const uint8_t m1 = DIR == 0 ? I.mask[node_of(I, i - 1, j)] : I.mask[node_of(I, i, j - 1)];
        active = (m0 | m1) != 0;
    }
    double g = 0.0, Rr[6] = {0, 0, 0, 0, 0, 0};
    if (active) {
        const int p2 = p0 + 2 * ps, p3 = p0 + 3 * ps;
        Roe q;
        double a6[6], b6[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) { a6[k] = sR[k][p3]; b6[k] = sR[k][p2]; }
        if (kExact) {
            Prim d3, d2;
            d3.u = a6[1]; d3.v = a6[2]; d3.e_e = a6[3]; d3.e_i = a6[4]; d3.e_r = a6[5];
            d2.u = b6[1]; d2.v = b6[2]; d2.e_e = b6[3]; d2.e_i = b6[4]; d2.e_r = b6[5];
            q = roe_average(sU[0][p3], d3, sU[0][p2], d2, P);
        } else {
            q = fastm::roe(a6, b6, P);
        }
        double Lc[6], lam;
        if (kExact) l_row<DIR>(c, q, P, Lc);
        else fastm::l_row<DIR>(c, q, P, Lc);
        r_row<DIR>(c, q, P, Rr, lam);
        const double a = fabs(lam);
        double fp[6], fm[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int p = p0 + k * ps;
            double cf = Lc[0] * sF[0][p] + Lc[1] * sF[1][p] + Lc[2] * sF[2][p] + Lc[3] * sF[3][p] +
                        Lc[4] * sF[4][p] + Lc[5] * sF[5][p];
            double cs = Lc[0] * sU[0][p] + Lc[1] * sU[1][p] + Lc[2] * sU[2][p] + Lc[3] * sU[3][p] +
                        Lc[4] * sU[4][p] + Lc[5] * sU[5][p];
            fp[k] = 0.5 * (cf + a * cs);
            fm[k] = 0.5 * (cf - a * cs);
        }
        g = weno5_any(fp[0], fp[1], fp[2], fp[3], fp[4], P.eps) + weno5_any(fm[5], fm[4], fm[3], fm[2], fm[1], P.eps);
    }
    // ---- exchange g among the six lanes of the face; lane c returns (R g)_c
    const int base = 6 * fw;
    double gall[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) gall[k] = __shfl_sync(0xffffffffu, g, base + k);
    if (!active) return;
    double out = Rr[0] * gall[0] + Rr[1] * gall[1] + Rr[2] * gall[2] + Rr[3] * gall[3] + Rr[4] * gall[4] +
                 Rr[5] * gall[5];
    long long fplane, fidx;
    double *fo, *dfo;
    if (DIR == 0) { fplane = (long long)(nx + 1) * ny; fidx = (long long)i * ny + j; fo = I.fx; dfo = I.dfx; }
    else { fplane = (long long)nx * (ny + 1); fidx = (long long)i * (ny + 1) + j; fo = I.fy; dfo = I.dfy; }
    fo[c * fplane + fidx] = out;
    if (diff && c >= 3) {
        // diffusion.rs:27-50: lane 3 -> ee (Te), 4 -> ei (Ti), 5 -> er (Tr^4)
        const int k = c - 3;
        double v[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            double x = sT[k][p0 + m * ps];
            v[m] = k == 2 ? pow4d(x) : x;
        }
        const double kap = k == 0 ? P.kappa_e : (k == 1 ? P.kappa_i : P.kappa_r);
        double term = kap * (2.0 * v[5] - 25.0 * v[4] + 245.0 * v[3] - 245.0 * v[2] + 25.0 * v[1] - 2.0 * v[0]);
        dfo[k * fplane + fidx] = term / 180.0;
    }
}

__global__ void __launch_bounds__(256) k_flux(const Inst* __restrict__ insts, const Tile* __restrict__ tx, int ntx,
                                              const Tile* __restrict__ ty, int nty, int stage) {
    __shared__ double sU[6][FLUX_NPT], sF[6][FLUX_NPT], sR[6][FLUX_NPT], sT[3][FLUX_NPT];
    const int b = blockIdx.x;
    if (b < ntx) {
        const Tile t = tx[b];
        const Inst& I = insts[t.inst];
        if (has_error(I)) return;
        flux_tile<0>(I, t, stage, sU, sF, sR, sT);
    } else if (b < ntx + nty) {
        const Tile t = ty[b - ntx];
        const Inst& I = insts[t.inst];
        if (has_error(I)) return;
        flux_tile<1>(I, t, stage, sU, sF, sR, sT);
    }
}

void launch_flux(cudaStream_t s, const Inst* insts, const Tile* tx, int ntx, const Tile* ty, int nty, int stage) {
    if (ntx + nty <= 0) return;
    k_flux<<<ntx + nty, 256, 0, s>>>(insts, tx, ntx, ty, nty, stage);
}

} // namespace rh3t
