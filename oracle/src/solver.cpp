// ORACLE — test infrastructure only (see physics.hpp).
// Restatement of the per-stage runtime of the reference: bc1.rs
// set_ghost_point_value (all BC kinds), ghost.rs update_values_parallel,
// main.rs l() / stage updates / rk3_ssp / calc_global_dt, the initial
// conditions of init.rs, and a C API used by the Python tests and bench.
// OpenMP loops stand where the reference has Rayon par_iter loops.
#include "model.hpp"
#include "jvp.hpp"
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <omp.h>

namespace oracle {

static bool state_finite(const State& s) {
    for (int k = 0; k < 6; ++k) if (!std::isfinite(s[k])) return false;
    return true;
}

// bc1.rs:467-469 solve6 — LAPACK dgesv (getrf + getrs) semantics: LU with
// partial pivoting (first maximal |a_ij|), reciprocal-scaled column,
// rank-1 trailing update, then unit-lower and upper triangular solves.
static bool solve6(double A[6][6], double b[6]) {
    int piv[6];
    for (int j = 0; j < 6; ++j) {
        int p = j;
        double mx = std::fabs(A[j][j]);
        for (int i = j + 1; i < 6; ++i)
            if (std::fabs(A[i][j]) > mx) { mx = std::fabs(A[i][j]); p = i; }
        piv[j] = p;
        if (A[p][j] == 0.0) return false;
        if (p != j) for (int k = 0; k < 6; ++k) std::swap(A[j][k], A[p][k]);
        double rcp = 1.0 / A[j][j];
        for (int i = j + 1; i < 6; ++i) A[i][j] *= rcp;
        for (int k = j + 1; k < 6; ++k)
            for (int i = j + 1; i < 6; ++i) A[i][k] -= A[i][j] * A[j][k];
    }
    for (int j = 0; j < 6; ++j) if (piv[j] != j) std::swap(b[j], b[piv[j]]);
    for (int k = 0; k < 6; ++k)
        for (int i = k + 1; i < 6; ++i) b[i] -= b[k] * A[i][k];
    for (int k = 5; k >= 0; --k) {
        b[k] /= A[k][k];
        for (int i = 0; i < k; ++i) b[i] -= b[k] * A[i][k];
    }
    return true;
}

// bc1.rs:424-440
static void local_pressure_and_a2(double rho, double u, double v, double ee, double ei, double er, const Params& P,
                                  double& p, double& a2) {
    double w2 = u * u + v * v;
    double ee1 = ee / rho - w2 / 6.0, ei1 = ei / rho - w2 / 6.0, er1 = er / rho - w2 / 6.0;
    double ge = P.gamma_e - 1.0, gi = P.gamma_i - 1.0, gr = P.gamma_r - 1.0;
    p = rho * (ge * ee1 + gi * ei1 + gr * er1);
    a2 = P.gamma_e * ge * ee1 + P.gamma_i * gi * ei1 + P.gamma_r * gr * er1;
}

// bc1.rs:448-465
static void build_ilw_row1(const double u0[6], const Params& P, double row[6]) {
    double u1 = u0[0], u3 = u0[2];
    double gi = P.gamma_i - 1.0, ge = P.gamma_e - 1.0, gr = P.gamma_r - 1.0;
    double gt = gi + ge + gr;
    row[0] = -gt * sq(u3) / (6.0 * sq(u1));
    row[1] = 0.0;
    row[2] = gt * u3 / (6.0 * u1);
    row[3] = -ge; row[4] = -gi; row[5] = -gr;
}

// bc1.rs:294-312 build_local_plain: L, R, lambda at the nearest fluid node,
// state rotated to the (normal, tangential) frame, X-direction matrices.
void build_local_plain(Vec2 n, const State& val, const Params& P, double L[6][6], double R[6][6], double lam[6]) {
    double mom_n = val.mx * n.x + val.my * n.y;
    double mom_t = -val.mx * n.y + val.my * n.x;
    State s1{val.rho, mom_n, mom_t, val.ee, val.ei, val.er};
    Derived d1 = derived_from_state(s1, P);
    build_l_plain(s1, s1, d1, d1, DIR_X, P, L);
    build_r_plain(s1, s1, d1, d1, DIR_X, P, lam, R);
}

// bc1.rs:193-255 weno_extrapolation_pre, evaluated for all k = 0..4 at once.
// The reference recomputes data, beta and alpha for every k (the loop at
// bc1.rs:673-675); they do not depend on k, so one pass gives the same values.
static void weno_extrapolation_all(const double L[6][6], const GhostBC& bc, const State* val, const Params& P,
                                   double v[5][6]) {
    Vec2 n = bc.normal;
    double alpha[6][5], vks[5][6][5], asum[6] = {0, 0, 0, 0, 0, 0};
    for (int r = 0; r <= 4; ++r) {
        int m = (r + 1) * (r + 1);
        double data[6][25];
        for (int a = 0; a < m; ++a) {
            const State& s = val[bc.stencil[BC_STENCIL_OFF[r] + a]];
            double mn = s.mx * n.x + s.my * n.y;
            double mt = -s.mx * n.y + s.my * n.x;
            double u6[6] = {s.rho, mn, mt, s.ee, s.ei, s.er};
            for (int c = 0; c < 6; ++c) {
                const double* row = L[c];
                data[c][a] = row[0] * u6[0] + row[1] * u6[1] + row[2] * u6[2] + row[3] * u6[3] + row[4] * u6[4] +
                             row[5] * u6[5];
            }
        }
        for (int c = 0; c < 6; ++c) {
            int soff = BC_S_OFF[r];
            double beta = 0.0;
            for (int a = 0; a < m; ++a) {
                int base = soff + a * m;
                double acc = 0.0;
                for (int b = 0; b < m; ++b) acc += bc.s[base + b] * data[c][b];
                beta += data[c][a] * acc;
            }
            for (int k = 0; k < 5; ++k) {
                double vk = 0.0;
                if (k <= r) {
                    int woff = BC_W_OFF[r] + k * m;
                    for (int a = 0; a < m; ++a) vk += bc.w[woff + a] * data[c][a];
                }
                vks[k][c][r] = vk;
            }
            alpha[c][r] = bc.d[r] / powf_ref(P.eps + beta, P.weno_q);
            asum[c] += alpha[c][r];
        }
    }
    for (int k = 0; k < 5; ++k)
        for (int c = 0; c < 6; ++c) {
            double res = 0.0;
            for (int r = 0; r <= 4; ++r) res += (alpha[c][r] / asum[c]) * vks[k][c][r];
            v[k][c] = res;
        }
}

static void mat_vec(const double M[6][6], const double x[6], double out[6]) {
    for (int i = 0; i < 6; ++i) {
        double acc = 0.0;
        for (int j = 0; j < 6; ++j) acc += M[i][j] * x[j];
        out[i] = acc;
    }
}

// bc1.rs:733-755 (same in 806-827 and 894-923): Taylor expansion to the
// ghost point and rotation back to the global frame.
static State taylor_rotate(double u[5][6], double d, Vec2 n) {
    double g[6];
    for (int c = 0; c < 6; ++c) g[c] = u[0][c];
    double coef = 1.0;
    for (int k = 1; k <= 4; ++k) {
        coef *= d / (double)k;
        for (int c = 0; c < 6; ++c) g[c] = g[c] + coef * u[k][c];
    }
    double mom_n = g[1], mom_t = g[2];
    return {g[0], mom_n * n.x - mom_t * n.y, mom_n * n.y + mom_t * n.x, g[3], g[4], g[5]};
}

// bc1.rs:930-1037 / 471-545: nearest fluid node to the mirror point 2 P0 - Pg
static bool mirror_source(long gi, long gj, const Projection& pr, const Field& f, long& oi, long& oj) {
    Point pg{f.grid.x(gi), f.grid.y(gj)};
    Point pi{2.0 * pr.point.x - pg.x, 2.0 * pr.point.y - pg.y};
    long ic, jc;
    f.grid.coord2idx(pi, ic, jc);
    const long cand[9][2] = {{ic, jc}, {ic - 1, jc}, {ic + 1, jc}, {ic, jc - 1}, {ic, jc + 1},
                             {ic - 1, jc - 1}, {ic - 1, jc + 1}, {ic + 1, jc - 1}, {ic + 1, jc + 1}};
    bool found = false;
    double best = INFINITY;
    for (int k = 0; k < 9; ++k) {
        if (!f.is_in_domain(cand[k][0], cand[k][1])) continue;
        double d2 = sq(f.grid.x(cand[k][0]) - pi.x) + sq(f.grid.y(cand[k][1]) - pi.y);
        if (d2 < best) { best = d2; oi = cand[k][0]; oj = cand[k][1]; found = true; }
    }
    return found;
}

// bc1.rs:609-928 set_ghost_point_value (precomputed fast path)
static State set_ghost_point_value(const GhostInfo& g, const Field& f, const State* val, double t,
                                   const GhostGrid& gg, const Params& P) {
    const BC& bc = (g.boundary == OUTER ? f.bc_outer : f.bc_inner)[g.side_id];
    const Projection& pr = g.project;
    switch (bc.kind) {
    case BC_CONSTANT: return bc.state;
    case BC_TIME_DEPENDENT: {
        double xs = bc.td_x0 + bc.td_speed * t;
        return pr.point.x <= xs ? bc.td_left : bc.td_right;
    }
    case BC_REFLECTIVE_WALL: {
        long oi, oj;
        if (!mirror_source(g.i, g.j, pr, f, oi, oj))
            throw OracleError(ERR_GEOMETRY, "cannot find reflected interior point for ghost", g.i, g.j);
        const State& s = val[f.linear_index(oi, oj)];
        Vec2 n = pr.normal;
        double mom_n = s.mx * n.x + s.my * n.y;
        return {s.rho, s.mx - 2.0 * mom_n * n.x, s.my - 2.0 * mom_n * n.y, s.ee, s.ei, s.er};
    }
    case BC_ZEROTH_ORDER: {
        long oi, oj;
        if (!mirror_source(g.i, g.j, pr, f, oi, oj))
            throw OracleError(ERR_GEOMETRY, "cannot find interior point for zeroth-order ghost", g.i, g.j);
        return val[f.linear_index(oi, oj)];
    }
    case BC_PERIODIC: {
        long np = (long)std::round(P.periodic_ly / f.grid.dy);
        long jw = ((g.j % np) + np) % np;
        if (!f.is_in_domain(g.i, jw)) throw OracleError(ERR_PERIODIC, "periodic wrapped point is not fluid", g.i, jw);
        return val[f.linear_index(g.i, jw)];
    }
    default: break;
    }
    const GhostBC& pre = gg.pre[g.pre];
    double L[6][6], R[6][6], lam[6];
    build_local_plain(pr.normal, val[f.linear_index(pre.nearest_i, pre.nearest_j)], P, L, R, lam);
    double v[5][6];
    weno_extrapolation_all(L, pre, val, P, v);
    return ghost_from_extrapolation(bc, pr, L, R, lam, v, P, g.i, g.j);
}

// bc1.rs:676-928: the Wall / Outflow / FarField rows from the extrapolated
// characteristic derivatives v[k] (k = 0..4) and L, R, lambda at the nearest
// node, then the Taylor sum to the ghost point (shared by the precomputed
// path above and the per-call path of slowpath.cpp, as in the reference).
// bc1.rs:691-702 the first ILW system of a Wall ghost: L with its first row
// replaced by the no-penetration row, right-hand side v^(0) with a zero first
// entry
static void wall_system0(const double L[6][6], const double v[5][6], double A0[6][6], double rhs0[6]) {
    std::memcpy(A0, L, 36 * sizeof(double));
    for (int c = 0; c < 6; ++c) A0[0][c] = c == 1 ? 1.0 : 0.0;
    for (int c = 0; c < 6; ++c) rhs0[c] = v[0][c];
    rhs0[0] = 0.0;
}
// bc1.rs:703-740 the second: L with the ILW momentum row at u^(0) first
static void wall_system1(const double L[6][6], const double v[5][6], const double u0[6], const Params& P,
                         double A1[6][6], double rhs1[6]) {
    double row1[6];
    std::memcpy(A1, L, 36 * sizeof(double));
    build_ilw_row1(u0, P, row1);
    for (int c = 0; c < 6; ++c) A1[0][c] = row1[c];
    for (int c = 0; c < 6; ++c) rhs1[c] = v[1][c];
    rhs1[0] = 0.0;
}

State ghost_from_extrapolation(const BC& bc, const Projection& pr, const double L[6][6], const double R[6][6],
                               const double lam[6], const double v[5][6], const Params& P, long gi, long gj) {
    double u[5][6];
    if (bc.kind == BC_WALL) {
        // bc1.rs:691-756
        double A0[6][6], rhs0[6];
        wall_system0(L, v, A0, rhs0);
        if (!solve6(A0, rhs0)) throw OracleError(ERR_SINGULAR, "singular ILW/extrapolation system at boundary", gi, gj);
        for (int c = 0; c < 6; ++c) u[0][c] = rhs0[c];
        double A1[6][6], rhs1[6];
        wall_system1(L, v, u[0], P, A1, rhs1);
        if (!solve6(A1, rhs1)) throw OracleError(ERR_SINGULAR, "singular ILW/extrapolation system at boundary", gi, gj);
        for (int c = 0; c < 6; ++c) u[1][c] = rhs1[c];
        for (int k = 2; k <= 4; ++k) mat_vec(R, v[k], u[k]);
    } else if (bc.kind == BC_OUTFLOW) {
        // bc1.rs:760-828
        mat_vec(R, v[0], u[0]);
        double rho0 = u[0][0];
        double un0 = u[0][1] / rho0, ut0 = u[0][2] / rho0;
        double p0, a2;
        local_pressure_and_a2(rho0, un0, ut0, u[0][3], u[0][4], u[0][5], P, p0, a2);
        double a = std::sqrt(a2);
        double lambda1 = un0 - a;
        double rhs1[6];
        for (int c = 0; c < 6; ++c) rhs1[c] = v[1][c];
        if (lambda1 < 0.0) {
            double m_local = std::fabs(un0 / a);
            double l1 = bc.sigma * (1.0 - sq(m_local)) * a / bc.l_domain * (p0 - bc.p_inf);
            rhs1[0] = l1 / lambda1;
        }
        mat_vec(R, rhs1, u[1]);
        for (int k = 2; k <= 4; ++k) mat_vec(R, v[k], u[k]);
    } else if (bc.kind == BC_FAR_FIELD) {
        // bc1.rs:829-924
        Vec2 n = pr.normal;
        const State& ui = bc.state;
        double uinf[6] = {ui.rho, ui.mx * n.x + ui.my * n.y, -ui.mx * n.y + ui.my * n.x, ui.ee, ui.ei, ui.er};
        double vinf[6];
        mat_vec(L, uinf, vinf);
        double rhs0[6];
        for (int c = 0; c < 6; ++c) rhs0[c] = lam[c] < 0.0 ? vinf[c] : v[0][c];
        mat_vec(R, rhs0, u[0]);
        for (int k = 1; k <= 4; ++k) {
            double rk[6];
            for (int c = 0; c < 6; ++c) rk[c] = lam[c] < 0.0 ? 0.0 : v[k][c];
            mat_vec(R, rk, u[k]);
        }
    } else {
        return State{0, 0, 0, 0, 0, 0};
    }
    return taylor_rotate(u, pr.distance, pr.normal);
}

// ---------------------------------------------------------------- main.rs
struct Solver {
    Field f;
    GhostGrid gg;
    Params P;
    std::vector<State> u1, u2, u3, fx, fy, dfx, dfy, rhs;
    std::vector<Derived> derived;
    double t1 = 0, t2 = 0, t3 = 0;
    int err_code = 0;
    long err_i = 0, err_j = 0;
    std::string err_msg;

    void init_buffers() {
        size_t n = f.grid.len();
        long nx = f.grid.nx, ny = f.grid.ny;
        State z{0, 0, 0, 0, 0, 0};
        u1.assign(n, z); u2.assign(n, z); u3.assign(n, z); rhs.assign(n, z);
        fx.assign((size_t)(nx + 1) * ny, z); fy.assign((size_t)nx * (ny + 1), z);
        dfx.assign((size_t)(nx + 1) * ny, z); dfy.assign((size_t)nx * (ny + 1), z);
        derived.assign(n, Derived{});
    }

    // ghost.rs:199-268
    void update_ghosts(const State* val, double t) {
        std::atomic<int> bad{-1};
        std::string msg; int code = 0; long ei = 0, ej = 0;
#pragma omp parallel for schedule(dynamic, 32)
        for (long g = 0; g < (long)gg.info.size(); ++g) {
            try {
                State r = set_ghost_point_value(gg.info[g], f, val, t, gg, P);
                if (!state_finite(r)) {
                    int exp = -1;
                    bad.compare_exchange_strong(exp, (int)g);
                }
                gg.values[g] = r;
                gg.derived[g] = derived_from_state(r, P);
            } catch (OracleError& e) {
#pragma omp critical
                { msg = e.what(); code = e.code; ei = e.i; ej = e.j; }
            }
        }
        if (code) throw OracleError(code, msg, ei, ej);
        if (bad.load() >= 0) {
            const GhostInfo& gi = gg.info[bad.load()];
            throw OracleError(ERR_NONFINITE_GHOST, "NON-FINITE GHOST STATE", gi.i, gi.j);
        }
    }

    State v_at(const State* val, uint32_t t) const { return t < f.grid.len() ? val[t] : gg.values[t - f.grid.len()]; }
    Derived d_at(uint32_t t) const { return t < derived.size() ? derived[t] : gg.derived[t - derived.size()]; }

    void gather6(const State* val, size_t anchor, long di0, Dir dir, State st[6], Derived dd[6]) const {
        for (long q = 0; q < 6; ++q) {
            long d = di0 + q;
            int k = dir == DIR_X ? gg.k_for(d, 0) : gg.k_for(0, d);
            uint32_t t = gg.access[anchor * gg.n_offsets + k];
            st[q] = v_at(val, t);
            dd[q] = d_at(t);
        }
    }
    void gather9d(size_t anchor, Dir dir, Derived dd[9]) const {
        for (long q = 0; q < 9; ++q) {
            long d = -4 + q;
            int k = dir == DIR_X ? gg.k_for(d, 0) : gg.k_for(0, d);
            dd[q] = d_at(gg.access[anchor * gg.n_offsets + k]);
        }
    }

    // main.rs:135-305
    void l(const State* val, double t) {
        long nx = f.grid.nx, ny = f.grid.ny;
        double dx = f.grid.dx, dy = f.grid.dy;
        update_ghosts(val, t);
        State z{0, 0, 0, 0, 0, 0};
#pragma omp parallel for schedule(static)
        for (long l = 0; l < nx * ny; ++l)
            if (f.fluid[l]) derived[l] = derived_from_state(val[l], P);
#pragma omp parallel for schedule(static)
        for (long lin = 0; lin < (nx + 1) * ny; ++lin) {
            long i = lin / ny;
            size_t anchor; long di0;
            if (i < nx && f.fluid[lin]) { anchor = lin; di0 = -3; }
            else if (i >= 1 && f.fluid[lin - ny]) { anchor = lin - ny; di0 = -2; }
            else { fx[lin] = z; continue; }
            State st[6]; Derived dd[6];
            gather6(val, anchor, di0, DIR_X, st, dd);
            fx[lin] = reconstruction_fast(st, dd, DIR_X, true, P);
        }
#pragma omp parallel for schedule(static)
        for (long lin = 0; lin < nx * (ny + 1); ++lin) {
            long j = lin / nx, i = lin % nx;
            size_t cell = (size_t)i * ny + j;
            size_t anchor; long di0;
            if (j < ny && f.fluid[cell]) { anchor = cell; di0 = -3; }
            else if (j >= 1 && f.fluid[cell - 1]) { anchor = cell - 1; di0 = -2; }
            else { fy[lin] = z; continue; }
            State st[6]; Derived dd[6];
            gather6(val, anchor, di0, DIR_Y, st, dd);
            fy[lin] = reconstruction_fast(st, dd, DIR_Y, true, P);
        }
        bool diff = P.diffusion_active();
        if (diff) {
#pragma omp parallel for schedule(static)
            for (long lin = 0; lin < (nx + 1) * ny; ++lin) {
                long i = lin / ny;
                size_t anchor; long di0;
                if (i < nx && f.fluid[lin]) { anchor = lin; di0 = -3; }
                else if (i >= 1 && f.fluid[lin - ny]) { anchor = lin - ny; di0 = -2; }
                else { dfx[lin] = z; continue; }
                State st[6]; Derived dd[6];
                gather6(val, anchor, di0, DIR_X, st, dd);
                dfx[lin] = diffusion_from_derived(dd, P);
            }
#pragma omp parallel for schedule(static)
            for (long lin = 0; lin < nx * (ny + 1); ++lin) {
                long j = lin / nx, i = lin % nx;
                size_t cell = (size_t)i * ny + j;
                size_t anchor; long di0;
                if (j < ny && f.fluid[cell]) { anchor = cell; di0 = -3; }
                else if (j >= 1 && f.fluid[cell - 1]) { anchor = cell - 1; di0 = -2; }
                else { dfy[lin] = z; continue; }
                State st[6]; Derived dd[6];
                gather6(val, anchor, di0, DIR_Y, st, dd);
                dfy[lin] = diffusion_from_derived(dd, P);
            }
        }
        bool src = P.source_active();
#pragma omp parallel for schedule(static)
        for (long lin = 0; lin < nx * ny; ++lin) {
            if (!f.fluid[lin]) { rhs[lin] = z; continue; }
            long i = lin / ny, j = lin % ny;
            const State& fl = fx[lin];
            const State& fr = fx[lin + ny];
            const State& fb = fy[j * nx + i];
            const State& ft = fy[(j + 1) * nx + i];
            double sx = 1.0 / dx, sy = 1.0 / dy;
            State fxt, fyt;
            for (int c = 0; c < 6; ++c) {
                fxt[c] = -(fr[c] - fl[c]) * sx;
                fyt[c] = -(ft[c] - fb[c]) * sy;
            }
            Derived dx9[9], dy9[9];
            gather9d(lin, DIR_X, dx9);
            gather9d(lin, DIR_Y, dy9);
            State ncx = nonconservative_pre(dx9, dx, DIR_X);
            State ncy = nonconservative_pre(dy9, dy, DIR_Y);
            State so = src ? source(val[lin], P) : z;
            State dif = z;
            if (diff) {
                double cx = -1.0 / (dx * dx), cy = -1.0 / (dy * dy);
                const State& a = dfx[lin];
                const State& b = dfx[lin + ny];
                const State& c2 = dfy[j * nx + i];
                const State& d2 = dfy[(j + 1) * nx + i];
                for (int c = 0; c < 6; ++c) dif[c] = (-(b[c] - a[c]) * cx) + (-(d2[c] - c2[c]) * cy);
            }
            State o;
            for (int c = 0; c < 6; ++c) o[c] = fxt[c] + fyt[c] + ncx[c] + ncy[c] + so[c] + dif[c];
            rhs[lin] = o;
        }
    }

    // main.rs:22-33 admissibility
    static bool admissible(const State& s) {
        if (!state_finite(s) || s.rho <= 0.0) return false;
        double ux = s.mx / s.rho, uy = s.my / s.rho;
        double k = (ux * ux + uy * uy) / 6.0;
        return !(s.ee / s.rho - k <= 0.0 || s.ei / s.rho - k <= 0.0 || s.er / s.rho - k <= 0.0);
    }

    // main.rs:308-349
    void stage(const State* base, const State* add, State* dst, double coef, double wb, double wa, const char* label) {
        long n = (long)f.grid.len();
        std::atomic<long> first{-1};
#pragma omp parallel for schedule(static)
        for (long l = 0; l < n; ++l) {
            if (!f.fluid[l]) continue;
            State v;
            if (!add) {
                for (int c = 0; c < 6; ++c) v[c] = base[l][c] + rhs[l][c] * coef;
            } else {
                for (int c = 0; c < 6; ++c) v[c] = base[l][c] * wb + add[l][c] * wa + rhs[l][c] * coef;
            }
            if (!admissible(v)) {
                long cur = first.load();
                while ((cur < 0 || l < cur) && !first.compare_exchange_weak(cur, l)) {}
            }
            dst[l] = v;
        }
        if (first.load() >= 0) {
            long l = first.load();
            throw OracleError(ERR_NONPHYSICAL, std::string("non-physical state in ") + label, l / f.grid.ny, l % f.grid.ny);
        }
    }

    // main.rs:351-373
    void rk3_ssp(double dt) {
        double t = f.time;
        l(f.value.data(), t);
        stage(f.value.data(), nullptr, u1.data(), dt, 0, 0, "RK1 state");
        t1 = t + dt;
        l(u1.data(), t1);
        stage(f.value.data(), u1.data(), u2.data(), dt / 4.0, 0.75, 0.25, "RK2 state");
        t2 = t + 0.5 * dt;
        l(u2.data(), t2);
        stage(f.value.data(), u2.data(), u3.data(), 2.0 * dt / 3.0, 1.0 / 3.0, 2.0 / 3.0, "RK3 state");
        t3 = t + dt;
        std::swap(f.value, u3);
        f.time = t3;
    }

    // main.rs:375-408
    double calc_global_dt() const {
        long nx = f.grid.nx, ny = f.grid.ny;
        double g = INFINITY;
#pragma omp parallel for reduction(min : g) schedule(static)
        for (long l = 0; l < nx * ny; ++l) {
            if (!f.fluid[l]) continue;
            double d = get_local_dt(f.value[l], f.grid.dx, f.grid.dy, P);
            g = std::fmin(g, d);
        }
        return g;
    }
};

// ---------------------------------------------------------------- init.rs
// init.rs:7-24
static State euler_to_three_energy(double rho, double ux, double uy, double p, double gamma) {
    double kinetic = 0.5 * rho * (ux * ux + uy * uy);
    double e_total = p / (gamma - 1.0) + kinetic;
    return {rho, rho * ux, rho * uy, e_total / 3.0, e_total / 3.0, e_total / 3.0};
}

static Polygon dummy_inner() {
    Polygon p;
    p.pts = {{-1002.0, -1002.0}, {-1001.0, -1002.0}, {-1001.0, -1001.0}, {-1002.0, -1001.0}};
    p.fluid = FLUID_OUTSIDE;
    return p;
}

// init.rs:116-510 init_cylinder, with the mesh width h, the inflow Mach number
// and the arc's y-shift as parameters (the reference fixes h = 1/40, M = 3 and
// the literal shift 0.0125).
static void init_cylinder(Field& u, double h, double mach, double shift) {
    double gamma = 1.4, rho_inf = 1.0, p_inf = 1.0;
    double a_inf = std::sqrt(gamma * p_inf / rho_inf);
    double ux_inf = mach * a_inf;
    State uinf = euler_to_three_energy(rho_inf, ux_inf, 0.0, p_inf, gamma);
    double x0 = -3.0, y0 = -6.0, lx = 3.0, ly = 12.0;
    long nx = (long)std::round(lx / h) + 1, ny = (long)std::round(ly / h) + 1;
    u.grid = {nx, ny, h, h, x0, y0};
    std::vector<Point> pts;
    std::vector<BC> bcs;
    BC ff; ff.kind = BC_FAR_FIELD; ff.state = uinf;
    BC rw; rw.kind = BC_REFLECTIVE_WALL;
    pts.push_back({-3.0, -6.0});
    pts.push_back({0.0, -6.0}); bcs.push_back(ff);
    pts.push_back({0.0, -1.0 + shift}); bcs.push_back(ff);
    long n_arc = 360;
    size_t arc_start = bcs.size();
    for (long k = 1; k <= n_arc; ++k) {
        double s = (double)k / (double)n_arc;
        double theta = -0.5 * M_PI - M_PI * s;
        pts.push_back({std::cos(theta), std::sin(theta) + shift});
        bcs.push_back(rw);
    }
    size_t arc_end = bcs.size() - 1;
    CircularArc arc = CircularArc::from_three_points({0.0, -1.0 + shift}, {-1.0, 0.0 + shift}, {0.0, 1.0 + shift},
                                                     FLUID_OUTSIDE);
    pts.push_back({0.0, 6.0}); bcs.push_back(ff);
    pts.push_back({-3.0, 6.0}); bcs.push_back(ff);
    bcs.push_back(ff);
    u.outer.pts = pts; u.outer.fluid = FLUID_INSIDE;
    u.inner = dummy_inner();
    u.bc_outer = bcs;
    BC wall; wall.kind = BC_WALL;
    u.bc_inner.assign(4, wall);
    u.time = 0.0;
    u.init_mask();
    u.outer_arcs.push_back({arc_start, arc_end, arc});
    u.value.assign(u.grid.len(), State{0, 0, 0, 0, 0, 0});
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j)
            if (u.is_in_domain(i, j)) u.value[u.linear_index(i, j)] = uinf;
}

// init.rs:26-113 init_double_mach (mesh width as a parameter; reference 1/320)
static void init_double_mach(Field& u, double h) {
    double sqrt3 = std::sqrt(3.0);
    Point a{-0.5 - sqrt3 / 12.0, 0.0}, b{0.0, 0.0}, c{23.0 * sqrt3 / 12.0, 23.0 / 12.0};
    Point d{c.x, 23.0 / 12.0 + sqrt3 / 2.0}, e{a.x, d.y};
    double x0 = a.x, y0 = 0.0, lx = c.x - a.x, ly = d.y;
    long nx = (long)std::ceil(lx / h) + 1, ny = (long)std::ceil(ly / h) + 1;
    u.grid = {nx, ny, h, h, x0, y0};
    double gamma = 1.4;
    State pre = euler_to_three_energy(1.4, 0.0, 0.0, 1.0, gamma);
    State post = euler_to_three_energy(8.0, 8.25, 0.0, 116.5, gamma);
    u.outer.pts = {a, b, c, d, e}; u.outer.fluid = FLUID_INSIDE;
    BC cpost; cpost.kind = BC_CONSTANT; cpost.state = post;
    BC cpre; cpre.kind = BC_CONSTANT; cpre.state = pre;
    BC wall; wall.kind = BC_WALL;
    BC zo; zo.kind = BC_ZEROTH_ORDER;
    u.bc_outer = {cpost, wall, cpre, zo, cpost};
    u.inner = dummy_inner();
    u.bc_inner.assign(4, wall);
    u.time = 0.0;
    u.init_mask();
    u.value.assign(u.grid.len(), State{0, 0, 0, 0, 0, 0});
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j) {
            if (!u.is_in_domain(i, j)) continue;
            u.value[u.linear_index(i, j)] = u.grid.x(i) <= 0.0 ? post : pre;
        }
}

// Translating Mach-2 planar shock, y-periodic (not in the reference, which has
// no such initializer): gamma = 1.4 normal-shock Rankine-Hugoniot on the total
// energy (valid because all three gammas are 1.4), pre-shock (1, 0, 1) with
// Te = Ti = Tr, post-shock Te:Ti:Tr = 1 : 1.5 : 0.8.
static double solve_temperature(double target, double ce, double ci, double cr, double rho, const Params& P) {
    // e_e + e_i + e_r = ce*T/Cve*Cve ... monotone in T: bisection to machine precision
    double lo = 0.0, hi = 1.0;
    auto f = [&](double T) {
        double te = ce * T, ti = ci * T, tr = cr * T;
        return P.cve * te + P.cvi * ti + P.a_rad * pow4(tr) / rho - target;
    };
    while (f(hi) < 0.0) hi *= 2.0;
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (f(mid) < 0.0) lo = mid; else hi = mid;
        if (hi - lo <= 0.0) break;
    }
    return 0.5 * (lo + hi);
}

static State three_temp_state(double rho, double u, double v, double te, double ti, double tr, const Params& P) {
    double e_e = P.cve * te, e_i = P.cvi * ti, e_r = P.a_rad * pow4(tr) / rho;
    double k = rho * (u * u + v * v) / 6.0;
    return {rho, rho * u, rho * v, rho * e_e + k, rho * e_i + k, rho * e_r + k};
}

static void init_planar_shock(Field& u, long nx, long ny, double lx, double ly, double x_shock, double mach,
                              double sigma, const Params& P) {
    u.grid = {nx, ny, lx / (double)nx, ly / (double)ny, 0.0, 0.0};
    double g = 1.4, rho1 = 1.0, u1 = 0.0, p1 = 1.0;
    double c1 = std::sqrt(g * p1 / rho1);
    double m2 = mach * mach;
    double rho2 = rho1 * (g + 1.0) * m2 / ((g - 1.0) * m2 + 2.0);
    double p2 = p1 * (2.0 * g * m2 - (g - 1.0)) / (g + 1.0);
    double ws = mach * c1;
    double u2 = ws * (1.0 - rho1 / rho2);
    double t1 = solve_temperature(p1 / ((g - 1.0) * rho1), 1.0, 1.0, 1.0, rho1, P);
    double t2 = solve_temperature(p2 / ((g - 1.0) * rho2), 1.0, 1.5, 0.8, rho2, P);
    State pre = three_temp_state(rho1, u1, 0.0, t1, t1, t1, P);
    State post = three_temp_state(rho2, u2, 0.0, t2, 1.5 * t2, 0.8 * t2, P);
    u.outer.pts = {{0.0, 0.0}, {lx, 0.0}, {lx, ly}, {0.0, ly}};
    u.outer.fluid = FLUID_INSIDE;
    BC per; per.kind = BC_PERIODIC;
    BC out; out.kind = BC_OUTFLOW; out.p_inf = p1; out.sigma = sigma; out.l_domain = lx;
    BC ff; ff.kind = BC_FAR_FIELD; ff.state = post;
    u.bc_outer = {per, out, per, ff};
    u.inner = dummy_inner();
    BC wall; wall.kind = BC_WALL;
    u.bc_inner.assign(4, wall);
    u.time = 0.0;
    u.init_mask();
    u.value.assign(u.grid.len(), State{0, 0, 0, 0, 0, 0});
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j)
            if (u.is_in_domain(i, j)) u.value[u.linear_index(i, j)] = u.grid.x(i) < x_shock ? post : pre;
}

// bc1.rs:1641-1702 make_rect_field (reference test fixture): [0,lx]x[0,ly]
// with one BC kind on all four sides.
static void init_rect(Field& u, long nx, long ny, double lx, double ly, const State& value, BCKind kind) {
    u.grid = {nx, ny, lx / (double)nx, ly / (double)ny, 0.0, 0.0};
    u.outer.pts = {{0.0, 0.0}, {lx, 0.0}, {lx, ly}, {0.0, ly}};
    u.outer.fluid = FLUID_INSIDE;
    BC b; b.kind = kind; b.state = value;
    u.bc_outer.assign(4, b);
    u.inner = dummy_inner();
    BC wall; wall.kind = BC_WALL;
    u.bc_inner.assign(4, wall);
    u.time = 0.0;
    u.init_mask();
    u.value.assign(u.grid.len(), value);
}


// ---------------------------------------------------------------- l() over a scalar type
// The functions above written over T (jvp.hpp): same operations, same order.
template <class T> static bool solve6_t(T A[6][6], T b[6]) {
    int piv[6];
    for (int j = 0; j < 6; ++j) {
        int p = j;
        double mx = std::fabs(val(A[j][j]));
        for (int i = j + 1; i < 6; ++i)
            if (std::fabs(val(A[i][j])) > mx) { mx = std::fabs(val(A[i][j])); p = i; }
        piv[j] = p;
        if (val(A[p][j]) == 0.0) return false;
        if (p != j) for (int k = 0; k < 6; ++k) std::swap(A[j][k], A[p][k]);
        T rcp = T(1.0) / A[j][j];
        for (int i = j + 1; i < 6; ++i) A[i][j] *= rcp;
        for (int k = j + 1; k < 6; ++k)
            for (int i = j + 1; i < 6; ++i) A[i][k] -= A[i][j] * A[j][k];
    }
    for (int j = 0; j < 6; ++j) if (piv[j] != j) std::swap(b[j], b[piv[j]]);
    for (int k = 0; k < 6; ++k)
        for (int i = k + 1; i < 6; ++i) b[i] -= b[k] * A[i][k];
    for (int k = 5; k >= 0; --k) {
        b[k] /= A[k][k];
        for (int i = 0; i < k; ++i) b[i] -= b[k] * A[i][k];
    }
    return true;
}

template <class T> static void mat_vec_t(const T M[6][6], const T x[6], T out[6]) {
    for (int i = 0; i < 6; ++i) {
        T acc = T(0.0);
        for (int j = 0; j < 6; ++j) acc += M[i][j] * x[j];
        out[i] = acc;
    }
}

template <class T>
static void build_local_plain_t(Vec2 n, const StateT<T>& val_, const Params& P, T L[6][6], T R[6][6], T lam[6]) {
    T mom_n = val_.mx * n.x + val_.my * n.y;
    T mom_t = -val_.mx * n.y + val_.my * n.x;
    StateT<T> s1{val_.rho, mom_n, mom_t, val_.ee, val_.ei, val_.er};
    DerivedT<T> d1 = derived_from_state(s1, P);
    build_l_plain(s1, s1, d1, d1, DIR_X, P, L);
    build_r_plain(s1, s1, d1, d1, DIR_X, P, lam, R);
}

template <class T>
static void weno_extrapolation_all_t(const T L[6][6], const GhostBC& bc, const StateT<T>* v_, const Params& P,
                                     T v[5][6]) {
    using std::pow;
    Vec2 n = bc.normal;
    T alpha[6][5], vks[5][6][5], asum[6];
    for (int c = 0; c < 6; ++c) asum[c] = T(0.0);
    for (int r = 0; r <= 4; ++r) {
        int m = (r + 1) * (r + 1);
        T data[6][25];
        for (int a = 0; a < m; ++a) {
            const StateT<T>& s = v_[bc.stencil[BC_STENCIL_OFF[r] + a]];
            T mn = s.mx * n.x + s.my * n.y;
            T mt = -s.mx * n.y + s.my * n.x;
            T u6[6] = {s.rho, mn, mt, s.ee, s.ei, s.er};
            for (int c = 0; c < 6; ++c) {
                const T* row = L[c];
                data[c][a] = row[0] * u6[0] + row[1] * u6[1] + row[2] * u6[2] + row[3] * u6[3] + row[4] * u6[4] +
                             row[5] * u6[5];
            }
        }
        for (int c = 0; c < 6; ++c) {
            int soff = BC_S_OFF[r];
            T beta = T(0.0);
            for (int a = 0; a < m; ++a) {
                int base = soff + a * m;
                T acc = T(0.0);
                for (int b = 0; b < m; ++b) acc += bc.s[base + b] * data[c][b];
                beta += data[c][a] * acc;
            }
            for (int k = 0; k < 5; ++k) {
                T vk = T(0.0);
                if (k <= r) {
                    int woff = BC_W_OFF[r] + k * m;
                    for (int a = 0; a < m; ++a) vk += bc.w[woff + a] * data[c][a];
                }
                vks[k][c][r] = vk;
            }
            alpha[c][r] = bc.d[r] / powf_ref(P.eps + beta, P.weno_q);
            asum[c] += alpha[c][r];
        }
    }
    for (int k = 0; k < 5; ++k)
        for (int c = 0; c < 6; ++c) {
            T res = T(0.0);
            for (int r = 0; r <= 4; ++r) res += (alpha[c][r] / asum[c]) * vks[k][c][r];
            v[k][c] = res;
        }
}

template <class T> static StateT<T> taylor_rotate_t(T u[5][6], double d, Vec2 n) {
    T g[6];
    for (int c = 0; c < 6; ++c) g[c] = u[0][c];
    double coef = 1.0;
    for (int k = 1; k <= 4; ++k) {
        coef *= d / (double)k;
        for (int c = 0; c < 6; ++c) g[c] = g[c] + coef * u[k][c];
    }
    T mom_n = g[1], mom_t = g[2];
    return {g[0], mom_n * n.x - mom_t * n.y, mom_n * n.y + mom_t * n.x, g[3], g[4], g[5]};
}

template <class T>
static StateT<T> set_ghost_point_value_t(const GhostInfo& g, const Field& f, const StateT<T>* v_, double t,
                                         const GhostGrid& gg, const Params& P, const Tangent& tg) {
    using std::sqrt; using std::fabs;
    const BC& bc = (g.boundary == OUTER ? f.bc_outer : f.bc_inner)[g.side_id];
    const Projection& pr = g.project;
    auto cst = [](const State& s) { return StateT<T>{T(s.rho), T(s.mx), T(s.my), T(s.ee), T(s.ei), T(s.er)}; };
    switch (bc.kind) {
    case BC_CONSTANT: return cst(bc.state);
    case BC_TIME_DEPENDENT: {
        double xs = bc.td_x0 + bc.td_speed * t;
        return cst(pr.point.x <= xs ? bc.td_left : bc.td_right);
    }
    case BC_REFLECTIVE_WALL: {
        long oi, oj;
        if (!mirror_source(g.i, g.j, pr, f, oi, oj))
            throw OracleError(ERR_GEOMETRY, "cannot find reflected interior point for ghost", g.i, g.j);
        const StateT<T>& s = v_[f.linear_index(oi, oj)];
        Vec2 n = pr.normal;
        T mom_n = s.mx * n.x + s.my * n.y;
        return {s.rho, s.mx - 2.0 * mom_n * n.x, s.my - 2.0 * mom_n * n.y, s.ee, s.ei, s.er};
    }
    case BC_ZEROTH_ORDER: {
        long oi, oj;
        if (!mirror_source(g.i, g.j, pr, f, oi, oj))
            throw OracleError(ERR_GEOMETRY, "cannot find interior point for zeroth-order ghost", g.i, g.j);
        return v_[f.linear_index(oi, oj)];
    }
    case BC_PERIODIC: {
        long np = (long)std::round(P.periodic_ly / f.grid.dy);
        long jw = ((g.j % np) + np) % np;
        if (!f.is_in_domain(g.i, jw)) throw OracleError(ERR_PERIODIC, "periodic wrapped point is not fluid", g.i, jw);
        return v_[f.linear_index(g.i, jw)];
    }
    default: break;
    }
    const GhostBC& pre = gg.pre[g.pre];
    T L[6][6], R[6][6], lam[6];
    build_local_plain_t(pr.normal, v_[f.linear_index(pre.nearest_i, pre.nearest_j)], P, L, R, lam);
    T v[5][6];
    weno_extrapolation_all_t(L, pre, v_, P, v);
    T u[5][6];
    if (bc.kind == BC_WALL) {
        T A0[6][6], rhs0[6];
        for (int i = 0; i < 6; ++i) for (int c = 0; c < 6; ++c) A0[i][c] = L[i][c];
        for (int c = 0; c < 6; ++c) A0[0][c] = T(c == 1 ? 1.0 : 0.0);
        for (int c = 0; c < 6; ++c) rhs0[c] = v[0][c];
        rhs0[0] = T(0.0);
        if (!solve6_t(A0, rhs0)) throw OracleError(ERR_SINGULAR, "singular ILW/extrapolation system at boundary", g.i, g.j);
        for (int c = 0; c < 6; ++c) u[0][c] = rhs0[c];
        T A1[6][6], rhs1[6], row1[6];
        for (int i = 0; i < 6; ++i) for (int c = 0; c < 6; ++c) A1[i][c] = L[i][c];
        double gi = P.gamma_i - 1.0, ge = P.gamma_e - 1.0, gr = P.gamma_r - 1.0;
        double gt = gi + ge + gr;
        T u1 = u[0][0], u3 = u[0][2];
        row1[0] = -gt * sq(u3) / (6.0 * sq(u1));
        row1[1] = T(0.0);
        row1[2] = gt * u3 / (6.0 * u1);
        row1[3] = T(-ge); row1[4] = T(-gi); row1[5] = T(-gr);
        for (int c = 0; c < 6; ++c) A1[0][c] = row1[c];
        for (int c = 0; c < 6; ++c) rhs1[c] = v[1][c];
        rhs1[0] = T(0.0);
        if (!solve6_t(A1, rhs1)) throw OracleError(ERR_SINGULAR, "singular ILW/extrapolation system at boundary", g.i, g.j);
        for (int c = 0; c < 6; ++c) u[1][c] = rhs1[c];
        for (int k = 2; k <= 4; ++k) mat_vec_t(R, v[k], u[k]);
    } else if (bc.kind == BC_OUTFLOW) {
        mat_vec_t(R, v[0], u[0]);
        T rho0 = u[0][0];
        T un0 = u[0][1] / rho0, ut0 = u[0][2] / rho0;
        T w2 = un0 * un0 + ut0 * ut0;
        T ee1 = u[0][3] / rho0 - w2 / 6.0, ei1 = u[0][4] / rho0 - w2 / 6.0, er1 = u[0][5] / rho0 - w2 / 6.0;
        double ge = P.gamma_e - 1.0, gi = P.gamma_i - 1.0, gr = P.gamma_r - 1.0;
        T p0 = rho0 * (ge * ee1 + gi * ei1 + gr * er1);
        T a2 = P.gamma_e * ge * ee1 + P.gamma_i * gi * ei1 + P.gamma_r * gr * er1;
        T a = sqrt(a2);
        T lambda1 = un0 - a;
        T rhs1[6];
        for (int c = 0; c < 6; ++c) rhs1[c] = v[1][c];
        if (val(lambda1) < 0.0) {
            T m_local = fabs(un0 / a);
            T l1 = bc.sigma * (1.0 - sq(m_local)) * a / bc.l_domain * (p0 - bc.p_inf);
            rhs1[0] = l1 / lambda1;
        }
        mat_vec_t(R, rhs1, u[1]);
        for (int k = 2; k <= 4; ++k) mat_vec_t(R, v[k], u[k]);
    } else if (bc.kind == BC_FAR_FIELD) {
        Vec2 n = pr.normal;
        StateT<T> ui;
        for (int c = 0; c < 6; ++c) ui[c] = seed<T>(bc.state[c], tg.duinf[c]);
        T uinf[6] = {ui.rho, ui.mx * n.x + ui.my * n.y, -ui.mx * n.y + ui.my * n.x, ui.ee, ui.ei, ui.er};
        T vinf[6];
        mat_vec_t(L, uinf, vinf);
        T rhs0[6];
        for (int c = 0; c < 6; ++c) rhs0[c] = val(lam[c]) < 0.0 ? vinf[c] : v[0][c];
        mat_vec_t(R, rhs0, u[0]);
        for (int k = 1; k <= 4; ++k) {
            T rk[6];
            for (int c = 0; c < 6; ++c) rk[c] = val(lam[c]) < 0.0 ? T(0.0) : v[k][c];
            mat_vec_t(R, rk, u[k]);
        }
    } else {
        return StateT<T>{};
    }
    return taylor_rotate_t(u, pr.distance, pr.normal);
}

// source.rs:7-21 with the exchange coefficients as T
template <class T> static StateT<T> source_t(const StateT<T>& s, const Params& P, T oei, T oer) {
    T te = state_te(s, P), tr = state_tr(s, P), ti = state_ti(s, P);
    return {T(0.0), T(0.0), T(0.0), -oei * (te - ti) - oer * (pow4(te) - pow4(tr)), oei * (te - ti),
            oer * (pow4(te) - pow4(tr))};
}

// main.rs:135-305 l() over T at state u (+ tangent), Field::time t
template <class T>
static void l_t(const Solver& S, const Tangent& tg, std::vector<StateT<T>>& rhs, std::vector<StateT<T>>& gval) {
    const Field& f = S.f;
    const GhostGrid& gg = S.gg;
    const Params& P = S.P;
    const long nx = f.grid.nx, ny = f.grid.ny, n = nx * ny;
    const double dx = f.grid.dx, dy = f.grid.dy;
    std::vector<StateT<T>> u((size_t)n);
    for (long l = 0; l < n; ++l)
        for (int c = 0; c < 6; ++c) u[l][c] = seed<T>(f.value[l][c], tg.du && f.fluid[l] ? tg.du[6 * l + c] : 0.0);
    gval.assign(gg.info.size(), StateT<T>{});
    std::vector<DerivedT<T>> gder(gg.info.size()), der((size_t)n);
    for (size_t g = 0; g < gg.info.size(); ++g) {
        gval[g] = set_ghost_point_value_t<T>(gg.info[g], f, u.data(), f.time, gg, P, tg);
        gder[g] = derived_from_state(gval[g], P);
    }
    for (long l = 0; l < n; ++l)
        if (f.fluid[l]) der[l] = derived_from_state(u[l], P);
    auto v_at = [&](uint32_t t) { return t < (uint32_t)n ? u[t] : gval[t - n]; };
    auto d_at = [&](uint32_t t) { return t < (uint32_t)n ? der[t] : gder[t - n]; };
    auto gather6 = [&](size_t anchor, long di0, Dir dir, StateT<T> st[6], DerivedT<T> dd[6]) {
        for (long q = 0; q < 6; ++q) {
            long d = di0 + q;
            int k = dir == DIR_X ? gg.k_for(d, 0) : gg.k_for(0, d);
            uint32_t t = gg.access[anchor * gg.n_offsets + k];
            st[q] = v_at(t);
            dd[q] = d_at(t);
        }
    };
    StateT<T> z{};
    std::vector<StateT<T>> fx((size_t)(nx + 1) * ny, z), fy((size_t)nx * (ny + 1), z);
    std::vector<StateT<T>> dfx((size_t)(nx + 1) * ny, z), dfy((size_t)nx * (ny + 1), z);
    const bool diff = P.diffusion_active();
    for (long lin = 0; lin < (nx + 1) * ny; ++lin) {
        long i = lin / ny;
        size_t anchor; long di0;
        if (i < nx && f.fluid[lin]) { anchor = lin; di0 = -3; }
        else if (i >= 1 && f.fluid[lin - ny]) { anchor = lin - ny; di0 = -2; }
        else continue;
        StateT<T> st[6]; DerivedT<T> dd[6];
        gather6(anchor, di0, DIR_X, st, dd);
        fx[lin] = reconstruction_fast(st, dd, DIR_X, true, P);
        if (diff) dfx[lin] = diffusion_from_derived(dd, P);
    }
    for (long lin = 0; lin < nx * (ny + 1); ++lin) {
        long j = lin / nx, i = lin % nx;
        size_t cell = (size_t)i * ny + j;
        size_t anchor; long di0;
        if (j < ny && f.fluid[cell]) { anchor = cell; di0 = -3; }
        else if (j >= 1 && f.fluid[cell - 1]) { anchor = cell - 1; di0 = -2; }
        else continue;
        StateT<T> st[6]; DerivedT<T> dd[6];
        gather6(anchor, di0, DIR_Y, st, dd);
        fy[lin] = reconstruction_fast(st, dd, DIR_Y, true, P);
        if (diff) dfy[lin] = diffusion_from_derived(dd, P);
    }
    const bool src = P.source_active() || tg.domega_ei != 0.0 || tg.domega_er != 0.0;
    const T oei = seed<T>(P.omega_ei, tg.domega_ei), oer = seed<T>(P.omega_er, tg.domega_er);
    rhs.assign((size_t)n, z);
    for (long lin = 0; lin < n; ++lin) {
        if (!f.fluid[lin]) continue;
        long i = lin / ny, j = lin % ny;
        const StateT<T>& fl = fx[lin];
        const StateT<T>& fr = fx[lin + ny];
        const StateT<T>& fb = fy[j * nx + i];
        const StateT<T>& ft = fy[(j + 1) * nx + i];
        double sx = 1.0 / dx, sy = 1.0 / dy;
        StateT<T> fxt, fyt;
        for (int c = 0; c < 6; ++c) {
            fxt[c] = -(fr[c] - fl[c]) * sx;
            fyt[c] = -(ft[c] - fb[c]) * sy;
        }
        DerivedT<T> dx9[9], dy9[9];
        for (long q = 0; q < 9; ++q) {
            dx9[q] = d_at(gg.access[lin * gg.n_offsets + gg.k_for(-4 + q, 0)]);
            dy9[q] = d_at(gg.access[lin * gg.n_offsets + gg.k_for(0, -4 + q)]);
        }
        StateT<T> ncx = nonconservative_pre(dx9, dx, DIR_X);
        StateT<T> ncy = nonconservative_pre(dy9, dy, DIR_Y);
        StateT<T> so = src ? source_t(u[lin], P, oei, oer) : z;
        StateT<T> dif = z;
        if (diff) {
            double cx = -1.0 / (dx * dx), cy = -1.0 / (dy * dy);
            const StateT<T>& a = dfx[lin];
            const StateT<T>& b = dfx[lin + ny];
            const StateT<T>& c2 = dfy[j * nx + i];
            const StateT<T>& d2 = dfy[(j + 1) * nx + i];
            for (int c = 0; c < 6; ++c) dif[c] = (-(b[c] - a[c]) * cx) + (-(d2[c] - c2[c]) * cy);
        }
        StateT<T> o;
        for (int c = 0; c < 6; ++c) o[c] = fxt[c] + fyt[c] + ncx[c] + ncy[c] + so[c] + dif[c];
        rhs[lin] = o;
    }
}

} // namespace oracle

// ================================================================ C API
using namespace oracle;

static void params_from(const double* p, Params& P) {
    if (!p) return;
    P.gamma_e = p[0]; P.gamma_i = p[1]; P.gamma_r = p[2];
    P.cve = p[3]; P.cvi = p[4]; P.a_rad = p[5];
    P.kappa_e = p[6]; P.kappa_i = p[7]; P.kappa_r = p[8];
    P.omega_ei = p[9]; P.omega_er = p[10];
    P.lambda = p[11]; P.weno_q = p[12]; P.eps = p[13]; P.periodic_ly = p[14];
}

struct Handle {
    Solver s;
    bool built = false;
};

static int finish_build(Handle* h, char* msg, int len) {
    try {
        h->s.gg.build(h->s.f, default_stencil_offsets());
        h->s.init_buffers();
        h->built = true;
        return 0;
    } catch (OracleError& e) {
        if (msg && len > 0) { std::strncpy(msg, e.what(), len - 1); msg[len - 1] = 0; }
        return e.code;
    }
}

static void set_err(Handle* h, const OracleError& e) {
    h->s.err_code = e.code; h->s.err_i = e.i; h->s.err_j = e.j; h->s.err_msg = e.what();
}

extern "C" {

void oracle_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int oracle_max_threads() { return omp_get_max_threads(); }

void* oracle_create_cylinder(double h, double mach, double shift, const double* params, char* msg, int len) {
    Handle* H = new Handle();
    params_from(params, H->s.P);
    try { init_cylinder(H->s.f, h, mach, shift); } catch (OracleError& e) { delete H; return nullptr; }
    if (finish_build(H, msg, len)) { delete H; return nullptr; }
    return H;
}

void* oracle_create_double_mach(double h, const double* params, char* msg, int len) {
    Handle* H = new Handle();
    params_from(params, H->s.P);
    init_double_mach(H->s.f, h);
    if (finish_build(H, msg, len)) { delete H; return nullptr; }
    return H;
}

void* oracle_create_planar_shock(long nx, long ny, double lx, double ly, double x_shock, double mach, double sigma,
                                 const double* params, char* msg, int len) {
    Handle* H = new Handle();
    params_from(params, H->s.P);
    init_planar_shock(H->s.f, nx, ny, lx, ly, x_shock, mach, sigma, H->s.P);
    if (finish_build(H, msg, len)) { delete H; return nullptr; }
    return H;
}

void* oracle_create_rect(long nx, long ny, double lx, double ly, const double* state6, int kind, const double* params,
                         char* msg, int len) {
    Handle* H = new Handle();
    params_from(params, H->s.P);
    State v{state6[0], state6[1], state6[2], state6[3], state6[4], state6[5]};
    init_rect(H->s.f, nx, ny, lx, ly, v, (BCKind)kind);
    if (finish_build(H, msg, len)) { delete H; return nullptr; }
    return H;
}

void oracle_destroy(void* h) { delete (Handle*)h; }

void oracle_dims(void* h, long* nx, long* ny, double* g4) {
    Field& f = ((Handle*)h)->s.f;
    *nx = f.grid.nx; *ny = f.grid.ny;
    g4[0] = f.grid.dx; g4[1] = f.grid.dy; g4[2] = f.grid.x0; g4[3] = f.grid.y0;
}
void oracle_params(void* h, double* p) {
    Params& P = ((Handle*)h)->s.P;
    double v[15] = {P.gamma_e, P.gamma_i, P.gamma_r, P.cve, P.cvi, P.a_rad, P.kappa_e, P.kappa_i, P.kappa_r,
                    P.omega_ei, P.omega_er, P.lambda, P.weno_q, P.eps, P.periodic_ly};
    std::memcpy(p, v, sizeof(v));
}
void oracle_fluid(void* h, uint8_t* out) {
    Field& f = ((Handle*)h)->s.f;
    std::memcpy(out, f.fluid.data(), f.fluid.size());
}
void oracle_get_state(void* h, double* out) {
    Field& f = ((Handle*)h)->s.f;
    std::memcpy(out, f.value.data(), f.value.size() * sizeof(State));
}
void oracle_set_state(void* h, const double* in) {
    Field& f = ((Handle*)h)->s.f;
    std::memcpy(f.value.data(), in, f.value.size() * sizeof(State));
}
double oracle_time(void* h) { return ((Handle*)h)->s.f.time; }
void oracle_set_time(void* h, double t) { ((Handle*)h)->s.f.time = t; }

// polygon description: n_outer/n_inner points, BC kinds and states
void oracle_geometry_sizes(void* h, long* sizes) {
    Field& f = ((Handle*)h)->s.f;
    sizes[0] = (long)f.outer.pts.size(); sizes[1] = (long)f.inner.pts.size();
    sizes[2] = (long)f.outer_arcs.size(); sizes[3] = (long)f.inner_arcs.size();
}
void oracle_geometry(void* h, double* outer_xy, double* inner_xy, int32_t* outer_kind, int32_t* inner_kind,
                     double* outer_bc /* n*24 */, double* inner_bc, int32_t* fluid_sides) {
    Field& f = ((Handle*)h)->s.f;
    auto put_bc = [](const BC& b, double* o) {
        for (int k = 0; k < 6; ++k) o[k] = b.state[k];
        o[6] = b.p_inf; o[7] = b.sigma; o[8] = b.l_domain; o[9] = b.td_x0; o[10] = b.td_speed;
        for (int k = 0; k < 6; ++k) { o[11 + k] = b.td_left[k]; o[17 + k] = b.td_right[k]; }
        o[23] = 0.0;
    };
    for (size_t k = 0; k < f.outer.pts.size(); ++k) {
        outer_xy[2 * k] = f.outer.pts[k].x; outer_xy[2 * k + 1] = f.outer.pts[k].y;
        outer_kind[k] = f.bc_outer[k].kind; put_bc(f.bc_outer[k], outer_bc + 24 * k);
    }
    for (size_t k = 0; k < f.inner.pts.size(); ++k) {
        inner_xy[2 * k] = f.inner.pts[k].x; inner_xy[2 * k + 1] = f.inner.pts[k].y;
        inner_kind[k] = f.bc_inner[k].kind; put_bc(f.bc_inner[k], inner_bc + 24 * k);
    }
    fluid_sides[0] = f.outer.fluid; fluid_sides[1] = f.inner.fluid;
}

long oracle_n_ghosts(void* h) { return (long)((Handle*)h)->s.gg.info.size(); }
long oracle_n_heavy(void* h) { return (long)((Handle*)h)->s.gg.pre.size(); }

// per ghost: ij[2], boundary, side, proj[5] (p0x p0y nx ny dist), nearest[2] (raw projection), pre index
void oracle_ghost_info(void* h, int32_t* ij, int32_t* boundary, int32_t* side, double* proj, int32_t* nearest,
                       int32_t* pre) {
    GhostGrid& gg = ((Handle*)h)->s.gg;
    for (size_t g = 0; g < gg.info.size(); ++g) {
        const GhostInfo& gi = gg.info[g];
        ij[2 * g] = (int32_t)gi.i; ij[2 * g + 1] = (int32_t)gi.j;
        boundary[g] = gi.boundary; side[g] = (int32_t)gi.side_id;
        proj[5 * g] = gi.project.point.x; proj[5 * g + 1] = gi.project.point.y;
        proj[5 * g + 2] = gi.project.normal.x; proj[5 * g + 3] = gi.project.normal.y;
        proj[5 * g + 4] = gi.project.distance;
        nearest[2 * g] = (int32_t)gi.nearest_i; nearest[2 * g + 1] = (int32_t)gi.nearest_j;
        pre[g] = gi.pre;
    }
}
void oracle_ghost_pre(void* h, int32_t* nearest, uint32_t* stencil, double* s, double* w, double* d) {
    GhostGrid& gg = ((Handle*)h)->s.gg;
    for (size_t k = 0; k < gg.pre.size(); ++k) {
        const GhostBC& b = gg.pre[k];
        nearest[2 * k] = (int32_t)b.nearest_i; nearest[2 * k + 1] = (int32_t)b.nearest_j;
        std::memcpy(stencil + 55 * k, b.stencil, sizeof(b.stencil));
        std::memcpy(s + 979 * k, b.s, sizeof(b.s));
        std::memcpy(w + 225 * k, b.w, sizeof(b.w));
        std::memcpy(d + 5 * k, b.d, sizeof(b.d));
    }
}
void oracle_access(void* h, uint32_t* out) {
    GhostGrid& gg = ((Handle*)h)->s.gg;
    std::memcpy(out, gg.access.data(), gg.access.size() * sizeof(uint32_t));
}

int oracle_last_error(void* h, long* ij, char* msg, int len) {
    Solver& s = ((Handle*)h)->s;
    ij[0] = s.err_i; ij[1] = s.err_j;
    if (msg && len > 0) { std::strncpy(msg, s.err_msg.c_str(), len - 1); msg[len - 1] = 0; }
    return s.err_code;
}

// l() on the current state/time; rhs_out nx*ny*6 (may be null); ghost_out n_ghosts*6 (may be null)
int oracle_l(void* h, double* rhs_out, double* ghost_out) {
    Solver& s = ((Handle*)h)->s;
    try {
        s.l(s.f.value.data(), s.f.time);
    } catch (OracleError& e) { set_err((Handle*)h, e); return e.code; }
    if (rhs_out) std::memcpy(rhs_out, s.rhs.data(), s.rhs.size() * sizeof(State));
    if (ghost_out) std::memcpy(ghost_out, s.gg.values.data(), s.gg.values.size() * sizeof(State));
    return 0;
}

// J_l(u) du of l() at the current state and time (forward mode, jvp.hpp):
// rhs/drhs nx*ny*6, ghost/dghost n_ghosts*6 (any may be null); duinf6: the
// direction of every FarField state; domega2: directions of omega_ei, omega_er.
int oracle_l_jvp(void* h, const double* du, const double* duinf6, const double* domega2, double* rhs,
                 double* drhs, double* ghost, double* dghost) {
    Solver& s = ((Handle*)h)->s;
    Tangent tg;
    tg.du = du;
    if (duinf6) for (int c = 0; c < 6; ++c) tg.duinf[c] = duinf6[c];
    if (domega2) { tg.domega_ei = domega2[0]; tg.domega_er = domega2[1]; }
    std::vector<StateT<Dual>> r, g;
    try { l_t<Dual>(s, tg, r, g); } catch (OracleError& e) { set_err((Handle*)h, e); return e.code; }
    for (size_t l = 0; l < r.size(); ++l)
        for (int c = 0; c < 6; ++c) {
            if (rhs) rhs[6 * l + c] = r[l][c].v;
            if (drhs) drhs[6 * l + c] = r[l][c].d;
        }
    for (size_t q = 0; q < g.size(); ++q)
        for (int c = 0; c < 6; ++c) {
            if (ghost) ghost[6 * q + c] = g[q][c].v;
            if (dghost) dghost[6 * q + c] = g[q][c].d;
        }
    return 0;
}

// double instantiation of the same templates (checks them against oracle_l)
int oracle_l_t(void* h, double* rhs, double* ghost) {
    Solver& s = ((Handle*)h)->s;
    Tangent tg;
    std::vector<StateT<double>> r, g;
    try { l_t<double>(s, tg, r, g); } catch (OracleError& e) { set_err((Handle*)h, e); return e.code; }
    if (rhs) std::memcpy(rhs, r.data(), r.size() * sizeof(State));
    if (ghost) std::memcpy(ghost, g.data(), g.size() * sizeof(State));
    return 0;
}

int oracle_rk3(void* h, double dt) {
    Solver& s = ((Handle*)h)->s;
    try { s.rk3_ssp(dt); } catch (OracleError& e) { set_err((Handle*)h, e); return e.code; }
    return 0;
}

double oracle_global_dt(void* h) { return ((Handle*)h)->s.calc_global_dt(); }

// main.rs:459-477 time loop without output clipping: dt = cfl_factor * dt_cfl
int oracle_run(void* h, long nsteps, double cfl_factor, double* dts_out) {
    Solver& s = ((Handle*)h)->s;
    for (long n = 0; n < nsteps; ++n) {
        double dt_cfl = s.calc_global_dt();
        double dt = cfl_factor * dt_cfl;
        if (dts_out) dts_out[n] = dt;
        if (!(dt > 0.0)) {
            s.err_code = ERR_NONPHYSICAL; s.err_msg = "non-positive dt"; return s.err_code;
        }
        int rc = oracle_rk3(h, dt);
        if (rc) return rc;
    }
    return 0;
}

// ---- known-answer helpers (pointwise functions of the reference)
void oracle_weno5(const double* u5, double* out) { *out = weno5(u5[0], u5[1], u5[2], u5[3], u5[4], 1e-12); }
void oracle_derived(const double* s6, const double* params, double* out11) {
    Params P; params_from(params, P);
    State s{s6[0], s6[1], s6[2], s6[3], s6[4], s6[5]};
    Derived d = derived_from_state(s, P);
    double v[11] = {d.u, d.v, d.e_e, d.e_i, d.e_r, d.pe, d.pi, d.pr, d.te, d.ti, d.tr};
    std::memcpy(out11, v, sizeof(v));
}
void oracle_flux(const double* s6, int dir, const double* params, double* out6) {
    Params P; params_from(params, P);
    State s{s6[0], s6[1], s6[2], s6[3], s6[4], s6[5]};
    State f = flux_from_derived(s, derived_from_state(s, P), (Dir)dir);
    for (int k = 0; k < 6; ++k) out6[k] = f[k];
}
void oracle_build_lr(const double* s1, const double* s2, int dir, const double* params, double* L36, double* R36,
                     double* lam6) {
    Params P; params_from(params, P);
    State a{s1[0], s1[1], s1[2], s1[3], s1[4], s1[5]}, b{s2[0], s2[1], s2[2], s2[3], s2[4], s2[5]};
    Derived da = derived_from_state(a, P), db = derived_from_state(b, P);
    double L[6][6], R[6][6];
    build_l_plain(a, b, da, db, (Dir)dir, P, L);
    build_r_plain(a, b, da, db, (Dir)dir, P, lam6, R);
    std::memcpy(L36, L, sizeof(L)); std::memcpy(R36, R, sizeof(R));
}
void oracle_reconstruction(const double* pts36, int dir, int recon, const double* params, double* out6) {
    Params P; params_from(params, P);
    State st[6]; Derived d[6];
    for (int i = 0; i < 6; ++i) {
        for (int k = 0; k < 6; ++k) st[i][k] = pts36[6 * i + k];
        d[i] = derived_from_state(st[i], P);
    }
    State r = reconstruction_fast(st, d, (Dir)dir, recon != 0, P);
    for (int k = 0; k < 6; ++k) out6[k] = r[k];
}
void oracle_noncon(const double* pts54, double ds, int dir, const double* params, double* out6) {
    Params P; params_from(params, P);
    Derived d[9];
    for (int i = 0; i < 9; ++i) {
        State s{pts54[6 * i], pts54[6 * i + 1], pts54[6 * i + 2], pts54[6 * i + 3], pts54[6 * i + 4], pts54[6 * i + 5]};
        d[i] = derived_from_state(s, P);
    }
    State r = nonconservative_pre(d, ds, (Dir)dir);
    for (int k = 0; k < 6; ++k) out6[k] = r[k];
}
void oracle_diffusion(const double* pts36, const double* params, double* out6) {
    Params P; params_from(params, P);
    Derived d[6];
    for (int i = 0; i < 6; ++i) {
        State s{pts36[6 * i], pts36[6 * i + 1], pts36[6 * i + 2], pts36[6 * i + 3], pts36[6 * i + 4], pts36[6 * i + 5]};
        d[i] = derived_from_state(s, P);
    }
    State r = diffusion_from_derived(d, P);
    for (int k = 0; k < 6; ++k) out6[k] = r[k];
}
void oracle_source(const double* s6, const double* params, double* out6) {
    Params P; params_from(params, P);
    State s{s6[0], s6[1], s6[2], s6[3], s6[4], s6[5]};
    State r = source(s, P);
    for (int k = 0; k < 6; ++k) out6[k] = r[k];
}
double oracle_local_dt(const double* s6, double dx, double dy, const double* params) {
    Params P; params_from(params, P);
    State s{s6[0], s6[1], s6[2], s6[3], s6[4], s6[5]};
    return get_local_dt(s, dx, dy, P);
}
double oracle_sixth_derivative(const double* q6, double dx) {
    return sixth_order_derivative(q6[0], q6[1], q6[2], q6[3], q6[4], q6[5], dx);
}
// least-squares fit (bc1.rs:1215-1254) and k-th x derivative (bc1.rs:1268-1304)
void oracle_fit_poly(const double* xyz, int n, int degree, double* coef_out) {
    std::vector<std::array<double, 3>> data(n);
    for (int k = 0; k < n; ++k) data[k] = {xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
    std::vector<double> c = fit_polynomial_surface(data, degree);
    for (size_t k = 0; k < c.size(); ++k) coef_out[k] = c[k];
}
double oracle_x_derivative(const double* coef, int degree, int k) {
    std::vector<double> c(coef, coef + (degree + 1) * (degree + 2) / 2);
    return x_derivative_at_origin(c, degree, k);
}
double oracle_smooth_indicator(const double* coef, int r, double h) {
    std::vector<double> c(coef, coef + (r + 1) * (r + 2) / 2);
    return smooth_indicator(c, r, h);
}
// E_r extraction for a projection on the handle's field (bc1.rs:1374-1485)
int oracle_extractor(void* h, const double* proj5, int r, int32_t* out) {
    Field& f = ((Handle*)h)->s.f;
    Projection p{{proj5[0], proj5[1]}, {proj5[2], proj5[3]}, proj5[4]};
    try {
        auto e = weno_stencil_extractor_indices(p, f, r);
        for (size_t k = 0; k < e.size(); ++k) { out[2 * k] = (int32_t)e[k].first; out[2 * k + 1] = (int32_t)e[k].second; }
        return (int)e.size();
    } catch (OracleError& e) { return -e.code; }
}
// projection of a grid point on the outer polygon (geometry.rs:121-138)
void oracle_project_outer(void* h, double x, double y, double* proj5) {
    Field& f = ((Handle*)h)->s.f;
    Projection p = project_polygon(f.outer, {x, y});
    proj5[0] = p.point.x; proj5[1] = p.point.y; proj5[2] = p.normal.x; proj5[3] = p.normal.y; proj5[4] = p.distance;
}
// single ghost value with the fast path, for a ghost index of the handle's grid
int oracle_ghost_value(void* h, long id, double* out6) {
    Solver& s = ((Handle*)h)->s;
    try {
        State r = set_ghost_point_value(s.gg.info[id], s.f, s.f.value.data(), s.f.time, s.gg, s.P);
        for (int k = 0; k < 6; ++k) out6[k] = r[k];
        return 0;
    } catch (OracleError& e) { return e.code; }
}
// V^(k) (k = 0..4, 6 characteristic components) of a heavy ghost: bc1.rs:193-255
int oracle_ghost_extrapolation(void* h, long id, double* v30) {
    Solver& s = ((Handle*)h)->s;
    const GhostInfo& g = s.gg.info[id];
    if (g.pre < 0) return -1;
    const GhostBC& pre = s.gg.pre[g.pre];
    double L[6][6], R[6][6], lam[6], v[5][6];
    build_local_plain(g.project.normal, s.f.value[s.f.linear_index(pre.nearest_i, pre.nearest_j)], s.P, L, R, lam);
    weno_extrapolation_all(L, pre, s.f.value.data(), s.P, v);
    std::memcpy(v30, v, sizeof(v));
    return 0;
}
// The two ILW systems of Wall ghost `id` as the ghost update hands them to
// solve6 (bc1.rs:691-740; the second is formed at the first one's solution),
// row-major; returns -1 for a ghost that is not a Wall ghost, 1 when the
// first system is singular, 0 otherwise.
int oracle_wall_systems(void* h, long id, double* A0, double* b0, double* A1, double* b1) {
    Solver& s = ((Handle*)h)->s;
    const GhostInfo& g = s.gg.info[id];
    if (g.pre < 0) return -1;
    const BC& bc = (g.boundary == OUTER ? s.f.bc_outer : s.f.bc_inner)[g.side_id];
    if (bc.kind != BC_WALL) return -1;
    const GhostBC& pre = s.gg.pre[g.pre];
    double L[6][6], R[6][6], lam[6], v[5][6];
    build_local_plain(g.project.normal, s.f.value[s.f.linear_index(pre.nearest_i, pre.nearest_j)], s.P, L, R, lam);
    weno_extrapolation_all(L, pre, s.f.value.data(), s.P, v);
    double M0[6][6], r0[6], M1[6][6], r1[6];
    wall_system0(L, v, M0, r0);
    std::memcpy(A0, M0, sizeof(M0));
    std::memcpy(b0, r0, sizeof(r0));
    if (!solve6(M0, r0)) return 1;
    wall_system1(L, v, r0, s.P, M1, r1);
    std::memcpy(A1, M1, sizeof(M1));
    std::memcpy(b1, r1, sizeof(r1));
    return 0;
}
// bc1.rs:467-469 solve6 on one system (row-major A, right-hand side b):
// x = A^-1 b; returns 0, or 1 when the LU factorisation meets a zero pivot
int oracle_solve6(const double* A36, const double* b6, double* x6) {
    double A[6][6], b[6];
    std::memcpy(A, A36, sizeof(A));
    std::memcpy(b, b6, sizeof(b));
    if (!solve6(A, b)) return 1;
    std::memcpy(x6, b, sizeof(b));
    return 0;
}
// weno.rs:599-679 Stencil6::reconstruction (the ndarray variant)
void oracle_reconstruction_slow(const double* pts36, int dir, int recon, const double* params, double* out6) {
    Params P;
    params_from(params, P);
    State pts[6];
    for (int i = 0; i < 6; ++i)
        for (int k = 0; k < 6; ++k) pts[i][k] = pts36[6 * i + k];
    State r = reconstruction_slow(pts, (Dir)dir, recon != 0, P);
    for (int k = 0; k < 6; ++k) out6[k] = r[k];
}
// The projection and side main.rs:567-596 give grid point (i, j) on the outer
// polygon: raw projection, BC-priority side, arc override or side geometry.
int oracle_ghost_probe(void* h, long i, long j, double* proj5) {
    const Field& f = ((Handle*)h)->s.f;
    Point p{f.grid.x(i), f.grid.y(j)};
    Projection raw = project_polygon(f.outer, p);
    size_t side = select_boundary_side(raw.point, f.outer, f.bc_outer);
    Projection pr;
    if (const CircularArc* arc = f.arc_for_side(OUTER, side)) {
        pr = arc->project(p);
    } else {
        Vec2 n = f.outer.outward_normal_of_side(side);
        double dx = p.x - raw.point.x, dy = p.y - raw.point.y;
        pr = {raw.point, n, dx * n.x + dy * n.y};
    }
    proj5[0] = pr.point.x; proj5[1] = pr.point.y; proj5[2] = pr.normal.x; proj5[3] = pr.normal.y;
    proj5[4] = pr.distance;
    return (int)side;
}
// set_ghost_point_value (bc1.rs:609-928) at grid point (i, j) with a given
// projection, boundary and side, on the handle's current state and time.
// mode 0: the precomputed path (precompute_ghost_bc for this projection,
// bc1.rs:108-188, then weno_extrapolation_pre); mode 1: the per-call path
// (bc1.rs:345-421); mode 2: the per-call path with the precomputed path's
// r = 0 smoothness indicator (2 h^2 v^2).
int oracle_ghost_value_at(void* h, long i, long j, const double* proj5, int boundary, int side, int mode,
                          double* out6) {
    Solver& s = ((Handle*)h)->s;
    const Field& f = s.f;
    GhostInfo g;
    g.i = i; g.j = j;
    g.project = {{proj5[0], proj5[1]}, {proj5[2], proj5[3]}, proj5[4]};
    g.boundary = (BoundaryKind)boundary;
    g.side_id = (size_t)side;
    find_nearest_grid_point(g.project, f, g.nearest_i, g.nearest_j);
    const BC& bc = (g.boundary == OUTER ? f.bc_outer : f.bc_inner)[g.side_id];
    try {
        State r;
        if (bc.kind != BC_WALL && bc.kind != BC_OUTFLOW && bc.kind != BC_FAR_FIELD) {
            r = set_ghost_point_value(g, f, f.value.data(), f.time, s.gg, s.P);
        } else {
            double L[6][6], R[6][6], lam[6], v[5][6];
            if (mode == 0) {
                double hh = std::sqrt(f.grid.dx * f.grid.dy);
                Matrix forms[5];
                for (int q = 0; q < 5; ++q) forms[q] = beta_quadratic_form(q, hh);
                GhostBC pre;
                precompute_ghost_bc(g.project, f, forms, pre);
                build_local_plain(g.project.normal, f.value[f.linear_index(pre.nearest_i, pre.nearest_j)], s.P, L, R,
                                  lam);
                weno_extrapolation_all(L, pre, f.value.data(), s.P, v);
            } else {
                build_local_plain(g.project.normal, f.value[f.linear_index(g.nearest_i, g.nearest_j)], s.P, L, R,
                                  lam);
                for (int k = 0; k < 5; ++k)
                    weno_extrapolation_slow(g.project, f, f.value.data(), s.P, k, mode == 2, v[k]);
            }
            r = ghost_from_extrapolation(bc, g.project, L, R, lam, v, s.P, i, j);
        }
        for (int k = 0; k < 6; ++k) out6[k] = r[k];
        return 0;
    } catch (OracleError& e) { return e.code; }
}
long oracle_ghost_id(void* h, long i, long j) {
    GhostGrid& gg = ((Handle*)h)->s.gg;
    auto it = gg.lookup.find({i, j});
    return it == gg.lookup.end() ? -1 : (long)it->second;
}

// arc description for the cylinder (three points used to build it)
void oracle_arc(void* h, int which, double* out) {
    Field& f = ((Handle*)h)->s.f;
    const ArcOverride& a = f.outer_arcs[which];
    out[0] = (double)a.side_start; out[1] = (double)a.side_end;
    out[2] = a.arc.center.x; out[3] = a.arc.center.y; out[4] = a.arc.radius;
    out[5] = a.arc.theta_start; out[6] = a.arc.sweep; out[7] = a.arc.fluid;
}
void oracle_circle_from_three(const double* pts6, int fluid, double* out5) {
    CircularArc a = CircularArc::from_three_points({pts6[0], pts6[1]}, {pts6[2], pts6[3]}, {pts6[4], pts6[5]},
                                                   (FluidSide)fluid);
    out5[0] = a.center.x; out5[1] = a.center.y; out5[2] = a.radius; out5[3] = a.theta_start; out5[4] = a.sweep;
}
void oracle_arc_project(const double* arc5, int fluid, double x, double y, double* proj5) {
    CircularArc a{{arc5[0], arc5[1]}, arc5[2], arc5[3], arc5[4], (FluidSide)fluid};
    Projection p = a.project({x, y});
    proj5[0] = p.point.x; proj5[1] = p.point.y; proj5[2] = p.normal.x; proj5[3] = p.normal.y; proj5[4] = p.distance;
}
int oracle_arc_contains(const double* arc5, int fluid, double theta) {
    CircularArc a{{arc5[0], arc5[1]}, arc5[2], arc5[3], arc5[4], (FluidSide)fluid};
    return a.contains_angle(theta) ? 1 : 0;
}

} // extern "C"
