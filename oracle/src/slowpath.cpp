// ORACLE — test infrastructure only (see physics.hpp).
// The reference's per-call ("slow") variants of two hot-path operations, which
// its own tests hold the hot path against:
//   * weno.rs:599-679 Stencil6::reconstruction: ndarray L and R
//     (weno.rs:15-26 build_l, 467-481 build_r_roe_ave), State::flux
//     (state.rs:37-117) and con2char (weno.rs:550-565) in place of
//     reconstruction_fast's Derived-based flux and l_dot
//     (main.rs:514-545 reconstruction_fast_matches_reconstruction);
//   * bc1.rs:345-421 weno_extrapolation with bc1.rs:1557-1579
//     weno_data_preprocess and bc1.rs:1039-1049 poly_regression: the E_r
//     least-squares fit of every characteristic component redone per call, the
//     path of set_ghost_point_value(.., None) (main.rs:548-613
//     ghost_bc_fast_matches_slow).
// The least-squares fit here is a Householder QR of the monomial matrix with
// its columns scaled by h^-degree, not nalgebra's truncated SVD solve: both
// give the unique least-squares solution when no singular value falls under
// the 1e-12 cut, and the arithmetic is independent of the builder's SVD.
#include "model.hpp"
#include <cmath>

namespace oracle {

// state.rs:37-45 pressure_tot / 47-54 pressure_spilit / 87-117 State::flux
static State state_flux(const State& s, Dir dir, const Params& P) {
    double u = s.mx / s.rho, v = s.my / s.rho;
    double pe = (P.gamma_e - 1.0) * (s.ee - s.rho * (sq(u) + sq(v)) / 6.0);
    double pi = (P.gamma_i - 1.0) * (s.ei - s.rho * (sq(u) + sq(v)) / 6.0);
    double pr = (P.gamma_r - 1.0) * (s.er - s.rho * (sq(u) + sq(v)) / 6.0);
    double p = pe + pi + pr;
    double rho = s.rho;
    if (dir == DIR_X) return {rho * u, rho * u * u + p, rho * u * v, (s.ee + pe) * u, (s.ei + pi) * u, (s.er + pr) * u};
    return {rho * v, rho * u * v, rho * v * v + p, (s.ee + pe) * v, (s.ei + pi) * v, (s.er + pr) * v};
}

// ndarray Array2::dot(Array1) without BLAS: each row a sequential sum from 0.0
static void nd_matvec(const double M[6][6], const double x[6], double out[6]) {
    for (int i = 0; i < 6; ++i) {
        double acc = 0.0;
        for (int j = 0; j < 6; ++j) acc = acc + M[i][j] * x[j];
        out[i] = acc;
    }
}

// weno.rs:599-679
State reconstruction_slow(const State pts[6], Dir dir, bool recon_type, const Params& P) {
    Derived d3 = derived_from_state(pts[3], P), d2 = derived_from_state(pts[2], P);
    double L[6][6], R[6][6], lam[6];
    build_l_plain(pts[3], pts[2], d3, d2, dir, P, L);
    build_r_plain(pts[3], pts[2], d3, d2, dir, P, lam, R);
    double fl[6][6], sl[6][6];
    for (int i = 0; i < 6; ++i) {
        State f = state_flux(pts[i], dir, P);
        double fv[6] = {f.rho, f.mx, f.my, f.ee, f.ei, f.er};
        double sv[6] = {pts[i].rho, pts[i].mx, pts[i].my, pts[i].ee, pts[i].ei, pts[i].er};
        if (recon_type) {
            nd_matvec(L, fv, fl[i]);
            nd_matvec(L, sv, sl[i]);
        } else {
            for (int c = 0; c < 6; ++c) { fl[i][c] = fv[c]; sl[i][c] = sv[c]; }
        }
    }
    double a[6];
    for (int c = 0; c < 6; ++c) a[c] = std::fabs(lam[c]);
    double fp[6][6], fm[6][6]; // [component][point]
    for (int i = 0; i < 6; ++i)
        for (int c = 0; c < 6; ++c) {
            fp[c][i] = 0.5 * (fl[i][c] + a[c] * sl[i][c]);
            fm[c][i] = 0.5 * (fl[i][c] - a[c] * sl[i][c]);
        }
    double flux[6];
    for (int c = 0; c < 6; ++c) {
        double plus = weno5(fp[c][0], fp[c][1], fp[c][2], fp[c][3], fp[c][4], P.eps);
        double minus = weno5(fm[c][5], fm[c][4], fm[c][3], fm[c][2], fm[c][1], P.eps);
        flux[c] = plus + minus;
    }
    double out[6];
    nd_matvec(R, flux, out);
    return {out[0], out[1], out[2], out[3], out[4], out[5]};
}

// Least-squares polynomial fit of bc1.rs:1215-1254 (coefficients in the
// reference's order: total degree t = 0..r, then x^i y^(t-i), i = 0..t):
// Householder QR of A D (D = diag(h^-degree)), back substitution, c = D y.
static void fit_poly_qr(const double xy[25][2], const double* val, int m, int r, double h, double* coef) {
    int nt = (r + 1) * (r + 2) / 2;
    double A[25][15], b[25], scale[15];
    for (int row = 0; row < m; ++row) {
        int col = 0;
        for (int t = 0; t <= r; ++t)
            for (int i = 0; i <= t; ++i) {
                int j = t - i;
                A[row][col] = powi(xy[row][0], i) * powi(xy[row][1], j);
                scale[col] = 1.0 / powi(h, t);
                col++;
            }
        b[row] = val[row];
    }
    for (int row = 0; row < m; ++row)
        for (int col = 0; col < nt; ++col) A[row][col] *= scale[col];
    for (int k = 0; k < nt; ++k) {
        double norm = 0.0;
        for (int i = k; i < m; ++i) norm += A[i][k] * A[i][k];
        norm = std::sqrt(norm);
        if (norm == 0.0) throw OracleError(ERR_STENCIL_FIT, "rank-deficient least-squares fit");
        double alpha = A[k][k] > 0 ? -norm : norm;
        double vk[25];
        for (int i = k; i < m; ++i) vk[i] = A[i][k];
        vk[k] -= alpha;
        double vnorm2 = 0.0;
        for (int i = k; i < m; ++i) vnorm2 += vk[i] * vk[i];
        for (int col = k; col < nt; ++col) {
            double dot = 0.0;
            for (int i = k; i < m; ++i) dot += vk[i] * A[i][col];
            double f = 2.0 * dot / vnorm2;
            for (int i = k; i < m; ++i) A[i][col] -= f * vk[i];
        }
        double dot = 0.0;
        for (int i = k; i < m; ++i) dot += vk[i] * b[i];
        double f = 2.0 * dot / vnorm2;
        for (int i = k; i < m; ++i) b[i] -= f * vk[i];
    }
    for (int k = nt - 1; k >= 0; --k) {
        double acc = b[k];
        for (int col = k + 1; col < nt; ++col) acc -= A[k][col] * coef[col];
        coef[k] = acc / A[k][k];
    }
    for (int k = 0; k < nt; ++k) coef[k] *= scale[k];
}

// bc1.rs:345-421 weno_extrapolation for derivative order k, every E_r and
// every characteristic component fitted afresh. beta0_as_fast: the r = 0
// smoothness indicator as the precomputed path has it (bc1.rs:167-168 and
// 222-231: S_0 = 2 h^2 used as a quadratic form, 2 h^2 v^2) instead of the
// constant 2 h^2 that smooth_indicator returns for r = 0 (bc1.rs:1087-1089).
void weno_extrapolation_slow(const Projection& pr, const Field& f, const State* val, const Params& P, int k,
                             bool beta0_as_fast, double out[6]) {
    double h = std::sqrt(f.grid.dx * f.grid.dy);
    double vk[5][6], beta[5][6];
    for (int r = 0; r < 5; ++r) {
        std::vector<std::pair<long, long>> idx = weno_stencil_extractor_indices(pr, f, r);
        int m = (int)idx.size();
        // bc1.rs:1557-1579 weno_data_preprocess: L at the nearest node, each
        // stencil state rotated to (n, t) and projected, coordinates local
        long ni, nj;
        find_nearest_grid_point(pr, f, ni, nj);
        double L[6][6], R[6][6], lam[6];
        build_local_plain(pr.normal, val[f.linear_index(ni, nj)], P, L, R, lam);
        double xy[25][2], cv[6][25];
        for (int a = 0; a < m; ++a) {
            const State& s = val[f.linear_index(idx[a].first, idx[a].second)];
            Vec2 n = pr.normal;
            double u6[6] = {s.rho, s.mx * n.x + s.my * n.y, -s.mx * n.y + s.my * n.x, s.ee, s.ei, s.er};
            double vm[6];
            nd_matvec(L, u6, vm);
            for (int c = 0; c < 6; ++c) cv[c][a] = vm[c];
            pr.global2local({f.grid.x(idx[a].first), f.grid.y(idx[a].second)}, xy[a][0], xy[a][1]);
        }
        // bc1.rs:1039-1049 poly_regression per component
        for (int c = 0; c < 6; ++c) {
            std::vector<double> coef((r + 1) * (r + 2) / 2);
            fit_poly_qr(xy, cv[c], m, r, h, coef.data());
            double b = smooth_indicator(coef, r, h);
            if (r == 0 && beta0_as_fast) b = 0.0 + cv[c][0] * (0.0 + b * cv[c][0]);
            beta[r][c] = b;
            vk[r][c] = x_derivative_at_origin(coef, r, k);
        }
    }
    double d0 = 2.0 * powi(h, 4), d1 = 2.0 * powi(h, 3), d2 = 2.0 * powi(h, 2), d3 = 2.0 * h;
    double d[5] = {d0, d1, d2, d3, 1.0 - d0 - d1 - d2 - d3};
    for (int c = 0; c < 6; ++c) {
        double alpha[5], alpha_sum = 0.0;
        for (int r = 0; r < 5; ++r) {
            alpha[r] = d[r] / powf_ref(P.eps + beta[r][c], P.weno_q);
            alpha_sum += alpha[r];
        }
        double res = 0.0;
        for (int r = 0; r < 5; ++r) res += (alpha[r] / alpha_sum) * vk[r][c];
        out[c] = res;
    }
}

} // namespace oracle
