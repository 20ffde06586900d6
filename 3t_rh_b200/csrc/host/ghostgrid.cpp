// Host side of the rh3t library: the mirror of the reference's Field::new
// (field1.rs:95-136) and GhostGrid::build (ghost.rs:50-118) that produces the
// tables rh3t_create() uploads (include/rh3t.h rh3t_geom_*).
//
// Ghost discovery, projection, side selection and the E_r stencils must be
// bit-identical to the reference, so every floating-point expression below
// keeps the reference's operation order (compiled with -ffp-contract=off).
// The least-squares pseudo-inverses (nalgebra SVD in the reference,
// bc1.rs:162-165) are a one-sided Jacobi SVD here; above the absolute 1e-12
// singular-value cut the pseudo-inverse is unique, so the tables agree with
// the reference's to rounding.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../../include/rh3t.h"
#include "lsbuild.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Pt { double x, y; };

struct Poly {
    std::vector<Pt> p;
    int fluid_side = 0; // 0 Inside, 1 Outside
    double area2 = 0.0;

    void finish() {
        size_t n = p.size();
        double a2 = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const Pt &a = p[i], &b = p[(i + 1) % n];
            a2 += a.x * b.y - b.x * a.y; // geometry.rs:165-178
        }
        area2 = a2;
    }
    // geometry.rs:254-278
    bool is_fluid(double px, double py) const {
        size_t n = p.size();
        if (n < 3) return false;
        bool inside = false;
        for (size_t i = 0; i < n; ++i) {
            const Pt &a = p[i], &b = p[(i + 1) % n];
            if ((a.y > py) != (b.y > py)) {
                double xi = a.x + (py - a.y) * (b.x - a.x) / (b.y - a.y);
                if (px < xi) inside = !inside;
            }
        }
        return fluid_side == 0 ? inside : !inside;
    }
    // geometry.rs:181-202
    static Pt seg_closest(double px, double py, const Pt& a, const Pt& b) {
        double abx = b.x - a.x, aby = b.y - a.y, apx = px - a.x, apy = py - a.y;
        double ab2 = abx * abx + aby * aby;
        if (ab2 <= 1e-30) return a;
        double t = (apx * abx + apy * aby) / ab2;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        return {a.x + t * abx, a.y + t * aby};
    }
    // index of the first side whose closest point is strictly nearest (geometry.rs:280-302, 332-347)
    size_t nearest_side(double px, double py, Pt& best_pt) const {
        size_t best = 0;
        double bd = INFINITY;
        best_pt = p[0];
        for (size_t i = 0; i < p.size(); ++i) {
            Pt c = seg_closest(px, py, p[i], p[(i + 1) % p.size()]);
            double dx = px - c.x, dy = py - c.y;
            double d2 = dx * dx + dy * dy;
            if (d2 < bd) { bd = d2; best = i; best_pt = c; }
        }
        return best;
    }
    // geometry.rs:212-250 (and the same left/right choice in 304-420)
    bool side_normal(size_t s, double& nx, double& ny) const {
        const Pt &a = p[s], &b = p[(s + 1) % p.size()];
        double tx = b.x - a.x, ty = b.y - a.y;
        double len = std::hypot(tx, ty);
        if (!(len > 1.0e-14)) return false;
        bool ccw = area2 > 0.0;
        bool right = fluid_side == 0 ? ccw : !ccw;
        if (right) { nx = ty / len; ny = -tx / len; }
        else { nx = -ty / len; ny = tx / len; }
        return true;
    }
};

constexpr double TWO_PI = 2.0 * 3.14159265358979323846;
inline double rem_2pi(double th) { // Rust f64::rem_euclid(2*PI)
    double r = std::fmod(th, TWO_PI);
    return r < 0.0 ? r + TWO_PI : r;
}

struct Arc {
    int boundary, side_start, side_end, fluid_side;
    double cx, cy, radius, th0, sweep;

    // geometry.rs:492-549
    bool from_three(const double s[2], const double m[2], const double e[2]) {
        double x1 = s[0], y1 = s[1], x2 = m[0], y2 = m[1], x3 = e[0], y3 = e[1];
        double d = 2.0 * (x1 * (y2 - y3) + x2 * (y3 - y1) + x3 * (y1 - y2));
        double chord = std::fmax(0.0, std::hypot(x1 - x2, y1 - y2));
        chord = std::fmax(chord, std::hypot(x2 - x3, y2 - y3));
        chord = std::fmax(chord, std::hypot(x1 - x3, y1 - y3));
        chord = std::fmax(chord, 1.0);
        if (!(std::fabs(d) > 1e-12 * chord * chord)) return false;
        double r1 = x1 * x1 + y1 * y1, r2 = x2 * x2 + y2 * y2, r3 = x3 * x3 + y3 * y3;
        cx = (r1 * (y2 - y3) + r2 * (y3 - y1) + r3 * (y1 - y2)) / d;
        cy = (r1 * (x3 - x2) + r2 * (x1 - x3) + r3 * (x2 - x1)) / d;
        radius = std::hypot(x1 - cx, y1 - cy);
        double ts = std::atan2(y1 - cy, x1 - cx), tm = std::atan2(y2 - cy, x2 - cx), te = std::atan2(y3 - cy, x3 - cx);
        double ccw = rem_2pi(te - ts), to_mid = rem_2pi(tm - ts);
        sweep = to_mid <= ccw + 1e-12 ? ccw : -rem_2pi(ts - te);
        th0 = ts;
        return radius > 0.0;
    }
    bool contains(double th) const {
        return sweep > 0.0 ? rem_2pi(th - th0) <= sweep + 1e-12 : rem_2pi(th0 - th) <= -sweep + 1e-12;
    }
    // geometry.rs:578-653
    bool project(double px, double py, double out[5]) const {
        double rx = px - cx, ry = py - cy;
        double rn = std::hypot(rx, ry);
        double qx, qy;
        bool done = false;
        if (rn > 1e-12) {
            double th = std::atan2(ry, rx);
            if (contains(th)) {
                double s = radius / rn;
                qx = cx + s * rx; qy = cy + s * ry;
                done = true;
            }
        }
        if (!done) {
            double sx = cx + radius * std::cos(th0), sy = cy + radius * std::sin(th0);
            double te = th0 + sweep;
            double ex = cx + radius * std::cos(te), ey = cy + radius * std::sin(te);
            double d2s = (px - sx) * (px - sx) + (py - sy) * (py - sy);
            double d2e = (px - ex) * (px - ex) + (py - ey) * (py - ey);
            if (d2s <= d2e) { qx = sx; qy = sy; } else { qx = ex; qy = ey; }
        }
        double dx = qx - cx, dy = qy - cy;
        double nrm = std::hypot(dx, dy);
        if (!(nrm > 1e-14)) return false;
        double nx = dx / nrm, ny = dy / nrm;
        if (fluid_side == 1) { nx = -nx; ny = -ny; }
        out[0] = qx; out[1] = qy; out[2] = nx; out[3] = ny;
        out[4] = (px - qx) * nx + (py - qy) * ny;
        return true;
    }
};

int priority(int kind) { // ghost.rs:285-305
    switch (kind) {
    case RH3T_BC_WALL: return 100;
    case RH3T_BC_REFLECTIVE_WALL: return 90;
    case RH3T_BC_CONSTANT: case RH3T_BC_TIME_DEPENDENT: return 70;
    case RH3T_BC_FAR_FIELD: return 20;
    case RH3T_BC_OUTFLOW: return 10;
    case RH3T_BC_ZEROTH_ORDER: return 5;
    default: return 0;
    }
}

inline bool on_segment(double px, double py, const Pt& a, const Pt& b, double eps) { // geometry.rs:12-33
    double abx = b.x - a.x, aby = b.y - a.y, apx = px - a.x, apy = py - a.y;
    if (std::fabs(abx * apy - aby * apx) > eps) return false;
    return px >= std::fmin(a.x, b.x) - eps && px <= std::fmax(a.x, b.x) + eps && py >= std::fmin(a.y, b.y) - eps &&
           py <= std::fmax(a.y, b.y) + eps;
}

inline double ipow(double a, int b) { // compiler-rt __powidf2 (Rust f64::powi)
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return r;
}

// ---- smoothness-indicator quadratic forms, bc1.rs:62-85 and 1070-1196
double integ1d(int power, double h) {
    if (power % 2 == 1) return 0.0;
    double half = 0.5 * h;
    return 2.0 * ipow(half, power + 1) / (double)(power + 1);
}
double smooth_ind(const double* coef, int r, double h) {
    if (r == 0) return 2.0 * h * h;
    double beta = 0.0;
    struct Term { int i, j; double c; };
    Term terms[15];
    for (int ax = 0; ax <= r; ++ax)
        for (int ay = 0; ay <= r - ax; ++ay) {
            int order = ax + ay;
            if (order == 0) continue;
            int nt = 0, k = 0;
            for (int tot = 0; tot <= r; ++tot)
                for (int i = 0; i <= tot; ++i) {
                    int j = tot - i;
                    double aij = coef[k++];
                    if (i < ax || j < ay) continue;
                    double f = 1.0;
                    for (int m = 0; m < ax; ++m) f *= (double)(i - m);
                    for (int m = 0; m < ay; ++m) f *= (double)(j - m);
                    terms[nt++] = {i - ax, j - ay, aij * f};
                }
            double integral = 0.0;
            for (int p = 0; p < nt; ++p)
                for (int q = 0; q < nt; ++q)
                    integral += terms[p].c * terms[q].c * integ1d(terms[p].i + terms[q].i, h) *
                                integ1d(terms[p].j + terms[q].j, h);
            beta += ipow(h, 2 * (order - 1)) * integral;
        }
    return beta;
}
void quad_form(int r, double h, std::vector<double>& M) {
    int n = (r + 1) * (r + 2) / 2;
    M.assign((size_t)n * n, 0.0);
    std::vector<double> ea(n), eb(n), eab(n);
    for (int a = 0; a < n; ++a)
        for (int b = a; b < n; ++b) {
            std::fill(ea.begin(), ea.end(), 0.0);
            std::fill(eb.begin(), eb.end(), 0.0);
            ea[a] = 1.0; eb[b] = 1.0;
            for (int q = 0; q < n; ++q) eab[q] = ea[q] + eb[q];
            double v = 0.5 * (smooth_ind(eab.data(), r, h) - smooth_ind(ea.data(), r, h) - smooth_ind(eb.data(), r, h));
            M[(size_t)a * n + b] = v;
            M[(size_t)b * n + a] = v;
        }
}

// Pseudo-inverse (n x m) of a tall m x n matrix (row-major), one-sided Jacobi
// SVD, singular values <= tol dropped.
void pinv(const double* A, int m, int n, double tol, double* P) {
    double U[25 * 15], V[15 * 15];
    std::memcpy(U, A, sizeof(double) * m * n);
    for (int i = 0; i < n * n; ++i) V[i] = 0.0;
    for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 80; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double al = 0, be = 0, ga = 0;
                for (int i = 0; i < m; ++i) {
                    al += U[i * n + p] * U[i * n + p];
                    be += U[i * n + q] * U[i * n + q];
                    ga += U[i * n + p] * U[i * n + q];
                }
                if (ga == 0.0) continue;
                double rel = std::fabs(ga) / std::sqrt(al * be);
                off = std::fmax(off, rel);
                if (rel < 1e-17) continue;
                double zeta = (be - al) / (2.0 * ga);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (int i = 0; i < m; ++i) {
                    double up = U[i * n + p], uq = U[i * n + q];
                    U[i * n + p] = c * up - s * uq;
                    U[i * n + q] = s * up + c * uq;
                }
                for (int i = 0; i < n; ++i) {
                    double vp = V[i * n + p], vq = V[i * n + q];
                    V[i * n + p] = c * vp - s * vq;
                    V[i * n + q] = s * vp + c * vq;
                }
            }
        if (off < 1e-16) break;
    }
    for (int i = 0; i < n * m; ++i) P[i] = 0.0;
    for (int j = 0; j < n; ++j) {
        double sig = 0.0;
        for (int i = 0; i < m; ++i) sig += U[i * n + j] * U[i * n + j];
        sig = std::sqrt(sig);
        if (!(sig > tol)) continue;
        for (int a = 0; a < m; ++a) {
            double sc = (U[a * n + j] / sig) / sig;
            for (int k = 0; k < n; ++k) P[k * m + a] += V[k * n + j] * sc;
        }
    }
}

} // namespace

struct rh3t_geom {
    rh3t_grid G;
    rh3t_params prm;
    Poly outer, inner;
    std::vector<rh3t_bc> bc_outer, bc_inner;
    std::vector<Arc> arcs;
    std::vector<uint8_t> fluid;
    // built ghost tables (SoA, the rh3t_ghost_table layout)
    std::vector<int32_t> idx, boundary, side, pre, nearest_raw;
    std::vector<double> proj;
    std::vector<int32_t> nearest;
    std::vector<uint32_t> stencil;
    std::vector<double> s, w, d;
    std::vector<uint32_t> access;
    // build intermediates: the sorted ghost list and the ghosts with a GhostBC slot
    std::vector<std::pair<long, long>> found;
    std::vector<long> heavy;
    std::string err;

    bool in_grid(long i, long j) const { return i >= 0 && i < G.nx && j >= 0 && j < G.ny; }
    double X(long i) const { return G.x0 + (double)i * G.dx; }
    double Y(long j) const { return G.y0 + (double)j * G.dy; }
    // field1.rs:179-192
    bool in_domain(long i, long j) const {
        if (!in_grid(i, j)) {
            double px = X(i), py = Y(j);
            return outer.is_fluid(px, py) && inner.is_fluid(px, py);
        }
        return fluid[(size_t)i * G.ny + j] != 0;
    }
    const Arc* arc_for(int b, long sd) const {
        for (const Arc& a : arcs)
            if (a.boundary == b && sd >= a.side_start && sd <= a.side_end) return &a;
        return nullptr;
    }
    // bc1.rs:257-281 (initial answer (0,0), strict improvement, 9 candidates)
    void nearest_node(double p0x, double p0y, long& oi, long& oj) const {
        long i = (long)std::round((p0x - G.x0) / G.dx), j = (long)std::round((p0y - G.y0) / G.dy);
        const long c[9][2] = {{i, j}, {i - 1, j}, {i + 1, j}, {i, j - 1}, {i, j + 1},
                              {i + 1, j + 1}, {i + 1, j - 1}, {i - 1, j + 1}, {i - 1, j - 1}};
        oi = 0; oj = 0;
        double best = 1e50;
        for (auto& q : c) {
            if (!in_domain(q[0], q[1])) continue;
            double dx = X(q[0]) - p0x, dy = Y(q[1]) - p0y;
            double dis = std::sqrt(dx * dx + dy * dy);
            if (dis < best) { best = dis; oi = q[0]; oj = q[1]; }
        }
    }
    // bc1.rs:1489-1549: whole-substencil shift search, nearest shift first
    bool fit_line(bool vertical, long line, long base, long width, long* out2) const {
        long max_shift = (vertical ? G.ny : G.nx) + width;
        for (long mag = 0; mag <= max_shift; ++mag)
            for (int sgn = 0; sgn < (mag == 0 ? 1 : 2); ++sgn) {
                long start = base + (sgn == 0 ? -mag : mag);
                bool ok = true;
                for (long a = 0; a < width && ok; ++a) {
                    long i = vertical ? line : start + a, j = vertical ? start + a : line;
                    ok = in_grid(i, j) && in_domain(i, j);
                }
                if (ok) {
                    for (long a = 0; a < width; ++a) {
                        out2[2 * a] = vertical ? line : start + a;
                        out2[2 * a + 1] = vertical ? start + a : line;
                    }
                    return true;
                }
            }
        return false;
    }
    // bc1.rs:1374-1485 E_r, (r+1)^2 nodes
    bool extract(const double* pr, int r, long* out2) const {
        double p0x = pr[0], p0y = pr[1], nx = pr[2], ny = pr[3];
        long width = r + 1;
        if (std::fabs(nx) >= std::fabs(ny)) {
            if (!(std::fabs(nx) > 1.0e-14)) return false;
            double q = (p0x - G.x0) / G.dx;
            long i0 = nx > 0.0 ? (long)std::ceil(q) - 1 : (long)std::floor(q) + 1;
            i0 = std::min(std::max(i0, 0L), (long)G.nx - 1);
            long step = nx > 0.0 ? -1 : 1;
            for (long l = 0; l <= r; ++l) {
                long il = i0 + l * step;
                double t = (p0x - X(il)) / nx;
                double ys = p0y - ny * t;
                long m = (long)std::floor((ys - G.y0) / G.dy);
                if (!fit_line(true, il, m - (long)(r / 2), width, out2 + 2 * l * width)) return false;
            }
        } else {
            if (!(std::fabs(ny) > 1.0e-14)) return false;
            double q = (p0y - G.y0) / G.dy;
            long j0 = ny > 0.0 ? (long)std::ceil(q) - 1 : (long)std::floor(q) + 1;
            j0 = std::min(std::max(j0, 0L), (long)G.ny - 1);
            long step = ny > 0.0 ? -1 : 1;
            for (long l = 0; l <= r; ++l) {
                long jl = j0 + l * step;
                double t = (p0y - Y(jl)) / ny;
                double xs = p0x - nx * t;
                long m = (long)std::floor((xs - G.x0) / G.dx);
                if (!fit_line(false, jl, m - (long)(r / 2), width, out2 + 2 * l * width)) return false;
            }
        }
        return true;
    }
};

static void fill_poly(Poly& P, int n, const double* xy, int fs) {
    P.p.resize((size_t)n);
    for (int k = 0; k < n; ++k) P.p[k] = {xy[2 * k], xy[2 * k + 1]};
    P.fluid_side = fs;
    P.finish();
}

extern "C" int rh3t_geom_create(const rh3t_grid* grid, const rh3t_params* params, int32_t n_outer,
                                const double* outer_xy, int32_t outer_fluid_side, const rh3t_bc* outer_bcs,
                                int32_t n_inner, const double* inner_xy, int32_t inner_fluid_side,
                                const rh3t_bc* inner_bcs, int32_t n_arcs, const rh3t_arc* arcs, rh3t_geom** out) {
    if (!out || !grid || !params || n_outer < 2 || !outer_xy || !outer_bcs || n_inner < 0 ||
        (n_inner && (!inner_xy || !inner_bcs)) || grid->nx <= 0 || grid->ny <= 0 || !(grid->dx > 0.0) ||
        !(grid->dy > 0.0) || n_arcs < 0 || (n_arcs && !arcs))
        return RH3T_ERR_INVALID_ARGUMENT;
    // field1.rs:104-105
    if (outer_fluid_side != 0 || inner_fluid_side != 1) return RH3T_ERR_GEOMETRY;
    rh3t_geom* g = new rh3t_geom();
    g->G = *grid;
    g->prm = *params;
    fill_poly(g->outer, n_outer, outer_xy, outer_fluid_side);
    fill_poly(g->inner, n_inner, inner_xy, inner_fluid_side);
    g->bc_outer.assign(outer_bcs, outer_bcs + n_outer);
    if (n_inner) g->bc_inner.assign(inner_bcs, inner_bcs + n_inner);
    for (int k = 0; k < n_arcs; ++k) {
        Arc a;
        a.boundary = arcs[k].boundary; a.side_start = arcs[k].side_start; a.side_end = arcs[k].side_end;
        a.fluid_side = arcs[k].fluid_side;
        if (!a.from_three(arcs[k].start, arcs[k].mid, arcs[k].end)) { delete g; return RH3T_ERR_GEOMETRY; }
        g->arcs.push_back(a);
    }
    const long nx = grid->nx, ny = grid->ny;
    g->fluid.assign((size_t)nx * ny, 0);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j) {
            double px = g->X(i), py = g->Y(j);
            g->fluid[(size_t)i * ny + j] = g->outer.is_fluid(px, py) && g->inner.is_fluid(px, py);
        }
    *out = g;
    return RH3T_OK;
}

extern "C" int rh3t_geom_fluid_mask(const rh3t_geom* g, uint8_t* out) {
    if (!g || !out) return RH3T_ERR_INVALID_ARGUMENT;
    std::memcpy(out, g->fluid.data(), g->fluid.size());
    return RH3T_OK;
}

extern "C" const char* rh3t_geom_last_error(const rh3t_geom* g) { return g ? g->err.c_str() : ""; }

extern "C" void rh3t_geom_destroy(rh3t_geom* g) { delete g; }

static inline uint64_t pack_ij(long i, long j) { return ((uint64_t)(uint32_t)(int32_t)i << 32) | (uint32_t)(int32_t)j; }

namespace {

const int SOFF[6] = {0, 1, 5, 14, 30, 55}, S2OFF[6] = {0, 1, 17, 98, 354, 979}, WOFF[6] = {0, 1, 9, 36, 100, 225};

// ghost.rs:352-468: discovery, per-ghost geometry, heavy slots
int build_geometry(rh3t_geom* g) {
    const long nx = g->G.nx, ny = g->G.ny;
    // ---- discovery (ghost.rs:352-376, default offsets ghost.rs:482-493: the radius-4 cross)
    std::vector<std::pair<long, long>>& found = g->found;
    found.clear();
#pragma omp parallel
    {
        std::vector<std::pair<long, long>> loc;
#pragma omp for schedule(static) nowait
        for (long i = 0; i < nx; ++i)
            for (long j = 0; j < ny; ++j) {
                if (!g->fluid[(size_t)i * ny + j]) continue;
                for (long d = -4; d <= 4; ++d) {
                    if (d == 0) continue;
                    if (!g->in_domain(i + d, j)) loc.push_back({i + d, j});
                    if (!g->in_domain(i, j + d)) loc.push_back({i, j + d});
                }
            }
#pragma omp critical
        found.insert(found.end(), loc.begin(), loc.end());
    }
    std::sort(found.begin(), found.end());
    found.erase(std::unique(found.begin(), found.end()), found.end());
    const long ng = (long)found.size();

    // ---- per-ghost geometry (ghost.rs:378-456)
    g->idx.assign(2 * ng, 0); g->boundary.assign(ng, 0); g->side.assign(ng, 0);
    g->proj.assign(5 * ng, 0.0); g->pre.assign(ng, -1); g->nearest_raw.assign(2 * ng, 0);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (long k = 0; k < ng; ++k) {
        long i = found[k].first, j = found[k].second;
        double px = g->X(i), py = g->Y(j);
        int b = g->outer.is_fluid(px, py) ? 1 : 0;
        const Poly& P = b == 0 ? g->outer : g->inner;
        const std::vector<rh3t_bc>& bcs = b == 0 ? g->bc_outer : g->bc_inner;
        Pt p0;
        size_t raw_side = P.nearest_side(px, py, p0);
        (void)raw_side;
        long ni, nj;
        g->nearest_node(p0.x, p0.y, ni, nj);
        // ghost.rs:307-348: all sides through P0, highest BC priority, first wins ties
        long best = -1;
        int bp = -1;
        for (size_t sdx = 0; sdx < P.p.size(); ++sdx)
            if (on_segment(p0.x, p0.y, P.p[sdx], P.p[(sdx + 1) % P.p.size()], 1e-12)) {
                int pr = priority(bcs[sdx].kind);
                if (best < 0 || pr > bp) { best = (long)sdx; bp = pr; }
            }
        if (best < 0 || bcs.size() != P.p.size()) { bad |= 1; continue; }
        double out5[5];
        if (const Arc* a = g->arc_for(b, best)) {
            if (!a->project(px, py, out5)) { bad |= 2; continue; }
        } else {
            double nx_, ny_;
            if (!P.side_normal((size_t)best, nx_, ny_)) { bad |= 2; continue; }
            out5[0] = p0.x; out5[1] = p0.y; out5[2] = nx_; out5[3] = ny_;
            out5[4] = (px - p0.x) * nx_ + (py - p0.y) * ny_;
        }
        g->idx[2 * k] = (int32_t)i; g->idx[2 * k + 1] = (int32_t)j;
        g->boundary[k] = b; g->side[k] = (int32_t)best;
        g->nearest_raw[2 * k] = (int32_t)ni; g->nearest_raw[2 * k + 1] = (int32_t)nj;
        for (int q = 0; q < 5; ++q) g->proj[5 * k + q] = out5[q];
    }
    if (bad) {
        g->err = (bad & 1) ? "projection point does not lie on any polygon side" : "degenerate boundary geometry";
        return RH3T_ERR_GEOMETRY;
    }
    // ---- heavy slots (Wall / Outflow / FarField), in ghost order (ghost.rs:461-468)
    g->heavy.clear();
    for (long k = 0; k < ng; ++k) {
        int kind = (g->boundary[k] == 0 ? g->bc_outer : g->bc_inner)[g->side[k]].kind;
        if (kind == RH3T_BC_WALL || kind == RH3T_BC_OUTFLOW || kind == RH3T_BC_FAR_FIELD) {
            g->pre[k] = (int32_t)g->heavy.size();
            g->heavy.push_back(k);
        }
    }
    return RH3T_OK;
}

// mesh width h and the r = 1..4 smoothness quadratic forms (bc1.rs:62-85)
double ls_h(const rh3t_geom* g) { return std::sqrt(g->G.dx * g->G.dy); }

// nearest fluid node, the d weights and the E_r stencils of every heavy ghost
// (bc1.rs:108-160, 1374-1549); tables sized for the least-squares step
int build_stencils(rh3t_geom* g) {
    const long ny = g->G.ny;
    const long nh = (long)g->heavy.size();
    g->nearest.assign(2 * nh, 0); g->stencil.assign(55 * nh, 0u);
    g->s.assign(979 * nh, 0.0); g->w.assign(225 * nh, 0.0); g->d.assign(5 * nh, 0.0);
    const double h = ls_h(g);
    const double dd[5] = {2.0 * ipow(h, 4), 2.0 * ipow(h, 3), 2.0 * ipow(h, 2), 2.0 * h, 0.0};
    const double d4 = 1.0 - dd[0] - dd[1] - dd[2] - dd[3];
    int fit_fail = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(| : fit_fail)
    for (long q = 0; q < nh; ++q) {
        long k = g->heavy[q];
        const double* pr = &g->proj[5 * k];
        long ni, nj;
        g->nearest_node(pr[0], pr[1], ni, nj);
        g->nearest[2 * q] = (int32_t)ni; g->nearest[2 * q + 1] = (int32_t)nj;
        for (int r = 0; r < 4; ++r) g->d[5 * q + r] = dd[r];
        g->d[5 * q + 4] = d4;
        for (int r = 0; r <= 4; ++r) {
            int m = (r + 1) * (r + 1);
            long e[50];
            if (!g->extract(pr, r, e)) { fit_fail = 1; break; }
            for (int a = 0; a < m; ++a) g->stencil[55 * q + SOFF[r] + a] = (uint32_t)((size_t)e[2 * a] * ny + e[2 * a + 1]);
        }
    }
    if (fit_fail) {
        g->err = "cannot fit paper substencil inside fluid domain";
        return RH3T_ERR_STENCIL_FIT;
    }
    return RH3T_OK;
}

// pseudo-inverses, S_r and w_r of every heavy ghost on the host (bc1.rs:120-186)
void build_ls_host(rh3t_geom* g) {
    const long ny = g->G.ny;
    const long nh = (long)g->heavy.size();
    const double h = ls_h(g);
    std::vector<double> M[5];
    for (int r = 1; r <= 4; ++r) quad_form(r, h, M[r]);
#pragma omp parallel for schedule(dynamic, 8)
    for (long q = 0; q < nh; ++q) {
        const double* pr = &g->proj[5 * g->heavy[q]];
        for (int r = 0; r <= 4; ++r) {
            int m = (r + 1) * (r + 1), nt = (r + 1) * (r + 2) / 2;
            double A[25 * 15], P[15 * 25];
            for (int a = 0; a < m; ++a) {
                const uint32_t l = g->stencil[55 * q + SOFF[r] + a];
                const long ei = (long)(l / (uint32_t)ny), ej = (long)(l % (uint32_t)ny);
                double dx = g->X(ei) - pr[0], dy = g->Y(ej) - pr[1];
                double nor = pr[2] * dx + pr[3] * dy;
                double tan = -dx * pr[3] + dy * pr[2];
                int col = 0;
                for (int t = 0; t <= r; ++t)
                    for (int i2 = 0; i2 <= t; ++i2) A[a * nt + col++] = ipow(nor, i2) * ipow(tan, t - i2);
            }
            pinv(A, m, nt, 1.0e-12, P);
            double* S = &g->s[979 * q + S2OFF[r]];
            if (r == 0) {
                S[0] = 2.0 * h * h; // bc1.rs:167-168
            } else {
                const std::vector<double>& Mr = M[r];
                double T[25 * 15];
                for (int a = 0; a < m; ++a)
                    for (int cc = 0; cc < nt; ++cc) {
                        double acc = 0.0;
                        for (int kk = 0; kk < nt; ++kk) acc += P[kk * m + a] * Mr[(size_t)kk * nt + cc];
                        T[a * nt + cc] = acc;
                    }
                for (int a = 0; a < m; ++a)
                    for (int b = 0; b < m; ++b) {
                        double acc = 0.0;
                        for (int kk = 0; kk < nt; ++kk) acc += T[a * nt + kk] * P[kk * m + b];
                        S[a * m + b] = acc;
                    }
            }
            double* W = &g->w[225 * q + WOFF[r]];
            double kf = 1.0;
            for (int kk = 0; kk <= r; ++kk) {
                if (kk > 0) kf *= (double)kk;
                int col = kk * (kk + 1) / 2 + kk; // x^k column (bc1.rs:89-101)
                for (int a = 0; a < m; ++a) W[kk * m + a] = kf * P[col * m + a];
            }
        }
    }
}

// ---- access table (ghost.rs:71-107), radius-4 cross in sorted offset order
int build_access(rh3t_geom* g) {
    const long nx = g->G.nx, ny = g->G.ny;
    const std::vector<std::pair<long, long>>& found = g->found;
    const long ng = (long)found.size();
    std::unordered_map<uint64_t, uint32_t> lookup;
    lookup.reserve((size_t)ng * 2);
    for (long k = 0; k < ng; ++k) lookup[pack_ij(found[k].first, found[k].second)] = (uint32_t)k;
    long offs[17][2];
    {
        int n = 0;
        for (long di = -4; di <= 4; ++di)
            for (long dj = -4; dj <= 4; ++dj)
                if ((di == 0) != (dj == 0) || (di == 0 && dj == 0)) { offs[n][0] = di; offs[n][1] = dj; ++n; }
    }
    g->access.assign((size_t)nx * ny * 17, 0u);
    int miss = 0;
#pragma omp parallel for schedule(static) reduction(| : miss)
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j) {
            size_t l = (size_t)i * ny + j;
            if (!g->fluid[l]) continue;
            for (int k = 0; k < 17; ++k) {
                long a = i + offs[k][0], b = j + offs[k][1];
                uint32_t t;
                if (g->in_grid(a, b) && g->fluid[(size_t)a * ny + b]) t = (uint32_t)((size_t)a * ny + b);
                else {
                    auto it = lookup.find(pack_ij(a, b));
                    if (it == lookup.end()) { miss = 1; continue; }
                    t = it->second + (uint32_t)(nx * ny);
                }
                g->access[l * 17 + k] = t;
            }
        }
    if (miss) {
        g->err = "ghost referenced by a fluid cell is not cached";
        return RH3T_ERR_GEOMETRY;
    }
    return RH3T_OK;
}

} // namespace

extern "C" int rh3t_geom_build_ghosts(rh3t_geom* g, int32_t n_threads) {
    if (!g) return RH3T_ERR_INVALID_ARGUMENT;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
    if (int rc = build_geometry(g)) return rc;
    if (int rc = build_stencils(g)) return rc;
    build_ls_host(g);
    return build_access(g);
}

extern "C" int rh3t_geom_build_ghosts_device(int32_t n, rh3t_geom* const* geoms, int32_t n_threads, int32_t device) {
    if (n <= 0 || !geoms) return RH3T_ERR_INVALID_ARGUMENT;
    for (int32_t k = 0; k < n; ++k)
        if (!geoms[k]) return RH3T_ERR_INVALID_ARGUMENT;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
    // host phases: one geometry at a time when there are few of them (the
    // loops inside are parallel), several at once otherwise
    std::vector<int> rc(n, RH3T_OK);
    const bool outer = n >= 4;
#pragma omp parallel for schedule(dynamic, 1) if (outer)
    for (int32_t k = 0; k < n; ++k) {
        rh3t_geom* g = geoms[k];
        int r = build_geometry(g);
        if (!r) r = build_stencils(g);
        if (!r) r = build_access(g);
        rc[k] = r;
    }
    for (int32_t k = 0; k < n; ++k)
        if (rc[k]) return rc[k];
    // least-squares tables of every heavy ghost of every geometry on the device
    std::vector<rh3t::LsGrid> grids(n);
    std::vector<double*> s_out(n), w_out(n);
    long long total = 0;
    for (int32_t k = 0; k < n; ++k) {
        const rh3t_geom* g = geoms[k];
        rh3t::LsGrid& L = grids[k];
        L.x0 = g->G.x0; L.y0 = g->G.y0; L.dx = g->G.dx; L.dy = g->G.dy; L.ny = g->G.ny;
        const double h = ls_h(g);
        L.s0 = 2.0 * h * h;
        int off = 0;
        for (int r = 1; r <= 4; ++r) {
            std::vector<double> Mr;
            quad_form(r, h, Mr);
            std::copy(Mr.begin(), Mr.end(), L.M + off);
            off += (int)Mr.size();
        }
        s_out[k] = geoms[k]->s.data();
        w_out[k] = geoms[k]->w.data();
        total += (long long)g->heavy.size();
    }
    std::vector<rh3t::LsJob> jobs((size_t)total);
    std::vector<uint32_t> st((size_t)total * rh3t::LS_STENCIL);
    long long o = 0;
    for (int32_t k = 0; k < n; ++k) {
        const rh3t_geom* g = geoms[k];
        const long nh = (long)g->heavy.size();
        for (long q = 0; q < nh; ++q, ++o) {
            const double* pr = &g->proj[5 * g->heavy[q]];
            jobs[o] = {pr[0], pr[1], pr[2], pr[3], k, (int32_t)q};
        }
        std::copy(g->stencil.begin(), g->stencil.end(), st.begin() + (o - nh) * rh3t::LS_STENCIL);
    }
    char err[200] = {0};
    if (rh3t::ls_tables_device(device, n, grids.data(), total, jobs.data(), st.data(), s_out.data(), w_out.data(),
                               err, (int)sizeof(err))) {
        for (int32_t k = 0; k < n; ++k) geoms[k]->err = err;
        return RH3T_ERR_CUDA;
    }
    return RH3T_OK;
}

extern "C" int rh3t_geom_ghost_table(const rh3t_geom* g, rh3t_ghost_table* v) {
    if (!g || !v) return RH3T_ERR_INVALID_ARGUMENT;
    v->n_ghosts = (int32_t)g->boundary.size();
    v->idx = g->idx.data(); v->boundary = g->boundary.data(); v->side = g->side.data();
    v->proj = g->proj.data(); v->pre = g->pre.data();
    v->n_heavy = (int32_t)(g->nearest.size() / 2);
    v->nearest = g->nearest.data(); v->stencil = g->stencil.data();
    v->s = g->s.data(); v->w = g->w.data(); v->d = g->d.data();
    return RH3T_OK;
}

extern "C" int rh3t_geom_access_table(const rh3t_geom* g, uint32_t* out) {
    if (!g || !out) return RH3T_ERR_INVALID_ARGUMENT;
    std::memcpy(out, g->access.data(), g->access.size() * sizeof(uint32_t));
    return RH3T_OK;
}
