// ORACLE — test infrastructure only (see physics.hpp).
// Restatement of geometry.rs, field1.rs, ghost.rs (static build) and the
// build-time part of bc1.rs (E_r stencil extraction, least-squares pinv,
// smoothness-indicator quadratic forms). Compile with -ffp-contract=off.
#include "model.hpp"
#include <algorithm>
#include <cmath>
#include <set>

namespace oracle {

static const double PI = 3.14159265358979323846;

// ---------------------------------------------------------------- geometry.rs
static double cross(Point a, Point b) { return a.x * b.y - a.y * b.x; }

// geometry.rs:12-33
bool point_on_segment(Point p, Point a, Point b, double eps) {
    Point ab{b.x - a.x, b.y - a.y};
    Point ap{p.x - a.x, p.y - a.y};
    if (std::fabs(cross(ab, ap)) > eps) return false;
    return p.x >= std::fmin(a.x, b.x) - eps && p.x <= std::fmax(a.x, b.x) + eps &&
           p.y >= std::fmin(a.y, b.y) - eps && p.y <= std::fmax(a.y, b.y) + eps;
}

// geometry.rs:35-55
std::vector<size_t> find_boundary_sides(Point p, const Polygon& g, double eps) {
    std::vector<size_t> sides;
    size_t n = g.pts.size();
    for (size_t i = 0; i < n; ++i)
        if (point_on_segment(p, g.pts[i], g.pts[(i + 1) % n], eps)) sides.push_back(i);
    return sides;
}

// geometry.rs:165-178
double Polygon::signed_area2() const {
    size_t n = pts.size();
    double a2 = 0.0;
    for (size_t i = 0; i < n; ++i) {
        Point a = pts[i], b = pts[(i + 1) % n];
        a2 += a.x * b.y - b.x * a.y;
    }
    return a2;
}

// geometry.rs:181-202
static Point closest_point_on_segment(Point p, Point a, Point b) {
    double abx = b.x - a.x, aby = b.y - a.y;
    double apx = p.x - a.x, apy = p.y - a.y;
    double ab2 = abx * abx + aby * aby;
    if (ab2 <= 1e-30) return a;
    double t = (apx * abx + apy * aby) / ab2;
    if (t < 0.0) t = 0.0;
    if (t > 1.0) t = 1.0;
    return {a.x + t * abx, a.y + t * aby};
}

static double distance2(Point a, Point b) {
    double dx = a.x - b.x, dy = a.y - b.y;
    return dx * dx + dy * dy;
}

static Vec2 side_normal(const Polygon& g, size_t side) {
    size_t n = g.pts.size();
    Point a = g.pts[side], b = g.pts[(side + 1) % n];
    double tx = b.x - a.x, ty = b.y - a.y;
    double len = std::hypot(tx, ty);
    if (!(len > 1.0e-14)) throw OracleError(ERR_GEOMETRY, "degenerate polygon edge");
    Vec2 left{-ty / len, tx / len};
    Vec2 right{ty / len, -tx / len};
    bool ccw = g.signed_area2() > 0.0;
    if (g.fluid == FLUID_INSIDE) return ccw ? right : left;
    return ccw ? left : right;
}

// geometry.rs:212-250
Vec2 Polygon::outward_normal_of_side(size_t side) const { return side_normal(*this, side); }

// geometry.rs:254-278 (crossing-number test)
bool Polygon::is_fluid(Point p) const {
    size_t n = pts.size();
    if (n < 3) return false;
    bool inside = false;
    for (size_t i = 0; i < n; ++i) {
        Point a = pts[i], b = pts[(i + 1) % n];
        bool crosses = (a.y > p.y) != (b.y > p.y);
        if (crosses) {
            double x_int = a.x + (p.y - a.y) * (b.x - a.x) / (b.y - a.y);
            if (p.x < x_int) inside = !inside;
        }
    }
    return fluid == FLUID_INSIDE ? inside : !inside;
}

// geometry.rs:280-302
Point Polygon::closest_point(Point p) const {
    size_t n = pts.size();
    Point closest = pts[0];
    double best = INFINITY;
    for (size_t i = 0; i < n; ++i) {
        Point c = closest_point_on_segment(p, pts[i], pts[(i + 1) % n]);
        double d2 = distance2(p, c);
        if (d2 < best) { best = d2; closest = c; }
    }
    return closest;
}

// geometry.rs:304-420
Vec2 Polygon::normal(Point p0) const {
    size_t n = pts.size();
    double area2 = signed_area2();
    if (!(std::fabs(area2) > 1e-14)) throw OracleError(ERR_GEOMETRY, "degenerate polygon");
    size_t best_edge = 0;
    double best = INFINITY;
    for (size_t i = 0; i < n; ++i) {
        Point c = closest_point_on_segment(p0, pts[i], pts[(i + 1) % n]);
        double d2 = distance2(p0, c);
        if (d2 < best) { best = d2; best_edge = i; }
    }
    return side_normal(*this, best_edge);
}

// geometry.rs:121-138
Projection project_polygon(const Polygon& g, Point p) {
    Point p0 = g.closest_point(p);
    Vec2 n = g.normal(p0);
    double dx = p.x - p0.x, dy = p.y - p0.y;
    return {p0, n, dx * n.x + dy * n.y};
}

// geometry.rs:435-437 (Rust f64::rem_euclid)
static double normalize_angle(double th) {
    double m = 2.0 * PI;
    double r = std::fmod(th, m);
    return r < 0.0 ? r + std::fabs(m) : r;
}
static const double ARC_ANGLE_TOL = 1e-12;

// geometry.rs:492-549
CircularArc CircularArc::from_three_points(Point s, Point m, Point e, FluidSide f) {
    double x1 = s.x, y1 = s.y, x2 = m.x, y2 = m.y, x3 = e.x, y3 = e.y;
    double d = 2.0 * (x1 * (y2 - y3) + x2 * (y3 - y1) + x3 * (y1 - y2));
    double chord = std::fmax(std::fmax(std::fmax(0.0, std::hypot(x1 - x2, y1 - y2)), std::hypot(x2 - x3, y2 - y3)),
                             std::hypot(x1 - x3, y1 - y3));
    chord = std::fmax(chord, 1.0);
    if (!(std::fabs(d) > 1e-12 * chord * chord)) throw OracleError(ERR_GEOMETRY, "points are (nearly) collinear");
    double r1 = x1 * x1 + y1 * y1, r2 = x2 * x2 + y2 * y2, r3 = x3 * x3 + y3 * y3;
    double ux = (r1 * (y2 - y3) + r2 * (y3 - y1) + r3 * (y1 - y2)) / d;
    double uy = (r1 * (x3 - x2) + r2 * (x1 - x3) + r3 * (x2 - x1)) / d;
    CircularArc a;
    a.center = {ux, uy};
    a.radius = std::hypot(x1 - ux, y1 - uy);
    double ts = std::atan2(y1 - uy, x1 - ux);
    double tm = std::atan2(y2 - uy, x2 - ux);
    double te = std::atan2(y3 - uy, x3 - ux);
    double ccw_sweep = normalize_angle(te - ts);
    double ccw_to_mid = normalize_angle(tm - ts);
    a.sweep = ccw_to_mid <= ccw_sweep + ARC_ANGLE_TOL ? ccw_sweep : -normalize_angle(ts - te);
    a.theta_start = ts;
    a.fluid = f;
    return a;
}

// geometry.rs:552-560
bool CircularArc::contains_angle(double theta) const {
    if (sweep > 0.0) return normalize_angle(theta - theta_start) <= sweep + ARC_ANGLE_TOL;
    return normalize_angle(theta_start - theta) <= -sweep + ARC_ANGLE_TOL;
}
Point CircularArc::start_point() const {
    return {center.x + radius * std::cos(theta_start), center.y + radius * std::sin(theta_start)};
}
Point CircularArc::end_point() const {
    double te = theta_start + sweep;
    return {center.x + radius * std::cos(te), center.y + radius * std::sin(te)};
}

// geometry.rs:578-607
Point CircularArc::closest_point(Point p) const {
    double rx = p.x - center.x, ry = p.y - center.y;
    double rnorm = std::hypot(rx, ry);
    if (rnorm > ARC_ANGLE_TOL) {
        double theta = std::atan2(ry, rx);
        if (contains_angle(theta)) {
            double s = radius / rnorm;
            return {center.x + s * rx, center.y + s * ry};
        }
    }
    Point st = start_point(), en = end_point();
    double d2s = sq(p.x - st.x) + sq(p.y - st.y);
    double d2e = sq(p.x - en.x) + sq(p.y - en.y);
    return d2s <= d2e ? st : en;
}

// geometry.rs:613-635
Vec2 CircularArc::outward_normal(Point p0) const {
    double dx = p0.x - center.x, dy = p0.y - center.y;
    double nrm = std::hypot(dx, dy);
    if (!(nrm > 1e-14)) throw OracleError(ERR_GEOMETRY, "point coincides with arc center");
    Vec2 radial{dx / nrm, dy / nrm};
    if (fluid == FLUID_INSIDE) return radial;
    return {-radial.x, -radial.y};
}

// geometry.rs:639-653
Projection CircularArc::project(Point p) const {
    Point p0 = closest_point(p);
    Vec2 n = outward_normal(p0);
    double dx = p.x - p0.x, dy = p.y - p0.y;
    return {p0, n, dx * n.x + dy * n.y};
}

// ---------------------------------------------------------------- field1.rs
// field1.rs:112-122
void Field::init_mask() {
    size_t n = grid.len();
    fluid.assign(n, 0);
    for (size_t l = 0; l < n; ++l) {
        long i = (long)(l / grid.ny), j = (long)(l % grid.ny);
        Point p{grid.x(i), grid.y(j)};
        fluid[l] = outer.is_fluid(p) && inner.is_fluid(p);
    }
}

// field1.rs:179-192
bool Field::is_in_domain(long i, long j) const {
    if (!grid.in_grid(i, j)) {
        Point p{grid.x(i), grid.y(j)};
        return outer.is_fluid(p) && inner.is_fluid(p);
    }
    return fluid[(size_t)i * grid.ny + (size_t)j] != 0;
}

// field1.rs:164-177
const CircularArc* Field::arc_for_side(BoundaryKind b, size_t side) const {
    const std::vector<ArcOverride>& arcs = b == OUTER ? outer_arcs : inner_arcs;
    for (const ArcOverride& ov : arcs)
        if (ov.contains_side(side)) return &ov.arc;
    return nullptr;
}

// ---------------------------------------------------------------- ghost.rs
// ghost.rs:285-305
int bc_priority(BCKind k) {
    switch (k) {
    case BC_WALL: return 100;
    case BC_REFLECTIVE_WALL: return 90;
    case BC_CONSTANT: case BC_TIME_DEPENDENT: return 70;
    case BC_FAR_FIELD: return 20;
    case BC_OUTFLOW: return 10;
    case BC_ZEROTH_ORDER: return 5;
    case BC_PERIODIC: return 0;
    }
    return 0;
}

// ghost.rs:307-348
size_t select_boundary_side(Point p0, const Polygon& g, const std::vector<BC>& bcs) {
    std::vector<size_t> cand = find_boundary_sides(p0, g, 1e-12);
    if (cand.empty()) throw OracleError(ERR_GEOMETRY, "projection point does not lie on any polygon side");
    if (g.pts.size() != bcs.size()) throw OracleError(ERR_GEOMETRY, "polygon side count and BC count disagree");
    size_t best = cand[0];
    int bp = bc_priority(bcs[best].kind);
    for (size_t k = 1; k < cand.size(); ++k) {
        int p = bc_priority(bcs[cand[k]].kind);
        if (p > bp) { best = cand[k]; bp = p; }
    }
    return best;
}

// ghost.rs:482-493
std::vector<std::pair<long, long>> default_stencil_offsets() {
    std::vector<std::pair<long, long>> o;
    for (long d = -4; d <= 4; ++d) { o.push_back({d, 0}); o.push_back({0, d}); }
    std::sort(o.begin(), o.end());
    o.erase(std::unique(o.begin(), o.end()), o.end());
    return o;
}

// ghost.rs:352-376
std::vector<std::pair<long, long>> discover_ghost_indices(const Field& f, const std::vector<std::pair<long, long>>& offs) {
    std::set<std::pair<long, long>> set;
    for (long i = 0; i < f.grid.nx; ++i)
        for (long j = 0; j < f.grid.ny; ++j) {
            if (!f.is_in_domain(i, j)) continue;
            for (auto& o : offs) {
                long a = i + o.first, b = j + o.second;
                if (!f.is_in_domain(a, b)) set.insert({a, b});
            }
        }
    return std::vector<std::pair<long, long>>(set.begin(), set.end());
}

// ---------------------------------------------------------------- bc1.rs (build time)
// bc1.rs:257-281
void find_nearest_grid_point(const Projection& p, const Field& f, long& oi, long& oj) {
    long i, j;
    f.grid.coord2idx(p.point, i, j);
    const long cand[9][2] = {{i, j}, {i - 1, j}, {i + 1, j}, {i, j - 1}, {i, j + 1},
                             {i + 1, j + 1}, {i + 1, j - 1}, {i - 1, j + 1}, {i - 1, j - 1}};
    oi = 0; oj = 0;
    double best = 1e50;
    for (int k = 0; k < 9; ++k) {
        if (!f.is_in_domain(cand[k][0], cand[k][1])) continue;
        double dx = f.grid.x(cand[k][0]) - p.point.x;
        double dy = f.grid.y(cand[k][1]) - p.point.y;
        double dis = std::sqrt(sq(dx) + sq(dy));
        if (dis < best) { oi = cand[k][0]; oj = cand[k][1]; best = dis; }
    }
}

// bc1.rs:1306-1350
static long clampl(long v, long lo, long hi) { return v < lo ? lo : (v > hi ? hi : v); }
static long first_interior_j(const Projection& p, const Field& f) {
    double q = (p.point.y - f.grid.y0) / f.grid.dy;
    long j = p.normal.y > 0.0 ? (long)std::ceil(q) - 1 : (long)std::floor(q) + 1;
    return clampl(j, 0, f.grid.ny - 1);
}
static long first_interior_i(const Projection& p, const Field& f) {
    double q = (p.point.x - f.grid.x0) / f.grid.dx;
    long i = p.normal.x > 0.0 ? (long)std::ceil(q) - 1 : (long)std::floor(q) + 1;
    return clampl(i, 0, f.grid.nx - 1);
}

// bc1.rs:1489-1549 — shift a whole substencil along its grid line, nearest shift first
static bool shifted_substencil(const Field& f, bool vertical, long line, long base, long width,
                               std::vector<std::pair<long, long>>& out) {
    long max_shift = (vertical ? f.grid.ny : f.grid.nx) + width;
    for (long mag = 0; mag <= max_shift; ++mag) {
        long shifts[2] = {-mag, mag};
        int count = mag == 0 ? 1 : 2;
        for (int s = 0; s < count; ++s) {
            long start = base + shifts[s];
            bool ok = true;
            for (long a = 0; a < width; ++a) {
                long i = vertical ? line : start + a;
                long j = vertical ? start + a : line;
                if (!f.grid.in_grid(i, j) || !f.is_in_domain(i, j)) { ok = false; break; }
            }
            if (ok) {
                for (long a = 0; a < width; ++a)
                    out.push_back(vertical ? std::make_pair(line, start + a) : std::make_pair(start + a, line));
                return true;
            }
        }
    }
    return false;
}

// bc1.rs:1374-1485
std::vector<std::pair<long, long>> weno_stencil_extractor_indices(const Projection& p, const Field& f, int r) {
    Vec2 n = p.normal;
    Point p0 = p.point;
    long width = r + 1;
    std::vector<std::pair<long, long>> e;
    if (std::fabs(n.x) >= std::fabs(n.y)) {
        if (!(std::fabs(n.x) > 1.0e-14)) throw OracleError(ERR_STENCIL_FIT, "normal too small");
        long i0 = first_interior_i(p, f);
        long step = p.normal.x > 0.0 ? -1 : 1;
        for (long l = 0; l <= r; ++l) {
            long il = i0 + l * step;
            double xl = f.grid.x(il);
            double t = (p0.x - xl) / n.x;
            double ys = p0.y - n.y * t;
            long m = (long)std::floor((ys - f.grid.y0) / f.grid.dy);
            long base = m - (long)(r / 2);
            if (!shifted_substencil(f, true, il, base, width, e))
                throw OracleError(ERR_STENCIL_FIT, "cannot fit paper substencil on vertical grid line", il, 0);
        }
    } else {
        if (!(std::fabs(n.y) > 1.0e-14)) throw OracleError(ERR_STENCIL_FIT, "normal too small");
        long j0 = first_interior_j(p, f);
        long step = p.normal.y > 0.0 ? -1 : 1;
        for (long l = 0; l <= r; ++l) {
            long jl = j0 + l * step;
            double yl = f.grid.y(jl);
            double t = (p0.y - yl) / n.y;
            double xs = p0.x - n.x * t;
            long m = (long)std::floor((xs - f.grid.x0) / f.grid.dx);
            long base = m - (long)(r / 2);
            if (!shifted_substencil(f, false, jl, base, width, e))
                throw OracleError(ERR_STENCIL_FIT, "cannot fit paper substencil on horizontal grid line", 0, jl);
        }
    }
    return e;
}

// bc1.rs:1119-1160
static void derivative_coeffs(const std::vector<double>& coef, int degree, int ax, int ay,
                              std::vector<std::array<double, 3>>& out) {
    out.clear();
    int k = 0;
    for (int total = 0; total <= degree; ++total)
        for (int i = 0; i <= total; ++i) {
            int j = total - i;
            double aij = coef[k];
            k++;
            if (i < ax || j < ay) continue;
            double factor = 1.0;
            for (int m = 0; m < ax; ++m) factor *= (double)(i - m);
            for (int m = 0; m < ay; ++m) factor *= (double)(j - m);
            out.push_back({(double)(i - ax), (double)(j - ay), aij * factor});
        }
}

// bc1.rs:1184-1196
static double integrate_1d_monomial(int power, double h) {
    if (power % 2 == 1) return 0.0;
    double half = 0.5 * h;
    return 2.0 * powi(half, power + 1) / (double)(power + 1);
}

// bc1.rs:1162-1182
static double integrate_square(const std::vector<std::array<double, 3>>& poly, double h) {
    double result = 0.0;
    for (auto& a : poly)
        for (auto& b : poly) {
            int px = (int)a[0] + (int)b[0], py = (int)a[1] + (int)b[1];
            double ix = integrate_1d_monomial(px, h), iy = integrate_1d_monomial(py, h);
            result += a[2] * b[2] * ix * iy;
        }
    return result;
}

// bc1.rs:1070-1117
double smooth_indicator(const std::vector<double>& coef, int r, double h) {
    if (r == 0) return 2.0 * h * h;
    double beta = 0.0;
    std::vector<std::array<double, 3>> der;
    for (int ax = 0; ax <= r; ++ax)
        for (int ay = 0; ay <= r - ax; ++ay) {
            int order = ax + ay;
            if (order == 0) continue;
            derivative_coeffs(coef, r, ax, ay, der);
            double integral = integrate_square(der, h);
            double scale = powi(h, 2 * (order - 1));
            beta += scale * integral;
        }
    return beta;
}

// bc1.rs:62-81
Matrix beta_quadratic_form(int r, double h) {
    int n = (r + 1) * (r + 2) / 2;
    Matrix m(n, n);
    for (int a = 0; a < n; ++a)
        for (int b = a; b < n; ++b) {
            std::vector<double> ea(n, 0.0), eb(n, 0.0), eab(n, 0.0);
            ea[a] = 1.0; eb[b] = 1.0;
            for (int q = 0; q < n; ++q) eab[q] = ea[q] + eb[q];
            double v = 0.5 * (smooth_indicator(eab, r, h) - smooth_indicator(ea, r, h) - smooth_indicator(eb, r, h));
            m(a, b) = v;
            m(b, a) = v;
        }
    return m;
}

// Pseudo-inverse with an absolute singular-value cut (nalgebra
// `svd(true,true).pseudo_inverse(tol)`: sigma > tol -> 1/sigma, else 0).
// nalgebra 0.33.3 is not in the reference tree; this is a one-sided Jacobi
// SVD of the same matrix (the maths of pinv is unique for sigma above the cut;
// the bit pattern of nalgebra's result is not reproduced).
Matrix pinv_svd(const Matrix& A, double tol) {
    int m = A.r, n = A.c;
    Matrix U = A, V(n, n);
    for (int i = 0; i < n; ++i) V(i, i) = 1.0;
    for (int sweep = 0; sweep < 80; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double al = 0, be = 0, ga = 0;
                for (int i = 0; i < m; ++i) {
                    al += U(i, p) * U(i, p);
                    be += U(i, q) * U(i, q);
                    ga += U(i, p) * U(i, q);
                }
                if (ga == 0.0) continue;
                double rel = std::fabs(ga) / std::sqrt(al * be);
                if (rel > off) off = rel;
                if (rel < 1e-17) continue;
                double zeta = (be - al) / (2.0 * ga);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (int i = 0; i < m; ++i) {
                    double up = U(i, p), uq = U(i, q);
                    U(i, p) = c * up - s * uq;
                    U(i, q) = s * up + c * uq;
                }
                for (int i = 0; i < n; ++i) {
                    double vp = V(i, p), vq = V(i, q);
                    V(i, p) = c * vp - s * vq;
                    V(i, q) = s * vp + c * vq;
                }
            }
        if (off < 1e-16) break;
    }
    Matrix P(n, m);
    for (int j = 0; j < n; ++j) {
        double sig = 0.0;
        for (int i = 0; i < m; ++i) sig += U(i, j) * U(i, j);
        sig = std::sqrt(sig);
        if (!(sig > tol)) continue;
        for (int a = 0; a < m; ++a) {
            double uij = U(a, j) / sig; // normalised left singular vector
            double scale = uij / sig;
            for (int k = 0; k < n; ++k) P(k, a) += V(k, j) * scale;
        }
    }
    return P;
}

static double factorial(int n) {
    double r = 1.0;
    for (int k = 1; k <= n; ++k) r *= (double)k;
    return r;
}

// bc1.rs:89-101
static int xk_coefficient_column(int k) {
    int col = 0;
    for (int t = 0; t <= k; ++t)
        for (int i2 = 0; i2 <= t; ++i2) {
            int j2 = t - i2;
            if (i2 == k && j2 == 0) return col;
            col++;
        }
    return -1;
}

// bc1.rs:108-188
void precompute_ghost_bc(const Projection& p, const Field& f, const Matrix forms[5], GhostBC& bc) {
    find_nearest_grid_point(p, f, bc.nearest_i, bc.nearest_j);
    double h = std::sqrt(f.grid.dx * f.grid.dy);
    double d0 = 2.0 * powi(h, 4), d1 = 2.0 * powi(h, 3), d2 = 2.0 * powi(h, 2), d3 = 2.0 * h;
    bc.normal = p.normal;
    bc.d[0] = d0; bc.d[1] = d1; bc.d[2] = d2; bc.d[3] = d3;
    bc.d[4] = 1.0 - d0 - d1 - d2 - d3;
    for (int k = 0; k < 55; ++k) bc.stencil[k] = 0;
    for (int k = 0; k < 979; ++k) bc.s[k] = 0.0;
    for (int k = 0; k < 225; ++k) bc.w[k] = 0.0;
    for (int r = 0; r <= 4; ++r) {
        int m = (r + 1) * (r + 1);
        int nt = (r + 1) * (r + 2) / 2;
        std::vector<std::pair<long, long>> idx = weno_stencil_extractor_indices(p, f, r);
        double xy[25][2];
        for (int a = 0; a < m; ++a) {
            bc.stencil[BC_STENCIL_OFF[r] + a] = (uint32_t)f.linear_index(idx[a].first, idx[a].second);
            Point q{f.grid.x(idx[a].first), f.grid.y(idx[a].second)};
            p.global2local(q, xy[a][0], xy[a][1]);
        }
        Matrix A(m, nt);
        for (int row = 0; row < m; ++row) {
            int col = 0;
            for (int t = 0; t <= r; ++t)
                for (int i2 = 0; i2 <= t; ++i2) {
                    int j2 = t - i2;
                    A(row, col) = powi(xy[row][0], i2) * powi(xy[row][1], j2);
                    col++;
                }
        }
        Matrix P = pinv_svd(A, 1.0e-12); // nt x m
        if (r == 0) {
            bc.s[0] = 2.0 * h * h;
        } else {
            const Matrix& M = forms[r];
            Matrix T1(m, nt); // P^T M
            for (int a = 0; a < m; ++a)
                for (int c = 0; c < nt; ++c) {
                    double acc = 0.0;
                    for (int k = 0; k < nt; ++k) acc += P(k, a) * M(k, c);
                    T1(a, c) = acc;
                }
            for (int a = 0; a < m; ++a)
                for (int b = 0; b < m; ++b) {
                    double acc = 0.0;
                    for (int k = 0; k < nt; ++k) acc += T1(a, k) * P(k, b);
                    bc.s[BC_S_OFF[r] + a * m + b] = acc;
                }
        }
        for (int k = 0; k <= r; ++k) {
            int col = xk_coefficient_column(k);
            double kf = factorial(k);
            for (int a = 0; a < m; ++a) bc.w[BC_W_OFF[r] + k * m + a] = kf * P(col, a);
        }
    }
}

// bc1.rs:1215-1254 (tests/slow path only): least-squares fit via the pinv.
std::vector<double> fit_polynomial_surface(const std::vector<std::array<double, 3>>& data, int degree) {
    int np = (int)data.size(), nt = (degree + 1) * (degree + 2) / 2;
    Matrix A(np, nt);
    for (int row = 0; row < np; ++row) {
        int col = 0;
        for (int t = 0; t <= degree; ++t)
            for (int i = 0; i <= t; ++i) {
                int j = t - i;
                A(row, col) = powi(data[row][0], i) * powi(data[row][1], j);
                col++;
            }
    }
    Matrix P = pinv_svd(A, 1.0e-12);
    std::vector<double> c(nt, 0.0);
    for (int k = 0; k < nt; ++k) {
        double acc = 0.0;
        for (int a = 0; a < np; ++a) acc += P(k, a) * data[a][2];
        c[k] = acc;
    }
    return c;
}

// bc1.rs:1268-1304
double x_derivative_at_origin(const std::vector<double>& c, int degree, int k) {
    if (k > degree) return 0.0;
    return c[xk_coefficient_column(k)] * factorial(k);
}

// ghost.rs:378-478 build_ghost_info
static GhostInfo build_ghost_info(const Field& f, long i, long j) {
    Point p{f.grid.x(i), f.grid.y(j)};
    bool outer_fluid = f.outer.is_fluid(p);
    BoundaryKind bk = outer_fluid ? INNER : OUTER;
    const Polygon& poly = bk == OUTER ? f.outer : f.inner;
    const std::vector<BC>& bcs = bk == OUTER ? f.bc_outer : f.bc_inner;
    Projection raw = project_polygon(poly, p);
    GhostInfo g;
    g.i = i; g.j = j;
    find_nearest_grid_point(raw, f, g.nearest_i, g.nearest_j);
    g.side_id = select_boundary_side(raw.point, poly, bcs);
    g.boundary = bk;
    if (const CircularArc* arc = f.arc_for_side(bk, g.side_id)) {
        g.project = arc->project(p);
    } else {
        Vec2 n = poly.outward_normal_of_side(g.side_id);
        double dx = p.x - raw.point.x, dy = p.y - raw.point.y;
        g.project = {raw.point, n, dx * n.x + dy * n.y};
    }
    return g;
}

// ghost.rs:50-118
void GhostGrid::build(const Field& f, const std::vector<std::pair<long, long>>& offsets) {
    std::vector<std::pair<long, long>> idx = discover_ghost_indices(f, offsets);
    info.clear(); pre.clear(); lookup.clear();
    double h = std::sqrt(f.grid.dx * f.grid.dy);
    Matrix forms[5];
    for (int r = 0; r < 5; ++r) forms[r] = beta_quadratic_form(r, h);
    info.resize(idx.size());
    std::vector<int> heavy(idx.size(), 0);
    // geometry per ghost (independent) then the heavy precompute in parallel
    std::string err; int err_code = 0;
#pragma omp parallel for schedule(dynamic, 16)
    for (long g = 0; g < (long)idx.size(); ++g) {
        try {
            info[g] = build_ghost_info(f, idx[g].first, idx[g].second);
        } catch (OracleError& e) {
#pragma omp critical
            { err = e.what(); err_code = e.code; }
        }
    }
    if (err_code) throw OracleError(err_code, err);
    for (size_t g = 0; g < idx.size(); ++g) {
        lookup[idx[g]] = g;
        const std::vector<BC>& bcs = info[g].boundary == OUTER ? f.bc_outer : f.bc_inner;
        BCKind k = bcs[info[g].side_id].kind;
        if (k == BC_WALL || k == BC_OUTFLOW || k == BC_FAR_FIELD) {
            info[g].pre = (int)pre.size();
            pre.emplace_back();
        }
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (long g = 0; g < (long)idx.size(); ++g) {
        if (info[g].pre < 0) continue;
        try {
            precompute_ghost_bc(info[g].project, f, forms, pre[info[g].pre]);
        } catch (OracleError& e) {
#pragma omp critical
            { err = e.what(); err_code = e.code; }
        }
    }
    if (err_code) throw OracleError(err_code, err);
    values.assign(info.size(), State{0, 0, 0, 0, 0, 0});
    derived.assign(info.size(), Derived{});

    long nx = f.grid.nx, ny = f.grid.ny;
    n_offsets = offsets.size();
    for (auto& row : off_map) for (int& v : row) v = -1;
    for (size_t k = 0; k < offsets.size(); ++k) off_map[offsets[k].first + 4][offsets[k].second + 4] = (int)k;
    access.assign((size_t)nx * ny * n_offsets, 0u);
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j) {
            size_t l = (size_t)i * ny + j;
            if (!f.fluid[l]) continue;
            for (size_t k = 0; k < offsets.size(); ++k) {
                long a = i + offsets[k].first, b = j + offsets[k].second;
                size_t t;
                if (f.grid.in_grid(a, b) && f.fluid[(size_t)a * ny + b]) {
                    t = (size_t)a * ny + b;
                } else {
                    auto it = lookup.find({a, b});
                    if (it == lookup.end()) throw OracleError(ERR_GEOMETRY, "ghost referenced by a fluid cell is not cached", a, b);
                    t = it->second + (size_t)nx * ny;
                }
                access[l * n_offsets + k] = (uint32_t)t;
            }
        }
}

} // namespace oracle
