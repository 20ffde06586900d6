// ORACLE — test infrastructure only (see physics.hpp). Restatement of the
// reference's geometry (geometry.rs), grid/field (field1.rs), BC types and
// ghost precompute (bc1.rs) and ghost grid (ghost.rs). Host-side, double only.
#pragma once
#include "physics.hpp"
#include <array>
#include <cstddef>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace oracle {

using State = StateT<double>;
using Derived = DerivedT<double>;

struct Point { double x, y; };
struct Vec2 { double x, y; };

// geometry.rs:88-108
struct Projection {
    Point point;
    Vec2 normal;
    double distance;
    void global2local(Point p, double& nor, double& tan) const {
        double dx = p.x - point.x, dy = p.y - point.y;
        nor = normal.x * dx + normal.y * dy;
        tan = -dx * normal.y + dy * normal.x;
    }
};

enum FluidSide { FLUID_INSIDE = 0, FLUID_OUTSIDE = 1 };

// geometry.rs:145-421
struct Polygon {
    std::vector<Point> pts;
    FluidSide fluid = FLUID_INSIDE;
    double signed_area2() const;
    bool is_fluid(Point p) const;
    Point closest_point(Point p) const;
    Vec2 normal(Point p0) const;
    Vec2 outward_normal_of_side(size_t side) const;
};

// geometry.rs:439-654
struct CircularArc {
    Point center;
    double radius, theta_start, sweep;
    FluidSide fluid;
    static CircularArc from_three_points(Point s, Point m, Point e, FluidSide f);
    bool contains_angle(double theta) const;
    Point start_point() const;
    Point end_point() const;
    Point closest_point(Point p) const;
    Vec2 outward_normal(Point p0) const;
    Projection project(Point p) const;
};

// geometry.rs:661-673
struct ArcOverride {
    size_t side_start, side_end;
    CircularArc arc;
    bool contains_side(size_t s) const { return s >= side_start && s <= side_end; }
};

Projection project_polygon(const Polygon& g, Point p);                // geometry.rs:121-138
bool point_on_segment(Point p, Point a, Point b, double eps);         // geometry.rs:12-33
std::vector<size_t> find_boundary_sides(Point p, const Polygon& g, double eps); // geometry.rs:35-55

// bc1.rs:17-28
enum BCKind {
    BC_REFLECTIVE_WALL = 0, BC_WALL = 1, BC_PERIODIC = 2, BC_CONSTANT = 3,
    BC_TIME_DEPENDENT = 4, BC_OUTFLOW = 5, BC_ZEROTH_ORDER = 6, BC_FAR_FIELD = 7
};
struct BC {
    BCKind kind = BC_WALL;
    State state{};                 // Constant / FarField
    double p_inf = 0, sigma = 0, l_domain = 1; // Outflow
    // TimeDependent: the reference's only closure (init.rs:61-65) is a moving
    // vertical shock: state = p.x <= td_x0 + td_speed*t ? td_left : td_right.
    double td_x0 = 0, td_speed = 0;
    State td_left{}, td_right{};
};
int bc_priority(BCKind k); // ghost.rs:285-305

// field1.rs:6-73
struct GridInfo {
    long nx = 0, ny = 0;
    double dx = 0, dy = 0, x0 = 0, y0 = 0;
    bool in_grid(long i, long j) const { return i >= 0 && i < nx && j >= 0 && j < ny; }
    double x(long i) const { return x0 + (double)i * dx; }
    double y(long j) const { return y0 + (double)j * dy; }
    size_t len() const { return (size_t)(nx * ny); }
    void coord2idx(Point p, long& i, long& j) const {
        i = (long)std::round((p.x - x0) / dx);
        j = (long)std::round((p.y - y0) / dy);
    }
};

enum BoundaryKind { OUTER = 0, INNER = 1 };

// field1.rs:75-136
struct Field {
    GridInfo grid;
    std::vector<State> value;
    Polygon outer, inner;
    std::vector<BC> bc_inner, bc_outer;
    double time = 0;
    std::vector<uint8_t> fluid;
    std::vector<ArcOverride> outer_arcs, inner_arcs;

    void init_mask();
    bool is_in_domain(long i, long j) const; // field1.rs:179-192
    size_t linear_index(long i, long j) const { return (size_t)i * grid.ny + (size_t)j; }
    const CircularArc* arc_for_side(BoundaryKind b, size_t side) const;
};

// bc1.rs:45-57
constexpr int BC_STENCIL_OFF[6] = {0, 1, 5, 14, 30, 55};
constexpr int BC_S_OFF[6] = {0, 1, 17, 98, 354, 979};
constexpr int BC_W_OFF[6] = {0, 1, 9, 36, 100, 225};
struct GhostBC {
    long nearest_i, nearest_j;
    Vec2 normal;
    double d[5];
    uint32_t stencil[55];
    double s[979];
    double w[225];
};

// ghost.rs:18-27
struct GhostInfo {
    long i, j;
    Projection project;
    long nearest_i, nearest_j;
    BoundaryKind boundary;
    size_t side_id;
    int pre = -1; // index into GhostGrid::pre, or -1
};

struct Matrix { // row-major dense matrix, only for the build-time precompute
    int r = 0, c = 0;
    std::vector<double> a;
    Matrix() {}
    Matrix(int r_, int c_) : r(r_), c(c_), a((size_t)r_ * c_, 0.0) {}
    double& operator()(int i, int j) { return a[(size_t)i * c + j]; }
    double operator()(int i, int j) const { return a[(size_t)i * c + j]; }
};

// ghost.rs:30-46
struct GhostGrid {
    std::vector<GhostInfo> info;
    std::vector<GhostBC> pre;
    std::vector<State> values;
    std::vector<Derived> derived;
    std::map<std::pair<long, long>, size_t> lookup;
    std::vector<uint32_t> access;
    size_t n_offsets = 0;
    int off_map[9][9];
    void build(const Field& f, const std::vector<std::pair<long, long>>& offsets);
    int k_for(long di, long dj) const { return off_map[di + 4][dj + 4]; }
};

std::vector<std::pair<long, long>> default_stencil_offsets();                           // ghost.rs:482-493
std::vector<std::pair<long, long>> discover_ghost_indices(const Field& f, const std::vector<std::pair<long, long>>& offs);
size_t select_boundary_side(Point p0, const Polygon& g, const std::vector<BC>& bcs);    // ghost.rs:307-348
void find_nearest_grid_point(const Projection& p, const Field& f, long& oi, long& oj);   // bc1.rs:257-281
std::vector<std::pair<long, long>> weno_stencil_extractor_indices(const Projection& p, const Field& f, int r);
Matrix beta_quadratic_form(int r, double h);                                           // bc1.rs:62-81
double smooth_indicator(const std::vector<double>& coef, int r, double h);              // bc1.rs:1070-1117
Matrix pinv_svd(const Matrix& A, double tol);                                           // nalgebra pseudo_inverse
void precompute_ghost_bc(const Projection& p, const Field& f, const Matrix forms[5], GhostBC& out);
std::vector<double> fit_polynomial_surface(const std::vector<std::array<double, 3>>& data, int degree);
double x_derivative_at_origin(const std::vector<double>& c, int degree, int k);

// bc1.rs:294-312 build_local_plain (solver.cpp)
void build_local_plain(Vec2 n, const State& val, const Params& P, double L[6][6], double R[6][6], double lam[6]);
// bc1.rs:676-928 Wall / Outflow / FarField rows + Taylor sum (solver.cpp)
State ghost_from_extrapolation(const BC& bc, const Projection& pr, const double L[6][6], const double R[6][6],
                               const double lam[6], const double v[5][6], const Params& P, long gi, long gj);

// slowpath.cpp: weno.rs:599-679 reconstruction; bc1.rs:345-421 weno_extrapolation
State reconstruction_slow(const State pts[6], Dir dir, bool recon_type, const Params& P);
void weno_extrapolation_slow(const Projection& pr, const Field& f, const State* val, const Params& P, int k,
                             bool beta0_as_fast, double out[6]);

struct OracleError : std::runtime_error {
    int code;
    long i, j;
    OracleError(int c, const std::string& m, long i_ = 0, long j_ = 0) : std::runtime_error(m), code(c), i(i_), j(j_) {}
};
enum ErrCode { ERR_OK = 0, ERR_NONPHYSICAL = 1, ERR_NONFINITE_GHOST = 2, ERR_SINGULAR = 3, ERR_PERIODIC = 4,
               ERR_STENCIL_FIT = 5, ERR_GEOMETRY = 6 };

} // namespace oracle
