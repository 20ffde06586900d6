// The 70 dot products of a heavy ghost's WENO extrapolation (bc1.rs:221-244)
// with its stencil data d (rows of S_0..S_4 and w_{r,k}), scheduled over the
// 32 lanes of a warp as pairs of rows of one order, and the row layout of d
// that keeps the loads of different orders in different shared-memory banks.
// Used by the ghost update (ghosts.cu) and its vector-Jacobian product
// (adjoint.cu).
#pragma once

namespace rh3t {

// Row of D holding stencil node a of order r: the order blocks start at
// kDOff[r], whose residues mod 8 differ, so the 16-byte loads of D rows of
// different orders at the same position fall in different banks.
static __constant__ int kDOff[5] = {0, 1, 5, 14, 31};
__host__ __device__ constexpr int d_row(int a) { return a + (a >= 30 ? 1 : 0); }

// Schedule of the 70 dot products with the stencil data d (55 rows of
// S_0..S_4 and the 15 rows w_{r,k}), all six fields at once, as 35 pairs of
// rows of one order (one load of a D row serves both), in two slots a warp
// runs one after the other (25 and 4 terms at most). Row code:
// w-row flag << 8 | r << 5 | a (S row) or k (w row); 0xffff = none.
constexpr unsigned short kRowNone = 0xffff;
__host__ __device__ constexpr unsigned short srow(int r, int a) { return (unsigned short)((r << 5) | a); }
__host__ __device__ constexpr unsigned short wrow(int r, int k) { return (unsigned short)(0x100 | (r << 5) | k); }
__host__ __device__ constexpr unsigned pair(unsigned short x, unsigned short y) { return (unsigned)x | ((unsigned)y << 16); }
constexpr unsigned kPairNone = 0xffffffffu;
static __constant__ unsigned kSlotA[32] = {  // orders 4 (lanes 0-14), 3 (15-24), 2 (25-30), 1 (31)
    pair(srow(4, 0), srow(4, 1)), pair(srow(4, 2), srow(4, 3)), pair(srow(4, 4), srow(4, 5)),
    pair(srow(4, 6), srow(4, 7)), pair(srow(4, 8), srow(4, 9)), pair(srow(4, 10), srow(4, 11)),
    pair(srow(4, 12), srow(4, 13)), pair(srow(4, 14), srow(4, 15)), pair(srow(4, 16), srow(4, 17)),
    pair(srow(4, 18), srow(4, 19)), pair(srow(4, 20), srow(4, 21)), pair(srow(4, 22), srow(4, 23)),
    pair(srow(4, 24), wrow(4, 0)), pair(wrow(4, 1), wrow(4, 2)), pair(wrow(4, 3), wrow(4, 4)),
    pair(srow(3, 0), srow(3, 1)), pair(srow(3, 2), srow(3, 3)), pair(srow(3, 4), srow(3, 5)),
    pair(srow(3, 6), srow(3, 7)), pair(srow(3, 8), srow(3, 9)), pair(srow(3, 10), srow(3, 11)),
    pair(srow(3, 12), srow(3, 13)), pair(srow(3, 14), srow(3, 15)), pair(wrow(3, 0), wrow(3, 1)),
    pair(wrow(3, 2), wrow(3, 3)),
    pair(srow(2, 0), srow(2, 1)), pair(srow(2, 2), srow(2, 3)), pair(srow(2, 4), srow(2, 5)),
    pair(srow(2, 6), srow(2, 7)), pair(srow(2, 8), wrow(2, 0)), pair(wrow(2, 1), wrow(2, 2)),
    pair(srow(1, 0), srow(1, 1))};
static __constant__ unsigned kSlotB[32] = {  // the rest of order 1, order 0
    pair(srow(1, 2), srow(1, 3)), pair(wrow(1, 0), wrow(1, 1)), pair(srow(0, 0), wrow(0, 0)),
    kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone,
    kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone,
    kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone, kPairNone,
    kPairNone, kPairNone};

// the six fields of one row of d (rows are 48 bytes, 16-byte aligned)
__device__ __forceinline__ void load_d6(const double* p, double d[6]) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = q[0], b = q[1], c = q[2];
    d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y; d[4] = c.x; d[5] = c.y;
}

__device__ __forceinline__ void store_d6(double* p, const double d[6]) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(d[0], d[1]);
    q[1] = make_double2(d[2], d[3]);
    q[2] = make_double2(d[4], d[5]);
}

} // namespace rh3t
