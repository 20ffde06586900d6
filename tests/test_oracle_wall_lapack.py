"""The oracle's Wall ILW solve against LAPACK, the library the reference calls
(bc1.rs:467-469: ndarray-linalg `solve_into`, LAPACK dgesv = dgetrf +
dgetrs).

The oracle restates dgesv as an LU factorisation with partial pivoting
(oracle/src/solver.cpp solve6). Here it is held to LAPACK as numpy and scipy
ship it (scipy.linalg.lu_factor = dgetrf, numpy.linalg.solve = dgesv):

  - every 6x6 system the ghost update solves on the Wall ghosts of a
    developed double Mach reflection (both ILW systems of each ghost): the
    same pivot sequence as dgetrf, and the same solution to a few units of
    the last place;
  - integer matrices with ties in the pivot column, where the first pivot
    choice rests on the tie rule alone (the first maximal |a_ij|, as
    LAPACK's idamax takes it): the same pivots up to the first step whose
    choice is a rounding-level tie (dgetrf's trailing update may round
    differently there), and the same solution.
"""
import numpy as np
import pytest

scipy_linalg = pytest.importorskip("scipy.linalg")


def _pivots(A):
    """the row interchanges of solve6 (first maximal |a_ij| of the column,
    the column scaled by the pivot's reciprocal, the trailing update one
    product and one difference per entry), as 0-based dgetrf ipiv; and per
    step whether the choice is decided by more than rounding (the largest
    magnitude ahead of the next by 1e-9 relative, or an exact tie of the
    input's own entries at the first step)"""
    A = np.array(A, dtype=np.float64)
    piv, decided = [], []
    for j in range(6):
        col = np.abs(A[j:, j])
        p = j + int(np.argmax(col))  # argmax returns the first maximum
        top = np.sort(col)[::-1]
        decided.append(j == 0 or len(top) == 1 or top[0] - top[1] > 1e-9 * top[0])
        piv.append(p)
        if p != j:
            A[[j, p]] = A[[p, j]]
        A[j + 1:, j] *= 1.0 / A[j, j]
        A[j + 1:, j + 1:] -= np.outer(A[j + 1:, j], A[j, j + 1:])
    return piv, decided


def _check(O, A, b):
    x = O.solve6(A, b)
    assert x is not None
    _, ipiv = scipy_linalg.lu_factor(A)
    piv, decided = _pivots(A)
    for j in range(6):
        if decided[j]:
            assert ipiv[j] == piv[j], (j, list(ipiv), piv)
        else:  # a rounding-level tie: the two factorisations may round differently
            break
    xl = np.linalg.solve(A, b)
    return np.abs(x - xl).max() / np.abs(xl).max()


def test_wall_ilw_systems_match_lapack(O):
    c = O.Case.double_mach(h=1.0 / 40.0)
    c.run(10, 0.05)
    gi = c.ghost_info()
    n, worst = 0, 0.0
    for gid in np.flatnonzero(gi["pre"] >= 0):
        try:
            sysm = c.wall_systems(int(gid))
        except ValueError:  # not a Wall ghost
            continue
        assert sysm is not None
        A0, b0, A1, b1 = sysm
        for A, b in ((A0, b0), (A1, b1)):
            worst = max(worst, _check(O, A, b))
            n += 1
    print(f"{n} Wall ILW systems: max relative difference from LAPACK dgesv {worst:.2e}")
    assert n > 500
    assert worst <= 1e-14


def test_pivot_ties_match_lapack(O):
    rng = np.random.default_rng(20261204)
    for _ in range(200):
        A = rng.integers(-3, 4, size=(6, 6)).astype(np.float64)
        if abs(np.linalg.det(A)) < 0.5:
            continue
        b = rng.integers(-5, 6, size=6).astype(np.float64)
        assert _check(O, A, b) <= 1e-13
