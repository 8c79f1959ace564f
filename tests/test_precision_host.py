"""Melt-pool extents and the error report on host arrays."""
import numpy as np

from spectral_galerkin_heat_b200.precision import compare_fields, melt_pool, melt_pool_nodal


def test_melt_pool_extents():
    T = np.full((4, 5, 6), 300.0)
    T[3, 1:4, 2:5] = 2000.0   # top layer, 3 x 3 cells
    T[2, 2, 3] = 2000.0       # one cell below
    mp = melt_pool(T, 1.0, 2.0, 0.5, 1723.0)
    assert mp == {"length": 3.0, "width": 6.0, "depth": 1.0, "cells": 10}
    assert melt_pool(np.full((2, 2, 2), 300.0), 1, 1, 1, 1723.0)["cells"] == 0


def test_compare_fields():
    T = np.full((3, 3, 3), 300.0)
    T2 = T.copy()
    T2[2, 1, 1] = 301.0
    r = compare_fields(T2, T, (1.0, 1.0, 1.0), 1723.0)
    assert r["peak_T_err_K"] == 1.0
    assert abs(r["rel_l2"] - 1.0 / np.linalg.norm(T)) < 1e-15


def test_melt_pool_nodal_interpolates_the_isotherm():
    """A field linear in x, y and z: the interpolated crossings are exact."""
    nx, ny, nz = 10, 8, 5
    L = (1.0, 2.0, 0.5)
    x = np.linspace(0, L[0], nx + 1)[:, None, None]
    y = np.linspace(0, L[1], ny + 1)[None, :, None]
    z = np.linspace(0, L[2], nz + 1)[None, None, :]
    # hot where x < 0.37, y < 1.23, and within 0.21 of the top
    T = 1000.0 - 1000.0 * np.maximum.reduce([np.broadcast_to(x - 0.37, (nx + 1, ny + 1, nz + 1)),
                                             np.broadcast_to((y - 1.23) / 2, (nx + 1, ny + 1, nz + 1)),
                                             np.broadcast_to((L[2] - z) - 0.21, (nx + 1, ny + 1, nz + 1))])
    mp = melt_pool_nodal(T, L, 1000.0)
    assert abs(mp["length"] - 0.37) < 1e-12
    assert abs(mp["width"] - 1.23) < 1e-12
    assert abs(mp["depth"] - 0.21) < 1e-12
    assert melt_pool_nodal(np.full((3, 3, 3), 300.0), L, 1000.0) == {"length": 0.0, "width": 0.0,
                                                                      "depth": 0.0}
