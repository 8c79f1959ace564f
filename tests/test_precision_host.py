"""Melt-pool extents and the error report on host arrays."""
import numpy as np

from spectral_galerkin_heat_b200.precision import compare_fields, melt_pool


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
