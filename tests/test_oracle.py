"""The CPU oracle against the reference's own outputs (golden fixtures) and
against the published DCT definition. CPU only."""
import numpy as np
import pytest
import scipy.fft

from conftest import golden_case, load_golden, make_context, rel_l2
from oracle.sgh_oracle import OracleSolver, dct2, dct3, dct_matrix

# Oracle vs reference on identical inputs: same FP64 algorithm, differing only
# in library summation order, so the bound is a few ulps times the step count.
TOL_ORACLE = 1e-12

BOX_CASES = ["box_const_24x12x8", "box_shallow_24x12x8", "box_tdep_16x12x8", "box_full_r1_20x12x30",
             "tdep03_box_25x15x24", "gcode_box_24x12x8"]
CASES = ["track_64x32x16", "raster_32x16x8", "odd_13x10x6_conv", "latent_const_24x12x8",
         "supergauss_20x18x5", "laser_off_8x6x4", "raster_128x64x32",
         "tdep03_grid_25x15x24", "gcode_track_30x16x8"] + BOX_CASES


def _run_oracle(name, upto=None):
    cfg, path, steps, snaps, block = golden_case(name)
    ctx = make_context(cfg, path)
    o = OracleSolver(ctx)
    o.initialize()
    g = load_golden(name)
    n = steps if upto is None else upto
    metrics = []
    snap_modes = {}
    flags = []
    for i in range(n):
        _, m = o.step(i * ctx.num.dt, ctx.num.dt)
        metrics.append(m)
        flags.append(o.box_flags)
        if (i + 1) in snaps:
            snap_modes[i + 1] = o.a.copy()
    if o.box is not None:
        snap_modes["box"] = (o.box, flags)
    return g, metrics, snap_modes, block


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_fixture(name):
    upto = 60 if name == "track_64x32x16" else None
    g, metrics, snaps, block = _run_oracle(name, upto)
    box = snaps.pop("box", None)
    if box is not None:
        fb, flags = box
        # box history, window and truncation flags after the last step
        assert tuple(g["box_shape"]) == fb.shape
        assert tuple(g["box_window"]) == fb.window
        assert rel_l2(fb.T_prev, g["box_T_prev"]) < TOL_ORACLE
        assert np.max(np.abs(fb.Q_prev - g["box_Q_prev"])) <= 1e-9 * np.max(np.abs(g["box_Q_prev"]))
        np.testing.assert_array_equal(flags, g["box_flags"])
        assert bool(g["box_truncation_warned"]) == any(flags)
    for step, a in snaps.items():
        ref = g[f"modes_step{step}"]
        got = a if block is None else a[:block[0], :block[1], :block[2]]
        assert rel_l2(got, ref) < TOL_ORACLE, (name, step)
        assert abs(np.linalg.norm(a) / float(g[f"modes_norm_step{step}"]) - 1) < TOL_ORACLE
    n = len(metrics)
    np.testing.assert_array_equal([m["n_evap_iter"] for m in metrics], g["metric_n_evap_iter"][:n])
    np.testing.assert_array_equal([float(m["picard_converged"]) for m in metrics],
                                  g["metric_picard_converged"][:n])
    np.testing.assert_allclose([m["T_surface_max"] for m in metrics], g["metric_T_surface_max"][:n],
                               rtol=1e-12)
    np.testing.assert_allclose([m["P_laser"] for m in metrics], g["metric_P_laser"][:n], rtol=1e-12)


def test_track_is_chaotic_beyond_60_steps():
    """One explicit forcing pass per step (max_picard_iter=1, omega=1) makes the
    evaporation feedback oscillate; a 1e-15 relative perturbation of the initial
    modes grows to O(1e-3) over 300 steps. No FP64 implementation with a
    different rounding can therefore match the reference there, and parity for
    this workload is checked over the first 60 steps."""
    cfg, path, *_ = golden_case("track_64x32x16")
    runs = []
    for eps in (0.0, 1e-15):
        ctx = make_context(cfg, path)
        o = OracleSolver(ctx)
        o.initialize()
        o.a[0, 0, 0] *= 1.0 + eps
        errs = {}
        base = None
        for i in range(300):
            o.step(i * ctx.num.dt, ctx.num.dt)
            if i + 1 in (60, 300):
                errs[i + 1] = o.a.copy()
        runs.append(errs)
    assert rel_l2(runs[1][60], runs[0][60]) < 1e-11
    assert rel_l2(runs[1][300], runs[0][300]) > 1e-6


@pytest.mark.parametrize("n", [1, 2, 3, 7, 16, 33, 64])
def test_dct_matrix_matches_scipy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    M = dct_matrix(n)
    np.testing.assert_allclose(M @ x, scipy.fft.dct(x, type=2, norm="ortho"), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(M.T @ x, scipy.fft.dct(x, type=3, norm="ortho"), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(M @ M.T, np.eye(n), atol=1e-13)


def test_dct_of_ones_is_impulse():
    # reference tests/unit_tests/physics/test_spectral_cpu_kernels.py:24-32
    out = dct2(np.ones((4, 4, 4)))
    assert out[0, 0, 0] == pytest.approx(4 ** 1.5, rel=1e-12)
    out[0, 0, 0] = 0.0
    assert np.allclose(out, 0.0, atol=1e-12)


def test_dct_roundtrip():
    x = np.random.default_rng(0).standard_normal((5, 6, 7))
    np.testing.assert_allclose(dct3(dct2(x)), x, atol=1e-13)


def test_propagators_known_values():
    # reference tests/unit_tests/physics/test_spectral_state.py:35-62
    from spectral_galerkin_heat_b200.config import MaterialParams
    mat = MaterialParams(rho=7900.0, k=15.0, Cp=500.0)
    dt = 1e-6
    K, KK = OracleSolver.propagators(mat, dt, (4, 6, 8), (1e-3, 2e-3, 4e-3))
    alpha = 15.0 / (7900.0 * 500.0)
    assert K[0, 0, 0] == 1.0
    assert KK[0, 0, 0] == pytest.approx(dt / (7900.0 * 500.0), rel=1e-15)
    assert K[1, 0, 0] == pytest.approx(np.exp(-alpha * (np.pi / 1e-3) ** 2 * dt), rel=1e-14)
    assert K[0, 0, 1] == pytest.approx(np.exp(-alpha * (np.pi / 4e-3) ** 2 * dt), rel=1e-14)
    assert K.shape == (4, 6, 8)


@pytest.mark.parametrize("name", ["outputs_odd_13x10x6", "outputs_raster_32x16x8"])
def test_output_reconstruction_matches_reference_fixtures(name):
    """The oracle's node field, point values and profiles equal the reference's
    (physics/spectral_helpers.py:146-333) on the fixture's modes."""
    from oracle.sgh_oracle import OracleSolver, nodal_temperature, points_temperature, temp_profiles
    g = load_golden(name)
    a, L = g["modes"], tuple(g["lengths"])
    assert rel_l2(nodal_temperature(a, L), g["nodal"]) < 1e-13
    assert rel_l2(points_temperature(a, L, g["coords"]), g["points"]) < 1e-13
    nz, ny, nx = a.shape
    surface = None
    for center in ("laser", "hotspot"):
        if center == "hotspot":
            case = name.replace("outputs_", "")
            cfg, path, *_ = golden_case({"odd_13x10x6": "odd_13x10x6_conv"}.get(case, case))
            o = OracleSolver(make_context(cfg, path))
            o.initialize()
            surface = o.surface_T(a, top=True)
        prof = temp_profiles(a, L, surface, tuple(g["laser_position"]), center=center, num_points=40)
        for key in "xyz":
            np.testing.assert_allclose(prof[key][0], g[f"profile_{center}_{key}_coords"], rtol=0, atol=0)
            assert rel_l2(prof[key][1], g[f"profile_{center}_{key}_T"]) < 1e-13


def test_points_reject_bad_shapes():
    from oracle.sgh_oracle import points_temperature
    with pytest.raises(ValueError, match=r"\(N, 3\)"):
        points_temperature(np.zeros((2, 2, 2)), (1.0, 1.0, 1.0), np.zeros((4, 2)))


def test_nodal_dct1_form_equals_series_form():
    from oracle.sgh_oracle import nodal_temperature, nodal_temperature_dct1
    g = load_golden("outputs_odd_13x10x6")
    a, L = g["modes"], tuple(g["lengths"])
    assert rel_l2(nodal_temperature_dct1(a, L), g["nodal"]) < 1e-13
    assert rel_l2(nodal_temperature_dct1(a, L), nodal_temperature(a, L)) < 1e-13
