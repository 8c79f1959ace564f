"""Parity of the CUDA path (through the C ABI) with the reference's outputs
(golden fixtures) and with the CPU oracle. Needs a CUDA device.

Tolerance: the plain path is FP64 throughout and must match the reference to
relative L2 <= 1e-10 on the modes (the stated target), with identical Picard
iteration counts.
"""
import numpy as np
import pytest
import scipy.fft

from conftest import golden_case, load_golden, make_context, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-10

GOLDEN = ["track_64x32x16", "raster_32x16x8", "odd_13x10x6_conv", "latent_const_24x12x8",
          "supergauss_20x18x5", "laser_off_8x6x4", "raster_128x64x32", "tdep03_grid_25x15x24",
          "gcode_track_30x16x8"]


def _solver(cfg, path):
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    s = B200SpectralSolver(None, make_context(cfg, path))
    s.initialize()
    return s


@pytest.mark.parametrize("shape", [(1,), (5,), (64,), (3, 5), (64, 128), (17, 33), (4, 5, 6),
                                   (16, 32, 64), (3, 1, 7), (32, 64, 128)])
@pytest.mark.parametrize("kind", [2, 3])
def test_dctn_matches_scipy(shape, kind):
    import torch
    from spectral_galerkin_heat_b200 import kernels
    x = np.random.default_rng(len(shape) * 100 + sum(shape)).standard_normal(shape)
    fn = kernels.DCT_II if kind == 2 else kernels.IDCT_II
    got = fn(torch.as_tensor(x, device="cuda")).cpu().numpy()
    ref = scipy.fft.dctn(x, type=kind, norm="ortho")
    assert rel_l2(got, ref) < 1e-14
    assert np.max(np.abs(got - ref)) < 1e-13 * max(1.0, np.max(np.abs(ref)))


def test_tables_and_initial_state():
    from oracle.sgh_oracle import OracleSolver
    cfg, path, *_ = golden_case("odd_13x10x6_conv")
    s = _solver(cfg, path)
    o = OracleSolver(make_context(cfg, path))
    o.initialize()
    assert rel_l2(s.state.K.cpu().numpy(), o.K) < 1e-15
    assert rel_l2(s.state.KK.cpu().numpy(), o.KK) < 1e-15
    a = s.state.a.cpu().numpy()
    assert a[0, 0, 0] == pytest.approx(o.a[0, 0, 0], rel=1e-15)
    assert np.count_nonzero(a) == 1
    T0 = float(s.context.mat.T0)
    np.testing.assert_allclose(s.surface_temperature().cpu().numpy(), T0, rtol=1e-13)
    np.testing.assert_allclose(s.volume_temperature().cpu().numpy(), T0, rtol=1e-13)
    s.finalize()


@pytest.mark.parametrize("name", GOLDEN)
def test_matches_reference_fixture(name):
    cfg, path, steps, snaps, block = golden_case(name)
    g = load_golden(name)
    s = _solver(cfg, path)
    dt = s.context.num.dt
    upto = 60 if name == "track_64x32x16" else steps
    metrics = []
    for i in range(upto):
        _, m = s.step(i * dt, dt)
        metrics.append(m)
        if (i + 1) in snaps:
            a = s.state.a.cpu().numpy()
            ref = g[f"modes_step{i + 1}"]
            got = a if block is None else a[:block[0], :block[1], :block[2]]
            err = rel_l2(got, ref)
            assert err < TOL, (name, i + 1, err)
            surf = s.surface_temperature().cpu().numpy()
            assert rel_l2(surf, g[f"surface_step{i + 1}"]) < TOL
    n = len(metrics)
    np.testing.assert_array_equal([m["n_evap_iter"] for m in metrics], g["metric_n_evap_iter"][:n])
    np.testing.assert_array_equal([float(m["picard_converged"]) for m in metrics],
                                  g["metric_picard_converged"][:n])
    np.testing.assert_allclose([m["T_surface_max"] for m in metrics], g["metric_T_surface_max"][:n],
                               rtol=TOL)
    np.testing.assert_allclose([m["P_laser"] for m in metrics], g["metric_P_laser"][:n], rtol=1e-12)
    s.finalize()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_matches_live_oracle_seeded_raster(seed):
    """Seeded raster jitter, reduced mode counts, against the oracle run now."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200 import workloads
    nx, ny, nz = [(24, 12, 6), (20, 16, 10), (30, 14, 8)][seed - 1]
    cfg, path = workloads.nonlinear_raster(nx=nx, ny=ny, nz=nz, seed=seed,
                                           size=(0.5e-3, 0.25e-3, 0.125e-3),
                                           line_length=0.1e-3, hatch=25e-6, steps=12)
    s = _solver(cfg, path)
    o = OracleSolver(make_context(cfg, path))
    o.initialize()
    dt = s.context.num.dt
    for i in range(12):
        _, m = s.step(i * dt, dt)
        _, mo = o.step(i * dt, dt)
        assert m["n_evap_iter"] == mo["n_evap_iter"]
    assert rel_l2(s.state.a.cpu().numpy(), o.a) < TOL
    assert rel_l2(s.state.T_prev.cpu().numpy(), o.T_prev_full) < TOL
    s.finalize()


def test_run_equals_step():
    """The multi-step device run (laser table, one launch) gives the same bits as step()."""
    cfg, path, *_ = golden_case("raster_32x16x8")
    a = _solver(cfg, path)
    b = _solver(cfg, path)
    dt = a.context.num.dt
    ms = [a.step(i * dt, dt)[1] for i in range(10)]
    mr = b.run(0.0, 10)
    assert np.array_equal(a.state.a.cpu().numpy(), b.state.a.cpu().numpy())
    assert [m["n_evap_iter"] for m in ms] == [m["n_evap_iter"] for m in mr]
    assert [m["T_surface_max"] for m in ms] == [m["T_surface_max"] for m in mr]
    a.finalize()
    b.finalize()


def test_full_size_roundtrip_and_laser_off():
    """Full 128x64x32 grid: set_state / reconstruction round trip, and a laser
    that is off keeps the field at T0 (size-independent properties)."""
    from spectral_galerkin_heat_b200 import workloads
    from spectral_galerkin_heat_b200.laser import FixedLaser
    cfg, _ = workloads.nonlinear_raster(steps=5)
    s = _solver(cfg, FixedLaser(1e-3, 0.5e-3, 200.0, is_on=False))
    T = 300.0 + 50.0 * np.random.default_rng(0).random(s.state.shape)
    s.set_state(T)
    assert rel_l2(s.volume_temperature().cpu().numpy(), T) < 1e-13
    s.reset()
    dt = s.context.num.dt
    for i in range(3):
        _, m = s.step(i * dt, dt)
        assert m["P_laser"] == 0.0
    np.testing.assert_allclose(s.volume_temperature().cpu().numpy(), 300.0, rtol=1e-12)
    s.finalize()


def test_dctn_alias_in_place():
    import torch
    from spectral_galerkin_heat_b200 import _lib
    import ctypes as C
    x = torch.as_tensor(np.random.default_rng(5).standard_normal(37), device="cuda")
    ref = scipy.fft.dct(x.cpu().numpy(), type=2, norm="ortho")
    shape = (C.c_int32 * 1)(37)
    n = C.c_uint64()
    L = _lib.lib()
    assert L.sgh_dctn_workspace_bytes(1, shape, C.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    assert L.sgh_dctn(2, 1, shape, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                      C.c_void_p(ws.data_ptr()), n.value, None) == 0
    torch.cuda.synchronize()
    assert rel_l2(x.cpu().numpy(), ref) < 1e-14


@pytest.mark.parametrize("which", ["precision_256x128x64", "serving_512x256x64"])
def test_large_grid_matches_live_oracle(which):
    """The largest grids the benchmarks step, in FP64, against the oracle run now:
    the 256x128x64 precision-study track (4 x 2 x 1 mm, seeded power and speed)
    and the largest serving class, 512x256x64 on the 2 x 1 x 0.5 mm cuboid with
    a serving raster. One forcing pass per step; 10 steps stay well inside the
    range over which this explicit scheme is not chaotic (about 60 steps)."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200 import workloads
    from spectral_galerkin_heat_b200.laser import RasterPath
    steps = 10
    if which.startswith("precision"):
        cfg, path = workloads.precision_track(seed=0, steps=steps)
    else:
        cfg = workloads.serving_config(512, 256, 64)
        cfg["simulation"]["duration"] = steps * cfg["simulation"]["dt"]
        path = RasterPath(0.25e-3, 0.2e-3, 1.5e-3, 50e-6, 2, 1.3, 350.0)
    s = _solver(cfg, path)
    o = OracleSolver(make_context(cfg, path))
    o.initialize()
    dt = s.context.num.dt
    for i in range(steps):
        _, m = s.step(i * dt, dt)
        _, mo = o.step(i * dt, dt)
        assert m["n_evap_iter"] == mo["n_evap_iter"]
        assert m["T_surface_max"] == pytest.approx(mo["T_surface_max"], rel=TOL)
        assert m["P_laser"] == pytest.approx(mo["P_laser"], rel=1e-12)
    assert mo["T_surface_max"] > 1000.0          # the beam has heated the surface
    assert rel_l2(s.state.a.cpu().numpy(), o.a) < TOL
    assert rel_l2(s.surface_temperature().cpu().numpy(), o.surface_T(o.a, top=True)) < TOL
    s.finalize()
