"""The mixed-precision form of the nonlinear volume step (latent heat in grid
and box mode, the T-dependent property correction): every DCT contraction as
split-BF16 products on the tensor cores (tcgen05), modal iterates in FP32,
the latent source, property correction, face fluxes and Picard norms in FP64.
Checked against the reference's own outputs (golden fixtures) and the FP64
plan. Tolerance: relative L2 <= 1e-4 on the modes, the bound stated for the
mixed forms."""
import numpy as np
import pytest
import scipy.fft

from conftest import golden_case, load_golden, make_context, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _solver(cfg, path, precision, **kw):
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    s = B200SpectralSolver(None, make_context(cfg, path), precision=precision, **kw)
    s.initialize()
    return s


def test_mixed_dct3d_matches_scipy():
    """The split-BF16 3-D transforms of a mixed plan: relative error of the
    order of the BF16 split (2^-16 per operand, FP32 accumulation)."""
    import torch
    cfg, path, *_ = golden_case("raster_32x16x8")
    s = _solver(cfg, path, "mixed")
    x = np.random.default_rng(3).standard_normal(s.state.shape)
    for kind in (2, 3):
        got = s.dct3d(torch.as_tensor(x, device="cuda"), kind).cpu().numpy()
        ref = scipy.fft.dctn(x, type=kind, norm="ortho")
        assert rel_l2(got, ref) < 2e-5
    s.finalize()


@pytest.mark.parametrize("mesh", [(300, 40, 20), (128, 80, 100), (33, 17, 129)])
def test_mixed_dct3d_tiles_and_ring(mesh):
    """Shapes that reach every tile path of the split-BF16 pass: 300 outputs
    (three 128-row tiles, a ragged last one), contraction lengths of 100 to
    300 slices (more 32-slice chunks than ring stages, so stages are refilled
    while MMAs run), 16-, 32- and 64-column tiles, and ragged columns."""
    import copy
    import torch
    cfg, path, *_ = golden_case("raster_32x16x8")
    cfg = copy.deepcopy(cfg)
    cfg["domain"]["mesh"] = list(mesh)
    s = _solver(cfg, path, "mixed")
    x = np.random.default_rng(sum(mesh)).standard_normal(s.state.shape)
    for kind in (2, 3):
        got = s.dct3d(torch.as_tensor(x, device="cuda"), kind).cpu().numpy()
        ref = scipy.fft.dctn(x, type=kind, norm="ortho")
        assert rel_l2(got, ref) < 2e-5, (mesh, kind, rel_l2(got, ref))
    s.finalize()


@pytest.mark.parametrize("name", ["raster_32x16x8", "tdep03_grid_25x15x24", "box_tdep_16x12x8",
                                  "tdep03_box_25x15x24"])
def test_mixed_volume_form_matches_reference(name):
    cfg, path, steps, snaps, block = golden_case(name)
    g = load_golden(name)
    s = _solver(cfg, path, "mixed")
    dt = s.context.num.dt
    for i in range(steps):
        _, m = s.step(i * dt, dt)
        assert s.last_status in ("converged", "capped"), s.last_status
        if (i + 1) in snaps:
            a = s.state.a.cpu().numpy()
            ref = g[f"modes_step{i + 1}"]
            got = a if block is None else a[:block[0], :block[1], :block[2]]
            assert rel_l2(got, ref) < TOL, (name, i + 1, rel_l2(got, ref))
            # the modal state is FP32
            assert np.array_equal(a, a.astype(np.float32).astype(np.float64))
    # a pointwise peak: held to the mixed forms' peak-temperature bound (1 K),
    # not to the L2 bound of the modes
    assert abs(m["T_surface_max"] - g["metric_T_surface_max"][steps - 1]) < 1.0
    s.finalize()


def test_mixed_matches_fp64_plan_on_the_c2_grid():
    """128 x 64 x 32 (the C2 grid), first steps of the raster: mixed against
    the FP64 plan, with the Picard tolerance at 1e-5 for the mixed plan (its
    residual floor is near 1e-6; at 1e-8 it would run every step to the cap)."""
    from spectral_galerkin_heat_b200 import workloads
    cfg, path = workloads.nonlinear_raster(steps=4)
    f64 = _solver(cfg, path, "fp64")
    mix = _solver(cfg, path, "mixed", convergence_tol=1e-5)
    dt = f64.context.num.dt
    for i in range(4):
        _, m64 = f64.step(i * dt, dt)
        _, mmx = mix.step(i * dt, dt)
        assert mix.last_status == "converged"
    assert rel_l2(mix.state.a.cpu().numpy(), f64.state.a.cpu().numpy()) < TOL
    assert abs(mmx["T_surface_max"] - m64["T_surface_max"]) < 1e-3 * m64["T_surface_max"]
    f64.finalize()
    mix.finalize()
