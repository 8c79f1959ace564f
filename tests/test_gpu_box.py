"""Box mode (laser-following fine box) on the device, through the C ABI,
against the reference's outputs (golden fixtures made by running the
reference) and the CPU oracle. Needs a CUDA device.

Tolerance: FP64 throughout, relative L2 <= 1e-10 on the modes and on the box
temperature history, identical Picard counts, windows and truncation flags.
The latent source Q_prev is compared in max norm relative to its peak
(<= 1e-8): it is a difference of clipped liquid fractions scaled by
rho L / dt, so cells on the edge of the mushy band carry large, sharp values.
"""
import numpy as np
import pytest

from conftest import golden_case, load_golden, make_context, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-10
BOX_CASES = ["box_const_24x12x8", "box_shallow_24x12x8", "box_tdep_16x12x8", "box_full_r1_20x12x30",
             "tdep03_box_25x15x24", "gcode_box_24x12x8"]


def _solver(cfg, path, **kw):
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    s = B200SpectralSolver(None, make_context(cfg, path), **kw)
    s.initialize()
    return s


def _q_err(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("name", BOX_CASES)
def test_box_matches_reference_fixture(name):
    cfg, path, steps, snaps, block = golden_case(name)
    g = load_golden(name)
    s = _solver(cfg, path)
    fm = s.state.fine_mesh
    assert fm is not None and fm.box_shape == tuple(g["box_shape"])
    assert fm.T_prev is None and fm.window() == (-1, -1)
    dt = s.context.num.dt
    metrics, flags = [], []
    for i in range(steps):
        _, m = s.step(i * dt, dt)
        metrics.append(m)
        flags.append(s.last_flags)
        if (i + 1) in snaps:
            a = s.state.a.cpu().numpy()
            assert rel_l2(a, g[f"modes_step{i + 1}"]) < TOL, (name, i + 1)
            assert rel_l2(s.surface_temperature().cpu().numpy(), g[f"surface_step{i + 1}"]) < TOL
    np.testing.assert_array_equal([m["n_evap_iter"] for m in metrics], g["metric_n_evap_iter"])
    np.testing.assert_array_equal([float(m["picard_converged"]) for m in metrics],
                                  g["metric_picard_converged"])
    np.testing.assert_allclose([m["T_surface_max"] for m in metrics], g["metric_T_surface_max"],
                               rtol=TOL)
    assert fm.window() == tuple(g["box_window"])
    assert rel_l2(fm.T_prev.cpu().numpy(), g["box_T_prev"]) < TOL
    assert _q_err(fm.Q_prev.cpu().numpy(), g["box_Q_prev"]) < 1e-8
    np.testing.assert_array_equal(flags, g["box_flags"])
    assert s._latent_truncation_warned == bool(g["box_truncation_warned"])
    s.finalize()


@pytest.mark.parametrize("name", ["box_const_24x12x8", "box_tdep_16x12x8", "gcode_box_24x12x8"])
def test_box_run_eager_and_graph_agree(name):
    """The device-graph run (``run``), graph steps and eager steps give the same
    field and metrics (same kernels, same order)."""
    cfg, path, steps, *_ = golden_case(name)
    res = []
    for mode in ("run", "step", "eager"):
        s = _solver(cfg, path)
        dt = s.context.num.dt
        if mode == "run":
            ms = s.run(0.0, steps)
        else:
            ms = [s.step(i * dt, dt, eager=(mode == "eager"))[1] for i in range(steps)]
        res.append((s.state.a.cpu().numpy(), [m["n_evap_iter"] for m in ms],
                    s.state.fine_mesh.T_prev.cpu().numpy()))
        s.finalize()
    for a, it, T in res[1:]:
        assert rel_l2(a, res[0][0]) < 1e-13
        assert it == res[0][1]
        assert rel_l2(T, res[0][2]) < 1e-13


def test_box_functions_match_oracle():
    """``reconstruct_temperature_box`` / ``project_box_to_modes`` on random modes
    and a random box field, at the window of the last step."""
    import torch
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200 import kernels
    cfg, path, *_ = golden_case("box_const_24x12x8")
    s = _solver(cfg, path)
    o = OracleSolver(make_context(cfg, path))
    o.initialize()
    dt = s.context.num.dt
    for i in range(3):
        s.step(i * dt, dt)
        o.step(i * dt, dt)
    assert s.state.fine_mesh.window() == o.box.window
    rng = np.random.default_rng(5)
    a = rng.standard_normal(s.state.shape)
    f = rng.standard_normal(o.box.shape)
    T = kernels.reconstruct_temperature_box(torch.as_tensor(a, device="cuda"), s.state).cpu().numpy()
    M = kernels.project_box_to_modes(torch.as_tensor(f, device="cuda"), s.state).cpu().numpy()
    assert rel_l2(T, o.box.reconstruct(a)) < 1e-13
    assert rel_l2(M, o.box.project(f)) < 1e-13
    # the bases: B_fine_full views against the oracle's tables
    for ax in range(3):
        got = s.state.fine_mesh.B_fine_full[ax].cpu().numpy()
        ref = o.box.B_fine_full[ax][:, :got.shape[1]]
        assert np.max(np.abs(got - ref)) <= 4 * np.finfo(np.float64).eps * np.max(np.abs(ref))
    s.finalize()


def test_box_refinement1_full_domain_matches_grid_mode():
    """Grid mode == box mode at refinement 1 over the whole domain: both evaluate
    the latent source at the same cell centres (the equivalence the reference
    tests in tests/integration/test_latent_grid_mode.py:57-96; same tolerance
    on the node-centred field, same Picard counts)."""
    import copy
    from spectral_galerkin_heat_b200 import kernels
    cfg, path, steps, *_ = golden_case("box_full_r1_20x12x30")
    grid = copy.deepcopy(cfg)
    grid.pop("fine_mesh")
    out = []
    for c in (grid, cfg):
        s = _solver(c, path)
        dt = s.context.num.dt
        ms = [s.step(i * dt, dt)[1] for i in range(steps)]
        assert all(m["picard_converged"] for m in ms)
        assert (s.state.fine_mesh is None) == (c is grid) and s._grid_latent == (c is grid)
        T = kernels.reconstruct_temperature_DCT(s.state.a, s.state).cpu().numpy()
        out.append((T, [m["n_evap_iter"] for m in ms]))
        s.finalize()
    (Tg, ig), (Tb, ib) = out
    assert Tg.max() > 1697.15
    np.testing.assert_allclose(Tg, Tb, rtol=1e-3, atol=0.2)
    assert ig == ib


def test_box_reset_and_dt_guard():
    cfg, path, *_ = golden_case("box_const_24x12x8")
    s = _solver(cfg, path)
    dt = s.context.num.dt
    s.step(0.0, dt)
    first = s.state.a.cpu().numpy()
    assert s.state.fine_mesh.T_prev is not None
    s.step(dt, dt)
    s.reset()
    assert s.state.fine_mesh.T_prev is None and s.state.fine_mesh.window() == (-1, -1)
    s.step(0.0, dt)
    assert rel_l2(s.state.a.cpu().numpy(), first) < 1e-14
    with pytest.raises(ValueError):
        s.step(dt, 0.5 * dt)
    s.finalize()
