"""Failure paths on the device, without a GPU fault: a non-finite field ends
the Picard loop with the "nonfinite" status; a bounded tensor-core wait that
can only run out records the batch's error flag, drains and returns, and the
context stays usable; and the per-iteration Picard history matches the
oracle's record of the same iterations (the reference's
``track_picard_history``)."""
import numpy as np
import pytest

from conftest import golden_case, make_context, rel_l2

pytestmark = pytest.mark.gpu


def _solver(cfg, path, **kw):
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    s = B200SpectralSolver(None, make_context(cfg, path), **kw)
    s.initialize()
    return s


@pytest.mark.parametrize("name", ["raster_32x16x8", "supergauss_20x18x5"])
def test_nonfinite_field_stops_the_picard_loop(name):
    """set_state with one NaN cell: the first residual is NaN, the convergence
    test stops the loop with SGH_STEP_NONFINITE after one iteration (the
    reference's ``rel < tol`` would never hold and it would run to the cap)."""
    cfg, path, *_ = golden_case(name)
    s = _solver(cfg, path)
    T = s.volume_temperature().cpu().numpy()
    T[T.shape[0] // 2, 1, 2] = np.nan
    s.set_state(T)
    dt = s.context.num.dt
    _, m = s.step(0.0, dt)
    assert s.last_status == "nonfinite"
    assert m["n_evap_iter"] == 1 and not m["picard_converged"]
    assert not np.isfinite(m["picard_rel_err"])
    # the plan is still usable: a reset brings back the initial condition
    s.reset()
    _, m = s.step(0.0, dt)
    assert s.last_status in ("converged", "capped") and np.isfinite(m["picard_rel_err"])
    s.finalize()


def _mixed_batch(n_steps):
    from spectral_galerkin_heat_b200 import workloads
    from spectral_galerkin_heat_b200.batch import BatchSolver
    from spectral_galerkin_heat_b200.laser import StraightTrack
    ctxs = []
    for nx, ny, nz in ((64, 32, 16), (128, 64, 16)):
        cfg, _ = workloads.straight_track(nx=nx, ny=ny, nz=nz, steps=n_steps,
                                          size=(2e-3 * nx / 64, 1e-3 * ny / 32, 0.5e-3))
        ctxs.append(make_context(cfg, StraightTrack(0.3e-3, cfg["domain"]["size"][1] / 2, 1.0,
                                                    0.0, 200.0)))
    b = BatchSolver(ctxs, "mixed")
    for i in range(len(ctxs)):
        b.start(i, n_steps)
    return b


def test_tensor_core_wait_runs_out_records_the_flag_and_returns():
    """Every face y-pass CTA first waits, with a bound of 2000 polls, on a
    barrier that nothing completes; each records the batch's error flag,
    waits for its bulk copies in flight (full bound), frees its tensor memory
    and returns. The host reads the flag; the context and a fresh batch still
    work."""
    import torch
    b = _mixed_batch(3)
    assert b.tensor_core_error() == 0
    b.set_wait_limit(2000, stall_test=True)
    b.step(1)
    b.synchronize()
    assert b.tensor_core_error() == 1
    b.set_wait_limit(0, stall_test=False)
    b.close()
    x = torch.arange(1024, device="cuda", dtype=torch.float64)
    assert float(x.sum()) == 1023 * 1024 / 2          # the context answers
    fresh = _mixed_batch(3)
    fresh.step(3)
    assert fresh.tensor_core_error() == 0
    assert all(int(st.step) == 3 for st in fresh.status())
    assert np.isfinite(fresh.modes(1).cpu().numpy()).all()
    fresh.close()


@pytest.mark.parametrize("name", ["raster_32x16x8", "box_tdep_16x12x8"])
def test_picard_history_matches_oracle(name):
    """rms of the residual, contraction ratio and relative residual of every
    Picard iteration of a step, against the oracle's record of the same step."""
    from oracle.sgh_oracle import OracleSolver
    cfg, path, *_ = golden_case(name)
    s = _solver(cfg, path)
    s.track_picard_history = True
    o = OracleSolver(make_context(cfg, path))
    o.initialize()
    o.track_picard_history = True
    dt = s.context.num.dt
    for i in range(3):
        _, m = s.step(i * dt, dt)
        o.step(i * dt, dt)
        h, ho = s.picard_history, o.picard_history
        assert len(h) == len(ho) == m["n_evap_iter"]
        assert [e["iter"] for e in h] == list(range(len(h)))
        # the residual near convergence is a difference of nearly equal fields,
        # so FP64 rounding differences (1e-16 of the field) are ~1e-8 of it
        got = np.array([[e["rms_diff"], e["true_rel_err"]] for e in h])
        ref = np.array([[e["rms_diff"], e["true_rel_err"]] for e in ho])
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=0.0)
        assert h[0]["rho"] is None and ho[0]["rho"] is None
        rho = np.array([e["rho"] for e in h[1:]])
        rho_o = np.array([e["rho"] for e in ho[1:]])
        np.testing.assert_allclose(rho, rho_o, rtol=1e-5)
        assert h[-1]["true_rel_err"] == pytest.approx(m["picard_rel_err"], rel=1e-15)
    s.finalize()
