"""Autotuner on the device: it times the candidates on the real step and
returns one of them; a plan built with any tile policy computes the same
step (the policy only changes the tiling, i.e. the rounding order)."""
import numpy as np
import pytest

from conftest import golden_case, make_context, rel_l2

pytestmark = pytest.mark.gpu


def test_tune_returns_a_candidate_and_policies_agree():
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    from spectral_galerkin_heat_b200.autotune import tune
    cfg, path, *_ = golden_case("raster_32x16x8")
    ctx = make_context(cfg, path)
    r = tune(ctx, candidates=(1, 1 << 30), steps=3, warmup=2)
    assert r["axis_min_ctas"] in (1, 1 << 30) and r["axis_cuda_cores"] in (0, 1)
    assert len(r["candidates"]) == 4
    assert all(v["ms_per_iter"] > 0 for v in r["candidates"].values())
    modes = []
    for policy, cores in ((1, False), (1 << 30, False), (1, True), (1 << 30, True)):
        s = B200SpectralSolver(None, make_context(cfg, path), axis_min_ctas=policy, axis_cuda_cores=cores)
        s.initialize()
        assert s.tile_policy == policy and s.kernel_policy == int(cores)
        dt = s.context.num.dt
        for k in range(5):
            s.step(k * dt, dt)
        modes.append(s.state.a.cpu().numpy())
        s.finalize()
    for m in modes[1:]:
        assert rel_l2(m, modes[0]) < 1e-12
