"""Modal checkpoints: an instance restored from a checkpoint continues exactly
as the instance that wrote it (same kernels, same inputs, deterministic
reductions), in grid mode with latent heat and the property correction, in
box mode and on the face-space path. Needs a CUDA device."""
import numpy as np
import pytest

from conftest import golden_case, make_context

pytestmark = pytest.mark.gpu

CASES = ["raster_32x16x8", "box_tdep_16x12x8", "box_const_24x12x8", "track_64x32x16"]


def _solver(name):
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    cfg, path, *_ = golden_case(name)
    s = B200SpectralSolver(None, make_context(cfg, path))
    s.initialize()
    return s


@pytest.mark.parametrize("name", CASES)
def test_restore_resumes_exactly(name, tmp_path):
    a = _solver(name)
    dt = a.context.num.dt
    k, m = 3, 3
    for i in range(k):
        a.step(i * dt, dt)
    f = a.save_checkpoint(tmp_path / "ck", t=k * dt, step=k)
    ck = a.checkpoint(t=k * dt, step=k)
    # the reference's modes.h5 layout for the modes
    assert ck["modes"].shape == (1, *a.state.shape) and ck["time"].shape == (1,) and ck["step"][0] == k
    ma = [a.step((k + i) * dt, dt)[1] for i in range(m)]
    end_a = a.state.a.cpu().numpy()

    b = _solver(name)
    t0, step0 = b.load_checkpoint(f)
    assert (t0, step0) == (k * dt, k)
    if b.state.fine_mesh is not None:
        assert b.state.fine_mesh.T_prev is not None
    mb = [b.step((k + i) * dt, dt)[1] for i in range(m)]
    np.testing.assert_array_equal(b.state.a.cpu().numpy(), end_a)
    assert [x["n_evap_iter"] for x in ma] == [x["n_evap_iter"] for x in mb]
    assert [x["T_surface_max"] for x in ma] == [x["T_surface_max"] for x in mb]
    a.finalize()
    b.finalize()


def test_restore_rejects_another_configuration():
    a = _solver("raster_32x16x8")
    ck = a.checkpoint()
    b = _solver("box_const_24x12x8")
    with pytest.raises(ValueError):
        b.restore(ck)
    a.finalize()
    b.finalize()


def test_fresh_state_checkpoint_flags():
    """Before the first step no warm start is present; after one latent step it is."""
    a = _solver("box_const_24x12x8")
    assert int(a.checkpoint()["flags"]) == 0
    a.step(0.0, a.context.num.dt)
    assert int(a.checkpoint()["flags"]) & 2
    a.finalize()
