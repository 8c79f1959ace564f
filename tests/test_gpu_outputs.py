"""Output reconstruction on the device (sgh_nodal_temperature,
sgh_points_temperature, and the profiles on top of them) against the
reference's own outputs (fixtures made by tests/golden/make_golden.py from
physics/spectral_helpers.py:146-333) and against the oracle."""
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import golden_case, load_golden, make_context, rel_l2

pytestmark = pytest.mark.gpu

CASES = {"outputs_odd_13x10x6": "odd_13x10x6_conv", "outputs_raster_32x16x8": "raster_32x16x8"}


@pytest.mark.parametrize("name", sorted(CASES))
def test_outputs_match_reference_fixtures(name):
    import torch

    from spectral_galerkin_heat_b200 import B200SpectralSolver
    from spectral_galerkin_heat_b200 import kernels as K
    g = load_golden(name)
    cfg, path, *_ = golden_case(CASES[name])
    s = B200SpectralSolver(None, make_context(cfg, path))
    state = s.initialize()
    a = torch.as_tensor(g["modes"], device="cuda")
    nodal = K.reconstruct_temperature_DCT(a, state)
    assert tuple(nodal.shape) == g["nodal"].shape
    assert rel_l2(nodal.cpu().numpy(), g["nodal"]) < 1e-12
    pts = K.reconstruct_temperature_volume_at_points(a, s.context.num, s.context.geom, state, g["coords"])
    assert rel_l2(pts.cpu().numpy(), g["points"]) < 1e-12
    for center in ("laser", "hotspot"):
        prof = K.save_temp_profiles(a, s.context.num, s.context.geom, state, tuple(g["laser_position"]),
                                    center=center, num_points=40)
        for key in "xyz":
            np.testing.assert_array_equal(prof[key][0], g[f"profile_{center}_{key}_coords"])
            assert rel_l2(prof[key][1].cpu().numpy(), g[f"profile_{center}_{key}_T"]) < 1e-12
    s.finalize()


def test_outputs_match_oracle_on_a_larger_random_field():
    import torch

    from oracle.sgh_oracle import nodal_temperature, points_temperature
    from spectral_galerkin_heat_b200 import kernels as K
    rng = np.random.default_rng(3)
    L = (2e-3, 1.3e-3, 0.7e-3)
    a = rng.standard_normal((24, 40, 64)) * np.exp(-0.05 * np.arange(64))[None, None, :]
    st = SimpleNamespace(size=L)
    ad = torch.as_tensor(a, device="cuda")
    assert rel_l2(K.reconstruct_temperature_DCT(ad, st).cpu().numpy(), nodal_temperature(a, L)) < 1e-12
    coords = rng.uniform(-0.2, 1.2, size=(777, 3)) * np.array(L)
    geom = SimpleNamespace(size=SimpleNamespace(x=L[0], y=L[1], z=L[2]))
    got = K.reconstruct_temperature_volume_at_points(ad, None, geom, st, coords).cpu().numpy()
    assert rel_l2(got, points_temperature(a, L, coords)) < 1e-12


def test_outputs_argument_errors():
    import torch

    from spectral_galerkin_heat_b200 import kernels as K
    st = SimpleNamespace(size=(1.0, 1.0, 1.0))
    a = torch.zeros((2, 3, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match=r"\(N, 3\)"):
        K.reconstruct_temperature_volume_at_points(a, None, None, st, np.zeros((5, 2)))
    with pytest.raises(ValueError, match="Laser position"):
        K.save_temp_profiles(a, None, None, st, None, center="laser", num_points=4)
    with pytest.raises(ValueError, match="Unknown center"):
        K.save_temp_profiles(a, None, None, st, (0.1, 0.1), center="middle", num_points=4)
    assert K.reconstruct_temperature_volume_at_points(a, None, None, st, np.zeros((0, 3))).numel() == 0
