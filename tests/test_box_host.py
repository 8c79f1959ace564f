"""Box mode on the host: the library's fine-box geometry against the oracle's
restatement of ``FineMeshState`` (plan creation runs no device code), config
validation, and the reference-named box functions' guard for grid mode."""
import ctypes as C

import pytest

from conftest import golden_case, make_context
from oracle.sgh_oracle import FineBox, subgrid_start
from spectral_galerkin_heat_b200 import _lib, kernels, workloads
from spectral_galerkin_heat_b200.solver import make_config

BOX_CASES = ["box_const_24x12x8", "box_shallow_24x12x8", "box_tdep_16x12x8", "box_full_r1_20x12x30"]


def _plan(c):
    p = C.c_void_p()
    rc = _lib.lib().sgh_plan_create(C.byref(c), C.byref(p))
    return rc, p


def _geometry(ctx):
    c = make_config(ctx, 0.1, 1e-8, 10)
    rc, p = _plan(c)
    assert rc == 0, _lib.lib().sgh_last_error()
    g = _lib.SghBoxGeom()
    assert _lib.lib().sgh_box_geometry(p, C.byref(g)) == 0
    _lib.lib().sgh_plan_destroy(p)
    return g


def _fine_box(ctx):
    g = ctx.geom
    return FineBox(ctx.fine, (g.d.x, g.d.y, g.d.z), (g.size.x, g.size.y, g.size.z),
                   (int(g.n.x), int(g.n.y), int(g.n.z)))


@pytest.mark.parametrize("name", BOX_CASES + ["bench"])
def test_box_geometry_matches_oracle(name):
    if name == "bench":
        cfg, path = workloads.box_track()
    else:
        cfg, path, *_ = golden_case(name)
    ctx = make_context(cfg, path)
    g = _geometry(ctx)
    fb = _fine_box(ctx)
    assert tuple(g.n_box) == (fb.nx_box, fb.ny_box, fb.nz_box)
    assert list(g.n_fine_total) == fb.n_fine_totals
    # bit-identical spacings and cell volume (same operations in the same order)
    assert tuple(g.d_fine) == (fb.dx_fine, fb.dy_fine, fb.dz_fine)
    assert g.dV_fine == fb.dV_fine
    assert g.z0 == float(ctx.geom.size.z) - float(ctx.fine.box_size[2])


def test_box_geometry_rounds_like_the_reference():
    """0.2e-3 / 12.5e-6 is 16.000000000000004 in FP64: the box gets 17 cells, as
    ``int(np.ceil(L / d))`` gives in the reference."""
    cfg, path, *_ = golden_case("box_const_24x12x8")
    g = _geometry(make_context(cfg, path))
    assert g.n_box[0] == 17


def test_window_start_rounds_half_to_even():
    # Python's round(): 2.5 -> 2, 3.5 -> 4 (the device uses rint)
    assert subgrid_start(2.5, 1.0, 100, 4) == 0
    assert subgrid_start(5.5, 1.0, 100, 4) == 4
    assert subgrid_start(6.5, 1.0, 100, 4) == 4
    assert subgrid_start(-3.0, 1.0, 100, 4) == 0
    assert subgrid_start(1e9, 1.0, 100, 4) == 96
    assert subgrid_start(50.0, 1.0, 10, 40) == 0


@pytest.mark.parametrize("over", [dict(box_refinement=0), dict(box_refinement=65),
                                  dict(box_size=(0.0, 1e-4, 1e-4)), dict(box_size=(1e-4, 1e-4, -1e-5))])
def test_plan_create_rejects_bad_box(over):
    cfg, path, *_ = golden_case("box_const_24x12x8")
    c = make_config(make_context(cfg, path), 0.1, 1e-8, 10)
    for k, v in over.items():
        if k == "box_size":
            for i in range(3):
                c.box_size[i] = v[i]
        else:
            setattr(c, k, v)
    rc, _ = _plan(c)
    assert rc == -1
    assert _lib.lib().sgh_last_error()


def test_box_mode_with_constant_properties_needs_a_band():
    cfg, path, *_ = golden_case("box_const_24x12x8")
    c = make_config(make_context(cfg, path), 0.1, 1e-8, 10)
    c.L_f = 0.0
    c.T_liquidus = c.T_solidus
    rc, _ = _plan(c)
    assert rc == -1 and b"T_liquidus" in _lib.lib().sgh_last_error()


def test_batch_rejects_box_mode():
    cfg, path, *_ = golden_case("box_const_24x12x8")
    c = make_config(make_context(cfg, path), 0.1, 1e-8, 10)
    arr = (_lib.SghConfig * 1)(c)
    b = C.c_void_p()
    rc = _lib.lib().sgh_batch_create(arr, 1, 0, C.byref(b))
    assert rc < 0 and b"box" in _lib.lib().sgh_last_error()


def test_grid_mode_plan_has_no_box():
    cfg, path = workloads.straight_track(nx=8, ny=6, nz=4, steps=1)
    c = make_config(make_context(cfg, path), 0.1, 1e-8, 10)
    assert c.box == 0
    rc, p = _plan(c)
    assert rc == 0
    g = _lib.SghBoxGeom()
    assert _lib.lib().sgh_box_geometry(p, C.byref(g)) == -3
    _lib.lib().sgh_plan_destroy(p)


class _GridState:
    fine_mesh = None


def test_box_functions_require_fine_mesh():
    """Grid-mode state -> RuntimeError, as ``project_box_to_modes`` and
    ``reconstruct_temperature_box`` raise in the reference
    (``tests/unit_tests/physics/test_spectral_ops.py:19-30``)."""
    with pytest.raises(RuntimeError):
        kernels.project_box_to_modes(None, _GridState())
    with pytest.raises(RuntimeError):
        kernels.reconstruct_temperature_box(None, _GridState())


def test_checkpoint_digest_ignores_tile_policy_only():
    """A checkpoint names the configuration it belongs to by a digest of the
    plan config with the tile-policy fields zeroed: a plan with other tiles may
    restore it, a plan with other physics may not (no device needed)."""
    from spectral_galerkin_heat_b200.solver import B200SpectralSolver
    cfg, path, *_ = golden_case("box_const_24x12x8")
    s = B200SpectralSolver(None, make_context(cfg, path))
    s._cfg = make_config(s.context, 0.1, 1e-8, 10)
    d0 = s._config_digest()
    s._cfg.axis_min_ctas, s._cfg.axis_cuda_cores = 264, 1
    assert s._config_digest() == d0
    s._cfg.dt *= 2.0
    assert s._config_digest() != d0
