"""Host-side logic: config parsing, property programs, laser paths, the backend
registry and the solver contract. CPU only."""
import copy
import math

import numpy as np
import pytest

from conftest import make_context
from spectral_galerkin_heat_b200 import (B200SpectralSolver, MathBackend, SimulationContext,
                                         build_solver, get_backend, register_backend, workloads)
from spectral_galerkin_heat_b200.laser import (RasterPath, StraightTrack, build_laser_profile,
                                               super_gaussian_area_factor)
from spectral_galerkin_heat_b200.properties import OPCODES, PropertyExpr


def run_program(ops, consts, T):
    """Host interpreter of the postfix programs (mirrors eval_program in sgh_device.cuh)."""
    inv = {v: k for k, v in OPCODES.items()}
    st = []
    i = 0
    fn1 = {"sqrt": np.sqrt, "exp": np.exp, "log": np.log, "log2": np.log2, "log10": np.log10,
           "sin": np.sin, "cos": np.cos, "tan": np.tan, "asin": np.arcsin, "acos": np.arccos,
           "atan": np.arctan, "sinh": np.sinh, "cosh": np.cosh, "tanh": np.tanh,
           "asinh": np.arcsinh, "acosh": np.arccosh, "atanh": np.arctanh, "fabs": np.abs,
           "ceil": np.ceil, "floor": np.floor, "trunc": np.trunc, "log1p": np.log1p,
           "expm1": np.expm1}
    while i < len(ops):
        name = inv[ops[i]]
        i += 1
        if name == "const":
            st.append(consts[ops[i]])
            i += 1
        elif name == "T":
            st.append(T)
        elif name in ("add", "sub", "mul", "div", "pow", "atan2"):
            b, a = st.pop(), st.pop()
            st.append({"add": a + b, "sub": a - b, "mul": a * b, "div": a / b,
                       "pow": a ** b, "atan2": np.arctan2(a, b)}[name])
        elif name == "neg":
            st.append(-st.pop())
        else:
            st.append(fn1[name](st.pop()))
    assert len(st) == 1
    return st[0]


EXPRS = ["15 + 20*(T - 300)/2700", "450 + 350*(T - 300)/2700", "7900", "9.248 + 0.01571 * T",
         "-T**2/1e6 + sqrt(T)*exp(-T/3000)", "atan2(T, 100) + fabs(T - 1500)/pi",
         "log(T) * e - +3", "tanh((T-1700)/50)*2 + floor(T/100)"]


_NUMPY_NS = {"sqrt": np.sqrt, "exp": np.exp, "log": np.log, "atan2": np.arctan2,
             "fabs": np.abs, "tanh": np.tanh, "floor": np.floor, "pi": math.pi, "e": math.e}


@pytest.mark.parametrize("src", EXPRS)
def test_program_matches_expression(src):
    """The device program (run by the test's own interpreter and by the host
    stack machine) gives the values of the expression evaluated directly by
    Python on NumPy arrays."""
    T = np.linspace(300.0, 4000.0, 37)
    e = PropertyExpr(src)
    ops, consts = e.program()
    direct = eval(src, {"__builtins__": {}}, dict(_NUMPY_NS, T=T)) + 0 * T
    np.testing.assert_array_equal(run_program(ops, consts, T), direct)
    np.testing.assert_array_equal(e(T), direct)


@pytest.mark.parametrize("bad", ["T.real", "T[0]", "foo(T)", "T < 3", "import os", "x + 1",
                                 "sqrt(T, 2)", "'abc'"])
def test_expression_whitelist(bad):
    with pytest.raises(ValueError):
        PropertyExpr(bad)


def test_config_parse_matches_reference_rules():
    cfg, _ = workloads.nonlinear_raster()
    ctx = SimulationContext.from_dict(copy.deepcopy(cfg))
    assert ctx.num.n_steps == 1000
    assert ctx.num.dt * ctx.num.n_steps == pytest.approx(2e-3, rel=1e-15)
    assert ctx.mat.k == 25.0 and ctx.mat.Cp == 625.0 and ctx.mat.rho == 7900.0
    assert ctx.mat.model is not None and not ctx.mat.model.is_constant
    assert ctx.num.picard_tol == 1e-8 and ctx.num.max_picard_iter == 400
    assert ctx.fine is None


def test_config_requires_reference_for_tdep():
    cfg, _ = workloads.nonlinear_raster()
    del cfg["material"]["k"]["reference"]
    with pytest.raises(ValueError, match="reference"):
        SimulationContext.from_dict(cfg)


@pytest.mark.parametrize("section,key", [("simulation", "bogus"), ("material", "kk"), ("oops", None)])
def test_config_rejects_unknown_keys(section, key):
    cfg, _ = workloads.straight_track()
    if key is None:
        cfg[section] = {}
    else:
        cfg[section][key] = 1
    with pytest.raises(ValueError):
        SimulationContext.from_dict(cfg)


def test_config_dtype_and_units():
    cfg, _ = workloads.straight_track()
    cfg["simulation"]["dtype"] = "float16"
    with pytest.raises(ValueError):
        SimulationContext.from_dict(cfg)
    cfg, _ = workloads.straight_track()
    cfg["simulation"]["dt"] = {"value": 5e-6, "unit": "s"}
    assert SimulationContext.from_dict(cfg).num.dt == pytest.approx(5e-6)
    cfg["simulation"]["dt"] = {"value": 5.0, "unit": "us"}
    with pytest.raises(ValueError):
        SimulationContext.from_dict(cfg)


def test_laser_profiles():
    assert super_gaussian_area_factor(2.0) == pytest.approx(math.pi / 2)
    assert build_laser_profile("flat_top").order == 12.0
    assert build_laser_profile("super_gaussian", 6.0).order == 6.0
    with pytest.raises(ValueError):
        build_laser_profile("square")
    p = build_laser_profile("gaussian")
    assert p.peak_intensity(200.0, 0.35, 50e-6 * 50e-6) == pytest.approx(
        0.35 * 200.0 / (math.pi / 2 * 2.5e-9))


def test_raster_path():
    r = RasterPath(0.8e-3, 0.3e-3, 0.4e-3, 1e-4, 5, 1.0, 200.0)
    s = r.get_state(0.0, 2e-6)
    assert (s.x, s.y, s.v, s.is_on) == (0.8e-3, 0.3e-3, (1.0, 0.0), True)
    s = r.get_state(0.5e-3, 2e-6)  # second line, running back
    assert s.y == pytest.approx(0.4e-3) and s.v[0] == -1.0
    assert s.x == pytest.approx(0.8e-3 + 0.4e-3 - 0.1e-3)
    assert not r.get_state(2.0e-3, 2e-6).is_on
    t = StraightTrack(0.25e-3, 0.5e-3, 1.0, 0.0, 200.0).get_state(1e-3, 5e-6)
    assert t.x == pytest.approx(1.25e-3)


def test_registry_contract():
    with pytest.raises(ValueError):
        get_backend("nope")
    with pytest.raises(ValueError):
        register_backend("b200")(lambda: None)

    @register_backend("unit-test-backend")
    def _make():
        return MathBackend("unit-test-backend", np, None)
    assert get_backend("unit-test-backend").name == "unit-test-backend"


def test_build_solver_cases():
    cfg, path = workloads.straight_track()
    ctx = make_context(cfg, path)
    assert isinstance(build_solver(ctx), B200SpectralSolver)
    ctx.backend = "tpu"
    with pytest.raises(ValueError):
        build_solver(ctx)


def test_solver_contract_errors_without_gpu_work():
    s = B200SpectralSolver()
    assert float(s.mixing_omega) == pytest.approx(0.1)
    assert float(s.convergence_tol) == pytest.approx(1e-4)
    assert s.max_picard_iter == 30
    with pytest.raises(RuntimeError):
        s.initialize()
    with pytest.raises(RuntimeError):
        s.set_state(np.zeros((4, 4, 4)))
    with pytest.raises(RuntimeError):
        s.step(0.0, 1e-6)


def test_picard_overrides_resolve_like_reference():
    cfg, path = workloads.straight_track()
    cfg["simulation"].update(max_picard_iter=55, picard_tol=1e-6, picard_omega=0.25)
    s = B200SpectralSolver(None, make_context(cfg, path))
    s._resolve_picard_params(np.float64)
    assert (s.max_picard_iter, float(s.convergence_tol), float(s.mixing_omega)) == (55, 1e-6, 0.25)
    s = B200SpectralSolver(None, make_context(cfg, path), mixing_omega=0.5)
    s._resolve_picard_params(np.float64)
    assert float(s.mixing_omega) == 0.5


def test_box_mode_is_rejected():
    cfg, path = workloads.straight_track()
    cfg["fine_mesh"] = {"refinement": 4}
    s = B200SpectralSolver(None, make_context(cfg, path))
    with pytest.raises((NotImplementedError, RuntimeError)):
        s.initialize()


@pytest.mark.parametrize("tag", ["dt2", "dt37", "dt0"])
def test_gcode_path_matches_reference_states(tag):
    """The G-code reader gives the reference reader's laser states bit for bit
    (float32 positions, velocities and powers; fixture from the reference's
    ``GCodeLaserPath``), one call at a time and as a vectorised step table."""
    import os
    from conftest import GOLDEN, load_golden
    from spectral_galerkin_heat_b200.laser import LASER_F32, GCodeLaserPath, laser_table
    g = load_golden("gcode_states")
    path = GCodeLaserPath(os.path.join(GOLDEN, "scan_two_segments.gcode"),
                          initial_position=(0.1, 0.2))
    dt = float(g[f"{tag}_dt"])
    times = g[f"{tag}_times"]
    for i, t in enumerate(times):
        st = path.get_state(float(t), dt)
        assert isinstance(st.x, np.float32) and isinstance(st.v[1], np.float32)
        assert (st.x, st.y) == tuple(g[f"{tag}_xy"][i])
        assert st.v == tuple(g[f"{tag}_v"][i])
        assert st.power == g[f"{tag}_power"][i] and st.is_on == bool(g[f"{tag}_on"][i])
    if dt > 0:
        tab = laser_table(path, 0.0, dt, len(times))
        np.testing.assert_array_equal(tab["x"], g[f"{tag}_xy"][:, 0])
        np.testing.assert_array_equal(tab["vy"], g[f"{tag}_v"][:, 1])
        np.testing.assert_array_equal(tab["power"], g[f"{tag}_power"])
        np.testing.assert_array_equal(tab["is_on"], g[f"{tag}_on"].astype(np.int32))
        assert np.all(tab["flags"] == LASER_F32)


def test_gcode_path_from_config():
    """A ``laser.path`` of type gcode is read into a GCodeLaserPath; a relative
    file name resolves under ``<config_dir>/paths`` as in the reference."""
    import os
    import shutil
    import tempfile
    from conftest import GOLDEN
    from spectral_galerkin_heat_b200.laser import GCodeLaserPath
    cfg, _ = workloads.straight_track()
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "paths"))
        shutil.copy(os.path.join(GOLDEN, "scan_two_segments.gcode"), os.path.join(d, "paths"))
        cfg["laser"]["path"] = {"type": "gcode", "file": "scan_two_segments.gcode"}
        ctx = SimulationContext.from_dict(cfg, config_dir=d)
        assert isinstance(ctx.laser_path, GCodeLaserPath)
        assert len(ctx.laser_path.segments) == 3
        assert cfg["laser"]["path"]["file"] == os.path.join(d, "paths", "scan_two_segments.gcode")
    cfg["laser"]["path"] = {"type": "gcode", "file": "x.gcode", "bogus": 1}
    with pytest.raises(ValueError):
        SimulationContext.from_dict(cfg)
