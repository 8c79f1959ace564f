"""The precision study's report on a small well-conditioned case: the mixed
form stays within 1e-4 relative L2 of FP64 with the same melt pool, and the
perturbed FP64 run stays within rounding of FP64."""
import pytest

pytestmark = pytest.mark.gpu


def test_precision_report_small_case():
    from spectral_galerkin_heat_b200 import workloads
    from spectral_galerkin_heat_b200.precision import run_study
    cfg, path = workloads.precision_track(seed=0, nx=64, ny=32, nz=16, steps=60)
    rep = run_study(cfg, path, [10, 40], picard={"max_picard_iter": 300, "picard_omega": 0.1,
                                                 "picard_tol": 1e-8})
    for r in rep:
        assert r["tensor_core_error"] == 0
        assert r["mixed"]["rel_l2"] < 1e-4
        assert r["fp64_perturbed"]["rel_l2"] < 1e-9
        assert abs(r["mixed"]["peak_T_err_K"]) < 1.0
    last = rep[-1]["mixed"]
    assert last["melt_pool_cells"]["cells"] > 0
    # nodal extents with interpolated isotherm crossings: a relative field
    # error of 1e-6 moves the liquidus by far less than a micrometre
    assert last["melt_pool"]["length"] > 0 and last["melt_pool"]["depth"] > 0
    assert all(abs(v) <= 1e-6 for v in last["melt_pool_err_m"].values())
    assert rep[-1]["fp64_fp32_rounded"]["rel_l2"] < 1e-5
    assert rep[-1]["fp64_fp32_every_step"]["rel_l2"] < 1e-4
    # the FP32 arm (FP32 CUDA-core contractions, FP32 modal iterates)
    for r in rep:
        assert r["fp32"]["rel_l2"] < 1e-4
        assert abs(r["fp32"]["peak_T_err_K"]) < 1.0


def test_volume_study_small_raster():
    """The volume-form study (nonlinear raster: latent heat, T-dependent k and
    c_p, evaporation, convection) on a small grid: the mixed and FP32 plans
    stay within 1e-4 of FP64, the perturbed FP64 run within rounding, and
    every form reports its device rate, Picard counts and step statuses."""
    from spectral_galerkin_heat_b200 import workloads
    from spectral_galerkin_heat_b200.precision import run_volume_study
    cfg, path = workloads.nonlinear_raster(nx=32, ny=16, nz=8, steps=10)
    rep = run_volume_study(cfg, path, [5, 10])
    assert [r["step"] for r in rep] == [5, 10]
    for r in rep:
        assert r["mixed"]["rel_l2"] < 1e-4
        assert r["fp32"]["rel_l2"] < 1e-4
        assert r["fp64_perturbed"]["rel_l2"] < 1e-9
        assert r["fp64_mixed_tol"]["rel_l2"] < 1e-4
        assert abs(r["mixed"]["peak_T_err_K"]) < 1.0
        for form in ("fp64", "mixed", "fp32", "fp64_mixed_tol", "fp64_perturbed"):
            t = r["timing"][form]
            assert t["steps_per_s"] > 0 and t["picard_iters_mean"] >= 1
            assert sum(t["step_status"].values()) == r["step"]
