"""Batched slots of uneven size: each slot equals its single-instance run and
the oracle, is the same alone and in a mix, and the mixed form (FP32 state,
split-BF16 tensor-core face contractions) stays within 1e-4 relative L2 of
the FP64 oracle on a converged-Picard case."""
import numpy as np
import pytest

from conftest import golden_case, make_context, rel_l2

pytestmark = pytest.mark.gpu


def _ctx(nx, ny, nz, seed, steps, **kw):
    from spectral_galerkin_heat_b200 import workloads
    from spectral_galerkin_heat_b200.laser import StraightTrack
    rng = np.random.default_rng(seed)
    cfg, _ = workloads.straight_track(nx=nx, ny=ny, nz=nz, steps=steps,
                                      size=(2e-3 * nx / 64, 1e-3 * ny / 32, 0.5e-3), **kw)
    cfg["simulation"].update({"max_picard_iter": 30, "picard_omega": 0.1, "picard_tol": 1e-4})
    power = float(rng.uniform(150.0, 400.0))
    v = float(rng.uniform(0.5, 2.0))
    path = StraightTrack(0.3e-3, cfg["domain"]["size"][1] / 2, v, 0.0, power)
    return make_context(cfg, path)


SHAPES = [(32, 16, 8), (48, 24, 16), (40, 20, 6), (64, 32, 16)]


def test_batch_matches_single_instance_and_oracle():
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 8
    ctxs = [_ctx(*sh, seed=i, steps=steps) for i, sh in enumerate(SHAPES)]
    b = BatchSolver(ctxs, "fp64")
    for i in range(len(ctxs)):
        b.start(i, steps)
    b.step(steps)
    info = b.status()
    assert all(x.step == steps and not x.active for x in info)
    for i, ctx in enumerate(ctxs):
        single = B200SpectralSolver(None, ctx)
        single.initialize()
        o = OracleSolver(ctx)
        o.initialize()
        dt = ctx.num.dt
        ms, mo = [], []
        for k in range(steps):
            ms.append(single.step(k * dt, dt)[1])
            mo.append(o.step(k * dt, dt)[1])
        a = b.modes(i).cpu().numpy()
        assert rel_l2(a, single.state.a.cpu().numpy()) < 1e-12
        assert rel_l2(a, o.a) < 1e-10
        mb = b.metrics(i)
        assert [m["n_evap_iter"] for m in mb] == [m["n_evap_iter"] for m in mo]
        np.testing.assert_allclose([m["T_surface_max"] for m in mb],
                                   [m["T_surface_max"] for m in mo], rtol=1e-10)
        single.finalize()
    b.close()


def test_slot_alone_equals_slot_in_mix():
    """Continuous-batching invariant: a slot's result does not depend on its neighbours."""
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 6
    ctxs = [_ctx(*sh, seed=10 + i, steps=steps) for i, sh in enumerate(SHAPES)]
    mix = BatchSolver(ctxs, "mixed")
    for i in range(len(ctxs)):
        mix.start(i, steps)
    mix.step(2)
    late = len(ctxs) - 1                    # restart one slot while the others run
    mix.start(late, steps)
    mix.step(steps)
    alone = BatchSolver([ctxs[late]], "mixed")
    alone.start(0, steps)
    alone.step(steps)
    assert mix.tensor_core_error() == 0 and alone.tensor_core_error() == 0
    assert np.array_equal(mix.modes(late).cpu().numpy(), alone.modes(0).cpu().numpy())
    assert [m["n_evap_iter"] for m in mix.metrics(late)] == \
        [m["n_evap_iter"] for m in alone.metrics(0)]
    mix.close()
    alone.close()


def test_mixed_precision_error_vs_fp64_oracle():
    """FP32 state: temperature rel L2 vs the FP64 oracle <= 1e-4 (stated target)."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 40
    ctx = _ctx(64, 32, 16, seed=3, steps=steps)
    ctx.num.picard_tol = 1e-8
    ctx.num.max_picard_iter = 300
    b = BatchSolver([ctx], "mixed")
    b.start(0, steps)
    b.step(steps)
    o = OracleSolver(ctx)
    o.initialize()
    for k in range(steps):
        o.step(k * ctx.num.dt, ctx.num.dt)
    from oracle.sgh_oracle import dct3
    T_mixed = dct3(b.modes(0).double().cpu().numpy())
    T_ref = dct3(o.a)
    assert b.tensor_core_error() == 0
    assert rel_l2(T_mixed, T_ref) < 1e-4
    b.close()


def test_batch_rejects_unsupported_physics():
    from spectral_galerkin_heat_b200.batch import BatchSolver
    cfg, path, *_ = golden_case("raster_32x16x8")
    with pytest.raises(Exception, match="face-space"):
        BatchSolver([make_context(cfg, path)], "fp64")


ODD = [(37, 19, 7), (50, 26, 9), (33, 17, 5)]   # nx % 8 != 0 and S % 4 != 0: scalar plane and volume paths


def test_odd_shapes_fp64_batch_matches_single_instance():
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 6
    ctxs = [_ctx(*sh, seed=20 + i, steps=steps) for i, sh in enumerate(ODD)]
    b = BatchSolver(ctxs, "fp64")
    for i in range(len(ctxs)):
        b.start(i, steps)
    b.step(steps)
    for i, ctx in enumerate(ctxs):
        s = B200SpectralSolver(None, ctx)
        s.initialize()
        dt = ctx.num.dt
        for k in range(steps):
            s.step(k * dt, dt)
        assert rel_l2(b.modes(i).cpu().numpy(), s.state.a.cpu().numpy()) < 1e-12
        s.finalize()
    b.close()


def test_odd_shapes_mixed_batch_vs_oracle_and_alone():
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 12
    ctxs = []
    for i, sh in enumerate(ODD):
        c = _ctx(*sh, seed=30 + i, steps=steps)
        c.num.picard_tol = 1e-8
        c.num.max_picard_iter = 300
        ctxs.append(c)
    mix = BatchSolver(ctxs, "mixed")
    for i in range(len(ctxs)):
        mix.start(i, steps)
    mix.step(steps)
    assert mix.tensor_core_error() == 0
    for i, ctx in enumerate(ctxs):
        o = OracleSolver(ctx)
        o.initialize()
        for k in range(steps):
            o.step(k * ctx.num.dt, ctx.num.dt)
        assert rel_l2(mix.modes(i).double().cpu().numpy(), o.a) < 1e-4
    alone = BatchSolver([ctxs[1]], "mixed")
    alone.start(0, steps)
    alone.step(steps)
    assert np.array_equal(alone.modes(0).cpu().numpy(), mix.modes(1).cpu().numpy())
    alone.close()
    mix.close()


def test_deep_slot_moves_the_mixed_volume_pass_off_the_ring_form_results_unchanged():
    """A slot deeper than the ring-staged volume pass's per-plane table (nz >
    256) moves its whole mixed batch to the float2 register form of the
    volume pass. Every variant groups the z-planes of the face sums alike, so
    the other slot's result is bit for bit that of the same slot alone (ring
    form), and the deep slot stays within 1e-4 of the FP64 oracle."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 6
    ctxs = [_ctx(16, 8, 264, seed=41, steps=steps), _ctx(32, 16, 24, seed=42, steps=steps)]
    for c in ctxs:
        c.num.picard_tol = 1e-8
        c.num.max_picard_iter = 300
    mix = BatchSolver(ctxs, "mixed")
    for i in range(2):
        mix.start(i, steps)
    mix.step(steps)
    assert mix.tensor_core_error() == 0
    alone = BatchSolver([ctxs[1]], "mixed")
    alone.start(0, steps)
    alone.step(steps)
    assert np.array_equal(alone.modes(0).cpu().numpy(), mix.modes(1).cpu().numpy())
    o = OracleSolver(ctxs[0])
    o.initialize()
    for k in range(steps):
        o.step(k * ctxs[0].num.dt, ctxs[0].num.dt)
    assert rel_l2(mix.modes(0).double().cpu().numpy(), o.a) < 1e-4
    alone.close()
    mix.close()


def test_mixed_batch_tall_faces_vs_oracle():
    """ny = 300 and nx = 72: three 128-row tiles per column block, the last
    one ragged, and a ragged second column block, in both face passes."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 4
    ctx = _ctx(72, 300, 8, seed=1, steps=steps)
    mix = BatchSolver([ctx], "mixed")
    mix.start(0, steps)
    mix.step(steps)
    assert mix.tensor_core_error() == 0
    o = OracleSolver(ctx)
    o.initialize()
    for k in range(steps):
        o.step(k * ctx.num.dt, ctx.num.dt)
    assert rel_l2(mix.modes(0).double().cpu().numpy(), o.a) < 1e-4
    mix.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_every_tile_policy_gives_the_same_result(precision):
    """The autotuner's candidate policies change only how the volume pass
    issues its loads, not the arithmetic: every candidate gives the same bits,
    and the result matches the oracle (FP64 to 1e-10, mixed to 1e-4)."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200.autotune import BATCH_CANDIDATES
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps = 6
    ctxs = [_ctx(*sh, seed=10 + i, steps=steps) for i, sh in enumerate(SHAPES)]
    modes = []
    for pol in BATCH_CANDIDATES:
        if precision == "fp64" and pol["vol_vec"] > 2:
            continue  # 4-wide vectors need FP32 modes
        b = BatchSolver(ctxs, precision, policy=pol)
        assert b.policy == pol
        for i in range(len(ctxs)):
            b.start(i, steps)
        b.step(steps)
        assert b.tensor_core_error() == 0
        modes.append([b.modes(i).double().cpu().numpy() for i in range(len(ctxs))])
        b.close()
    for other in modes[1:]:
        for x, y in zip(modes[0], other):
            assert np.array_equal(x, y)
    tol = 1e-10 if precision == "fp64" else 1e-4
    for i, ctx in enumerate(ctxs):
        o = OracleSolver(ctx)
        o.initialize()
        for k in range(steps):
            o.step(k * ctx.num.dt, ctx.num.dt)
        assert rel_l2(modes[0][i], o.a) < tol


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_slot_export_import_resumes_bit_for_bit(precision):
    """A request exported after some steps and resumed in another batch (a
    different slot, another slot mix) ends with the same bits as the same
    request run through without a stop."""
    from spectral_galerkin_heat_b200.batch import BatchSolver
    steps, cut = 10, 4
    ctx = _ctx(48, 24, 16, seed=3, steps=steps)
    other = _ctx(32, 16, 8, seed=4, steps=steps)
    ref = BatchSolver([ctx], precision)
    ref.start(0, steps)
    ref.step(steps)
    want = ref.modes(0).double().cpu().numpy()
    a = BatchSolver([other, ctx], precision)
    a.start(1, steps)
    a.step(cut)
    state = a.export_slot(1)
    assert state["step"] == cut and state["n_steps"] == steps
    table = a._tables[1]
    a.close()
    b = BatchSolver([ctx, other, ctx], precision)
    b.start(1, steps)                 # a neighbour running alongside
    b.import_slot(2, state, table)
    b.step(steps - cut)
    info = b.status()[2]
    assert info.step == steps and not info.active
    assert np.array_equal(b.modes(2).double().cpu().numpy(), want)
    assert b.tensor_core_error() == 0
    b.close()
    ref.close()


def test_lanes_give_the_same_bits_as_one_batch():
    """Slots dealt to two batches on their own streams and stepped
    concurrently end with the same bits as in one batch."""
    from spectral_galerkin_heat_b200.batch import BatchSolver, LaneBatch
    steps = 7
    ctxs = [_ctx(*sh, seed=20 + i, steps=steps) for i, sh in enumerate(SHAPES + SHAPES)]
    one = BatchSolver(ctxs, "mixed")
    two = LaneBatch(ctxs, "mixed", lanes=2)
    assert len(two.lanes) == 2
    for b in (one, two):
        for i in range(len(ctxs)):
            b.start(i, steps, record=False)
        b.step(3)
        b.step(steps - 3)
        assert b.tensor_core_error() == 0
    info = two.status()
    assert all(x.step == steps and not x.active for x in info)
    for i in range(len(ctxs)):
        assert np.array_equal(one.modes(i).cpu().numpy(), two.modes(i).cpu().numpy())
    one.close()
    two.close()
