"""Serving on the device: requests that arrive while others run are admitted
into free slots and batched with them; each result is the same alone and in
the mix (bitwise in mixed precision), the FP64 engine matches the
single-instance FP64 solver, and mixed results stay within 1e-4 relative L2
of the FP64 oracle (Picard-converged evaporation)."""
import copy

import numpy as np
import pytest

from conftest import make_context, rel_l2

pytestmark = pytest.mark.gpu

MESHES = [(32, 16, 8), (48, 24, 8), (64, 32, 16)]


def _stream(n=9, seed=5, picard=None):
    from spectral_galerkin_heat_b200 import workloads
    from spectral_galerkin_heat_b200.laser import StraightTrack
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        mesh = MESHES[i % len(MESHES)]
        cfg = workloads.serving_config(*mesh)
        if picard:
            cfg["simulation"].update(picard)
        steps = int(rng.integers(15, 60))
        path = StraightTrack(0.3e-3, 0.5e-3, float(rng.uniform(0.5, 2.0)), 0.0,
                             float(rng.uniform(150, 400)))
        out.append((mesh, cfg, path, steps, 0.002 * i))
    return out


def _requests(stream):
    from spectral_galerkin_heat_b200.serving import Request
    return [Request(id=i, key=mesh, context=make_context(cfg, path), steps=steps, arrival=arr)
            for i, (mesh, cfg, path, steps, arr) in enumerate(stream)]


def _classes(stream):
    return {mesh: make_context(cfg, path) for mesh, cfg, path, _, _ in stream}


def _alone(req, precision):
    from spectral_galerkin_heat_b200.batch import BatchSolver
    b = BatchSolver([req.context], precision)
    b.start(0, req.steps, record=False)
    b.step(req.steps)
    m = b.modes(0).clone()
    b.close()
    return m


@pytest.mark.parametrize("realtime", [False, True])
def test_each_request_same_alone_and_in_mix(realtime):
    from spectral_galerkin_heat_b200.serving import ServingEngine
    stream = _stream()
    eng = ServingEngine(_classes(stream), precision="mixed",
                        slots={m: 2 for m in MESHES}, keep_modes=True)
    reqs = eng.run(_requests(stream), realtime=realtime)
    assert eng.stats.completed == len(reqs)
    assert eng.batch.tensor_core_error() == 0
    # with two slots per class and three requests per class, one request waited
    assert any(r.admitted > r.arrival for r in reqs) or realtime
    for r in reqs:
        got = r.modes.cpu().numpy()
        ref = _alone(r, "mixed").cpu().numpy()
        assert np.array_equal(got, ref), f"request {r.id} differs from its solo run"
    eng.close()


def test_fp64_engine_matches_single_instance_solver():
    from spectral_galerkin_heat_b200 import B200SpectralSolver
    from spectral_galerkin_heat_b200.serving import ServingEngine
    stream = _stream(n=4, seed=9)
    eng = ServingEngine(_classes(stream), precision="fp64", slots={m: 1 for m in MESHES},
                        keep_modes=True)
    reqs = eng.run(_requests(stream), realtime=False)
    for r in reqs:
        s = B200SpectralSolver(None, copy.copy(r.context))
        s.initialize()
        dt = r.context.num.dt
        for k in range(r.steps):
            s.step(k * dt, dt)
        assert rel_l2(r.modes.cpu().numpy(), s.state.a.cpu().numpy()) < 1e-12
        s.finalize()
    eng.close()


def test_mixed_serving_error_vs_fp64_oracle():
    """Mixed vs the FP64 oracle where the comparison is well posed: evaporation
    solved to its Picard fixed point (tol 1e-8). With a single explicit
    forcing pass (max_picard_iter = 1) the evaporation feedback is stiff: at
    high power the FP64 solution itself turns unstable, and any two solutions
    (FP64 ones with reordered sums included) part ways after some steps."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200.serving import ServingEngine
    stream = _stream(n=3, seed=11, picard={"max_picard_iter": 300, "picard_omega": 0.1,
                                           "picard_tol": 1e-8})
    eng = ServingEngine(_classes(stream), precision="mixed", slots={m: 1 for m in MESHES},
                        keep_modes=True)
    reqs = eng.run(_requests(stream), realtime=False)
    for r in reqs:
        o = OracleSolver(r.context)
        o.initialize()
        dt = r.context.num.dt
        for k in range(r.steps):
            o.step(k * dt, dt)
        assert rel_l2(r.modes.double().cpu().numpy(), o.a) < 1e-4
    eng.close()


def test_preempted_request_resumes_bit_for_bit():
    """A request taken out of its slot and queued again (its modes and warm
    start exported to the device and imported into the next free slot) ends
    with the same bits as run alone without a stop."""
    from spectral_galerkin_heat_b200.serving import ServingEngine
    stream = _stream(n=4, seed=11)
    eng = ServingEngine(_classes(stream), precision="mixed", slots={m: 1 for m in MESHES},
                        keep_modes=True, max_chunk=5)
    reqs = _requests(stream)
    eng.preempt(reqs[0])
    eng.run(reqs, realtime=False)
    assert reqs[0].preempted == 1 and all(r.status == "done" for r in reqs)
    for r in reqs:
        assert np.array_equal(r.modes.cpu().numpy(), _alone(r, "mixed").cpu().numpy()), r.id
    eng.close()


def test_adaptive_engine_plans_capacity_by_free_memory():
    """An adaptive engine declared with one class only: requests of the other
    classes bring their classes, the engine re-plans its slots by demand
    within its memory budget and moves requests in flight into the new batch
    with their state; every result is the same as alone."""
    from spectral_galerkin_heat_b200.serving import ServingEngine
    stream = _stream(n=9, seed=12)
    first = MESHES[0]
    eng = ServingEngine({first: _classes(stream)[first]}, precision="mixed", slots={first: 1},
                        keep_modes=True, adaptive=True, rebalance_interval=0.0, max_slots=3,
                        max_chunk=7)
    reqs = _requests(stream)
    eng.run(reqs, realtime=False)
    assert all(r.status == "done" for r in reqs)
    assert eng.rebalances >= 1 and set(eng.slots_per_class) >= set(MESHES)
    assert eng.batch.tensor_core_error() == 0
    for r in reqs:
        assert np.array_equal(r.modes.cpu().numpy(), _alone(r, "mixed").cpu().numpy()), r.id
    eng.close()


def test_serving_lanes_same_result_as_alone():
    """A two-lane engine (two batches on their own streams, stepped
    concurrently) serves every request with the bits it has alone."""
    from spectral_galerkin_heat_b200.serving import ServingEngine
    stream = _stream(n=8, seed=13)
    eng = ServingEngine(_classes(stream), precision="mixed", slots={m: 2 for m in MESHES},
                        keep_modes=True, lanes=2)
    reqs = _requests(stream)
    eng.run(reqs, realtime=False)
    assert all(r.status == "done" for r in reqs)
    for r in reqs:
        assert np.array_equal(r.modes.cpu().numpy(), _alone(r, "mixed").cpu().numpy()), r.id
    eng.close()


@pytest.mark.parametrize("mesh", [(512, 256, 16), (256, 128, 16)])
def test_mixed_largest_classes_first_steps_vs_fp64(mesh):
    """The largest serving classes in the benchmarked one-pass form (eight and
    four 64-column blocks, two and one 128-row tiles per face transform),
    two steps from the start, before the evaporation feedback can amplify
    rounding: the mixed batch stays within 1e-4 of the FP64 solver."""
    from spectral_galerkin_heat_b200 import B200SpectralSolver, workloads
    from spectral_galerkin_heat_b200.batch import BatchSolver
    from spectral_galerkin_heat_b200.laser import StraightTrack
    steps = 2
    cfg = workloads.serving_config(*mesh)
    ctx = make_context(cfg, StraightTrack(0.3e-3, 0.5e-3, 1.0, 0.0, 300.0))
    mix = BatchSolver([ctx], "mixed")
    mix.start(0, steps)
    mix.step(steps)
    assert mix.tensor_core_error() == 0
    s = B200SpectralSolver(None, copy.copy(ctx))
    s.initialize()
    s.run(0.0, steps)
    assert rel_l2(mix.modes(0).double().cpu().numpy(), s.state.a.cpu().numpy()) < 1e-4
    s.finalize()
    mix.close()
