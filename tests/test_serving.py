"""Serving loop scheduling on the host: admission by free slots of a class,
slot capacity from the memory budget, chunks that stop at the next
completion, and per-request accounting. The batch is a stand-in that advances
slot counters, so no device is needed."""
from types import SimpleNamespace

import numpy as np
import pytest

from spectral_galerkin_heat_b200.serving import Request, ServingEngine, latency_percentiles


class FakeBatch:
    def __init__(self, contexts, precision):
        self.n = len(contexts)
        self.workspace_bytes = 1000 * self.n
        self.st = [SimpleNamespace(active=0, step=0, n_steps=0, iters=0,
                                   last=SimpleNamespace(T_surface_max=0.0, P_laser=0.0, n_iter=1,
                                                        converged=1, picard_rel_err=0.0))
                   for _ in range(self.n)]
        self.starts, self.chunks = [], []
        self.umma_err = 0
        self.fail_after_chunks = None

    def tensor_core_error(self):
        return self.umma_err

    def launch_counts(self):
        return 5, 3, 4

    def upload_table(self, t):
        return t

    def start(self, slot, n_steps, t0=0.0, record=True, table=None):
        assert not self.st[slot].active, "slot reused while active"
        self.starts.append(slot)
        self.st[slot].active, self.st[slot].step, self.st[slot].n_steps = 1, 0, n_steps

    def step(self, k):
        self.chunks.append(k)
        if self.fail_after_chunks is not None and len(self.chunks) > self.fail_after_chunks:
            self.umma_err = 1
        for s in self.st:
            if s.active:
                s.step = min(s.n_steps, s.step + k)
                s.last.T_surface_max = float(s.step)
                if s.step >= s.n_steps:
                    s.active = 0

    def status(self):
        return [SimpleNamespace(**vars(s)) for s in self.st]

    def stop(self, slot):
        self.st[slot].active = 0

    def export_slot(self, slot):
        st = self.st[slot]
        return {"step": st.step, "n_steps": st.n_steps, "value": st.last.T_surface_max}

    def import_slot(self, slot, state, table):
        assert not self.st[slot].active, "slot reused while active"
        st = self.st[slot]
        st.active, st.step, st.n_steps = 1, state["step"], state["n_steps"]
        st.last.T_surface_max = state["value"]
        self.imports = getattr(self, "imports", 0) + 1

    def fetch(self, slot, name):
        return np.zeros(4)

    def snapshot(self, slot, name):
        return np.zeros(4)

    def synchronize(self):
        pass

    def close(self):
        pass


def _engine(slots, **kw):
    return ServingEngine({"a": object(), "b": object()}, precision="mixed", slots=slots,
                         batch_factory=FakeBatch, mem_info=lambda: (10**9, 10**9),
                         slot_bytes=lambda ctx: 1000, **kw)


def _reqs(spec):
    return [Request(id=i, key=k, context=None, steps=n, arrival=0.0,
                    table=np.zeros(n, dtype=np.float64)) for i, (k, n) in enumerate(spec)]


def test_every_request_completes_with_its_steps():
    eng = _engine({"a": 1, "b": 2})
    reqs = _reqs([("a", 10), ("b", 7), ("a", 5), ("b", 12), ("b", 3), ("a", 8)])
    eng.run(reqs, realtime=False)
    assert all(np.isfinite(r.finished) for r in reqs)
    assert eng.stats.completed == len(reqs)
    assert eng.stats.slot_steps == sum(r.steps for r in reqs)
    assert all(r.last["T_surface_max"] == r.steps for r in reqs)


def test_class_slots_serialise_and_chunks_stop_at_completions():
    eng = _engine({"a": 1, "b": 1})
    reqs = _reqs([("a", 10), ("a", 5), ("b", 4)])
    eng.run(reqs, realtime=False)
    a0, a1, b0 = reqs
    assert a1.admitted >= a0.finished      # one slot of class a: the second waits
    assert b0.admitted <= a0.finished      # class b is admitted independently
    # first chunk ends when the shortest active request (4 steps) completes
    assert eng.batch.chunks[0] == 4
    assert sum(eng.batch.chunks) == 15     # 10 then 5 on the single a-slot


def test_capacity_follows_memory_budget_and_weights():
    eng = ServingEngine({"small": object(), "big": object()}, slots=None, memory_fraction=1.0,
                        max_slots=100, weights={"small": 1.0, "big": 1.0},
                        batch_factory=FakeBatch, mem_info=lambda: (10_000, 20_000),
                        slot_bytes=lambda ctx: 1000)
    assert sum(eng.slots_per_class.values()) == 10
    assert eng.slots_per_class == {"small": 5, "big": 5}
    with pytest.raises(RuntimeError, match="budget"):
        ServingEngine({"x": object()}, slots=None, memory_fraction=0.5, batch_factory=FakeBatch,
                      mem_info=lambda: (100, 100), slot_bytes=lambda ctx: 1000)


def test_latency_percentiles():
    reqs = _reqs([("a", 1)] * 4)
    for i, r in enumerate(reqs):
        r.arrival, r.finished = 0.0, float(i + 1)
    p = latency_percentiles(reqs)
    assert p["p50"] == pytest.approx(2.5) and p["p99"] == pytest.approx(3.97)


def test_max_steps_bounds_the_batched_steps_and_reset_frees_slots():
    eng = _engine({"a": 2, "b": 1})
    reqs = _reqs([("a", 50), ("a", 40), ("b", 30), ("a", 20)])
    eng.run(reqs, realtime=False, max_steps=25)
    assert sum(eng.batch.chunks) == 25
    assert eng.in_flight == 3 and eng.stats.completed == 0
    eng.reset()
    assert eng.in_flight == 0 and len(eng.free["a"]) == 2 and len(eng.free["b"]) == 1


def test_vectorised_laser_tables_equal_get_state_bitwise():
    from spectral_galerkin_heat_b200 import laser, workloads
    for r in workloads.serving_stream(n_requests=12, seed=4):
        p, n = r["path"], r["steps"]
        tab = laser.laser_table(p, 0.0, 5e-6, n)
        for i in range(0, n, 5):
            s = p.get_state(0.0 + i * 5e-6, 5e-6)
            assert tuple(tab[i])[:6] == (s.x, s.y, s.power, s.v[0], s.v[1], int(s.is_on))
    track = laser.StraightTrack(1e-4, 2e-4, 0.7, -0.1, 250.0)
    tab = laser.laser_table(track, 1e-5, 2e-6, 40)
    for i in range(40):
        s = track.get_state(1e-5 + i * 2e-6, 2e-6)
        assert tuple(tab[i])[:6] == (s.x, s.y, s.power, s.v[0], s.v[1], 1)


def test_unknown_class_is_refused_before_anything_runs():
    eng = _engine({"a": 1, "b": 1})
    reqs = _reqs([("a", 5), ("c", 5)])
    with pytest.raises(ValueError, match="no slots"):
        eng.run(reqs, realtime=False)
    assert eng.batch.starts == [] and eng.stats.admitted == 0


def test_cancel_running_and_queued_requests():
    eng = _engine({"a": 1, "b": 1}, max_chunk=4)
    reqs = _reqs([("a", 40), ("a", 10), ("b", 12)])
    eng.cancel(reqs[0])            # running once admitted: stopped at the first boundary
    eng.cancel(reqs[1])            # still queued behind it: never runs
    eng.run(reqs, realtime=False)
    a0, a1, b0 = reqs
    assert a0.status == "cancelled" and a0.last is None
    assert a1.status in ("cancelled", "done")
    assert b0.status == "done" and b0.last["T_surface_max"] == 12
    assert eng.stats.cancelled >= 1 and len(eng.free["a"]) == 1 and eng.in_flight == 0


def test_deadline_stops_a_request_and_frees_its_slot():
    clock = iter(float(i) for i in range(10_000))
    eng = _engine({"a": 1, "b": 1}, max_chunk=2)
    reqs = _reqs([("a", 100), ("a", 4), ("b", 6)])
    reqs[0].deadline = 3.0          # host seconds after arrival (the fake clock ticks 1 per call)
    eng.run(reqs, realtime=False, clock=lambda: next(clock))
    assert reqs[0].status == "timed_out" and np.isfinite(reqs[0].finished)
    assert reqs[1].status == "done" and reqs[2].status == "done"
    assert eng.stats.timed_out == 1 and eng.in_flight == 0


def test_tensor_core_error_fails_requests_in_flight():
    eng = _engine({"a": 1, "b": 1})
    eng.batch.fail_after_chunks = 1
    reqs = _reqs([("a", 30), ("b", 50)])
    with pytest.raises(RuntimeError, match="tensor-core"):
        eng.run(reqs, realtime=False)
    assert {r.status for r in reqs} <= {"failed", "done"} and any(r.status == "failed" for r in reqs)


def test_preempted_request_resumes_and_completes_its_steps():
    eng = _engine({"a": 1, "b": 1}, max_chunk=4)
    reqs = _reqs([("a", 20), ("a", 6), ("b", 9)])
    eng.preempt(reqs[0])          # taken out at the first chunk boundary, queued again
    eng.run(reqs, realtime=False)
    a0, a1, b0 = reqs
    assert a0.status == "done" and a0.preempted == 1
    assert a0.last["T_surface_max"] == 20          # the fake slot's step counter went on
    assert eng.stats.slot_steps == 35 and eng.batch.imports >= 1
    assert all(r.status == "done" for r in reqs)


def _adaptive(slots, budget_slots, **kw):
    """An adaptive engine on a fake device whose free memory is 2 x budget_slots
    slots' worth minus what the engine's batch holds (the budget is half)."""
    holder = {}

    def mem_info():
        used = holder["eng"].batch.workspace_bytes if "eng" in holder else 0
        return 1000 * budget_slots * 2 - used, 10**9
    eng = ServingEngine({k: object() for k in slots}, precision="mixed", slots=slots,
                        batch_factory=FakeBatch, mem_info=mem_info,
                        slot_bytes=lambda ctx: 1000, adaptive=True, rebalance_interval=0.0,
                        memory_fraction=0.5, max_slots=8, **kw)
    holder["eng"] = eng
    return eng


def test_adaptive_engine_admits_a_new_class_by_free_memory():
    from types import SimpleNamespace
    eng = _adaptive({"a": 2}, budget_slots=6)
    reqs = _reqs([("a", 12), ("c", 7), ("c", 5), ("c", 9)])
    for r in reqs:
        r.context = SimpleNamespace(laser_path=None)
    eng.run(reqs, realtime=False)
    assert all(r.status == "done" for r in reqs)
    assert "c" in eng.slots_per_class and eng.rebalances >= 1
    assert sum(eng.slots_per_class.values()) <= 6 + 1   # budget: half of free + own workspace
    assert eng.stats.slot_steps == 12 + 7 + 5 + 9


def test_adaptive_engine_moves_idle_capacity_to_the_busy_class():
    eng = _adaptive({"a": 4, "b": 1}, budget_slots=5)
    reqs = _reqs([("a", 30)] + [("b", 10)] * 6)
    eng.run(reqs, realtime=False)
    assert all(r.status == "done" for r in reqs)
    assert eng.rebalances >= 1 and eng.slots_per_class.get("b", 0) > 1
    assert eng.stats.slot_steps == 30 + 60
