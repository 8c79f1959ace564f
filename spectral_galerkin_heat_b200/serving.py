"""Continuous-batching serving loop for laser-scan solves of uneven size.

A request is one solve: a grid and physics (a :class:`SimulationContext`), a
laser path and a step count. Requests arrive over time. The engine holds ONE
batch (``sgh_batch_*`` of the C ABI) whose slots are grouped into classes of
identical configuration (same grid and physics; only the laser differs). Its
capacity is sized from the free device memory when the engine starts: slots
are handed to the classes in proportion to their expected share of the
traffic until the memory budget is spent (admission by free HBM). A request
is admitted as soon as a slot of its class is free: its laser table goes to
the device, the slot restarts at the initial condition, and its modal state
stays resident in the slot until the solve completes. Every chunk of steps
advances all active requests together, one launch per stage of the time step,
so a request that arrives while others are on the GPU overlaps with them. A
chunk ends at the next completion (and, with an arrival due, after an
estimate of the steps that fit before it), so slots free up promptly.

A slot's result does not depend on what else runs in the batch (the batch
kernels reduce per slot in a fixed order), so a request gives the same result
alone and in the mix.

Latency is completion minus arrival on the host clock; throughput is the
timesteps of all completed requests divided by the span from the first
arrival to the last completion.

Failure handling (the host side of what the reference does with a warning or
an exception, ``solvers/spectral.py:486-499``):

* a request of a grid class the engine holds no slots for is refused with a
  ``ValueError`` before anything runs;
* ``cancel(request)`` stops a queued or running request at the next chunk
  boundary and frees its slot (``status = "cancelled"``);
* a request with a ``deadline`` (seconds after its arrival) that has not
  finished by then is stopped the same way (``status = "timed_out"``);
* after every chunk the batch's tensor-core error flag is read: if a bounded
  wait of a tensor-core face pass ran out, every request in flight is marked
  ``"failed"`` (its slot results are not trusted) and ``run`` raises
  ``RuntimeError``.

Preemption and adaptive capacity. A slot's state between steps is its modes
and its evaporation warm start (``BatchSolver.export_slot``); a request moved
with that state resumes bit for bit (``import_slot``). ``preempt(request)``
takes a running request out of its slot at the next chunk boundary and queues
it again with its state, to resume when a slot of its class frees. With
``adaptive=True`` the engine also re-plans its capacity by free HBM while it
runs: when queued requests find no free slot of their class -- a class it has
never seen included -- it re-divides the memory budget (a fraction of the free
device memory plus its own workspace) among the classes in proportion to
their demand (requests running and waiting), builds the new batch, and moves
every request in flight into it with its state. Freed slot bytes of one class
thus go to another, and admission follows free memory rather than a fixed
class plan.
"""
from __future__ import annotations

import copy
import functools
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .batch import BatchSolver, LaneBatch
from .laser import laser_table

__all__ = ["Request", "ServingEngine", "latency_percentiles"]


@dataclass
class Request:
    """One solve. ``key`` names its class (requests of a class share the
    context's grid and physics); ``table`` may hold its laser records already
    (host NumPy structured array or a device tensor of raw bytes)."""

    id: int
    key: Tuple
    context: object
    steps: int
    arrival: float = 0.0
    table: object = None
    deadline: Optional[float] = None   # seconds after arrival; None = no limit
    # filled in by the engine
    admitted: float = float("nan")
    finished: float = float("nan")
    slot: int = -1
    status: str = "new"   # queued | running | done | cancelled | timed_out | failed
    last: Optional[dict] = None
    modes: object = None
    surface: object = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def latency_percentiles(requests: Sequence[Request], qs=(50, 99)) -> Dict[str, float]:
    lat = np.array([r.latency for r in requests if np.isfinite(r.finished)])
    if lat.size == 0:
        return {f"p{q}": float("nan") for q in qs}
    return {f"p{q}": float(np.percentile(lat, q)) for q in qs}


@dataclass
class _Stats:
    chunks: int = 0
    steps_launched: int = 0
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    admitted: int = 0
    completed: int = 0
    slot_steps: int = 0
    class_steps: dict = field(default_factory=dict)   # slot-steps per class key
    cancelled: int = 0
    timed_out: int = 0
    busy_s: float = 0.0
    launches: int = 0
    extra: dict = field(default_factory=dict)


class ServingEngine:
    """Continuous batching of solve requests on one device.

    ``classes`` maps a class key to a template context (its laser path is not
    used) and ``weights`` gives each class's expected share of the device
    memory demand (default: equal). ``lanes`` > 1 splits the slots over that
    many batches on their own CUDA streams, stepped concurrently
    (:class:`LaneBatch`), so one lane's latency-bound face transforms overlap
    another's bandwidth-bound volume pass. Slot capacity: starting from one slot per
    class, slots go to the class with the lowest slots/weight ratio while the
    batch workspace fits in ``memory_fraction`` of the free device memory and
    stays within ``max_slots`` slots per class.
    """

    def __init__(self, classes: Dict[Tuple, object], precision: str = "mixed",
                 memory_fraction: float = 0.5, max_slots: int = 16,
                 weights: Optional[Dict[Tuple, float]] = None, slots: Optional[Dict[Tuple, int]] = None,
                 keep_modes: bool = False, max_chunk: int = 64,
                 batch_factory: Optional[Callable] = None, mem_info: Optional[Callable] = None,
                 slot_bytes: Optional[Callable] = None, adaptive: bool = False,
                 rebalance_interval: float = 1.0, lanes: int = 1):
        if batch_factory is None:
            import torch
            if not torch.cuda.is_available():
                raise RuntimeError("ServingEngine needs a CUDA device (no CPU fallback)")
            if int(lanes) > 1:
                batch_factory = functools.partial(LaneBatch, lanes=int(lanes))
            else:
                batch_factory = BatchSolver
            mem_info = mem_info or torch.cuda.mem_get_info
        self._slot_bytes_fn = slot_bytes or (lambda ctx: BatchSolver.workspace_bytes_for([ctx], precision))
        self._batch_factory = batch_factory
        self._mem_info = mem_info
        self.precision = precision
        self.memory_fraction = float(memory_fraction)
        self.max_slots = int(max_slots)
        self.adaptive = bool(adaptive)
        self.rebalance_interval = float(rebalance_interval)
        self.keys = list(classes)
        self.templates = {k: classes[k] for k in self.keys}
        self.keep_modes = keep_modes
        self.max_chunk = int(max_chunk)
        self._per_slot: Dict[Tuple, int] = {}
        free, total = mem_info()
        self.budget = int(self.memory_fraction * free)
        if slots is None:
            w = {k: float((weights or {}).get(k, 1.0)) for k in self.keys}
            slots = self._allocate(w, {}, self.budget)
        self.stats = _Stats()
        self._active: Dict[int, Request] = {}
        self._done_steps: Dict[int, int] = {}
        self._cancel: set = set()
        self._preempt: set = set()
        self._last_rebalance = -float("inf")
        self.rebalances = 0
        self._build(slots)
        self.memory = {"free_bytes_at_start": int(free), "total_bytes": int(total),
                       "budget_bytes": self.budget, "workspace_bytes": self.batch.workspace_bytes,
                       "slots": len(self.slot_key)}

    # ---- capacity ------------------------------------------------------------
    def slot_bytes(self, key) -> int:
        """Device bytes one slot of class ``key`` adds to the batch workspace."""
        if key not in self._per_slot:
            self._per_slot[key] = int(self._slot_bytes_fn(self.templates[key]))
        return self._per_slot[key]

    def _allocate(self, weights: Dict[Tuple, float], floor: Dict[Tuple, int], budget: int) -> Dict[Tuple, int]:
        """Slots per class: ``floor`` (at least one per weighted class), then one
        at a time to the class with the fewest slots per unit of weight, while
        the workspace fits in ``budget`` and a class holds at most max_slots."""
        keys = [k for k in self.keys if weights.get(k, 0.0) > 0 or floor.get(k, 0) > 0]
        slots = {k: max(1, floor.get(k, 0)) for k in keys}
        used = sum(self.slot_bytes(k) * n for k, n in slots.items())
        if used > budget:
            raise RuntimeError(f"the classes in use need {used} bytes; the budget is {budget}")
        while True:
            cand = [k for k in keys if slots[k] < self.max_slots and used + self.slot_bytes(k) <= budget]
            if not cand:
                break
            k = min(cand, key=lambda c: slots[c] / max(weights.get(c, 0.0), 1e-12))
            slots[k] += 1
            used += self.slot_bytes(k)
        return slots

    def _build(self, slots: Dict[Tuple, int]) -> None:
        """A new batch holding ``slots[k]`` slots of each class (empty)."""
        self.slots_per_class = {k: n for k, n in slots.items() if n > 0}
        contexts, self.slot_key = [], []
        for k in self.keys:
            for _ in range(self.slots_per_class.get(k, 0)):
                contexts.append(self.templates[k])
                self.slot_key.append(k)
        self.batch = self._batch_factory(contexts, self.precision)
        self.free = {k: deque(i for i, kk in enumerate(self.slot_key) if kk == k) for k in self.keys}

    def _rebalance(self, queue: List[Request], now: float) -> bool:
        """Re-divide the memory budget among the classes by demand and move
        every request in flight into the new batch with its state."""
        demand = {k: 0.0 for k in self.keys}
        active_n = {k: 0 for k in self.keys}
        for r in self._active.values():
            demand[r.key] += 1.0
            active_n[r.key] += 1
        for r in queue:
            demand[r.key] += 1.0
        free, _ = self._mem_info()
        budget = int(self.memory_fraction * (free + self.batch.workspace_bytes))
        try:
            slots = self._allocate(demand, active_n, budget)
        except RuntimeError:
            return False
        if slots == self.slots_per_class:
            return False
        states = {}
        for s, r in list(self._active.items()):
            states[id(r)] = (r, self.batch.export_slot(s), self._done_steps[s])
        self.batch.synchronize()
        self.batch.close()
        self._build(slots)
        self._active, self._done_steps = {}, {}
        for r, st, done in states.values():
            slot = self.free[r.key].popleft()
            self.batch.import_slot(slot, st, r._dev_table)
            r.slot = slot
            self._active[slot] = r
            self._done_steps[slot] = done
        self.budget = budget
        self.memory.update(budget_bytes=budget, workspace_bytes=self.batch.workspace_bytes,
                           slots=len(self.slot_key))
        self.rebalances += 1
        return True

    def _short_of_slots(self, queue: List[Request]) -> bool:
        """Some class has more requests waiting than free slots."""
        need: Dict[Tuple, int] = {}
        for r in queue:
            need[r.key] = need.get(r.key, 0) + 1
        return any(n > len(self.free[k]) for k, n in need.items())

    def _add_class(self, req: Request) -> None:
        """Adaptive mode: a request of a new class brings its class (its
        context, without the laser path, is the template)."""
        tpl = copy.copy(req.context)
        tpl.laser_path = None
        self.keys.append(req.key)
        self.templates[req.key] = tpl
        self.free[req.key] = deque()

    # ---- one request -------------------------------------------------------
    def _device_table(self, req: Request):
        if req.table is None:
            ctx = req.context
            req.table = laser_table(ctx.laser_path, 0.0, float(ctx.num.dt), req.steps)
        if isinstance(req.table, np.ndarray):
            self.stats.h2d_bytes += req.table.nbytes
            return self.batch.upload_table(req.table)
        return req.table

    def _admit(self, req: Request, now: float) -> bool:
        fr = self.free[req.key]
        if not fr:
            return False
        slot = fr.popleft()
        table = self._device_table(req)
        resume = getattr(req, "_resume", None)
        if resume is not None:  # a preempted request continues where it stopped
            self.batch.import_slot(slot, resume, table)
            req._resume = None
            self._done_steps_pending = resume["step"]
        else:
            self.batch.start(slot, req.steps, table=table, record=False)
            self._done_steps_pending = 0
        req.slot, req.admitted, req.status = slot, now, "running"
        req._dev_table = table  # keep the device table alive while the slot runs
        self.stats.admitted += 1
        return True

    def _complete(self, req: Request, info, now: float) -> None:
        req.finished = now
        o = info.last
        req.last = {"T_surface_max": o.T_surface_max, "P_laser": o.P_laser, "n_evap_iter": o.n_iter,
                    "picard_converged": bool(o.converged), "picard_rel_err": o.picard_rel_err}
        req.surface = self.batch.fetch(req.slot, "surface")  # device -> host
        self.stats.d2h_bytes += req.surface.nbytes
        if self.keep_modes:
            req.modes = self.batch.snapshot(req.slot, "modes")  # device copy
        req._dev_table = None
        req.status = "done"
        self.free[req.key].append(req.slot)
        self.stats.completed += 1

    def preempt(self, req: Request) -> None:
        """Take ``req`` out of its slot at the next chunk boundary of
        :meth:`run` and queue it again with its state (modes and warm start);
        it resumes, bit for bit, when a slot of its class is free."""
        self._preempt.add(id(req))

    def cancel(self, req: Request) -> None:
        """Stop ``req`` (queued or running) at the next chunk boundary of
        :meth:`run`; its slot is freed and ``req.status`` becomes "cancelled"."""
        self._cancel.add(id(req))

    def _stop(self, req: Request, status: str, now: float) -> None:
        """Stop a running request: free its slot, no result."""
        self.batch.stop(req.slot)
        self.free[req.key].append(req.slot)
        req._dev_table = None
        req.status, req.finished = status, now
        self._active.pop(req.slot, None)
        self._done_steps.pop(req.slot, None)

    def _expired(self, req: Request, now: float) -> bool:
        return req.deadline is not None and now > req.arrival + req.deadline

    def _check_classes(self, requests: Sequence[Request]) -> None:
        for r in requests:
            if r.key not in self.free and self.adaptive:
                self._add_class(r)
            elif r.key not in self.free:
                declared = ", ".join(map(str, self.keys))
                raise ValueError(f"request {r.id} is of class {r.key!r}, for which this engine holds "
                                 f"no slots (declared classes: {declared}); create the engine with "
                                 f"that class")

    # ---- the loop ------------------------------------------------------------
    def run(self, requests: Sequence[Request], realtime: bool = True, max_steps: Optional[int] = None,
            clock: Callable[[], float] = time.perf_counter) -> List[Request]:
        """Serve ``requests`` (``arrival`` in seconds from the start of this call).

        ``realtime``: a request becomes visible at its arrival time on the host
        clock; otherwise all are queued at once (a saturated queue).
        ``max_steps``: stop after this many batched steps (one batched step
        advances every active request by one time step); requests still in
        flight then stay in their slots until :meth:`reset`. Returns the
        requests with their timings and results filled in.
        """
        self._check_classes(requests)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        if not realtime:
            for r in pending:
                r.arrival = 0.0
        for r in pending:
            r.status = "queued"
        queue: List[Request] = []
        active, done_steps = self._active, self._done_steps
        pre, per_it, post = self.batch.launch_counts()
        launched = 0
        t0 = clock()
        step_time = None  # running estimate of one batched step (s)
        while (pending or queue or active) and (max_steps is None or launched < max_steps):
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            # cancellations and deadlines, at chunk boundaries only
            for s, r in list(active.items()):
                if id(r) in self._cancel:
                    self._cancel.discard(id(r))
                    self._stop(r, "cancelled", now)
                    self.stats.cancelled += 1
                elif self._expired(r, now):
                    self._stop(r, "timed_out", now)
                    self.stats.timed_out += 1
            if queue:
                kept = []
                for r in queue:
                    if id(r) in self._cancel:
                        self._cancel.discard(id(r))
                        r.status, r.finished = "cancelled", now
                        self.stats.cancelled += 1
                    elif self._expired(r, now):
                        r.status, r.finished = "timed_out", now
                        self.stats.timed_out += 1
                    else:
                        kept.append(r)
                queue = kept
            # preemption: export the state, free the slot, queue again
            for s, r in list(active.items()):
                if id(r) in self._preempt:
                    self._preempt.discard(id(r))
                    r._resume = self.batch.export_slot(s)
                    self.batch.stop(s)
                    self.free[r.key].append(s)
                    active.pop(s)
                    done_steps.pop(s)
                    r.status = "queued"
                    r.preempted = getattr(r, "preempted", 0) + 1
                    queue.insert(0, r)
            if (self.adaptive and queue and now - self._last_rebalance >= self.rebalance_interval
                    and self._short_of_slots(queue)):
                self._last_rebalance = now
                if self._rebalance(queue, now):
                    active, done_steps = self._active, self._done_steps
            if queue:
                still = []
                for r in queue:
                    if self._admit(r, now):
                        active[r.slot] = r
                        done_steps[r.slot] = self._done_steps_pending
                    else:
                        still.append(r)
                queue = still
            if not active:
                if pending:
                    wait = pending[0].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
                continue
            chunk = min(r.steps - done_steps[s] for s, r in active.items())
            if pending and step_time:
                until = pending[0].arrival - now
                chunk = min(chunk, max(1, int(until / step_time)))
            if max_steps is not None:
                chunk = min(chunk, max_steps - launched)
            chunk = max(1, min(chunk, self.max_chunk))
            c0 = clock()
            self.batch.step(chunk)
            info = self.batch.status()  # synchronises
            if self.batch.tensor_core_error():
                now = clock() - t0
                for r in active.values():
                    r.status, r.finished = "failed", now
                raise RuntimeError("a bounded tensor-core wait ran out in the batch's face "
                                   "transforms; the results of the requests in flight are not "
                                   "trusted (marked failed)")
            dt_chunk = clock() - c0
            self.stats.busy_s += dt_chunk
            self.stats.d2h_bytes += len(info) * 64
            est = dt_chunk / chunk
            step_time = est if step_time is None else 0.7 * step_time + 0.3 * est
            launched += chunk
            self.stats.chunks += 1
            self.stats.steps_launched += chunk
            self.stats.launches += 1 + chunk * (pre + post + per_it)
            now = clock() - t0
            iters = 1
            for s in list(active):
                st = info[s]
                self.stats.slot_steps += st.step - done_steps[s]
                key = active[s].key
                self.stats.class_steps[key] = self.stats.class_steps.get(key, 0) + st.step - done_steps[s]
                iters = max(iters, st.last.n_iter)
                done_steps[s] = st.step
                if not st.active:
                    self._complete(active.pop(s), st, now)
            # Picard iterations beyond the first (upper bound: the largest count
            # of the last step, for every step of the chunk)
            self.stats.launches += chunk * per_it * (iters - 1)
        self.batch.synchronize()
        return list(requests)

    def reset(self) -> None:
        """Stop every request in flight and free its slot."""
        for s, r in list(self._active.items()):
            self.batch.stop(s)
            self.free[r.key].append(s)
            r._dev_table = None
        self._active.clear()
        self._done_steps.clear()
        self.batch.synchronize()

    @property
    def in_flight(self) -> int:
        return len(self._active)

    def close(self) -> None:
        self.batch.close()


def requests_from_stream(stream: Sequence[dict], contexts: Dict[Tuple, object]) -> List[Request]:
    """Requests of a ``workloads.serving_stream`` list; ``contexts`` holds one
    template context per mesh (built with ``SimulationContext.from_dict``)."""
    out = []
    for r in stream:
        ctx = copy.copy(contexts[r["mesh"]])
        ctx.laser_path = r["path"]
        out.append(Request(id=r["id"], key=r["mesh"], context=ctx, steps=r["steps"], arrival=r["arrival"]))
    return out
