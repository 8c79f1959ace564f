"""Batched stepping of many independent cuboids (``sgh_batch_*`` of the C ABI).

:class:`BatchSolver` holds a fixed set of slots, each with its own
:class:`SimulationContext` (grid shape and physics may differ between slots).
A slot is started with a laser path and a step count; every call of
:meth:`BatchSolver.step` advances all active slots together, one launch per
stage. Each slot runs the reference step (``solvers/spectral.py:219-543``) in
its face-space form, so the supported physics is laser + evaporation without
convection, latent heat or a T-dependent model.

``precision="fp64"`` keeps the modes and K/KK in FP64; ``precision="mixed"``
stores the modes in FP32 (K and KK formed from FP64 1-D tables), with FP64 face
fields (fluxes, sigma, surface) and norms and FP32 face sums and weights,
moving a third of the bytes per step.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .solver import laser_struct, make_config

__all__ = ["BatchSolver", "LaneBatch"]


def _torch_stream(stream):
    import torch
    return torch.cuda.stream(stream)


def _picard(ctx, omega=None, tol=None, max_iter=None):
    num = ctx.num

    def pick(explicit, attr, default):
        if explicit is not None:
            return explicit
        v = getattr(num, attr, None)
        return default if v is None else v

    return (float(pick(omega, "picard_omega", 0.1)), float(pick(tol, "picard_tol", 1e-4)),
            int(pick(max_iter, "max_picard_iter", 30)))


class BatchSolver:
    """A bound batch of slots on one device."""

    def __init__(self, contexts: Sequence, precision: str = "fp64", device=None,
                 policy: Optional[dict] = None, stream=None):
        """``policy``: the kernels' tile policy, ``{"vol_unroll": 2 | 4 | 8,
        "vol_vec": 0 | 1 | 2 | 4}`` (0: the widest vector);
        None takes the autotuner's entry for this grid mix (``tuned.json`` or
        ``SGH_TUNE_TABLE``) and the built-in default without one. ``stream``:
        the CUDA stream of every launch and copy of this batch (default: the
        device's current stream)."""
        import torch
        if precision not in _lib.PRECISION:
            raise ValueError(f"precision must be one of {sorted(_lib.PRECISION)}")
        if not torch.cuda.is_available():
            raise RuntimeError("BatchSolver needs a CUDA device (no CPU fallback)")
        self.contexts = list(contexts)
        self.precision = precision
        self.n = len(self.contexts)
        cfgs = (_lib.SghConfig * self.n)()
        for i, ctx in enumerate(self.contexts):
            if getattr(ctx, "fine", None) is not None:
                raise NotImplementedError("box mode (fine_mesh) is not supported")
            cfgs[i] = make_config(ctx, *_picard(ctx))
        self._cfgs = cfgs
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check("sgh_batch_create", L.sgh_batch_create(cfgs, self.n, _lib.PRECISION[precision],
                                                          C.byref(h)))
        self._h = h
        if policy is None:
            from .autotune import lookup_batch
            policy = lookup_batch(cfgs, precision) or {}
        self.policy = {"vol_unroll": int(policy.get("vol_unroll", 4)),
                       "vol_vec": int(policy.get("vol_vec", 0))}
        pol = _lib.SghBatchPolicy()
        pol.vol_unroll = self.policy["vol_unroll"]
        pol.vol_vec = self.policy["vol_vec"]
        _lib.check("sgh_batch_set_policy", L.sgh_batch_set_policy(h, C.byref(pol)))
        nbytes = C.c_uint64()
        _lib.check("sgh_batch_workspace_bytes", L.sgh_batch_workspace_bytes(h, C.byref(nbytes)))
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        self.workspace = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        self.stream = torch.cuda.current_stream(self.device) if stream is None else stream
        _lib.check("sgh_batch_bind", L.sgh_batch_bind(h, C.c_void_p(self.workspace.data_ptr()),
                                                      nbytes.value, self._s()))
        self._tables = [None] * self.n
        self._outs = [None] * self.n

    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    @staticmethod
    def workspace_bytes_for(contexts: Sequence, precision: str = "fp64") -> int:
        """Device bytes a batch of these contexts would bind (computed on the host)."""
        n = len(contexts)
        cfgs = (_lib.SghConfig * n)()
        for i, ctx in enumerate(contexts):
            cfgs[i] = make_config(ctx, *_picard(ctx))
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check("sgh_batch_create", L.sgh_batch_create(cfgs, n, _lib.PRECISION[precision], C.byref(h)))
        try:
            nbytes = C.c_uint64()
            _lib.check("sgh_batch_workspace_bytes", L.sgh_batch_workspace_bytes(h, C.byref(nbytes)))
            return int(nbytes.value)
        finally:
            L.sgh_batch_destroy(h)

    @property
    def workspace_bytes(self) -> int:
        return self.workspace.numel()

    def laser_table(self, ctx, t0: float, n_steps: int):
        """Device table of ``sgh_laser`` for steps ``t0 + i*dt`` of ``ctx.laser_path``."""
        import torch
        dt = float(ctx.num.dt)
        arr = (_lib.SghLaser * n_steps)()
        for i in range(n_steps):
            arr[i] = laser_struct(ctx.laser_path.get_state(t0 + i * dt, dt), dt, dt)
        return torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(self.device)

    def start(self, slot: int, n_steps: int, t0: float = 0.0, record: bool = True,
              table=None) -> None:
        """Restart ``slot`` at the initial condition for ``n_steps`` steps of its path."""
        import torch
        ctx = self.contexts[slot]
        if table is None:
            table = self.laser_table(ctx, t0, n_steps)
        self._tables[slot] = table
        outs = None
        if record:
            outs = torch.zeros(max(1, n_steps) * C.sizeof(_lib.SghStepOut), dtype=torch.uint8,
                               device=self.device)
        self._outs[slot] = outs
        _lib.check("sgh_batch_slot_start", _lib.lib().sgh_batch_slot_start(
            self._h, int(slot), C.c_void_p(table.data_ptr()), int(n_steps),
            C.c_void_p(outs.data_ptr()) if outs is not None else None, self._s()))

    def export_slot(self, slot: int) -> dict:
        """The state a slot carries between steps, as device copies: its modes
        (FP64 or FP32), its evaporation warm start ``q_evap_old`` and its
        progress (``step`` of ``n_steps``). The slot keeps running unless it is
        stopped; a checkpoint of a request in flight (preemption)."""
        info = self.status()[slot]
        return {"modes": self.snapshot(slot, "modes"), "q_evap_old": self.snapshot(slot, "q_evap_old"),
                "step": int(info.step), "n_steps": int(info.n_steps), "precision": self.precision,
                "shape": tuple(self.buffer(slot, "modes").shape)}

    def import_slot(self, slot: int, state: dict, table) -> None:
        """Continue an exported request in ``slot`` (same grid, physics and
        precision) with its laser ``table`` (all of the request's steps): it
        resumes at the exported step and gives the same bits as if it had run
        on uninterrupted."""
        if state["precision"] != self.precision:
            raise ValueError("a slot state moves between batches of the same precision only")
        dst = self.buffer(slot, "modes")
        if tuple(dst.shape) != tuple(state["shape"]):
            raise ValueError(f"slot {slot} has modes {tuple(dst.shape)}, the state {state['shape']}")
        with _torch_stream(self.stream):
            dst.copy_(state["modes"])
            self.buffer(slot, "q_evap_old").copy_(state["q_evap_old"])
        self._tables[slot] = table
        self._outs[slot] = None
        _lib.check("sgh_batch_slot_resume", _lib.lib().sgh_batch_slot_resume(
            self._h, int(slot), C.c_void_p(table.data_ptr()), int(state["n_steps"]), int(state["step"]),
            None, self._s()))

    def stop(self, slot: int) -> None:
        _lib.check("sgh_batch_slot_stop", _lib.lib().sgh_batch_slot_stop(self._h, int(slot), self._s()))

    def step(self, n_steps: int = 1) -> None:
        """Advance every active slot by ``n_steps`` steps (asynchronous)."""
        _lib.check("sgh_batch_step", _lib.lib().sgh_batch_step(self._h, int(n_steps), self._s()))

    def step_eager(self) -> None:
        """One step with the kernels launched one by one (profilers, debugging)."""
        _lib.check("sgh_batch_step_eager", _lib.lib().sgh_batch_step_eager(self._h, self._s()))

    def status(self):
        """Per-slot ``SghBatchSlotInfo`` (synchronises the stream)."""
        arr = (_lib.SghBatchSlotInfo * self.n)()
        _lib.check("sgh_batch_status", _lib.lib().sgh_batch_status(self._h, arr, self._s()))
        return list(arr)

    def metrics(self, slot: int):
        """Per-step metric dicts recorded for ``slot`` since its start."""
        info = self.status()[slot]
        outs = self._outs[slot]
        if outs is None:
            return []
        host = outs.cpu().numpy().tobytes()
        sz = C.sizeof(_lib.SghStepOut)
        res = []
        for i in range(info.step):
            o = _lib.SghStepOut.from_buffer_copy(host[i * sz:(i + 1) * sz])
            res.append({"T_surface_max": o.T_surface_max, "P_laser": o.P_laser,
                        "n_evap_iter": o.n_iter, "picard_converged": bool(o.converged),
                        "picard_rel_err": o.picard_rel_err})
        return res

    def buffer(self, slot: int, name: str):
        """torch view of a slot buffer: ``modes``, ``K``, ``KK`` (FP64 or FP32),
        ``q_evap_old``, ``surface`` (FP64)."""
        import torch
        ptr, nb = C.c_void_p(), C.c_uint64()
        _lib.check("sgh_batch_buffer", _lib.lib().sgh_batch_buffer(
            self._h, int(slot), _lib.BUF[name], C.byref(ptr), C.byref(nb)))
        off = ptr.value - self.workspace.data_ptr()
        c = self._cfgs[slot]
        vol = name in ("modes", "K", "KK")
        dt = torch.float32 if (vol and self.precision == "mixed") else torch.float64
        view = self.workspace[off:off + nb.value].view(dt)
        return view.view(c.nz, c.ny, c.nx) if vol else view.view(c.ny, c.nx)

    def modes(self, slot: int):
        return self.buffer(slot, "modes")

    def upload_table(self, records: np.ndarray):
        """Device copy (raw bytes) of a host table of ``sgh_laser`` records,
        from pinned memory on this batch's stream."""
        import torch
        host = torch.from_numpy(np.ascontiguousarray(records).view(np.uint8)).pin_memory()
        with torch.cuda.stream(self.stream):
            return host.to(self.device, non_blocking=True)

    def fetch(self, slot: int, name: str) -> np.ndarray:
        """Host copy of a slot buffer (synchronises the stream)."""
        return self.buffer(slot, name).to("cpu").numpy()

    def snapshot(self, slot: int, name: str):
        """Device copy of a slot buffer (the slot may be reused afterwards)."""
        return self.buffer(slot, name).clone()

    def volume_pass(self) -> None:
        """The step's volume pass alone over every active slot (timing, profiling)."""
        _lib.check("sgh_batch_volume_pass", _lib.lib().sgh_batch_volume_pass(self._h, self._s()))

    def active_modes(self) -> int:
        """Modes of the slots that are active now (synchronises)."""
        return sum(int(c.nx) * int(c.ny) * int(c.nz) for c, st in zip(self._cfgs, self.status()) if st.active)

    def synchronize(self) -> None:
        self.stream.synchronize()

    def tensor_core_error(self) -> int:
        """Nonzero once a tensor-core wait expired in a mixed-precision face pass."""
        e = C.c_int32()
        _lib.check("sgh_batch_error", _lib.lib().sgh_batch_error(self._h, C.byref(e), self._s()))
        return e.value

    def set_wait_limit(self, polls: int = 0, stall_test: bool = False) -> None:
        """Bound the tensor-core data waits to ``polls`` polls (0: the default);
        ``stall_test`` makes the face transforms wait on a barrier nothing
        completes, so the bounded-wait error path runs (tests only)."""
        _lib.check("sgh_batch_set_wait_limit", _lib.lib().sgh_batch_set_wait_limit(
            self._h, int(polls), 1 if stall_test else 0, self._s()))

    def launch_counts(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        _lib.check("sgh_batch_launch_counts", _lib.lib().sgh_batch_launch_counts(
            self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            self.stream.synchronize()
            _lib.lib().sgh_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LaneBatch:
    """Several batches ("lanes") driven as one, each on its own CUDA stream.

    The slots are dealt to the lanes class by class, so every lane holds a
    share of each grid class. A step launches every lane's step graph on its
    own stream before any is waited for, so the lanes run concurrently: while
    one lane is in its latency-bound face transforms, another streams its
    volume pass from HBM. Results do not depend on the lane count (each slot's
    arithmetic is its own). The interface is BatchSolver's, with global slot
    numbers."""

    def __init__(self, contexts: Sequence, precision: str = "fp64", lanes: int = 2, device=None,
                 policy: Optional[dict] = None):
        import torch
        self.contexts = list(contexts)
        self.precision = precision
        self.n = len(self.contexts)
        lanes = max(1, min(int(lanes), self.n))
        # deal the slots of each class round-robin over the lanes
        by_key = {}
        for i, c in enumerate(self.contexts):
            key = (int(c.num.nx), int(c.num.ny), int(c.num.nz))
            by_key.setdefault(key, []).append(i)
        members = [[] for _ in range(lanes)]
        turn = 0
        for key in sorted(by_key):
            for i in by_key[key]:
                members[turn % lanes].append(i)
                turn += 1
        members = [m for m in members if m]
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.lanes = []
        self.where = [None] * self.n   # global slot -> (lane, local slot)
        for li, m in enumerate(members):
            st = torch.cuda.Stream(dev)
            self.lanes.append(BatchSolver([self.contexts[i] for i in m], precision, device=dev,
                                          policy=policy, stream=st))
            for local, g in enumerate(m):
                self.where[g] = (li, local)
        self.policy = self.lanes[0].policy
        self.stream = torch.cuda.current_stream(dev)
        self.device = dev

    def _l(self, slot):
        li, local = self.where[slot]
        return self.lanes[li], local

    @property
    def workspace_bytes(self) -> int:
        return sum(b.workspace_bytes for b in self.lanes)

    @property
    def _cfgs(self):
        out = [None] * self.n
        for g, (li, local) in enumerate(self.where):
            out[g] = self.lanes[li]._cfgs[local]
        return out

    def upload_table(self, records):
        import torch
        host = torch.from_numpy(np.ascontiguousarray(records).view(np.uint8)).pin_memory()
        return host.to(self.device, non_blocking=True)

    def start(self, slot, n_steps, t0=0.0, record=True, table=None):
        b, local = self._l(slot)
        b.stream.wait_stream(self.stream)   # the table was uploaded on the engine's stream
        b.start(local, n_steps, t0=t0, record=record, table=table)

    def stop(self, slot):
        b, local = self._l(slot)
        b.stop(local)

    def step(self, n_steps: int = 1) -> None:
        for b in self.lanes:               # every lane's graph is in flight before any wait
            b.step(n_steps)

    def step_eager(self) -> None:
        for b in self.lanes:
            b.step_eager()

    def status(self):
        infos = [b.status() for b in self.lanes]
        return [infos[li][local] for li, local in self.where]

    def buffer(self, slot, name):
        b, local = self._l(slot)
        return b.buffer(local, name)

    def modes(self, slot):
        return self.buffer(slot, "modes")

    def fetch(self, slot, name):
        b, local = self._l(slot)
        self.stream.wait_stream(b.stream)
        return b.fetch(local, name)

    def snapshot(self, slot, name):
        b, local = self._l(slot)
        out = b.snapshot(local, name)
        self.stream.wait_stream(b.stream)
        return out

    def export_slot(self, slot):
        b, local = self._l(slot)
        state = b.export_slot(local)
        self.stream.wait_stream(b.stream)
        return state

    def import_slot(self, slot, state, table):
        b, local = self._l(slot)
        b.stream.wait_stream(self.stream)
        b.import_slot(local, state, table)

    def volume_pass(self):
        # bracketed by the engine's stream, so events on it time every lane
        for b in self.lanes:
            b.stream.wait_stream(self.stream)
        for b in self.lanes:
            b.volume_pass()
        for b in self.lanes:
            self.stream.wait_stream(b.stream)

    def active_modes(self) -> int:
        return sum(b.active_modes() for b in self.lanes)

    def synchronize(self):
        for b in self.lanes:
            b.synchronize()
        self.stream.synchronize()

    def tensor_core_error(self) -> int:
        return max(b.tensor_core_error() for b in self.lanes)

    def launch_counts(self):
        pre, it, post = self.lanes[0].launch_counts()
        k = len(self.lanes)
        return pre * k, it * k, post * k

    def metrics(self, slot):
        b, local = self._l(slot)
        return b.metrics(local)

    def close(self):
        for b in self.lanes:
            b.close()
