"""Continuous batching of UVLM cases on one GPU.

Cases of uneven lattice and wake sizes arrive over time.  Each admitted case keeps its
wake, circulation history and cached factors resident in HBM (its ``DeviceCase``); the
loop advances every active case by one time step per iteration with a single set of
kernel launches (``fj_step_batched``), admits waiting cases as device memory frees up
(admission by footprint), and retires finished cases.  Per-step latency is the device
time of the batched iteration a case's step ran in, measured with CUDA events.

With ``overlap_admission`` (the default) ``admission_workers`` host threads admit cases,
each on its own CUDA stream -- static solve and first, factorising step, which are
latency-bound LU panels -- while the batched steps of the active cases run on the main
stream; a case joins the batch once its admission event has completed.
"""
from __future__ import annotations

import ctypes as C
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .runtime import DeviceCase


class BatchStepper:
    """Advances a set of device cases by one step each, in one batched call."""

    def __init__(self, max_items: int, device=None):
        import torch

        from .runtime import device_of

        self.torch = torch
        self.dev = device_of(device)
        self.max_items = max_items
        n = C.c_size_t()
        _lib.call("fj_batch_workspace_size", max_items, C.byref(n))
        self.ws = torch.empty(n.value, dtype=torch.uint8, device=self.dev)

    def step(self, cases: list[DeviceCase], slots: list[int], reuse: list[bool], stream=None, graph: bool = True):
        """One step of each case.  ``graph``: replay the batch's captured CUDA graph when the
        batch has the launch signature of the last call (fj_step_batched); False launches
        every kernel directly (same results)."""
        if not cases:
            return
        if len(cases) > self.max_items:
            raise ValueError(f"batch of {len(cases)} exceeds {self.max_items}")
        items = (_lib.FjBatchItem * len(cases))()
        for k, (dc, i, r) in enumerate(zip(cases, slots, reuse)):
            items[k].cfg = C.pointer(dc.cfg)
            items[k].bufs = C.pointer(dc._bufs)
            items[k].d_ws = dc.ws.data_ptr()
            items[k].ws_bytes = dc.ws.numel()
            items[k].i_ts = int(i)
            items[k].flags = (_lib.FJ_REUSE_FACTORS if r else 0) | (0 if graph else _lib.FJ_NO_GRAPH)
        s = (stream or self.torch.cuda.current_stream(self.dev)).cuda_stream
        _lib.call("fj_step_batched", items, len(cases), self.ws.data_ptr(), self.ws.numel(), s)

    def close(self):
        """Drops the captured graph of this stepper's batch workspace."""
        if self.ws is not None:
            self.torch.cuda.synchronize(self.dev)
            _lib.call("fj_batch_release", self.ws.data_ptr())
            self.ws = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the process releases everything
            pass


def graph_stats() -> dict:
    """Batched-step graph replays and captures since the library was loaded."""
    r, c = C.c_int64(), C.c_int64()
    _lib.call("fj_batch_graph_stats", C.byref(r), C.byref(c))
    return {"replays": int(r.value), "captures": int(c.value)}


def residual(dc: DeviceCase, i: int) -> float:
    out = C.c_double()
    _lib.call("fj_case_residual", C.byref(dc.cfg), dc.ws.data_ptr(), dc.ws.numel(), int(i), C.byref(out),
              dc._stream())
    return out.value


def case_footprint_bytes(uvlm, n_tstep: int) -> int:
    """Device bytes a case holds while active: time-batched outputs, node frames,
    workspace (AIC, factors, streams, partials)."""
    cfg = uvlm._config(n_tstep, uvlm.hg_ref.shape[0])
    n = C.c_size_t()
    _lib.call("fj_case_workspace_size", C.byref(cfg), C.byref(n))
    lay = uvlm._layout()
    per_slot = 0
    for f in ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
              "f_unsteady", "alpha"):
        per_slot += lay.blocks(f)[1]
    per_slot += 4 + 2 * cfg.n_nodes * 16
    return int(n.value) + per_slot * n_tstep * 8


@dataclass
class Request:
    """One case: a configured ``UVLM`` (design variables set), its motion and length."""

    uvlm: object
    hg_t: np.ndarray
    hg_dot_t: np.ndarray
    arrival: float = 0.0
    tag: object = None


@dataclass
class _Active:
    req: Request
    dc: DeviceCase
    next_slot: int
    n_tstep: int
    footprint: int
    admitted_at: float
    step_ms: list = field(default_factory=list)


@dataclass
class ServeResult:
    results: dict
    step_latency_ms: np.ndarray
    case_steps: int
    wall_s: float
    gpu_busy_s: float
    admit_latency_s: np.ndarray
    max_active: int

    def summary(self):
        lat = self.step_latency_ms
        return {
            "case_steps": self.case_steps,
            "wall_s": self.wall_s,
            "steps_per_s": self.case_steps / self.wall_s if self.wall_s > 0 else None,
            "gpu_steps_per_s": self.case_steps / self.gpu_busy_s if self.gpu_busy_s > 0 else None,
            "p50_step_ms": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_step_ms": float(np.percentile(lat, 99)) if lat.size else None,
            "mean_step_ms": float(lat.mean()) if lat.size else None,
            "p50_admit_s": float(np.percentile(self.admit_latency_s, 50)) if self.admit_latency_s.size else None,
            "p99_admit_s": float(np.percentile(self.admit_latency_s, 99)) if self.admit_latency_s.size else None,
            "max_active": self.max_active,
        }


class ServingLoop:
    """Continuous batching over one GPU.

    ``memory_budget`` bounds the sum of active case footprints (bytes); ``max_active``
    bounds the batch width.  ``realtime``: requests become visible at their ``arrival``
    (seconds after ``run`` starts); otherwise all are queued at once.
    """

    def __init__(self, memory_budget: int, max_active: int = 256, device=None, keep_results=True,
                 admit_per_iteration: int = 4, overlap_admission: bool = True, admission_workers: int = 4):
        import torch

        from .runtime import device_of

        self.torch = torch
        self.dev = device_of(device)
        self.memory_budget = int(memory_budget)
        self.max_active = max_active
        self.stepper = BatchStepper(max_active, self.dev)
        self.keep_results = keep_results
        self.admit_per_iteration = admit_per_iteration
        self.overlap_admission = overlap_admission
        self.admission_workers = max(1, int(admission_workers))

    def _admit(self, req: Request, now: float, stream=None) -> _Active:
        """Static solve and the first (factorising) step run for the case alone, so the
        batched steps it joins reuse its cached factors and stay uniform.  The static
        solve writes slot 0 of the case in place (the frames of the reference
        configuration, ``UVLM.solve_static()``), so nothing crosses to the host."""
        uv = req.uvlm
        n_tstep = req.hg_t.shape[0]
        dc = uv.make_device_case(n_tstep, req.hg_t.shape[1], stream=stream)
        dc.set_hg(req.hg_t, req.hg_dot_t)
        dc.hg_t[0].copy_(self.torch.from_numpy(np.ascontiguousarray(uv.hg_ref, dtype=np.float64)))
        dc.solve_static(False, 0.0)
        dc.hg_t[0].copy_(self.torch.from_numpy(np.ascontiguousarray(req.hg_t[0], dtype=np.float64)))
        first = 1
        if n_tstep > 1:
            dc.solve_dynamic(1, 2)
            first = 2
        return _Active(req, dc, first, n_tstep, case_footprint_bytes(uv, n_tstep), now)

    def _retire(self, a: _Active, results: dict):
        if self.keep_results:
            results[a.req.tag if a.req.tag is not None else id(a.req)] = a.req.uvlm._to_case(a.dc)
        a.dc = None

    def run(self, requests: list[Request], realtime: bool = True) -> ServeResult:
        if self.overlap_admission:
            return self._run_overlapped(requests, realtime)
        return self._run_serial(requests, realtime)

    def _run_overlapped(self, requests: list[Request], realtime: bool) -> ServeResult:
        torch = self.torch
        pending = sorted(requests, key=lambda r: r.arrival)
        n_total = len(pending)
        cond = threading.Condition()
        state = {"used": 0, "inflight": 0, "error": None, "next": 0}
        ready: queue.Queue = queue.Queue()
        t0 = time.perf_counter()

        def worker():
            try:
                torch.cuda.set_device(self.dev)
                adm_stream = torch.cuda.Stream(self.dev)
                while True:
                    with cond:  # requests are taken in arrival order
                        k = state["next"]
                        if k >= n_total or state["error"] is not None:
                            return
                        state["next"] = k + 1
                    req = pending[k]
                    if realtime:
                        wait = req.arrival - (time.perf_counter() - t0)
                        if wait > 0:
                            time.sleep(wait)
                    est = case_footprint_bytes(req.uvlm, req.hg_t.shape[0])
                    with cond:
                        # footprint budget and batch width; an empty system always admits
                        while state["inflight"] > 0 and (state["used"] + est > self.memory_budget
                                                         or state["inflight"] >= self.max_active):
                            cond.wait()
                        state["used"] += est
                        state["inflight"] += 1
                    with torch.cuda.stream(adm_stream):
                        a = self._admit(req, time.perf_counter() - t0, stream=adm_stream)
                        a.footprint = est
                        ev = torch.cuda.Event()
                        ev.record(adm_stream)
                    ready.put((a, ev, time.perf_counter() - t0))
            except BaseException as e:  # surfaced by the stepping loop
                state["error"] = e
                ready.put(None)

        threads = [threading.Thread(target=worker, daemon=True) for _ in range(self.admission_workers)]
        for th in threads:
            th.start()
        active: list[_Active] = []
        results = {}
        lat, admit_lat = [], []
        busy_s = 0.0
        steps = 0
        max_act = 0
        received = 0
        stream = torch.cuda.current_stream(self.dev)

        def release(a):
            with cond:
                state["used"] -= a.footprint
                state["inflight"] -= 1
                cond.notify_all()

        while received < n_total or active:
            # take every admitted case; block only when nothing is running
            while received < n_total:
                try:
                    item = ready.get(block=not active, timeout=None if not active else 0)
                except queue.Empty:
                    break
                if item is None:
                    raise state["error"]
                a, ev, done_at = item
                received += 1
                stream.wait_event(ev)
                a.dc.stream = None  # from here on the case lives on the stepping stream
                if a.next_slot > 1:
                    steps += 1
                admit_lat.append(max(0.0, done_at - a.req.arrival) if realtime else 0.0)
                if a.next_slot >= a.n_tstep:
                    ev.synchronize()
                    self._retire(a, results)
                    release(a)
                else:
                    active.append(a)
            if not active:
                continue
            max_act = max(max_act, len(active))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            self.stepper.step([a.dc for a in active], [a.next_slot for a in active],
                              [a.next_slot > 1 for a in active], stream)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            busy_s += ms * 1e-3
            for a in active:
                a.step_ms.append(ms)
                lat.append(ms)
                a.next_slot += 1
                steps += 1
            done = [a for a in active if a.next_slot >= a.n_tstep]
            for a in done:
                self._retire(a, results)
                active.remove(a)
                release(a)
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        return ServeResult(results, np.asarray(lat), steps, wall, busy_s, np.asarray(admit_lat), max_act)

    def _run_serial(self, requests: list[Request], realtime: bool) -> ServeResult:
        torch = self.torch
        pending = sorted(requests, key=lambda r: r.arrival)
        active: list[_Active] = []
        used = 0
        results = {}
        lat, admit_lat = [], []
        busy_s = 0.0
        steps = 0
        max_act = 0
        t0 = time.perf_counter()
        stream = torch.cuda.current_stream(self.dev)
        while pending or active:
            now = time.perf_counter() - t0
            # admission: arrived requests, while the footprint budget and batch width allow
            # (a few per iteration, so a burst of arrivals does not stall running cases)
            admitted = 0
            while (pending and (not realtime or pending[0].arrival <= now) and len(active) < self.max_active
                   and (admitted < self.admit_per_iteration or not active)):
                est = case_footprint_bytes(pending[0].uvlm, pending[0].hg_t.shape[0])
                if active and used + est > self.memory_budget:
                    break
                req = pending.pop(0)
                a = self._admit(req, now)
                used += a.footprint
                admitted += 1
                if a.next_slot > 1:
                    steps += 1
                if a.next_slot >= a.n_tstep:
                    self._retire(a, results)
                    used -= a.footprint
                else:
                    active.append(a)
                done_at = time.perf_counter() - t0
                admit_lat.append(max(0.0, done_at - req.arrival) if realtime else 0.0)
            if not active:
                if pending and realtime:
                    time.sleep(max(0.0, min(pending[0].arrival - now, 0.002)))
                continue
            max_act = max(max_act, len(active))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            self.stepper.step([a.dc for a in active], [a.next_slot for a in active],
                              [a.next_slot > 1 for a in active], stream)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            busy_s += ms * 1e-3
            for a in active:
                a.step_ms.append(ms)
                lat.append(ms)
                a.next_slot += 1
                steps += 1
            done = [a for a in active if a.next_slot >= a.n_tstep]
            for a in done:
                self._retire(a, results)
                active.remove(a)
                used -= a.footprint
        wall = time.perf_counter() - t0
        return ServeResult(results, np.asarray(lat), steps, wall, busy_s, np.asarray(admit_lat), max_act)
