"""Serving: continuous batching of flood scenarios on one GPU (hf_server_*).

Requests arrive over time; each is admitted into a slot as soon as a slot is
free and its fields fit the HBM budget, then advances together with every
other admitted scenario (one launch per stage over all their tiles; a
scenario that fills the GPU by itself gets its own launches). A
finished scenario is collected, freeing its slot and memory for the next
request. `serve_stream` drives an arrival stream and reports per-request
latency (arrival -> result) and throughput.
"""
from __future__ import annotations

import collections
import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import abi
from ._lib import lib
from .ensemble import _Desc
from .sim import raise_for
from .workloads import Scenario, uniform, valley


class Server:
    def __init__(self, hbm_budget_bytes: int, max_slots: int = 1024, device: int = 0,
                 max_steps: int = 10_000_000):
        h = C.c_void_p()
        raise_for(lib().hf_server_create(int(device), int(hbm_budget_bytes), int(max_slots),
                                         C.byref(h)))
        self._h = h
        self._max_steps = max_steps
        self._shapes: Dict[int, tuple] = {}

    def try_admit(self, s: Scenario) -> Optional[int]:
        """Slot id, or None when there is no capacity right now."""
        d = _Desc(s, self._max_steps)
        slot = C.c_int()
        rc = lib().hf_server_admit(self._h, C.byref(d.c), C.byref(slot))
        if rc == abi.HF_ERR_CAPACITY:
            return None
        raise_for(rc)
        self._shapes[slot.value] = s.shape
        return slot.value

    def advance(self, n_batch_steps: int) -> int:
        n = C.c_int()
        raise_for(lib().hf_server_advance(self._h, int(n_batch_steps), C.byref(n)))
        return n.value

    def finished(self) -> List[int]:
        buf = (C.c_int * 4096)()
        n = C.c_int()
        raise_for(lib().hf_server_finished(self._h, buf, 4096, C.byref(n)))
        return list(buf[:n.value])

    def collect(self, slot: int, with_state: bool = True):
        shape = self._shapes.pop(slot)
        out = [np.empty(shape) for _ in range(3)] if with_state else [None] * 3
        t, st, status = C.c_double(), C.c_uint64(), C.c_int()
        ptrs = [o.ctypes.data if o is not None else None for o in out]
        raise_for(lib().hf_server_collect(self._h, int(slot), *ptrs, C.byref(t), C.byref(st),
                                          C.byref(status)))
        return {"state": tuple(out) if with_state else None, "t": t.value, "steps": st.value,
                "status": status.value}

    def usage(self):
        b, n = C.c_uint64(), C.c_int()
        raise_for(lib().hf_server_usage(self._h, C.byref(b), C.byref(n)))
        return b.value, n.value

    def close(self):
        if getattr(self, "_h", None):
            lib().hf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class Request:
    rid: int
    arrival: float
    make: Callable[[], Scenario]
    admitted: Optional[float] = None
    done: Optional[float] = None
    result: Optional[dict] = None
    scenario: Optional[Scenario] = None  # the payload, once built (prepare)

    def prepare(self) -> Scenario:
        if self.scenario is None:
            self.scenario = self.make()
        return self.scenario

    def work(self) -> float:
        """Work estimate: cells x horizon."""
        s = self.prepare()
        return float(s.n_cells) * float(s.t_end)


def serve_stream(requests: Sequence[Request], hbm_budget_bytes: int, chunk: int = 8,
                 max_slots: int = 1024, device: int = 0, keep_state: bool = False,
                 time_scale: float = 1.0, policy: str = "fifo",
                 max_active_cells: Optional[int] = None) -> dict:
    """Run an arrival stream (arrival times in seconds of wall clock, scaled
    by time_scale) through a server. Admission: "fifo" in arrival order, or
    "srpt", the arrived request with the least work (cells x horizon) first.
    max_active_cells caps the cells advancing together (a request is admitted
    while the cap holds, or when nothing runs); the HBM budget and max_slots
    always apply. Payloads are built when first needed (Request.prepare; call
    it beforehand to keep generation out of the served time). Returns
    per-request latencies and the throughput."""
    if policy not in ("fifo", "srpt"):
        raise ValueError("policy must be 'fifo' or 'srpt'")
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    arrived: List[Request] = []
    by_slot: Dict[int, Request] = {}
    active_cells = 0
    with Server(hbm_budget_bytes, max_slots=max_slots, device=device) as srv:
        t0 = time.perf_counter()
        now = lambda: (time.perf_counter() - t0) / time_scale  # noqa: E731
        while pending or arrived or by_slot:
            while pending and pending[0].arrival <= now():
                arrived.append(pending.popleft())
            if policy == "srpt":
                arrived.sort(key=lambda r: r.work())
            while arrived:
                r = arrived[0]
                s = r.prepare()
                if (max_active_cells is not None and by_slot
                        and active_cells + s.n_cells > max_active_cells):
                    break
                slot = srv.try_admit(s)
                if slot is None:
                    break
                arrived.pop(0)
                r.admitted = now()
                by_slot[slot] = r
                active_cells += s.n_cells
            if not by_slot and arrived:
                raise RuntimeError(f"request {arrived[0].rid} does not fit the server "
                                   "(HBM budget or slots)")
            if not by_slot:
                if pending:
                    time.sleep(max(0.0, min(0.01, (pending[0].arrival - now()) * time_scale)))
                continue
            srv.advance(chunk)
            for slot in srv.finished():
                res = srv.collect(slot, with_state=keep_state)
                r = by_slot.pop(slot)
                active_cells -= r.scenario.n_cells
                r.done = now()
                r.result = res
        makespan = now()
    lat = np.array([r.done - r.arrival for r in requests])
    return {"latency_p50": float(np.percentile(lat, 50)), "latency_p99": float(np.percentile(lat, 99)),
            "solves_per_s": len(requests) / makespan, "makespan": makespan,
            "n": len(requests), "failed": sum(1 for r in requests if r.result["status"] != 0),
            "latencies": lat.tolist()}


def request_stream(count: int, rate: float, seed: int = 0, sides=(128, 256, 512, 1024, 2048),
                   horizon_min: float = 300.0, horizon_max: float = 3600.0,
                   max_dt: float = 60.0) -> List[Request]:
    """Poisson arrivals at `rate` per second; side uniform over `sides`,
    horizon uniform in [horizon_min, horizon_max] s, valley scenario with a
    per-request seed (built lazily at admission), step cap `max_dt`."""
    gaps = -np.log1p(-uniform(seed, 200, count)) / rate
    arrivals = np.cumsum(gaps)
    side_idx = np.minimum((uniform(seed, 201, count) * len(sides)).astype(int), len(sides) - 1)
    horizons = uniform(seed, 202, count, horizon_min, horizon_max)
    out = []
    for k in range(count):
        side = int(sides[side_idx[k]])
        hz = float(horizons[k])
        sd = seed * 1000003 + k + 1
        out.append(Request(k, float(arrivals[k]),
                           (lambda side=side, hz=hz, sd=sd: _capped(valley(n=side, dx=5.0,
                                                                          seed=sd, t_end=hz),
                                                                   max_dt))))
    return out


def _capped(s: Scenario, max_dt: float) -> Scenario:
    s.max_dt = max_dt
    return s
