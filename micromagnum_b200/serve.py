"""Serving: a request loop with continuous batching over `Batch`.

Requests (a relax or a timed switching solve of one box, with its arrival time) go, by size, to
one of a few size classes.  Each class is a `Batch` driven by its own host thread on its own CUDA
stream, so the classes' rounds overlap on the device and a small request never waits for the
rounds of a large one.  Within a class, requests are admitted in arrival order as soon as they
have arrived and their device memory (resident + set-up peak) fits the shared budget; admitted
requests join the running ones' lock-step rounds at the next tick (their tensor and spectra are
built while the other rounds run), keep state, tensor and spectra resident until they finish,
and leave the batch, freeing their memory, as soon as they finish.  Latency is the time from a
request's arrival to the host seeing its result.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import omf
from .batch import Batch, Instance


@dataclass
class Request:
    id: int
    instance: Instance
    M0: object  # (3, N) array in A/m, or the bytes of an OMF file of the instance's mesh
    arrival: float  # seconds after the start of the run


@dataclass
class Completed:
    id: int
    status: int  # 1 finished, 2 stopped on a non-finite state
    arrival: float
    admitted: float
    finished: float
    steps: int
    attempts: int
    M: object = None  # with keep_results: the final M, (3, N) array or (keep_results="omf") OMF bytes

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class ServeStats:
    completed: List[Completed] = field(default_factory=list)
    makespan: float = 0.0
    rebuilds: int = 0
    rounds: int = 0
    peak_resident: int = 0
    unfinished: int = 0  # requests not finished when the deadline passed
    progress: dict = field(default_factory=dict)  # request id -> accepted steps made (admitted requests)

    def percentile(self, q: float) -> float:
        return float(np.percentile([c.latency for c in self.completed], q)) if self.completed else float("nan")

    @property
    def solves_per_s(self) -> float:
        return len(self.completed) / self.makespan if self.makespan > 0 else 0.0


class _Class:
    """One size class: a batch, its queue of arrived requests and its running requests."""

    def __init__(self, batch: Batch, max_live: Optional[int] = None):
        self.batch = batch
        self.max_live = max_live
        self.queue = deque()
        self.live = {}  # slot -> (request, resident bytes, admitted)


class Server:
    def __init__(self, memory_budget: int, precision: str = "f32", eps_abs: float = 1e-3, eps_rel: float = 1e-4,
                 max_torque: float = 1e-4, check_every_nth_step: int = 1, rounds_per_tick: int = 8,
                 keep_results=False, class_bounds: Sequence[int] = (1 << 17, 1 << 20),
                 max_live: Optional[Sequence[int]] = None):
        """class_bounds: upper cell counts of the size classes (a last class takes the rest).
        keep_results: False, True (final M as a (3, N) array) or "omf" (final M as the bytes of an
        OMF binary-8 file, the wire format requests may also use for M0).
        max_live: the most requests each class runs at once (None: as many as memory allows).
        Under overload, running every admitted request at once shares the device among all of
        them and finishes none early; a bound serves them in arrival order, a batch at a time."""
        self.budget = int(memory_budget)
        self.precision = precision
        self.rounds_per_tick = int(rounds_per_tick)
        self.keep_results = keep_results
        self.bounds = list(class_bounds)
        self.max_live = list(max_live) if max_live is not None else [None] * (len(self.bounds) + 1)
        if len(self.max_live) != len(self.bounds) + 1:
            raise ValueError("max_live needs one bound per size class")
        self.classes = [_Class(Batch([], precision=precision, eps_abs=eps_abs, eps_rel=eps_rel,
                                     max_torque=max_torque, check_every_nth_step=check_every_nth_step), cap)
                        for cap in self.max_live]

    def _class_of(self, req: Request) -> _Class:
        n = req.instance.n
        for b, c in zip(self.bounds, self.classes):
            if n <= b:
                return c
        return self.classes[-1]

    def run(self, requests: List[Request], clock=time.perf_counter, deadline: Optional[float] = None) -> ServeStats:
        """Serves `requests`; with `deadline` (seconds) it stops admitting and running once the
        deadline has passed and counts the requests left over in `unfinished`."""
        stats = ServeStats()
        lock = threading.Lock()
        state = {"used": 0, "dispatching": True}
        t0 = clock()
        for r in requests:
            need = sum(r.instance.device_bytes(self.precision))
            if need > self.budget:
                raise MemoryError(f"request {r.id} needs {need} bytes, over the budget {self.budget}")

        def expired():
            return deadline is not None and clock() - t0 > deadline

        def worker(cl: _Class):
            while not expired():
                admitted = False
                while True:  # admit in arrival order while memory allows
                    with lock:
                        if not cl.queue or (cl.max_live is not None and len(cl.live) >= cl.max_live):
                            break
                        req = cl.queue[0]
                        res, trans = req.instance.device_bytes(self.precision)
                        # the budget is shared by every class, so an idle class waits too; each
                        # request fits alone (checked before the run), so memory freed by the
                        # other classes eventually admits it
                        if state["used"] + res + trans > self.budget:
                            break
                        state["used"] += res + trans  # set-up scratch held until add() returns
                        stats.peak_resident = max(stats.peak_resident, state["used"])
                        cl.queue.popleft()
                    slot = cl.batch.add(req.instance, req.M0)
                    with lock:
                        state["used"] -= trans
                    cl.live[slot] = (req, res, clock() - t0)
                    admitted = True
                if not cl.live:
                    with lock:
                        if not state["dispatching"] and not cl.queue:
                            return
                    time.sleep(0.0005)
                    continue
                rounds = cl.batch.relax(max_rounds=self.rounds_per_tick, check_interval=self.rounds_per_tick)
                results = cl.batch.results()
                now = clock() - t0
                done = []
                for slot in list(cl.live):
                    r = results[slot]
                    if r["status"] in (1, 2):
                        req, res, adm = cl.live.pop(slot)
                        M = None
                        if self.keep_results == "omf":
                            M = omf.format(cl.batch.get_M(slot), req.instance.dims, req.instance.delta,
                                           omf.BINARY_8, title=f"request {req.id}")
                        elif self.keep_results:
                            M = cl.batch.get_M(slot).cpu().numpy()
                        done.append((Completed(req.id, r["status"], req.arrival, adm, now, r["steps"], r["attempts"],
                                               M), slot, res))
                for c, slot, res in done:
                    cl.batch.remove(slot)
                with lock:
                    stats.rounds += rounds
                    stats.rebuilds += len(done) + (1 if admitted else 0)
                    for c, slot, res in done:
                        stats.completed.append(c)
                        state["used"] -= res

        threads = [threading.Thread(target=worker, args=(cl,), daemon=True) for cl in self.classes]
        for th in threads:
            th.start()
        for req in sorted(requests, key=lambda r: r.arrival):  # dispatch at arrival times
            wait = req.arrival - (clock() - t0)
            if wait > 0:
                time.sleep(wait)
            if expired():
                break
            with lock:
                self._class_of(req).queue.append(req)
        with lock:
            state["dispatching"] = False
        for th in threads:
            th.join()
        stats.makespan = clock() - t0
        for c in stats.completed:
            stats.progress[c.id] = c.steps
        for cl in self.classes:
            if cl.live:
                res = cl.batch.results()
                for slot, (req, _, _) in cl.live.items():
                    stats.progress[req.id] = res[slot]["steps"]
            for slot in list(cl.live):
                cl.batch.remove(slot)
            cl.live.clear()
            cl.queue.clear()
        stats.unfinished = len(requests) - len(stats.completed)
        stats.completed.sort(key=lambda c: c.id)
        return stats

    def close(self) -> None:
        for cl in self.classes:
            cl.batch.close()
