"""Serving: a request loop with continuous batching over `Batch`.

Requests (a relax or a timed switching solve of one box, with its arrival time) are admitted in
arrival order as soon as they have arrived and their device memory fits the budget; admitted
requests join the lock-step rounds of the running ones (their tensor and spectra are built while
the others' rounds are on the device), keep their state, tensor and spectra resident until they
finish, and leave the batch, freeing their memory, as soon as they finish.  Latency is the time
from a request's arrival to the host seeing its result.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .batch import Batch, Instance


@dataclass
class Request:
    id: int
    instance: Instance
    M0: np.ndarray
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
    M: Optional[np.ndarray] = None

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

    def percentile(self, q: float) -> float:
        return float(np.percentile([c.latency for c in self.completed], q)) if self.completed else float("nan")

    @property
    def solves_per_s(self) -> float:
        return len(self.completed) / self.makespan if self.makespan > 0 else 0.0


class Server:
    def __init__(self, memory_budget: int, precision: str = "f32", eps_abs: float = 1e-3, eps_rel: float = 1e-4,
                 max_torque: float = 1e-4, check_every_nth_step: int = 1, rounds_per_tick: int = 8,
                 keep_results: bool = False):
        self.budget = int(memory_budget)
        self.batch = Batch([], precision=precision, eps_abs=eps_abs, eps_rel=eps_rel, max_torque=max_torque,
                           check_every_nth_step=check_every_nth_step)
        self.precision = precision
        self.rounds_per_tick = int(rounds_per_tick)
        self.keep_results = keep_results

    def run(self, requests: List[Request], clock=time.perf_counter, deadline: Optional[float] = None) -> ServeStats:
        """Serves `requests`; with `deadline` (seconds) it stops admitting and running once the
        deadline has passed and counts the requests left over in `unfinished`."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        live = {}  # slot -> (request, resident bytes, admitted)
        used = 0
        stats = ServeStats()
        t0 = clock()
        while pending or live:
            now = clock() - t0
            if deadline is not None and now > deadline:
                break
            while pending and pending[0].arrival <= now:
                req = pending[0]
                res, trans = req.instance.device_bytes(self.precision)
                if live and used + res + trans > self.budget:
                    break  # wait until running requests free memory
                if res + trans > self.budget:
                    raise MemoryError(f"request {req.id} needs {res + trans} bytes, over the budget {self.budget}")
                slot = self.batch.add(req.instance, req.M0)
                used += res
                stats.peak_resident = max(stats.peak_resident, used)
                live[slot] = (req, res, clock() - t0)
                pending.popleft()
                stats.rebuilds += 1
            if not live:
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - (clock() - t0)))
                continue
            stats.rounds += self.batch.relax(max_rounds=self.rounds_per_tick, check_interval=self.rounds_per_tick)
            results = self.batch.results()
            now = clock() - t0
            for slot in list(live):
                r = results[slot]
                if r["status"] in (1, 2):
                    req, res, adm = live.pop(slot)
                    M = self.batch.get_M(slot).cpu().numpy() if self.keep_results else None
                    stats.completed.append(Completed(req.id, r["status"], req.arrival, adm, now, r["steps"],
                                                     r["attempts"], M))
                    self.batch.remove(slot)
                    used -= res
                    stats.rebuilds += 1
        stats.makespan = clock() - t0
        stats.unfinished = len(pending) + len(live)
        for slot in list(live):
            self.batch.remove(slot)
        return stats

    def close(self) -> None:
        self.batch.close()
