"""Device-resident serving loop for carrier-step requests.

A request asks for k steps of the fixed-box carrier on a fresh box of a given
edge, initialised with a seeded random-Fourier velocity. The loop is
continuous batching, not a queue: every admitted request owns a resident
carrier (its own CUDA stream and step graph), each request's next step is
launched as soon as its previous one finishes, and requests that arrive while
others are on the device are admitted as soon as a carrier slot fits in the
HBM budget. Their steps overlap on the device. The host only launches step
graphs and polls for completion.

Carriers are pooled by edge and reused: admission costs one device-side
initialisation, not an allocation, once a carrier of that size exists. The
pool never holds more than the budget; idle carriers of other sizes are
released (least recently used first) to make room.

Multi-GPU: requests are sharded across ranks by request id (independent boxes,
no collective on the data path); latencies are merged on rank 0.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import CarrierConfig, CarrierSimulation, GridGeometry, StepParams
from . import workloads as W

MAXF = 1.7976931348623157e308


@dataclass
class Request:
    rid: int
    arrival: float      # seconds after the start of the run
    edge: int           # cells per axis
    steps: int
    seed: int


@dataclass
class Completion:
    rid: int
    edge: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    status: int
    iterations: List[int] = field(default_factory=list)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def make_requests(count: int, rate_hz: float, seed: int = W.DEFAULT_SEED, edge_min: int = 32, edge_max: int = 256,
                  max_steps: int = 20) -> List[Request]:
    """Poisson arrivals at rate_hz; edge log-uniform in [edge_min, edge_max]
    rounded to a multiple of 8; steps uniform in [1, max_steps]; all drawn
    from counter-based SplitMix64 streams of `seed`."""
    u_gap = (W.uniform(seed, 32, count) + 1.0) * 0.5
    u_edge = (W.uniform(seed, 33, count) + 1.0) * 0.5
    u_steps = (W.uniform(seed, 34, count) + 1.0) * 0.5
    gaps = -np.log1p(-np.minimum(u_gap, 1.0 - 1e-16)) / rate_hz if rate_hz > 0 else np.zeros(count)
    arrivals = np.cumsum(gaps) - (gaps[0] if count else 0.0)
    log_e = math.log(edge_min) + u_edge * (math.log(edge_max) - math.log(edge_min))
    edges = np.clip(np.round(np.exp(log_e) / 8.0) * 8, edge_min, edge_max).astype(int)
    steps = np.minimum(max_steps, 1 + np.floor(u_steps * max_steps)).astype(int)
    return [Request(i, float(arrivals[i]), int(edges[i]), int(steps[i]), int(seed + 7919 * (i + 1)))
            for i in range(count)]


def shard_requests(requests: Sequence[Request], rank: int, world: int) -> List[Request]:
    """Requests of one rank: id modulo world size (independent boxes)."""
    return [r for r in requests if r.rid % world == rank]


def percentiles(latencies: Sequence[float]) -> Dict[str, float]:
    if not latencies:
        return {"p50": float("nan"), "p95": float("nan"), "p99": float("nan")}
    a = np.sort(np.asarray(latencies, dtype=np.float64))
    return {f"p{q}": float(np.percentile(a, q)) for q in (50, 95, 99)}


def merge_completions(per_rank: Sequence[Sequence[Completion]]) -> List[Completion]:
    out: List[Completion] = []
    for part in per_rank:
        out.extend(part)
    return sorted(out, key=lambda c: c.rid)


def carrier_bytes_estimate(edge: int, config: CarrierConfig) -> int:
    """Device bytes of one carrier (three face buffers, solver vectors, the
    FP32 multigrid hierarchy), before it is created."""
    n = edge ** 3
    faces = 3 * edge * edge * (edge + 1)
    elem = 4 if config.storage == "f32" else 8
    per_cell = 8 * 7 + (6 if config.implementation == 3 else 0) + (8 if config.warm_start else 0)
    return 3 * faces * elem + n * per_cell + (1 << 20)


class CarrierPool:
    """Resident carriers keyed by edge, bounded by an HBM byte budget."""

    def __init__(self, config: CarrierConfig, budget_bytes: int):
        self.config = config
        self.budget = int(budget_bytes)
        self.used = 0
        self.free: Dict[int, List[CarrierSimulation]] = collections.defaultdict(list)
        self.lru: "collections.OrderedDict[int, None]" = collections.OrderedDict()
        self.created = 0

    def acquire(self, edge: int) -> Optional[CarrierSimulation]:
        if self.free[edge]:
            self.lru.pop(id(self.free[edge][-1]), None)
            return self.free[edge].pop()
        need = carrier_bytes_estimate(edge, self.config)
        while self.used + need > self.budget and self._evict_one(except_edge=edge):
            pass
        if self.used + need > self.budget:
            return None
        sim = CarrierSimulation(GridGeometry((edge, edge, edge)), self.config)
        self.used += sim.allocated_bytes()
        self.created += 1
        return sim

    def release(self, edge: int, sim: CarrierSimulation) -> None:
        self.free[edge].append(sim)
        self.lru[id(sim)] = None

    def _evict_one(self, except_edge: int) -> bool:
        for key in list(self.lru.keys()):
            for edge, sims in self.free.items():
                if edge == except_edge:
                    continue
                for i, sim in enumerate(sims):
                    if id(sim) == key:
                        sims.pop(i)
                        self.lru.pop(key, None)
                        self.used -= sim.allocated_bytes()
                        sim.close()
                        return True
        return False

    def close(self) -> None:
        for sims in self.free.values():
            for sim in sims:
                sim.close()
        self.free.clear()
        self.lru.clear()
        self.used = 0


class ServingLoop:
    """Continuous-batching loop over resident carriers (see module docstring)."""

    def __init__(self, config: CarrierConfig, budget_bytes: int, params: Optional[StepParams] = None,
                 max_in_flight: int = 1 << 30):
        self.pool = CarrierPool(config, budget_bytes)
        self.params = params or StepParams(MAXF, cfl=0.5)
        self.max_in_flight = max_in_flight

    def run(self, requests: Sequence[Request], keep_state: bool = False,
            on_complete: Optional[Callable[[Completion, CarrierSimulation], None]] = None) -> List[Completion]:
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        active: Dict[int, dict] = {}
        done: List[Completion] = []
        self.final_states: Dict[int, list] = {}
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            # admission: arrivals whose time has come, while a carrier fits
            while pending and pending[0].arrival <= now and len(active) < self.max_in_flight:
                req = pending[0]
                sim = self.pool.acquire(req.edge)
                if sim is None:
                    break
                pending.popleft()
                sim.init_fourier(req.seed)
                sim.step_async(self.params)
                active[req.rid] = {"req": req, "sim": sim, "done": 0, "admitted": now, "its": []}
            progressed = False
            for rid in list(active):
                slot = active[rid]
                sim = slot["sim"]
                if not sim.step_done():
                    continue
                progressed = True
                status = 0
                try:
                    rep = sim.step_wait()
                    slot["its"].append(rep.pressure.iterations)
                except Exception as e:  # a rejected step ends the request
                    status = getattr(e, "status", -1)
                slot["done"] += 1
                req = slot["req"]
                if status == 0 and slot["done"] < req.steps:
                    sim.step_async(self.params)
                    continue
                finished = time.perf_counter() - t0
                comp = Completion(req.rid, req.edge, slot["done"], req.arrival, slot["admitted"], finished, status,
                                  slot["its"])
                done.append(comp)
                if keep_state:
                    self.final_states[req.rid] = sim.download()
                if on_complete:
                    on_complete(comp, sim)
                self.pool.release(req.edge, sim)
                del active[rid]
            if not progressed:
                if pending and not active:
                    wait = pending[0].arrival - (time.perf_counter() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
                else:
                    time.sleep(0.00005)
        self.elapsed = time.perf_counter() - t0
        return sorted(done, key=lambda c: c.rid)

    def close(self) -> None:
        self.pool.close()


def summarize(completions: Sequence[Completion], elapsed: float) -> dict:
    from . import status_name

    ok = [c for c in completions if c.status == 0]
    rejected: Dict[str, int] = {}
    for c in completions:
        if c.status != 0:
            name = status_name(c.status) if c.status >= 0 else "Error"
            rejected[name] = rejected.get(name, 0) + 1
    cell_steps = sum(c.edge ** 3 * c.steps for c in ok)
    lat = percentiles([c.latency for c in ok])
    return {
        "requests": len(completions),
        "accepted": len(ok),
        "rejected": rejected,
        "elapsed_s": elapsed,
        "requests_per_s": len(ok) / elapsed if elapsed > 0 else float("nan"),
        "cell_steps_per_s": cell_steps / elapsed if elapsed > 0 else float("nan"),
        "latency_s": lat,
    }
