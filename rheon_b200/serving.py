"""Device-resident serving loop for carrier-step and projection requests.

A step request asks for k steps of the fixed-box carrier on a fresh box of a
given edge, initialised with a seeded random-Fourier velocity. A projection
request supplies a velocity (here the seeded random-Fourier field, generated
on the device) that is projected once with its own dt
(ProjectionStepWorkspace::project, src/projection_step.rs:863-1033): the
corrected faces and the pressure are its result. The loop is
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
    steps: int          # 1 for a projection
    seed: int
    kind: str = "step"  # "step" or "projection"
    dt: float = 0.0     # a projection's dt


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
    kind: str = "step"
    # device interval of the request's work (ms after the loop's reference
    # event): from before its first launch to after its last one
    device_start_ms: float = float("nan")
    device_end_ms: float = float("nan")

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def make_requests(count: int, rate_hz: float, seed: int = W.DEFAULT_SEED, edge_min: int = 32, edge_max: int = 256,
                  max_steps: int = 20, projection_share: float = 0.0, projection_dt: float = 0.01) -> List[Request]:
    """Poisson arrivals at rate_hz; edge log-uniform in [edge_min, edge_max]
    rounded to a multiple of 8; steps uniform in [1, max_steps]; a share of
    the requests are projections (one projection with dt = projection_dt);
    all drawn from counter-based SplitMix64 streams of `seed`."""
    u_gap = (W.uniform(seed, 32, count) + 1.0) * 0.5
    u_edge = (W.uniform(seed, 33, count) + 1.0) * 0.5
    u_steps = (W.uniform(seed, 34, count) + 1.0) * 0.5
    u_kind = (W.uniform(seed, 35, count) + 1.0) * 0.5
    gaps = -np.log1p(-np.minimum(u_gap, 1.0 - 1e-16)) / rate_hz if rate_hz > 0 else np.zeros(count)
    arrivals = np.cumsum(gaps) - (gaps[0] if count else 0.0)
    log_e = math.log(edge_min) + u_edge * (math.log(edge_max) - math.log(edge_min))
    edges = np.clip(np.round(np.exp(log_e) / 8.0) * 8, edge_min, edge_max).astype(int)
    steps = np.minimum(max_steps, 1 + np.floor(u_steps * max_steps)).astype(int)
    out = []
    for i in range(count):
        proj = bool(u_kind[i] < projection_share)
        out.append(Request(i, float(arrivals[i]), int(edges[i]), 1 if proj else int(steps[i]),
                           int(seed + 7919 * (i + 1)), "projection" if proj else "step",
                           projection_dt if proj else 0.0))
    return out


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
        # make room by the estimate, then book the carrier's actual bytes:
        # a carrier that turns out larger than estimated makes more room or
        # is released, so the pool never exceeds the budget
        need = carrier_bytes_estimate(edge, self.config)
        while self.used + need > self.budget and self._evict_one(except_edge=edge):
            pass
        if self.used + need > self.budget:
            return None
        sim = CarrierSimulation(GridGeometry((edge, edge, edge)), self.config)
        actual = sim.allocated_bytes()
        while self.used + actual > self.budget and self._evict_one(except_edge=edge):
            pass
        if self.used + actual > self.budget:
            sim.close()
            return None
        self.used += actual
        self.created += 1
        assert self.used <= self.budget
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
                 max_in_flight: int = 1 << 30, device_times: bool = False):
        self.pool = CarrierPool(config, budget_bytes)
        self.params = params or StepParams(MAXF, cfl=0.5)
        self.max_in_flight = max_in_flight
        self.device_times = device_times

    def _event(self, sim: Optional[CarrierSimulation]):
        """A timing event recorded on the carrier's stream (None: the current
        stream), or None without device timing."""
        if not self.device_times:
            return None
        import torch

        ev = torch.cuda.Event(enable_timing=True)
        if sim is None:
            ev.record()
        else:
            ev.record(torch.cuda.ExternalStream(sim.stream()))
        return ev

    def _launch(self, req: Request, sim: CarrierSimulation) -> None:
        if req.kind == "projection":
            sim.project_async(req.dt)
        else:
            sim.step_async(self.params)

    def run(self, requests: Sequence[Request], keep_state: bool = False,
            on_complete: Optional[Callable[[Completion, CarrierSimulation], None]] = None) -> List[Completion]:
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        active: Dict[int, dict] = {}
        done: List[Completion] = []
        self.final_states: Dict[int, list] = {}
        self.final_pressures: Dict[int, np.ndarray] = {}
        ref = self._event(None)
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
                start = self._event(sim)
                sim.init_fourier(req.seed)
                self._launch(req, sim)
                active[req.rid] = {"req": req, "sim": sim, "done": 0, "admitted": now, "its": [],
                                   "start": start, "end": self._event(sim)}
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
                    self._launch(req, sim)
                    slot["end"] = self._event(sim)
                    continue
                finished = time.perf_counter() - t0
                comp = Completion(req.rid, req.edge, slot["done"], req.arrival, slot["admitted"], finished, status,
                                  slot["its"], req.kind)
                if ref is not None:
                    comp.device_start_ms = ref.elapsed_time(slot["start"])
                    comp.device_end_ms = ref.elapsed_time(slot["end"])
                done.append(comp)
                if keep_state:
                    self.final_states[req.rid] = sim.download()
                    self.final_pressures[req.rid] = sim.pressure()
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
    kinds = sorted({c.kind for c in completions})
    return {
        "requests": len(completions),
        "accepted": len(ok),
        "rejected": rejected,
        "elapsed_s": elapsed,
        "requests_per_s": len(ok) / elapsed if elapsed > 0 else float("nan"),
        "cell_steps_per_s": cell_steps / elapsed if elapsed > 0 else float("nan"),
        "latency_s": lat,
        "by_kind": {k: {"requests": sum(1 for c in ok if c.kind == k),
                        "latency_s": percentiles([c.latency for c in ok if c.kind == k])} for k in kinds},
        # the first rejected requests, to be rerun alone
        "rejections": [{"rid": c.rid, "edge": c.edge, "kind": c.kind, "steps_done": c.steps, "status": c.status,
                        "iterations": list(c.iterations)} for c in completions if c.status != 0][:10],
    }


def overlapping_pairs(completions: Sequence[Completion]) -> int:
    """Pairs of requests whose device intervals overlap (work of both on the
    GPU at the same time)."""
    iv = sorted((c.device_start_ms, c.device_end_ms) for c in completions
                if c.device_start_ms == c.device_start_ms and c.device_end_ms == c.device_end_ms)
    pairs = 0
    for a in range(len(iv)):
        for b in range(a + 1, len(iv)):
            if iv[b][0] < iv[a][1]:
                pairs += 1
            else:
                break
    return pairs
