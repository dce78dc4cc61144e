"""Continuous-batching brick service over the batched volume codec.

Requests ask to encode a brick (a device float32 volume) or to decode one of
the compressed bricks kept resident on the device.  The server keeps one
batched codec (cc_volume_batch) per (brick edge, operation) with a fixed
number of slots, each on its own CUDA stream, so that work for different
sizes and operations overlaps on the GPU.  Every time a batch is idle the
loop fills it with the oldest waiting requests of its kind - as many as
slots and the HBM admission budget allow - and launches it (replayed as a
CUDA graph per fill level); requests that arrive meanwhile wait for the next
launch of their batch, not for the whole queue to drain.  Latency is
arrival -> result ready (the host sees the batch's completion event).

Results do not depend on the mix: every brick has its own Huffman tables and
its own stream, so a brick decoded alone and in a full batch is bit-identical.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from .codec import Instance, VolumeBatch

ENCODE, DECODE = 0, 1


@dataclass
class Request:
    rid: int
    op: int                    # ENCODE or DECODE
    edge: int
    arrival: float             # seconds after the start of the run
    brick: int = 0             # DECODE: index of the resident brick; ENCODE: index of the source brick
    done: float = -1.0
    result: Optional[object] = None


@dataclass
class _Lane:
    """One batched codec with its slots, stream and in-flight state."""
    edge: int
    op: int
    batch: VolumeBatch
    stream: torch.cuda.Stream
    outs: List[torch.Tensor]
    queue: List[Request] = field(default_factory=list)
    inflight: List[Request] = field(default_factory=list)
    event: Optional[torch.cuda.Event] = None
    bytes_inflight: int = 0


class BrickServer:
    """edges: brick edge lengths served; slots: slots per edge; sources: per
    edge a list of device float32 bricks (encode inputs, and what the resident
    compressed store holds); budget: HBM bytes admitted requests may hold
    (outputs of decodes, inputs of encodes) on top of the resident store."""

    def __init__(self, device: int, sources: Dict[int, List[torch.Tensor]], slots: Dict[int, int], levels: int,
                 q0: float, budget_bytes: int = 4 << 30, graph: bool = True, keep_results: bool = False):
        self.inst = Instance(device, 7, 1 << 12, 128, 14)
        self.levels = levels
        self.q0 = q0
        self.budget = budget_bytes
        self.keep = keep_results
        self.sources = sources
        self.lanes: Dict[Tuple[int, int], _Lane] = {}
        for edge, k in slots.items():
            for op in (ENCODE, DECODE):
                b = VolumeBatch(self.inst, [(edge, edge, edge)] * k, levels, [q0] * k, graph=graph)
                st = torch.cuda.Stream(device=device)
                b.set_stream(st)
                outs = [torch.empty((edge,) * 3, dtype=torch.float32, device=f"cuda:{device}") for _ in range(k)] \
                    if op == DECODE else []
                self.lanes[(edge, op)] = _Lane(edge, op, b, st, outs)
        # resident compressed store: every source brick, compressed once
        self.store: Dict[int, List[Tuple[torch.Tensor, int]]] = {}
        self.store_bytes = 0
        for edge, bricks in sources.items():
            lane = self.lanes[(edge, ENCODE)]
            entries = []
            for i in range(0, len(bricks), len(lane.batch.shapes)):
                chunk = bricks[i:i + len(lane.batch.shapes)]
                lane.batch.set_active(len(chunk))
                lane.batch.compress(chunk)
                for j in range(len(chunk)):
                    words, bits = lane.batch.read_stream(j)
                    t = torch.from_numpy(words.view(np.int32)).to(f"cuda:{device}")
                    entries.append((t, bits))
                    self.store_bytes += t.numel() * 4
            self.store[edge] = entries
        torch.cuda.synchronize()

    def close(self):
        for lane in self.lanes.values():
            lane.batch.close()
        self.inst.close()

    # ------------------------------------------------------------------ loop
    @staticmethod
    def _request_bytes(r: Request) -> int:
        return r.edge ** 3 * 4

    def _launch(self, lane: _Lane, used: int) -> int:
        """Fills an idle lane from its queue within the budget; returns bytes admitted."""
        k = len(lane.batch.shapes)
        take = []
        budget_left = self.budget - self.store_bytes - used
        while lane.queue and len(take) < k and self._request_bytes(lane.queue[0]) <= budget_left:
            r = lane.queue.pop(0)
            budget_left -= self._request_bytes(r)
            take.append(r)
        if not take:
            return 0
        b = lane.batch
        b.set_active(len(take))
        if lane.op == ENCODE:
            b.compress([self.sources[lane.edge][r.brick] for r in take])
        else:
            entries = [self.store[lane.edge][r.brick] for r in take]
            b.load_streams([w for w, _ in entries], [bits for _, bits in entries])
            b.decompress(lane.outs[:len(take)])
        ev = torch.cuda.Event()
        ev.record(lane.stream)
        lane.event = ev
        lane.inflight = take
        lane.bytes_inflight = sum(self._request_bytes(r) for r in take)
        return lane.bytes_inflight

    def _complete(self, lane: _Lane, now: float) -> int:
        freed = lane.bytes_inflight
        for j, r in enumerate(lane.inflight):
            r.done = now
            if self.keep:
                if lane.op == DECODE:
                    with torch.cuda.stream(lane.stream):
                        r.result = lane.outs[j].clone()
                else:
                    r.result = lane.batch.read_stream(j)
        if self.keep:
            lane.stream.synchronize()
        lane.inflight = []
        lane.event = None
        lane.bytes_inflight = 0
        return freed

    def run(self, requests: List[Request]) -> List[Request]:
        """Open-loop run: requests (sorted by arrival) are admitted when their
        arrival time has come; returns them with completion times."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        nxt = 0
        used = 0
        pending = len(reqs)
        t0 = time.perf_counter()
        while pending:
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                r = reqs[nxt]
                self.lanes[(r.edge, r.op)].queue.append(r)
                nxt += 1
            progressed = False
            for lane in self.lanes.values():
                if lane.event is not None and lane.event.query():
                    t = time.perf_counter() - t0
                    pending -= len(lane.inflight)
                    used -= self._complete(lane, t)
                    progressed = True
                if lane.event is None and lane.queue:
                    got = self._launch(lane, used)
                    used += got
                    progressed = progressed or got > 0
            if not progressed and nxt < len(reqs) and all(l.event is None for l in self.lanes.values()) \
                    and not any(l.queue for l in self.lanes.values()):
                # idle until the next arrival
                wait = reqs[nxt].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        return reqs


def poisson_requests(n: int, rate: float, edges, decode_frac: float, bricks_per_edge: int, seed: int) -> List[Request]:
    """Open-loop Poisson arrivals; edge uniform over `edges`; decode with
    probability decode_frac, else encode."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for i in range(n):
        edge = int(rng.choice(edges))
        op = DECODE if rng.random() < decode_frac else ENCODE
        out.append(Request(i, op, edge, float(t[i]), int(rng.integers(0, bricks_per_edge))))
    return out


def latency_stats(reqs: List[Request]) -> dict:
    lat = np.array([r.done - r.arrival for r in reqs]) * 1e3
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    return {"requests": len(reqs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "bricks_per_s": len(reqs) / span if span > 0 else None}
