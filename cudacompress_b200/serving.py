"""Continuous-batching brick service over the batched volume codec.

Requests ask to encode a brick (a device float32 volume) or to decode one of
the compressed bricks kept resident on the device.  The server keeps, per
(brick edge, operation), a lane of two batched codecs (cc_volume_batch) with
a fixed number of slots each, every codec on its own CUDA stream.  While one
codec of a lane is on the GPU the other admits the requests that arrived
meanwhile - as many as its slots and the HBM admission budget allow - and
launches at once (replayed as a CUDA graph per fill level), so a request waits
for a free slot group, not for the lane's running batch to drain.  Decode
lanes run on high-priority streams and are filled first, so small decodes are
not held behind large encodes.  Latency is arrival -> result ready (the host
sees the batch's completion event).

Admission: a request holds its output (decode) or input (encode) volume,
edge^3 * 4 bytes, from launch to completion; the resident compressed store
plus everything admitted stays within `budget_bytes`.  A budget that cannot
hold the store plus one request of the largest edge is rejected at
construction, so every request fits once the GPU drains and the loop always
makes progress.

Fill levels: a launch takes a power of two of the admitted requests (or all
of a codec's slots), so a codec replays one of log2(slots) + 1 graphs; they
are all captured when the server is built, so no graph capture (tens of
milliseconds of host time) ever falls inside a run.  The requests a launch
leaves stay at the head of the queue for the lane's other codec.

Results do not depend on the mix: every brick has its own Huffman tables and
its own stream, so a brick decoded alone and in a full batch is bit-identical.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional, Sequence, Tuple

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
    launched: float = -1.0     # when its batch was launched (seconds after the start of the run)


@dataclass
class _Group:
    """One batched codec of a lane: its slots, stream and in-flight state."""
    batch: VolumeBatch
    stream: torch.cuda.Stream
    outs: List[torch.Tensor]
    inflight: List[Request] = field(default_factory=list)
    event: Optional[torch.cuda.Event] = None
    bytes_inflight: int = 0


@dataclass
class _Lane:
    edge: int
    op: int
    groups: List[_Group]
    queue: Deque[Request] = field(default_factory=deque)


def request_bytes(edge: int) -> int:
    """Device bytes a request of this edge holds while admitted."""
    return edge ** 3 * 4


def validate_budget(store_bytes: int, edges: Sequence[int], budget_bytes: int) -> None:
    """Raises ValueError unless the budget holds the resident store plus one
    request of the largest edge (otherwise such a request could never run)."""
    need = store_bytes + request_bytes(max(edges))
    if need > budget_bytes:
        raise ValueError(f"HBM admission budget {budget_bytes} B cannot hold the resident store ({store_bytes} B) "
                         f"plus one {max(edges)}^3 request ({request_bytes(max(edges))} B)")


def admit(queue_bytes: Sequence[int], slots: int, budget_left: int) -> int:
    """How many requests from the head of a queue (their bytes, in arrival
    order) one launch takes: at most `slots`, in order, while they fit."""
    take = 0
    for b in queue_bytes:
        if take == slots or b > budget_left:
            break
        budget_left -= b
        take += 1
    return take


def fill_levels(slots: int) -> List[int]:
    """The active counts a codec of `slots` slots launches with: powers of
    two below `slots`, and `slots`."""
    out, k = [], 1
    while k < slots:
        out.append(k)
        k *= 2
    out.append(slots)
    return out


def fill_level(n: int, slots: int) -> int:
    """The largest fill level not above n (0 for n == 0)."""
    best = 0
    for k in fill_levels(slots):
        if k <= n:
            best = k
    return best


class BrickServer:
    """sources: per edge a list of device float32 bricks (encode inputs, and
    what the resident compressed store holds); slots: slots per codec of each
    edge's lanes; groups: codecs per lane; budget_bytes: HBM bytes the store
    plus admitted requests may hold."""

    def __init__(self, device: int, sources: Dict[int, List[torch.Tensor]], slots: Dict[int, int], levels: int,
                 q0: float, budget_bytes: int = 4 << 30, graph: bool = True, keep_results: bool = False,
                 groups: int = 2):
        self.inst = Instance(device, 7, 1 << 12, 128, 14)
        self.levels = levels
        self.q0 = q0
        self.budget = budget_bytes
        self.keep = keep_results
        self.sources = sources
        self.lanes: Dict[Tuple[int, int], _Lane] = {}
        for edge, k in slots.items():
            for op in (ENCODE, DECODE):
                gs = []
                for _ in range(groups):
                    b = VolumeBatch(self.inst, [(edge, edge, edge)] * k, levels, [q0] * k, graph=graph)
                    st = torch.cuda.Stream(device=device, priority=-1 if op == DECODE else 0)
                    b.set_stream(st)
                    outs = [torch.empty((edge,) * 3, dtype=torch.float32, device=f"cuda:{device}")
                            for _ in range(k)] if op == DECODE else []
                    gs.append(_Group(b, st, outs))
                self.lanes[(edge, op)] = _Lane(edge, op, gs)
        # filling order: decodes before encodes, small edges first
        self.order = sorted(self.lanes.values(), key=lambda ln: (ln.op != DECODE, ln.edge))
        # resident compressed store: every source brick, compressed once
        self.store: Dict[int, List[Tuple[torch.Tensor, int]]] = {}
        self.store_bytes = 0
        for edge, bricks in sources.items():
            g = self.lanes[(edge, ENCODE)].groups[0]
            k = len(g.batch.shapes)
            entries = []
            for i in range(0, len(bricks), k):
                chunk = bricks[i:i + k]
                g.batch.set_active(len(chunk))
                g.batch.compress(chunk)
                for j in range(len(chunk)):
                    words, bits = g.batch.read_stream(j)
                    t = torch.from_numpy(words.view(np.int32)).to(f"cuda:{device}")
                    entries.append((t, bits))
                    self.store_bytes += t.numel() * 4
            self.store[edge] = entries
        torch.cuda.synchronize()
        validate_budget(self.store_bytes, list(slots), budget_bytes)
        self.peak_admitted = 0
        if graph:
            self._capture_fill_levels()

    def _capture_fill_levels(self) -> None:
        """Runs every codec once at every fill level (capturing its graph)."""
        for lane in self.lanes.values():
            srcs = self.sources[lane.edge]
            entries = self.store[lane.edge]
            for g in lane.groups:
                for k in fill_levels(len(g.batch.shapes)):
                    g.batch.set_active(k)
                    if lane.op == ENCODE:
                        g.batch.compress([srcs[i % len(srcs)] for i in range(k)])
                    else:
                        pick = [entries[i % len(entries)] for i in range(k)]
                        g.batch.load_streams([w for w, _ in pick], [bits for _, bits in pick])
                        g.batch.decompress(g.outs[:k])
        torch.cuda.synchronize()

    def close(self):
        for lane in self.lanes.values():
            for g in lane.groups:
                g.batch.close()
        self.inst.close()

    # ------------------------------------------------------------------ loop
    def _launch(self, lane: _Lane, g: _Group, used: int, now: float) -> int:
        """Fills an idle codec from its lane's queue within the budget;
        returns the bytes admitted."""
        k = len(g.batch.shapes)
        n = admit([request_bytes(r.edge) for r in list(lane.queue)[:k]], k, self.budget - self.store_bytes - used)
        n = fill_level(n, k)
        if n == 0:
            return 0
        take = [lane.queue.popleft() for _ in range(n)]
        b = g.batch
        b.set_active(n)
        if lane.op == ENCODE:
            b.compress([self.sources[lane.edge][r.brick] for r in take])
        else:
            entries = [self.store[lane.edge][r.brick] for r in take]
            b.load_streams([w for w, _ in entries], [bits for _, bits in entries])
            b.decompress(g.outs[:n])
        ev = torch.cuda.Event()
        ev.record(g.stream)
        g.event = ev
        g.inflight = take
        for r in take:
            r.launched = now
        g.bytes_inflight = sum(request_bytes(r.edge) for r in take)
        return g.bytes_inflight

    def _complete(self, lane: _Lane, g: _Group, now: float) -> int:
        freed = g.bytes_inflight
        for j, r in enumerate(g.inflight):
            r.done = now
            if self.keep:
                if lane.op == DECODE:
                    with torch.cuda.stream(g.stream):
                        r.result = g.outs[j].clone()
                else:
                    r.result = g.batch.read_stream(j)
        if self.keep:
            g.stream.synchronize()
        g.inflight = []
        g.event = None
        g.bytes_inflight = 0
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
            for lane in self.order:
                for g in lane.groups:
                    if g.event is not None and g.event.query():
                        pending -= len(g.inflight)
                        used -= self._complete(lane, g, time.perf_counter() - t0)
                        progressed = True
            busy = False
            for lane in self.order:
                for g in lane.groups:
                    if g.event is None and lane.queue:
                        got = self._launch(lane, g, used, time.perf_counter() - t0)
                        used += got
                        progressed = progressed or got > 0
                    busy = busy or g.event is not None
            self.peak_admitted = max(self.peak_admitted, used)
            queued = any(lane.queue for lane in self.order)
            if queued and not busy:
                # nothing on the GPU and still nothing admitted: cannot happen
                # with a validated budget; fail instead of spinning
                raise RuntimeError("a queued request does not fit the HBM budget on an idle GPU")
            if not progressed and not busy and not queued and nxt < len(reqs):
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
