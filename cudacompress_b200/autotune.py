"""Autotuner of the batched volume codec.

For a given set of brick shapes it times one compress + decompress pass of a
batch for every candidate Huffman coding block size (the reference allows
32..256 symbols per block; a larger block means fewer offsets in the stream
and fewer, longer decode threads) and returns the fastest.  The choice
changes only the entropy-coding blocking, never the quantized data, so the
reconstruction - and the PSNR - is the same for every candidate.
"""
from __future__ import annotations

from typing import Dict, Sequence, Tuple

import torch

from .codec import Instance, VolumeBatch


def tune_coding_block(device: int, volumes: Sequence[torch.Tensor], levels: int, steps: Sequence[float],
                      candidates=(64, 128, 256), passes: int = 2) -> Tuple[int, Dict[int, float]]:
    """Returns (best coding block size, {candidate: ms per pass})."""
    times: Dict[int, float] = {}
    shapes = [tuple(v.shape) for v in volumes]
    outs = [torch.empty_like(v) for v in volumes]
    for cb in candidates:
        inst = Instance(device, 7, 1 << 12, cb, 14)
        with VolumeBatch(inst, shapes, levels, steps, graph=True) as b:
            b.compress(volumes)
            b.decompress(outs)
            b.status()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            for _ in range(passes):
                b.compress(volumes)
                b.decompress(outs)
            e.record()
            torch.cuda.synchronize()
            b.status()
            times[cb] = s.elapsed_time(e) / passes
        inst.close()
    best = min(times, key=times.get)
    return best, times
