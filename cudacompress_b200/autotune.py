"""Autotuner of the batched volume codec.

For a given set of brick shapes it times one compress + decompress pass of a
batch for every candidate pair of

* Huffman coding block size (the reference allows 32..256 symbols per block;
  a larger block means fewer offsets in the stream and fewer, longer decode
  lanes), and
* forward-transform tile depth (z_chunk: output slices per CTA of a level's
  fused pass; deeper tiles re-read fewer halo slices, shallower ones give
  small bricks more CTAs),

and returns the fastest.  Neither changes the quantized data: the coding
block changes only the entropy blocking and the tile depth not a single
coefficient, so the reconstruction - and the PSNR - is the same for every
candidate.
"""
from __future__ import annotations

from typing import Dict, Sequence, Tuple

import torch

from .codec import Instance, VolumeBatch


def _time_pass(device: int, volumes, shapes, levels: int, steps, cb: int, z_chunk: int, passes: int) -> float:
    outs = [torch.empty_like(v) for v in volumes]
    inst = Instance(device, 7, 1 << 12, cb, 14)
    try:
        with VolumeBatch(inst, shapes, levels, steps, graph=True, z_chunk=z_chunk) as b:
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
            return s.elapsed_time(e) / passes
    finally:
        inst.close()


def tune(device: int, volumes: Sequence[torch.Tensor], levels: int, steps: Sequence[float],
         coding_blocks=(64, 128, 256), z_chunks=(16, 32, 64), passes: int = 2) -> Tuple[int, int, Dict[str, float]]:
    """Returns (coding block, z_chunk, {"cb/z_chunk": ms per pass})."""
    shapes = [tuple(v.shape) for v in volumes]
    times: Dict[str, float] = {}
    best = None
    for cb in coding_blocks:
        for zc in z_chunks:
            t = _time_pass(device, volumes, shapes, levels, steps, cb, zc, passes)
            times[f"{cb}/{zc}"] = t
            if best is None or t < best[0]:
                best = (t, cb, zc)
    return best[1], best[2], times


def tune_coding_block(device: int, volumes: Sequence[torch.Tensor], levels: int, steps: Sequence[float],
                      candidates=(64, 128, 256), passes: int = 2) -> Tuple[int, Dict[int, float]]:
    """The coding block alone (default tile depth): (best, {candidate: ms per pass})."""
    shapes = [tuple(v.shape) for v in volumes]
    times = {cb: _time_pass(device, volumes, shapes, levels, steps, cb, 0, passes) for cb in candidates}
    return min(times, key=times.get), times
