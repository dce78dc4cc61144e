"""A small, self-contained case of the batched codec for profilers: one batch
of `--comps` seeded n^3 float32 fields (the vector-field workload's
generator), one warm-up encode + decode, then `--steps` more.  Launch order
per step: the forward transform (per level: k_bRows, k_bCols Y, k_bCols Z
with the quantizer fused), the encoders, then the decoder and the inverse
transform (per level: k_bCols Z from symbols, k_bCols Y, k_bRows).

    python -m cudacompress_b200.profile_case --n 256 --comps 3 --steps 1
"""
from __future__ import annotations

import argparse

import torch

from . import codec as cc
from . import fields


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--comps", type=int, default=3)
    ap.add_argument("--levels", type=int, default=3)
    ap.add_argument("--q0", type=float, default=0.01)
    ap.add_argument("--steps", type=int, default=1)
    args = ap.parse_args()
    n = args.n
    vols = [torch.from_numpy(fields.turbulence_field(n, 1024, min(64, n // 4), seed=1002 + c)).cuda()
            for c in range(args.comps)]
    outs = [torch.empty_like(v) for v in vols]
    with cc.Instance(0, 7, (n // 2) ** 3, 128, 14) as inst:
        with cc.VolumeBatch(inst, [v.shape for v in vols], args.levels, [args.q0] * args.comps) as batch:
            for _ in range(1 + args.steps):
                batch.compress(vols)
                batch.decompress(outs)
            torch.cuda.synchronize()
            batch.status()
    print("profile case done:", n, args.comps)


if __name__ == "__main__":
    main()
