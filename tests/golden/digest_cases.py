"""The full-size cases pinned by digests of the reference's own output
(tests/golden/ref_digests.json, written by make_golden.py --only digests):
their parameters and their inputs, regenerated from seeds.

* the 128^3 lossy volume (3 levels, q0 = 0.01 std);
* each component of the 3 x 256^3 vector field at q0 in {0.002, 0.01, 0.05}
  std (3 levels; the largest symbol at q0 = 0.002 is 11085, so the default
  2^14-symbol Huffman alphabet holds every band);
* the first bricks of the 4096 uneven bricks (2 levels, per-brick q0);
* the 2048^2 lossless heightfield (4 integer levels).
"""
import hashlib

import numpy as np

from cudacompress_b200 import fields

C2_Q0 = (0.002, 0.01, 0.05)
BRICK_COUNT, BRICK_SEED, BRICK_LEVELS, BRICK_SAMPLE = 4096, 1005, 2, 32
HEIGHTFIELD = dict(name="heightfield-2048", n=2048, seed=fields.SEED_C1, levels=4)


def volume_cases():
    out = [dict(name="volume-128", n=128, modes=512, kmax=32, seed=fields.SEED_C0, levels=3, q0=0.01)]
    for seed in fields.SEED_C2:
        for q0 in C2_Q0:
            out.append(dict(name=f"vector-field-256-seed{seed}-q{q0}", n=256, modes=1024, kmax=64, seed=seed,
                            levels=3, q0=q0))
    return out


def volume_input(case):
    return fields.turbulence_field(case["n"], case["modes"], case["kmax"], case["seed"])


def brick_inputs():
    """The sampled bricks (z, y, x float32 arrays) and their steps."""
    bricks, q = fields.brick_set(BRICK_COUNT, BRICK_SEED)
    return bricks[:BRICK_SAMPLE], [float(v) for v in q[:BRICK_SAMPLE]]


def heightfield_input():
    return fields.fbm_heightfield(HEIGHTFIELD["n"], HEIGHTFIELD["seed"])


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
