"""Baseline infrastructure (not shipped): times the reference's own GPU codec
(examples/CompressVolume.cpp over src/cudaCompress, compiled unmodified for
sm_100a by oracle/ref/Makefile into oracle/_ref/libref_gpu.so) on the
vector-field workload's components, beside this library's plain
per-component path driven the same way: device field -> host bit stream
(compressVolumeFloat) and host bit stream -> device field
(decompressVolumeFloat), every call synchronous.  Prints one JSON line.

Run from the repository root on a GPU host, after `make -C oracle/ref`:
    python oracle/ref/time_ref_gpu.py [--reps 5] [--comps 3]
"""
import argparse
import ctypes as c
import json
import os
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import cudacompress_b200 as cc  # noqa: E402
from cudacompress_b200 import fields  # noqa: E402

# the vector-field workload: 256^3 components, 3 levels, q0 = 0.01 std
N, LEVELS, Q0, MODES, KMAX, SEEDS = 256, 3, 0.01, 1024, 64, (1002, 1003, 1004)


def time_reference(lib, d, out, reps):
    u32p = c.POINTER(c.c_uint32)
    lib.ref_volume_time.argtypes = [c.c_void_p, c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32,
                                    c.c_float, c.c_uint32, c.POINTER(c.c_double), c.POINTER(c.c_double), u32p]
    enc, dec, nw = c.c_double(), c.c_double(), c.c_uint32()
    r = lib.ref_volume_time(c.c_void_p(d.data_ptr()), c.c_void_p(out.data_ptr()), N, N, N, LEVELS, Q0, reps,
                            c.byref(enc), c.byref(dec), c.byref(nw))
    if r != 0:
        raise RuntimeError(f"ref_volume_time failed: {r}")
    return enc.value, dec.value, nw.value


def time_ours(inst, d, out, reps):
    cap = cc.volume_stream_capacity_words(N, N, N)
    dw = torch.empty(cap, dtype=torch.int32, device="cuda")
    hw = torch.empty(cap, dtype=torch.int32).pin_memory()
    enc = dec = 0.0
    warm = 3   # the instance makes its volume batch on the fifth consecutive call of a shape
    for r in range(reps + warm):
        t0 = time.perf_counter()
        _, bits = cc.compress_volume_float(inst, d, LEVELS, Q0, dw)
        nw = (bits + 31) // 32
        hw[:nw].copy_(dw[:nw])                      # the stream to host memory, as the reference returns it
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        dw[:nw].copy_(hw[:nw])                      # and back (synchronous copy)
        cc.decompress_volume_float(inst, out, LEVELS, Q0, dw, bits)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if r >= warm:
            enc += (t1 - t0) * 1e3
            dec += (t2 - t1) * 1e3
    return enc / reps, dec / reps, nw


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--comps", type=int, default=3)
    args = ap.parse_args()
    lib = c.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so"))
    inst = cc.Instance(0, 7, (N // 2) ** 3, 128, 14)
    rows = []
    for seed in SEEDS[: args.comps]:
        v = fields.turbulence_field(N, MODES, KMAX, seed)
        d = torch.from_numpy(v).cuda()
        out_ref = torch.empty_like(d)
        out_ours = torch.empty_like(d)
        re, rd, rw = time_reference(lib, d, out_ref, args.reps)
        oe, od, ow = time_ours(inst, d, out_ours, args.reps)
        same = rw == ow and torch.equal(out_ref, out_ours)
        rows.append({"seed": seed, "ref_encode_ms": re, "ref_decode_ms": rd, "ours_plain_encode_ms": oe,
                     "ours_plain_decode_ms": od, "words": rw, "same_stream_size_and_reconstruction": bool(same)})
    raw = N ** 3 * 4
    tot = lambda k: sum(r[k] for r in rows)  # noqa: E731
    out = {"workload": f"{len(rows)} x {N}^3 f32, {LEVELS} levels, q0 = {Q0} std",
           "ref_gpu": {"encode_gbs": raw * len(rows) / tot("ref_encode_ms") / 1e6,
                       "decode_gbs": raw * len(rows) / tot("ref_decode_ms") / 1e6,
                       "ms_per_step": tot("ref_encode_ms") + tot("ref_decode_ms")},
           "ours_plain": {"encode_gbs": raw * len(rows) / tot("ours_plain_encode_ms") / 1e6,
                          "decode_gbs": raw * len(rows) / tot("ours_plain_decode_ms") / 1e6,
                          "ms_per_step": tot("ours_plain_encode_ms") + tot("ours_plain_decode_ms")},
           "components": rows, "reps": args.reps,
           "note": "wall time per synchronous call, device field in, host stream between, device field out"}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
