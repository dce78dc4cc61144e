"""Stream container files: volume bit streams with the codec, levels, sizes
and steps needed to decode them (cc_container_*; layout documented in
csrc/container.cu).  The reference's example writes the words alone
(examples.cpp:527-536)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from ._ffi import check, lib

FLOAT, QUANT_FIRST, HEIGHTFIELD = 0, 1, 2


class _Info(ctypes.Structure):
    _fields_ = [("codec", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("levels", ctypes.c_uint32),
                ("coding_block_size", ctypes.c_uint32), ("log2_symbol_count", ctypes.c_uint32)]


class _Entry(ctypes.Structure):
    _fields_ = [("size_x", ctypes.c_uint32), ("size_y", ctypes.c_uint32), ("size_z", ctypes.c_uint32),
                ("quant_step", ctypes.c_float), ("bit_size", ctypes.c_uint64), ("words", ctypes.c_void_p)]


@dataclass
class ContainerInfo:
    codec: int = FLOAT
    flags: int = 0
    levels: int = 3
    coding_block_size: int = 128
    log2_symbol_count: int = 14


@dataclass
class Stream:
    shape: Tuple[int, int, int]      # (z, y, x)
    quant_step: float
    bit_size: int
    words: np.ndarray                # uint32


def pack(info: ContainerInfo, streams: Sequence[Stream]) -> bytes:
    """The container's bytes."""
    words = [np.ascontiguousarray(s.words, np.uint32) for s in streams]
    ents = (_Entry * max(len(streams), 1))()
    for i, (s, w) in enumerate(zip(streams, words)):
        if w.size * 32 < s.bit_size:
            raise ValueError(f"stream {i}: {w.size} words hold fewer than {s.bit_size} bits")
        z, y, x = s.shape
        ents[i] = _Entry(x, y, z, s.quant_step, s.bit_size, w.ctypes.data)
    bits = (ctypes.c_uint64 * max(len(streams), 1))(*[s.bit_size for s in streams])
    n = lib().cc_container_bytes(len(streams), bits)
    buf = ctypes.create_string_buffer(n)
    written = ctypes.c_uint64()
    inf = _Info(info.codec, info.flags, info.levels, info.coding_block_size, info.log2_symbol_count)
    check(lib().cc_container_write(buf, n, ctypes.byref(inf), ents, len(streams), ctypes.byref(written)),
          "cc_container_write")
    return buf.raw[: written.value]


def unpack(data: bytes) -> Tuple[ContainerInfo, List[Stream]]:
    buf = ctypes.create_string_buffer(data, len(data))
    inf = _Info()
    count = ctypes.c_uint32()
    check(lib().cc_container_read(buf, len(data), ctypes.byref(inf), None, 0, ctypes.byref(count)), "cc_container_read")
    ents = (_Entry * max(count.value, 1))()
    check(lib().cc_container_read(buf, len(data), ctypes.byref(inf), ents, count.value, ctypes.byref(count)),
          "cc_container_read")
    base = ctypes.addressof(buf)
    out = []
    for i in range(count.value):
        e = ents[i]
        nw = (e.bit_size + 31) // 32
        off = e.words - base
        w = np.frombuffer(data, np.uint32, count=nw, offset=off).copy()
        out.append(Stream((e.size_z, e.size_y, e.size_x), float(e.quant_step), int(e.bit_size), w))
    return ContainerInfo(inf.codec, inf.flags, inf.levels, inf.coding_block_size, inf.log2_symbol_count), out


def save(path: str, info: ContainerInfo, streams: Sequence[Stream]) -> None:
    with open(path, "wb") as f:
        f.write(pack(info, streams))


def load(path: str) -> Tuple[ContainerInfo, List[Stream]]:
    with open(path, "rb") as f:
        return unpack(f.read())
