"""FP64 error of the FP32 float DWT and of the lossy volume codec.

The float DWT computes in FP32 with the reference's tap order and FMA chain
(util/DWTFloatKernels.cui:68-79; taps util/DWTFloatFilters.cuh:42-49), which is
what makes its output bit-identical to the reference's.  This module states
the cost of FP32 against the same transform in FP64: the same taps (the
reference's float constants, promoted to double), the same whole-sample
symmetric extension (util/DWTCommon.cuh:54-55) and [L|H] layout per axis,
accumulated in double - computed with torch float64 on the volume's device.

error_report() gives, for an L-level forward transform, the max-abs and RMS
difference of the library's FP32 coefficients from the FP64 ones, and per
quantization step q0: the codec's FP32 reconstruction against the FP64
inverse of the very symbols it coded (dequantized in FP64), with the PSNR of
both against the original field.
"""
from __future__ import annotations

import numpy as np
import torch

from . import codec

# CDF 9/7 analysis (even / odd output) and synthesis taps as float32 constants
# (util/DWTFloatFilters.cuh:42-49); the centre tap is index 4.
TAPS_FORWARD = np.array([
    [0.0267488, -0.0168641, -0.0782233, 0.2668641, 0.6029490, 0.2668641, -0.0782233, -0.0168641, 0.0267488],
    [0.0, 0.0456359, -0.0287718, -0.2956359, 0.5575435, -0.2956359, -0.0287718, 0.0456359, 0.0]], np.float32)
TAPS_INVERSE = np.array([
    [0.0, 0.0337282, -0.0575435, -0.5337281, 1.1150871, -0.5337281, -0.0575435, 0.0337282, 0.0],
    [0.0534975, -0.0912718, -0.1564465, 0.5912718, 1.2058980, 0.5912718, -0.1564465, -0.0912718, 0.0534975]],
    np.float32)


def _fir_axis(a: torch.Tensor, dim: int, inverse: bool) -> torch.Tensor:
    """One 9-tap pass along `dim` of a float64 tensor: forward writes the even
    outputs to the first half and the odd ones to the second; inverse reads
    the halves as the interleaved signal and writes it in order."""
    n = a.shape[dim]
    h = n // 2
    dev = a.device
    x = a.movedim(dim, -1)
    if inverse:
        inter = torch.empty(n, dtype=torch.long, device=dev)
        inter[0::2] = torch.arange(h, device=dev)
        inter[1::2] = h + torch.arange(h, device=dev)
        x = x[..., inter]
    pos = torch.arange(n, device=dev)
    idx = (pos[:, None] + torch.arange(-4, 5, device=dev)[None, :]).abs()
    idx = torch.where(idx > n - 1, 2 * (n - 1) - idx, idx)                  # whole-sample mirror
    taps = torch.from_numpy((TAPS_INVERSE if inverse else TAPS_FORWARD).astype(np.float64)).to(dev)[pos & 1]
    out = torch.zeros_like(x)
    for i in range(9):                                                      # one tap at a time: bounded memory
        out += x[..., idx[:, i]] * taps[:, i]
    if not inverse:
        out = torch.cat([out[..., 0::2], out[..., 1::2]], dim=-1)
    return out.movedim(-1, dim).contiguous()


def dwt_fp64(a: torch.Tensor, inverse: bool = False) -> torch.Tensor:
    """One level of the 3D (z, y, x) or 2D (y, x) transform in float64:
    forward X, Y, Z; inverse Z, Y, X (util/DWTFloat.cu:84-202, 204-323)."""
    dims = [a.dim() - 1 - k for k in range(a.dim())]                        # x, y[, z]
    if inverse:
        dims = dims[::-1]
    for d in dims:
        a = _fir_axis(a, d, inverse)
    return a


def multilevel_fp64(vol: torch.Tensor, levels: int, inverse: bool = False) -> torch.Tensor:
    """L levels in the codec's layout: level l transforms the low octant of
    extent n / 2^l (CompressVolume.cpp:341-347)."""
    out = vol.to(torch.float64).clone()
    order = range(levels - 1, -1, -1) if inverse else range(levels)
    for lvl in order:
        sl = tuple(slice(0, s >> lvl) for s in out.shape)
        out[sl] = dwt_fp64(out[sl].contiguous(), inverse)
    return out


def multilevel_fp32(vol: torch.Tensor, levels: int) -> torch.Tensor:
    """The library's FP32 forward transform (cc_dwt_float_forward), L levels
    in the same layout."""
    nz, ny, nx = vol.shape
    out = vol.clone()
    t1 = torch.empty_like(vol)
    t2 = torch.empty_like(vol)
    for lvl in range(levels):
        sz, sy, sx = nz >> lvl, ny >> lvl, nx >> lvl
        sub = out[:sz, :sy, :sx].contiguous()
        res = torch.empty_like(sub)
        codec.dwt_float_forward(res, t2, t1, sub, sx, sy, sz)
        out[:sz, :sy, :sx] = res
    return out


def _symbols_fp64(coef32: torch.Tensor, levels: int, q0: float) -> torch.Tensor:
    """The codec's symbols of every band (the library's quantizer, level l's
    step q0 / 2^l, the lowpass at the coarsest step; CompressVolume.cpp:353-366),
    dequantized in float64 as (q + sign(q) / 2) * step (util/Quantize.cuh:75-147)."""
    nz, ny, nx = coef32.shape
    out = torch.zeros(coef32.shape, dtype=torch.float64, device=coef32.device)
    for lvl in range(levels):
        step = np.float32(q0) / np.float32(1 << lvl)
        hz, hy, hx = nz >> (lvl + 1), ny >> (lvl + 1), nx >> (lvl + 1)
        blocks = range(0 if lvl == levels - 1 else 1, 8)
        for b in blocks:
            x0, y0, z0 = (b & 1) * hx, ((b >> 1) & 1) * hy, (b >> 2) * hz
            band = coef32[z0:z0 + hz, y0:y0 + hy, x0:x0 + hx]
            sym = torch.empty((hz, hy, hx), dtype=torch.int16, device=coef32.device)
            codec.quantize_to_symbols(sym, band, hx, hy, hz, float(step), nx, nx * ny)
            s = sym.to(torch.int32) & 0xFFFF
            q = torch.where(s & 1 == 1, -((s + 1) >> 1), s >> 1).to(torch.float64)
            out[z0:z0 + hz, y0:y0 + hy, x0:x0 + hx] = (q + torch.sign(q) * 0.5) * float(step)
    return out


def psnr(orig: torch.Tensor, rec: torch.Tensor) -> float:
    """20 log10((max - min) / RMSE) in float64 (tools/imgtools.h:32-44, 114-143)."""
    o = orig.to(torch.float64)
    rmse = float(torch.sqrt(torch.mean((o - rec.to(torch.float64)) ** 2)))
    return float("inf") if rmse == 0.0 else 20.0 * np.log10(float(o.max() - o.min()) / rmse)


def _err(a: torch.Tensor, b: torch.Tensor) -> dict:
    d = a.to(torch.float64) - b.to(torch.float64)
    return {"max_abs": float(d.abs().max()), "rms": float(torch.sqrt(torch.mean(d * d)))}


def error_report(inst: codec.Instance, vol: torch.Tensor, levels: int, q0s) -> dict:
    """FP32-vs-FP64 error of the transform and of the codec on one (z, y, x)
    float32 CUDA volume (see the module docstring)."""
    coef32 = multilevel_fp32(vol, levels)
    coef64 = multilevel_fp64(vol, levels)
    rep = {"coefficients": dict(_err(coef32, coef64), max_abs_coefficient=float(coef64.abs().max()))}
    nz, ny, nx = vol.shape
    per_q0 = {}
    cap = codec.volume_stream_capacity_words(nx, ny, nz, inst.log2_huffman_distinct_symbol_count_max)
    words = torch.empty(cap, dtype=torch.int32, device=vol.device)
    rec32 = torch.empty_like(vol)
    for q0 in q0s:
        _, bits = codec.compress_volume_float(inst, vol, levels, q0, words)
        codec.decompress_volume_float(inst, rec32, levels, q0, words, bits)
        rec64 = multilevel_fp64(_symbols_fp64(coef32, levels, q0), levels, inverse=True)
        per_q0[str(q0)] = dict(_err(rec32, rec64), psnr_fp32=psnr(vol, rec32), psnr_fp64=psnr(vol, rec64),
                               bits_per_voxel=bits / vol.numel())
    rep["reconstruction"] = per_q0
    return rep
