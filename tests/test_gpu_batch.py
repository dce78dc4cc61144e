"""Batched volume codec (cc_volume_batch_*): uneven bricks in one batch, each
stream byte-identical to the CPU oracle's (and so to the plain codec's), each
reconstruction bit-identical to the oracle's; the same with the whole
sequence replayed as a CUDA graph, on repeated calls and with new inputs."""
import numpy as np
import pytest

from helpers import Oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402
from cudacompress_b200 import fields  # noqa: E402


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def bricks(count, levels, seed):
    rng = np.random.default_rng(seed)
    src = fields.turbulence_field(64, 128, 16, seed=seed)
    f = 1 << levels
    edges = [e for e in (16, 24, 32, 48, 64) if e % f == 0 and (e >> (levels - 1)) >= 8]
    out, steps = [], []
    for _ in range(count):
        nz, ny, nx = (int(rng.choice(edges)) for _ in range(3))
        z0, y0, x0 = (int(rng.integers(0, 64 - n + 1)) for n in (nz, ny, nx))
        out.append(np.ascontiguousarray(src[z0:z0 + nz, y0:y0 + ny, x0:x0 + nx]))
        steps.append(float(np.exp(rng.uniform(np.log(0.002), np.log(0.05)))) * float(src.std()))
    return out, steps


def shifted(shape, shift):
    """A contiguous device float32 volume whose data starts `shift` elements
    into its allocation (shift 1: 4-byte but not 16-byte aligned)."""
    n = int(np.prod(shape))
    return torch.empty(n + shift, dtype=torch.float32, device="cuda")[shift:].view(shape)


def check_batch(oracle, vols, steps, levels, graph, rounds=2, shift=0):
    inst = cc.Instance(0, 7, 1 << 12, 128, 14)
    with cc.VolumeBatch(inst, [v.shape for v in vols], levels, steps, graph=graph) as b:
        ref = [oracle.compress_volume(v, levels, q) for v, q in zip(vols, steps)]
        recs = [oracle.decompress_volume(w, bits, v.shape, levels, q) for (w, bits), v, q in zip(ref, vols, steps)]
        dev = [shifted(v.shape, shift) for v in vols]
        for d, v in zip(dev, vols):
            d.copy_(torch.from_numpy(v))
        outs = [shifted(v.shape, shift).fill_(float("nan")) for v in vols]
        for r in range(rounds):
            b.compress(dev)
            b.decompress(outs)
            b.status()
            for i, v in enumerate(vols):
                words, bits = b.read_stream(i)
                assert bits == ref[i][1], (r, i, bits, ref[i][1])
                assert np.array_equal(words, ref[i][0]), (r, i)
                got = outs[i].cpu().numpy()
                assert np.array_equal(got.view(np.uint32), recs[i].view(np.uint32)), (r, i)
            for o in outs:
                o.fill_(float("nan"))
    inst.close()


def test_batch_uneven_bricks_match_oracle(oracle):
    vols, steps = bricks(12, 2, seed=1005)
    check_batch(oracle, vols, steps, 2, graph=False)


def test_batch_of_many_tables_matches_oracle(oracle):
    """600 bricks: 8400 highpass streams, 16800 encode tables and 17400
    decode tables, so the encode's histogram plan and the decode's symbol
    plan run as several chunk CTAs plus a carry pass over the chunks' sums."""
    vols, steps = bricks(600, 2, seed=1007)
    check_batch(oracle, vols, steps, 2, graph=True, rounds=1)


def test_batch_graph_replay_matches_oracle(oracle):
    vols, steps = bricks(9, 2, seed=1006)
    check_batch(oracle, vols, steps, 2, graph=True, rounds=3)


def test_batch_three_levels_and_new_inputs(oracle):
    vols, steps = bricks(4, 3, seed=77)
    check_batch(oracle, vols, steps, 3, graph=True)
    # same shapes, other data through the same (graph) batch
    vols2 = [np.ascontiguousarray(v[::-1]) for v in vols]
    check_batch(oracle, vols2, steps, 3, graph=True)


def test_batch_unaligned_volume_pointers(oracle):
    """Inputs and outputs 4 bytes past a 16-byte boundary take the scalar
    row path; results are unchanged."""
    vols, steps = bricks(6, 2, seed=4242)
    check_batch(oracle, vols, steps, 2, graph=True, shift=1)
    check_batch(oracle, vols, steps, 2, graph=False, shift=3)


def test_batch_wide_rows(oracle):
    """Rows wider than one row tile (2048): a full and a partial tile per
    row, with the vector path (x % 8 == 0) and the scalar one."""
    rng = np.random.default_rng(99)
    vols = []
    for nx in (2200, 2058):
        v = np.cumsum(rng.standard_normal((8, 8, nx)).astype(np.float32), axis=2) * np.float32(0.05)
        vols.append(np.ascontiguousarray(v.astype(np.float32)))
    steps = [0.02 * float(v.std()) for v in vols]
    check_batch(oracle, vols, steps, 1, graph=False)


def test_batch_rejects_bad_sizes():
    inst = cc.Instance(0, 7, 1 << 12, 128, 14)
    with pytest.raises(cc.CudaCompressError):
        cc.VolumeBatch(inst, [(16, 16, 18)], 2, [0.1])
    inst.close()


def test_batch_decodes_streams_of_the_plain_codec(oracle):
    """Streams written by cc_compress_volume_float, loaded into a batch and
    decoded there, give the oracle's reconstruction."""
    vols, steps = bricks(5, 2, seed=31)
    inst = cc.Instance(0, 7, 32 ** 3, 128, 14)
    words, bits = [], []
    for v, q in zip(vols, steps):
        w, b = cc.compress_volume_float(inst, torch.from_numpy(v).cuda(), 2, q)
        words.append(w[: (b + 31) // 32].cpu().numpy().view(np.uint32).copy())
        bits.append(b)
    with cc.VolumeBatch(inst, [v.shape for v in vols], 2, steps) as bt:
        bt.load_streams(words, bits)
        outs = [torch.empty(v.shape, dtype=torch.float32, device="cuda") for v in vols]
        bt.decompress(outs)
        bt.status()
        for i, (v, q) in enumerate(zip(vols, steps)):
            ref = oracle.decompress_volume(words[i], bits[i], v.shape, 2, q)
            assert np.array_equal(outs[i].cpu().numpy().view(np.uint32), ref.view(np.uint32)), i
    inst.close()


def test_batch_stream_download_upload(oracle):
    """Streams through page-locked host memory without a host wait: the
    download holds each volume's words at its offset (byte-identical to the
    oracle's stream), the upload restores them for a decode, and an
    undersized host buffer is reported."""
    vols, steps = bricks(9, 2, 77)
    inst = cc.Instance(0, 7, 1 << 12, 128, 14)
    s = torch.cuda.Stream()
    with cc.VolumeBatch(inst, [v.shape for v in vols], 2, steps, graph=True) as b:
        b.set_stream(s)
        dv = [torch.from_numpy(v).cuda() for v in vols]
        torch.cuda.synchronize()
        cap = sum(cc.volume_stream_capacity_words(*v.shape[::-1]) for v in vols)
        hw = torch.zeros(cap, dtype=torch.int32).pin_memory()
        he = torch.zeros(2 * len(vols), dtype=torch.int64).pin_memory()
        b.compress(dv)
        b.download_streams(hw, he)
        s.synchronize()
        b.status()
        ext = he.numpy()
        words = hw.numpy().view(np.uint32)
        for i, (v, q) in enumerate(zip(vols, steps)):
            w, bits = oracle.compress_volume(v, 2, q)
            off, nb = int(ext[i]), int(ext[len(vols) + i])
            assert nb == bits
            assert np.array_equal(words[off: off + (nb + 31) // 32], w), i
        # scramble the device streams, then restore them from the host copy
        b.compress([torch.zeros_like(v) for v in dv])
        b.upload_streams(hw, he)
        outs = [torch.full_like(v, float("nan")) for v in dv]
        b.decompress(outs)
        s.synchronize()
        b.status()
        for o, v, q in zip(outs, vols, steps):
            w, bits = oracle.compress_volume(v, 2, q)
            assert np.array_equal(o.cpu().numpy(), oracle.decompress_volume(w, bits, v.shape, 2, q))
        small = torch.zeros(16, dtype=torch.int32).pin_memory()
        b.compress(dv)
        b.download_streams(small, he)
        s.synchronize()
        with pytest.raises(cc.CudaCompressError):
            b.status()
        with pytest.raises(cc.CudaCompressError):       # pageable host memory is refused
            b.download_streams(torch.zeros(cap, dtype=torch.int32), he)
    inst.close()


def test_batch_back_to_back_encodes_are_deterministic():
    """Many encodes enqueued back to back (no host wait; the lowpass tables
    build beside the highpass encode and the previous call's tail) give the
    same bytes every time.  Guards the table builder's block-cooperative sort,
    whose round counter once could be reset before a slower warp read it."""
    bricks_, q = fields.brick_set(512, 1005)
    dv = [torch.from_numpy(b).cuda() for b in bricks_]
    inst = cc.Instance(0, 7, 32 ** 3, 128, 14)
    with cc.VolumeBatch(inst, [b.shape for b in bricks_], 2, [float(v) for v in q], graph=True) as b:
        cap = sum(cc.volume_stream_capacity_words(*v.shape[::-1]) for v in bricks_)
        n = 20
        hw = [torch.zeros(cap, dtype=torch.int32).pin_memory() for _ in range(n)]
        he = [torch.zeros(2 * len(bricks_), dtype=torch.int64).pin_memory() for _ in range(n)]
        for i in range(n):
            b.compress(dv)
            b.download_streams(hw[i], he[i])
        torch.cuda.synchronize()
        b.status()
        ext = he[0].numpy()
        total = int(ext[len(bricks_) - 1] + (ext[-1] + 31) // 32)
        for i in range(1, n):
            assert np.array_equal(he[i].numpy(), ext), i
            assert np.array_equal(hw[i].numpy()[:total], hw[0].numpy()[:total]), i
    inst.close()


@pytest.mark.parametrize("z_chunk", [8, 16, 64, 256])
def test_tile_depth_does_not_change_the_streams(oracle, z_chunk):
    """The forward transform's tile depth (an autotuner knob) changes no
    coefficient: streams and reconstructions equal the oracle's for every
    depth, including depths larger than the volumes."""
    vols, steps = bricks(6, 2, seed=77)
    dev = [torch.from_numpy(v).cuda() for v in vols]
    outs = [torch.full_like(d, float("nan")) for d in dev]
    with cc.Instance(0, 7, 1 << 12, 128, 14) as inst:
        with cc.VolumeBatch(inst, [v.shape for v in vols], 2, steps, graph=True, z_chunk=z_chunk) as b:
            b.compress(dev)
            b.decompress(outs)
            b.status()
            for i, (v, q) in enumerate(zip(vols, steps)):
                words, bits = b.read_stream(i)
                rw, rb = oracle.compress_volume(v, 2, q)
                assert bits == rb and np.array_equal(words, rw), i
                want = oracle.decompress_volume(rw, rb, v.shape, 2, q)
                assert np.array_equal(outs[i].cpu().numpy().view(np.uint32), want.view(np.uint32)), i


def test_tile_depth_out_of_range_is_rejected():
    vols, steps = bricks(2, 2, seed=78)
    with cc.Instance(0, 7, 1 << 12, 128, 14) as inst:
        for bad in (4, 9, 257):
            with pytest.raises(cc.CudaCompressError):
                cc.VolumeBatch(inst, [v.shape for v in vols], 2, steps, z_chunk=bad)
