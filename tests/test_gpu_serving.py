"""Continuous-batching brick service (cudacompress_b200.serving): every
result in a mixed, continuously batched run is bit-identical to the same
request served alone (a server run holding only that request) and to the
plain single-volume codec."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402
from cudacompress_b200 import fields, serving  # noqa: E402


@pytest.fixture(scope="module")
def server():
    src = fields.turbulence_field(64, 128, 16, seed=1006)
    sources = {32: [torch.from_numpy(np.ascontiguousarray(src[i * 8:i * 8 + 32, :32, i * 4:i * 4 + 32])).cuda()
                    for i in range(5)],
               64: [torch.from_numpy(np.ascontiguousarray(np.roll(src, 7 * i, axis=2))).cuda() for i in range(3)]}
    s = serving.BrickServer(0, sources, {32: 6, 64: 3}, levels=3, q0=0.02, keep_results=True)
    yield s
    s.close()


def check(server, reqs):
    inst = cc.Instance(0, 7, 32 ** 3, 128, 14)
    for r in reqs:
        assert r.done >= r.arrival
        if r.op == serving.DECODE:
            words, bits = server.store[r.edge][r.brick]
            alone = torch.empty((r.edge,) * 3, dtype=torch.float32, device="cuda")
            cc.decompress_volume_float(inst, alone, 3, server.q0, words, bits)
            torch.cuda.synchronize()
            assert torch.equal(alone.view(torch.int32), r.result.view(torch.int32)), r.rid
        else:
            w, b = cc.compress_volume_float(inst, server.sources[r.edge][r.brick], 3, server.q0)
            torch.cuda.synchronize()
            words, bits = r.result
            assert bits == b and np.array_equal(words, w[: (b + 31) // 32].cpu().numpy().view(np.uint32)), r.rid
    inst.close()


def test_mixed_run_equals_alone(server):
    reqs = serving.poisson_requests(80, 20000.0, (32, 64), 0.8, 3, seed=5)
    for r in reqs:
        r.brick %= len(server.sources[r.edge])
    done = server.run(reqs)
    assert all(r.done > 0 for r in done)
    check(server, done)
    # the same requests one at a time
    for r in done[:12]:
        one = serving.Request(r.rid, r.op, r.edge, 0.0, r.brick)
        server.run([one])
        if r.op == serving.DECODE:
            assert torch.equal(one.result.view(torch.int32), r.result.view(torch.int32))
        else:
            assert one.result[1] == r.result[1] and np.array_equal(one.result[0], r.result[0])


def test_latency_stats(server):
    reqs = serving.poisson_requests(40, 2000.0, (32,), 0.9, 5, seed=9)
    done = server.run(reqs)
    st = serving.latency_stats(done)
    assert st["requests"] == 40 and st["p99_ms"] >= st["p50_ms"] > 0


def test_budget_defers_requests_and_results_stay_equal():
    """A budget that holds the resident store plus eight 32^3 requests: forty
    32^3 decodes arriving at once run in launches the budget cuts short,
    never more than the budget admitted, each result equal to the brick
    decoded alone."""
    src = fields.turbulence_field(64, 128, 16, seed=1007)
    sources = {32: [torch.from_numpy(np.ascontiguousarray(src[i * 8:i * 8 + 32, :32, :32])).cuda() for i in range(4)],
               64: [torch.from_numpy(src.copy()).cuda()]}
    probe = serving.BrickServer(0, sources, {32: 6, 64: 1}, levels=3, q0=0.02)
    store = probe.store_bytes
    probe.close()
    budget = store + serving.request_bytes(64)          # = eight 32^3 requests
    with pytest.raises(ValueError):
        serving.BrickServer(0, sources, {32: 6, 64: 1}, levels=3, q0=0.02, budget_bytes=budget - 1)
    s = serving.BrickServer(0, sources, {32: 6, 64: 1}, levels=3, q0=0.02, budget_bytes=budget, keep_results=True)
    try:
        reqs = [serving.Request(i, serving.DECODE, 32, 0.0, i % 4) for i in range(40)]
        done = s.run(reqs)
        assert all(r.done > 0 for r in done)
        assert 0 < s.peak_admitted <= budget - s.store_bytes
        assert s.peak_admitted == 8 * serving.request_bytes(32)  # the budget, not the 12 slots, bound the run
        check(s, done)
    finally:
        s.close()
