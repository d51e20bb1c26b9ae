"""GPU tests of the continuous-batching server (no reference counterpart;
each request keeps sgemm()'s contract, src/sgemm.cuh:19-30)."""
import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu

MIX = [(64, 4096, 4096), (512, 512, 512), (200, 4096, 4096), (1024, 1024, 1024),
       (16, 4096, 4096), (777, 777, 777)]


def _expected(m, n, k, seed, path):
    """The same request run directly through the library, outside any server."""
    import torch
    A = torch.empty((m, k), device="cuda")
    B = torch.empty((k, n), device="cuda")
    C = torch.empty((m, n), device="cuda")
    sg.fill_random(A, seed, 1, sg.DIST_UNIFORM_PM1)
    sg.fill_random(B, seed, 2, sg.DIST_UNIFORM_PM1)
    sg.fill_random(C, seed, 3, sg.DIST_UNIFORM_PM1)
    if path == "plain":
        sg.sgemm(A, B, C, 1.5, 0.5)
    else:
        sg.sgemm_split(path, A, B, C, 1.5, 0.5)
    torch.cuda.synchronize()
    return C.cpu().numpy()


@pytest.mark.parametrize("path", ["plain", "bf16x6"])
def test_result_same_alone_and_in_the_mix(path):
    target = (300, 520, 1001)
    seed = 4242
    alone = sg.Server(1 << 33, slots=2, max_batch=8, path=path, keep_results=True)
    rid = alone.submit(*target, alpha=1.5, beta=0.5, seed=seed)
    alone.drain()
    c_alone = alone.read_result(rid, target[0], target[1])
    assert alone.result(rid)["batch_size"] == 1
    alone.close()

    mix = sg.Server(1 << 33, slots=2, max_batch=8, path=path, keep_results=True)
    ids = []
    for i, shape in enumerate(MIX * 2):
        ids.append(mix.submit(*shape, alpha=1.5, beta=0.5, seed=100 + i))
        if i == 5:
            rid = mix.submit(*target, alpha=1.5, beta=0.5, seed=seed)
    mix.drain()
    c_mix = mix.read_result(rid, target[0], target[1])
    st = mix.stats()
    bs = mix.result(rid)["batch_size"]
    mix.close()
    print(path, "batch size in the mix:", bs, st)
    assert np.array_equal(c_alone, c_mix)  # same bits alone and in the mix
    assert np.array_equal(c_alone, _expected(*target, seed, path))
    if path == "plain":  # and equal to the oracle's restatement of the reference
        m, n, k = target
        A = oracle.fill(m, k, seed, 1, 0)
        B = oracle.fill(k, n, seed, 2, 0)
        C = oracle.fill(m, n, seed, 3, 0)
        assert np.array_equal(c_alone, oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False))


def test_continuous_batching_overlaps_batches():
    srv = sg.Server(64 << 30, slots=2, max_batch=16, path="plain")
    st = srv.run_poisson(rate_per_s=3000.0, n_requests=400, seed=5)
    srv.close()
    print(st)
    assert st["completed"] == 400 and st["failed"] == 0 and st["rejected"] == 0
    assert st["max_batches_in_flight"] == 2  # a new batch started while one ran
    assert st["max_batch_size"] > 1          # arrivals during a batch joined the next one
    assert st["batches"] < 400
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]


def test_admission_waits_for_memory_and_refuses_oversize():
    budget = 420 << 20  # two 4096^2 requests (3 x 64 MiB each) fit, three do not
    srv = sg.Server(budget, slots=2, max_batch=4, path="plain")
    with pytest.raises(sg.SgemmError) as e:
        srv.submit(8192, 8192, 8192)  # 768 MiB: can never fit
    assert e.value.status == sg.ERR_REJECTED
    for i in range(8):
        srv.submit(4096, 4096, 4096, seed=i)
    srv.drain()
    st = srv.stats()
    srv.close()
    print(st)
    assert st["completed"] == 8 and st["rejected"] == 1
    assert st["peak_pool_bytes"] <= budget
    assert st["peak_waiting"] >= 1  # requests queued for memory


def test_injected_allocation_failures_and_delays():
    srv = sg.Server(8 << 30, slots=2, max_batch=4, path="plain", inject_alloc_failure_every=3,
                    inject_batch_delay_ms=20)
    for i in range(9):
        srv.submit(256, 256, 256, seed=i)
    with pytest.raises(sg.SgemmError):
        srv.drain()  # reports the failed admissions
    st = srv.stats()
    srv.close()
    print(st)
    assert st["failed"] == 3 and st["completed"] == 6
    assert st["p50_ms"] >= 20.0  # every batch waited the injected delay


@pytest.mark.parametrize("path", ["plain", "bf16x6"])
def test_trace_accounts_for_every_request(path):
    srv = sg.Server(64 << 30, slots=2, max_batch=16, path=path)
    st = srv.run_poisson(rate_per_s=2000.0, n_requests=120, seed=9)
    tr = srv.trace()
    srv.close()
    assert st["completed"] == 120 and len(tr) == 120
    assert len({r["request_id"] for r in tr}) == 120
    eps = 1e-9
    for r in tr:
        assert -eps <= r["submit_ms"] <= r["admit_ms"] + eps
        assert r["admit_ms"] <= r["launch_ms"] + eps <= r["done_ms"] + 2 * eps
        # device span: after the window's epoch, ends before the host hears of
        # it (the host and device axes differ by the epoch's enqueue delay)
        assert 0.0 <= r["device_start_ms"] <= r["device_end_ms"]
        assert r["device_end_ms"] <= r["done_ms"] + 0.5
    # every batch's records: all of its requests, one launch and one completion
    by_batch = {}
    for r in tr:
        by_batch.setdefault(r["batch"], []).append(r)
    assert len(by_batch) == st["batches"]
    for recs in by_batch.values():
        assert len(recs) == recs[0]["batch_size"]
        assert len({r["launch_ms"] for r in recs}) == 1 and len({r["done_ms"] for r in recs}) == 1
    # the statistics are the trace's percentiles (nearest rank)
    def pct(v, q):
        v = sorted(v)
        return v[min(len(v) - 1, int(np.ceil(q * len(v))) - 1)]
    lat = [r["done_ms"] - r["submit_ms"] for r in tr]
    que = [r["launch_ms"] - r["submit_ms"] for r in tr]
    svc = [r["done_ms"] - r["launch_ms"] for r in tr]
    assert pct(lat, 0.99) == pytest.approx(st["p99_ms"], abs=1e-6)
    assert pct(que, 0.99) == pytest.approx(st["queue_p99_ms"], abs=1e-6)
    assert pct(svc, 0.50) == pytest.approx(st["service_p50_ms"], abs=1e-6)


def test_destroy_cancels_requests_that_can_never_be_admitted():
    # two kept 4096^2 results fill the budget, so the third request waits for
    # memory that never frees; destroy must cancel it rather than wait
    import threading
    import time
    budget = 420 << 20
    srv = sg.Server(budget, slots=2, max_batch=4, path="plain", keep_results=True)
    for i in range(3):
        srv.submit(4096, 4096, 4096, seed=i)
    t_end = time.time() + 30
    while srv.stats()["completed"] < 2 and time.time() < t_end:
        time.sleep(0.01)
    st = srv.stats()
    assert st["completed"] == 2 and st["peak_waiting"] >= 1
    closer = threading.Thread(target=srv.close)
    closer.start()
    closer.join(timeout=60)
    assert not closer.is_alive(), "destroy waited for a request that could never run"
