"""GPU tests of the persistent grouped GEMM (no reference counterpart; each
problem keeps sgemm()'s contract, src/sgemm.cuh:19-30)."""
import json
import time

import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _table(path, split, tile=1, stages=3, depth=None):
    torch = _torch()
    p = torch.cuda.get_device_properties(0)
    buckets = [{"mn": a, "k": b, "tile": tile, "split": split} for a in range(3) for b in range(3)]
    if depth is not None:  # the buckets' own stage count
        for x in buckets:
            x["stages"] = depth
    lines = ",\n".join("  " + json.dumps(x) for x in buckets)
    path.write_text(f'{{\n "device": "{p.name}",\n "sm_count": {p.multi_processor_count},\n'
                    f' "stages": {stages},\n "buckets": [\n{lines}\n ]\n}}\n')
    return str(path)


def _make(shapes, seed, lds=None):
    """Problems with seeded inputs; returns (specs, host inputs, C0 copies)."""
    torch = _torch()
    specs, host = [], []
    for i, (m, n, k) in enumerate(shapes):
        A = oracle.fill(m, k, seed + i, 1, 0)
        B = oracle.fill(k, n, seed + i, 2, 0)
        C = oracle.fill(m, n, seed + i, 3, 0)
        ld = lds[i] if lds else (None, None, None)

        def dev(x, l):
            r, c = x.shape
            big = torch.full((r, max(l or c, 1)), float("nan"), device="cuda")
            if c:
                big[:, :c] = torch.from_numpy(x).cuda()
            return big[:, :c] if c else big[:, :0]

        dA, dB, dC = dev(A, ld[0]), dev(B, ld[1]), dev(C, ld[2])
        alpha, beta = (1.5, 0.5) if i % 3 else (1.0, 0.0)
        specs.append((dA, dB, dC, alpha, beta))
        host.append((A, B, C, alpha, beta))
    return specs, host


SHAPES = [(1, 1, 1), (64, 64, 64), (300, 520, 1001), (129, 257, 33), (1031, 97, 263),
          (97, 1031, 61), (50, 70, 0), (640, 512, 2048), (130, 270, 77), (256, 256, 512)]
LDS = [None, None, None, None, None, None, None, None, (79, 275, 273), (None, None, 260)]


def _lds():
    return [x if x else (None, None, None) for x in LDS]


def test_grouped_bit_exact_with_plain_path():
    torch = _torch()
    specs, host = _make(SHAPES, 100, _lds())
    plan = sg.GroupedPlan(specs)
    plan.launch(use_graph=False)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    for (dA, dB, dC, a, b), (A, B, C, _, _) in zip(specs, host):
        want = oracle.sgemm_basic(A, B, C, a, b, basic=False)
        got = dC.cpu().numpy()
        assert np.array_equal(got, want), f"{A.shape}x{B.shape}"
    info = plan.info()
    assert info["work_items"] == info["tiles"]
    plan.close()


def test_grouped_graph_replay_equals_direct():
    torch = _torch()
    specs, host = _make(SHAPES, 200, _lds())
    C0 = [s[2].clone() for s in specs]
    plan = sg.GroupedPlan(specs)
    plan.launch(use_graph=True)
    torch.cuda.synchronize()
    first = [s[2].clone() for s in specs]
    for s, c in zip(specs, C0):
        s[2].copy_(c)
    plan.launch(use_graph=True)  # replay of the captured graph
    torch.cuda.synchronize()
    for s, f in zip(specs, first):
        assert torch.equal(s[2], f)
    plan.close()


@pytest.mark.parametrize("split", [2, 4])
def test_grouped_split_k_deterministic_and_accurate(tmp_path, split):
    torch = _torch()
    shapes = [(64, 64, 4096), (128, 256, 3000), (200, 136, 1001), (300, 520, 2048)]
    specs, host = _make(shapes, 300)
    C0 = [s[2].clone() for s in specs]
    table = _table(tmp_path / "t.json", split)
    plan = sg.GroupedPlan(specs, tuning_json=table)
    assert plan.info()["work_items"] > plan.info()["tiles"]
    plan.launch()
    torch.cuda.synchronize()
    first = [s[2].clone() for s in specs]
    for s, c in zip(specs, C0):
        s[2].copy_(c)
    plan.launch()
    torch.cuda.synchronize()
    for s, f, (A, B, C, a, b) in zip(specs, first, host):
        assert torch.equal(s[2], f)  # same bits on every launch
        ref, mag = oracle.dgemm(A, B, C, a, b)
        e = oracle.error_stats(f.cpu().numpy(), ref, mag)
        ep = oracle.error_stats(oracle.sgemm_basic(A, B, C, a, b, basic=False), ref, mag)
        assert e["max_componentwise"] <= 1.5 * ep["max_componentwise"] + 2.0 ** -23
    plan.close()


SKINNY = [(16, 4096, 4096), (1, 1000, 300), (31, 129, 1000), (33, 4100, 64), (48, 640, 2048),
          (8, 8, 8), (20, 3000, 3001), (200, 300, 50)]


def test_grouped_skinny_tiles_bit_exact_with_plain_path():
    # tall-skinny problems (the serving loop's common case) run on 32 x 128
    # tiles; every element keeps the plain path's FMA chain, so bits agree
    torch = _torch()
    lds = [(None, None, None)] * (len(SKINNY) - 1) + [(53, 307, 301)]
    specs, host = _make(SKINNY, 700, lds)
    plan = sg.GroupedPlan(specs)
    plan.launch(use_graph=True)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    for (dA, dB, dC, a, b), (A, B, C, _, _) in zip(specs, host):
        want = oracle.sgemm_basic(A, B, C, a, b, basic=False)
        assert np.array_equal(dC.cpu().numpy(), want), f"{A.shape}x{B.shape}"
    plan.close()


def test_grouped_skinny_split_k_deterministic_and_accurate(tmp_path):
    torch = _torch()
    shapes = [(16, 1024, 4096), (40, 520, 3000)]
    specs, host = _make(shapes, 800)
    C0 = [s[2].clone() for s in specs]
    plan = sg.GroupedPlan(specs, tuning_json=_table(tmp_path / "t.json", 4))
    assert plan.info()["work_items"] > plan.info()["tiles"]
    plan.launch()
    torch.cuda.synchronize()
    first = [s[2].clone() for s in specs]
    for s, c in zip(specs, C0):
        s[2].copy_(c)
    plan.launch()
    torch.cuda.synchronize()
    for s, f, (A, B, C, a, b) in zip(specs, first, host):
        assert torch.equal(s[2], f)
        ref, mag = oracle.dgemm(A, B, C, a, b)
        e = oracle.error_stats(f.cpu().numpy(), ref, mag)
        ep = oracle.error_stats(oracle.sgemm_basic(A, B, C, a, b, basic=False), ref, mag)
        assert e["max_componentwise"] <= 1.5 * ep["max_componentwise"] + 2.0 ** -23
    plan.close()


def _workload(n, seed):
    """The 512-problem grouped workload: M, N, K log-uniform on [64, 4096], multiples of 8."""
    rng = np.random.default_rng(seed)
    vals = np.exp(rng.uniform(np.log(64), np.log(4096), size=(n, 3)))
    return [tuple(int(max(8, round(v / 8) * 8)) for v in row) for row in vals]


def test_grouped_512_problems_vs_sequential():
    torch = _torch()
    shapes = _workload(512, 7)
    specs = []
    for i, (m, n, k) in enumerate(shapes):
        A = torch.empty((m, k), device="cuda")
        B = torch.empty((k, n), device="cuda")
        C = torch.empty((m, n), device="cuda")
        sg.fill_random(A, 500 + i, 1, 0)
        sg.fill_random(B, 500 + i, 2, 0)
        sg.fill_random(C, 500 + i, 3, 0)
        specs.append((A, B, C, 1.5, 0.5))
    C0 = [s[2].clone() for s in specs]
    probs = sg.make_problems(specs)
    sg.grouped_sequential(probs)
    torch.cuda.synchronize()
    seq = [s[2].clone() for s in specs]
    for s, c in zip(specs, C0):
        s[2].copy_(c)
    plan = sg.GroupedPlan(specs)
    plan.launch()
    torch.cuda.synchronize()
    for s, want in zip(specs, seq):
        assert torch.equal(s[2], want)
    # timing, reported not asserted (bench.py carries the measured numbers)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    plan.launch()
    ev[1].record()
    ev[2].record()
    sg.grouped_sequential(probs)
    ev[3].record()
    torch.cuda.synchronize()
    flop = sum(2.0 * m * n * k for m, n, k in shapes)
    tg, ts = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
    print(f"grouped {tg:.3f} ms ({flop / tg * 1e-9:.1f} GFLOP/s), sequential {ts:.3f} ms "
          f"({flop / ts * 1e-9:.1f} GFLOP/s), info {plan.info()}")
    plan.close()


def test_autotuner_writes_table_and_plan_uses_it(tmp_path):
    torch = _torch()
    shapes = _workload(48, 11)
    specs = []
    for i, (m, n, k) in enumerate(shapes):
        A = torch.empty((m, k), device="cuda")
        B = torch.empty((k, n), device="cuda")
        C = torch.zeros((m, n), device="cuda")
        sg.fill_random(A, 900 + i, 1, 0)
        sg.fill_random(B, 900 + i, 2, 0)
        specs.append((A, B, C, 1.0, 0.0))
    probs = sg.make_problems(specs)
    path = str(tmp_path / "tuned.json")
    t0 = time.time()
    sg.autotune_grouped(probs, path)
    print(f"autotune took {time.time() - t0:.1f} s")
    text = open(path).read()
    table = json.loads(text)
    assert table["device"] == torch.cuda.get_device_properties(0).name
    assert table["sm_count"] == torch.cuda.get_device_properties(0).multi_processor_count
    assert len(table["buckets"]) == 9
    print(text)
    plan = sg.GroupedPlan(specs, tuning_json=path)
    plan.launch()
    torch.cuda.synchronize()
    for (A, B, C, a, b) in specs[:6]:
        want = A.double() @ B.double()
        assert torch.allclose(C.double(), want, rtol=0, atol=1e-5 * want.abs().max().item())
    plan.close()


@pytest.mark.parametrize("depth", [2, 3])
def test_bucket_stage_count_keeps_results(tmp_path, depth):
    """A bucket's stage count changes only how many k blocks each item keeps
    in flight through the ring, never the arithmetic: results stay equal to
    the plain path's, bit for bit (4-stage ring, split 1)."""
    torch = _torch()
    specs, host = _make(SHAPES, 300, _lds())
    plan = sg.GroupedPlan(specs, tuning_json=_table(tmp_path / "t.json", 1, tile=0, stages=4,
                                                    depth=depth))
    plan.launch(use_graph=True)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    for (dA, dB, dC, a, b), (A, B, C, _, _) in zip(specs, host):
        assert np.array_equal(dC.cpu().numpy(), oracle.sgemm_basic(A, B, C, a, b, basic=False))
    plan.close()


def test_autotuner_beats_default_on_k_heavy_problems(tmp_path):
    """16 problems of 128 x 128 x 65536: 32 tiles leave almost every resident
    slot idle, so the default plan (no split-K) is far from the tuned one,
    which splits K; the tuned plan is several times faster and its results
    stay within FP32 accuracy (the split sums are reduced in a fixed order)."""
    torch = _torch()
    specs = []
    for i in range(16):
        A = torch.empty((128, 65536), device="cuda")
        B = torch.empty((65536, 128), device="cuda")
        C = torch.zeros((128, 128), device="cuda")
        sg.fill_random(A, 1200 + i, 1, 0)
        sg.fill_random(B, 1200 + i, 2, 0)
        specs.append((A, B, C, 1.0, 0.0))
    probs = sg.make_problems(specs)
    path = str(tmp_path / "tuned.json")
    sg.autotune_grouped(probs, path)
    table = json.loads(open(path).read())
    print(table)
    assert any(b["split"] > 1 for b in table["buckets"])

    def time_plan(plan):
        plan.launch()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            plan.launch()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return sorted(ts)[2]

    default, tuned = sg.GroupedPlan(specs), sg.GroupedPlan(specs, tuning_json=path)
    t_default, t_tuned = time_plan(default), time_plan(tuned)
    print(f"default {t_default:.3f} ms, tuned {t_tuned:.3f} ms")
    assert t_tuned < 0.5 * t_default
    for (A, B, C, a, b) in specs[:4]:
        want = A.double() @ B.double()
        assert torch.allclose(C.double(), want, rtol=0, atol=1e-5 * want.abs().max().item())
    default.close()
    tuned.close()
