"""Serving (cvl_server_*): continuous batching with memory-budget admission.
Every result equals the same map run alone through cvl_run, whatever it was
batched with; waits time out instead of blocking; admission holds the budget."""
import threading

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import _abi, synth

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.num_curvelets == b.num_curvelets
    assert np.array_equal(a.chains, b.chains)
    assert np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))
    assert (a.valid_pairs, a.total_neighbor_pairs, a.max_num_of_neighbors) == \
        (b.valid_pairs, b.total_neighbor_pairs, b.max_num_of_neighbors)


def _mix():
    maps = [synth.plain_small(s) for s in range(8)]
    maps += [synth.mixed_map(2000 + s) for s in (0, 1, 4, 5)]  # 14k .. 129k edges
    maps += [synth.plain_hd(1000)]                            # 242k: the large lane below
    return maps


def test_server_results_same_alone_and_in_the_mix(engine):
    maps = _mix()
    alone = [engine.run(m) for m in maps]
    with cvl.Server(workers=3, large_map_edges=200_000, max_batch_edges=300_000) as srv:
        ids = [None] * len(maps)
        order = np.random.default_rng(0).permutation(len(maps))

        def submitter(part):
            for k in part:
                ids[k] = srv.submit(maps[k])

        ts = [threading.Thread(target=submitter, args=(order[i::3],)) for i in range(3)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        got = [srv.wait(ids[k], timeout_s=120.0) for k in range(len(maps))]
        st = srv.stats()
    for a, g in zip(alone, got):
        _same(a, g)
    assert st["completed"] == len(maps) and st["failed"] == 0
    assert st["in_flight"] == 0 and st["queued"] == 0 and st["admitted_bytes"] == 0
    assert st["launches"] < len(maps), "waiting maps were not folded into shared launches"
    assert 0 < st["p50_ms"] <= st["p95_ms"] <= st["p99_ms"] <= st["max_ms"]


def test_server_wait_times_out_and_poll_reports_pending(engine):
    hd = synth.plain_hd(1000)
    ref = engine.run(hd)
    with cvl.Server(workers=1) as srv:
        rid = srv.submit(hd)
        with pytest.raises(cvl.CvlError) as ei:
            srv.wait(rid, timeout_s=1e-6)
        assert ei.value.code == _abi.CVL_ETIMEDOUT
        got = srv.wait(rid, timeout_s=120.0)
        _same(ref, got)
        with pytest.raises(cvl.CvlError) as ei:  # handed out once
            srv.poll(rid)
        assert ei.value.code == _abi.CVL_EINVAL
        rid2 = srv.submit(synth.plain_small(3))
        r = None
        for _ in range(200000):
            r = srv.poll(rid2)
            if r is not None:
                break
        assert r is not None
        _same(engine.run(synth.plain_small(3)), r)


def test_server_admission_budget(engine):
    maps = [synth.plain_small(s) for s in range(6)]
    largest = max(m.shape[0] for m in maps)
    # room for the largest map alone: launches hold one map at a time
    with cvl.Server(workers=2, mem_budget_bytes=largest * 2048, admit_bytes_per_edge=2048) as srv:
        ids = [srv.submit(m) for m in maps]
        got = [srv.wait(i, timeout_s=120.0) for i in ids]
        st = srv.stats()
        with pytest.raises(cvl.CvlError) as ei:
            srv.submit(synth.plain_hd(1000))
        assert ei.value.code == _abi.CVL_ENOMEM
        ms, ed = srv.latencies()
        rt = srv.request_times()
    for m, g in zip(maps, got):
        _same(engine.run(m), g)
    assert st["completed"] == 6 and st["launches"] == 6 and st["admitted_bytes"] == 0
    assert len(ms) == 6 and sorted(ed.tolist()) == sorted(m.shape[0] for m in maps)
    # the per-request breakdown: one entry per request, its parts within its total
    assert len(rt) == 6 and sorted(rt["edges"].tolist()) == sorted(m.shape[0] for m in maps)
    assert np.all(rt["launch_maps"] == 1)
    parts = rt["queue_ms"] + rt["upload_ms"] + rt["run_ms"] + rt["result_ms"]
    assert np.all(parts <= rt["total_ms"] + 0.5) and np.all(rt["run_ms"] > 0)


def test_server_next_hands_out_in_completion_order(engine):
    maps = [synth.plain_small(s) for s in range(5)]
    with cvl.Server(workers=2) as srv:
        ids = [srv.submit(m) for m in maps]
        seen = {}
        for _ in maps:
            rid, res = srv.next(timeout_s=120.0)
            seen[rid] = res
        assert srv.next(timeout_s=1.0) is None  # nothing queued or running
    assert sorted(seen) == sorted(ids)
    for rid, m in zip(ids, maps):
        _same(engine.run(m), seen[rid])


def test_engine_reserved_workspace_runs_without_allocation():
    """cvl_engine_reserve_workspace: runs within the reserved shape allocate no
    device memory, and give the same results as an engine that grew on demand."""
    maps = [synth.plain_small(0), synth.plain_hd(1000), synth.mixed_map(2004), synth.plain_small(3)]
    n = max(m.shape[0] for m in maps)
    with cvl.Engine() as grown, cvl.Engine() as eng:
        tot, chunk = eng.workspace_bytes(n, 40 * n, 8 * n)
        eng.reserve_workspace(n, 40 * n, 8 * n)
        m0 = eng.memory()
        assert m0["held_bytes"] >= tot - (1 << 20), (m0, tot)
        for m in maps:
            _same(grown.run(m), eng.run(m))
        m1 = eng.memory()
    assert m1["device_grows"] == m0["device_grows"], (m0, m1)
    print(f"[reserve] {n} edges: workspace {tot / 2**30:.2f} GiB (bundle chunk {chunk / 2**30:.2f} GiB), "
          f"{len(maps)} runs, no allocation")


def test_server_stream_allocates_no_device_memory(engine):
    """The default server reserves each worker's workspace at creation: a Poisson
    stream over every size class, a 3.79M-edge map included, then runs with no
    device allocation (device_grows unchanged after creation), and its results
    equal the maps run alone."""
    import time
    big = synth.mixed_map(2038)  # 3,791,782 edges: the largest map of the 64-map batch
    small = [synth.plain_small(s) for s in range(6)]
    mid = [synth.mixed_map(s) for s in (2000, 2004, 2005)] + [synth.plain_hd(1000)]
    maps = small + mid + [synth.dense_4k(4000), big] + small[:3]
    rng = np.random.default_rng(3)
    with cvl.Server() as srv:
        st0 = srv.stats()
        ids = []
        for k in rng.permutation(len(maps)):
            ids.append((k, srv.submit(maps[k])))
            time.sleep(float(rng.exponential(0.02)))
        got = {k: srv.wait(i, timeout_s=300.0) for k, i in ids}
        st = srv.stats()
    assert st["completed"] == len(maps) and st["failed"] == 0
    assert st["device_grows"] == st0["device_grows"], (st0["device_grows"], st["device_grows"])
    for k in range(len(small) + len(mid)):
        _same(engine.run(maps[k]), got[k])
    print(f"[server] reserved {st['reserved_bytes'] / 2**30:.1f} GiB at creation; {len(maps)} maps, "
          f"{st['launches']} launches, device allocations in the stream: {st['device_grows'] - st0['device_grows']}")
