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
    for m, g in zip(maps, got):
        _same(engine.run(m), g)
    assert st["completed"] == 6 and st["launches"] == 6 and st["admitted_bytes"] == 0
    assert len(ms) == 6 and sorted(ed.tolist()) == sorted(m.shape[0] for m in maps)


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
