"""CUDA graphs of the path, one per size bucket: every run that replays a graph
gives the same results, bit for bit, as the kernel-by-kernel path, including the
runs that exceed a graph's capacity and are run again kernel by kernel."""
import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert (a.num_curvelets, a.valid_pairs, a.total_neighbor_pairs, a.max_num_of_neighbors, a.truncated_anchors) == \
        (b.num_curvelets, b.valid_pairs, b.total_neighbor_pairs, b.max_num_of_neighbors, b.truncated_anchors)
    assert np.array_equal(a.chains, b.chains)
    assert np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))


@pytest.fixture(scope="module")
def direct():
    eng = cvl.Engine()
    eng.set_graphs(False)
    yield eng
    eng.close()


def test_graph_runs_equal_direct_runs(direct, golden_kat):
    maps = [synth.plain_small(s) for s in range(4)] + [synth.mixed_map(2000), synth.plain_hd(1000)]
    kats = [golden_kat[k] for k in golden_kat.files if k.endswith("/edges")]
    with cvl.Engine() as eng:
        for m in maps + [k for k in kats if k.shape[1] == 4]:
            _same(eng.run(m), direct.run(m))
        st = eng.graph_stats()
    assert st["replays"] >= len(maps) and st["captures"] >= 2 and st["fallbacks"] == 0, st
    print(f"[graphs] {st}")


def test_graph_batches_equal_direct(direct):
    small = [synth.plain_small(100 + s, 640, 480) for s in range(40)]
    with cvl.Engine() as eng:
        for maps in (small[:8], small, [synth.mixed_map(2001)] + small[:5]):
            b, bd = eng.upload_batch(maps), direct.upload_batch(maps)
            r, rd = eng.run_batch(b), direct.run_batch(bd)
            for k in range(len(maps)):
                _same(r.map(k), rd.map(k))
            r.close(), rd.close(), b.close(), bd.close()
        st = eng.graph_stats()
    assert st["replays"] >= 3 and st["fallbacks"] == 0, st


def test_graph_params_and_truncation(direct, golden_kat):
    e = golden_kat["blob150/edges"]
    p2 = cvl.CurveletParams(nrad=4.5, dx=0.3, dt_deg=10.0, max_k=0.5, sx=0.15, st=0.05, group_max_sz=6)
    with cvl.Engine() as eng:
        _same(eng.run(e), direct.run(e))
        m = synth.plain_small(9)[:3000]
        _same(eng.run(m, p2), direct.run(m, p2))
        _same(eng.run(m), direct.run(m))
        assert eng.graph_stats()["captures"] >= 2


def test_graph_capacity_overflow_falls_back(direct):
    """Bucket 0 with 64 Ki-pair chunks holds 128 Ki pairs: a 60k-edge map has more,
    is flagged on the device and run kernel by kernel, with the same results."""
    m = synth.mixed_map(2000)  # 49,622 edges
    with cvl.Engine() as eng:
        eng.set_tuning(0, chunk_pairs=1 << 16)
        _same(eng.run(m), direct.run(m))
        st = eng.graph_stats()
        assert st["fallbacks"] == 1, st
        small = synth.plain_small(2)
        _same(eng.run(small), direct.run(small))
        assert eng.graph_stats()["fallbacks"] == 1


def test_warmup_then_runs_equal_a_fresh_engine(engine):
    """cvl_engine_warmup runs its built-in maps through every form; the engine's later
    results equal a fresh engine's, and its graph switch is as it was."""
    maps = [synth.plain_small(11), synth.plain_hd(1000)]
    with cvl.Engine() as warm:
        warm.warmup()
        assert warm.graph_stats()["enabled"] == 1
        got = [warm.run(m) for m in maps]
    for a, m in zip(got, maps):
        b = engine.run(m)
        assert np.array_equal(a.chains, b.chains) and np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))
