"""Parity at the full sizes of the workloads (the 64-map batch of 33.7M edges;
the dense 3840x2160 stress map with high-curvature arcs and 40% clutter):
against the oracle where it finishes in seconds, and otherwise through the
size-independent property that each map's curvelets in a ragged batch are
bit-identical to the same map run alone."""
import os

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth
from tests.parity import assert_same_curvelets

pytestmark = pytest.mark.gpu

CORES = os.cpu_count() or 1


def _identical(a, b, label):
    assert a.num_curvelets == b.num_curvelets, label
    assert np.array_equal(a.chains, b.chains), label
    assert np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64)), label
    assert (a.valid_pairs, a.total_neighbor_pairs, a.max_num_of_neighbors, a.truncated_anchors) == \
        (b.valid_pairs, b.total_neighbor_pairs, b.max_num_of_neighbors, b.truncated_anchors), label


def test_dense_stress_map_vs_oracle(engine, oracle):
    e = synth.dense_4k(4000)
    r = engine.run(e)
    o = oracle.run(e, nthreads=CORES)
    assert (r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == \
        (o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors)
    st = assert_same_curvelets(r, o, label="dense_4k")
    print(f"[fullsize] dense_4k: edges={e.shape[0]} curvelets={st['rows']} max_rel={st['max_rel']}")


def test_full_64_map_batch_equals_each_map_alone(engine, oracle):
    maps = synth.mixed64(2000, 64)
    with cvl.Engine() as beng:  # the batch's outputs stay on its own engine while the plain runs go on
        batch = beng.upload_batch(maps)
        res = beng.run_batch(batch)
        stats = res.stats()
        assert stats["num_maps"] == 64
        total = 0
        for k, m in enumerate(maps):
            got = res.take_map(k)
            _identical(got, engine.run(m), f"map {k}")
            total += got.num_curvelets
            del got
        assert total == stats["num_curvelets"]
        res.close()
        batch.close()
    # and four maps of different sizes against the oracle
    order = np.argsort([m.shape[0] for m in maps])
    for k in (int(order[0]), int(order[20]), int(order[40]), int(order[52])):
        r = engine.run(maps[k])
        o = oracle.run(maps[k], nthreads=CORES)
        assert (r.valid_pairs, r.total_neighbor_pairs) == (o.valid_pairs, o.total_neighbor_pairs)
        assert_same_curvelets(r, o, label=f"mixed map {k} ({maps[k].shape[0]} edges)")
