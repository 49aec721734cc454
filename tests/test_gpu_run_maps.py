"""cvl_run_maps: many maps host to host with the result copies overlapping the
compute; every map's result equals the map run alone (cvl_run), bit for bit,
whatever the grouping."""
import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth

pytestmark = pytest.mark.gpu


def _same(a, b):
    return (np.array_equal(a.chains, b.chains) and np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))
            and (a.valid_pairs, a.total_neighbor_pairs, a.max_num_of_neighbors, a.truncated_anchors, a.num_edges)
            == (b.valid_pairs, b.total_neighbor_pairs, b.max_num_of_neighbors, b.truncated_anchors, b.num_edges))


def test_run_maps_equals_single_runs(engine):
    maps = [synth.plain_small(s, 480 + 40 * (s % 4), 320) for s in range(10)] + [synth.plain_hd(1000)]
    maps.insert(3, synth.plain_small(77, 64, 48)[:40])  # a tiny map
    singles = [engine.run(m) for m in maps]
    for group_edges in (0, 1, 30_000, 1 << 30):
        got = engine.run_maps(maps, group_edges=group_edges)
        assert len(got) == len(maps)
        for k, (a, b) in enumerate(zip(got, singles)):
            assert _same(a, b), (group_edges, k)
    # the concatenated form, and results that outlive later calls
    allrows = np.concatenate(maps)
    got = engine.run_maps(allrows, counts=[m.shape[0] for m in maps], group_edges=50_000)
    engine.run(maps[0])
    assert all(_same(a, b) for a, b in zip(got, singles))


def test_run_maps_params_and_errors(engine):
    maps = [synth.plain_small(s) for s in range(3)]
    prm = cvl.CurveletParams(group_max_sz=6, max_k=0.4)
    got = engine.run_maps(maps, prm, group_edges=1)
    assert all(_same(a, engine.run(m, prm)) for a, m in zip(got, maps))
    with pytest.raises(cvl.CvlError):
        engine.run_maps(np.concatenate(maps), counts=[maps[0].shape[0], 0, maps[1].shape[0] + maps[2].shape[0]])
    assert _same(engine.run_maps(maps[:1])[0], engine.run(maps[0]))


def test_run_maps_gated_copies_on_large_groups(engine):
    """Groups above the graph buckets (512 Ki edges) run kernel by kernel in chunks,
    and each group's result copies are released during the next group's growth
    kernels: the results still equal the maps run alone, bit for bit."""
    # 598k, 621k, 1.25M and 1.31M edges, and two small maps folded with the large ones
    maps = [synth.mixed_map(s) for s in (2037, 2041, 2010, 2009)] + [synth.plain_small(3), synth.plain_small(4)]
    singles = [engine.run(m) for m in maps]
    with cvl.Engine() as eng:
        for b in range(4):
            eng.set_tuning(b, chunk_pairs=1 << 18)  # more chunks: more gated releases
        # group_edges 1: one map per group (four groups above the graph buckets);
        # 2 Mi: groups of several maps
        for group_edges in (1, 2 << 20):
            got = eng.run_maps(maps, group_edges=group_edges)
            assert all(_same(a, b) for a, b in zip(got, singles)), group_edges
