"""Every tuning of the engine gives the same curvelets bit for bit; the
autotuner installs a valid tuning for the batch's bucket."""
import json

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import _abi, autotune, synth

pytestmark = pytest.mark.gpu

VARIANTS = [
    dict(cell_size=2), dict(cell_size=8), dict(bundle_blocks_per_sm=3), dict(growth_blocks_per_sm=6), dict(growth_blocks_per_sm=4),
    dict(seeds_per_group=8), dict(anchors_per_warp=1), dict(anchors_per_warp=16), dict(chunk_pairs=1 << 16),
    dict(cell_size=8, seeds_per_group=8, anchors_per_warp=2, bundle_blocks_per_sm=3, chunk_pairs=1 << 18),
]


def _same(a, b):
    assert np.array_equal(a.chains, b.chains)
    assert np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))
    assert (a.valid_pairs, a.total_neighbor_pairs, a.max_num_of_neighbors) == \
        (b.valid_pairs, b.total_neighbor_pairs, b.max_num_of_neighbors)


@pytest.mark.parametrize("knobs", VARIANTS, ids=lambda k: ",".join(f"{a}={b}" for a, b in k.items()))
def test_tuning_variants_give_identical_results(knobs):
    maps = [synth.plain_small(1), synth.mixed_map(2000 + 1), synth.plain_hd(1000)]
    with cvl.Engine() as ref_eng, cvl.Engine() as eng:
        eng.set_tuning(-1, **knobs)
        for m in maps:
            _same(ref_eng.run(m), eng.run(m))
        # a ragged batch goes through the same tuned kernels
        b = eng.upload_batch(maps[:2])
        r = eng.run_batch(b)
        for k, m in enumerate(maps[:2]):
            _same(ref_eng.run(m), r.take_map(k))
        r.close()
        b.close()


def test_set_tuning_rejects_out_of_range():
    with cvl.Engine() as eng:
        for bad in (dict(cell_size=3), dict(bundle_blocks_per_sm=5), dict(seeds_per_group=6),
                    dict(anchors_per_warp=0), dict(chunk_pairs=10)):
            with pytest.raises(cvl.CvlError) as ei:
                eng.set_tuning(0, **bad)
            assert ei.value.code == _abi.CVL_EINVAL


def test_autotune_installs_a_tuning(tmp_path):
    m = synth.plain_hd(1000)
    with cvl.Engine() as eng:
        table = autotune.tune(eng, {autotune.bucket_of(m.shape[0]): [m]})
        bucket = autotune.bucket_of(m.shape[0])
        assert bucket in table and table[bucket]["device_ms"] > 0
        assert eng.get_tuning(bucket) == table[bucket]["tuning"]
        path = tmp_path / "tuning.json"
        autotune.save(str(path), table, "B200")
        assert json.loads(path.read_text())["device"] == "B200"
        with cvl.Engine() as eng2:
            autotune.load(str(path), eng2)
            assert eng2.get_tuning(bucket) == table[bucket]["tuning"]
            _same(eng.run(m), eng2.run(m))
