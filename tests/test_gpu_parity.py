"""GPU parity: every stage of the CUDA path, through the C ABI, against the
reference fixtures and the pinned CPU restatement on the same inputs.

Rules (tests/parity.py): neighbour lists and chains bit-identical; info columns
without transcendental input bit-identical; the others within 1e-9 relative
(column-scale floor)."""
import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth
from tests.parity import assert_same_curvelets, compare_info

pytestmark = pytest.mark.gpu


def _report(label, st):
    print(f"[parity] {label}: rows={st['rows']} max_rel={st.get('max_rel')} "
          f"bit_identical={st.get('bit_identical_frac')}")


# ---- (c) bundle transport, pair by pair ---------------------------------------
def test_pair_bundles_vs_reference(engine, golden_pairs):
    pairs = golden_pairs["pairs"]
    bmin, bmax, valid = engine.pair_bundles(pairs)
    assert bmin.shape == golden_pairs["bmin"].shape
    assert np.array_equal(valid, golden_pairs["valid"].astype(bool))
    rmin, rmax = golden_pairs["bmin"], golden_pairs["bmax"]
    # cell validity (max > min) is a threshold decision: must match exactly
    assert np.array_equal(bmax > bmin, rmax > rmin)
    for a, b in ((bmin, rmin), (bmax, rmax)):
        d = np.abs(a - b)
        bound = np.maximum(1e-9 * np.maximum(np.abs(a), np.abs(b)), 1e-9 * 0.3)
        assert np.all(d <= bound), float(d.max())
    print(f"[parity] pair bundles: bit-identical cells "
          f"{np.mean(bmin.view(np.uint64) == rmin.view(np.uint64)):.4f} / "
          f"{np.mean(bmax.view(np.uint64) == rmax.view(np.uint64)):.4f}")


# ---- (a)+(b) neighbour graph ---------------------------------------------------
@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_neighbor_graph_vs_reference(engine, golden_files, key):
    e = golden_files[f"{key}/edges"]
    g = engine.build_neighbor_graph(e, 3.5, 3, 128)
    assert np.array_equal(g.neighbor_offsets, golden_files[f"{key}/csr_offsets"])
    assert np.array_equal(g.neighbor_ids, golden_files[f"{key}/csr_ids"])
    assert np.array_equal(g.neighbor_dist2.view(np.uint64), golden_files[f"{key}/csr_dist2"].view(np.uint64))
    assert g.max_num_of_neighbors == int(golden_files[f"{key}/counts"][3])


def test_neighbor_graph_vs_oracle_synthetic(engine, oracle):
    for e in (synth.plain_small(3), synth.mixed_map(2004)):
        g = engine.build_neighbor_graph(e, 3.5, 3, 128)
        c = oracle.build_csr(e, nthreads=16)
        assert np.array_equal(g.neighbor_offsets, c.offsets)
        assert np.array_equal(g.neighbor_ids, c.ids)
        assert np.array_equal(g.neighbor_dist2.view(np.uint64), c.dist2.view(np.uint64))
        assert g.truncated_anchors == c.truncated_anchors


# ---- the whole path ---------------------------------------------------------------
class _Ref:
    def __init__(self, chains, info):
        self.chains, self.info = chains, info


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_run_vs_reference_fixture(engine, golden_files, key):
    e = golden_files[f"{key}/edges"]
    r = engine.run(e)
    n_cv, vp, tp, md = golden_files[f"{key}/counts"].tolist()
    assert (r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == (n_cv, vp, tp, md)
    st = assert_same_curvelets(r, _Ref(golden_files[f"{key}/chains"], golden_files[f"{key}/info"]), label=key)
    _report(key, st)


def test_run_vs_oracle_TO_edges(engine, oracle, golden_files):
    e = golden_files["TO_edges/edges"]
    r = engine.run(e)
    o = oracle.run(e, nthreads=16)
    n_cv, vp, tp, md = golden_files["TO_edges/counts"].tolist()
    assert (r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == (n_cv, vp, tp, md)
    _report("TO_edges", assert_same_curvelets(r, o, label="TO_edges"))


def test_kat_maps(engine, oracle, golden_kat):
    names = sorted({k.split("/")[0] for k in golden_kat.files})
    for name in names:
        e = golden_kat[f"{name}/edges"]
        gms, mc = golden_kat[f"{name}/params"].tolist()
        p = cvl.CurveletParams(group_max_sz=gms, max_candidates=mc, edge_data_sz=e.shape[1])
        r = engine.run(e, p)
        o = oracle.run(e, group_max_sz=gms, max_candidates=mc)
        assert (r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == \
            (o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors), name
        assert r.truncated_anchors == o.truncated_anchors, name
        assert_same_curvelets(r, o, label=name)
        if not o.truncated_anchors:
            ref = _Ref(golden_kat[f"{name}/chains"], golden_kat[f"{name}/info"])
            assert_same_curvelets(r, ref, label=name + " vs reference")


@pytest.mark.parametrize("seed", [0, 7])
def test_plain_small_vs_oracle(engine, oracle, seed):
    e = synth.plain_small(seed)
    r = engine.run(e)
    o = oracle.run(e, nthreads=16)
    assert (r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == \
        (o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors)
    _report(f"plain_small[{seed}]", assert_same_curvelets(r, o, label="plain_small"))


def test_plain_hd_full_size_vs_oracle(engine, oracle):
    """The 1920x1080, ~250k-edge map at full size."""
    e = synth.plain_hd(1000)
    r = engine.run(e)
    o = oracle.run(e, nthreads=16)
    assert (r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == \
        (o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors)
    _report("plain_hd", assert_same_curvelets(r, o, label="plain_hd"))


def test_nondefault_params_vs_oracle(engine, oracle):
    e = synth.plain_small(5)[:3000]
    kw = dict(nrad=4.5, dx=0.3, dt_deg=10.0, max_k=0.5, sx=0.15, st=0.05, group_max_sz=6)
    r = engine.run(e, cvl.CurveletParams(**kw))
    o = oracle.run(e, nthreads=16, **kw)
    assert (r.valid_pairs, r.total_neighbor_pairs) == (o.valid_pairs, o.total_neighbor_pairs)
    assert_same_curvelets(r, o, max_k=0.5, label="nondefault")


# ---- the staged template API ------------------------------------------------------
def test_staged_api_matches_one_shot(engine, golden_files):
    e = golden_files["TO_edges_ABC_0006_thresh1/edges"]
    g = cvl.GPUNeighborGraph()
    assert cvl.build_neighbor_csr_graph(e.shape[0], 4, e, 3.5, 3, 128, 1, g, engine=engine)
    dt = (15.0 / 180.0) * cvl.M_PI
    obj = cvl.CurveletGPU(e.shape[0], 4, g, 0.4, dt, 0.1, 0.08, 0.3, 4, 1, e, 3.5, engine=engine)
    res = cvl.CurveletFormationResult()
    assert obj.form_pairwise_bundles(res)
    obj.build_curvelets_greedy()
    one = engine.run(e)
    assert res.valid_pairs == one.valid_pairs
    assert obj.num_curvelets() == one.num_curvelets and obj.chain_width() == 5
    assert np.array_equal(obj._edge_chain_final, one.chains)
    assert np.array_equal(obj._curvelet_info.T.view(np.uint64), one.info.view(np.uint64))
    assert not cvl.build_neighbor_csr_graph(0, 4, e, 3.5, 3, 128, 1, g, engine=engine)
    assert not cvl.build_neighbor_csr_graph(10, 3, e, 3.5, 3, 128, 1, g, engine=engine)


# ---- batches: each map identical alone and in the mix -----------------------------
def test_batch_equals_plain(engine):
    maps = [synth.plain_small(11), synth.plain_small(12)[:50], np.array([[5.0, 5.0, 0.1, 3.0]]),
            synth.mixed_map(2001), synth.plain_small(13)]
    b = engine.upload_batch(maps)
    br = engine.run_batch(b)
    mixed = [br.map(m) for m in range(len(maps))]  # results live in the engine's workspace until fetched
    for m, e in enumerate(maps):
        alone = engine.run(e)
        inmix = mixed[m]
        assert np.array_equal(alone.chains, inmix.chains), m
        assert np.array_equal(alone.info.view(np.uint64), inmix.info.view(np.uint64)), m
        assert (alone.valid_pairs, alone.total_neighbor_pairs, alone.max_num_of_neighbors) == \
            (inmix.valid_pairs, inmix.total_neighbor_pairs, inmix.max_num_of_neighbors), m
    st = br.stats()
    assert st["num_curvelets"] == sum(r.num_curvelets for r in mixed)
    # a result whose outputs were overwritten by a later run refuses to serve stale data
    br2 = engine.run_batch(b)
    engine.run(maps[0])
    with pytest.raises(cvl.CvlError):
        br2.map(0)


# ---- edge cases -------------------------------------------------------------------------
def test_edge_cases(engine):
    with pytest.raises(cvl.CvlError) as ei:
        engine.run(np.zeros((0, 4)))
    assert ei.value.code == cvl._abi.CVL_EINVAL
    with pytest.raises(cvl.CvlError):
        engine.run(np.zeros((5, 3)))
    bad = synth.plain_small(1)[:100].copy()
    bad[17, 0] = np.nan
    with pytest.raises(cvl.CvlError) as ei:
        engine.run(bad)
    assert ei.value.code == cvl._abi.CVL_EINVAL
    with pytest.raises(cvl.CvlError) as ei:
        engine.run(synth.plain_small(1)[:100], cvl.CurveletParams(group_max_sz=17))
    assert ei.value.code == cvl._abi.CVL_EUNSUPPORTED
    one = engine.run(np.array([[1.0, 2.0, 0.3, 4.0]]))
    assert one.num_curvelets == 0 and one.total_neighbor_pairs == 0 and one.valid_pairs == 0
    # engine still usable after the errors
    e = synth.plain_small(2)
    a, b = engine.run(e), engine.run(e)
    assert np.array_equal(a.chains, b.chains) and np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))


@pytest.mark.parametrize("gms", [1, 2, 3, 5, 8, 16])
def test_group_max_sz_range(engine, oracle, gms):
    e = synth.plain_small(4)[:2500]
    r = engine.run(e, cvl.CurveletParams(group_max_sz=gms))
    o = oracle.run(e, group_max_sz=gms)
    assert r.chains.shape[1] == gms + 1
    assert_same_curvelets(r, o, label=f"gms={gms}")


@pytest.mark.parametrize("case", ["blob150", "blob600_mc128", "blob600_mc40"])
def test_truncated_vs_reference_stage(engine, golden_trunc, case):
    """Every anchor truncated at max_candidates: the engine (lowest edge indices
    inside a pixel cell) against the reference's own CurveletCPU stage run on the
    same lowest-index neighbour lists (tests/golden/make_golden_truncated.py)."""
    k = f"{case}/double"
    e = golden_trunc[f"{k}/edges"]
    gms, mc = golden_trunc[f"{k}/params"].tolist()
    r = engine.run(e, cvl.CurveletParams(group_max_sz=gms, max_candidates=mc, edge_data_sz=e.shape[1]))
    assert [r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors,
            r.truncated_anchors] == golden_trunc[f"{k}/counts"].tolist()
    _report(f"truncated {case}", assert_same_curvelets(
        r, _Ref(golden_trunc[f"{k}/chains"], golden_trunc[f"{k}/info"]), label=case + " vs reference stage"))


def test_truncation_blob(engine, oracle):
    rng = np.random.Generator(np.random.PCG64(3))
    e = np.stack([50 + rng.uniform(-2, 2, 600), 50 + rng.uniform(-2, 2, 600), rng.uniform(-3, 3, 600),
                  rng.uniform(1, 5, 600)], 1)
    for mc in (128, 40):
        p = cvl.CurveletParams(max_candidates=mc)
        r = engine.run(e, p)
        o = oracle.run(e, max_candidates=mc)
        assert r.truncated_anchors == o.truncated_anchors and r.truncated_anchors > 0
        assert (r.valid_pairs, r.total_neighbor_pairs) == (o.valid_pairs, o.total_neighbor_pairs)
        assert_same_curvelets(r, o, label=f"blob mc={mc}")
        g = engine.build_neighbor_graph(e, 3.5, 3, mc)
        c = oracle.build_csr(e, max_candidates=mc)
        assert np.array_equal(g.neighbor_ids, c.ids)
