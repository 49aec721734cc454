"""The CPU checker is pinned before it is trusted: the C restatement
(oracle/cvl_oracle.c) must reproduce the reference's own outputs bit for bit
on the committed fixtures (generated by tests/golden/make_golden.py from the
reference's cpu_curvelet code) and, where the reference harness is built, on
fresh runs of the reference itself."""
import hashlib

import numpy as np
import pytest

from curvelet_construction_on_gpu_b200 import synth


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1", "TO_edges"])
def test_restatement_matches_reference_fixtures(oracle, golden_files, key):
    e = golden_files[f"{key}/edges"]
    r = oracle.run(e, nthreads=4)
    n_cv, vp, tp, md = golden_files[f"{key}/counts"].tolist()
    assert (r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == (n_cv, vp, tp, md)
    csr = oracle.build_csr(e, nthreads=4)
    d = golden_files[f"{key}/digests"].tolist()
    assert _digest(r.chains) == d[0]
    assert _digest(r.info) == d[1]
    assert _digest(csr.offsets) == d[2] and _digest(csr.ids) == d[3] and _digest(csr.dist2) == d[4]
    if f"{key}/chains" in golden_files.files:
        assert np.array_equal(r.chains, golden_files[f"{key}/chains"])
        assert np.array_equal(r.info.view(np.uint64), golden_files[f"{key}/info"].view(np.uint64))


def _kat_names(z):
    return sorted({k.split("/")[0] for k in z.files})


def test_restatement_matches_reference_kats(oracle, golden_kat):
    for name in _kat_names(golden_kat):
        e = golden_kat[f"{name}/edges"]
        gms, mc = golden_kat[f"{name}/params"].tolist()
        r = oracle.run(e, group_max_sz=gms, max_candidates=mc)
        csr = oracle.build_csr(e, max_candidates=mc)
        if csr.truncated_anchors:
            # Where the cap cuts inside a pixel cell the reference keeps the cell's
            # edges in libstdc++'s unstable-sort order and the restatement keeps the
            # lowest indices; every anchor whose list was not cut must still match.
            ref_off, ref_ids = golden_kat[f"{name}/csr_offsets"], golden_kat[f"{name}/csr_ids"]
            assert np.array_equal(csr.offsets, ref_off)
            deg = np.diff(ref_off)
            full = deg < mc
            for a in np.nonzero(full)[0]:
                assert np.array_equal(csr.ids[ref_off[a]:ref_off[a + 1]], ref_ids[ref_off[a]:ref_off[a + 1]])
            continue
        assert np.array_equal(csr.ids, golden_kat[f"{name}/csr_ids"]), name
        assert np.array_equal(csr.dist2.view(np.uint64), golden_kat[f"{name}/csr_dist2"].view(np.uint64)), name
        assert np.array_equal(r.chains, golden_kat[f"{name}/chains"]), name
        assert np.array_equal(r.info.view(np.uint64), golden_kat[f"{name}/info"].view(np.uint64)), name


def test_restatement_pair_bundles_match_reference(oracle, golden_pairs):
    pairs = golden_pairs["pairs"]
    for k, q in enumerate(pairs):
        v, mn, mx = oracle.pair_bundle(q[:3], q[3:])
        assert v == bool(golden_pairs["valid"][k])
        assert np.array_equal(mn.view(np.uint64), golden_pairs["bmin"][k].view(np.uint64))
        assert np.array_equal(mx.view(np.uint64), golden_pairs["bmax"][k].view(np.uint64))


@pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).ref_available()")
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_restatement_matches_live_reference_on_synthetic(oracle, seed):
    e = synth.plain_small(seed)
    r = oracle.ref_run(e, nthreads=4)
    o = oracle.run(e, nthreads=4)
    assert np.array_equal(r.chains, o.chains)
    assert np.array_equal(r.info.view(np.uint64), o.info.view(np.uint64))
    assert (r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors) == \
        (o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors)


@pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).ref_available()")
def test_restatement_matches_live_reference_nondefault_params(oracle):
    e = synth.plain_small(5)[:3000]
    kw = dict(nrad=4.5, dx=0.3, dt_deg=10.0, max_k=0.5, sx=0.15, st=0.05, group_max_sz=6)
    r = oracle.ref_run(e, nthreads=4, **kw)
    o = oracle.run(e, nthreads=4, **kw)
    assert np.array_equal(r.chains, o.chains)
    assert np.array_equal(r.info.view(np.uint64), o.info.view(np.uint64))


def test_float_fixtures_reproduce_with_live_reference(oracle):
    """The --float fixtures are the reference's run_curvelet<float>: where the
    harness is built, running it again gives the same bits (KATs, digit1)."""
    import os
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_files_f32.npz"))
    for name in sorted({k.split("/")[1] for k in z.files if k.startswith("kat/")}):
        gms, mc = z[f"kat/{name}/params"].tolist()
        r = oracle.ref_run(z[f"kat/{name}/edges"], scalar="float", group_max_sz=gms, max_candidates=mc)
        assert np.array_equal(r.chains, z[f"kat/{name}/chains"]), name
        assert np.array_equal(r.info.view(np.uint64), z[f"kat/{name}/info"].view(np.uint64)), name
    r = oracle.ref_run(z["TO_edges_digit1/edges"], scalar="float")
    assert np.array_equal(r.chains, z["TO_edges_digit1/chains"])
    assert np.array_equal(r.info.view(np.uint64), z["TO_edges_digit1/info"].view(np.uint64))


# ---- truncated anchors (max_candidates cuts inside a pixel cell)

def _csr_digest(offsets, ids, dist2=None):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(offsets, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(ids, dtype=np.int32).tobytes())
    if dist2 is not None:
        h.update(np.ascontiguousarray(dist2, dtype=np.float32).tobytes())
    return h.hexdigest()


def test_restatement_truncated_matches_reference_stage(oracle, golden_trunc):
    """On maps where every anchor is truncated, the C restatement equals, bit for
    bit, the reference's own CurveletCPU stage run on the same lowest-index
    neighbour lists (tests/golden/make_golden_truncated.py)."""
    from tests.conftest import truncated_cases
    cases = [c for c, s in truncated_cases(golden_trunc) if s == "double"]
    assert len(cases) == 3
    for case in cases:
        k = f"{case}/double"
        e = golden_trunc[f"{k}/edges"]
        gms, mc = golden_trunc[f"{k}/params"].tolist()
        csr = oracle.build_csr(e, max_candidates=mc)
        assert _csr_digest(csr.offsets, csr.ids) == str(golden_trunc[f"{k}/csr_sha256"]), case
        o = oracle.run(e, group_max_sz=gms, max_candidates=mc)
        assert [o.chains.shape[0], o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors,
                o.truncated_anchors] == golden_trunc[f"{k}/counts"].tolist(), case
        assert np.array_equal(o.chains, golden_trunc[f"{k}/chains"]), case
        assert np.array_equal(o.info.view(np.uint64), golden_trunc[f"{k}/info"].view(np.uint64)), case


def test_float_csr_restatement_pinned(oracle, golden_trunc):
    """oracle.build_csr_f32 (run_curvelet<float>'s neighbour lists) equals the
    reference's own float CSR, distances included, on every map without a
    truncated anchor, and gives the lists the float truncation fixtures used."""
    import os
    from tests.conftest import truncated_cases
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_files_f32.npz"))
    pins = sorted({k.split("/")[1] for k in golden_trunc.files if k.startswith("pin_f32/")})
    assert len(pins) == 9
    for name in pins:
        key = name if name.startswith("TO_edges") else f"kat/{name}"
        mc = int(z[f"{key}/params"][1]) if f"{key}/params" in z.files else 128
        c = oracle.build_csr_f32(z[f"{key}/edges"], max_candidates=mc)
        assert c.truncated_anchors == 0, name
        assert _csr_digest(c.offsets, c.ids, c.dist2) == str(golden_trunc[f"pin_f32/{name}/csr_sha256"]), name
    for case in [c for c, s in truncated_cases(golden_trunc) if s == "float"]:
        k = f"{case}/float"
        mc = int(golden_trunc[f"{k}/params"][1])
        c = oracle.build_csr_f32(golden_trunc[f"{k}/edges"], max_candidates=mc)
        assert c.truncated_anchors == int(golden_trunc[f"{k}/counts"][4]) > 0, case
        assert _csr_digest(c.offsets, c.ids) == str(golden_trunc[f"{k}/csr_sha256"]), case


def test_truncated_fixtures_reproduce_with_live_reference(oracle, golden_trunc):
    """Where the harness is built: the reference stage on the lowest-index lists
    gives the fixtures' bits again, and on the reference's own lists it gives
    what the whole reference run gives (the list override changes nothing else)."""
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    from tests.conftest import truncated_cases
    for case, scalar in truncated_cases(golden_trunc):
        k = f"{case}/{scalar}"
        e = golden_trunc[f"{k}/edges"]
        gms, mc = golden_trunc[f"{k}/params"].tolist()
        c = oracle.build_csr_f32(e, max_candidates=mc) if scalar == "float" else oracle.build_csr(e, max_candidates=mc)
        r = oracle.ref_run_csr(e, c.offsets, c.ids, scalar=scalar, group_max_sz=gms, max_candidates=mc)
        assert np.array_equal(r.chains, golden_trunc[f"{k}/chains"]), k
        assert np.array_equal(r.info.view(np.uint64), golden_trunc[f"{k}/info"].view(np.uint64)), k
        full = oracle.ref_run(e, scalar=scalar, group_max_sz=gms, max_candidates=mc)
        own = oracle.ref_run_csr(e, full.csr.offsets, full.csr.ids, scalar=scalar, group_max_sz=gms,
                                 max_candidates=mc)
        assert np.array_equal(own.chains, full.chains) and own.valid_pairs == full.valid_pairs, k
        assert np.array_equal(own.info.view(np.uint64), full.info.view(np.uint64)), k


def test_reference_stage_rejects_malformed_lists(oracle, golden_trunc):
    """cvlref_run_csr refuses lists that are not a CSR over the map's edges: a
    first offset other than 0, a decreasing offset, an id out of range, a self pair."""
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    e = golden_trunc["blob150/double/edges"]
    c = oracle.build_csr(e)
    bad = []
    off = c.offsets.copy()
    off[0] = 1
    bad.append((off, c.ids))
    off = c.offsets.copy()
    off[5] = off[4] - 1
    bad.append((off, c.ids))
    ids = c.ids.copy()
    ids[3] = e.shape[0]
    bad.append((c.offsets, ids))
    ids = c.ids.copy()
    ids[c.offsets[7]] = 7
    bad.append((c.offsets, ids))
    for o, i in bad:
        with pytest.raises(ValueError):
            oracle.ref_run_csr(e, o, i)
    # and the untouched lists run
    assert oracle.ref_run_csr(e, c.offsets, c.ids).chains.shape[0] == int(golden_trunc["blob150/double/counts"][0])
