"""Failure paths under host-side allocation failures (cvl_debug_fail_allocations).

The injector fails the library's own device and page-locked allocations on the
host, as if the memory were exhausted: nothing on the GPU faults or waits. Each
test checks that the call that needed the memory returns CVL_ENOMEM with a
message, that nothing is left half done, and that the same engine or server
works again, with the same results, once memory is available."""
import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import _abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture
def injector():
    lib = _abi.load()
    yield lib.cvl_debug_fail_allocations
    lib.cvl_debug_fail_allocations(-1)


def _same(a, b):
    assert np.array_equal(a.chains, b.chains)
    assert np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))


def test_engine_run_fails_cleanly_and_recovers(engine, injector):
    small, big = synth.plain_small(1), synth.plain_hd(1000)
    ref = engine.run(big)
    with cvl.Engine() as eng:
        eng.run(small)                 # a workspace for the small map
        assert injector(0) == 0        # from now on every allocation fails
        with pytest.raises(cvl.CvlError) as ei:
            eng.run(big)               # needs a larger workspace
        assert ei.value.code == _abi.CVL_ENOMEM
        assert "allocation" in str(ei.value)
        injector(-1)
        _same(eng.run(small), engine.run(small))  # the same engine runs again
        _same(eng.run(big), ref)                  # and grows once memory is back


def test_engine_fails_after_some_allocations(engine, injector):
    """The k-th allocation of a first run fails, for several k: each run fails with
    CVL_ENOMEM and the engine then gives the right result."""
    e = synth.plain_small(2)
    ref = engine.run(e)
    for k in (0, 3, 11, 25):
        with cvl.Engine() as eng:
            injector(k)
            with pytest.raises(cvl.CvlError) as ei:
                eng.run(e)
            assert ei.value.code == _abi.CVL_ENOMEM, k
            injector(-1)
            _same(eng.run(e), ref)


def test_server_create_and_submit_fail_cleanly(injector):
    injector(0)
    with pytest.raises(cvl.CvlError) as ei:
        cvl.Server(workers=2)          # its workspace reservation fails
    assert ei.value.code == _abi.CVL_ENOMEM
    injector(-1)
    # no page-locked staging set aside: the first submit must pin memory
    with cvl.Server(workers=2, host_reserve_bytes=0, max_map_edges=1 << 20, max_batch_edges=1 << 18) as srv:
        injector(0)
        with pytest.raises(cvl.CvlError) as ei:
            srv.submit(synth.plain_small(4))
        assert ei.value.code == _abi.CVL_ENOMEM
        injector(-1)
        m = synth.plain_small(4)
        rid = srv.submit(m)
        got = srv.wait(rid, timeout_s=120.0)
        st = srv.stats()
    assert st["completed"] == 1 and st["failed"] == 0
    with cvl.Engine() as eng:
        _same(got, eng.run(m))
