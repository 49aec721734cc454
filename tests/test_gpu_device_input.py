"""cvl_run_device: edges that stay in device memory (written there by a producer
on the same GPU, handed over with an event) give exactly cvl_run's results, and
the outputs can stay on the device for a consumer there."""
import numpy as np
import pytest
import torch

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth

pytestmark = pytest.mark.gpu


class _DevArray:
    """A device buffer seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def _same(a, b):
    return (np.array_equal(a.chains, b.chains) and np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))
            and (a.valid_pairs, a.total_neighbor_pairs, a.max_num_of_neighbors) ==
            (b.valid_pairs, b.total_neighbor_pairs, b.max_num_of_neighbors))


def test_device_edges_with_producer_event(engine):
    e = synth.plain_hd(1000)
    ref = engine.run(e)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):  # the "producer": writes the edges on its own stream
        d = torch.empty(e.shape, dtype=torch.float64, device="cuda")
        d.copy_(torch.from_numpy(e).pin_memory(), non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(side)
    r = engine.run_device(d.data_ptr(), e.shape[0], e.shape[1], ready_event=ev.cuda_event)
    assert _same(r, ref)
    # a wider edge row (edge_data_sz 6) read in place
    e6 = np.column_stack([e, np.zeros((e.shape[0], 2))])
    d6 = torch.from_numpy(e6).cuda()
    torch.cuda.synchronize()
    assert _same(engine.run_device(d6.data_ptr(), e.shape[0], 6, cvl.CurveletParams(edge_data_sz=6)), ref)


def test_device_resident_outputs(engine):
    e = synth.plain_small(4)
    ref = engine.run(e)
    d = torch.from_numpy(e).cuda()
    torch.cuda.synchronize()
    assert engine.run_device(d.data_ptr(), e.shape[0], 4, to_host=False) is None
    v = engine.device_results()
    assert v["num_curvelets"] == ref.num_curvelets and v["chain_width"] == ref.chains.shape[1]
    torch.cuda.synchronize()  # the outputs' done_event has passed
    n = v["num_curvelets"] * v["chain_width"]
    chains = torch.as_tensor(_DevArray(v["chains"], n, "<i4"), device="cuda").cpu().numpy().view(np.uint32)
    info = torch.as_tensor(_DevArray(v["info"], v["num_curvelets"] * 10, "<f8"), device="cuda").cpu().numpy()
    assert np.array_equal(chains.reshape(ref.chains.shape), ref.chains)
    assert np.array_equal(info.reshape(ref.info.shape).view(np.uint64), ref.info.view(np.uint64))
    engine.run(e)  # another run: the device outputs are gone
    with pytest.raises(cvl.CvlError):
        engine.device_results()


def test_device_input_rejects_host_memory(engine):
    e = np.ascontiguousarray(synth.plain_small(1))
    with pytest.raises(cvl.CvlError):
        engine.run_device(e.ctypes.data, e.shape[0], 4)
    with pytest.raises(cvl.CvlError):
        engine.run_device(0, 10, 4)
