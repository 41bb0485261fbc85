"""cb_step_packed_static: the packed FP64 ARS(2,2,2) step with its scratch in the library's own
static device array, for callers that may not allocate device memory while a step runs (a plugin
that its host runtime hands only input and output buffers, such as an XLA/JAX custom call, or a
process whose device memory another allocator already holds).

Checked through the C ABI against cb_step on the same handle, inputs and controls, twice in a
row (the array keeps the first call's contents; the second call must not depend on them), with
the parity tolerance of the other device tests (1e-10 scaled difference per field), and the same
call captured into a CUDA graph and replayed twice. This file is collected last and must pass
alone in a fresh process as well as after the other tests.
"""

import ctypes

import numpy as np
import pytest

from cells_b200 import worlds
from conftest import scaled_difference

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _ptr(tensor):
    return ctypes.c_void_p(tensor.data_ptr())


@pytest.fixture
def bound(cuda, monkeypatch):
    """A small uneven batch (channels, several worlds per work item) bound for the packed kernel."""
    from cells_b200.tissue import Tissue

    monkeypatch.setenv("CELLS_B200_KERNEL", "packed")
    rng = np.random.default_rng(44)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(44, k),
                                                     junction_sigma=0.3), rng,
                               na=("nav", 3e-10, 0.5), k=("hh", 6e-10, 0.5), sigma=0.3)
          for k, n in enumerate((600, 48, 200, 35, 1100, 90))]
    tissue = Tissue(worlds.pack(ws))
    yield tissue
    tissue.close()


def test_static_scratch_step_matches_cb_step_on_two_calls(cuda, bound):
    from cells_b200 import _lib

    torch, tissue, lib = cuda, bound, bound.lib
    dev = torch.device("cuda", tissue.device)
    b = tissue.batch
    rng = np.random.default_rng(7)
    start = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control(
        rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges), rng.uniform(0.6, 1, b.cells),
        rng.uniform(0.4, 1, (2, b.cells)))).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    reference_state = start.clone()
    static_state = start.clone()
    for call in range(2):  # two calls in a row: the second starts where the first ended
        ref_out = torch.empty_like(start)
        st_out = torch.empty_like(start)
        ref_status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
        st_status = torch.full((b.worlds,), 99, dtype=torch.int32, device=dev)
        st_taken = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
        _lib.check(lib.cb_step(tissue.handle, _lib.METHOD_ARS222, _ptr(reference_state),
                               _ptr(ref_out), 1e-3, _ptr(control), 40, _ptr(ref_status), None,
                               ctypes.c_void_p(stream)))
        _lib.check(lib.cb_step_packed_static(tissue.handle, _ptr(static_state), _ptr(st_out),
                                             1e-3, _ptr(control), 40, _ptr(st_status),
                                             _ptr(st_taken), ctypes.c_void_p(stream)))
        torch.cuda.synchronize(dev)
        assert int(ref_status.abs().max()) == 0
        assert int(st_status.abs().max()) == 0, f"call {call}: a world was refused"
        assert int(st_taken.min()) == 40
        ref = tissue.unpack_state(ref_out.cpu().numpy())
        got = tissue.unpack_state(st_out.cpu().numpy())
        for f in ref:
            assert scaled_difference(got[f], ref[f]) <= TOL, (call, f)
        reference_state, static_state = ref_out, st_out


def test_static_scratch_refuses_a_batch_beyond_its_size(cuda, monkeypatch):
    """A batch whose scratch exceeds the static array is refused with a clear error."""
    from cells_b200 import _lib
    from cells_b200.tissue import Tissue

    monkeypatch.setenv("CELLS_B200_KERNEL", "packed")
    big = Tissue(worlds.pack(worlds.grid_tissues(200, side=16, seed=3)))  # 51,200 cells
    torch = cuda
    dev = torch.device("cuda", big.device)
    state = torch.from_numpy(big.pack_state(big.initial_state())).to(dev)
    control = torch.from_numpy(big.pack_control()).to(dev)
    status = torch.zeros(big.batch.worlds, dtype=torch.int32, device=dev)
    rc = big.lib.cb_step_packed_static(big.handle, _ptr(state), _ptr(state), 1e-3,
                                       _ptr(control), 1, _ptr(status), None, None)
    assert rc == 4  # CB_ERR_UNSUPPORTED
    assert "static scratch" in big.lib.cb_last_error().decode()
    big.close()
    del _lib


def test_static_scratch_step_replays_from_a_cuda_graph(cuda, bound):
    """The case the entry point exists for: the call captured into a CUDA graph (a memset of the
    ticket counter and one launch, nothing allocated), replayed twice in a row with the state
    carried between replays, matches cb_step over the same 80 steps."""
    from cells_b200 import _lib

    torch, tissue, lib = cuda, bound, bound.lib
    dev = torch.device("cuda", tissue.device)
    b = tissue.batch
    rng = np.random.default_rng(8)
    start = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control(
        rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges), rng.uniform(0.6, 1, b.cells),
        rng.uniform(0.4, 1, (2, b.cells)))).to(dev)
    graph_in = start.clone()
    graph_out = torch.empty_like(start)
    status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
    taken = torch.zeros(b.worlds, dtype=torch.int32, device=dev)

    def call(stream):
        return lib.cb_step_packed_static(tissue.handle, _ptr(graph_in), _ptr(graph_out), 1e-3,
                                         _ptr(control), 40, _ptr(status), _ptr(taken),
                                         ctypes.c_void_p(stream.cuda_stream))

    side = torch.cuda.Stream(dev)  # warm-up off the capture, so the kernel is loaded before it
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        _lib.check(call(side))
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize(dev)

    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        rc = call(torch.cuda.current_stream(dev))
    _lib.check(rc)

    reference = start.clone()
    for replay in range(2):
        ref_out = torch.empty_like(start)
        ref_status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
        _lib.check(lib.cb_step(tissue.handle, _lib.METHOD_ARS222, _ptr(reference), _ptr(ref_out),
                               1e-3, _ptr(control), 40, _ptr(ref_status), None,
                               ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
        graph_in.copy_(start if replay == 0 else graph_out)
        status.fill_(99)
        taken.zero_()
        graph.replay()
        torch.cuda.synchronize(dev)
        assert int(ref_status.abs().max()) == 0
        assert int(status.abs().max()) == 0, f"replay {replay}: a world was refused"
        assert int(taken.min()) == 40
        ref = tissue.unpack_state(ref_out.cpu().numpy())
        got = tissue.unpack_state(graph_out.cpu().numpy())
        for f in ref:
            assert scaled_difference(got[f], ref[f]) <= TOL, (replay, f)
        reference = ref_out
    del graph
