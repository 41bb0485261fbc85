"""Helpers of the GPU tests: run the device step through the C ABI on packed states."""

import numpy as np


def run_device(torch, tissue, state, control, dt, n_steps, *, chunks=None):
    """Advance a host state dict n_steps on the device (cb_step), optionally in several launches
    (chunks = list of step counts). Returns (state dict, status[W], accepted[W] of the last call)."""
    dev = torch.device("cuda", tissue.device)
    src = torch.from_numpy(tissue.pack_state(state)).to(dev)
    dst = torch.empty_like(src)
    ctl = torch.from_numpy(np.asarray(control, dtype=np.float64)).to(dev)
    status = torch.zeros(tissue.batch.worlds, dtype=torch.int32, device=dev)
    taken = torch.zeros(tissue.batch.worlds, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    plan = [n_steps] if chunks is None else list(chunks)
    assert sum(plan) == n_steps
    for k in plan:
        tissue.step(src, dst, ctl, dt, k, status, taken, stream=stream)
        src, dst = dst, src
    torch.cuda.synchronize(dev)
    return tissue.unpack_state(src.cpu().numpy()), status.cpu().numpy(), taken.cpu().numpy()


def oracle_state(st):
    return {f: np.asarray(getattr(st, f)) for f in st._fields}
