"""neat_create_samples_noalloc: the sampler for callers that cannot allocate.

Some callers of the sampler cannot hand the library a workspace: a host
framework that has reserved the GPU's memory for its own pool, a loop that
must not stall on the device synchronisation a cudaMalloc costs, or a binding
that only passes input and output arrays.  For them the library keeps the
sampler's per-ray scratch in one static device array (at most
NEAT_NOALLOC_MAX_RAYS rays).  These tests call it through the C ABI and check
its SampleList against the workspace entry point, bit for bit, on two calls in
a row whose second batch is smaller than the first (a stale first call would
show), and that an oversize batch is refused before any kernel launch, with
its count zeroed.

Collected last (file name) so a failure here cannot hide the other tests.
"""
import numpy as np
import pytest
import torch

from tests.cases import cfg1_case

pytestmark = pytest.mark.gpu

FIELDS = ("coords", "ray_t", "weight", "ray_index", "local_index", "node_id")


def _buffers(cap):
    return dict(coords=torch.empty((cap, 3), device="cuda"), ray_t=torch.empty(cap, device="cuda"),
                weight=torch.empty(cap, device="cuda"), ray_index=torch.empty(cap, dtype=torch.int64, device="cuda"),
                local_index=torch.empty(cap, dtype=torch.int64, device="cuda"),
                node_id=torch.empty(cap, dtype=torch.int64, device="cuda"))


def _run(neat, fn_name, case, origin, direction, seed, step, cap):
    t = case.tree.device_tables("cuda")
    R = origin.shape[0]
    b = _buffers(cap)
    cnt = torch.full((2,), -1, dtype=torch.int64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    args = [t["table"].data_ptr(), case.A, case.tree.max_depth, origin.data_ptr(), direction.data_ptr(), R, case.M,
            1, seed, step, cap] + [b[k].data_ptr() for k in FIELDS] + [cnt.data_ptr(), st.data_ptr()]
    if fn_name == "neat_create_samples":
        ws = torch.empty(max(neat.neat_samples_workspace_bytes(R), 16), dtype=torch.uint8, device="cuda")
        args.append(ws.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream
    rc = getattr(neat, fn_name)(*args, stream)
    torch.cuda.synchronize()
    assert rc == 0, fn_name
    assert int(st.item()) == 0, fn_name
    S = int(cnt[0])
    return S, int(cnt[1]), {k: v[:S].cpu().numpy() for k, v in b.items()}


def test_noalloc_matches_workspace_entry_point_two_calls(neat, oracle):
    from neat_b200.api import CameraModel, GetRays
    case = cfg1_case(R=4096, oracle=oracle)
    rays = GetRays(CameraModel(case.w, case.h, case.intr, case.rot, case.trans),
                   torch.from_numpy(case.uv).cuda(), torch.from_numpy(case.img).cuda())
    cap = 4096 * 64
    # first call: the whole batch; second call: a smaller batch, new seed/step
    for R, seed, step in ((4096, 21, 1), (1500, 22, 2)):
        o = rays.origin[:R].contiguous()
        d = rays.direction[:R].contiguous()
        S_ref, mx_ref, ref = _run(neat, "neat_create_samples", case, o, d, seed, step, cap)
        S, mx, out = _run(neat, "neat_create_samples_noalloc", case, o, d, seed, step, cap)
        assert S == S_ref > 0 and mx == mx_ref
        for k in FIELDS:  # integer/ordering work and identical arithmetic: bit-exact
            np.testing.assert_array_equal(out[k], ref[k], err_msg=k)


def test_noalloc_rejects_batches_beyond_its_array(neat):
    from neat_b200 import _lib
    R = _lib.NEAT_NOALLOC_MAX_RAYS + 1
    cnt = torch.full((2,), -1, dtype=torch.int64, device="cuda")
    rc = neat.neat_create_samples_noalloc(None, 0, 2, None, None, R, 16, 0, 0, 1, 0, None, None, None, None, None,
                                          None, cnt.data_ptr(), None, None)
    torch.cuda.synchronize()
    assert rc == _lib.NEAT_ERR_CAPACITY
    # the count is zeroed before the refusal, so a caller that skips rc reads 0
    assert cnt.tolist() == [0, 0]
