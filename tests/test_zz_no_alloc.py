"""The allocation-free probe generator (slq_generate_probes_noalloc).

It serves callers that cannot allocate device memory -- code whose device
memory belongs entirely to a caching allocator or a fixed arena, and paths
that must not take the synchronisation cudaFree can cause -- by keeping its
scratch in a fixed array inside the library.  Its output must equal the
workspace-based slq_generate_probes bit for bit (probes are +-1 integers),
on two calls in a row, whether this file runs alone in a fresh process or
after the rest of the suite.  Collected last on purpose (file name)."""

import ctypes

import numpy as np
import pytest

from imate_b200 import _lib

pytestmark = pytest.mark.gpu

CASES = [
    # (seed, rng, len, first, count, width, dtype)
    (3, 0, 1000, 0, 8, 8, _lib.SLQ_F64),
    (7, 0, 70001, 5, 50, 64, _lib.SLQ_F32),
    (1, 0, 65, 2, 1, 1, _lib.SLQ_F32),
    (11, 1, 4097, 3, 200, 256, _lib.SLQ_F32),
    (0, 0, 262144, 0, 256, 256, _lib.SLQ_F32),
    # 531,251 words per probe: more than the fixed scratch's 8192 chunks of
    # 64 words, so this call takes 128-word chunks where the workspace path
    # keeps 64 (136 MB of output)
    (5, 0, 34_000_000, 1, 1, 1, _lib.SLQ_F32),
]


def _with_workspace(lib, seed, rng, n, first, count, width, dtype):
    import torch
    tdt = torch.float64 if dtype == _lib.SLQ_F64 else torch.float32
    out = torch.full((n, width), 5.0, dtype=tdt, device="cuda")
    nb = ctypes.c_size_t(0)
    _lib.check(lib.slq_generate_probes_workspace_bytes(n, width,
                                                       ctypes.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    _lib.check(lib.slq_generate_probes(
        seed, rng, n, first, count, width, dtype, out.data_ptr(),
        ws.data_ptr(), ws.numel(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _without_workspace(lib, seed, rng, n, first, count, width, dtype):
    import torch
    tdt = torch.float64 if dtype == _lib.SLQ_F64 else torch.float32
    out = torch.full((n, width), -5.0, dtype=tdt, device="cuda")
    _lib.check(lib.slq_generate_probes_noalloc(
        seed, rng, n, first, count, width, dtype, out.data_ptr(),
        torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_probes_equal_workspace_probes_twice(cuda):
    for case in CASES:
        want = _with_workspace(cuda, *case)
        first_call = _without_workspace(cuda, *case)
        second_call = _without_workspace(cuda, *case)
        assert np.array_equal(first_call, want), case
        assert np.array_equal(second_call, want), case


def test_noalloc_rejects_width_beyond_its_scratch(cuda):
    import torch
    out = torch.empty((64, 2048), dtype=torch.float32, device="cuda")
    st = cuda.slq_generate_probes_noalloc(
        0, 0, 64, 0, 2048, 2048, _lib.SLQ_F32, out.data_ptr(),
        torch.cuda.current_stream().cuda_stream)
    assert st == 1  # SLQ_ERR_BAD_ARG
    assert b"1024" in cuda.slq_last_error()


def test_noalloc_calls_leave_device_free_memory_unchanged(cuda):
    """The point of this entry point: after a first call on the device has
    resolved the scratch array's address and loaded the kernels, further
    calls take no device memory (free bytes before and after are equal)."""
    import torch
    seed, rng, n, first, count, width, dtype = 7, 0, 70001, 5, 50, 64, \
        _lib.SLQ_F32
    out = torch.empty((n, width), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for r in (0, 1):  # warm-up: both probe streams' kernels loaded
        _lib.check(cuda.slq_generate_probes_noalloc(
            seed, r, n, first, count, width, dtype, out.data_ptr(), stream))
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for r in (0, 1, 0, 1):
        _lib.check(cuda.slq_generate_probes_noalloc(
            seed, r, n, first, count, width, dtype, out.data_ptr(), stream))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_parity_mode_refuses_a_capturing_stream(cuda):
    """Parity mode copies its scratch from host staging and waits for the
    copies; on a stream that is being captured it must return
    SLQ_ERR_BAD_ARG without touching the stream, so the caller's capture
    stays valid, and the next ordinary call still gives the right probes."""
    import torch
    case = (3, 0, 1000, 0, 8, 8, _lib.SLQ_F32)
    want = _with_workspace(cuda, *case)
    out = torch.zeros((1000, 8), dtype=torch.float32, device="cuda")
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        st = cuda.slq_generate_probes_noalloc(
            3, 0, 1000, 0, 8, 8, _lib.SLQ_F32, out.data_ptr(),
            side.cuda_stream)
        msg = cuda.slq_last_error()
        out.add_(1.0)  # the capture itself stays usable
    del graph
    torch.cuda.synchronize()
    assert st == 1  # SLQ_ERR_BAD_ARG
    assert b"capture" in msg
    assert np.array_equal(_without_workspace(cuda, *case), want)
