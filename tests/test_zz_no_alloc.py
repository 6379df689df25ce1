"""sc_sample_static: sampling for callers that cannot allocate device memory.

Frameworks that own all device memory through their own pool, and serving loops
that forbid allocation after start-up, hold the state in their own device memory;
sc_sample_static samples it into their device buffer using a fixed scratch array
inside the library.  Checked through the C ABI against the context sampler
(sc_sample) on the same state and uniforms: outcomes are integers and must be
identical, on two calls in a row.  This file is collected last so a failure here
cannot hide the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

import randcirc as RCirc
from statecraft_b200 import _abi as A
from statecraft_b200.engine import B200Config, NativeContext, serialize_circuit

pytestmark = pytest.mark.gpu


def _device_state(ctx, n, dtype):
    import torch

    host = ctx.state(n)  # interleaved doubles
    t = torch.from_numpy(host).to("cuda")
    if dtype == A.SC_C64:
        t = t.to(torch.float32)
    return t.contiguous()


@pytest.mark.parametrize("dtype", [A.SC_C128, A.SC_C64])
def test_static_sampler_matches_context_sampler(dtype):
    import torch

    n, shots = 14, 4096
    ctx = NativeContext(B200Config(dtype=dtype))
    c = RCirc.random_circuit(n, 60, seed=99)
    ctx.run_ops(n, *serialize_circuit(c))
    qubits = list(range(n))
    rng = np.random.default_rng(7)
    u = rng.random(shots)
    want_u = ctx.sample(qubits, shots, None, u)
    want_seeded = ctx.sample(qubits, shots, 1234)

    state = _device_state(ctx, n, dtype)
    d_u = torch.from_numpy(u).to("cuda")
    d_out = torch.empty(shots, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = A.load()
    for _ in range(2):
        d_out.fill_(-1)
        rc = lib.sc_sample_static(ctypes.c_void_p(state.data_ptr()), n, dtype, shots, 0,
                                  ctypes.c_void_p(d_u.data_ptr()),
                                  ctypes.c_void_p(d_out.data_ptr()), stream)
        A.raise_for(rc, lib)
        np.testing.assert_array_equal(d_out.cpu().numpy(), want_u)
    for _ in range(2):
        d_out.fill_(-1)
        rc = lib.sc_sample_static(ctypes.c_void_p(state.data_ptr()), n, dtype, shots, 1234, None,
                                  ctypes.c_void_p(d_out.data_ptr()), stream)
        A.raise_for(rc, lib)
        np.testing.assert_array_equal(d_out.cpu().numpy(), want_seeded)
    ctx.close()


def test_static_sampler_rejects_oversized_state():
    lib = A.load()
    # 31 qubits is one past the scratch size; 64 and 200 would overflow a shift
    for n in (31, 64, 200):
        rc = lib.sc_sample_static(ctypes.c_void_p(16), n, A.SC_C128, 8, 1, None,
                                  ctypes.c_void_p(16), None)
        assert rc == A.SC_EINVAL
        assert b"2^30" in lib.sc_last_error()


def test_static_sampler_refuses_capturing_stream():
    """A call on a stream that is recording a CUDA graph returns SC_EINVAL and
    enqueues nothing: it would end by waiting for the stream, which a capturing
    stream does not allow.  The caller's capture stays valid and replays."""
    import torch

    lib = A.load()
    n, shots = 10, 8
    state = torch.zeros(2 << n, dtype=torch.float64, device="cuda")
    state[0] = 1.0
    d_out = torch.full((shots,), -1, dtype=torch.int32, device="cuda")
    x = torch.zeros(4, device="cuda")
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        g.capture_begin()
        x.add_(1)
        rc = lib.sc_sample_static(ctypes.c_void_p(state.data_ptr()), n, A.SC_C128, shots, 3, None,
                                  ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(s.cuda_stream))
        x.add_(1)
        g.capture_end()
    assert rc == A.SC_EINVAL
    assert b"capturing" in lib.sc_last_error()
    g.replay()
    torch.cuda.synchronize()
    assert x.tolist() == [2.0] * 4
    assert d_out.tolist() == [-1] * shots
    # the same buffers sample normally once the capture is over
    rc = lib.sc_sample_static(ctypes.c_void_p(state.data_ptr()), n, A.SC_C128, shots, 3, None,
                              ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(s.cuda_stream))
    A.raise_for(rc, lib)
    assert d_out.tolist() == [0] * shots
