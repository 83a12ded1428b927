"""The allocation-free entry point against the regular one (needs a GPU).

gpz_compress_member_static is for callers that cannot allocate GPU memory
while they compress; it keeps all working memory in one fixed device array
inside the library.  Its output must be byte-identical to gpz_compress_chunk
on the same input (integer path: no tolerance), call after call: the array
keeps the previous call's contents, so consecutive calls with different
sizes also check that nothing stale leaks into the next result.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_member_matches_regular_path():
    import torch

    from gpzip_b200 import native
    from gpzip_b200 import workloads as W

    L = native.load()
    ctx = native.Context()
    inputs = [
        W.text(131072, seed=31).tobytes(),              # full member
        W.binary(70001, seed=32).tobytes(),             # smaller, after a larger call
        b"",                                            # empty member
        W.logs(90000, seed=33).tobytes(),
    ]
    for data in inputs:
        want = ctx.compress_chunk(data)
        host = np.frombuffer(b"\0" + data, dtype=np.uint8)
        d_buf = torch.from_numpy(host.copy()).cuda()
        d_in = d_buf[1:]  # deliberately unaligned device input
        cap = L.gpz_bound(len(data))
        d_out = torch.zeros(cap + 1, dtype=torch.uint8, device="cuda")[1:]
        n = ctypes.c_size_t()
        torch.cuda.synchronize()
        rc = L.gpz_compress_member_static(ctypes.c_void_p(d_in.data_ptr()), len(data),
                                          ctypes.c_void_p(d_out.data_ptr()), cap, ctypes.byref(n), None)
        assert rc == native.GPZ_OK, native.STATUS.get(rc, rc)
        got = d_out[:n.value].cpu().numpy().tobytes()
        assert got == want
    ctx.close()


def test_static_member_rejects_oversize_and_short_output():
    import torch

    from gpzip_b200 import native

    L = native.load()
    d_in = torch.zeros(131073, dtype=torch.uint8, device="cuda")
    d_out = torch.zeros(L.gpz_bound(131073), dtype=torch.uint8, device="cuda")
    n = ctypes.c_size_t()
    rc = L.gpz_compress_member_static(ctypes.c_void_p(d_in.data_ptr()), 131073, ctypes.c_void_p(d_out.data_ptr()),
                                      d_out.numel(), ctypes.byref(n), None)
    assert rc == 5  # GPZ_E_ARG: above GPZ_STATIC_MAX_BYTES
    rc = L.gpz_compress_member_static(ctypes.c_void_p(d_in.data_ptr()), 4096, ctypes.c_void_p(d_out.data_ptr()),
                                      8, ctypes.byref(n), None)
    assert rc == 6  # GPZ_E_SPACE
