"""The allocation-free norms entry point against the workspace one.

``cvfes_solid_norms_noalloc_f32`` serves callers that cannot give the library a
device workspace and must not make it allocate (a watchdog between steps of an
ensemble that fills the GPU, or a framework whose pool owns all device memory).
It keeps its partial sums in a fixed device array instead; this file checks,
through the C ABI, that it returns what ``cvfes_solid_norms_f32`` returns, call
after call, and that it refuses sizes beyond its fixed array.  It is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from cvfes_b200 import _lib

pytestmark = pytest.mark.gpu
RTOL = 1e-12  # FP64 sums of the same values in a different chunk order


def _state(dev, n_nodes, S, seed, nan_at=None):
    g = torch.Generator(device="cpu").manual_seed(seed)
    u = torch.randn((3 * n_nodes, S), generator=g, dtype=torch.float32)
    up = u + 1e-3 * torch.randn((3 * n_nodes, S), generator=g, dtype=torch.float32)
    invm = torch.rand((n_nodes, S), generator=g, dtype=torch.float32) + 0.5
    invm[:7] = 0.0  # zero-mass rows count as m = 0
    if nan_at is not None:
        u[nan_at] = float("nan")
    return u.to(dev), up.to(dev), invm.to(dev)


def _norms_workspace(lib, u, up, invm, S, n_nodes, stream):
    work = torch.empty(int(lib.cvfes_norms_work_size(n_nodes, S)), dtype=torch.float64,
                       device=u.device)
    out = torch.empty((S, 4), dtype=torch.float64, device=u.device)
    rc = lib.cvfes_solid_norms_f32(n_nodes, S, u.data_ptr(), up.data_ptr(), invm.data_ptr(),
                                   work.data_ptr(), out.data_ptr(), 0, stream)
    assert rc == 0, _lib.last_error()
    return out.cpu().numpy()


def _norms_fixed(lib, u, up, invm, S, n_nodes, stream, check=0):
    out = torch.full((S, 4), -1.0, dtype=torch.float64, device=u.device)
    rc = lib.cvfes_solid_norms_noalloc_f32(n_nodes, S, u.data_ptr(), up.data_ptr(),
                                           invm.data_ptr(), out.data_ptr(), check, stream)
    return rc, out.cpu().numpy()


def test_fixed_scratch_norms_match_workspace_norms():
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # two sizes: the second needs fewer, longer chunks to fit the fixed array
    for n_nodes, S in ((5000, 64), (70000, 512)):
        for call, nan_at in enumerate((None, (3 * 1234 + 1, 5), None)):
            u, up, invm = _state(dev, n_nodes, S, seed=10 * S + call, nan_at=nan_at)
            ref = _norms_workspace(lib, u, up, invm, S, n_nodes, stream)
            rc, got = _norms_fixed(lib, u, up, invm, S, n_nodes, stream)
            assert rc == 0, _lib.last_error()
            np.testing.assert_allclose(got, ref, rtol=RTOL, atol=0, equal_nan=True)
            # the non-finite count restarts from zero on every call
            assert got[:, 3].sum() == (1 if nan_at is not None else 0)
        # the watchdog form reports the NaN it is shown
        u, up, invm = _state(dev, n_nodes, S, seed=7, nan_at=(11, 0))
        rc, _ = _norms_fixed(lib, u, up, invm, S, n_nodes, stream, check=1)
        assert rc == _lib.CVFES_ERR_NONFINITE


def test_fixed_scratch_rejects_oversized_requests():
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    S = 131072  # one more sample than the fixed array holds
    x = torch.zeros(4, dtype=torch.float32, device=dev)
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    rc = lib.cvfes_solid_norms_noalloc_f32(1, S, x.data_ptr(), x.data_ptr(), x.data_ptr(),
                                           out.data_ptr(), 0, None)
    assert rc == _lib.CVFES_ERR_ARG
    assert "at most 131071 samples" in _lib.last_error()
