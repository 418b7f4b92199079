"""qs_invert_batched_noalloc: the batched Dyson inversion for callers that cannot allocate
GPU memory (an enclosing application owns all of it, or the loop cannot take cudaMalloc's
synchronisation). The caller's device buffers are passed through the C ABI; the result
must equal the allocating entry point's (qs_invert_batched) within the FP64 tolerance of
the other inversion tests (1e-13 relative), on two calls in a row (the fixed scratch array
keeps the previous call's contents). This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import quichotte_b200 as qb

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def run_noalloc(torch, A):
    """A: (batch, N, N) host complex; returns (inverses, info) from the no-alloc entry point."""
    batch, N, _ = A.shape
    cm = np.ascontiguousarray(A.transpose(0, 2, 1))  # column-major matrices
    dA = torch.from_numpy(cm.view(np.float64).copy()).cuda()
    dinfo = torch.full((batch,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    rc = qb._lib.qs_invert_batched_noalloc(N, batch, ctypes.c_void_p(dA.data_ptr()),
                                           ctypes.c_void_p(dinfo.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0
    torch.cuda.synchronize()
    inv = dA.cpu().numpy().view(np.complex128).reshape(batch, N, N).transpose(0, 2, 1)
    return inv, dinfo.cpu().numpy()


@pytest.mark.parametrize("N", [6, 120, 200])
def test_noalloc_matches_allocating_entry_point_twice(N):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(100 + N)
    for call in range(2):  # two calls in a row reuse the same scratch
        batch = 41 + call
        A = rng.standard_normal((batch, N, N)) + 1j * rng.standard_normal((batch, N, N)) + 3 * np.sqrt(N) * np.eye(N)
        ref, info_ref = qb.invert_batched(A)
        got, info = run_noalloc(torch, A)
        assert not info.any() and not info_ref.any()
        assert rel(got, ref) < 1e-13


def test_noalloc_reports_zero_pivot_and_rejects_oversize():
    torch = pytest.importorskip("torch")
    A = np.tile(np.eye(6, dtype=np.complex128), (3, 1, 1))
    A[1, 3, :] = 0.0
    got, info = run_noalloc(torch, A)
    _, info_ref = qb.invert_batched(A)
    assert list(info) == list(info_ref) == [0, 4, 0]
    assert np.allclose(got[0], np.eye(6))
    rc = qb._lib.qs_invert_batched_noalloc(513, 1, None, None, None)
    assert rc == qb.QS_ERR_NOALLOC_LIMIT
