"""mset_batch_gradient_noalloc: the allocation-free batched pass for callers
that cannot allocate device memory (work issued during CUDA graph capture,
device memory owned by a framework allocator or MATLAB gpuArrays, real-time
pipelines).  Called through the C ABI with caller-owned device buffers, twice
in a row (the shared scratch keeps the previous call's contents, so the
second call checks that everything that must start at zero is cleared), and
compared with mset_batch_gradient on the same inputs at the parity tolerance
of the other GPU tests (relative L2 <= 1e-4).

Kept in a file that pytest collects last, so a run that stops at the first
failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest

from mset_b200 import MSET_ADJOINT_EXACT, MSET_ADJOINT_REF, MSET_MODE_MSET, MSET_MODE_SSET, load
from mset_b200._lib import check
from mset_b200.batch import BatchSession
from tests.helpers import rel_l2, small_case

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,nz,b,method,adjoint", [
    (64, 6, 2, MSET_MODE_MSET, MSET_ADJOINT_REF),
    (128, 5, 1, MSET_MODE_MSET, MSET_ADJOINT_EXACT),
    (24, 4, 1, MSET_MODE_SSET, MSET_ADJOINT_REF),
])
def test_noalloc_matches_batch_gradient(gpu_available, n, nz, b, method, adjoint):
    import torch

    npos = 6
    c = small_case(n=n, nz=nz, npos=npos, b=b, seed=40 + n, defocus=15.0, jitter=6.0, strength=20.0)
    ns = 1 if method == MSET_MODE_SSET else -(-nz // b)

    # existing entry point
    bs = BatchSession(n=n, nz=nz, npos=[npos], prop=c["prop"], sigma=c["sigma"], potential_pixelsize=c["dz"],
                      slice_binning=b, method=method, adjoint=adjoint)
    bs.set_tilt(0, probe=c["probe"], scan_x=c["sx"], scan_y=c["sy"], measured=c["meas"], volume=c["V"])
    ref = bs.gradient()
    bs.close()

    # caller-owned device buffers
    V = _dev(c["V"], torch)
    pr = _dev(c["probe"].view(np.float32).reshape(n, n, 2), torch)
    pp = _dev(c["prop"].view(np.float32).reshape(n, n, 2), torch)
    sx, sy = _dev(c["sx"], torch), _dev(c["sy"], torch)
    me = _dev(c["meas"], torch)
    lib = load()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        g = torch.full((ns, n, n), float("nan"), dtype=torch.float64, device="cuda")
        po = torch.full((n, n, 2), float("nan"), dtype=torch.float64, device="cuda")
        pd = torch.full((npos, 2), float("nan"), dtype=torch.float64, device="cuda")
        er = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        ptrs = [t.data_ptr() for t in (V, pr, pp, sx, sy, me, g, po, pd, er)]
        check("mset_batch_gradient_noalloc", lib.mset_batch_gradient_noalloc(
            torch.cuda.current_device(), C.c_void_p(stream), n, nz, b, method, adjoint, c["sigma"], c["dz"], npos,
            *[C.c_void_p(p) for p in ptrs]))
        torch.cuda.synchronize()
        probe = po.cpu().numpy()
        assert rel_l2(g.cpu().numpy(), ref["grad"][0]) < TOL, call
        assert rel_l2(probe[..., 0] + 1j * probe[..., 1], ref["probe"][0]) < TOL, call
        # scan-position directions at n = 128 are cancellation-limited sums; the
        # other GPU tests allow 3e-4 there (tests/test_gpu_parity.py)
        assert rel_l2(pd.cpu().numpy(), ref["posdir"]) < (TOL if n <= 96 else 3e-4), call
        assert abs(er.item() - ref["err"][0]) <= TOL * ref["err"][0], call


def test_noalloc_rejects_oversized_request(gpu_available):
    lib = load()
    null = C.c_void_p(8)  # never dereferenced: the size check comes first
    # 128 x 128 with 600 slabs needs 601 saved waves (78.8 MB) > the 64 MiB scratch
    rc = lib.mset_batch_gradient_noalloc(0, None, 128, 600, 1, MSET_MODE_MSET, MSET_ADJOINT_REF, 1e-3, 0.3, 4,
                                         *([null] * 10))
    assert rc == -2  # MSET_E_UNSUPPORTED
    assert b"64 MiB" in lib.mset_last_error()
    rc = lib.mset_batch_gradient_noalloc(0, None, 96, 4, 1, MSET_MODE_MSET, MSET_ADJOINT_REF, 1e-3, 0.3, 4,
                                         *([null] * 10))
    assert rc == -2 and b"window size" in lib.mset_last_error()
