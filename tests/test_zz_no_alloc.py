"""The scratch-free entry point fg_chi_reduce_noalloc, called through the C ABI.

It serves callers that must not allocate device memory (their GPU memory belongs to an allocator they do not
control, so they cannot hand fg_chi_reduce a workspace): its scratch is a fixed 32 MiB array inside the library,
which holds the exact row sums of up to about 5,200 rows at 401 k points (any number of paths).
Checked here against the existing entry point fg_chi_reduce on the same batch, on two calls in a row (the array keeps
the previous call's contents), within the fused stage's tolerance; and an oversized batch must be refused before
any work is launched.  This file is collected last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.fixtures import groups, phase

pytestmark = pytest.mark.gpu


def _ref_rows(st, b, q, S, span):
    """rows from the existing entry point fg_chi_reduce with a torch-allocated workspace."""
    from feffgpu_b200 import _lib
    ps = st._paths_struct(b, b.coords, None)
    NK = q.shape[0]
    rows = torch.empty(b.nrows, NK, dtype=torch.float64, device="cuda")
    n = int(st._lib.fg_chi_reduce_workspace(st._h, C.byref(ps), NK))
    ws = torch.empty(n, dtype=torch.uint8, device="cuda")
    _lib.check(st._lib.fg_chi_reduce(st._h, st.prec, C.byref(ps), NK, q.data_ptr(), S.data_ptr(), span.data_ptr(),
                                     rows.data_ptr(), None, None, ws.data_ptr(), n,
                                     torch.cuda.current_stream().cuda_stream))
    return rows


def _noalloc_rows(st, b, q, S, span, rows=None):
    from feffgpu_b200 import _lib
    ps = st._paths_struct(b, b.coords, None)
    if rows is None:
        rows = torch.full((b.nrows, q.shape[0]), float("nan"), dtype=torch.float64, device="cuda")
    _lib.check(st._lib.fg_chi_reduce_noalloc(st._h, st.prec, C.byref(ps), q.shape[0], q.data_ptr(), S.data_ptr(),
                                             span.data_ptr(), rows.data_ptr(), torch.cuda.current_stream().cuda_stream))
    return rows


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_no_alloc_entry_point_equals_fg_chi_reduce(dtype):
    from feffgpu_b200 import GPUPathStage, PathBatch
    st = GPUPathStage(phase("case_L001"), device="cuda", dtype=dtype)
    gs = groups("case_L001")
    b = PathBatch([(c, i, d, np.arange(len(c)) % 3) for c, i, d in gs.values()], nrows=3, device="cuda")
    q = torch.tensor(np.arange(1, 401) * 0.05, dtype=torch.float64, device="cuda")
    S = st.linear_matrix(q.cpu().numpy()).double().contiguous()
    span = st._span(S)
    ref = _ref_rows(st, b, q, S, span)
    scale = float(ref.abs().max())
    for _ in range(2):   # the fixed scratch still holds the previous call's data on the second call
        rows = _noalloc_rows(st, b, q, S, span)
        torch.cuda.synchronize()
        assert torch.isfinite(rows).all()
        np.testing.assert_allclose(rows.cpu().numpy(), ref.cpu().numpy(), rtol=0, atol=1e-12 * scale)
    # a different, smaller batch after the larger one: the stale contents beyond it must not leak in
    b2 = PathBatch([(gs[3][0][:5], gs[3][1][:5], gs[3][2][:5])], device="cuda")
    np.testing.assert_allclose(_noalloc_rows(st, b2, q, S, span).cpu().numpy(),
                               _ref_rows(st, b2, q, S, span).cpu().numpy(), rtol=0, atol=1e-12 * scale)
    # the defining property: once the scratch address is known (the calls above), calls take no device memory --
    # the GPU's free memory is the same before and after two more calls into a buffer allocated beforehand
    out = torch.empty(b.nrows, q.shape[0], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        _noalloc_rows(st, b, q, S, span, out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=0, atol=1e-12 * scale)


def test_no_alloc_entry_point_refuses_a_batch_beyond_its_scratch():
    """The fixed scratch holds the exact row sums (two 64-bit words per row entry): a batch with more rows than fit is
    refused before any work is launched, whatever its number of paths."""
    from feffgpu_b200 import GPUPathStage, PathBatch, _lib
    st = GPUPathStage(phase("case_L001"), device="cuda", dtype=torch.complex64)
    NK = 401
    nrows = _lib.NOALLOC_SCRATCH_BYTES // (2 * NK * 8) + 10          # the rows' sums alone exceed the scratch
    rng = np.random.default_rng(0)
    coords = np.concatenate([np.zeros((nrows, 1, 3)), rng.normal(0, 2.0, (nrows, 1, 3)) + 2.0], 1)
    ipots = np.tile([0, 1], (nrows, 1))
    b = PathBatch([(coords, ipots, None, np.arange(nrows))], nrows=nrows, device="cuda")
    q = torch.tensor(np.arange(NK) * 0.05, dtype=torch.float64, device="cuda")
    S = st.linear_matrix(q.cpu().numpy()).double().contiguous()
    with pytest.raises(ValueError, match="fixed scratch"):
        _noalloc_rows(st, b, q, S, st._span(S))
