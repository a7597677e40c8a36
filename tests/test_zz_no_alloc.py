"""aldic_subpb2_noalloc -- Subproblem 2 for callers that cannot allocate
device memory (a host framework that owns every device byte, a real-time loop
that must not stall on an allocation, a process with audited or capped
allocations).  Its work vectors live in the library's fixed static device
array, so the test checks, through the C ABI, that two calls in a row give
the same Uhat as the allocating entry point aldic_subpb2 (which solves
directly; this entry point's PCG stops at 1e-11 relative residual; results
compared to 1e-8) and that oversize grids are refused.  Kept in its own file
that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_subpb2_noalloc_matches_subpb2(aldic):
    import torch
    assert torch.cuda.is_available(), "GPU test"
    ctx = aldic.Context(0)
    call = aldic._lib.call
    rng = np.random.default_rng(2024)
    M, N, h, mu = 61, 47, 8.0, 1e-3
    n = M * N
    dev = torch.device("cuda", 0)
    for k, beta in enumerate((6.4e-5, 2.0e-2)):
        U = rng.standard_normal(2 * n)
        F = 0.01 * rng.standard_normal(4 * n)
        ud = 0.001 * rng.standard_normal(4 * n)
        vd = 0.01 * rng.standard_normal(2 * n)
        ref = np.empty(2 * n)
        call("aldic_subpb2", ctx.h, M, N, h, beta, mu, *[C.c_void_p(a.ctypes.data) for a in (U, F, ud, vd, ref)])
        dU, dF, dud, dvd = (torch.from_numpy(a).to(dev) for a in (U, F, ud, vd))
        out = torch.full((2 * n,), float("nan"), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev)
        call("aldic_subpb2_noalloc", M, N, h, beta, mu, *[C.c_void_p(t.data_ptr()) for t in (dU, dF, dud, dvd, out)],
             C.c_void_p(stream.cuda_stream))
        np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-8, atol=1e-10)
    # oversize grids are refused with a clear error, nothing launched
    big = torch.zeros(2 * 300 * 300, dtype=torch.float64, device=dev)
    with pytest.raises(aldic.AldicError) as e:
        call("aldic_subpb2_noalloc", 300, 300, h, 1e-3, mu, *[C.c_void_p(big.data_ptr())] * 5, None)
    assert "65536 nodes" in str(e.value)
