"""iblgf_conv_block_noalloc against iblgf_conv_block (both through the C ABI).

The allocation-free entry point keeps its temporaries in a static device
array; it must give the same block as the allocating entry point, on two calls
in a row (the second reuses the scratch the first left behind). Tolerance:
1e-12 relative L-inf in FP64, 1e-5 in FP32 (both run the same kernels, so the
results are expected to agree exactly).
"""
import ctypes

import numpy as np
import pytest

import iblgf_b200 as B
import oracle_lib as O

pytestmark = pytest.mark.gpu


def _solver(N, precision):
    return B.Solver((-4 * N,) * 3, (8 * N,) * 3, N - 2, 1.0, [((-2 * N + 4,) * 3, ((N - 2) * 2,) * 3)],
                    precision=precision)


@pytest.mark.parametrize("N", [8, 18])
@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
def test_conv_block_noalloc_matches_allocating_entry(N, precision, tol):
    torch = pytest.importorskip("torch")
    P = 2 * N - 1
    g = _solver(N, precision)
    L = B.lib()
    rng = np.random.default_rng(N)
    for call in range(2):
        src = rng.standard_normal((N, N, N))
        ker = rng.standard_normal((P, P, P))
        ts = torch.tensor(src.ravel(order="F"), device="cuda", dtype=torch.float64)
        tk = torch.tensor(ker.ravel(order="F"), device="cuda", dtype=torch.float64)
        base = rng.standard_normal(N ** 3)
        ref_out = torch.tensor(base, device="cuda", dtype=torch.float64)
        out = torch.tensor(base, device="cuda", dtype=torch.float64)
        g.conv_block(ts.data_ptr(), tk.data_ptr(), ref_out.data_ptr(), 0.5)
        rc = L.iblgf_conv_block_noalloc(g.h, ctypes.c_void_p(ts.data_ptr()), ctypes.c_void_p(tk.data_ptr()),
                                        ctypes.c_void_p(out.data_ptr()), 0.5)
        assert rc == 0, L.iblgf_last_error(g.h)
        assert L.iblgf_synchronize(g.h) == 0
        a = out.cpu().numpy() - base
        b = ref_out.cpu().numpy() - base
        rel = float(np.abs(a - b).max() / np.abs(b).max())
        assert rel < tol, (call, rel)
        if N == 8 and precision == B.FP64:
            ora = O.block_conv(src, ker, 0.5).ravel(order="F")
            assert float(np.abs(a - ora).max() / np.abs(ora).max()) < tol


def test_conv_block_noalloc_rejects_null():
    g = _solver(8, B.FP64)
    L = B.lib()
    assert L.iblgf_conv_block_noalloc(g.h, None, None, None, 1.0) == 1  # IBLGF_EINVAL


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
def test_conv_block_noalloc_is_capturable_without_allocation(precision, tol):
    """After its one-time set-up call, the entry point allocates, frees and
    synchronises nothing: a second call recorded under global-mode stream
    capture (where cudaMalloc, cudaFree and synchronisation from any thread
    fail the capture) succeeds, and the replayed graph gives the allocating
    entry point's block."""
    torch = pytest.importorskip("torch")
    N = 18
    P = 2 * N - 1
    s = torch.cuda.Stream()
    g = B.Solver((-4 * N,) * 3, (8 * N,) * 3, N - 2, 1.0, [((-2 * N + 4,) * 3, ((N - 2) * 2,) * 3)],
                 precision=precision, stream=s.cuda_stream)
    L = B.lib()
    rng = np.random.default_rng(11)
    src = torch.tensor(rng.standard_normal(N ** 3), device="cuda", dtype=torch.float64)
    ker = torch.tensor(rng.standard_normal(P ** 3), device="cuda", dtype=torch.float64)
    base = rng.standard_normal(N ** 3)
    out = torch.tensor(base, device="cuda", dtype=torch.float64)
    ref = torch.tensor(base, device="cuda", dtype=torch.float64)

    def call(o):
        return L.iblgf_conv_block_noalloc(g.h, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(ker.data_ptr()),
                                          ctypes.c_void_p(o.data_ptr()), 0.5)

    warm = torch.zeros(N ** 3, device="cuda", dtype=torch.float64)
    assert call(warm) == 0  # one-time set-up, outside any capture
    assert L.iblgf_synchronize(g.h) == 0
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="global"):
        rc = call(out)
    assert rc == 0, L.iblgf_last_error(g.h)
    graph.replay()
    torch.cuda.synchronize()
    g.conv_block(src.data_ptr(), ker.data_ptr(), ref.data_ptr(), 0.5)
    assert L.iblgf_synchronize(g.h) == 0
    a = out.cpu().numpy() - base
    b = ref.cpu().numpy() - base
    assert float(np.abs(a - b).max() / np.abs(b).max()) < tol
    del graph
    g.close()
