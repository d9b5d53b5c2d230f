"""Failure detection without a GPU fault. The reference has none (it ignores
most CUDA return codes, convolution_GPU.cu:144-154, and stops CG silently at
cg_max_itr, linsys.hpp:202-229); the library reports every failure as a
status code and keeps the context usable:

* a bounded device wait that runs out (an mbarrier nothing arrives on) ->
  IBLGF_ETIMEOUT, and the next solve is still exact;
* a device allocation that fails (host-side fault injector, no real
  out-of-memory) -> IBLGF_ENOMEM from context creation or from the first
  solve that allocates, and the context can be destroyed or used again;
* non-finite values in host inputs -> found by the device scan; the solve
  itself does not mask them.
CG that stops at its iteration limit (IBLGF_ENOTCONVERGED) is covered in
test_gpu_ib.py."""
import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S
import oracle_lib as O

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def make(case, precision=B.FP64):
    return B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                    n_levels=getattr(case, "n_levels", 0), predicate=getattr(case, "predicate", None),
                    precision=precision)


def oracle(case):
    return O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                    n_levels=getattr(case, "n_levels", 0), predicate=getattr(case, "predicate", None))


def test_bounded_wait_reports_timeout_and_context_stays_usable():
    case = S.GaussianPoisson("amr_small")
    g, o = make(case), oracle(case)
    with pytest.raises(B.IblgfError) as e:
        g.wait_selftest(1000)
    assert e.value.code == B.ETIMEOUT
    # the status word was cleared: a second run reports the same, once
    with pytest.raises(B.IblgfError) as e:
        g.wait_selftest(10)
    assert e.value.code == B.ETIMEOUT
    with pytest.raises(B.IblgfError) as e:
        g.wait_selftest(0)
    assert e.value.code == B.EINVAL
    src = case.fields(g)
    fs, ft = g.field(src), g.field()
    g.apply_lgf(fs, ft)
    assert rel_linf(g.download(ft), o.apply_lgf(src)) < 1e-12
    g.close()


@pytest.mark.parametrize("after", [0, 3, 20])
def test_allocation_failure_is_reported(after):
    """The injector fails the (after+1)-th allocation: creation or the first
    solve (plans, spectra, sweep buffers) returns ENOMEM; a context that
    survived creation is destroyed cleanly, and a fresh one solves exactly."""
    case = S.GaussianPoisson("amr_small")
    src = None
    B.debug_fail_alloc(after)
    try:
        try:
            g = make(case)
        except B.IblgfError as e:
            assert e.code == B.ENOMEM
            g = None
        if g is not None:
            src = case.fields(g)
            with pytest.raises(B.IblgfError) as e:
                fs, ft = g.field(src), g.field()
                g.apply_lgf(fs, ft)
                g.synchronize()
            assert e.value.code == B.ENOMEM
            g.close()
    finally:
        B.debug_fail_alloc(-1)
    g, o = make(case), oracle(case)
    src = case.fields(g)
    fs, ft = g.field(src), g.field()
    g.apply_lgf(fs, ft)
    assert rel_linf(g.download(ft), o.apply_lgf(src)) < 1e-12
    g.close()


def test_nonfinite_host_input_is_found():
    case = S.GaussianPoisson("amr_small")
    g = make(case)
    src = case.fields(g)
    fs, ft = g.field(src), g.field()
    assert g.first_nonfinite(fs) == -1
    bad = src.copy()
    leaves = np.nonzero(g.leaf)[0]  # the solve reads leaf interiors only
    idx = (int(leaves[len(leaves) // 2]), 3, 4, 5)
    bad[idx] = np.nan
    bad[int(leaves[-1]), 1, 1, 1] = np.inf
    g.upload(fs, bad)
    assert g.first_nonfinite(fs) == int(np.ravel_multi_index(idx, bad.shape))
    g.apply_lgf(fs, ft)
    out = g.download(ft)
    assert g.first_nonfinite(ft) >= 0 and not np.isfinite(out).all()
    g.upload(fs, src)
    g.apply_lgf(fs, ft)
    assert g.first_nonfinite(ft) == -1
    g.close()
