"""The block convolution against the reference's own GPU implementation:
fft::Convolution_GPU<3> (include/iblgf/utilities/convolution_GPU.hpp,
src/utilities/convolution_GPU.cu, cuFFT, FP64), built from the reference
tree into oracle/_ref/ref_conv_gpu by oracle/ref_gpu/Makefile and driven
through its stock apply_forward_add / apply_backward for one (source, LGF
block) pair. The library's iblgf_conv_block on the same random kernel block
and source must agree to 1e-12 relative L-inf (FP64)."""
import os
import subprocess

import numpy as np
import pytest

import iblgf_b200 as B

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_conv_gpu")


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference GPU convolution not built (needs the reference tree)")
@pytest.mark.parametrize("N", [8, 18])
def test_conv_block_matches_reference_cufft_convolution(tmp_path, N):
    torch = pytest.importorskip("torch")
    P = 2 * N - 1
    rng = np.random.default_rng(N)
    ker = rng.standard_normal((P, P, P))
    src = rng.standard_normal((N, N, N))
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        f.write(ker.ravel(order="F").tobytes())
        f.write(src.ravel(order="F").tobytes())
    r = subprocess.run([REF_BIN, "check", str(N), str(fin), str(fout)], capture_output=True, text=True, timeout=120)
    print(r.stderr)
    assert r.returncode == 0, r.stderr
    ref = np.fromfile(fout, dtype=np.float64)
    g = B.Solver((-4 * N,) * 3, (8 * N,) * 3, N - 2, 1.0, [((-2 * N + 4,) * 3, ((N - 2) * 2,) * 3)])
    ts = torch.tensor(src.ravel(order="F"), device="cuda", dtype=torch.float64)
    tk = torch.tensor(ker.ravel(order="F"), device="cuda", dtype=torch.float64)
    to = torch.zeros(N ** 3, device="cuda", dtype=torch.float64)
    g.conv_block(ts.data_ptr(), tk.data_ptr(), to.data_ptr(), 1.0)
    out = to.cpu().numpy()
    assert np.abs(out - ref).max() / np.abs(ref).max() < 1e-12
