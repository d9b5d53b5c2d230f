"""Learned warm start of the IB force CG (iblgf_ib_warmstart, iblgf_ws_check).

* The device network's forward pass, loss and parameter gradients against a
  float64 numpy restatement of the same network (the checker), FP32
  tolerance 1e-4 relative.
* In the IF-HERK step past the sphere: training on the solver's own samples
  lowers the loss, the CG still converges to its tolerance and the velocity
  agrees with the reference warm start (previous force) to the CG tolerance.
  The CG iterations of the three warm starts (previous force, its linear
  extrapolation, previous force + the network's correction) are reported:
  on this flow neither alternative needs fewer iterations than the previous
  force (the measured numbers are in the bench line).
"""
import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S
import oracle_lib as O

pytestmark = pytest.mark.gpu
C, K, I = 64, 5, 9


def offsets():
    o = [0]
    for n in (C * I * K, C, C * C * K, C, 3 * C * K, 3):
        o.append(o[-1] + n)
    return o


def conv(x, W, b):
    N = x.shape[2]
    xp = np.pad(x, ((0, 0), (0, 0), (2, 2)))
    y = np.zeros((x.shape[0], W.shape[0], N)) + b[None, :, None]
    for k in range(K):
        y += np.einsum("oc,scn->son", W[:, :, k], xp[:, :, k:k + N])
    return y, xp


def conv_back(dy, xp, W):
    N = dy.shape[2]
    dW = np.zeros_like(W)
    dxp = np.zeros_like(xp)
    for k in range(K):
        dW[:, :, k] = np.einsum("son,scn->oc", dy, xp[:, :, k:k + N])
        dxp[:, :, k:k + N] += np.einsum("oc,son->scn", W[:, :, k], dy)
    return dW, dy.sum((0, 2)), dxp[:, :, 2:2 + N]


def reference(params, x, t):
    o = offsets()
    p = params.astype(np.float64)
    W1, b1 = p[o[0]:o[1]].reshape(C, I, K), p[o[1]:o[2]]
    W2, b2 = p[o[2]:o[3]].reshape(C, C, K), p[o[3]:o[4]]
    W3, b3 = p[o[4]:o[5]].reshape(3, C, K), p[o[5]:o[6]]
    a1, x0p = conv(x.astype(np.float64), W1, b1)
    h1 = np.maximum(a1, 0)
    a2, h1p = conv(h1, W2, b2)
    h2 = np.maximum(a2, 0)
    y, h2p = conv(h2, W3, b3)
    d = y - t
    loss = float((d * d).mean())
    dy = 2 * d / d.size
    dW3, db3, dh2 = conv_back(dy, h2p, W3)
    dh2 = dh2 * (h2 > 0)
    dW2, db2, dh1 = conv_back(dh2, h1p, W2)
    dh1 = dh1 * (h1 > 0)
    dW1, db1, _ = conv_back(dh1, x0p, W1)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return y, g, loss


def test_network_forward_backward_matches_reference():
    case = S.SphereIB("small")
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks)
    rng = np.random.default_rng(3)
    n = offsets()[-1]
    params = (rng.standard_normal(n) * 0.1).astype(np.float32)
    x = rng.standard_normal((2, I, 37)).astype(np.float32)
    t = rng.standard_normal((2, 3, 37)).astype(np.float32)
    y, grads, loss = g.ws_check(params, x, t)
    yr, gr, lr = reference(params, x, t)
    assert np.abs(y - yr).max() / np.abs(yr).max() < 1e-4
    assert np.abs(grads - gr).max() / np.abs(gr).max() < 1e-4
    assert abs(loss - lr) / lr < 1e-4


def _run(mode, steps=12):
    case = S.SphereIB("small")
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    X = O.sphere_points(case.dx_base, g.depth - 1 - g.base_level, case.ibph)
    g.ib_set_points(X, case.Re)
    # a tight CG tolerance, so that both warm starts reach the same solution
    g.ns_options((-1.0, 0.0, 0.0), cg_threshold=1e-6, cg_max_iter=200)
    g.ib_warmstart(mode, train_steps=4, epochs=1500, lr=2e-3, seed=7)
    u0 = case.velocity(g, U=(0.0, 0.0, 0.0))
    uf = [g.field(u0[k]) for k in range(3)]
    pf = g.field()
    T, its = 0.0, []
    for _ in range(steps):
        T = g.ns_step(uf, pf, 0.01, case.Re, T, 1)
        its.append(g.ib_iterations())
    u = np.stack([g.download(uf[k]) for k in range(3)])
    return u, its, g.ib_warmstart_info()


def test_learned_warm_start_in_ns_step():
    u0, its0, _ = _run(0)
    u2, its2, _ = _run(2)
    u1, its1, info = _run(1)
    # samples from steps 2..5 (3 stages each), trained after step 5
    assert info["trained"] and info["samples"] == 12 and info["params"] == 24451
    assert info["loss_last"] < info["loss_first"]
    assert max(max(s) for s in its1) < 200  # every stage's CG converged before its limit
    assert float(np.abs(u1 - u0).max() / np.abs(u0).max()) < 1e-4
    after = slice(6, None)  # steps 7-12: the trained network predicts
    n0 = sum(sum(s) for s in its0[after])
    n2 = sum(sum(s) for s in its2[after])
    n1 = sum(sum(s) for s in its1[after])
    print("CG iterations over steps 7-12: previous force %d, extrapolation %d, learned %d" % (n0, n2, n1))
    print("warm-start training: %s" % info)
    assert n0 > 0 and n1 > 0 and n2 > 0
