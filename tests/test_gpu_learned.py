"""The learned term of the two-level flexible-CG preconditioner (one-ring message-passing network,
BF16 weights on tensor cores, FP32 accumulate), trained on the GPU by the library's own forward
and backward kernels on samples that the pressure solves record.

* gradient check: loss and parameter gradient of the device kernels against the oracle's double
  restatement (same bf16 rounding points) on the same recorded samples and parameters;
* training: the A-angle loss decreases; the kept scale gamma never makes the held-out solves take
  more iterations than the preconditioner without the term (gamma = 0 is kept on ties);
* ablation: the next time steps (solves the gate never saw) with and without the trained term:
  when the gate kept the term (gamma > 0) it must take strictly fewer iterations there; when it
  switched the term off, the two runs are the same solve.  The flow still meets the divergence
  bound.  The measured iterations are printed.
"""
import ctypes as C

import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200.solver import Solver
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _fcg_solver(nx, ny, nz):
    case = cases.channel_config(nx=nx, ny=ny, nz=nz)
    p = case.make_params()
    p.p_solver = abi.PSOLVER_TWOLEVEL_FCG
    s = Solver(case, params=p)
    s.initialise()
    return s


def test_learned_gradient_matches_oracle():
    s = _fcg_solver(24, 16, 12)
    assert s.learn_collect(1) > 4
    d = s.learn_export()
    rng = np.random.default_rng(7)
    prm = (rng.uniform(-0.5, 0.5, 561)).astype(np.float32)
    prm[560] = 0.0  # omega of order 0.2: the term is well away from zero
    loss_g, grad_g = s.learn_loss_grad(prm)
    loss_o = C.c_double(0.0)
    grad_o = np.zeros(561)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    O.lib().orc_lp_loss_grad(d["n"], d["C"], d["WL"], d["lpk"].ctypes.data, d["feat"].ctypes.data, d["WA"],
                             d["col"].ctypes.data, dp(d["val"]), d["S"], dp(d["R"]), dp(d["Z"]), dp(d["U"]),
                             dp(d["E"]), prm.ctypes.data, C.byref(loss_o), dp(grad_o))
    assert abs(loss_g - loss_o.value) <= 1e-6 * abs(loss_o.value), (loss_g, loss_o.value)
    err = np.linalg.norm(grad_g - grad_o) / np.linalg.norm(grad_o)
    assert err <= 2e-3, err
    for blk in ((0, 256), (256, 272), (272, 528), (528, 544), (544, 560)):  # every layer is reached
        assert np.linalg.norm(grad_o[blk[0]:blk[1]]) > 0.0, blk


def test_learned_training_and_ablation():
    s = _fcg_solver(48, 32, 32)
    k = s.learn_collect(3)
    assert k >= 16
    rep = s.learn_train(epochs=80, lr=1e-2)
    print("learned-term training:", rep)
    assert rep["loss_final"] < rep["loss_initial"]
    assert rep["gamma"] in (0.0, 0.5, 1.0)
    assert rep["its_val_learned"] <= rep["its_val_base"]
    # ablation on the following steps: same state, with and without the term
    host = s.sync_host()
    its = {}
    for g in (0.0, rep["gamma"]):
        s.to_device(U=host["U"], p=host["p"])
        s.learn_set_gamma(g)
        tot = 0
        for _ in range(2):
            s.advance()
            st = s.stats()
            tot += st["p_iters"]
            assert st["max_abs_divU"] <= 1e-6
        its[g] = tot
    print("ablation iterations (gamma -> total over 2 steps):", its)
    if rep["gamma"] > 0.0:
        assert its[rep["gamma"]] < its[0.0], its


def test_learned_term_on_the_multilevel_form():
    """The learned term on the multilevel form (p_solver = DPM_PSOLVER_MULTILEVEL_FCG): samples
    recorded by the multilevel kernel, the same training kernels, gamma gated on the held-out
    solve; then an ablation from the same state with the gated gamma: the steps converge
    (divergence <= 1e-8, no fallback), and a kept term (gamma > 0) must take strictly fewer
    iterations on those unseen solves.  On
    the channel the V-cycle leaves the one-ring term little to correct (A-angle loss ~0.12 against
    ~0.7 under the two-level preconditioner) and the gate measured gamma = 0."""
    case = cases.channel_config(nx=48, ny=32, nz=32)
    p = case.make_params()
    p.p_solver = abi.PSOLVER_MULTILEVEL_FCG
    s = Solver(case, params=p)
    s.initialise()
    k = s.learn_collect(3)
    assert k >= 8, k
    rep = s.learn_train(epochs=80, lr=1e-2)
    print("multilevel learned-term training:", rep)
    assert rep["loss_final"] <= rep["loss_initial"]
    assert rep["gamma"] in (0.0, 0.5, 1.0)
    assert rep["its_val_learned"] <= rep["its_val_base"]
    host = s.sync_host()
    its = {}
    for g in sorted({0.0, rep["gamma"]}):
        s.to_device(U=host["U"], p=host["p"])
        s.learn_set_gamma(g)
        tot = 0
        for _ in range(2):
            s.advance()
            st = s.stats()
            tot += st["p_iters"]
            assert st["max_abs_divU"] <= 1e-8 and st["p_fallbacks"] == 0
        its[g] = tot
    print("multilevel ablation iterations (gamma -> total over 2 steps):", its)
    if rep["gamma"] > 0.0:
        assert its[rep["gamma"]] < its[0.0], its
