"""The learned SCF start's kernels (include/imago_learned.h) against the CPU
oracle (oracle/mlp.py): forward pass, backward pass (the oracle's analytic
gradient is itself checked by finite differences), Adam, descriptors; and
what the trained network gains over the plain start.

The library computes in FP32 with FP32 accumulation; the oracle in FP64.
Tolerances are written per check: 1e-5 relative to the largest output for
the forward pass, 1e-4 relative to the largest gradient element."""
import os

import numpy as np
import pytest

from oracle import mlp as omlp

NI, NH, NO = 35, 128, 20


def _problem(seed=0, n=300):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, NI))
    t = rng.normal(size=(n, NO))
    m = (rng.random((n, NO)) > 0.25).astype(float)
    return x, t, m


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    ni, nh, no = 6, 9, 4
    npar = ni * nh + nh + nh * nh + nh + nh * no + no
    p = rng.normal(size=npar) * 0.3
    x, t = rng.normal(size=(13, ni)), rng.normal(size=(13, no))
    m = (rng.random((13, no)) > 0.3).astype(float)
    g = omlp.grad(p, x, t, m, ni, nh, no)
    fd = omlp.finite_difference(p, x, t, m, ni, nh, no, range(npar))
    assert np.abs(g - fd).max() < 1e-7 * max(np.abs(g).max(), 1.0)


def _net():
    from imago_b200 import learned
    return learned.Mlp(NI, NO, NH, seed=5)


@pytest.mark.gpu
def test_forward_matches_oracle(imago_lib):
    import torch
    net = _net()
    x, _, _ = _problem()
    y = net.forward(torch.as_tensor(x, dtype=torch.float32, device="cuda").contiguous())
    ref, _ = omlp.forward(net.params().astype(np.float64), x.astype(np.float32).astype(np.float64),
                          NI, NH, NO)
    assert np.abs(y.cpu().numpy() - ref).max() < 1e-5 * np.abs(ref).max()
    net.close()


@pytest.mark.gpu
def test_backward_matches_oracle_gradient(imago_lib):
    import torch
    net = _net()
    x, t, m = _problem(1)
    xs = x.astype(np.float32).astype(np.float64)
    ts = t.astype(np.float32).astype(np.float64)
    dev = "cuda"
    loss, g = net.loss_grad(torch.as_tensor(xs, dtype=torch.float32, device=dev).contiguous(),
                            torch.as_tensor(ts, dtype=torch.float32, device=dev).contiguous(),
                            torch.as_tensor(m, dtype=torch.float32, device=dev).contiguous(),
                            want_grad=True)
    p = net.params().astype(np.float64)
    ref = omlp.grad(p, xs, ts, m, NI, NH, NO)
    assert abs(loss - omlp.loss(p, xs, ts, m, NI, NH, NO)) < 1e-5 * loss
    assert np.abs(g - ref).max() < 1e-4 * np.abs(ref).max()
    # and against finite differences of the oracle's loss on a sample of
    # parameters from every block
    idx = np.linspace(0, len(p) - 1, 40).astype(int)
    fd = omlp.finite_difference(p, xs, ts, m, NI, NH, NO, idx)
    assert np.abs(g[idx] - fd).max() < 1e-4 * np.abs(ref).max()
    net.close()


@pytest.mark.gpu
def test_adam_step_matches_oracle(imago_lib):
    import torch
    net = _net()
    x, t, m = _problem(2)
    args = [torch.as_tensor(a, dtype=torch.float32, device="cuda").contiguous() for a in (x, t, m)]
    p0 = net.params().astype(np.float64)
    _, g = net.loss_grad(*args, want_grad=True)
    net.adam_step(1e-3)
    p1 = net.params().astype(np.float64)
    ref, _, _ = omlp.adam(p0, g.astype(np.float64), np.zeros_like(p0), np.zeros_like(p0), 1,
                          1e-3)
    assert np.abs(p1 - ref).max() < 1e-6
    net.close()


@pytest.mark.gpu
def test_descriptors_match_oracle(imago_lib):
    from imago_b200 import configs, learned
    for s in (configs.silicon_cubic8(kmesh=(1, 1, 1)),
              configs.graphite_cell(reps=(2, 1, 1), kmesh=(1, 1, 1))):
        x = learned.descriptors(s)
        z = [int(round(s.pot_types[t - 1].nuc_charge)) for t in s.pot_site_type]
        ref = omlp.descriptors(s.real_vectors, s.pot_site_pos,
                               [learned.SPECIES.index(v) for v in z], len(learned.SPECIES),
                               learned.CUTOFF, learned.NRAD, learned.WIDTH)
        assert np.abs(x - ref).max() < 1e-5 * np.abs(ref).max()


@pytest.mark.gpu
def test_training_fits_a_smooth_map(imago_lib):
    # full-batch Adam through the library's kernels learns y = sin(x W) to
    # a small fraction of its variance
    from imago_b200 import learned
    rng = np.random.default_rng(7)
    x = rng.normal(size=(512, 8))
    t = np.sin(x @ rng.normal(size=(8, 4)) * 0.5)
    m = np.ones_like(t)
    _, _, hist = learned.train(x, t, m, steps=1500, lr=3e-3)
    assert hist[-1][1] < 0.02 * hist[0][1]


WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "imago_b200", "data", "learned_start.npz")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained network")
def test_learned_start_gain_on_an_unseen_cell(imago_lib):
    # a strained, jittered Si16 cell the network was not trained on, at
    # 2x2x2 k: the learned start must reach the plain start's energy within
    # 1e-6 Ha in no more iterations, and start closer to the converged
    # potential (a smaller first testableDelta)
    from imago_b200 import configs, learned, scf
    e = np.array([[0.012, 0.004, 0.0], [0.004, -0.02, 0.006], [0.0, 0.006, 0.015]])
    s = configs.cubic_supercell("si", reps=(2, 1, 1), kmesh=(2, 2, 2), seed=99, strain=e)
    ls = learned.LearnedStart.load()
    r = learned.compare(s, ls)
    assert r["kept"], (r["plain"]["iterations"], r["learned"]["iterations"],
                       r["plain"]["energies"][-1], r["learned"]["energies"][-1])
    assert r["learned"]["deltas"][0] < r["plain"]["deltas"][0]
