"""GPU tests of the learned-guess kernels (forward, backward, loss, Adam)
against the FP64 numpy oracle, training on the GPU, and the guess in SCF."""
import os

import numpy as np
import pytest

from oracle import mlp_ref

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GUESS_FILE = os.path.join(os.path.dirname(__file__), "..", "librint_b200", "data", "guess_ch.npz")


def _net(sizes, seed=1):
    from librint_b200.guess import MLP
    net = MLP(sizes, seed=seed)
    g = np.random.default_rng(seed + 100)
    for b in net.b:
        b.copy_(torch.tensor(g.normal(size=b.shape[0]) * 0.1, dtype=torch.float32))
    return net


def _np_params(net):
    return [p.double().cpu().numpy() for p in net.params]


@pytest.mark.parametrize("M,sizes", [(1, [3, 5, 2]), (77, [63, 256, 256, 225]),
                                     (2048, [63, 128, 128, 225]), (33, [40, 33, 31, 17])])
def test_forward_backward_vs_oracle(M, sizes):
    from librint_b200.guess import mse
    net = _net(sizes)
    g = np.random.default_rng(M)
    X = g.normal(size=(M, sizes[0]))
    T = g.normal(size=(M, sizes[-1]))
    W = (g.random(size=T.shape) > 0.2).astype(np.float64)
    Xd = torch.tensor(X, dtype=torch.float32, device="cuda")
    out, acts, zs = net.forward(Xd, keep=True)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    inv = 1.0 / T.size
    dY = mse(out, torch.tensor(T, dtype=torch.float32, device="cuda"),
             torch.tensor(W, dtype=torch.float32, device="cuda"), loss, inv)
    grads = net.backward(acts, zs, dY)
    torch.cuda.synchronize()
    params = _np_params(net)
    Xr = Xd.double().cpu().numpy()
    ref_loss, ref_grads, ref_Y = mlp_ref.loss_and_grad(params, Xr, T, W, inv)
    Y = out.double().cpu().numpy()
    # FP32 arithmetic: errors relative to the magnitude of each tensor
    assert np.abs(Y - ref_Y).max() <= 1e-5 * max(1.0, np.abs(ref_Y).max())
    assert abs(loss.item() - ref_loss) <= 1e-5 * ref_loss
    for g_gpu, g_ref in zip(grads, ref_grads):
        gg = g_gpu.double().cpu().numpy()
        assert np.abs(gg - g_ref).max() <= 2e-5 * max(1e-6, np.abs(g_ref).max())


def test_adam_vs_oracle():
    from librint_b200.guess import Adam
    g = np.random.default_rng(3)
    p = torch.tensor(g.normal(size=1000), dtype=torch.float32, device="cuda")
    opt = Adam([p], lr=1e-2)
    pn = p.double().cpu().numpy()
    m = np.zeros_like(pn)
    v = np.zeros_like(pn)
    for t in range(1, 6):
        gr = g.normal(size=1000)
        opt.step([torch.tensor(gr, dtype=torch.float32, device="cuda")])
        pn, m, v = mlp_ref.adam_step(pn, gr, m, v, 1e-2, 0.9, 0.999, 1e-8, t)
    torch.cuda.synchronize()
    np.testing.assert_allclose(p.double().cpu().numpy(), pn, atol=2e-6)


def test_training_fits_a_smooth_function():
    """GPU training with the library's kernels drives a regression loss down."""
    from librint_b200.guess import MLP, Adam, mse
    g = np.random.default_rng(0)
    X = g.uniform(-1, 1, size=(4096, 8))
    T = np.stack([np.sin(2 * X[:, 0]) * X[:, 1], X[:, 2] ** 2 - X[:, 3], np.cos(X[:, 4] + X[:, 5])], 1)
    net = MLP([8, 64, 64, 3], seed=0)
    opt = Adam(net.params, lr=3e-3)
    Xd = torch.tensor(X, dtype=torch.float32, device="cuda")
    Td = torch.tensor(T, dtype=torch.float32, device="cuda")
    losses = []
    for it in range(600):
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        out, acts, zs = net.forward(Xd, keep=True)
        dY = mse(out, Td, None, loss)
        opt.step(net.backward(acts, zs, dY))
        if it % 100 == 0 or it == 599:
            losses.append(loss.item())
    assert losses[-1] < 0.02 * losses[0]


@pytest.mark.skipif(not os.path.exists(GUESS_FILE), reason="trained network not present")
def test_learned_guess_scf_same_energy_fewer_iterations():
    """Held-out ring geometries: the learned start converges to the energy of
    the core-Hamiltonian start (|dE| <= 1e-9 Eh) in fewer iterations."""
    from librint_b200.guess import LearnedGuess
    from librint_b200.scf import MolContext
    from librint_b200.train_guess import SCF_OPTS, geometry
    g = LearnedGuess.load(GUESS_FILE)
    its_core, its_learned = [], []
    for i in (2300, 2301, 2302):               # outside the training and held-out ranges
        m = geometry(i)
        assert g.applies(m)
        ctx = MolContext(m)
        S = ctx.int1e(0)
        P0 = g.predict(m, S=S)
        assert abs(np.sum(P0 * S) - m.nelec) < 1e-9
        rb = ctx.scf(conv=1e-8, **SCF_OPTS)
        rl = ctx.scf(conv=1e-8, P0=P0, **SCF_OPTS)
        ctx.close()
        assert abs(rb.energy - rl.energy) <= 1e-9
        its_core.append(rb.iterations)
        its_learned.append(rl.iterations)
    assert sum(its_learned) < sum(its_core), (its_core, its_learned)
