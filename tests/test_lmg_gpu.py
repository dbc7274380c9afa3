"""Learned multigrid preconditioner on the B200 (no reference counterpart).

1. The network's forward output and its parameter gradients (tcgen05 forward
   and input-gradient convolutions, CUDA-core weight gradients) against the
   numpy oracle (oracle/cnn.py), which rounds weights and stored activations
   to BF16 where the kernels do. The kernels also store gradients in BF16 and
   sum in another order, so the check is relative L2 per layer: within 5e-2
   for gradients (a wrong backward is off by O(1)) and 2e-2 for the network
   part of M(r).
2. Training on residual/error pairs from Jacobi-PCG lowers the loss.
3. Flexible CG with the trained network reaches the FP64 residual 1e-10 on
   held-out fields in fewer iterations than Jacobi-PCG: the gain the network
   brings over the same method without it."""
import numpy as np
import pytest

from oracle import cnn as ref

pytestmark = pytest.mark.gpu


def small_problem(n=2, h=32, w=32, seed=3):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, h + 2, w + 2))
    e = np.zeros_like(r)
    r[:, 1:-1, 1:-1] = rng.standard_normal((n, h, w))
    e[:, 1:-1, 1:-1] = rng.standard_normal((n, h, w))
    Kx = np.zeros_like(r)
    Ky = np.zeros_like(r)
    Kx[:, 1:-1, 2:-1] = rng.uniform(0.01, 5.0, (n, h, w - 1))
    Ky[:, 2:-1, 1:-1] = rng.uniform(0.01, 5.0, (n, h - 1, w))
    return r, Kx, Ky, e


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_forward_and_gradients_match_oracle(gpu_runtime):
    import torch
    from ops_b200 import lmg
    r, Kx, Ky, e = small_problem()
    p = ref.init_params(seed=1, out_scale=0.5)
    net = lmg.Net(seed=1)
    try:
        net.set_params(p)
        out = torch.zeros_like(cuda(r))
        net.apply(cuda(r), cuda(Kx), cuda(Ky), 30.0, 30.0, out)
        M_ref, A = ref.net_forward(p, r, Kx, Ky, 30.0, 30.0)
        got = out.cpu().numpy()[:, 1:-1, 1:-1]
        assert rel(got - A["z"], M_ref - A["z"]) < 2e-2
        for kind in ("l2", "anorm"):
            loss = net.train_step(cuda(r), cuda(Kx), cuda(Ky), cuda(e), 30.0, 30.0, 0.0, loss=kind)
            L_ref, g_ref = ref.net_loss_grad(p, r, Kx, Ky, e, 30.0, 30.0, anorm=kind == "anorm")
            assert abs(loss - L_ref) < 1e-3 * L_ref, kind
            g = net.grads().astype(np.float64)
            o = 0
            for l, (ci, co) in enumerate(ref.LAYERS):
                k = 9 * ci * co + co
                assert rel(g[o:o + k], g_ref[o:o + k]) < 5e-2, (kind, l, rel(g[o:o + k], g_ref[o:o + k]))
                o += k
            assert rel(g[o:], g_ref[o:]) < 1e-2, kind
        assert np.array_equal(net.params(), p)   # lr = 0: no step
    finally:
        net.close()


def test_untrained_network_is_jacobi(gpu_runtime):
    import torch
    from ops_b200 import lmg
    r, Kx, Ky, _ = small_problem(seed=4)
    net = lmg.Net(seed=2)
    try:
        out = torch.zeros_like(cuda(r))
        net.apply(cuda(r), cuda(Kx), cuda(Ky), 30.0, 30.0, out)
        _, A = ref.net_forward(net.params(), r, Kx, Ky, 30.0, 30.0)
        np.testing.assert_allclose(out.cpu().numpy()[:, 1:-1, 1:-1], A["z"], rtol=1e-15, atol=0)
    finally:
        net.close()


@pytest.fixture(scope="module")
def trained(gpu_runtime):
    """The training recipe (PCG pairs, then three rounds of on-policy pairs from
    the learned FCG's own iterates) on 64 x 64 seeded fields."""
    from ops_b200 import lmg
    net = lmg.Net(seed=5)
    hists = lmg.fit(net, n=64, nfields=300, steps=1500, rounds=3)
    yield net, hists
    net.close()


def test_training_lowers_loss(trained):
    _, hists = trained
    first = hists[0]
    assert np.mean(first[-40:]) < 0.7 * np.mean(first[:10])


def test_learned_fcg_beats_jacobi_pcg(trained):
    import torch
    from ops_b200 import lmg
    net, _ = trained
    n, rx = 64, 400.0
    its_pcg, its_fcg = [], []
    for seed in (90001, 90002, 90003):
        rho, en = lmg.density_field(n, seed)
        Kx, Ky, u0 = lmg.padded_problem(rho, en)
        kx, ky, b = cuda(Kx), cuda(Ky), cuda(u0)
        u = b.clone()
        sp = lmg.solve(kx, ky, b, u, rx, rx, method=lmg.PCG_TRUE, eps=1e-10)
        u2 = b.clone()
        sj = lmg.solve(kx, ky, b, u2, rx, rx, method=lmg.FCG_JACOBI, eps=1e-10)
        u3 = b.clone()
        sl = lmg.solve(kx, ky, b, u3, rx, rx, method=lmg.FCG_LEARNED, net=net.h, eps=1e-10, window=40)
        for s in (sp, sj, sl):
            assert s["converged"] and s["final_residual"] < 1.5e-10 * s["initial_residual"]
        assert abs(sj["iterations"] - sp["iterations"]) <= 0.1 * sp["iterations"] + 2
        ua, uc = u.cpu().numpy(), u3.cpu().numpy()
        assert rel(uc, ua) < 1e-8
        its_pcg.append(sp["iterations"])
        its_fcg.append(sl["iterations"])
    assert sum(its_fcg) < 0.8 * sum(its_pcg), (its_fcg, its_pcg)


@pytest.mark.parametrize("n", [256, 512])
def test_learned_fcg_gain_beyond_the_training_size(trained, n):
    """Trained on 64 x 64 fields, the network still cuts the iterations of the
    heat solve on larger grids: fewer than half of Jacobi-PCG's at 256^2 and
    512^2 (measured about a sixth and a fifth). Each application costs about
    ten PCG iterations, so the wall time is not lower (bench.py --workload
    learned, grid_sweep_rx400); at 1024^2 the gain falls to 1.6x and at
    4096^2 it is gone."""
    from ops_b200 import lmg
    net, _ = trained
    rho, en = lmg.density_field(n, 91000 + n)
    Kx, Ky, u0 = lmg.padded_problem(rho, en)
    kx, ky, b = cuda(Kx), cuda(Ky), cuda(u0)
    u = b.clone()
    sp = lmg.solve(kx, ky, b, u, 400.0, 400.0, method=lmg.PCG_TRUE, eps=1e-10)
    u2 = b.clone()
    sl = lmg.solve(kx, ky, b, u2, 400.0, 400.0, method=lmg.FCG_LEARNED, net=net.h, eps=1e-10, window=40)
    for st in (sp, sl):
        assert st["converged"] and st["final_residual"] < 1.5e-10 * st["initial_residual"]
    assert rel(u2.cpu().numpy(), u.cpu().numpy()) < 1e-8
    assert sl["iterations"] < 0.5 * sp["iterations"], (sl["iterations"], sp["iterations"])


@pytest.mark.parametrize("n", [64, 256])
def test_replayed_fcg_chunks_match_the_host_loop(trained, n):
    """The learned and Jacobi flexible-CG solves run their iterations from
    replayed graph chunks (stopping and restart tests on the device); with the
    option off they run the host loop. Same iterations, same restarts, and
    the same solution bit for bit."""
    from ops_b200 import lmg
    from ops_b200 import ops as O
    net, _ = trained
    rho, en = lmg.density_field(n, 91000 + n)
    Kx, Ky, u0 = lmg.padded_problem(rho, en)
    kx, ky, b = cuda(Kx), cuda(Ky), cuda(u0)
    for method, h in ((lmg.FCG_LEARNED, net.h), (lmg.FCG_JACOBI, -1)):
        out = {}
        for chunks in (1, 0):
            O.set_option("fcg_chunks", chunks)
            try:
                u = b.clone()
                st = lmg.solve(kx, ky, b, u, 400.0, 400.0, method=method, net=h, eps=1e-10, window=40)
            finally:
                O.set_option("fcg_chunks", 1)
            out[chunks] = (st, u.cpu().numpy())
        (s1, u1), (s0, u0_) = out[1], out[0]
        assert s1["converged"] and s0["converged"]
        assert (s1["iterations"], s1["fallbacks"]) == (s0["iterations"], s0["fallbacks"]), (method, s1, s0)
        assert np.array_equal(u1, u0_), method


def test_untrained_learned_multigrid_is_the_vcycle(gpu_runtime):
    """FCG_LEARNED_MG applies V-cycle(r) + (network output - r / D); with the
    output layer at zero that is the V-cycle exactly, so the solve repeats
    FCG_MG bit for bit."""
    import torch
    from ops_b200 import lmg
    rho, en = lmg.density_field(96, 77)
    kx, ky, b = (cuda(a) for a in lmg.padded_problem(rho, en))
    net = lmg.Net(seed=3)
    try:
        u1, u2 = b.clone(), b.clone()
        s1 = lmg.solve(kx, ky, b, u1, 300.0, 300.0, method=lmg.FCG_MG, eps=1e-10, window=40)
        s2 = lmg.solve(kx, ky, b, u2, 300.0, 300.0, method=lmg.FCG_LEARNED_MG, net=net.h, eps=1e-10, window=40)
        assert s1["converged"] and s2["converged"] and s2["fallbacks"] == 0
        assert s1["iterations"] == s2["iterations"]
        assert torch.equal(u1, u2)
    finally:
        net.close()
