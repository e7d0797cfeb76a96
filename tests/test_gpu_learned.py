"""The learned con2prim seed on the GPU: backward kernels against the CPU
oracle, training, the Newton refinement judged by Cardano, the ablation
against the same Newton without the network, and the learned path inside a
run of the solver."""
import numpy as np
import pytest

from conftest import rel_l1_field

pytestmark = pytest.mark.gpu

PRIMS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]


@pytest.fixture(scope="module")
def trained():
    from cueva.learned import LearnedSeed, synthetic_pairs
    cons, prims = synthetic_pairs(400_000, seed=1234)
    net = LearnedSeed(seed=11)
    net.fit_normalisation(cons, prims)
    first = net.train(cons, prims, steps=10, batch=4096, lr=2e-3)
    last = net.train(cons, prims, steps=3000, batch=4096, lr=2e-3)
    yield net, first, last
    net.close()


def test_gradients_match_oracle():
    import mlp_oracle as mo
    from cueva.learned import LearnedSeed, synthetic_pairs
    cons, prims = synthetic_pairs(512, seed=77)
    net = LearnedSeed(seed=3)
    net.fit_normalisation(cons, prims)
    g_gpu, loss_gpu = net.gradients(cons, prims)
    params = net.params()
    loss_cpu, g_cpu = mo.forward_backward(params[:mo.NPARAM], params[mo.NPARAM:].astype(np.float64),
                                          cons.cpu().numpy(), prims[1].cpu().numpy())
    assert abs(loss_gpu - loss_cpu) <= 1e-4 * abs(loss_cpu)
    for name, (o, n) in mo.OFF.items():
        a, b = g_gpu[o:o + n].astype(np.float64), g_cpu[o:o + n]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert err <= 2e-3, (name, err)
    net.close()


def test_training_reduces_loss(trained):
    net, first, last = trained
    assert last < 0.05 * first, (first, last)
    assert last < 5e-3


def test_network_seed_newton_judged_by_cardano(trained):
    """On held-out synthetic states the network seed + Newton reaches the
    pressure root; Cardano (the reference recovery) is the judge: both agree
    where Cardano itself is accurate, and the Newton answer satisfies the
    primitive->conserved map to round-off."""
    import torch
    from cueva.learned import CARDANO, NETWORK, synthetic_pairs
    net = trained[0]
    cons, prims = synthetic_pairs(200_000, seed=4321)
    out_n, it_n = net.c2p(NETWORK, cons, prims)
    out_c, _ = net.c2p(CARDANO, cons, prims)
    it = it_n.cpu().numpy()
    assert (it > 0).mean() > 0.999              # Newton converged from the network seed
    rel_p = (out_n[1] - prims[1]).abs() / prims[1]
    print(f"p rel error vs generator: median {float(torch.median(rel_p)):.2e}, 99% {float(torch.quantile(rel_p, 0.99)):.2e}")
    assert float(torch.quantile(rel_p, 0.99)) < 1e-7
    rel_pc = (out_n[1] - out_c[1]).abs() / out_c[1]
    print(f"network+Newton vs Cardano: median {float(torch.median(rel_pc)):.2e}, 99% {float(torch.quantile(rel_pc, 0.99)):.2e}")
    assert float(torch.median(rel_pc)) < 1e-6


def test_ablation_network_vs_plain_newton(trained):
    """What the network buys: Newton from its seed against the same Newton
    from the cold-start guess p = (gamma-1)/gamma (tau - |E|^2/2 - |B|^2/2 - D)."""
    import torch
    from cueva.learned import NETWORK, SEEDED, synthetic_pairs
    net = trained[0]
    cons, prims = synthetic_pairs(200_000, seed=999)
    Ef = cons[1] - 0.5 * (cons[5:11] ** 2).sum(0)
    cold = torch.clamp(0.25 * (Ef - cons[0]), min=1e-12)
    _, it_net = net.c2p(NETWORK, cons, prims)
    _, it_cold = net.c2p(SEEDED, cons, prims, seed=cold)
    n_net, n_cold = it_net.cpu().numpy(), it_cold.cpu().numpy()
    ok_net, ok_cold = (n_net > 0).mean(), (n_cold > 0).mean()
    mean_net = n_net[n_net > 0].mean()
    mean_cold = n_cold[n_cold > 0].mean() if (n_cold > 0).any() else float("inf")
    print(f"network seed: converged {ok_net:.4f}, mean iterations {mean_net:.2f}; "
          f"cold seed: converged {ok_cold:.4f}, mean iterations {mean_cold:.2f}")
    assert ok_net >= ok_cold
    assert mean_net < mean_cold


def test_learned_path_in_solver(oracle_mod, trained):
    """c2p = 2 inside the fused step, against the Cardano run of the same KH
    set-up; the Newton root and Cardano's approximate inversion differ at the
    round-off level of the latter."""
    from cueva import Cueva
    from cueva.learned import learned_stats
    net = trained[0]
    kw = dict(order=2, flux_solver=7, rec_mp=0, sigma=1e3)
    ref = Cueva(64, 32, c2p=1, **kw)
    lrn = Cueva(64, 32, c2p=2, **kw)
    for g in (ref, lrn):
        g.kh_init(v0=0.5, a=0.05)
        g.upload()
    net.attach(lrn)
    for g in (ref, lrn):
        g.step(20)
        g.download()
    r = {n: ref.interior(n) for n in PRIMS}
    for n in PRIMS:
        assert rel_l1_field(n, lrn.interior(n), r[n], r) <= 1e-6, n
    its, pts, fails = learned_stats(lrn)
    assert pts == 20 * 65 * 33
    assert fails <= pts // 1000
    print(f"learned path: {its / pts:.2f} Newton iterations per point, {fails} Cardano fall-backs")
    ref.close(); lrn.close()


def test_ablation_inside_a_run(trained):
    """Inside a time loop the previous step's pressure is already a seed (the
    reference's NR seed, 12_varprimitive_nr.f95:150-151).  On the states of a
    KH run (steps 10 -> 11): the previous pressure beats the network alone,
    and the step's seed choice (network or previous pressure by residual)
    needs about as few iterations as the previous pressure (within 0.05 per
    point; a smaller residual does not always mean fewer iterations) and
    fewer than the network alone.  After a restart whose pressures are off by 30 %, the
    previous pressure is a poor seed and the choice follows the network."""
    import torch
    from cueva import Cueva
    from cueva.learned import BEST, NETWORK, SEEDED, snapshot_pairs
    net = trained[0]
    g = Cueva(128, 64, order=2, flux_solver=7, sigma=1e3)
    g.kh_init(v0=0.5, a=0.05)
    g.upload()
    g.step(10)
    _, prims_n = snapshot_pairs(g)
    g.upload()           # re-prepare the state from the downloaded prims
    g.step(1)
    cons, prims = snapshot_pairs(g)
    prev = prims_n.contiguous()
    _, it_net = net.c2p(NETWORK, cons, prev)
    _, it_prev = net.c2p(SEEDED, cons, prev, seed=prims_n[1].contiguous())
    _, it_best = net.c2p(BEST, cons, prev)
    a, b, c = (x.cpu().numpy() for x in (it_net, it_prev, it_best))
    print(f"KH states: network seed {a.mean():.2f} iterations, previous-step seed {b.mean():.2f}, "
          f"seed choice {c.mean():.2f}")
    assert (a > 0).all() and (b > 0).all() and (c > 0).all()
    assert b.mean() < a.mean()
    assert c.mean() < a.mean() and c.mean() <= b.mean() + 0.05
    # a restart with the pressures off by 30 %
    bad = prev.clone()
    bad[1] *= 1.3
    _, it_bad_prev = net.c2p(SEEDED, cons, bad, seed=bad[1].contiguous())
    _, it_bad_best = net.c2p(BEST, cons, bad)
    d, e = it_bad_prev.cpu().numpy(), it_bad_best.cpu().numpy()
    print(f"pressures off by 30 %: previous-step seed {d[d > 0].mean():.2f} iterations "
          f"({(d <= 0).sum()} failed), seed choice {e.mean():.2f}")
    assert (e > 0).all()
    assert e.mean() < d[d > 0].mean()
    g.close()


def test_tensor_core_inference_matches_fp32(trained):
    """The warp-cooperative bf16 MMA forward (bf16 activations) against the
    per-thread FP32 forward of the same network: seeds agree to the bf16
    activation rounding, far inside what the Newton refinement absorbs."""
    import torch
    from cueva.learned import synthetic_pairs
    net = trained[0]
    cons, prims = synthetic_pairs(100_003, seed=555)     # not a multiple of 32: a partial last warp
    a = net.predict(cons, tensor_cores=True)
    b = net.predict(cons, tensor_cores=False)
    d = (torch.log(a) - torch.log(b)).abs()
    print(f"log-seed difference tensor cores vs FP32: median {float(d.median()):.2e}, max {float(d.max()):.2e}")
    assert float(d.median()) < 2e-2 and float(d.max()) < 0.5
    e = (torch.log(a) - torch.log(prims[1])).abs()
    assert float(e.median()) < 0.1


def test_tcgen05_inference_matches_fp32(trained):
    """The tcgen05 form (tiles of 128 states, accumulator in tensor memory,
    SiLU through tanh.approx) against the per-thread FP32 forward and the
    mma.sync form: the same network with bf16 activations, so the seeds
    agree to the activation rounding."""
    import torch
    from cueva.learned import synthetic_pairs
    net = trained[0]
    cons, prims = synthetic_pairs(100_003, seed=556)     # a partial last tile
    a = net.predict(cons, tensor_cores=2)
    b = net.predict(cons, tensor_cores=0)
    c = net.predict(cons, tensor_cores=1)
    assert torch.isfinite(a).all()
    d_fp32 = (torch.log(a) - torch.log(b)).abs()
    d_warp = (torch.log(a) - torch.log(c)).abs()
    print(f"tcgen05 log-seed difference: vs FP32 median {float(d_fp32.median()):.2e} max {float(d_fp32.max()):.2e}; "
          f"vs mma.sync median {float(d_warp.median()):.2e} max {float(d_warp.max()):.2e}")
    assert float(d_fp32.median()) < 2e-2 and float(d_fp32.max()) < 0.5
    assert float(d_warp.median()) < 5e-3 and float(d_warp.max()) < 0.2


@pytest.mark.parametrize("solver,order", [(7, 2), (5, 3)])
def test_learned_kernel_modes_agree(trained, solver, order):
    """The learned con2prim as a tcgen05 kernel after the last stage and
    inside the last stage: both Newton roots to 1e-12, so the runs agree far
    below the 1e-6 bar; both count every point once."""
    from cueva import Cueva
    from cueva.learned import learned_stats
    net = trained[0]
    kw = dict(order=order, flux_solver=solver, rec_mp=0, sigma=1e3, c2p=2)
    runs = []
    for mode in (1, 0):
        g = Cueva(45, 38, **kw)   # ragged: partial tiles of 128 points
        g.kh_init(v0=0.5, a=0.05)
        g.upload()
        net.attach(g)
        g.set_learned_kernel(mode)
        g.step(10)
        g.download()
        its, pts, fails = learned_stats(g)
        assert pts == 10 * 46 * 39 and fails <= pts // 1000, (mode, pts, fails)
        runs.append({n: g.interior(n).copy() for n in PRIMS})
        g.close()
    for n in PRIMS:
        assert rel_l1_field(n, runs[0][n], runs[1][n], runs[1]) <= 1e-9, n


def test_tcgen05_bounded_wait_reports_and_recovers(trained):
    """The timeout path of the tensor-core waits: in the self-test mode no
    MMA is issued, the bounded mbarrier wait runs out, the kernel frees its
    tensor memory and the call reports status 64; the next call works."""
    import torch
    from cueva import CuevaError
    from cueva.learned import synthetic_pairs
    net = trained[0]
    cons, _ = synthetic_pairs(10_000, seed=7)
    with pytest.raises(CuevaError) as e:
        net.predict(cons, tensor_cores=3)
    assert e.value.code == 4 and "64" in str(e.value)
    a = net.predict(cons, tensor_cores=2)
    b = net.predict(cons, tensor_cores=0)
    assert torch.isfinite(a).all()
    assert float((torch.log(a) - torch.log(b)).abs().median()) < 2e-2
