"""The learned cooling step: labels, gradients against the CPU oracle, training, and inference
with its hull and a-posteriori checks (the network has no counterpart in the reference)."""

import time

import numpy as np
import pytest

from oracle import cooling as ocool
from oracle import mlp as omlp
from tests.conftest import check


def test_bf16_rounding_matches_torch():
    import torch

    x = np.random.default_rng(0).normal(size=4096).astype(np.float32) * 10
    ref = torch.tensor(x).to(torch.bfloat16).to(torch.float32).numpy()
    check("bf16 round to nearest even", ref, omlp.bf16_round(x))


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    w = rng.normal(0, 0.3, 8641)
    X = rng.uniform(-1, 1, (64, 3))
    Y = rng.uniform(0, 1, 64)
    loss, g = omlp.loss_and_grad(w, X, Y)
    # biases are not rounded, so their finite differences check the backward pass exactly
    for k in (8640, 192 + 5, 192 + 64 + 4096 + 7):
        e = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[k] += e
        wm[k] -= e
        fd = (omlp.loss_and_grad(wp, X, Y)[0] - omlp.loss_and_grad(wm, X, Y)[0]) / (2 * e)
        check(f"d loss / d w[{k}]", fd, g[k], rtol=1e-6, atol=1e-10)


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import _lib, cooling
    from blackhole_nebula_simulator_b200.device import ctx, ptr, stream

    return _lib, cooling, ctx, ptr, stream


@pytest.mark.gpu
def test_labels_match_exact_integrator(gpu):
    import torch

    _lib, cooling, ctx, ptr, stream = gpu
    prm = cooling.mlp_params()
    n = 20000
    X = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    Y = torch.empty(n, dtype=torch.float32, device="cuda")
    U = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    c = ctx()
    _lib.check(c, _lib.lib().nb_mlp_data(c, n, 7, prm, ptr(X), ptr(Y), ptr(U), stream()))
    u, rho, dt = U.cpu().numpy().T
    consts = ocool.brems_constants()
    check("labels = exact f", omlp.label(u, rho, dt, consts), Y.cpu().numpy(), atol=2e-7)
    assert np.all(np.abs(X.cpu().numpy()) <= 1.0 + 1e-6)


@pytest.mark.gpu
def test_gradients_match_oracle(gpu):
    import torch

    _lib, cooling, ctx, ptr, stream = gpu
    rng = np.random.default_rng(3)
    w = rng.normal(0, 0.25, 8641).astype(np.float32)
    X = rng.uniform(-1, 1, (1000, 3)).astype(np.float32)
    Y = rng.uniform(0, 1, 1000).astype(np.float32)
    wt, Xt, Yt = (torch.tensor(a, device="cuda") for a in (w, X, Y))
    g = torch.empty(8641, dtype=torch.float32, device="cuda")
    loss = __import__("ctypes").c_double(0)
    c = ctx()
    _lib.check(c, _lib.lib().nb_mlp_grad(c, 1000, ptr(Xt), ptr(Yt), ptr(wt), ptr(g),
                                         __import__("ctypes").byref(loss), stream()))  # fmt: skip
    ref_loss, ref_g = omlp.loss_and_grad(w, X, Y)
    check("loss", ref_loss, loss.value, rtol=1e-5)
    gn = np.abs(ref_g).max()
    check("gradient (relative to its largest entry)", ref_g / gn, g.cpu().numpy() / gn, atol=2e-5)


@pytest.mark.gpu
def test_training_inference_checks_and_gain(gpu):
    """Train on 4M samples, then: accepted network results within 1e-3 u of the exact integrator,
    inputs outside the hull and failed checks fall back to it, and the time of the network step
    beside the exact step on the same 4M particles: the network is the slower (a net cost)."""
    import torch

    _lib, cooling, ctx, ptr, stream = gpu
    net = cooling.train_network(n_samples=4 * 2**20, batch=65536, epochs=12, lr=3e-3, seed=11)
    assert net.loss_history[-1] < net.loss_history[0]
    consts = cooling.brems_constants()
    rng = np.random.default_rng(12)
    n = 4 * 2**20
    h = cooling.Hull()
    lr = rng.uniform(*h.lrho, n)
    lt = rng.uniform(*h.lt, n)
    ld = rng.uniform(*h.ldt, n)
    p = net.params
    rho = 10**lr / p.rho_unit_cgs
    u = 10**lt / consts.tfac
    dt = 10**ld / p.t_unit_s
    u_t, rho_t, dt_t = (torch.tensor(a, device="cuda") for a in (u, rho, dt))
    out, mode = cooling.mlp_cool(u_t, rho_t, dt_t, net)
    exact = cooling.brems_cool(u_t, rho_t, dt_t, consts)
    err = (torch.abs(out - exact) / u_t).cpu().numpy()
    m = mode.cpu().numpy()
    frac_net = float(np.mean(m == 1))
    print(f"network used for {frac_net:.3f} of hull samples, fallback {np.mean(m == 2):.3f}")
    assert frac_net > 0.2
    # accepted results are within 2 check_tol = 1e-3 of u by construction of the check
    check("accepted network results vs exact (|du| / u)", 0.0, err[m == 1].max(), atol=1e-3)
    check("fallback results are exact", 0.0, err[m == 2].max() if np.any(m == 2) else 0.0, atol=1e-12)
    # outside the hull: exact
    out2, mode2 = cooling.mlp_cool(u_t[:1000] * 1e7, rho_t[:1000], dt_t[:1000], net)
    assert not np.any(mode2.cpu().numpy() == 1)
    # time per particle of the two methods on the same particles
    times = {}
    for name, fn in (("exact", lambda: cooling.brems_cool(u_t, rho_t, dt_t, consts)),
                     ("network", lambda: cooling.mlp_cool(u_t, rho_t, dt_t, net))):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        times[name] = (time.perf_counter() - t0) / 5
    print(f"exact {times['exact'] * 1e3:.3f} ms, network {times['network'] * 1e3:.3f} ms "
          f"per {n} particles: gain x{times['exact'] / times['network']:.2f}")
    # What the network gains: nothing in time.  The exact integrator of this bremsstrahlung law
    # is a closed form (an arctangent falling linearly in rho dt), so one evaluation per
    # particle beats the network's four layers and its a-posteriori check; the bench line and
    # the design notes state the network as a net cost, and this is the measurement behind it.
    check("the network costs more than the closed-form exact integrator", True,
          times["network"] > times["exact"])  # fmt: skip
