"""Learned return-map surrogate: oracle self-check (CPU), GPU training kernels against the
oracle, tensor-core inference, and what the trained network gains inside the step (GPU)."""
import numpy as np
import pytest

from oracle import mlp_ref


def _batch(n=256, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 10)) * np.array([0.01, 0.01, 0.01, 5, 5, 5, 30, 0.01, 0.1, 1e4]) + \
        np.array([0, 0, 0, 0, 0, 0, 100, 0.02, 0.6, 5e4])
    t = rng.normal(size=(n, 6)) * np.array([1e-3, 1e-3, 1e-3, 1, 1, 1])
    return x.astype(np.float32), t.astype(np.float32)


def test_oracle_gradient_matches_finite_differences():
    x, t = _batch(64)
    p = mlp_ref.init_params(x, t, seed=1).astype(np.float64)
    loss, g = mlp_ref.loss_grad(p, x, t)
    rng = np.random.default_rng(2)
    idx = np.concatenate([rng.integers(mlp_ref.O_W1, mlp_ref.NPARAMS, 40), [mlp_ref.O_B3, mlp_ref.O_B1]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp_ref.loss_grad(pp, x, t)[0] - mlp_ref.loss_grad(pm, x, t)[0]) / (2 * h)
        assert fd == pytest.approx(g[i], rel=1e-5, abs=1e-9), i


@pytest.mark.gpu
def test_gpu_training_gradients_match_oracle():
    """pm_mlp_loss_grad (the GPU training kernels, FP32) against the float64 oracle."""
    from pigment_mixing_b200 import surrogate
    x, t = _batch(1000, seed=3)
    p = mlp_ref.init_params(x, t, seed=4)
    loss_g, g_g = surrogate.loss_grad(p, x, t)
    loss_o, g_o = mlp_ref.loss_grad(p.astype(np.float64), x, t)
    assert loss_g == pytest.approx(loss_o, rel=1e-4)
    trained = slice(32, mlp_ref.NPARAMS)
    err = np.abs(g_g[trained] - g_o[trained]).max() / np.abs(g_o[trained]).max()
    assert err < 1e-4, err


@pytest.mark.gpu
def test_tensor_core_inference_matches_fp32_oracle():
    """BF16 mma inference against the float64 forward pass (BF16 operands, FP32 accumulation)."""
    from pigment_mixing_b200 import surrogate
    x, t = _batch(999, seed=5)
    p = mlp_ref.init_params(x, t, seed=6)
    y_gpu = surrogate.infer(p, x)
    y_ref = mlp_ref.predict(p.astype(np.float64), x)
    osd = p[mlp_ref.O_OS:mlp_ref.O_OS + 6]
    err = np.abs((y_gpu - y_ref) / osd).max()  # in units of the output standard deviation
    assert err < 0.05, err


@pytest.mark.gpu
def test_trained_surrogate_gains_over_plain_return_map():
    """Log samples from the plain solver, train on the GPU, then step the same state both ways:
    the surrogate path needs far fewer Newton updates, every estimate is checked against the
    Perzyna consistency condition, and positions and latents stay within the parity tolerance."""
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Simulation, scenes, surrogate
    sc = scenes.config1(seed=0)
    log = Simulation(0)
    scenes.apply(sc, log)
    log.enableSampleLog(1 << 21)
    log.prepareSimulation()
    log.advance(60)
    x, y = log.samples()
    assert len(x) > 50000
    p, hist = surrogate.train(x, y, epochs=12, batch=4096, lr=3e-3, seed=0)
    assert hist[-1] < 0.2 * hist[0], hist
    sims = {}
    for mode in ("plain", "surrogate"):
        s = Simulation(0)
        scenes.apply(sc, s)
        if mode == "surrogate":
            s.setSurrogate(p)
            s.setReturnMap(RETURN_MAP_SURROGATE)
        s.prepareSimulation()
        s.advance(20)
        iters = solves = accepted = 0
        for _ in range(10):
            s.advance(1)
            st = s.returnMapStats()
            iters += st["newton_iters"]
            solves += st["solves"]
            accepted += st["accepted"]
        sims[mode] = (s, iters, solves, accepted)
    _, it_p, sv_p, _ = sims["plain"]
    _, it_s, sv_s, acc_s = sims["surrogate"]
    assert sv_p > 0 and sv_s > 0
    assert it_s < 0.7 * it_p, (it_s, it_p)  # observed about 0.5 after 12 epochs
    pp = sims["plain"][0].getParticles(fields=("x", "latent"))
    ps = sims["surrogate"][0].getParticles(fields=("x", "latent"))
    assert np.abs(pp.x - ps.x).max() <= 1e-3
    assert np.abs(pp.latent - ps.latent).max() <= 1e-3
