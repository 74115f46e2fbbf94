"""The learned correction on the GPU against the FP64 oracle (oracle/mlp.py):
gradients of the fused training kernel, one Adam step, FP16 tensor-core
inference, the feature gather, and what training gains over the plain
cheap ensemble."""
import numpy as np
import pytest

import oracle
from oracle import mlp, pipeline as pl

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _model(seed=0, base_mode=0):
    from mog_solver_b200.learned import Model, norm_vector

    p = (mlp.init(seed) + np.random.default_rng(seed).normal(0, 0.05, mlp.N_PARAMS)).astype(np.float32)
    return Model(p, norm_vector(np.zeros(12), np.ones(12), 1.0, 1.0, 1.0, base_mode)), p


def _batch(n, seed=0):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 16), np.float32)
    x[:, :12] = rng.normal(0, 1, (n, 12))
    t = np.zeros((n, 4), np.float32)
    t[:, :3] = rng.normal(0, 1, (n, 3))
    return x, t


@pytest.mark.parametrize("batch", [1, 100, 128, 1000])
def test_gradient_matches_fp64_oracle(batch):
    m, p = _model(1)
    x, t = _batch(batch + 50, seed=batch)
    idx = np.random.default_rng(3).choice(batch + 50, batch, replace=False).astype(np.int32)
    X, T, I = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(idx).cuda()
    grad = torch.empty(mlp.N_PARAMS, dtype=torch.float32, device="cuda")
    loss = m.train_step(X, T, I, lr=0.0, want_loss=True, grad_out=grad)
    ref_loss, ref_grad = mlp.loss_and_grad(p.astype(np.float64), x[idx, :12].astype(np.float64),
                                           t[idx, :3].astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-5 * max(1, ref_loss)
    g = grad.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - ref_grad) <= 1e-4 * np.linalg.norm(ref_grad)
    m.close()


def test_adam_step_matches_fp64():
    m, p = _model(2)
    x, t = _batch(512, seed=9)
    idx = np.arange(512, dtype=np.int32)
    X, T, I = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(idx).cuda()
    lr = 1e-3
    m.train_step(X, T, I, lr=lr)
    _, g = mlp.loss_and_grad(p.astype(np.float64), x[:, :12].astype(np.float64), t[:, :3].astype(np.float64))
    mm = 0.1 * g
    vv = 0.001 * g * g
    ref = p - lr * (mm / 0.1) / (np.sqrt(vv / 0.001) + 1e-8)
    got, _ = m.get()
    # lr * g / (|g| + eps) is ill-conditioned where g ~ 0: compare elsewhere
    live = np.abs(g) > 1e-4 * np.abs(g).max()
    assert np.abs(got - ref)[live].max() <= 1e-5
    assert np.abs(got - p).max() <= lr * 1.0001
    m.close()


@pytest.mark.parametrize("base_mode", [0, 1])
def test_fp16_inference_matches_fp64_forward(base_mode):
    from mog_solver_b200 import Simulation
    from mog_solver_b200.learned import features, learned_forces

    n, k, g, L = 5000, 8, 16, 100.0
    m, p = _model(4, base_mode)
    sim = Simulation({"n_grids": k, "grid_size": g, "world_size": L, "num_particles": n, "G": 100.0,
                      "dt": 1e-5, "seed": 3})
    rng = np.random.default_rng(4)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0, L, (n, 3))
    pos[:, 3] = 1.0 / n
    sim.set_particles(pos)
    mean, feat = features(sim, m)
    acc = learned_forces(sim, m)
    y, _ = mlp.forward(p.astype(np.float64), feat.cpu().numpy()[:, :12].astype(np.float64))
    base = mean.cpu().numpy()[:, :3].astype(np.float64)
    if base_mode:
        base = base + feat.cpu().numpy()[:, 12:15].astype(np.float64)
    ref = base + y
    got = acc.cpu().numpy()[:, :3].astype(np.float64)
    # FP16 weights and activations, GELU in FP16: a few parts in 1e3 of the output scale
    assert np.abs(got - ref).max() <= 2e-2 * max(1.0, np.abs(y).max())
    assert pl.relative_l2(got - base, y) < 2e-2
    sim.close()
    m.close()


def test_features_match_fp64_oracle():
    from mog_solver_b200 import Simulation
    from mog_solver_b200.learned import Model, features, norm_vector

    n, k, g, L, G = 20000, 8, 16, 100.0, 100.0
    sim = Simulation({"n_grids": k, "grid_size": g, "world_size": L, "num_particles": n, "G": G,
                      "dt": 1e-5, "seed": 5})
    rng = np.random.default_rng(5)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.mod(rng.normal(50, 12, (n, 3)), L)
    pos[:, 3] = 1.0 / n
    sim.set_particles(pos)
    fs, rho_ref = 0.3, 1.0 / g ** 3
    mu = rng.normal(0, 0.1, 12)
    isd = rng.uniform(0.5, 2, 12)
    m = Model(norm=norm_vector(mu, isd, fs, rho_ref, 1.0))
    mean, feat = features(sim, m)
    # plain mean force: bit-identical to the plain path
    assert torch.equal(mean[:, :3], sim.forces()[:, :3])
    mass = sim.mass_grid().cpu().numpy().view(np.uint64).astype(np.float64) * 2.0 ** -sim.scale_bits
    F = sim.solve_grid(sim.mass_grid()).cpu().numpy()[..., :3].astype(np.float64).reshape(k, -1, 3)
    M = pl.rotations_fp64(sim.rotations)
    Fw = np.einsum("kab,kcb->kca", M, F)
    cells = oracle.cells(pos, sim.rotations, sim.offsets, g, L)
    rows = oracle.fast_rows(sim.rotations, sim.offsets, L, g).astype(np.float64).reshape(k, 3, 4)
    c = pos[:, :3].astype(np.float64) - L / 2
    t = np.einsum("krj,nj->nkr", rows[:, :, :3], c) + rows[:, :, 3][None]
    ref, ref_mean, ref_corr = mlp.features(cells, Fw, mass.reshape(k, -1), t, sim.rotations, L / g,
                                           {"force_scale": fs, "rho_ref": rho_ref, "mu": mu,
                                            "inv_sigma": isd})
    got = feat.cpu().numpy()[:, :12].astype(np.float64)
    err = np.abs(got - ref)
    assert np.quantile(err, 0.999) < 1e-3 * (1 + np.abs(ref).max())
    corr = feat.cpu().numpy()[:, 12:15].astype(np.float64)
    assert np.quantile(np.abs(corr - ref_corr), 0.999) < 1e-3 * fs * (1 + np.abs(ref_corr / fs).max())
    assert np.abs(feat.cpu().numpy()[:, 15]).max() == 0
    sim.close()
    m.close()


def test_network_gains_over_least_squares_alone():
    """The committed network against the method without it: the cheap
    ensemble's mean plus its least-squares correction (the network's output
    zeroed).  Against the k = 240 force, on a clump set held out of training
    and on the evaluation disks (N = 2^20 each), the learned force must be
    closer than least squares alone, which must be closer than the plain
    k = 32 mean."""
    from mog_solver_b200 import ics
    from mog_solver_b200.learned import Model, residual_errors
    from mog_solver_b200.train_learned import DEFAULT_MODEL

    model = Model.load(DEFAULT_MODEL)
    try:
        sets = [ics.clumps(1 << 20, 100.0, seed=901)[0], ics.two_disks(1 << 20, 100.0, seed=1)[0]]
        rows = residual_errors(model, sets, alphas=(1.0,))
    finally:
        model.close()
    for name, r in zip(("held-out clumps", "disks"), rows):
        assert r["net_x1"] < r["ls"] < r["plain"], (name, r)


def test_training_gains_over_plain_cheap_ensemble():
    """Train briefly on clump sets; on held-out particles the corrected
    k=16 force is closer to the k=128 force than the plain k=16 mean is."""
    from mog_solver_b200 import Simulation, ics
    from mog_solver_b200.learned import Model, generate_dataset, learned_forces, train

    data = generate_dataset(n_sets=4, n=65536, k_small=16, k_big=128, seed0=500)
    model = Model(seed=0)
    hist = train(model, data, steps=400, batch=4096, lr=2e-3)
    assert hist[-1][1] < hist[0][1]
    n, L = 65536, 100.0
    small = Simulation({"n_grids": 16, "grid_size": 16, "world_size": L, "num_particles": n,
                        "G": 100.0, "dt": 1e-5, "seed": 1000})
    big = Simulation({"n_grids": 128, "grid_size": 16, "world_size": L, "num_particles": n,
                      "G": 100.0, "dt": 1e-5, "seed": 2000})
    pos, _ = ics.clumps(n, L, seed=999)
    small.set_particles(pos)
    big.set_particles(pos)
    ref = big.forces()[:, :3].double()
    plain = small.forces()[:, :3].double()
    corrected = learned_forces(small, model)[:, :3].double()
    e_plain = float(torch.linalg.norm(plain - ref) / torch.linalg.norm(ref))
    e_learned = float(torch.linalg.norm(corrected - ref) / torch.linalg.norm(ref))
    assert e_learned < e_plain, (e_learned, e_plain)
    small.close()
    big.close()
    model.close()


def _clump_sim(k, n=20000, seed=7):
    from mog_solver_b200 import Simulation, ics

    sim = Simulation({"n_grids": k, "grid_size": 16, "world_size": 100.0, "num_particles": n,
                      "G": 100.0, "dt": 1e-5, "seed": seed})
    pos, _ = ics.clumps(n, 100.0, seed=seed)
    sim.set_particles(pos)
    return sim


def test_step_statistics_match_feature_pass():
    """The force spread and mean-force magnitude summed inside
    mog_learned_step are the means that mog_features gives for the same
    positions."""
    from mog_solver_b200.learned import LearnedSimulation

    sim = _clump_sim(16)
    m, _ = _model(5)
    ls = LearnedSimulation(sim, m)
    before = ls.feature_stats()
    ls.step()
    after = ls.step_stats()
    assert before[0] > 0 and before[1] > 0
    for a, b in zip(after, before):
        assert abs(a - b) <= 1e-4 * b
    sim.close()
    m.close()


def test_learned_step_profiled_matches_step():
    import ctypes

    from mog_solver_b200 import _lib

    a, b = _clump_sim(16), _clump_sim(16)
    m, _ = _model(6)
    lib = _lib.lib()
    ph = (ctypes.c_float * 4)()
    for _ in range(3):
        _lib.check(lib.mog_learned_step(a.handle, m.handle, a.pos.data_ptr(), a.vel.data_ptr(),
                                        a.n_particles, 1e-3, None), "step")
        _lib.check(lib.mog_learned_step_profiled(b.handle, m.handle, b.pos.data_ptr(),
                                                 b.vel.data_ptr(), b.n_particles, 1e-3, ph, None),
                   "profiled")
    torch.cuda.synchronize()
    assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
    assert all(v >= 0 for v in ph) and ph[3] > 0
    a.close()
    b.close()
    m.close()


@pytest.mark.parametrize("factor,expect_fallback", [(0.0, True), (1e9, False)])
def test_variance_gate(factor, expect_fallback):
    """gate_factor 0 hands every step after a gate check to the plain
    expensive ensemble; a huge factor never does."""
    from mog_solver_b200.learned import LearnedSimulation

    cheap, big = _clump_sim(16), _clump_sim(64)
    m, _ = _model(7)
    ls = LearnedSimulation(cheap, m, fallback=big, train_ratio=1.0, gate_factor=factor,
                           gate_every=2)
    ls.step(6)
    torch.cuda.synchronize()
    assert ls.steps == 6
    assert (ls.fallback_steps == 4) if expect_fallback else (ls.fallback_steps == 0)
    assert torch.isfinite(ls.pos).all()
    cheap.close()
    big.close()
    m.close()
