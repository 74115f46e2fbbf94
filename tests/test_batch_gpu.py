"""A batch of uneven simulations stepped as one graph equals each
simulation stepped on its own, bit for bit."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SPECS = [(20000, 16, 16), (70000, 24, 16), (5000, 8, 32), (1000, 3, 8)]


def _sims(seed_base=0):
    from mog_solver_b200 import Simulation, ics

    sims = []
    for i, (n, k, g) in enumerate(SPECS):
        s = Simulation({"n_grids": k, "grid_size": g, "world_size": 100.0, "num_particles": n,
                        "G": 100.0, "dt": 1e-3, "damping": 0.999, "seed": 10 + i})
        pos, vel = ics.plummer(n, 100.0, seed=seed_base + i)
        vel[:, :3] = np.random.default_rng(i).normal(0, 1, (n, 3))
        s.set_particles(pos, vel)
        sims.append(s)
    return sims


@pytest.mark.parametrize("stream", ["default", "side"])
def test_batch_equals_individual_steps(stream):
    from mog_solver_b200.batch import Batch

    a = _sims()
    b = _sims()
    batch = Batch(a)
    if stream == "side":
        st = torch.cuda.Stream()
        st.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(st):
            batch.step(3)
            batch.step(2)
        st.synchronize()
    else:
        batch.step(5)
    for s in b:
        for _ in range(5):
            s.step()
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x.pos, y.pos) and torch.equal(x.vel, y.vel)
    batch.close()


def test_autotune_keeps_results_bit_exact(tmp_path):
    from mog_solver_b200 import Simulation, ics
    from mog_solver_b200.autotune import autotune

    def make():
        s = Simulation({"n_grids": 24, "grid_size": 16, "world_size": 100.0, "num_particles": 200000,
                        "G": 100.0, "dt": 1e-3, "seed": 4})
        pos, vel = ics.plummer(200000, 100.0, seed=4)
        s.set_particles(pos, vel)
        return s

    a, b = make(), make()
    entry = autotune(a, reps=2, cache=tmp_path / "t.json")
    assert (tmp_path / "t.json").exists() and "tuning" in entry
    assert torch.equal(a.pos, b.pos)  # tuning restored the particles it advanced
    for _ in range(3):
        a.step()
        b.step()
    torch.cuda.synchronize()
    assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
