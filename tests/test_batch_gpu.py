"""A batch of uneven simulations stepped as one graph equals each
simulation stepped on its own, bit for bit: with the persistent work-queue
deposit and gather over all simulations (the default) and with one graph
branch per simulation."""
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
@pytest.mark.parametrize("queue", [1, 0])
def test_batch_equals_individual_steps(stream, queue):
    from mog_solver_b200.batch import Batch

    a = _sims()
    b = _sims()
    batch = Batch(a)
    batch.tune(work_queue=queue)
    assert batch.tuning()["active_work_queue"] == queue
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


@pytest.mark.parametrize("mass_mode,chunk,split", [("u64", 0, 0), ("u64", 4096, 0), ("u32x1000", 20000, 0),
                                                   ("u64", 0, 1), ("u64", 4096, 1), ("u64", 0, 2),
                                                   ("u64", 4096, 2)])
def test_work_queue_tiles_are_bit_exact(mass_mode, chunk, split):
    """Tile sizes that split every simulation into many deposit tiles (and
    a chunk that is not a multiple of the block), both mass modes, and the
    one-word histograms at every grid size (deposit_split 1: high words, the
    non-zero low halves of these masses as global atomics; 2: counts of each
    tile's first mass, the other masses as global atomics)."""
    from mog_solver_b200 import Simulation, ics
    from mog_solver_b200.batch import Batch

    def make():
        sims = []
        for i, (n, k, g) in enumerate([(30000, 7, 16), (9000, 13, 8), (12000, 5, 32), (1, 2, 16)]):
            s = Simulation({"n_grids": k, "grid_size": g, "world_size": 100.0, "num_particles": n,
                            "G": 100.0, "dt": 1e-3, "damping": 0.99, "seed": 30 + i,
                            "mass_mode": mass_mode})
            pos, vel = ics.clumps(n, 100.0, seed=40 + i)
            if mass_mode == "u32x1000":
                pos[:, 3] = 1.0
            vel[:, :3] = np.random.default_rng(i).normal(0, 1, (n, 3))
            s.set_particles(pos, vel)
            sims.append(s)
        return sims

    a, b = make(), make()
    batch = Batch(a)
    batch.tune(deposit_chunk=chunk, deposit_split=split)
    assert batch.tuning()["active_work_queue"] == 1 and batch.tuning()["deposit_split"] == split
    batch.step(4)
    for s in b:
        s.step(4)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x.pos, y.pos) and torch.equal(x.vel, y.vel)
        assert x.status() == y.status() == 0
    batch.close()


def test_work_queue_does_not_apply_to_mixed_mass_modes():
    from mog_solver_b200 import Simulation
    from mog_solver_b200.batch import Batch

    sims = [Simulation({"n_grids": 2, "grid_size": 8, "world_size": 100.0, "num_particles": 100,
                        "G": 1.0, "dt": 1e-3, "mass_mode": m}) for m in ("u64", "u32x1000")]
    for s in sims:
        s.init_particles("uniform")
    batch = Batch(sims)
    assert batch.tuning()["active_work_queue"] == 0
    batch.step(1)
    batch.close()
