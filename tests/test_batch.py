"""Batched scenes (pm_batch_*): the batched kernels give each scene the result of stepping it on
its own, scenes of different sizes and grids stay independent, a scene that outgrows its grid
inside a batch is regrown without holding the others back, and the autotuner keeps the
scenes in step.  The scene builders are checked on the CPU."""
import numpy as np
import pytest

from conftest import ROOT  # noqa: F401


def test_batch_scene_builder_ranges():
    from pigment_mixing_b200 import scenes
    b = scenes.batch_scenes(16, seed=3)
    n = np.array([len(s["x"]) for s in b])
    assert len(b) == 16
    assert n.min() >= 8 * 2 * 2 * 2 * 2 * 2 and n.max() <= 1.3 * 400000
    for s in b:
        g = round(1.0 / s["params"]["dx"])
        assert 64 <= g <= 160
        assert 50.0 <= s["params"]["q_max"] <= 200.0
        assert s["x"].min() >= 0.0 and s["x"].max() <= 1.0
        assert s["latent"].shape == (len(s["x"]), 7)
    again = scenes.batch_scenes(16, seed=3)
    assert all(np.array_equal(a["x"], c["x"]) for a, c in zip(b, again))
    assert len(scenes.RGB_SEEDS) == 6
    assert [len(s["x"]) for s in _small_scenes()] == [2 * 8 * 4 * c ** 3 for c in (4, 6, 7)]


def _small_scenes():
    from pigment_mixing_b200 import scenes
    return [scenes.palette_scene(3000, 48, (0, 1), 80.0, seed=1, steps=30),
            scenes.palette_scene(12000, 64, (2, 3), 150.0, seed=2, steps=30),
            scenes.palette_scene(25000, 80, (4, 5), 60.0, seed=3, steps=30)]


def _make(sc):
    from pigment_mixing_b200 import Simulation, scenes
    g = Simulation(0)
    scenes.apply(sc, g)
    g.prepareSimulation()
    return g


@pytest.mark.gpu
def test_batch_matches_scenes_stepped_alone():
    from pigment_mixing_b200 import Batch
    scs = _small_scenes()
    alone = [_make(s) for s in scs]
    for g in alone:
        g.advance(25)
    members = [_make(s) for s in scs]
    b = Batch(members)
    b.step(10)
    b.step(15)
    for g, m in zip(alone, members):
        assert m.steps_done == g.steps_done == 25
        pa = g.getParticles(fields=("x", "v", "latent"))
        pm = m.getParticles(fields=("x", "v", "latent"))
        # same kernels per scene; only the order of floating-point atomics differs
        assert np.abs(pa.x - pm.x).max() <= 1e-5
        assert np.abs(pa.latent - pm.latent).max() <= 1e-5
        assert np.abs(pa.v - pm.v).max() <= 1e-3 * max(1.0, np.abs(pa.v).max())
        assert m.errorFlags() == 0
        assert abs(float(m.time) - float(g.time)) <= 1e-9 * max(1.0, float(g.time))
    b.close()
    # members keep working on their own after the batch
    members[0].advance(2)
    assert members[0].steps_done == 27


@pytest.mark.gpu
def test_batch_member_matches_fp64_oracle():
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import Batch, scenes
    scs = _small_scenes()
    members = [_make(s) for s in scs]
    b = Batch(members)
    b.step(20)
    o = OracleSim(64)
    o.set(n_threads=8)
    scenes.apply(scs[0], o)
    o.prepare()
    o.advance(20)
    po = o.particles_f64()
    pg = members[0].getParticles(fields=("x", "latent"))
    assert np.abs(pg.x - po["x"]).max() <= 1e-4
    assert np.abs(pg.latent - po["latent"]).max() <= 1e-4
    b.close()


@pytest.mark.gpu
def test_batch_regrows_one_scene_and_keeps_the_others_in_step():
    """An expanding block outgrows its initial grid inside a batch; it sits rounds out while the
    host regrows it, and every scene still ends exactly n steps further."""
    from pigment_mixing_b200 import Batch, Simulation, scenes
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=5, steps=10, knife=False, material="vmvisc")
    sc["params"].update(plastic_model=0, E=1.0, rho=1000.0, particle_mass=1000.0 * (1.0 / 32) ** 3 / 8.0)
    sc["vectors"]["gravity"] = [0.0, 0.0, 0.0]
    sc["params"]["use_particle_boundaries"] = 0  # unbounded: the grid is sized from the blocks and must grow
    c = sc["x"].mean(0)
    c[1] = 0.0
    v = (3.0 * (sc["x"] - c)).astype(np.float32)

    def expanding():
        g = Simulation(0)
        scenes.apply(sc, g)
        g.setParticles(sc["x"], sc["latent"], v)
        g.prepareSimulation()
        return g

    alone = expanding()
    alone.advance(82)
    grow = expanding()
    nodes0 = grow.grid_capacity_nodes
    other = _make(_small_scenes()[1])
    other_alone = _make(_small_scenes()[1])
    other_alone.advance(82)
    b = Batch([grow, other])
    b.step(82)
    assert grow.steps_done == 82 and other.steps_done == 82
    assert int(grow.regrowths) >= 1 and grow.grid_capacity_nodes > nodes0
    pa, pb = alone.getParticles(fields=("x",)), grow.getParticles(fields=("x",))
    assert np.abs(pa.x - pb.x).max() <= 1e-5
    pa, pb = other_alone.getParticles(fields=("x",)), other.getParticles(fields=("x",))
    assert np.abs(pa.x - pb.x).max() <= 1e-5
    b.close()


@pytest.mark.gpu
def test_batch_autotune_and_profile():
    from pigment_mixing_b200 import Batch
    members = [_make(s) for s in _small_scenes()]
    b = Batch(members)
    t0 = b.tuning()
    best, ms = b.autotune(trial_rounds=2)
    assert ms > 0.0
    assert best["flat_threads"] in (128, 256, 512)
    steps = [m.steps_done for m in members]
    assert len(set(steps)) == 1 and steps[0] > 0  # autotuning advances all scenes alike
    prof = b.profile(2)
    assert "kb_p2g" in prof and "kb_defgrad_tail" in prof and len(prof) == b.kernels_per_round
    assert all(v >= 0.0 for v in prof.values())
    b.step(3)
    assert len({m.steps_done for m in members}) == 1
    assert set(t0) == set(best)
    b.close()


@pytest.mark.gpu
def test_batch_with_learned_return_map():
    """Scenes on the surrogate return map inside a batch: the batched inference and finish
    passes run, and positions stay within the parity tolerance of the plain batch."""
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Batch, Simulation, scenes, surrogate
    scs = _small_scenes()
    log = Simulation(0)
    scenes.apply(scs[2], log)
    log.enableSampleLog(1 << 20)
    log.prepareSimulation()
    log.advance(30)
    xs, ys = log.samples()
    log.close()
    params, _ = surrogate.train(xs, ys, epochs=8, batch=4096, lr=3e-3, seed=0)
    plain = [_make(s) for s in scs]
    sur = []
    for s in scs:
        g = Simulation(0)
        scenes.apply(s, g)
        g.setSurrogate(params)
        g.setReturnMap(RETURN_MAP_SURROGATE)
        g.prepareSimulation()
        sur.append(g)
    bp, bs = Batch(plain), Batch(sur)
    assert bs.kernels_per_round == bp.kernels_per_round + 2
    bp.step(20)
    bs.step(20)
    for a, c in zip(plain, sur):
        pa, pc = a.getParticles(fields=("x", "latent")), c.getParticles(fields=("x", "latent"))
        assert np.abs(pa.x - pc.x).max() <= 1e-3
        assert np.abs(pa.latent - pc.latent).max() <= 1e-3
    st = sur[2].returnMapStats()
    assert st["solves"] > 0
    bp.close()
    bs.close()
