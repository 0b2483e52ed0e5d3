"""The reference's set-up path through the C ABI: its own configuration files through the JSON
readers, its full knife animation through pm_add_spatula_file, the render loop's
step / frameFinished / isFinished idiom, and setupScene's blob scene (pm_setup_scene_blobs).

Fixtures (tests/golden, written by make_golden.py from the reference tree): sim_config.json and
pigment_config.json (matter/), spatula_motion.bin (matter/animations/, 3,601 frames).
"""
import json
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

SIM_CFG = os.path.join(GOLDEN, "sim_config.json")
PIG_CFG = os.path.join(GOLDEN, "pigment_config.json")
ANIM = os.path.join(GOLDEN, "spatula_motion.bin")


def _sim():
    from pigment_mixing_b200 import Simulation
    return Simulation(0)


def test_reference_config_files_through_the_json_readers():
    """simulation_units.cpp:31-64: every key of the reference's two files lands in its field
    (friction_angle as M = tan(angle)); keys the files leave out keep the readers' defaults."""
    g = _sim()
    g.loadPigmentConfig(PIG_CFG)
    g.loadSimConfig(SIM_CFG)
    pig = json.load(open(PIG_CFG))
    cfg = json.load(open(SIM_CFG))
    pig_fields = dict(D_max="pigment_D_max", D_edge0="pigment_D_edge0", D_edge1="pigment_D_edge1",
                      start_boost_time="start_boost_time", end_boost_time="end_boost_time",
                      boost_factor="boost_factor")
    pig_default = dict(D_max=0.1, D_edge0=0.5, D_edge1=0.8, start_boost_time=20.0, end_boost_time=40.0,
                       boost_factor=2.0)
    for key, field in pig_fields.items():
        assert g.param(field) == pytest.approx(pig.get(key, pig_default[key]), rel=1e-12), key
    sim_default = dict(cfl=0.2, flip_ratio=-0.8, E=5e5, nu=0.3, rho=1000.0, q_cohesion=500.0, perzyna_exp=1.0,
                       perzyna_visc=0.1)
    for key, d in sim_default.items():
        assert g.param(key) == pytest.approx(cfg.get(key, d), rel=1e-12), key
    assert g.param("M") == pytest.approx(math.tan(math.radians(cfg.get("friction_angle", 5.0))), rel=1e-12)
    g.close()


def test_json_readers_absent_keys_and_missing_files(tmp_path):
    """An absent key takes the reader's default; a missing sim_config.json applies the reference's
    file-missing defaults (simulation_units.cpp:66-80); a missing pigment file keeps the fields;
    a malformed file is an error (PM_ERR_IO)."""
    from pigment_mixing_b200._lib import PMError
    g = _sim()
    p = tmp_path / "partial.json"
    p.write_text('{"E": 1234.5, "D_max": 7}')
    g.set(cfl=0.9, flip_ratio=-1.5)
    g.loadSimConfig(str(p))
    assert g.param("E") == 1234.5 and g.param("cfl") == pytest.approx(0.2) and g.param("flip_ratio") == pytest.approx(-0.8)
    assert g.param("M") == pytest.approx(math.tan(math.radians(5.0)))
    g.loadPigmentConfig(str(p))
    assert g.param("pigment_D_max") == 7 and g.param("pigment_D_edge0") == pytest.approx(0.5)
    g.set(cfl=0.9)
    g.loadSimConfig(str(tmp_path / "absent.json"))
    assert g.param("cfl") == pytest.approx(0.2) and g.param("E") == pytest.approx(5e5)
    g.set(pigment_D_max=3.0)
    g.loadPigmentConfig(str(tmp_path / "absent.json"))
    assert g.param("pigment_D_max") == 3.0
    bad = tmp_path / "bad.json"
    bad.write_text('{"E": }')
    with pytest.raises(PMError):
        g.loadSimConfig(str(bad))
    g.close()


def test_setup_scene_with_reference_files_and_full_animation():
    """pm_setup_scene with the reference's files and knife: setupScene's fixed settings
    (simulation_units.cpp:82-131) are applied and the knife is the animated spatula."""
    from pigment_mixing_b200 import scenes
    g = _sim()
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=1, steps=5, knife=False, material="dpvisc")
    g.setParticles(sc["x"] - np.float32([0.5, 0.0, 0.5]), sc["latent"])
    g.set(dx=sc["params"]["dx"], particle_volume=sc["params"]["particle_volume"],
          particle_mass=sc["params"]["particle_mass"])
    g.setupScene(60.0, PIG_CFG, SIM_CFG, ANIM)
    assert g.param("end_frame") == 1800 and g.param("fps") == 60.0
    assert g.param("plastic_model") == 6 and g.param("use_pradhana") == 1
    assert g.param("q_prefac") == pytest.approx(1.0 / math.sqrt(2.0))
    g.prepareSimulation()
    g.advance(10)
    assert g.getSpatulaObject() is not None
    p = g.getParticles(fields=("x", "active"))
    assert np.isfinite(p.x).all() and p.active.all()
    assert g.errorFlags() == 0
    g.close()


def test_spatula_file_full_animation_matches_oracle():
    """pm_add_spatula_file on the whole 3,601-frame animation: one-second steps (no gravity, a soft
    material, fps 1) walk the knife through every part of the file and past its end (the last
    frame holds); its pose equals the FP64 oracle's, given the same frames, at every step."""
    from oracle.oracle import OracleSim
    frames = np.fromfile(ANIM, dtype=np.float32).reshape(-1, 7)
    assert frames.shape == (3601, 7)
    dx = 0.1
    x = (np.stack(np.meshgrid(*[np.arange(2)] * 3, indexing="ij"), -1).reshape(-1, 3) * 0.05 + [3.0, 0.2, 3.0])
    x = x.astype(np.float32)
    lat = np.tile(np.float32([1, 0, 0, 0, 0, 0, 0]), (len(x), 1))
    params = dict(E=1e-2, rho=1000.0, nu=0.3, fps=1.0, end_frame=10000, dx=dx, particle_volume=dx ** 3 / 8,
                  particle_mass=1000.0 * dx ** 3 / 8, flip_ratio=-1.5)
    g = _sim()
    g.setParticles(x, lat)
    g.set(**params)
    g.addSpatula(2, 0.0, anim_path=ANIM)
    g.prepareSimulation()
    o = OracleSim(64)
    o.set_particles(x, lat)
    o.set(**params)
    o.add_spatula(2, 0.0, frames)
    o.prepare()
    for k in range(62):
        g.advance(1)
        o.advance(1)
        assert g.time == pytest.approx(o.get("time"), rel=1e-12)
        kg, ko = g.getSpatulaObject()[0], o.knife()[0]
        assert np.allclose(kg, ko, atol=2e-5), (k, np.abs(kg - ko).max())
    assert g.time > len(frames) / 60.0
    g.close()


def test_render_loop_matches_oracle():
    """The render loop (raytracing/src/main.cpp:270-285, simulation_units.cpp:217-245):
    step(); frameFinished(); until isFinished(): same steps, frames and state as the oracle."""
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import scenes
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=7, steps=10)
    sc["params"]["end_frame"] = 3
    g = _sim()
    scenes.apply(sc, g)
    g.prepareSimulation()
    o = OracleSim(64)
    o.set(n_threads=4)
    scenes.apply(sc, o)
    o.prepare()
    steps_g = frames_g = 0
    while not g.isFinished():
        g.step()
        steps_g += 1
        frames_g += int(g.frameFinished())
        assert steps_g < 1000
    steps_o = frames_o = 0
    while not o.is_finished():
        o.step(1)
        steps_o += 1
        frames_o += int(o.frame_finished())
    assert (steps_g, frames_g) == (steps_o, frames_o) and frames_g == 3
    assert g.frame == o.get("frame") == 3
    assert g.time == pytest.approx(3.0 / 60.0, rel=1e-12) and o.get("time") == pytest.approx(3.0 / 60.0, rel=1e-12)
    pg = g.getParticles(fields=("x", "latent"))
    po = o.particles_f64()
    assert np.abs(pg.x - po["x"]).max() <= 1e-5
    assert np.abs(pg.latent - po["latent"]).max() <= 1e-5


def test_setup_scene_blobs_builds_the_blob_recipe():
    """pm_setup_scene_blobs (setupScene's signature: fps, colour ratios, latents, animation) builds
    the same particles as the Python restatement of the blob recipe (scenes.blob_scene, which
    centres the scene at (0.5, 0, 0.5) instead of the origin), then applies setupScene's
    settings; the scene then steps with the reference knife."""
    from pigment_mixing_b200 import scenes
    ratios = [0.25, 0.5, 0.75]
    lat = np.asarray([scenes.MIXBOX_LATENTS[scenes.RGB_SEEDS[i]] for i in range(3)], np.float32)
    g = _sim()
    g.setupSceneBlobs(60.0, ratios, lat, PIG_CFG, SIM_CFG, ANIM)
    ref = scenes.blob_scene(ratios, lat, knife=False)
    p = g.getParticles(fields=("x", "latent"))
    assert len(p.x) == len(ref["x"])
    assert np.abs(p.x + np.float32([0.5, 0.0, 0.5]) - ref["x"]).max() <= 1e-6
    assert np.array_equal(p.latent, ref["latent"])
    assert g.param("dx") == pytest.approx(ref["params"]["dx"], rel=1e-12)
    cfg = json.load(open(SIM_CFG))
    assert g.param("particle_mass") == pytest.approx(cfg.get("rho", 1000.0) * g.param("dx") ** 3 / 27.0, rel=1e-12)
    # touching blobs, centred on the origin in x and z, resting on y = 0
    assert abs(0.5 * (p.x[:, 0].min() + p.x[:, 0].max())) < 0.02 and p.x[:, 1].min() >= 0.0
    g.prepareSimulation()
    g.advance(5)
    q = g.getParticles(fields=("x", "active"))
    assert np.isfinite(q.x).all() and q.active.all() and g.errorFlags() == 0
    g.close()


def test_simulate_stops_at_max_steps_and_trim_memory_keeps_working():
    """pm_simulate with a step bound below the run's length reports PM_ERR_STATE after exactly that
    many steps; pm_trim_memory hands the pool's cached memory back, and simulations created
    afterwards allocate and step as before."""
    import ctypes as C
    from pigment_mixing_b200 import Simulation, scenes
    from pigment_mixing_b200._lib import PMError, call
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=8, steps=5)
    sc["params"]["end_frame"] = 5
    g = Simulation(0)
    scenes.apply(sc, g)
    with pytest.raises(PMError):
        g.simulate(max_steps=7)
    assert g.steps_done == 7 and g.frame < 5
    g.close()
    call("pm_trim_memory", 0, C.c_uint64(0))
    g = Simulation(0)
    scenes.apply(sc, g)
    steps = g.simulate()
    assert g.frame == 5 and steps > 7 and g.errorFlags() == 0
    g.close()
    call("pm_trim_memory", 0, C.c_uint64(1 << 30))
