"""Output files and checkpoints: the PLY files of save_data.cpp (property set, binary layout,
values against the particle state and the FP64 oracle), info.txt, and checkpoint save -> load ->
continue matching an uninterrupted run."""
import os

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401


def _write_reference_style_ply(path, names, rows):
    """A PLY exactly as the reference writes it (tinyply binary little-endian, float32)."""
    with open(path, "wb") as f:
        f.write(b"ply\nformat binary_little_endian 1.0\n")
        f.write(f"element vertex {len(rows)}\n".encode())
        for n in names:
            f.write(f"property float {n}\n".encode())
        f.write(b"end_header\n")
        f.write(np.ascontiguousarray(rows, "<f4").tobytes())


def test_ply_reader_round_trip(tmp_path):
    from pigment_mixing_b200.ply import read_ply
    names = ["x", "y", "z", "vx", "vy", "vz", "p", "q", "Je"]
    rows = np.random.default_rng(0).normal(size=(17, len(names))).astype(np.float32)
    path = os.path.join(tmp_path, "a.ply")
    _write_reference_style_ply(path, names, rows)
    d = read_ply(path)
    assert list(d) == names
    for k, n in enumerate(names):
        assert np.array_equal(d[n], rows[:, k])


def _scene():
    from pigment_mixing_b200 import scenes
    return scenes.two_block_scene(1.0 / 32, (8, 8, 4), seed=4, steps=20)


@pytest.mark.gpu
def test_particle_and_grid_ply_match_state_and_oracle(tmp_path):
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import Simulation, scenes
    from pigment_mixing_b200.ply import read_ply
    sc = _scene()
    g = Simulation(0)
    g.initializeBasic("plyrun")
    scenes.apply(sc, g)
    g.prepareSimulation()
    g.advance(12)
    os.makedirs(os.path.join(tmp_path, "plyrun"))
    d = str(tmp_path) + "/"
    g.saveParticleData(d)
    g.saveGridData(d, "x")
    g.saveInfo(d)
    frame = int(g.frame)
    names = ["x", "y", "z", "vx", "vy", "vz", "p", "q", "Je", "eps_pl_vol", "eps_pl_dev", "delta_gamma"]
    pl = read_ply(os.path.join(d, "plyrun", f"particles_f{frame}.ply"))
    assert list(pl) == names
    assert open(os.path.join(d, "plyrun", "last_written.txt")).read().strip() == str(frame)
    st = g.getParticles(fields=("x", "v", "F", "plastic"))
    assert np.array_equal(np.stack([pl["x"], pl["y"], pl["z"]], 1), st.x)
    assert np.array_equal(np.stack([pl["vx"], pl["vy"], pl["vz"]], 1), st.v)
    assert np.allclose(pl["Je"], np.linalg.det(st.F.astype(np.float64)), rtol=1e-5, atol=1e-6)
    assert np.array_equal(pl["eps_pl_vol"], st.plastic[:, 1])
    assert np.array_equal(pl["eps_pl_dev"], st.plastic[:, 0])
    assert np.array_equal(pl["delta_gamma"], st.plastic[:, 3])
    # p and q from the FP64 oracle's F through the reference's Hencky stress (save_data.cpp:15-31)
    o = OracleSim(64)
    scenes.apply(sc, o)
    o.prepare()
    o.advance(12)
    F = o.particles()["F"].astype(np.float64)
    U, s, Vt = np.linalg.svd(F)
    prm = sc["params"]
    mu = prm["E"] / (2 * (1 + prm["nu"]))
    lam = prm["nu"] * prm["E"] / ((1 + prm["nu"]) * (1 - 2 * prm["nu"]))
    h = np.log(s)
    dvals = 2 * mu * h + lam * h.sum(1, keepdims=True)
    tau = np.einsum("nij,nj,nkj->nik", U, dvals, U)
    p_ref = -np.trace(tau, axis1=1, axis2=2) / 3
    dev = tau + p_ref[:, None, None] * np.eye(3)
    q_ref = prm["q_prefac"] * np.sqrt((dev * dev).sum((1, 2)))
    scale = np.abs(p_ref).max() + np.abs(q_ref).max()
    assert np.abs(pl["p"] - p_ref).max() <= 1e-4 * scale
    assert np.abs(pl["q"] - q_ref).max() <= 1e-4 * scale
    gr = read_ply(os.path.join(d, "plyrun", f"grid_fx{frame}.ply"))
    assert list(gr) == ["x", "y", "z", "vx", "vy", "vz", "mass"]
    gg = g.grid()
    assert np.array_equal(gr["mass"], gg["mass"])
    assert np.allclose(gr["x"].reshape(gg["dims"])[:, 0, 0], gg["origin"][0] + np.arange(gg["dims"][0]) * prm["dx"],
                       atol=1e-6)
    info = open(os.path.join(d, "plyrun", "info.txt")).read().split()
    assert int(info[3]) == len(sc["x"]) and float(info[2]) == pytest.approx(prm["dx"])


@pytest.mark.gpu
def test_checkpoint_resume_continues_the_run(tmp_path):
    from pigment_mixing_b200 import Simulation, scenes
    sc = _scene()

    def make():
        g = Simulation(0)
        scenes.apply(sc, g)
        g.prepareSimulation()
        return g

    a = make()
    a.advance(10)
    path = os.path.join(tmp_path, "run.ckpt")
    a.saveCheckpoint(path)
    t10, f10 = float(a.time), int(a.frame)
    a.advance(10)
    b = make()
    b.loadCheckpoint(path)
    assert b.steps_done == 10 and float(b.time) == t10 and int(b.frame) == f10
    b.advance(10)
    assert b.steps_done == a.steps_done == 20
    assert b.time == pytest.approx(a.time, rel=1e-6)
    pa = a.getParticles(fields=("x", "v", "latent", "F"))
    pb = b.getParticles(fields=("x", "v", "latent", "F"))
    assert np.abs(pa.x - pb.x).max() <= 1e-5
    assert np.abs(pa.latent - pb.latent).max() <= 1e-5
    assert np.abs(pa.F - pb.F).max() <= 1e-4
    c = Simulation(0)
    other = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=1, steps=5)
    scenes.apply(other, c)
    c.prepareSimulation()
    from pigment_mixing_b200._lib import PMError
    with pytest.raises(PMError):
        c.loadCheckpoint(path)  # particle count differs
