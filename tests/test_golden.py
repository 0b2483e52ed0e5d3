"""Golden fixtures produced by the reference's own code (tests/golden/make_golden.py)."""
import ctypes as C
import json
import os

import numpy as np

from conftest import GOLDEN


def _golden():
    with open(os.path.join(GOLDEN, "mixbox_latents.json")) as f:
        return json.load(f)


def test_scene_latents_match_reference_mixbox():
    """The scene builders' latents are the reference Mixbox rgb->latent outputs (mixbox.cpp:120-170)."""
    from pigment_mixing_b200 import scenes
    g = _golden()["rgb_to_latent"]
    for rgb, lat in scenes.MIXBOX_LATENTS.items():
        key = repr(tuple(float(c) for c in rgb)).replace("0.1,", "0.1,")
        ref = g[repr(tuple(rgb))]
        assert np.allclose(np.asarray(lat, np.float32), np.asarray(ref, np.float32), atol=0, rtol=0), rgb


def test_latent_concentrations_sum_to_one():
    """Mixbox latents hold 4 concentrations that sum to 1 (mixbox.cpp:165: c3 = 1 - (c0+c1+c2))."""
    for lat in _golden()["rgb_to_latent"].values():
        assert abs(sum(lat[:4]) - 1.0) < 1e-6


def test_reference_mixbox_reproduces_golden_when_built():
    """When oracle/_ref (the reference mixbox compiled in place) exists, it reproduces the fixture."""
    from oracle.oracle import mixbox_ref_lib
    lib = mixbox_ref_lib()
    if lib is None:
        import pytest
        pytest.skip("oracle/_ref not built (reference tree absent)")
    g = _golden()
    for rgb_s, lat in g["rgb_to_latent"].items():
        rgb = eval(rgb_s)
        out = (C.c_float * 7)()
        lib.mixbox_float_rgb_to_latent(C.c_float(rgb[0]), C.c_float(rgb[1]), C.c_float(rgb[2]), out)
        assert np.array_equal(np.asarray(list(out), np.float32), np.asarray(lat, np.float32))
    for m in g["latent_mix_to_rgb"]:
        z = (C.c_float * 7)(*m["latent"])
        r, gg, b = C.c_float(), C.c_float(), C.c_float()
        lib.mixbox_latent_to_float_rgb(z, C.byref(r), C.byref(gg), C.byref(b))
        assert np.allclose([r.value, gg.value, b.value], m["rgb"], rtol=0, atol=0)


def test_spatula_frames_fixture():
    """Keyframes of the reference knife animation: 7 float32 per frame, unit quaternions."""
    fr = np.load(os.path.join(GOLDEN, "spatula_frames_head.npy"))
    assert fr.shape == (481, 7) and fr.dtype == np.float32
    qn = np.linalg.norm(fr[:, 3:7].astype(np.float64), axis=1)
    assert np.all(np.abs(qn - 1.0) < 1e-5)
