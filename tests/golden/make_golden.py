"""Regenerate the golden fixtures in this folder from the reference tree.

Run in a container where the reference is mounted (it reads it, the tests never do):

    make -C oracle ref REF=<reference tree>     # compiles the reference's mixbox.cpp in place
    python tests/golden/make_golden.py <reference tree>

Writes
  mixbox_latents.json    Mixbox float RGB -> 7-float latent for the scene colours, produced by
                         the reference's own raytracing/src/mixbox/mixbox.cpp
                         (mixbox_float_rgb_to_latent, mixbox.cpp:120-170), plus latent -> RGB of
                         a few 50/50 latent mixes (mixbox_latent_to_float_rgb, mixbox.cpp:172-179).
  spatula_frames_head.npy  the first 481 keyframes (8 s at 60 fps) of the reference's knife
                         animation matter/animations/spatula_motion.bin (7 float32 per frame:
                         position xyz, quaternion xyzw; object_spatula.hpp:7-10).
  spatula_motion.bin     that animation whole (3,601 frames), byte for byte, for the tests of
                         pm_add_spatula_file and pm_setup_scene.
  sim_config.json,       the reference's own configuration files (matter/sim_config.json,
  pigment_config.json    matter/pigment_config.json), byte for byte, for the tests of the JSON
                         readers (simulation_units.cpp:31-80).
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import mixbox_ref_lib  # noqa: E402

# Scene colours: the two paint colours of the single-scene workloads and four more seeds used by
# the four-pigment and batched workloads.
RGB_SEEDS = [
    (0.99, 0.86, 0.08),
    (0.10, 0.20, 0.60),
    (0.80, 0.10, 0.12),
    (0.05, 0.45, 0.25),
    (0.95, 0.95, 0.93),
    (0.45, 0.25, 0.05),
]


def main(ref_root: str) -> None:
    lib = mixbox_ref_lib()
    if lib is None:
        raise SystemExit("oracle/_ref/libmixbox_ref.so missing: run `make -C oracle ref` first")
    lat = {}
    for rgb in RGB_SEEDS:
        out = (C.c_float * 7)()
        lib.mixbox_float_rgb_to_latent(C.c_float(rgb[0]), C.c_float(rgb[1]), C.c_float(rgb[2]), out)
        lat[repr(rgb)] = [float(v) for v in out]
    mixes = []
    keys = list(lat)
    for i in range(len(keys)):
        for j in range(i + 1, len(keys)):
            z = (np.asarray(lat[keys[i]], np.float32) + np.asarray(lat[keys[j]], np.float32)) * np.float32(0.5)
            zc = (C.c_float * 7)(*[float(v) for v in z])
            r, g, b = C.c_float(), C.c_float(), C.c_float()
            lib.mixbox_latent_to_float_rgb(zc, C.byref(r), C.byref(g), C.byref(b))
            mixes.append(dict(a=keys[i], b=keys[j], latent=[float(v) for v in z], rgb=[r.value, g.value, b.value]))
    with open(os.path.join(HERE, "mixbox_latents.json"), "w") as f:
        json.dump(dict(source="raytracing/src/mixbox/mixbox.cpp (reference, compiled in place)",
                       rgb_to_latent=lat, latent_mix_to_rgb=mixes), f, indent=1)

    anim = os.path.join(ref_root, "matter", "animations", "spatula_motion.bin")
    frames = np.fromfile(anim, dtype=np.float32).reshape(-1, 7)
    np.save(os.path.join(HERE, "spatula_frames_head.npy"), frames[:481].copy())
    for src, dst in ((anim, "spatula_motion.bin"), (os.path.join(ref_root, "matter", "sim_config.json"), "sim_config.json"),
                     (os.path.join(ref_root, "matter", "pigment_config.json"), "pigment_config.json")):
        with open(src, "rb") as f, open(os.path.join(HERE, dst), "wb") as g:
            g.write(f.read())
    print("wrote mixbox_latents.json, spatula_frames_head.npy, spatula_motion.bin (%d frames), sim_config.json, "
          "pigment_config.json" % len(frames))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden.py <reference tree>")
    main(sys.argv[1])
