"""The C-ABI library loads and exports every entry point that include/*.h declares (no GPU calls)."""
import ctypes as C
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        with open(h) as f:
            txt = f.read()
        names |= set(re.findall(r"^PM_API\s+[\w\s\*]+?\b(pm_\w+)\s*\(", txt, flags=re.M))
    return names


def test_header_declares_entry_points():
    names = _declared()
    for required in ("pm_create", "pm_destroy", "pm_prepare", "pm_step", "pm_advance", "pm_set_particles",
                     "pm_get_particles", "pm_add_plate", "pm_add_spatula", "pm_add_box_knife", "pm_setup_scene",
                     "pm_frame_finished", "pm_is_finished", "pm_get_grid_boundaries", "pm_get_knife",
                     "pm_load_sim_config", "pm_load_pigment_config", "pm_set_return_map"):
        assert required in names, required


def test_library_exports_every_declared_symbol():
    from pigment_mixing_b200 import build
    path = build.build()
    lib = C.CDLL(path)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_signatures_cover_header():
    from pigment_mixing_b200._lib import SIGNATURES
    names = _declared() - {"pm_last_error_message", "pm_kernel_name", "pm_batch_kernel_name",
                           "pm_batch_kernels_per_round"}
    assert names <= set(SIGNATURES), sorted(names - set(SIGNATURES))


def test_create_without_gpu_fails_cleanly():
    """Without a usable GPU pm_create returns an error status (never a CPU fallback)."""
    from conftest import gpu_available
    if gpu_available():
        import pytest
        pytest.skip("GPU present")
    from pigment_mixing_b200 import Simulation
    from pigment_mixing_b200._lib import PMError
    import pytest
    with pytest.raises(PMError):
        Simulation(0)
