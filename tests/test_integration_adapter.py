"""The C++ adapter that INTEGRATION.md gives the reference's caller (MPMIntegrationSim.cpp) compiles
against include/pigment_mpm.h and links against the library with every symbol it calls resolved."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _adapter_source() -> str:
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    sec = text[text.index("## C++"):]
    m = re.search(r"```cpp\n(.*?)```", sec, re.S)
    assert m, "no C++ block in the C++ section of INTEGRATION.md"
    return m.group(1)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_integration_adapter_compiles_and_links(tmp_path):
    src = tmp_path / "adapter.cpp"
    src.write_text(_adapter_source() + "\n// instantiate every member\ntemplate struct std::vector<float>;\n"
                   "void use_adapter() { PmSimAdapter a; a.setupScene(60.f, {0.5f}, {{}}, \"anim.bin\"); a.simStep();\n"
                   "  a.isTimeToRender(); a.isFinished(); a.recountParticles(); a.getGridBoundaries();\n"
                   "  std::array<double, 16> m; std::array<double, 3> h; a.getSpatulaInvTransform(m, h); }\n")
    inc = os.path.join(ROOT, "include")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-c", str(src), "-I", inc, "-o", str(tmp_path / "a.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lib_dir = os.path.join(ROOT, "pigment_mixing_b200")
    if not os.path.exists(os.path.join(lib_dir, "libpigment_mpm.so")):
        pytest.skip("library not built")
    r = subprocess.run(["g++", "-shared", "-fPIC", "-Wl,--no-undefined", "-o", str(tmp_path / "a.so"), str(src), "-I", inc,
                        "-L", lib_dir, "-lpigment_mpm", "-Wl,--allow-shlib-undefined"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
