"""The drop-in reference program: the reference's own host sources (main, planner, factory,
FDKReconstructor, reader, writer -- unmodified) linked with listctrecons_b200/dropin/Stages.cpp
and liblct.so in place of its CUDA files (built by listctrecons_b200/dropin/Makefile where the
reference tree is present).  CPU part: it loads and behaves like the reference's main."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
DROPIN = ROOT / "listctrecons_b200" / "dropin" / "_build" / "LISTCTRecons"


@pytest.mark.skipif(not DROPIN.exists(), reason="drop-in not built (needs the reference tree)")
def test_dropin_binary_loads_and_prints_usage():
    r = subprocess.run([str(DROPIN)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1  # Src/main.cpp:17-21
    assert "Usage LISTCTRecons <PRM filename>" in r.stdout
    r = subprocess.run([str(DROPIN), "/nonexistent.prm"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Parameter file not found" in r.stdout  # Src/FileParams.cpp:31-35
