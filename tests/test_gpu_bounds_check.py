"""The bounds-checked build (lib/libifc_bc.so, compiled with IFC_BOUNDS_CHECK):
every field-array index of the handle's kernels is checked on the device, and
an index out of range would come back as IFC_BAD_ARGUMENT instead of touching
memory.  The step-by-step parity tests on odd grid sizes (every boundary type,
2D and 3D, and the cooperative sweeps without norms), the multi-tile
single-launch tests and the slab decomposition tests run against it in a
child process and must pass: no kernel indexes outside its arrays on those
grids."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_BC = os.path.join(ROOT, "incompflow-cuda_b200", "lib", "libifc_bc.so")


def test_parity_tests_pass_under_the_bounds_checked_build(gpu_ok):
    assert os.path.exists(LIB_BC), "build it with make -C incompflow-cuda_b200 lib_bc"
    env = dict(os.environ, IFC_LIB=LIB_BC)
    probe = subprocess.run([sys.executable, "-c", "import ifc; print(ifc.load().ifc_build_flags())"], env=env,
                           cwd=os.path.join(ROOT, "incompflow-cuda_b200", "python"), capture_output=True, text=True)
    assert probe.returncode == 0 and probe.stdout.strip() == "1", probe.stdout + probe.stderr
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
                        "tests/test_gpu_parity_steps.py", "tests/test_gpu_persist_mt.py", "tests/test_gpu_slabs.py"],
                       env=env, cwd=ROOT, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
