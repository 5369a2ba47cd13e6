"""The Fortran drop-in module (pmlib3d_b200/fortran/pmlib_gpu_mod.f90) compiled
against stand-ins of the pmlib3d modules it USEs, for the double and the
single-precision build.  Needs a Fortran compiler; skipped where there is none."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FC = shutil.which("gfortran")


@pytest.mark.skipif(FC is None, reason="no gfortran on this machine")
@pytest.mark.parametrize("single", [False, True])
def test_drop_in_module_compiles(tmp_path, single):
    stubs = os.path.join(ROOT, "tests", "fortran", "pmlib_stub_modules.f90")
    mod = os.path.join(ROOT, "pmlib3d_b200", "fortran", "pmlib_gpu_mod.f90")
    cmd = [FC, "-cpp", "-fsyntax-only", "-std=f2008", "-Wall", "-J", str(tmp_path)]
    if single:
        cmd.append("-D__single")
    r = subprocess.run(cmd + [stubs, mod], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
