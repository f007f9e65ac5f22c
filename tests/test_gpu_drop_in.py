"""Drop-in check: the reference's own GPU test programs
(tests/test_gpu_pdhg.cpp, tests/test_pdhg_kernel.cpp and
tests/test_precision_ladder.cpp with the reference's own controller
src/gpu/precision_ladder.cpp), compiled unmodified from its sources and linked
against libpramaan_b200 through the C++ facade
(pramaan_b200/csrc/facade/pdhg_solver.cpp), must pass.  The same programs
linked against the reference's own GPU library are run beside them.

The binaries are built by oracle/build.py into oracle/_ref/ (needs the
reference tree at build time; they travel with the working tree)."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


def run(exe: str):
    path = REF / exe
    if not path.exists():
        pytest.skip(f"{path} not built (oracle/build.py needs the reference tree)")
    r = subprocess.run([str(path)], cwd=REF / "run", capture_output=True, text=True, timeout=600)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("prog", ["test_gpu_pdhg", "test_pdhg_kernel", "test_precision_ladder"])
def test_reference_program_passes_on_pramaan_b200(prog):
    rc, out = run(f"{prog}__pramaan_b200")
    assert rc == 0 and "TEST SUITE PASSED" in out, out[-4000:]


@pytest.mark.parametrize("prog", ["test_gpu_pdhg", "test_pdhg_kernel", "test_precision_ladder"])
def test_reference_program_on_reference_library(prog):
    rc, out = run(f"{prog}__reference")
    print(out[-3000:])
    assert "checks run" in out


def test_cuda_backend_matches_the_cpu_backend():
    """pramaan::gpu::make_cuda_backend() (the facade's Backend,
    include/pramaan/gpu/backend.hpp:36-57) against the reference's CPU backend
    on the same models (tests/cpp/check_cuda_backend.cpp)."""
    rc, out = run("check_cuda_backend")
    assert rc == 0 and "CUDA BACKEND CHECK PASSED" in out, out[-3000:]
