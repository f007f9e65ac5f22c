"""Build recipe for the oracle (test infrastructure only).

* ``oracle/_build/liborc.so`` — the C restatement in ``pdhg_oracle.c``.
* ``oracle/_ref/`` — the reference's own code, compiled from its sources where
  they lie (``/root/reference``) when that tree is present: its CPU core
  (simplex, dual simplex, IPM, MPS parser, certificate), its GPU PDHG
  (``src/gpu/pdhg_solver.cu``, ``src/gpu/pdhg.cu``) built for sm_100a, C shims
  over both (``ref_shim.cpp``), and the reference's GPU test programs linked
  once against its own GPU library and once against libpramaan_b200 through
  the C++ facade.  Nothing is copied into the repository; outputs stay in
  ``oracle/_ref/`` (git-ignored, shipped with the working tree).

Usage: ``python -m oracle.build [--ref] [--force]``
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
REF_SRC = Path(os.environ.get("PRAMAAN_REFERENCE_ROOT", "/root/reference"))
ORC_LIB = BUILD / "liborc.so"

# The reference's CPU core (its CMakeLists.txt pramaan_core source list).
REF_CORE = [
    "src/io/mps_parser.cpp", "src/ir/model_ir.cpp", "src/linalg/sparse_matrix.cpp",
    "src/presolve/presolve.cpp", "src/presolve/scaling.cpp",
    "src/presolve/transformation_ledger.cpp", "src/simplex/revised_simplex.cpp",
    "src/simplex/dual_simplex.cpp", "src/certificate/certificate.cpp", "src/mip/node.cpp",
    "src/mip/branch_and_bound.cpp", "src/structure/fingerprint.cpp",
    "src/ipm/interior_point.cpp", "src/gpu/backend_cpu.cpp",
]
REF_GPU = ["src/gpu/pdhg_solver.cu", "src/gpu/pdhg.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _newer(out: Path, *deps: Path) -> bool:
    return out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps if d.exists())


def build_oracle(force: bool = False) -> Path:
    src = HERE / "pdhg_oracle.c"
    BUILD.mkdir(exist_ok=True)
    if force or not _newer(ORC_LIB, src):
        tmp = ORC_LIB.with_suffix(".tmp.so")
        _run(["gcc", "-O3", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              "-mfma", "-fvisibility=hidden", str(src), "-o", str(tmp), "-lm"])
        os.replace(tmp, ORC_LIB)
    return ORC_LIB


def reference_available() -> bool:
    return (REF_SRC / "src" / "gpu" / "pdhg_solver.cu").exists()


def build_reference(force: bool = False) -> dict[str, Path]:
    """Compiles the reference pieces into oracle/_ref (needs the reference tree)."""
    if not reference_available():
        raise RuntimeError(f"reference sources not found under {REF_SRC}")
    REF_OUT.mkdir(exist_ok=True)
    obj_dir = REF_OUT / "obj"
    obj_dir.mkdir(exist_ok=True)
    inc = ["-I", str(REF_SRC / "include")]
    cxx = ["g++", "-O2", "-std=c++17", "-fPIC", "-w"]
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

    def obj_for(rel: str) -> Path:
        return obj_dir / (rel.replace("/", "__") + ".o")

    jobs = []
    for rel in REF_CORE:
        src, obj = REF_SRC / rel, obj_for(rel)
        if force or not _newer(obj, src):
            jobs.append([*cxx, *inc, "-c", str(src), "-o", str(obj)])
    for rel in REF_GPU:
        src, obj = REF_SRC / rel, obj_for(rel)
        if force or not _newer(obj, src):
            jobs.append([nvcc, *ARCH, "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-w",
                         *inc, "-c", str(src), "-o", str(obj)])
    shim = HERE / "ref_shim.cpp"
    shim_cpu, shim_gpu = obj_dir / "ref_shim_cpu.o", obj_dir / "ref_shim_gpu.o"
    if force or not _newer(shim_cpu, shim):
        jobs.append([*cxx, *inc, "-c", str(shim), "-o", str(shim_cpu)])
    if force or not _newer(shim_gpu, shim):
        jobs.append([*cxx, *inc, "-DREF_WITH_GPU", "-I/usr/local/cuda/include", "-c", str(shim),
                     "-o", str(shim_gpu)])
    facade = REPO / "pramaan_b200" / "csrc" / "facade" / "pdhg_solver.cpp"
    facade_obj = obj_dir / "facade_pdhg_solver.o"
    if force or not _newer(facade_obj, facade):
        jobs.append([*cxx, *inc, "-I", str(REPO / "include"), "-c", str(facade), "-o",
                     str(facade_obj)])
    # the GPU Backend of the facade and its check program (ours, against the reference's headers)
    backend = REPO / "pramaan_b200" / "csrc" / "facade" / "cuda_backend.cpp"
    backend_obj = obj_dir / "facade_cuda_backend.o"
    if force or not _newer(backend_obj, backend, backend.with_suffix(".hpp")):
        jobs.append([*cxx, *inc, "-I", str(REPO / "include"), "-c", str(backend), "-o", str(backend_obj)])
    bcheck = REPO / "tests" / "cpp" / "check_cuda_backend.cpp"
    bcheck_obj = obj_dir / "check_cuda_backend.o"
    if force or not _newer(bcheck_obj, bcheck, backend.with_suffix(".hpp")):
        jobs.append([*cxx, *inc, "-I", str(backend.parent), "-c", str(bcheck), "-o", str(bcheck_obj)])
    # the reference's precision-ladder controller, compiled with its GPU rung enabled
    ladder_src = REF_SRC / "src" / "gpu" / "precision_ladder.cpp"
    ladder_obj = obj_dir / "precision_ladder_cuda.o"
    if force or not _newer(ladder_obj, ladder_src):
        jobs.append([*cxx, *inc, "-DPRAMAAN_ENABLE_CUDA", "-c", str(ladder_src), "-o", str(ladder_obj)])
    tests = {}
    for t in ("test_gpu_pdhg", "test_pdhg_kernel", "test_precision_ladder"):
        src = REF_SRC / "tests" / f"{t}.cpp"
        obj = obj_dir / f"{t}.o"
        tests[t] = obj
        extra = ["-DPRAMAAN_ENABLE_CUDA"] if t == "test_precision_ladder" else []
        if force or not _newer(obj, src):
            jobs.append([*cxx, *inc, *extra, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        list(ex.map(_run, jobs))

    core_objs = [str(obj_for(r)) for r in REF_CORE]
    gpu_objs = [str(obj_for(r)) for r in REF_GPU]
    cuda_lib = ["-L/usr/local/cuda/lib64", "-lcudart"]
    out = {}
    # CPU shim: the reference's simplex / dual simplex / IPM / MPS parser.
    out["cpu"] = REF_OUT / "libref_cpu.so"
    _run(["g++", "-shared", "-o", str(out["cpu"]), str(shim_cpu), *core_objs])
    # GPU shim: additionally the reference's PDHG solver and launchers (sm_100a).
    out["gpu"] = REF_OUT / "libref_gpu.so"
    _run([nvcc, *ARCH, "-shared", "-o", str(out["gpu"]), str(shim_gpu), *core_objs, *gpu_objs])
    # The reference's GPU test programs, against its own library ...
    for t, obj in tests.items():
        exe = REF_OUT / f"{t}__reference"
        extra = [str(ladder_obj)] if t == "test_precision_ladder" else []
        _run([nvcc, *ARCH, "-o", str(exe), str(obj), *extra, *core_objs, *gpu_objs])
        out[f"{t}__reference"] = exe
    # ... and against libpramaan_b200 through the C++ facade (drop-in check;
    # the precision ladder is the reference's own controller calling the
    # facade's PdhgSolver).
    lib_dir = REPO / "pramaan_b200"
    for t, obj in tests.items():
        exe = REF_OUT / f"{t}__pramaan_b200"
        extra = [str(ladder_obj)] if t == "test_precision_ladder" else []
        _run(["g++", "-o", str(exe), str(obj), *extra, str(facade_obj), *core_objs,
              f"-L{lib_dir}", "-lpramaan_b200", f"-Wl,-rpath,$ORIGIN/../../pramaan_b200"])
        out[f"{t}__pramaan_b200"] = exe
    exe = REF_OUT / "check_cuda_backend"
    _run(["g++", "-o", str(exe), str(bcheck_obj), str(backend_obj), *core_objs,
          f"-L{lib_dir}", "-lpramaan_b200", f"-Wl,-rpath,$ORIGIN/../../pramaan_b200"])
    out["check_cuda_backend"] = exe
    # The reference's MPS fixtures, for the programs above (they open
    # tests/data/*.mps relative to their working directory).
    data = REF_OUT / "run" / "tests" / "data"
    data.mkdir(parents=True, exist_ok=True)
    for mps in ("afiro.mps", "adlittle.mps"):
        shutil.copy2(REF_SRC / "tests" / "data" / mps, data / mps)
    return out


def build(force: bool = False, ref: bool = True) -> None:
    build_oracle(force)
    if ref and reference_available():
        build_reference(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, ref="--no-ref" not in sys.argv)
