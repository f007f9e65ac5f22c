"""Records golden vectors from the reference's own GPU PDHG.

Runs the reference's GPU solver and launchers — src/gpu/pdhg_solver.cu and
src/gpu/pdhg.cu compiled for sm_100a from the reference's sources by
oracle/build.py into oracle/_ref/libref_gpu.so — on small seeded inputs and
stores inputs and outputs in one compressed .npz:

* ``solve/<case>/…``: PdhgSolver::solve (src/gpu/pdhg_solver.cu:169-411) on
  the reference's known-answer LPs (tests/test_gpu_pdhg.cpp:263-404), on
  seeded random LPs and on afiro: status, iterations, residuals, objective,
  x and row activity, plus the LP itself and the options;
* ``spmv/<case>/…`` and ``spmv_t/<case>/…``: launch_spmv / launch_spmv_t
  (src/gpu/pdhg.cu:156-241) on seeded random CSR matrices;
* ``step/<case>/…``: launch_pdhg_iteration (src/gpu/pdhg.cu:77-150).

It needs a CUDA device and the reference build, so it runs on a GPU machine:
``python tests/golden/make_ref_golden.py <out.npz>``; the result is
committed as tests/golden/ref_gpu_golden.npz and read by
tests/test_golden_reference.py (no GPU, no reference needed to read it).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
from lp_cases import KNOWN, mps_model, random_csr  # noqa: E402
from pramaan_b200.generators import random_sparse_lp  # noqa: E402

SOLVE_OPTS = dict(tolerance=1e-4, max_iterations=50000, check_frequency=100)


def lp_arrays(model) -> dict:
    return dict(c=model.obj_coeffs, row_ptr=model.row_ptr, col_idx=model.col_idx, values=model.values,
                row_lower=model.row_lower, row_upper=model.row_upper, var_lower=model.var_lower,
                var_upper=model.var_upper, obj_sense=np.int32(int(model.obj_sense)),
                obj_offset=np.float64(model.obj_offset))


def solve_cases():
    cases = {name: KNOWN[name][0] for name in sorted(KNOWN)}
    for seed in (0, 1, 2):
        cases[f"random_{seed}"] = random_sparse_lp(30, 90, 4, seed=seed)
    afiro = mps_model("afiro")
    if afiro is not None:
        cases["afiro"] = afiro
    return cases


def main(out: str) -> None:
    h = oracle.ref_gpu()
    if h is None:
        raise SystemExit("oracle/_ref/libref_gpu.so is not built")
    rec: dict[str, np.ndarray] = {}
    for name, model in solve_cases().items():
        opts = dict(SOLVE_OPTS)
        if name == "afiro":
            opts.update(tolerance=1e-5, max_iterations=200000, check_frequency=500)
        r = oracle.ref_solve("pdhg", model, max_iterations=opts["max_iterations"], tolerance=opts["tolerance"],
                             check_frequency=opts["check_frequency"], lib=h)
        p = f"solve/{name}/"
        for k, v in lp_arrays(model).items():
            rec[p + "lp_" + k] = np.asarray(v)
        rec[p + "opts"] = np.array([opts["tolerance"], opts["max_iterations"], opts["check_frequency"]])
        for k in ("status", "iterations", "primal_residual", "dual_residual", "objective_value"):
            rec[p + k] = np.asarray(r[k])
        rec[p + "x"] = r["x"]
        rec[p + "row_activity"] = r["row_activity"]
        print(name, r["status"], r["iterations"], r["objective_value"], flush=True)

    rng = np.random.default_rng(20240611)
    import ctypes as C
    ptr = oracle.ptr
    for i, (m, n) in enumerate([(1, 1), (7, 5), (64, 33), (300, 200), (1000, 3000)]):
        rp, ci, v = random_csr(m, n, rng, empty_frac=0.1 if m > 10 else 0.0)
        x = rng.standard_normal(n).astype(np.float32)
        yv = rng.standard_normal(m).astype(np.float32)
        y = np.zeros(m, np.float32)
        assert h.ref_launch_spmv(ptr(rp), ptr(ci), ptr(v), len(v), ptr(x), ptr(y), m, n) == 0
        yt = np.zeros(n, np.float32)
        assert h.ref_launch_spmv_t(ptr(rp), ptr(ci), ptr(v), len(v), ptr(yv), ptr(yt), m, n) == 0
        p = f"spmv/case{i}/"
        rec.update({p + "row_ptr": rp, p + "col_idx": ci, p + "values": v, p + "x": x, p + "y": y,
                    p + "dims": np.array([m, n])})
        rec.update({f"spmv_t/case{i}/yin": yv, f"spmv_t/case{i}/out": yt})

    for i, (n, m) in enumerate([(1, 1), (37, 19), (1000, 700)]):
        x = rng.standard_normal(n).astype(np.float32)
        y = rng.standard_normal(m).astype(np.float32)
        g = rng.standard_normal(n).astype(np.float32)
        ax = rng.standard_normal(m).astype(np.float32)
        b = rng.standard_normal(m).astype(np.float32)
        tau, sigma = np.float32(0.37), np.float32(0.61)
        xo, yo = x.copy(), y.copy()
        assert h.ref_launch_pdhg_iteration(ptr(xo), ptr(yo), ptr(g), ptr(ax), ptr(b), n, m,
                                           C.c_float(tau), C.c_float(sigma)) == 0
        p = f"step/case{i}/"
        rec.update({p + "x": x, p + "y": y, p + "g": g, p + "ax": ax, p + "b": b,
                    p + "tau_sigma": np.array([tau, sigma], np.float32), p + "x_out": xo, p + "y_out": yo})

    Path(out).parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out, **rec)
    print("wrote", out, len(rec), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(HERE / "ref_gpu_golden.npz"))
