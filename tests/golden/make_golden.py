"""Generate the golden fixtures in tests/golden/*.npz from the reference's own CPU
solver (oracle/_ref/libmmref.so, built from the unmodified reference sources by
oracle/Makefile). Run here, where the reference is present:

    make -C oracle && python tests/golden/make_golden.py

Each fixture stores the complete inputs (so it does not depend on the workload
generators staying unchanged), the chunk sequence passed to computeLawsonRK,
and getResult()'s output. The reference publishes no tests or golden vectors of
its own, so these are the pins for the oracle restatement and the GPU path.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref_lib  # noqa: E402
from mm_propagation_b200 import workloads as W  # noqa: E402


def cases():
    """name -> (problem, chunks). chunks None entries = computeLawsonRK()."""
    out = {}
    # the pair-slot case: lexicographic insertion makes unique_pairs [0,2,1,3]
    out["grin2_quirk_raman"] = (W.grin2(seed=11, nt=512, n_steps=1000, fiber_length=0.1,
                                        peak_scale=0.01), [24])
    out["grin2_quirk_noraman"] = (W.grin2(seed=12, nt=256, n_steps=1000, fiber_length=0.1,
                                          peak_scale=0.01, raman=False), [24])
    out["grin2_literal"] = (W.grin2(seed=13, nt=256, n_steps=1000, fiber_length=0.1,
                                    peak_scale=0.003, literal=True), [12])
    out["m3_order6_raman"] = (W.small_case(seed=21, M=3, nt=256, n_steps=16, order=6), [16])
    out["m4_order8_raman"] = (W.small_case(seed=22, M=4, nt=128, n_steps=8, order=8), [8])
    out["m2_order4_noraman_beta5"] = (W.small_case(seed=23, M=2, nt=512, n_steps=20, raman=False,
                                                   n_beta=5), [20])
    out["m3_physical_order"] = (W.small_case(seed=24, M=3, nt=256, n_steps=16, physical_order=True), [16])
    out["m3_chunked_zreset"] = (W.small_case(seed=25, M=3, nt=256, n_steps=20), [5, 7, 8])
    out["m2_noarg"] = (W.small_case(seed=26, M=2, nt=256, n_steps=12), [None])
    out["m1_single_mode"] = (W.small_case(seed=27, M=1, nt=1024, n_steps=30, peak_w=400.0), [30])
    out["m5_order4_raman_nt2048"] = (W.small_case(seed=28, M=5, nt=2048, n_steps=10, nnz_target=40), [10])
    return out


def save(name, prob, chunks, phi, seconds):
    c = prob.coupling
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        n_modes=prob.n_modes, nt=prob.nt, dispersion=prob.dispersion,
        coup_p=c["p"], coup_k=c["k"], coup_l=c["l"], coup_m=c["m"], coup_value=c["value"],
        initial_fields=prob.initial_fields, time_window=prob.time_window,
        pulse_width=prob.pulse_width, fiber_length=prob.fiber_length, n_steps=prob.n_steps,
        method_order=prob.method_order, nonlinearity_const=prob.nonlinearity_const,
        raman_proportion=prob.raman_proportion,
        raman_response=(prob.raman_response if prob.raman_response is not None else np.zeros(0)),
        raman=int(prob.raman),
        chunks=np.array([-1 if x is None else x for x in chunks], dtype=np.int64),
        result=phi)
    return {"name": name, "seconds": seconds, "chunks": [x for x in chunks],
            "finite": bool(np.isfinite(phi).all()), **{k: v for k, v in prob.manifest().items()
                                                          if k in ("n_modes", "nt", "method_order",
                                                                   "raman", "n_nonzeros")}}


def dropin_golden():
    """Build tests/dropin/two_mode_driver.cpp against the reference's own headers and
    CPU objects (oracle/_ref, from `make -C oracle`), run it, store its output."""
    import subprocess
    import tempfile
    ref_dir = os.environ.get("REF_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
    objs = sorted(os.path.join(ROOT, "oracle", "_ref", f) for f in os.listdir(os.path.join(ROOT, "oracle", "_ref"))
                  if f.startswith("ref_") and f.endswith(".o") and f != "ref_driver.o")
    objs.append(os.path.join(ROOT, "oracle", "_ref", "fftw3_shim.o"))
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "drv_ref")
        subprocess.run(["/usr/bin/g++", "-O3", "-std=c++11", "-fopenmp", "-DMMP_REFERENCE_BUILD",
                        "-I" + os.path.join(ref_dir, "include"), "-I" + os.path.join(ROOT, "oracle", "fftw_shim"),
                        os.path.join(ROOT, "tests", "dropin", "two_mode_driver.cpp"), *objs, "-o", exe], check=True)
        out = os.path.join(td, "out.txt")
        subprocess.run([exe, out], check=True)
        a = np.loadtxt(out)
    phi = (a[:, 0] + 1j * a[:, 1]).reshape(2, -1)
    assert np.isfinite(phi).all()
    np.savez_compressed(os.path.join(HERE, "dropin_two_mode.npz"), result=phi)
    print(f"dropin_two_mode: |phi|max {np.abs(phi).max():.3e}")


def main():
    dropin_golden()
    manifest = []
    for name, (prob, chunks) in cases().items():
        phi, sec = ref_lib.run(prob, chunks)
        assert np.isfinite(phi).all(), f"{name}: reference output not finite"
        manifest.append(save(name, prob, chunks, phi, sec))
        print(f"{name}: |phi|max {np.abs(phi).max():.3e} ({sec:.3f}s)")
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "source": "oracle/_ref/libmmref.so "
                   "(reference CPU solver, unmodified sources, FFTW-API shim)", "cases": manifest}, f,
                  indent=1)


if __name__ == "__main__":
    main()
