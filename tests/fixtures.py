"""Load tests/golden/*.npz into workload Problems (see tests/golden/make_golden.py)."""
import glob
import os

import numpy as np

from mm_propagation_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """Solver fixtures (the drop-in driver's output fixture is used by test_dropin.py)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("dropin_"))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    coup = np.zeros(len(z["coup_p"]), dtype=W.NZ_DTYPE)
    for f in ("p", "k", "l", "m"):
        coup[f] = z["coup_" + f]
    coup["value"] = z["coup_value"]
    raman = bool(int(z["raman"]))
    prob = W.Problem(
        n_modes=int(z["n_modes"]), nt=int(z["nt"]), dispersion=z["dispersion"], coupling=coup,
        initial_fields=z["initial_fields"], time_window=float(z["time_window"]),
        pulse_width=float(z["pulse_width"]), fiber_length=float(z["fiber_length"]),
        n_steps=int(z["n_steps"]), method_order=int(z["method_order"]),
        nonlinearity_const=float(z["nonlinearity_const"]),
        raman_proportion=float(z["raman_proportion"]),
        raman_response=z["raman_response"] if raman else None, raman=raman, name=name)
    chunks = [None if c < 0 else int(c) for c in z["chunks"]]
    return prob, chunks, z["result"]
