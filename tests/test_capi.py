"""CPU checks of the C-ABI library: it loads, exports every entry point the
headers in include/ declare, and validates parameters on the host. No kernel
is launched here."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from mm_propagation_b200 import capi, workloads as W
import mm_propagation_b200 as mmp


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms |= set(re.findall(r"\b(mmp_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_library_loads_and_exports_every_declared_symbol():
    lib = capi.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) <= set(capi.SIGNATURES), "capi.SIGNATURES lags the header"


def test_version_and_strerror():
    lib = capi.load()
    assert b"sm_100a" in lib.mmp_version()
    for code in range(-8, 1):
        assert lib.mmp_strerror(code)


def _rc(prob):
    return mmp.validate(prob)


def test_validate_accepts_workloads():
    for prob in (W.grin2(nt=256, n_steps=10), W.small_case(), W.grin6(nt=256, n_steps=10)):
        rc, msg = _rc(prob)
        assert rc == 0, msg


@pytest.mark.parametrize("mutate,code", [
    (lambda p: p.replace(n_modes=0), capi.MMP_EINVAL),
    (lambda p: p.replace(dispersion=p.dispersion[:, :2]), capi.MMP_EINVAL),
    (lambda p: p.replace(dispersion=p.dispersion * np.array([1, 1, 0, 1])), capi.MMP_EINVAL),
    (lambda p: p.replace(pulse_width=0.0), capi.MMP_EINVAL),
    (lambda p: p.replace(time_window=-1.0), capi.MMP_EINVAL),
    (lambda p: p.replace(n_steps=0), capi.MMP_EINVAL),
    (lambda p: p.replace(nt=100, initial_fields=p.initial_fields[:, :100],
                         raman_response=p.raman_response[:100]), capi.MMP_ENOTSUP),
    (lambda p: p.replace(raman_response=None), capi.MMP_EINVAL),
    # the reference's conversion factor sqrt(|gamma| LD max|Q|) is then 0 and its result 0/0
    (lambda p: p.replace(nonlinearity_const=0.0), capi.MMP_EINVAL),
])
def test_validate_rejects(mutate, code):
    base = W.grin2(nt=256, n_steps=10)
    rc, msg = _rc(mutate(base))
    assert rc == code, (rc, msg)
    assert msg


def test_validate_rejects_bad_coupling():
    p = W.grin2(nt=256, n_steps=10)
    bad = p.coupling.copy()
    bad["l"][0] = 7
    assert _rc(p.replace(coupling=bad))[0] == capi.MMP_EINVAL
    zero = p.coupling.copy()
    zero["value"] = 0.0
    assert _rc(p.replace(coupling=zero))[0] == capi.MMP_EINVAL
    nan = p.initial_fields.copy()
    nan[0, 3] = np.nan
    assert _rc(p.replace(initial_fields=nan))[0] == capi.MMP_EINVAL


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly():
    with pytest.raises(mmp.MMPError):
        mmp.Solver(W.small_case())
    with pytest.raises(mmp.MMPError):
        mmp.Server()


def test_server_structs_match_header():
    # field order and sizes of the two serving structs as include/mmp.h lays them out
    assert C.sizeof(capi.mmp_server_config) == 24
    assert C.sizeof(capi.mmp_request_info) == 48
    assert [f for f, _ in capi.mmp_request_info._fields_][:4] == ["status", "n_modes", "nt", "steps"]
