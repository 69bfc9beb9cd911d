"""The C-ABI library: loads without a GPU, exports every declared symbol, and
its structs have the layout the ctypes mirror assumes."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT
from openferric_b200 import _abi as A
from openferric_b200 import _lib

HEADER = os.path.join(ROOT, "include", "of_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(of_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_match_binding_list():
    assert declared_functions() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert L.of_abi_version() == 1
    assert L.of_status_str(A.OF_ERR_INVALID_INPUT).decode() == "invalid input"


STRUCTS = {
    "of_model": A.OfModel,
    "of_payoff": A.OfPayoff,
    "of_mc_config": A.OfMcConfig,
    "of_mc_result": A.OfMcResult,
    "of_book_entry": A.OfBookEntry,
    "of_book_config": A.OfBookConfig,
    "of_greeks_params": A.OfGreeksParams,
    "of_greeks_result": A.OfGreeksResult,
    "of_lsm_contract": A.OfLsmContract,
    "of_lsm_config": A.OfLsmConfig,
    "of_lsm_result": A.OfLsmResult,
    "of_heston_adjoint_params": A.OfHestonAdjointParams,
    "of_adjoint_result": A.OfAdjointResult,
    "of_device_peaks": A.OfDevicePeaks,
    "of_tune_candidate": A.OfTuneCandidate,
    "of_stderr_target": A.OfStderrTarget,
    "of_stderr_round": A.OfStderrRound,
    "of_bermudan_contract": A.OfBermudanContract,
    "of_boundary_point": A.OfBoundaryPoint,
    "of_qmc_params": A.OfQmcParams,
    "of_dividend_event": A.OfDividendEvent,
    "of_book_greeks": A.OfBookGreeks,
    "of_lsm_barrier_contract": A.OfLsmBarrierContract,
}


def test_struct_layout_matches_ctypes():
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["/usr/bin/gcc", "-std=c11", "-o", exe, src], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for cname, py in STRUCTS.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly_without_cpu_fallback():
    from openferric_b200 import MonteCarloPricingEngine, Market, VanillaOption
    market = Market.builder().spot(100).rate(0.05).flat_vol(0.2).build()
    with pytest.raises(_lib.GpuUnavailable):
        MonteCarloPricingEngine(1000, 10, 1).price(VanillaOption.european_call(100, 1.0), market)


def _noalloc(model, strikes, **cfg_fields):
    """of_mc_strip_noalloc on host arguments only; the requests below fail in
    its validation, before any CUDA call, so this runs without a GPU."""
    L = _lib.load()
    ks = (C.c_double * len(strikes))(*strikes)
    cfg = A.OfMcConfig(num_paths=1024, seed=1, precision=A.OF_PREC_FP32_PHILOX, discount_factor=1.0, **cfg_fields)
    out = (A.OfMcResult * len(strikes))()
    err = C.create_string_buffer(256)
    st = L.of_mc_strip_noalloc(None, C.byref(model), A.OF_CALL, ks, len(strikes), C.byref(cfg), out, err, len(err))
    return st, err.value.decode()


def test_noalloc_strip_validates_like_of_mc_strip():
    """The no-allocation strip runs of_mc_strip's own validation: the same
    status for the same request, then its static-scratch strike limit."""
    from openferric_b200 import Heston, HestonPathGenerator
    gen = HestonPathGenerator(Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04), 100.0, 1.0, 8)
    model = gen.to_abi()
    st, msg = _noalloc(model, [100.0], tile_ilp=4)
    assert st == A.OF_ERR_INVALID_INPUT and "tile_ilp" in msg
    st, msg = _noalloc(model, [100.0], control_variate=A.OF_CV_TERMINAL_SPOT)
    assert st == A.OF_ERR_UNSUPPORTED and "control variate" in msg
    big = HestonPathGenerator(Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04), 100.0, 1.0, (1 << 30) + 1).to_abi()
    st, msg = _noalloc(big, [100.0])
    assert st == A.OF_ERR_INVALID_INPUT and "num_steps" in msg
    st, msg = _noalloc(model, [100.0 + k for k in range(65)])
    assert st == A.OF_ERR_INVALID_INPUT and "64" in msg
    st, msg = _noalloc(model, [100.0 + k for k in range(129)])
    assert st == A.OF_ERR_UNSUPPORTED and "128" in msg
