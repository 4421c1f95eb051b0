"""The C-ABI library loads and exports every symbol include/bv_pairhmm.h
declares; host-only entry points behave without a device."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from biovoltron_b200 import native as N
from biovoltron_b200 import workloads as W

pytestmark = pytest.mark.skipif(not os.path.exists(N.LIB_PATH), reason="native library not built")


def test_exports_every_header_function():
    lib = N.load()
    names = N.header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert f" T {n}" in out, n


def test_shacc_hook_symbol_has_cpp_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    # shacc_pairhmm::calculate(shacc_pairhmm::Batch&)
    assert "_ZN13shacc_pairhmm9calculateERNS_5BatchE" in out


def test_built_for_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", N.LIB_PATH], capture_output=True, text=True).stdout
    assert "sm_100a" in out
    assert "sm_90" not in out and "sm_80" not in out


def test_default_options_and_abi():
    lib = N.load()
    o = N.Options()
    lib.bv_phmm_default_options(C.byref(o))
    assert o.struct_size == C.sizeof(N.Options)
    assert o.rescue_threshold == 1e-28
    assert o.precision == N.BV_PRECISION_AUTO and o.mode == N.BV_MODE_FULL
    assert lib.bv_phmm_abi_version() == 3
    assert lib.bv_phmm_status_string(N.BV_ERR_INVALID_ARG) == b"invalid argument"


def test_default_band_options():
    """The ctypes mirror has the C struct's size, and the defaults are the
    documented ones: fixed band of +-8 diagonals, margin 2, ring threshold
    1e-3, no audit, rescore 12 log10 units below the read's best."""
    lib = N.load()
    o = N.BandOptions()
    lib.bv_phmm_default_band_options(C.byref(o))
    assert o.struct_size == C.sizeof(N.BandOptions) == 56
    assert (o.enabled, o.use_mlp, o.fixed_half, o.margin, o.audit_period) == (1, 0, 8, 2, 0)
    assert o.edge_threshold == 1e-3 and o.cap_margin == 12.0
    assert list(o.reserved) == [0] * 5


def test_create_rejects_bad_options_before_touching_a_device():
    lib = N.load()
    h = C.c_void_p()
    o = N.Options()
    lib.bv_phmm_default_options(C.byref(o))
    o.struct_size = 3
    assert lib.bv_phmm_create(C.byref(o), C.byref(h)) == N.BV_ERR_INVALID_ARG
    lib.bv_phmm_default_options(C.byref(o))
    o.precision = 9
    assert lib.bv_phmm_create(C.byref(o), C.byref(h)) == N.BV_ERR_INVALID_ARG
    assert lib.bv_phmm_create(C.byref(o), None) == N.BV_ERR_INVALID_ARG


def test_null_context_calls_fail_cleanly():
    lib = N.load()
    assert lib.bv_phmm_compute_regions(None, None, None, None) == N.BV_ERR_INVALID_ARG
    assert lib.bv_phmm_run_staged(None, None) == N.BV_ERR_INVALID_ARG
    assert lib.bv_phmm_fetch_results(None, None, 0) == N.BV_ERR_INVALID_ARG
    assert lib.bv_phmm_last_error(None) == b"null context"


def test_region_result_count():
    from biovoltron_b200.pairhmm import _BatchView
    b = W.config1(seed=5, n_regions=9)
    v = _BatchView(b)
    assert N.load().bv_phmm_region_results(C.byref(v.c)) == b.n_pairs


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = N.load()
    h = C.c_void_p()
    assert lib.bv_phmm_create(None, C.byref(h)) == N.BV_ERR_NO_DEVICE
    assert not h.value


def test_new_entry_points_reject_bad_arguments_without_a_device():
    lib = N.load()
    h = C.c_void_p()
    o = N.Options()
    for field, value in (("pipeline_chunks", -1), ("pipeline_chunks", 65), ("pipeline_min_pairs", -5)):
        lib.bv_phmm_default_options(C.byref(o))
        setattr(o, field, value)
        assert lib.bv_phmm_create(C.byref(o), C.byref(h)) == N.BV_ERR_INVALID_ARG
    assert lib.bv_phmm_set_transitions(None, None) == N.BV_ERR_INVALID_ARG
    assert lib.bv_phmm_get_transitions(None, None) == 0
    assert lib.bv_phmm_genotype_staged(None, None, None, None, None, None, None, None) == N.BV_ERR_INVALID_ARG
    assert lib.bv_phmm_debug_chunks(None, 4, None, 0) == -1
    lib.bv_phmm_default_options(C.byref(o))
    assert o.pipeline_chunks == 0 and o.pipeline_min_pairs == 0
