"""The C ABI library loads without a GPU, exports every entry point that
include/edm_b200.h declares, and its structs match the ctypes mirrors."""
import ctypes as C
import re
from pathlib import Path

import pytest

from flim_microscopy_simulator_with_causal_inference_b200 import engine as E
from flim_microscopy_simulator_with_causal_inference_b200 import params as PR

HEADER = Path(__file__).resolve().parents[1] / "include" / "edm_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"static inline[^{]*\{[^}]*\}", "", text)  # header-only helpers are not exported
    return sorted(set(re.findall(r"\b(edm_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    E.build_library()
    return E.load_library()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "edm_create" in names and "edm_dynamics_step" in names and "edm_pipeline_steps" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    raw = C.CDLL(str(E.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(raw, n)]
    assert not missing, f"missing exports: {missing}"


def test_abi_struct_sizes_match(lib):
    assert lib.edm_abi_version() == 3
    for which, cls in ((0, PR.EdmDynParams), (1, PR.EdmPhotParams), (2, PR.EdmScopeParams), (3, PR.EdmHostState),
                       (4, PR.EdmFlimParams)):
        assert lib.edm_abi_sizeof(which) == C.sizeof(cls), cls.__name__
    assert lib.edm_abi_sizeof(99) == -1


def test_create_rejects_bad_arguments_without_touching_the_gpu(lib):
    out = C.c_void_p()
    rc = lib.edm_create(None, None, None, 1, None, 0, 64, 0, C.byref(out))
    assert rc == -1
    assert b"null" in lib.edm_last_error()
    dp = PR.EdmDynParams()
    rc = lib.edm_create(C.byref(dp), None, None, 1, None, 0, 16, 0, C.byref(out))
    assert rc == -1 and b"precision" in lib.edm_last_error()


def test_engine_refuses_to_run_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        E.Engine([PR.EdmDynParams()], PR.np.zeros(0))


def test_flim_create_rejects_bad_parameters_without_touching_the_gpu(lib):
    out = C.c_void_p()
    assert lib.edm_flim_create(None, 0, C.byref(out)) == -1
    fp = PR.EdmFlimParams(nx=128, ny=128, n_replicas=1, n_bins=256)
    assert lib.edm_flim_create(C.byref(fp), 0, C.byref(out)) == -4
    assert b"256 x 256" in lib.edm_last_error()
    fp = PR.EdmFlimParams(nx=256, ny=256, n_replicas=1, n_emitters=10, n_bins=100, half_taps=3)
    assert lib.edm_flim_create(C.byref(fp), 0, C.byref(out)) == -1
    assert b"n_bins" in lib.edm_last_error()
    fp = PR.EdmFlimParams(nx=256, ny=256, n_replicas=1, n_emitters=10, n_bins=256, half_taps=3,
                          bin_width_ns=0.1, sigma_irf_ns=0.06, sigma_psf_px=3.0, tau_free_ns=-1.0,
                          tau_bound_ns=1.0)
    assert lib.edm_flim_create(C.byref(fp), 0, C.byref(out)) == -1
    assert not out.value
