"""CPU checks of the C-ABI library: it loads without a GPU and exports every
entry point the public header declares."""
import ctypes as C
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def header_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"^NB_API\s+[\w\s\*]+?\b(nb_\w+)\s*\(", h.read_text(), re.M))
    return names


def test_header_declares_the_binding_list(nbp):
    assert header_symbols() == set(nbp.EXPORTS)


def test_library_exports_every_declared_symbol(nbp):
    lib = nbp.load()
    for name in header_symbols():
        assert hasattr(lib, name), name


def test_status_strings(nbp):
    lib = nbp.load()
    assert lib.nb_status_string(0) == b"ok"
    assert lib.nb_status_string(3) == b"device capacity exceeded"
    assert lib.nb_last_error(None) == b"null context"


def test_params_default(nbp):
    lib = nbp.load()
    p = nbp.NbParams()
    assert lib.nb_params_default(C.byref(p)) == 0
    assert (p.G, p.timestep, p.theta, p.epsilon_squared, p.mode) == (1.0, 1e-4, 0.5, 1e-4, 0)


def test_invalid_arguments_rejected_before_any_device_call(nbp):
    lib = nbp.load()
    h = C.c_void_p()
    p = nbp.NbParams()
    lib.nb_params_default(C.byref(p))
    p.theta = -1.0
    one = (C.c_double * 2)(0.0, 0.0)
    assert lib.nb_create(C.byref(p), 1, one, one, one, C.byref(h)) == 1
    lib.nb_params_default(C.byref(p))
    assert lib.nb_create(C.byref(p), 0, one, one, one, C.byref(h)) == 1
    assert lib.nb_create(None, 1, one, one, one, C.byref(h)) == 1
    assert lib.nb_destroy(None) == 0
    # context calls with no context, and empty or missing arrays
    assert lib.nb_upload_async(None, one, one, one) == 1
    assert lib.nb_download_async(None, one, one) == 1
    params = (C.c_float * nbp.NB_MLP_PARAMS)()
    feats = (C.c_float * 12)()
    out = (C.c_float * 2)()
    assert lib.nb_mlp_forward(0, params, 0, feats, out) == 1
    assert lib.nb_mlp_forward(0, None, 1, feats, out) == 1


def test_batch_create_rejects_bad_batches_before_any_device_call(nbp):
    lib = nbp.load()
    h = C.c_void_p()
    p = nbp.NbParams()
    lib.nb_params_default(C.byref(p))
    one = (C.c_double * 8)(*([0.0] * 8))
    counts = (C.c_uint64 * 2)(1, 1)
    # FP64 parity mode holds one universe
    assert lib.nb_batch_create(C.byref(p), 2, counts, one, one, one, C.byref(h)) == 1
    p.mode = nbp.NB_MODE_SPLIT
    assert lib.nb_batch_create(C.byref(p), 0, counts, one, one, one, C.byref(h)) == 1
    assert lib.nb_batch_create(C.byref(p), 1025, counts, one, one, one, C.byref(h)) == 1
    assert lib.nb_batch_create(C.byref(p), 2, None, one, one, one, C.byref(h)) == 1
    empty = (C.c_uint64 * 2)(1, 0)
    assert lib.nb_batch_create(C.byref(p), 2, empty, one, one, one, C.byref(h)) == 1
    p.flags = nbp.NB_FLAG_LEARNED
    assert lib.nb_batch_create(C.byref(p), 2, counts, one, one, one, C.byref(h)) == 1
    assert lib.nb_autotune(None, 1, None, None) == 1


def test_bmax_ratio_validated(nbp):
    lib = nbp.load()
    h = C.c_void_p()
    p = nbp.NbParams()
    lib.nb_params_default(C.byref(p))
    assert p.bmax_ratio == 0.0
    one = (C.c_double * 2)(0.0, 0.0)
    for bad in (-0.5, float("nan"), float("inf")):
        p.bmax_ratio = bad
        assert lib.nb_create(C.byref(p), 1, one, one, one, C.byref(h)) == 1
