"""C ABI: the built library loads, exports every function the header
declares, and behaves on a machine without a GPU (no compute calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from sph_3_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "sph3.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sph3_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from sph_3_b200 import build
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name


def test_defaults_and_strings(lib):
    cfg = _lib.default_config()
    assert cfg.n_ngb == 64 and cfg.n_ngb_tol == 5 and cfg.theta == 0.5 and cfg.eps == 0.01
    assert cfg.gamma == pytest.approx(5.0 / 3.0) and cfg.alpha == 1.0 and cfg.beta == 2.0
    assert lib.sph3_version() >= 10000
    for code in range(8):
        assert lib.sph3_error_string(code)
    assert _lib.C["SPH3_STATUS_H_NOT_CONVERGED"] == 1


def test_config_struct_layout_matches_header(lib):
    # sph3_default_config writes the full struct; a layout mismatch would
    # leave the trailing doubles at 0
    cfg = _lib.Config()
    ctypes.memset(ctypes.byref(cfg), 0xFF, ctypes.sizeof(cfg))
    lib.sph3_default_config(ctypes.byref(cfg))
    assert cfg.eps == 0.01 and list(cfg.box) == [0.0, 0.0, 0.0] and list(cfg.reserved_d) == [0.0] * 4


def test_ref_binding_config_matches_package_config(lib):
    # the stand-alone ctypes stub (copied next to the reference's sph_code/)
    # must declare the same struct as the package's own binding
    from sph_3_b200 import ref_binding
    a = [(n, getattr(_lib.Config, n).offset, getattr(_lib.Config, n).size) for n, _ in _lib.Config._fields_]
    b = [(n, getattr(ref_binding.Config, n).offset, getattr(ref_binding.Config, n).size)
         for n, _ in ref_binding.Config._fields_]
    assert a == b and ctypes.sizeof(_lib.Config) == ctypes.sizeof(ref_binding.Config)
    cfg = ref_binding.Config()
    lib.sph3_default_config(ctypes.byref(cfg))
    assert cfg.list_cap == 128 and cfg.stack_cap == 768 and cfg.theta == 0.5


def test_invalid_arguments_rejected_without_device(lib):
    out = ctypes.c_void_p()
    cfg = _lib.default_config()
    cfg.leaf_size = 0
    assert lib.sph3_ctx_create(ctypes.byref(cfg), -1, ctypes.byref(out)) == _lib.C["SPH3_ERR_INVALID_ARG"]
    cfg = _lib.default_config()
    cfg.box[0] = 1.0  # periodic with gravity on
    assert lib.sph3_ctx_create(ctypes.byref(cfg), -1, ctypes.byref(out)) == _lib.C["SPH3_ERR_UNSUPPORTED"]
    cfg = _lib.default_config()
    cfg.stack_cap = 64  # below 7 (max_level + 2) + 32
    assert lib.sph3_ctx_create(ctypes.byref(cfg), -1, ctypes.byref(out)) == _lib.C["SPH3_ERR_INVALID_ARG"]
    assert lib.sph3_ctx_create(None, -1, None) == _lib.C["SPH3_ERR_INVALID_ARG"]


def test_no_gpu_fails_loudly(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    out = ctypes.c_void_p()
    rc = lib.sph3_ctx_create(None, -1, ctypes.byref(out))
    assert rc == _lib.C["SPH3_ERR_NO_DEVICE"]
    from sph_3_b200 import Context, Sph3Error
    with pytest.raises(Sph3Error):
        Context()
    # the roofline probe too: no CPU stand-in for a measured GPU rate
    v = ctypes.c_double(-1.0)
    assert lib.sph3_probe_fp32_rate(0, ctypes.byref(v), None) == _lib.C["SPH3_ERR_NO_DEVICE"]
    assert v.value == -1.0
    assert lib.sph3_probe_fp32_rate(0, None, None) == _lib.C["SPH3_ERR_INVALID_ARG"]


def test_python_config_roundtrip(lib):
    from sph_3_b200 import Config
    c = Config(precision="fp64", h_mode="refstep", visc="balsara", n_ngb=50, box=(1.0, 2.0, 0.5),
               gravity=False).to_c()
    assert c.precision == _lib.C["SPH3_PREC_FP64"] and c.h_mode == _lib.C["SPH3_H_REFSTEP"]
    assert c.visc == _lib.C["SPH3_VISC_BALSARA"] and c.n_ngb == 50 and list(c.box) == [1.0, 2.0, 0.5]
    assert c.gravity == 0
