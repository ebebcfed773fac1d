"""The C ABI without a GPU: the shared library loads, exports every function include/*.h declares,
and rejects malformed arguments with HF_ERR_INVALID and a message before touching the device."""
import ctypes as C

import pytest

import holoflow_b200 as hf
from holoflow_b200 import pipeline as pl


def test_library_exports_every_declared_symbol():
    lib = hf.lib()
    names = hf.declared_symbols()
    assert len(names) >= 39
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    # and the binding declares a prototype for each of them
    assert sorted(set(names) - set(hf._PROTOS)) == []


def test_version_and_launch_counter():
    lib = hf.lib()
    assert lib.hf_version() >= 1
    lib.hf_reset_launch_count()
    assert lib.hf_launch_count() == 0


def _expect_invalid(rc, fragment):
    assert rc == hf.HF_ERR_INVALID
    msg = hf.lib().hf_last_error().decode()
    assert fragment in msg, msg


def test_null_pointers_are_rejected():
    lib = hf.lib()
    _expect_invalid(lib.hf_covariance(None, hf.HF_MONO12P, 1, 64, 1024, None, None, None), "null")
    _expect_invalid(lib.hf_covariance_noalloc(None, hf.HF_MONO12P, 1, 64, 1024, None, None), "null")
    _expect_invalid(lib.hf_eigh_jacobi_f64(None, None, None, None, 64, 1, None), "null")
    _expect_invalid(lib.hf_pipeline_exec(None, None, 64, 0, 1, None, None), "null")
    _expect_invalid(lib.hf_stream_create(None, 256, None), "null")


def test_bad_extents_are_rejected():
    lib = hf.lib()
    buf = (C.c_uint8 * 64)()
    g = (C.c_double * 64)()
    _expect_invalid(lib.hf_covariance(buf, hf.HF_MONO12P, 0, 64, 1024, g, buf, None), "extents")
    _expect_invalid(lib.hf_covariance(buf, hf.HF_MONO12P, 1, 64, 1023, g, buf, None), "even P")
    _expect_invalid(lib.hf_covariance(buf, 99, 1, 64, 1024, g, buf, None), "dtype")
    _expect_invalid(lib.hf_covariance_noalloc(buf, hf.HF_MONO12P, 70000, 64, 1024, g, None), "extents")


@pytest.mark.parametrize("field,value,fragment", [
    ("height", 0, "frame size"),
    ("frames", 1, "frames per window"),
    ("frames", 129, "frames per window"),
    ("hop", 0, "hop"),
    ("z_end", 65, "band"),
    ("input_dtype", 7, ""),
    ("clutter_rank", 64, "clutter rank"),
    ("moment_mask", 8, "moment mask"),
    ("max_batch", 0, "max_batch"),
    ("form", 5, "form"),
    ("lambda_", 0.0, "wavelength"),
])
def test_plan_descriptor_validation(field, value, fragment):
    cfg = pl.PipelineConfig(height=256, width=256, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.25,
                            clutter_rank=4)
    d = cfg.desc()
    setattr(d, field, value)
    plan = C.c_void_p()
    _expect_invalid(hf.lib().hf_plan_create(C.byref(d), C.byref(plan), None), fragment)
    assert not plan.value
