"""The autofocus C ABI without a GPU: argument validation with the reference factories' messages
(graph_builder.cc:311-334, short_time_fresnel_diffraction.cu:609-625, shack_hartmann_slopes.cu:
334-370, zernike_from_slopes.cc:290-320), which returns before any device call, and the
defocus-to-distance estimate (zernike_defocus_z_prop.cc:84-97) against the oracle."""
import ctypes as C
import math

import pytest

import holoflow_b200 as hf
from oracle import shack as SH

LAM, DX, Z = 852e-9, 20e-6, 0.25


def lib():
    return hf.lib()


def err(rc):
    return rc, lib().hf_last_error().decode()


def ints(v):
    return (C.c_int * max(1, len(v)))(*v), len(v)


@pytest.mark.parametrize("nb,msg", [(4, "autofocus_nb_subaps must be odd"), (0, "autofocus_nb_subaps must be positive"),
                                    (65, "autofocus_nb_subaps is too large for the current frame size")])
def test_autofocus_create_validation(nb, msg):
    h = C.c_void_p()
    arr, n = ints([4])
    rc, text = err(lib().hf_autofocus_create(2, 64, 64, nb, 1, LAM, DX, Z, 0.5, 1, arr, n, 0.0, None, C.byref(h)))
    assert rc == hf.HF_ERR_INVALID and msg in text and not h


def test_autofocus_iterations_and_orders_validation():
    h = C.c_void_p()
    arr, n = ints([4])
    rc, text = err(lib().hf_autofocus_create(2, 64, 64, 5, 0, LAM, DX, Z, 0.5, 1, arr, n, 0.0, None, C.byref(h)))
    assert rc == hf.HF_ERR_INVALID and "autofocus_nb_iter must be positive" in text
    arr, n = ints([4, 11])
    rc, text = err(lib().hf_autofocus_create(2, 64, 64, 5, 1, LAM, DX, Z, 0.5, 1, arr, n, 0.0, None, C.byref(h)))
    assert rc == hf.HF_ERR_INVALID and "only Noll indexes 2..10 are supported" in text


@pytest.mark.parametrize("kw,msg", [
    (dict(dy=2 * DX), "dx must equal dy"), (dict(z=0.0), "z must be non-zero"), (dict(lam=0.0), "lambda must be positive"),
    (dict(win=(128, 64)), "window dimensions exceed field size"), (dict(stride=(0, 8)), "strides must be >= 1"),
])
def test_stfd_create_validation(kw, msg):
    a = dict(lam=LAM, dx=DX, dy=DX, z=Z, win=(32, 32), stride=(32, 32))
    a.update(kw)
    h = C.c_void_p()
    rc, text = err(lib().hf_stfd_create(1, 64, 64, 0, a["win"][0], a["win"][1], a["stride"][0], a["stride"][1],
                                        a["lam"], a["dx"], a["dy"], a["z"], hf.HF_STFD_GLOBAL, hf.HF_STFD_COMPLEX, 1, 0,
                                        None, C.byref(h)))
    assert rc == hf.HF_ERR_INVALID and "ShortTimeFresnelDiffractionFactory: " + msg in text


def test_stfd_sides_beyond_the_transform_are_unsupported():
    h = C.c_void_p()
    rc, text = err(lib().hf_stfd_create(1, 2048, 2048, 0, 2048, 2048, 2048, 2048, LAM, DX, DX, Z, hf.HF_STFD_LOCAL,
                                        hf.HF_STFD_COMPLEX, 1, 0, None, C.byref(h)))
    assert rc == hf.HF_ERR_UNSUPPORTED and "window sides must be in 2..1024" in text


@pytest.mark.parametrize("args,msg", [
    ((4, 5, 32, 32), "subaperture grid dimensions must be odd for an unambiguous center reference"),
    ((5, 5, 1, 32), "reconstruction dimensions must be at least 2"),
])
def test_slopes_create_validation(args, msg):
    h = C.c_void_p()
    roi = hf.HfEllipse(0.5, 0.5, 0.5, 0.5, 0.0)
    rc, text = err(lib().hf_shslopes_create(*args, 0, 0, 0, 0, LAM, DX, DX, Z, C.byref(roi), 1, None, C.byref(h)))
    assert rc == hf.HF_ERR_INVALID and "ShackHartmannSlopesFactory inference error: " + msg in text
    roi = hf.HfEllipse(0.5, 0.5, 0.0, 0.5, 0.0)
    rc, text = err(lib().hf_shslopes_create(5, 5, 32, 32, 0, 0, 0, 0, LAM, DX, DX, Z, C.byref(roi), 1, None,
                                            C.byref(h)))
    assert rc == hf.HF_ERR_INVALID and "correlation ROI radii must be positive" in text


@pytest.mark.parametrize("idx,msg", [([], "indexes must not be empty"), ([4, 4], "indexes must be unique"),
                                     ([1], "only Noll indexes 2..10 are supported"),
                                     (list(range(2, 11)) + [4], "too many requested Zernike modes")])
def test_zernike_fit_create_validation(idx, msg):
    h = C.c_void_p()
    arr, n = ints(idx)
    rc, text = err(lib().hf_zernike_fit_create(5, 5, 10, 10, 10, 10, 0.5, 1.0, 1.0, 1, arr, n, C.byref(h)))
    assert rc == hf.HF_ERR_INVALID and "ZernikeFromSlopesFactory inference error: " + msg in text


@pytest.mark.parametrize("a4", [0.0, 1.7, -3.2, 12.0])
def test_defocus_estimate_matches_oracle(a4):
    d = [C.c_double() for _ in range(3)]
    assert lib().hf_defocus_z(a4, LAM, Z, 5e-3, *[C.byref(v) for v in d]) == hf.HF_OK
    exp = SH.defocus_z(a4, float(C.c_float(LAM).value), Z, float(C.c_float(5e-3).value))
    for got, want in zip(d, exp):
        assert math.isclose(got.value, want, rel_tol=1e-6, abs_tol=1e-12)


def test_defocus_estimate_validation():
    d = [C.c_double() for _ in range(3)]
    rc, text = err(lib().hf_defocus_z(1.0, LAM, 0.0, 5e-3, *[C.byref(v) for v in d]))
    assert rc == hf.HF_ERR_INVALID and "z_curr must be non-zero" in text
    rc, text = err(lib().hf_defocus_z(1.0, LAM, Z, 0.0, *[C.byref(v) for v in d]))
    assert rc == hf.HF_ERR_INVALID and "pupil_radius must be positive" in text
