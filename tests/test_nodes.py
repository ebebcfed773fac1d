"""The node layer without a GPU: kinds are registered under the reference's strings, settings are
parsed with the reference's keys, and infer() returns the reference's output descriptors or fails
with its "<Factory> inference error: ..." messages (restated from fresnel_diffraction.cu:94-99,
466-508, angular_spectrum.cu:446-494, pca.cc:157-193, conversion.cu:389-410, mean.cu:30-70)."""
import pytest

import holoflow_b200 as hf
from holoflow_b200 import nodes as N

U8, U16, F32, CF32 = 0, 1, 2, 3


def desc(shape, dtype=F32, device=True, strides=None):
    d = hf.HfTDesc()
    d.rank, d.dtype, d.mem_loc = len(shape), dtype, 1 if device else 0
    for i, n in enumerate(shape):
        d.shape[i] = n
    if strides:
        for i, s in enumerate(strides):
            d.strides[i] = s
    return d


FRESNEL = {"lambda": 852e-9, "dx": 12e-6, "dy": 12e-6, "z": 0.25}
AS = {"lambda": 852e-9, "dx": 12e-6, "dy": 12e-6, "z": 0.30}


def out_of(kind, settings, descs):
    (o,) = N.infer(kind, settings, descs)
    return N.shape_of(o), o.dtype


def invalid(kind, settings, descs, fragment):
    with pytest.raises(hf.HfError) as e:
        N.infer(kind, settings, descs)
    assert e.value.code == hf.HF_ERR_INVALID
    assert fragment in str(e.value), str(e.value)


def test_reference_kinds_are_registered():
    assert set(N.kinds()) == {"FresnelDiffraction", "AngularSpectrum", "Pca", "FFT", "RFFT", "Mean", "MeanAbs",
                              "Conversion", "Holofile", "FFTShiftNp", "Flatfield", "Filter2D", "PctClip",
                              "DopplerMoments", "ShortTimeFresnelDiffraction", "ShackHartmannSlopes",
                              "ZernikeFromSlopes", "ZernikePhase", "CorrectPhase", "Wrap2Pi", "ZernikeDefocusZProp",
                              "Slice", "Reshape", "Copy", "Concatenate", "Arange", "Multiply", "Abs",
                              "CausalSlidingAverage", "BatchQueue", "DualReaderBatchQueue", "SlidingAverage"}


def test_unknown_kind_and_bad_settings():
    invalid("Fresnel", FRESNEL, [desc([4, 8, 8], CF32)], "no synchronous task of kind 'Fresnel'")
    invalid("FresnelDiffraction", {"lambda": 1.0}, [desc([4, 8, 8], CF32)], "settings")


def test_fresnel_infer():
    assert out_of("FresnelDiffraction", FRESNEL, [desc([3, 64, 32], CF32)]) == ((3, 64, 32), CF32)
    assert out_of("FresnelDiffraction", FRESNEL, [desc([3, 64, 32], F32)]) == ((3, 64, 32), CF32)
    assert out_of("FresnelDiffraction", {**FRESNEL, "output_magnitude": True}, [desc([64, 32], CF32)]) == ((64, 32), F32)
    p = "FresnelDiffractionFactory inference error: "
    invalid("FresnelDiffraction", {**FRESNEL, "dy": 10e-6}, [desc([8, 8], CF32)], p + "dx must equal dy")
    invalid("FresnelDiffraction", {**FRESNEL, "lambda": 0.0}, [desc([8, 8], CF32)], p + "wavelength must be positive")
    invalid("FresnelDiffraction", FRESNEL, [desc([8], CF32)], p + "input must be a tensor of rank 2 or higher")
    invalid("FresnelDiffraction", FRESNEL, [desc([8, 8], U16)], p + "input must be complex float32 or real float32")
    invalid("FresnelDiffraction", FRESNEL, [desc([8, 8], CF32, device=False)], p + "input must be in device memory")
    invalid("FresnelDiffraction", {**FRESNEL, "axes": [0]}, [desc([8, 8], CF32)], p + "axes must contain exactly two")
    invalid("FresnelDiffraction", {**FRESNEL, "axes": [-1, -1]}, [desc([8, 8], CF32)], p + "axes must be distinct")
    # any two axes whose strides nest (fresnel_diffraction.cu:482-484)
    assert out_of("FresnelDiffraction", {**FRESNEL, "axes": [0, 1]}, [desc([64, 32, 3], CF32)]) == ((64, 32, 3), CF32)
    invalid("FresnelDiffraction", {**FRESNEL, "axes": [1, 0]}, [desc([64, 32], CF32)],
            p + "stride of ax0 (H) must be a multiple of stride of ax1 (W)")
    invalid("FresnelDiffraction", FRESNEL, [desc([2, 8, 8], CF32)] * 2, p + "expected exactly one input")


def test_angular_spectrum_infer():
    (o,) = N.infer("AngularSpectrum", AS, [desc([2, 64, 64], CF32)])
    assert N.shape_of(o) == (2, 64, 64) and o.dtype == CF32
    pad = {**AS, "padding": {"width": 96, "height": 80}}
    assert out_of("AngularSpectrum", pad, [desc([2, 64, 64], F32)]) == ((2, 80, 96), CF32)
    p = "AngularSpectrumFactory inference error: "
    invalid("AngularSpectrum", {**AS, "padding": {"width": 65, "height": 64}}, [desc([64, 64], CF32)],
            p + "horizontal padding must be even")
    invalid("AngularSpectrum", {**AS, "padding": {"width": 32, "height": 64}}, [desc([64, 64], CF32)],
            p + "padding width must be at least the input width")
    invalid("AngularSpectrum", AS, [desc([64, 64], CF32, strides=[1024, 8])], p + "input must be C-contiguous")


def test_pca_infer():
    assert out_of("Pca", {"begin": 2, "end": 5}, [desc([3, 16, 8, 8])]) == ((3, 3, 8, 8), F32)
    p = "PcaFactory inference error: "
    invalid("Pca", {"begin": 3, "end": 3}, [desc([16, 8, 8])], p + "expected begin < end")
    invalid("Pca", {"begin": -1, "end": 3}, [desc([16, 8, 8])], p + "expected begin >= 0")
    invalid("Pca", {"begin": 0, "end": 17}, [desc([16, 8, 8])], p + "expected end <= n_features")
    invalid("Pca", {"begin": 0, "end": 2}, [desc([8, 8])], p + "expected input rank >= 3")


def test_fft_rfft_infer():
    assert out_of("FFT", {"axis": 1, "norm": "ortho"}, [desc([2, 32, 8, 8], U16)]) == ((2, 32, 8, 8), CF32)
    assert out_of("RFFT", {"axis": 1}, [desc([2, 64, 8, 8])]) == ((2, 33, 8, 8), CF32)
    assert out_of("RFFT", {}, [desc([4, 10])]) == ((4, 6), CF32)  # axis defaults to -1
    invalid("FFT", {"axis": 4}, [desc([2, 32, 8, 8])], "FFTFactory inference error: axis out of range")
    invalid("RFFT", {"axis": 1}, [desc([2, 32, 8], CF32)], "RFFTFactory inference error: input must be real")
    with pytest.raises(hf.HfError, match="unsupported norm"):
        N.infer("FFT", {"axis": 1, "norm": "unitary"}, [desc([2, 32, 8])])


def test_mean_infer():
    assert out_of("Mean", {"axis": -3, "keepdims": True}, [desc([1, 28, 8, 8])]) == ((1, 1, 8, 8), F32)
    assert out_of("Mean", {"axis": 0}, [desc([1, 8, 8])]) == ((8, 8), F32)
    assert out_of("Mean", {"axes": [1, 2]}, [desc([2, 3, 4, 5], CF32)]) == ((2, 5), CF32)
    assert out_of("Mean", {"axis": None}, [desc([2, 3])]) == ((), F32)
    assert out_of("MeanAbs", {"axis": -3, "keepdims": True}, [desc([1, 28, 8, 8], CF32)]) == ((1, 1, 8, 8), F32)
    invalid("Mean", {"axis": 5}, [desc([2, 3])], "MeanFactory inference error: axis out of range")
    with pytest.raises(hf.HfError, match="axis must be int, array, or null"):
        N.infer("Mean", {"axis": "x"}, [desc([2, 3])])


def test_conversion_infer():
    conv = lambda t, s: {"target": t, "strategy": s}
    assert out_of("Conversion", conv("CF32", "Real"), [desc([4, 4], U16)]) == ((4, 4), CF32)
    assert out_of("Conversion", conv("U8", "Scaled"), [desc([4, 4], F32)]) == ((4, 4), U8)
    assert out_of("Conversion", conv("F32", "Argument"), [desc([4, 4], CF32)]) == ((4, 4), F32)
    invalid("Conversion", conv("F32", "Real"), [desc([4, 4], U16)],
            "ConversionFactory inference error: Unsupported conversion configuration")
    with pytest.raises(hf.HfError, match="Unknown strategy type for conversion: Linear"):
        N.infer("Conversion", conv("F32", "Linear"), [desc([4, 4], U8)])


def test_doppler_moments_infer():
    s = {"time_z_begin": 6, "time_z_end": 16, "propagation": "angular_spectrum", "lambda": 852e-9, "dx": 12e-6,
         "z": 0.3, "input_format": "u16", "padding": {"width": 96, "height": 80}}
    assert out_of("DopplerMoments", s, [desc([2, 32, 64, 64], U16)]) == ((2, 3, 80, 96), F32)
    s12 = {"time_z_begin": 4, "time_z_end": 32, "propagation": "fresnel", "lambda": 852e-9, "dx": 12e-6, "z": 0.25,
           "clutter_rank": 4, "input_format": "mono12p", "height": 64, "width": 64, "moments": ["M0"],
           "form": "chosen"}
    assert out_of("DopplerMoments", s12, [desc([3, 64, 64 * 64 * 3 // 2], U8)]) == ((3, 1, 64, 64), F32)
    p = "DopplerMomentsFactory inference error: "
    invalid("DopplerMoments", {**s12, "width": 32}, [desc([3, 64, 64 * 64 * 3 // 2], U8)],
            p + "height x width must match the packed frame size")
    invalid("DopplerMoments", {**s, "time_z_end": 40}, [desc([2, 32, 64, 64], U16)], p + "bad band")
    invalid("DopplerMoments", {**s, "moments": ["M3"]}, [desc([2, 32, 64, 64], U16)], p + "moments must be among")


def test_display_chain_infer():
    """FFTShiftNp (fftshift.cu:185-210), Flatfield (flatfield.cu:296-323), PctClip
    (pct_clip.cu:230-270): output descriptors and messages."""
    assert out_of("FFTShiftNp", {"axes": [-2, -1]}, [desc([1, 64, 48])]) == ((1, 64, 48), F32)
    assert out_of("FFTShiftNp", {}, [desc([3, 5], U8)]) == ((3, 5), U8)
    for s, msg in [({"axes": [2]}, "axis out of range"), ({"axes": [0, -2]}, "axes must be unique")]:
        invalid("FFTShiftNp", s, [desc([4, 4])], "FFTShift: " + msg)
    invalid("FFTShiftNp", {}, [desc([4, 4], device=False)], "FFTShift: only Device tensors are supported")
    assert out_of("Flatfield", {"sigma_y": 3.0, "sigma_x": 2.0}, [desc([2, 64, 64])]) == ((2, 64, 64), F32)
    p = "FlatfieldFactory inference error: "
    invalid("Flatfield", {"sigma_y": 0.0, "sigma_x": 2.0}, [desc([64, 64])], p + "sigma_y must be positive")
    invalid("Flatfield", {"sigma_y": 1.0, "sigma_x": -1.0}, [desc([64, 64])], p + "sigma_x must be positive")
    invalid("Flatfield", {"sigma_y": 1.0, "sigma_x": 1.0}, [desc([64])], p + "input must be a tensor of rank 2 or higher")
    invalid("Flatfield", {"sigma_y": 1.0, "sigma_x": 1.0}, [desc([8, 8], U16)], p + "input must be float32")
    roi = {"cx": 0.5, "cy": 0.5, "rx": 0.5, "ry": 0.5, "angle": 0.0}
    pc = {"min_pct": 1.0, "max_pct": 99.0, "roi": roi}
    assert out_of("PctClip", pc, [desc([1, 32, 32])]) == ((1, 32, 32), F32)
    p = "PctClipFactory inference error: "
    invalid("PctClip", {**pc, "min_pct": 99.0}, [desc([1, 8, 8])], p + "min_pct must be < max_pct")
    invalid("PctClip", {**pc, "max_pct": 101.0}, [desc([1, 8, 8])], p + "max_pct must be <= 100")
    invalid("PctClip", {**pc, "roi": {**roi, "rx": 0.0}}, [desc([1, 8, 8])], p + "roi.rx must be > 0")
    invalid("PctClip", {**pc, "roi": {**roi, "cy": 1.5}}, [desc([1, 8, 8])], p + "roi.cy must be <= 1")
    invalid("PctClip", pc, [desc([8, 8])], p + "input must be 3D")


def test_doppler_moments_two_sided_time_method():
    s = {"time_z_begin": 4, "time_z_end": 32, "propagation": "fresnel", "lambda": 852e-9, "dx": 12e-6, "z": 0.25,
         "input_format": "u16", "time_method": "fft"}
    assert out_of("DopplerMoments", s, [desc([1, 64, 64, 64], U16)]) == ((1, 3, 64, 64), F32)
    p = "DopplerMomentsFactory inference error: "
    invalid("DopplerMoments", {**s, "time_method": "stft"}, [desc([1, 64, 64, 64], U16)],
            p + "time_method must be rfft or fft")
    invalid("DopplerMoments", {**s, "time_z_begin": 0, "time_z_end": 33}, [desc([1, 64, 64, 64], U16)],
            p + "at most 64 band planes")


def test_filter2d_infer():
    f = {"r_inner": 2, "r_outer": 40, "s_inner": 3, "s_outer": 5}
    assert out_of("Filter2D", f, [desc([2, 64, 64], CF32)]) == ((2, 64, 64), CF32)
    assert out_of("Filter2D", f, [desc([64, 64], F32)]) == ((64, 64), F32)
    p = "Filter2DFactory inference error: "
    invalid("Filter2D", f, [desc([64, 64], U16)], p + "input must be complex float32 or real float32")
    invalid("Filter2D", f, [desc([64])], p + "input must be a tensor of rank 2 or higher")
    invalid("Filter2D", f, [desc([64, 64], CF32, device=False)], p + "input must be in device memory")


STFD = {"lambda": 852e-9, "dx": 20e-6, "dy": 20e-6, "z": 0.25, "win_h": 102, "win_w": 102, "stride_y": 102,
        "stride_x": 102, "phase_ref": "GLOBAL"}
SLOPES = {"lambda": 852e-9, "dx": 20e-6, "dy": 20e-6, "z": 0.25, "subaperture_height": 102, "subaperture_width": 102,
          "stride_y": 102, "stride_x": 102, "correlation_roi": {"rx": 0.5, "ry": 0.5}}
FIT = {"indexes": [4, 5, 6], "lambda": 852e-9, "dx": 20e-6, "dy": 20e-6, "subaperture_height": 102,
       "subaperture_width": 102, "stride_y": 102, "stride_x": 102}


def test_autofocus_kinds_infer():
    """ShortTimeFresnelDiffraction (short_time_fresnel_diffraction.cu:604-649), ShackHartmannSlopes
    (shack_hartmann_slopes.cu:326-388), ZernikeFromSlopes (zernike_from_slopes.cc:283-323),
    ZernikePhase (zernike_phase.cu:290-334), CorrectPhase (correct_phase.cu:160-190), Wrap2Pi,
    ZernikeDefocusZProp (zernike_defocus_z_prop.cc:173-211): output descriptors and messages."""
    assert out_of("ShortTimeFresnelDiffraction", STFD, [desc([2, 510, 510], CF32)]) == ((2, 5, 5, 102, 102), CF32)
    mag = dict(STFD, output_magnitude=True, stride_y=51, stride_x=34)
    assert out_of("ShortTimeFresnelDiffraction", mag, [desc([512, 520], F32)]) == ((9, 13, 102, 102), F32)
    p = "ShortTimeFresnelDiffractionFactory inference error: "
    invalid("ShortTimeFresnelDiffraction", dict(STFD, dy=1e-5), [desc([1, 64, 64], CF32)], p + "dx must equal dy")
    invalid("ShortTimeFresnelDiffraction", STFD, [desc([1, 64, 64], CF32)], p + "window dimensions exceed field size")
    invalid("ShortTimeFresnelDiffraction", STFD, [desc([1, 512, 512], U16)], p + "input must be CF32 or F32")
    invalid("ShortTimeFresnelDiffraction", dict(STFD, axes=[0, 1]), [desc([4, 512, 512], CF32)],
            p + "only trailing axes (-2, -1) are supported")

    assert out_of("ShackHartmannSlopes", SLOPES, [desc([1, 5, 5, 102, 102])]) == ((1, 5, 5, 2), F32)
    outs = N.infer("ShackHartmannSlopes", dict(SLOPES, output_xcorr_maps=True), [desc([1, 5, 5, 102, 102])])
    assert [N.shape_of(o) for o in outs] == [(1, 5, 5, 2), (1, 5, 5, 102, 102)]
    p = "ShackHartmannSlopesFactory inference error: "
    invalid("ShackHartmannSlopes", SLOPES, [desc([1, 4, 5, 102, 102])],
            p + "subaperture grid dimensions must be odd for an unambiguous center reference")
    invalid("ShackHartmannSlopes", SLOPES, [desc([5, 5, 102, 102])], p + "input rank must be 5")
    invalid("ShackHartmannSlopes", dict(SLOPES, z=-1.0), [desc([1, 5, 5, 102, 102])],
            p + "propagation distance must be > 0")
    invalid("ShackHartmannSlopes", dict(SLOPES, correlation_roi={"rx": 0.0}), [desc([1, 5, 5, 102, 102])],
            p + "correlation ROI radii must be positive")

    assert out_of("ZernikeFromSlopes", FIT, [desc([1, 5, 5, 2], device=False)]) == ((1, 1, 3), F32)
    p = "ZernikeFromSlopesFactory inference error: "
    invalid("ZernikeFromSlopes", dict(FIT, indexes=[4, 11]), [desc([1, 5, 5, 2])], p + "only Noll indexes 2..10")
    invalid("ZernikeFromSlopes", dict(FIT, indexes=[4, 4]), [desc([1, 5, 5, 2])], p + "indexes must be unique")
    invalid("ZernikeFromSlopes", dict(FIT, ny=2), [desc([1, 5, 5, 2])], p + "only global fitting with ny = nx = 1")
    invalid("ZernikeFromSlopes", FIT, [desc([1, 5, 5, 3])], p + "last input dimension must contain [dW/dx, dW/dy]")

    zp = {"indexes": [4, 5], "ny": 96, "nx": 130, "output": "Device"}
    assert out_of("ZernikePhase", zp, [desc([2])]) == ((96, 130), F32)
    p = "ZernikePhaseFactory inference error: "
    invalid("ZernikePhase", zp, [desc([2], device=False)], p + "Input coefficients must be in the output memory location")
    invalid("ZernikePhase", zp, [desc([3])], p + "Input coefficient count must match settings.indexes size")

    (o,) = N.infer("CorrectPhase", {}, [desc([4, 64, 48], CF32), desc([64, 48])])
    assert (N.shape_of(o), o.dtype) == ((4, 64, 48), CF32)
    invalid("CorrectPhase", {}, [desc([4, 64, 48], CF32), desc([64, 40])],
            "CorrectPhaseFactory inference error: phase mask width must match the input")
    assert out_of("Wrap2Pi", {}, [desc([7, 9])]) == ((7, 9), F32)
    zd = {"indexes": [4, 5], "lambda": 852e-9, "z_curr": 0.25, "pupil_radius": 5e-3}
    assert N.infer("ZernikeDefocusZProp", zd, [desc([2])]) == []
    invalid("ZernikeDefocusZProp", dict(zd, indexes=[5, 6]), [desc([2])],
            "ZernikeDefocusZPropFactory inference error: indexes must contain Z4 defocus")


def test_doppler_moments_autofocus_settings():
    """DopplerMoments takes the reference's autofocus settings names (settings.hh autofocus_*)."""
    s = {"time_z_begin": 3, "time_z_end": 9, "propagation": "fresnel", "lambda": 852e-9, "dx": 20e-6, "z": 0.25,
         "input_format": "f32", "autofocus_enabled": True, "autofocus_nb_subaps": 5, "autofocus_zernike_orders": [4, 5]}
    assert out_of("DopplerMoments", s, [desc([1, 32, 256, 256])]) == ((1, 3, 256, 256), F32)
    p = "DopplerMomentsFactory inference error: "
    invalid("DopplerMoments", {**s, "autofocus_nb_subaps": 4}, [desc([1, 32, 256, 256])], p + "autofocus_nb_subaps must be odd")
    invalid("DopplerMoments", {**s, "propagation": "angular_spectrum"}, [desc([1, 32, 256, 256])],
            p + "Shack-Hartmann autofocus needs fresnel propagation")


# ---- the thin holonp kinds and the queues GraphBuilder wires around the path -------------------
def test_slice_is_a_strided_view():
    """Slice (slice.cu:185-250): [8, 33, 4, 6] CF32 with [:, 4:32] is a view: shape [8, 28, 4, 6],
    the input's byte strides, offset 4 x stride(1); an integer item drops its dimension."""
    d = desc([8, 33, 4, 6], CF32)
    (o,) = N.infer("Slice", {"slices": [{}, {"start": 4, "stop": 32}, {}, {}]}, [d])
    assert N.shape_of(o) == (8, 28, 4, 6) and o.dtype == CF32
    assert [o.strides[i] for i in range(4)] == [33 * 24 * 8, 24 * 8, 6 * 8, 8] and o.offset == 4 * 24 * 8
    (o,) = N.infer("Slice", {"slices": [1, {"start": -3, "step": 2}, {}, {}]}, [d])
    assert N.shape_of(o) == (2, 4, 6) and o.offset == 33 * 24 * 8 + 30 * 24 * 8
    invalid("Slice", {"slices": [{}, {}]}, [d], "Slice: number of slice items must match input ndim")
    invalid("Slice", {"slices": [{}, {"step": -1}, {}, {}]}, [d], "Slice: only positive step is supported")


def test_reshape_copy_concatenate_infer():
    (o,) = N.infer("Reshape", {"shape": [1, 32, 4, -1]}, [desc([32, 4, 8])])
    assert N.shape_of(o) == (1, 32, 4, 8)
    invalid("Reshape", {"shape": [-1, -1]}, [desc([4, 8])], "Reshape: Only one dimension can be -1")
    invalid("Reshape", {"shape": [5, 7]}, [desc([4, 8])], "Reshape: Total elements mismatch")
    strided = desc([4, 8], F32, strides=[64, 4])          # rows 16 floats apart: no flat view
    invalid("Reshape", {"shape": [32], "copy": False}, [strided], "a view is not possible")
    (o,) = N.infer("Reshape", {"shape": [32]}, [strided])   # falls back to a contiguous copy
    assert N.shape_of(o) == (32,) and o.strides[0] == 4
    assert out_of("Copy", {}, [strided]) == ((4, 8), F32)
    invalid("Copy", {}, [desc([4, 8], F32, device=False)], "Copy: only Device tensors are supported")
    assert out_of("Concatenate", {"axis": 1}, [desc([2, 3, 5], CF32), desc([2, 4, 5], CF32)]) == ((2, 7, 5), CF32)
    invalid("Concatenate", {"axis": 1}, [desc([2, 3, 5], CF32), desc([2, 4, 5], F32)],
            "Concatenate: all inputs must share the same dtype")
    invalid("Concatenate", {"axis": 3}, [desc([2, 3, 5])], "Concatenate: axis out of range")


def test_arange_multiply_abs_infer():
    df = 37e3 / 64
    assert out_of("Arange", {"start": 4 * df, "stop": 32 * df, "step": df, "dtype": "F32"}, []) == ((28,), F32)
    invalid("Arange", {"start": 0.0, "stop": 1.0, "step": 0.0}, [], "ArangeFactory inference error: step must be non-zero")
    assert out_of("Multiply", {}, [desc([1, 28, 1, 1]), desc([1, 28, 16, 16], CF32)]) == ((1, 28, 16, 16), CF32)
    invalid("Multiply", {}, [desc([1, 28, 1, 1]), desc([1, 27, 16, 16])], "Multiply: input shapes are not broadcastable")
    assert out_of("Abs", {}, [desc([1, 28, 8, 8], CF32)]) == ((1, 28, 8, 8), F32)
    invalid("Abs", {}, [desc([4, 8], CF32, strides=[128, 8])], "Abs: input tensor must be contiguous")


def test_queue_kinds_infer():
    """BatchQueue (batch_queue.cc:188-222) and DualReaderBatchQueue (dual_reader_batch_queue.cc:
    231-262): owned inputs and outputs, the reference's messages."""
    (o,) = N.infer("BatchQueue", {"target_capacity": 16, "output_size": 8, "output_stride": 8}, [desc([1, 32, 8, 8])])
    assert N.shape_of(o) == (8, 32, 8, 8)
    invalid("BatchQueue", {"target_capacity": 16, "output_size": 8, "output_stride": 4}, [desc([1, 32, 8, 8])],
            "BatchQueueFactory inference error: BatchQueue task output stride must be a multiple of output size")
    outs = N.infer("DualReaderBatchQueue", {"target_capacity": 16, "window_size": 3}, [desc([8, 28, 8, 8], CF32)])
    assert [N.shape_of(o) for o in outs] == [(1, 28, 8, 8), (1, 28, 8, 8), (1,)]
    assert outs[2].dtype == U8 and outs[2].mem_loc == 0
    invalid("DualReaderBatchQueue", {"target_capacity": 16, "window_size": 0}, [desc([8, 28, 8, 8], CF32)],
            "DualReaderBatchQueueFactory inference error: window_size must be positive")
    assert out_of("SlidingAverage", {"target_capacity": 4, "window_size": 3}, [desc([1, 16, 16])]) == ((1, 16, 16), F32)
    invalid("CausalSlidingAverage", {"window_size": 2}, [desc([1, 16, 16], CF32)],
            "CausalSlidingAverageFactory inference error: input dtype must be F32")
