"""The C ABI: libmdwt.so loads, exports every entry point of include/mdwt.h, and its
host-side logic answers without a GPU (host-only contexts)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mdwtracker_b200 import MDWT_HOST_ONLY, MdwtError, Renderer

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for h in ("mdwt.h", "mdwt_denoiser.h", "mdwt_batch.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms |= set(re.findall(r"\b(mdwt_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_header_declares_the_renderer_surface():
    syms = header_symbols()
    for must in ["mdwt_create", "mdwt_destroy", "mdwt_push_channel_raw", "mdwt_push_channel", "mdwt_init",
                 "mdwt_set_tf", "mdwt_set_opacity_scale", "mdwt_set_tf_range", "mdwt_set_dt", "mdwt_reset_dt",
                 "mdwt_set_camera", "mdwt_resize", "mdwt_render", "mdwt_reset_accumulation",
                 "mdwt_get_framebuffer", "mdwt_get_accum", "mdwt_get_majorants"]:
        assert must in syms


def test_library_exports_every_declared_symbol(mdwt_lib):
    syms = header_symbols()
    for must in ["mdwt_denoiser_create", "mdwt_denoiser_train_step", "mdwt_denoiser_infer", "mdwt_denoise",
                 "mdwt_render_expected", "mdwt_accum_rmse", "mdwt_set_features", "mdwt_batch_render",
                 "mdwt_batch_autotune", "mdwt_autotune_macrocells"]:
        assert must in syms
    missing = [s for s in syms if not hasattr(mdwt_lib, s)]
    assert not missing, missing


def test_denoiser_parameter_count_matches_the_reference_layout(mdwt_lib):
    from mdwtracker_b200 import Denoiser
    from oracle import denoiser_ref
    assert Denoiser.numParams(mdwt_lib) == denoiser_ref.num_params()


def test_status_strings(mdwt_lib):
    mdwt_lib.mdwt_status_string.restype = C.c_char_p
    assert mdwt_lib.mdwt_status_string(0) == b"ok"
    assert mdwt_lib.mdwt_status_string(4) == b"too many channels"
    assert mdwt_lib.mdwt_version() >> 16 == 1


def test_null_arguments_are_rejected(mdwt_lib):
    assert mdwt_lib.mdwt_create(None, 0) == 1
    assert mdwt_lib.mdwt_destroy(None) == 1
    assert mdwt_lib.mdwt_render(None, None) == 1


def test_host_only_context_refuses_init():
    r = Renderer(MDWT_HOST_ONLY)
    r.PushMesh(np.zeros((4, 4, 4), np.uint8))
    with pytest.raises(MdwtError) as e:
        r.Init(0)
    assert e.value.status == 6


def test_too_many_channels():
    r = Renderer(MDWT_HOST_ONLY)
    for _ in range(12):
        r.PushMesh(np.zeros((2, 2, 2), np.uint8))
    with pytest.raises(MdwtError) as e:
        r.PushMesh(np.zeros((2, 2, 2), np.uint8))
    assert e.value.status == 4


def test_bad_arguments():
    r = Renderer(MDWT_HOST_ONLY)
    with pytest.raises(MdwtError):
        r.PushMesh(np.zeros((4, 4, 4), np.complex64))
    with pytest.raises(MdwtError):
        r.setSpp(0)
    with pytest.raises(MdwtError):
        r.Resize((0, 10))
    with pytest.raises(MdwtError):
        r.channelInfo(0)
    with pytest.raises(MdwtError) as e:
        r.PushMesh("/nonexistent/vol_8x8x8_uint8.raw")
    assert e.value.status == 3
    with pytest.raises(MdwtError) as e:
        r.PushMesh("/nonexistent/volume_uint8.raw")
    assert e.value.status == 9
    with pytest.raises(MdwtError) as e:
        r.setLight(True, False, (0.0, 0.0, 0.0))
    assert e.value.status == 1
    r.setLight(False, True, (0.0, 0.0, 0.0))      # gradient alone: NdotL clamps to 0
    r.setLight(True, True, (0.0, -1.0, 0.0))


def test_gpu_absent_is_an_error_not_a_fallback():
    """Without a device the product refuses to create a render context."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(MdwtError) as e:
        Renderer(0)
    assert e.value.status == 2


def test_seed_block_accepts_powers_of_two_only():
    r = Renderer(MDWT_HOST_ONLY)
    for edge in (0, 1, 16, 1024):
        r.setSeedBlock(edge)
    for edge in (-1, 3, 12, 2048):
        with pytest.raises(MdwtError):
            r.setSeedBlock(edge)


def test_tuning_knobs_read_back():
    r = Renderer(MDWT_HOST_ONLY)
    # pool, batch, trips, quorum, regroup (off by default without -m 2), regrouped-tracker blocks
    assert [r.getTuning(k) for k in (0, 1, 2, 3, 4, 5)] == [8, 0, 4, 16, 0, 0]
    r.setTuning(4, 1)
    r.setTuning(2, 7)
    r.setTuning(5, 3)
    assert r.getTuning(4) == 1 and r.getTuning(2) == 7 and r.getTuning(5) == 3
    with pytest.raises(MdwtError):
        r.setTuning(4, 2)
    with pytest.raises(MdwtError):
        r.setTuning(5, 9)
    with pytest.raises(MdwtError):
        r.getTuning(9)


def test_arithmetic_is_exact_until_set():
    r = Renderer(MDWT_HOST_ONLY)
    assert r.arithmetic() == 0
    r.setArithmetic(True)
    assert r.arithmetic() == 1
    r.setArithmetic(False)
    assert r.arithmetic() == 0
    for bad in (-1, 2):
        with pytest.raises(MdwtError) as e:
            r.setArithmetic(bad)
        assert e.value.status == 1
    assert r.arithmetic() == 0
