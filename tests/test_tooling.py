"""Image/TF files and the headless offline front end (CPU: driven through the oracle)."""
import os

import numpy as np
import pytest

from mdwtracker_b200 import cli, imageio
from mdwtracker_b200 import synthetic as syn


def test_png_roundtrip_and_flip(tmp_path):
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (7, 5, 4), dtype=np.uint8)
    p = str(tmp_path / "a.png")
    imageio.write_png(p, img, flip=True)
    np.testing.assert_array_equal(imageio.read_png(p), img[::-1])
    imageio.write_png(p, img, flip=False)
    np.testing.assert_array_equal(imageio.read_png(p), img)
    fb = img.copy().view(np.uint32)[..., 0]
    imageio.write_png(p, fb, flip=False)
    np.testing.assert_array_equal(imageio.read_png(p), img)


def test_ppm_pfm_headers(tmp_path):
    img = np.zeros((3, 4, 4), np.uint8)
    imageio.write_ppm(str(tmp_path / "a.ppm"), img)
    assert open(tmp_path / "a.ppm", "rb").read().startswith(b"P6\n4 3\n255\n")
    acc = np.ones((3, 4, 4), np.float32)
    imageio.write_pfm(str(tmp_path / "a.pfm"), acc)
    data = open(tmp_path / "a.pfm", "rb").read()
    assert data.startswith(b"PF\n4 3\n-1.0\n") and len(data) == len(b"PF\n4 3\n-1.0\n") + 3 * 4 * 3 * 4


def test_tf_file_roundtrip(tmp_path):
    cm = syn.ramp_tf((1.0, 0.5, 0.25))
    p = str(tmp_path / "a.tf")
    imageio.save_tf(p, cm, 2.5, (0.1, 0.9))
    cm2, os_, rng = imageio.load_tf(p)
    np.testing.assert_array_equal(cm2, cm)
    assert os_ == 2.5 and rng == (0.1, 0.9)


def test_cli_argument_checks():
    parse = cli.build_parser().parse_args
    with pytest.raises(SystemExit):
        cli.validate(parse([]))
    with pytest.raises(SystemExit):
        cli.validate(parse(["-fr", "x_2x2x2_uint8.raw", "-mc", "0"]))
    with pytest.raises(SystemExit):
        cli.validate(parse(["-fr", "x_2x2x2_uint8.raw", "-mc", "2", "3"]))
    with pytest.raises(SystemExit):
        cli.validate(parse(["-fr", "x_2x2x2_uint8.raw", "-cb", "1", "2"]))
    a = parse(["-fr", "x_2x2x2_uint8.raw", "-mc", "4", "-c"] + ["1"] * 10 + ["-l", "0", "0", "0", "-1", "0"])
    cli.validate(a)
    assert a.macrocells == [4] and len(a.camera) == 10


def _write_scene(tmp_path):
    vol = syn.value_noise_sparse(24, 0.3, 5, octaves=3)
    raw = str(tmp_path / "vol_24x24x24_uint8.raw")
    vol.tofile(raw)
    tf = str(tmp_path / "a.tf")
    imageio.save_tf(tf, syn.ramp_tf(syn.HUES[0]), 1.5, (0.0, 0.9))
    return raw, tf


def test_cli_frame_loop_on_the_oracle(tmp_path, oracle, capsys):
    raw, tf = _write_scene(tmp_path)
    out = str(tmp_path / "shot")
    a = cli.build_parser().parse_args(["-fr", raw, "-t", tf, "-mc", "3", "-r", "20", "16", "-m", "2", "-spp", "2",
                                       "-n", "3", "-wu", "1", "-nt", "2", "-o", out, "-bg", "0.1", "0.2", "0.3"])
    cli.validate(a)
    r = cli.setup(a, oracle.OracleRenderer())
    res = cli.run(a, r)
    assert res["frames"] == 3
    txt = capsys.readouterr().out
    assert "avg. fps" in txt and "Mode: AMMB" in txt
    final = imageio.read_png(out + "_AMMB_w_3_shadows_off_frames.png")
    np.testing.assert_array_equal(final, imageio.rgba8_to_array(r.framebuffer())[::-1])
    assert os.path.exists(out + "_AMMB_w_2_shadows_off_frames.png")
