"""Output formats (wholistic_registration_b200/IO.py, utils/IO.py:737-1033):
TIFF pages checked with an independent reader (Pillow), ImageJ hyperstack
shape and description, BigTIFF, zarr v2 stores (directory and zip) against
the format's rules and by round trip."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

PIL = pytest.importorskip("PIL.Image")


def _pil_pages(path):
    from PIL import Image

    im = Image.open(path)
    pages = []
    for i in range(getattr(im, "n_frames", 1)):
        im.seek(i)
        pages.append(np.array(im))
    return pages, im


@pytest.mark.parametrize("dtype", [np.uint16, np.float32, np.uint8])
def test_volume_tiff_pages_match_an_independent_reader(tmp_path, dtype):
    from wholistic_registration_b200 import IO

    rng = np.random.default_rng(3)
    vol = (rng.uniform(0, 250, (5, 40, 48))).astype(dtype)
    fname = IO.write_volume_as_ome_tiff(vol, str(tmp_path), "ch1", 7, "cfg.toml", spacing_x=0.5, spacing_y=0.25)
    assert os.path.basename(fname) == "vol_ch1_000007.tif"
    pages, im = _pil_pages(fname)
    assert len(pages) == 5
    for z in range(5):
        np.testing.assert_array_equal(pages[z].astype(dtype), vol[z])
    arr, desc = IO.readTiff(fname)
    assert arr.shape == (5, 40, 48) and arr.dtype == dtype
    np.testing.assert_array_equal(arr, vol)
    assert desc.startswith("ImageJ=") and "slices=5" in desc and "spacing_x=0.5" in desc and "config=cfg.toml" in desc
    np.testing.assert_array_equal(IO.read_reg_tiff(str(tmp_path), 7, 1), vol)
    im.seek(0)
    assert abs(float(im.tag_v2[282]) - 2.0) < 1e-9 and abs(float(im.tag_v2[283]) - 4.0) < 1e-9


def test_multichannel_hyperstack_page_order(tmp_path):
    from wholistic_registration_b200 import IO

    rng = np.random.default_rng(4)
    vols = [rng.uniform(0, 100, (4, 16, 20)).astype(np.float32) for _ in range(3)]
    IO.write_multichannel_volume_as_ome_tiff(vols, str(tmp_path), 12, label="rgb")
    fname = os.path.join(str(tmp_path), "vol_rgb_000012.tif")
    pages, _ = _pil_pages(fname)
    assert len(pages) == 12
    for z in range(4):
        for c in range(3):   # ImageJ order: channel fastest within a slice
            np.testing.assert_array_equal(pages[z * 3 + c], vols[c][z])
    arr, desc = IO.readTiff(fname)
    assert arr.shape == (4, 3, 16, 20) and "channels=3" in desc and "hyperstack=true" in desc
    np.testing.assert_array_equal(arr, np.stack(vols, axis=1))


def test_bigtiff_with_config_description(tmp_path):
    from wholistic_registration_b200 import IO

    cfg = tmp_path / "c.toml"
    cfg.write_text('[pyramid]\nr = 16\nlayer = 3\n[mask]\nthresFactor = 3.0\n')
    frames = [np.full((6, 9), k, np.uint16) + np.arange(54, dtype=np.uint16).reshape(6, 9) for k in range(3)]
    path = str(tmp_path / "s.tif")
    IO.saveTiff(frames, str(cfg), path)
    with open(path, "rb") as fh:
        assert fh.read(4) == b"II+\0"   # BigTIFF
    arr, desc = IO.readTiff(path)
    np.testing.assert_array_equal(arr, np.stack(frames))
    assert json.loads(desc) == {"pyramid": {"r": 16, "layer": 3}, "mask": {"thresFactor": 3.0}}
    pages, _ = _pil_pages(path)
    assert len(pages) == 3
    np.testing.assert_array_equal(pages[2], frames[2])


def test_frame_tags_follow_the_reference():
    from wholistic_registration_b200 import IO

    assert IO._frame_tag(5) == "000005"
    assert IO._frame_tag("100~200") == "000100_000200"
    assert IO._frame_tag("100-200") == "000100_000200"
    assert IO._frame_tag("1~2_vs_3~4") == "0001~0002_vs_0003~0004"
    with pytest.raises(ValueError):
        IO._frame_tag("a~b")
    with pytest.raises(TypeError):
        IO._frame_tag(1.5)


@pytest.mark.parametrize("single_file,compressor", [(False, None), (True, None), (False, "raw")])
def test_zarr_store_round_trip_and_format(tmp_path, single_file, compressor):
    from wholistic_registration_b200 import IO

    cfg = tmp_path / "c.toml"
    cfg.write_text('[channels]\ndual_channel = true\nk = 0.5\n')
    rng = np.random.default_rng(5)
    mem = rng.uniform(0, 1000, (5, 37, 41)).astype(np.float32)
    ca = rng.uniform(0, 1000, (5, 37, 41)).astype(np.float32)
    ref = rng.uniform(0, 1000, (37, 41)).astype(np.float32)
    path = str(tmp_path / "out.zarr")
    IO.saveZarr_fast(mem, ca, ref, str(cfg), path, chunks=(2, 16, 16), compressor=compressor, single_file=single_file)
    arrays, attrs = IO.readZarr(path + ".zip" if single_file else path)
    np.testing.assert_array_equal(arrays["membrane"], mem)
    np.testing.assert_array_equal(arrays["calcium"], ca)
    np.testing.assert_array_equal(arrays["reference"], ref)
    assert json.loads(attrs["config"]) == {"channels": {"dual_channel": True, "k": 0.5}}
    if not single_file:
        meta = json.load(open(os.path.join(path, "membrane", ".zarray")))
        assert meta["zarr_format"] == 2 and meta["shape"] == [5, 37, 41] and meta["chunks"] == [2, 16, 16]
        assert meta["dtype"] == "<f4" and meta["order"] == "C" and meta["filters"] is None
        assert meta["compressor"] == (None if compressor == "raw" else {"id": "zlib", "level": 1})
        assert json.load(open(os.path.join(path, ".zgroup"))) == {"zarr_format": 2}
        # 3 x 3 x 3 chunks, edge chunks stored at the full chunk shape
        assert sorted(os.listdir(os.path.join(path, "membrane")))[:2] == [".zarray", "0.0.0"]
        assert len([f for f in os.listdir(os.path.join(path, "membrane")) if not f.startswith(".")]) == 27
        if compressor == "raw":
            assert os.path.getsize(os.path.join(path, "membrane", "2.2.2")) == 2 * 16 * 16 * 4


def test_saveZarr_default_chunks(tmp_path):
    from wholistic_registration_b200 import IO

    cfg = tmp_path / "c.toml"
    cfg.write_text('[a]\nb = 1\n')
    mem = np.arange(3 * 20 * 30, dtype=np.float32).reshape(3, 20, 30)
    IO.saveZarr(mem, mem * 2, mem[0], str(cfg), str(tmp_path / "z"))
    arrays, _ = IO.readZarr(str(tmp_path / "z"))
    np.testing.assert_array_equal(arrays["calcium"], mem * 2)
    meta = json.load(open(tmp_path / "z" / "membrane" / ".zarray"))
    assert meta["chunks"] == [1, 20, 30]   # (1, 512, 512) clipped to the array
