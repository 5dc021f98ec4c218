"""The reference's text image format (Image::initSelfFromFile, ImageUtils.cu:84-146) through
cpx_image_load_text / cpx_image_mask_pixels -- host code, run on the CPU: planes read back,
the mask bounds of readMask (Utils.cu:508-552) and processMasksInfo's rectangle of pixels."""
import numpy as np
import pytest


def _write(path, a, rows, cols):
    with open(path, "w") as f:
        for r in range(rows):
            f.write("".join("%d " % int(v) for v in a[r * cols:(r + 1) * cols]) + "\n")


def test_image_text_round_trip(tmp_path):
    import cpx

    w, h = 37, 23
    rng = np.random.default_rng(5)
    planes = [rng.integers(0, 256, w * h).astype(np.uint8) for _ in range(3)]
    mask = np.zeros((h, w), np.uint8)
    mask[4:17, 9:30] = 255
    mask[5, 3] = 7  # any nonzero value widens the bounds
    prefix = str(tmp_path / "img_000")
    for name, p in zip(("red", "green", "blue"), planes):
        _write(prefix + "_%s.txt" % name, p, h, w)
    _write(prefix + "_mask.txt", mask.reshape(-1), h, w)
    img, box, pix = cpx.load_image_text(prefix, w, h)
    for got, want in zip(img, planes + [mask.reshape(-1)]):
        assert np.array_equal(got, want)
    assert box == (4, 16, 3, 29)  # rows 4..16, cols 3..29
    rows, cols = np.meshgrid(np.arange(4, 17), np.arange(3, 30), indexing="ij")
    assert np.array_equal(pix, (rows * w + cols).reshape(-1))


def test_missing_files_and_empty_masks_are_errors(tmp_path):
    import cpx

    with pytest.raises(cpx.CpxError):
        cpx.load_image_text(str(tmp_path / "nothing"), 8, 8)
    prefix = str(tmp_path / "blank")
    z = np.zeros(64, np.uint8)
    for name in ("red", "green", "blue", "mask"):
        _write(prefix + "_%s.txt" % name, z, 8, 8)
    with pytest.raises(cpx.CpxError):  # the reference asserts a nonempty rectangle
        cpx.load_image_text(prefix, 8, 8)
    img, box, pix = cpx.load_image_text(prefix, 8, 8, use_mask=False)
    assert pix is None and box == (7, 0, 7, 0)
