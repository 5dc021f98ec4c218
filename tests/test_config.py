"""The reference's positional config.txt (readConfig, Utils.cu:765-932) through cpx_config_read
-- host code, run on the CPU.  A file written here in the reference's key order parses to the
values written; a missing or misordered line is an error that names it; where the reference
tree is present its shipped config_linux.txt parses to the values the reference reads."""
import os
import pathlib

import pytest

KEYS = [
    ("SceneSize", "256 128 64"), ("RenderSize", "800 600"), ("Graylized", "0"), ("SphericalHarmonicsBand", "2"),
    ("HierarchyBandStrategy", "1"), ("SHsForTargetResolutionOnly", "1"), ("Hierarchy", "3"),
    ("MinimumHierarchy", "0"), ("ToSparseHierarchy", "-2"), ("SilhouetteBound", "1"), ("SilhouetteInitial", "5"),
    ("SilhouetteRadius", "8"), ("MaskAreaOnly", "1"), ("InitialFromFile", "0"), ("InitialFileDirBase", "/a/b"),
    ("AvailableSHBands", "3"), ("RenderOnly", "0"), ("ViewDirectory", "/views"), ("CameraPoseFile", "/p/train.txt"),
    ("ValidationPoseFile", "/p/val.txt"), ("NovelViewPoseFile", "/p/test.txt"), ("CameraDistance", "4.031129"),
    ("ViewCount", "100"), ("ValidationCount", "100"), ("TestCount", "200"), ("TrainProcessViewIndex", "-1"),
    ("WhiteBG", "1"), ("TestSkip", "5"), ("RepeatLayers", "5"), ("RandomSeed", "7"), ("LearningRate", "0.3"),
    ("SHLearningRate", "1."), ("DensityOptimizer", "6"), ("ColorChannelOptimizer", "6"), ("Momentum", "0.9"),
    ("Epochs", "6"), ("ValidationInterval", "10000"), ("BatchSize", "8192"), ("FixBatchSize", "0"),
    ("BaseDir", "/out/run"), ("SaveIntervals", "10"), ("HalfLR", "100"), ("LowestLR", "0.00009"),
    ("PruneEpoch", "60"), ("PruneThreshold", "8."), ("Skips", "3"), ("SkipIndex", "4 9 17"), ("StepSize", "0.5"),
    ("SolidStrategy", "0"), ("InitialDensity", "0.1"), ("InitialColor", "0."), ("VarianceLossInterval", "3"),
    ("VarianceCoefficient", "0.00001"), ("ColorDisparityCoefficient", "0.000001"), ("MaskRayCoefficient", "1."),
    ("VarianceType", "0"), ("NeighboorNumsForTVLoss", "6"), ("DiffuseRatio", "0.0"), ("ExportModel", "2"),
    ("ShuffleRays", "1"), ("JustModel", "0"), ("HuberDelta", "0.25"),
]


def _write(path, keys):
    path.write_text("".join("%s:%s\n" % kv for kv in keys))


def test_config_parses_in_the_reference_order(tmp_path):
    import cpx

    p = tmp_path / "config.txt"
    _write(p, KEYS)
    c = cpx.read_config(p)
    assert (c["width"], c["height"], c["depth"]) == (256, 128, 64)
    assert (c["render_width"], c["render_height"]) == (800, 600)
    assert c["sh_band"] == 2 and c["silhouette_initial"] == 1  # a nonzero flag reads as true
    assert c["initial_file_dir_base"] == "/a/b" and c["base_dir"] == "/out/run"
    assert c["camera_distance"] == 4.031129 and c["random_seed"] == 7
    assert c["learning_rate"] == 0.3 and c["sh_learning_rate"] == 1.0 and c["batch_size"] == 8192
    assert c["skips"] == 3 and c["skip_index"] == [4, 9, 17]
    assert c["step_size"] == pytest.approx(0.5) and c["solid_strategy"] == 0
    assert c["variance_coefficient"] == 1e-5 and c["sh_coefficient"] == 1e-6
    assert c["export_model"] == 0  # true only at 1 (Utils.cu:904-906)
    assert c["shuffle_rays"] == 1 and c["huber_delta"] == pytest.approx(0.25)


@pytest.mark.parametrize("drop", ["RandomSeed", "HuberDelta", "SceneSize"])
def test_missing_line_is_named(tmp_path, drop):
    import cpx

    p = tmp_path / "config.txt"
    _write(p, [kv for kv in KEYS if kv[0] != drop])
    with pytest.raises(cpx.CpxError) as ei:
        cpx.read_config(p)
    assert ei.value.name == "CPX_ERR_INVALID_ARGUMENT"
    assert drop in str(ei.value)


def test_misordered_lines_are_an_error(tmp_path):
    import cpx

    keys = list(KEYS)
    keys[3], keys[4] = keys[4], keys[3]
    p = tmp_path / "config.txt"
    _write(p, keys)
    with pytest.raises(cpx.CpxError):
        cpx.read_config(p)
    with pytest.raises(cpx.CpxError):
        cpx.read_config(tmp_path / "absent.txt")


def test_reference_shipped_config():
    import cpx

    ref = pathlib.Path(os.environ.get("CPX_REF_DIR", "/root/reference/SparseVolumeRadianceField")) / \
        "config_linux.txt"
    if not ref.exists():
        pytest.skip("the reference tree is not present")
    c = cpx.read_config(ref)
    assert (c["width"], c["height"], c["depth"]) == (512, 512, 512)
    assert c["learning_rate"] == 0.3 and c["sh_learning_rate"] == 1.0
    assert c["variance_coefficient"] == 1e-5 and c["sh_coefficient"] == 1e-6 and c["mask_ray_coefficient"] == 1.0
    assert c["step_size"] == 0.5 and c["solid_strategy"] == 1 and c["huber_delta"] == pytest.approx(0.1)
    assert c["skips"] == 0 and c["neighbour_nums"] == 6
