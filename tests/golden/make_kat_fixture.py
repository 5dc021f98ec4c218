"""Generate tests/golden/kat_test_render.json from the reference's own testRender().

testRender (SparseVolumeRadianceField/VolumeFieldRender.cu:111-183) is the only
hand-written known-answer routine in the reference: a 10-sample compositing and
gradient check with inline inputs that prints its results.  This script reads
the inline inputs out of the reference source, runs the routine as the
reference compiled it (oracle/_ref/ref_kat, built by oracle/Makefile), parses
the printed values and writes both into the fixture.  It needs the reference
tree, so it runs in the build container only; the fixture is committed.
"""
import json
import os
import pathlib
import re
import subprocess
import sys

REPO = pathlib.Path(__file__).resolve().parents[2]
# the reference's source tree (SparseVolumeRadianceField/); CPX_REF_DIR overrides the default
REF_DIR = pathlib.Path(os.environ.get("CPX_REF_DIR", "/root/reference/SparseVolumeRadianceField"))
REF_SRC = REF_DIR / "VolumeFieldRender.cu"
KAT_BIN = REPO / "oracle" / "_ref" / "ref_kat"
OUT = REPO / "tests" / "golden" / "kat_test_render.json"


def _numbers(text):
    return [float(x) for x in re.findall(r"[-+]?\d*\.\d+(?:[eE][-+]?\d+)?|[-+]?\d+\.", text)]


def read_inputs():
    src = REF_SRC.read_text()
    body = src[src.index("void testRender()"):]
    body = body[: body.index("printArray(renderRes")]
    # drop commented-out alternatives before parsing
    body = re.sub(r"//[^\n]*", "", body)
    op = re.search(r"double opacity\[samples\]\s*=\s*\{(.*?)\};", body, re.S).group(1)
    col = re.search(r"double density\[3\]\[samples\]\s*=\s*\{(.*?)\};", body, re.S).group(1)
    gt = re.search(r"double GT\[3\]\s*=\s*\{(.*?)\};", src, re.S).group(1)
    opacity = _numbers(op)
    colour = _numbers(col)
    return opacity, [colour[0:10], colour[10:20], colour[20:30]], _numbers(gt)


def run_reference():
    out = subprocess.run([str(KAT_BIN)], check=True, capture_output=True, text=True).stdout
    blocks = {}
    name = None
    for line in out.splitlines():
        line = line.strip()
        if line.endswith(":"):
            name = line[:-1]
            blocks[name] = []
        elif line and name:
            blocks[name] += [float(v) for v in line.split()]
    return blocks


def main():
    opacity, colour, gt = read_inputs()
    assert len(opacity) == 10 and all(len(c) == 10 for c in colour) and len(gt) == 3
    printed = run_reference()
    fixture = {
        "source": "SparseVolumeRadianceField/VolumeFieldRender.cu:111-183 (testRender), printed with %.6f",
        "opacity": opacity,
        "colour": colour,
        "gt": gt,
        "render_res": printed["RenderRes"],
        "weights": printed["weights"],
        "opacity_grad": printed["OpacityGradient"],
        "colour_grad": [printed["redGradient"], printed["greenGradient"], printed["blueGradient"]],
        "print_resolution": 5e-7,
    }
    OUT.write_text(json.dumps(fixture, indent=1) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    sys.exit(main())
