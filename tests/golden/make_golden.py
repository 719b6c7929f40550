"""Regenerate the golden fixtures in this directory from the reference's own
golden generator (tests/fixtures/gen_golden_isp_nodes.cpp in the reference tree).

The reference ships its goldens as git-LFS pointers, so the pixel data is not in
the tree; the generator source is.  `make -C oracle ref` compiles that source
unmodified (against stand-in OIIO/OCIO headers that write raw float files) into
oracle/_ref/gen_golden.  This script runs it and packs each in-scope node's
input/output pair into `<fixture>.npz` (float32 arrays, HxW or HxWx4), plus the
17^3 LUT values of the color.3d_lut fixture.

Run in an environment that has the reference tree:  python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

FIXTURES = [
    "linearize.dng_lut", "blacklevel.dng_levels", "lens.shading_gainmap", "demosaic.bilinear",
    "demosaic.rcd", "demosaic.amaze", "demosaic.quad_bayer_remosaic", "lens.dng_opcode_list_3",
    "wb.dual_illuminant", "colormatrix.dng_to_working", "denoise.bm3d", "denoise.guided_filter",
    "denoise.wavelet_bayes_shrink", "tone.filmic_rgb", "color.3d_lut", "sharpen.edge_aware_usm",
    "tone.aces_filmic", "tone.reinhard", "wb.greyworld_auto", "tone.mertens_local",
]


def read_raw(path):
    with open(path, "rb") as f:
        data = f.read()
    assert data[:4] == b"CPF1", path
    w, h, c = np.frombuffer(data[4:16], dtype=np.int32)
    px = np.frombuffer(data[16:], dtype=np.float32).copy()
    return px.reshape(h, w, c) if c > 1 else px.reshape(h, w)


def read_cube(path):
    vals = []
    size = None
    for line in open(path):
        parts = line.split()
        if not parts or parts[0] in ("TITLE", "DOMAIN_MIN", "DOMAIN_MAX"):
            continue
        if parts[0] == "LUT_3D_SIZE":
            size = int(parts[1])
            continue
        vals.extend(float(p) for p in parts[:3])
    return size, np.asarray(vals, dtype=np.float32)


def main():
    gen = os.path.join(ROOT, "oracle", "_ref", "gen_golden")
    if not os.path.exists(gen):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    with tempfile.TemporaryDirectory() as tmp:
        out_root = os.path.join(tmp, "tests", "golden")
        subprocess.check_call([gen, out_root])
        for name in FIXTURES:
            d = os.path.join(out_root, name)
            if name == "tone.mertens_local":  # an exposure stack: under / normal / over in
                arrays = {k: read_raw(os.path.join(d, k + ".exr")) for k in ("under", "normal", "over")}
                arrays["output"] = read_raw(os.path.join(d, "out.exr"))
                np.savez(os.path.join(HERE, name + ".npz"), **arrays)
                print("wrote", name, arrays["normal"].shape, arrays["output"].shape)
                continue
            arrays = {"input": read_raw(os.path.join(d, "in.exr")),
                      "output": read_raw(os.path.join(d, "out.exr"))}
            if name == "color.3d_lut":
                size, vals = read_cube(os.path.join(d, "look.cube"))
                arrays["lut_size"] = np.int32(size)
                arrays["lut"] = vals
            np.savez(os.path.join(HERE, name + ".npz"), **arrays)
            print("wrote", name, arrays["input"].shape, arrays["output"].shape)
    return 0


if __name__ == "__main__":
    sys.exit(main())
