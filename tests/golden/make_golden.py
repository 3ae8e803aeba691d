"""Regenerates the golden fixtures in this folder from the reference checkout.

shot_1.bin is the one known-answer artefact the reference ships (its
run.jl synthetic single shot, 800 x 100 Float32 vz gather, column-major).
It is copied verbatim; runjl_case.json records the run.jl recipe
(run.jl:36-61, 90-131) that produced it, so the tests can rebuild the inputs
without the reference being present.

Usage:  python tests/golden/make_golden.py /path/to/reference-checkout
"""
import hashlib
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "shot_1.bin")
    dst = os.path.join(HERE, "shot_1.bin")
    shutil.copyfile(src, dst)
    digest = hashlib.sha256(open(dst, "rb").read()).hexdigest()
    recipe = {
        "source": "run.jl main_synthetic() + run_simulation() of Wuheng10086/Fomo_julia",
        "nx": 400, "nz": 200, "dx": 10.0, "dz": 10.0,
        "vp": 3000.0, "vs": 1800.0, "rho": 2200.0,
        "layer_from_row": 100, "vp_layer": 4000.0, "vs_layer": 2400.0,
        "nbc": 50, "fd_order": 8, "free_surface": True,
        "f0": 15.0, "total_time": 1.0, "cfl": 0.5,
        "rec_x_start": 500, "rec_x_stop": 3500, "n_rec": 100, "rec_z": 100.0,
        "src_z": 50.0, "rec_type": "vz",
        "gather_shape": [800, 100], "gather_layout": "column-major [nt x n_rec], little-endian Float32",
        "sha256": digest,
    }
    with open(os.path.join(HERE, "runjl_case.json"), "w") as f:
        json.dump(recipe, f, indent=1)
    print("wrote", dst, digest)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference-checkout")
    main(sys.argv[1])
