"""Regenerate tests/golden/*.json from the reference's own test fixtures.

Reads (text only) the camera files under test/inputs/test_Camera and the expected
values under test/solutions/test_Camera of the reference checkout (the argument,
else $OLPT_REFERENCE_DIR, else the tree the oracle Makefile built from), as used by its test_Camera.cpp test_function_2/3/5, and writes
camera_golden.json.  Run: python tests/golden/make_golden.py [reference_root]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.refdir import reference_dir  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else reference_dir()


def numbers(path):
    out = []
    with open(path) as f:
        for line in f:
            out += [float(x) for x in line.replace(",", " ").split()]
    return out


def main():
    inp = os.path.join(REF, "test", "inputs", "test_Camera")
    sol = os.path.join(REF, "test", "solutions", "test_Camera")
    cams = {}
    for name in ["cam1", "cam2", "cam3", "cam4", "cam5", "cam1_poly", "cam2_poly"]:
        with open(os.path.join(inp, name + ".txt")) as f:
            cams[name] = f.read()
    g = {
        "source": "reference test/inputs/test_Camera + test/solutions/test_Camera "
                  "(test_Camera.cpp test_function_2, 3, 5)",
        "cameras": cams,
        # test_function_2: world (1,2,3) -> worldToUndistImg, distort, project for cam1..5
        "f2_world": [1.0, 2.0, 3.0],
        "f2": numbers(os.path.join(sol, "test_function_2.txt")),
        # test_function_3: pixel (461,441) -> undistort, pinholeLine, lineOfSight for cam1..5
        "f3_pixel": [461.0, 441.0],
        "f3": numbers(os.path.join(sol, "test_function_3.txt")),
        # test_function_5: world (1,0,3) -> polyProject, project for cam1_poly, cam2_poly
        "f5_world": [1.0, 0.0, 3.0],
        "f5": numbers(os.path.join(sol, "test_function_5.txt")),
    }
    with open(os.path.join(HERE, "camera_golden.json"), "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", os.path.join(HERE, "camera_golden.json"))


if __name__ == "__main__":
    main()
