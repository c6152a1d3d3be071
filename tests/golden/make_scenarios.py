"""Copies the reference's two scenario files (scenarios/threebody.json, scenarios/test.json of
JacksonCampolattaro/n-body) into this folder as test fixtures, byte for byte, and prints their
SHA-256 so a later copy can be compared.

    python tests/golden/make_scenarios.py <path to the reference checkout>

The files are data in the reference's JSON scenario schema (Simulation.cpp:154-228); the tests
read them from here, so they need no reference checkout at run time.
"""
import hashlib
import os
import shutil
import sys

NAMES = ("threebody.json", "test.json")


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for name in NAMES:
        src = os.path.join(ref_root, "scenarios", name)
        dst = os.path.join(here, name)
        shutil.copyfile(src, dst)
        print(name, hashlib.sha256(open(dst, "rb").read()).hexdigest())


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else ".")
