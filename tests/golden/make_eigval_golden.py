"""Collect the reference's own EIGVAL.OUT files as text fixtures.

Reads ``test/test_farm/<case>/ref/EIGVAL.OUT`` of the exciting source tree
(its path is the required argument) and writes
``eigval_fixtures.json`` beside this script: {case: file text} for every
case whose file is at most 20 kB.  They pin the EIGVAL.OUT writer
(exciting_b200.fileio.write_eigval, the I6 / G18.10 layout of
src/writeeval.f90) byte for byte.  Run once where the reference is present;
the JSON is committed.
"""
from __future__ import annotations

import glob
import json
import os
import sys


def main(root):
    out = {}
    for path in sorted(glob.glob(os.path.join(root, "test", "test_farm", "*", "ref", "EIGVAL.OUT"))):
        if os.path.getsize(path) <= 20000:
            case = os.path.basename(os.path.dirname(os.path.dirname(path)))
            out[case] = open(path).read()
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "eigval_fixtures.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print(f"{len(out)} cases -> {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_eigval_golden.py <exciting source tree>")
    main(sys.argv[1])
