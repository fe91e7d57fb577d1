"""Extract golden counts from the reference's own test-farm outputs.

Reads ``test/test_farm/<case>/ref/{INFO.OUT,KPOINTS.OUT}`` of the exciting
source tree (its path is the required argument) and writes
``reference_counts.json`` beside this script: per case the lattice, the muffin
tin radii, the atomic positions, rgkmax, gmaxvr, the FFT box (``G-vector grid
sizes``), the number of G-vectors, the unit-cell volume, the number of local
orbitals and, per k-point, vkl and nmat (KPOINTS.OUT).

These pin the host-side G-vector and G+k construction (gridsize, gengvec,
gengpvec, nmat = ngk + nlotot) against numbers printed by the reference.
Run once in a tree where the reference is present; the JSON is committed.
"""
from __future__ import annotations

import json
import os
import re
import sys
from fractions import Fraction

CASES = [
    "groundstate-GGA_PBE-properties-Si",
    "groundstate-LDA_PW-properties_ldos-Si",
    "groundstate-LDA_PW-gw-Si",
    "groundstate-GGA_PBE-BSE-LiF",
    "groundstate-LDA_PW-PbTiO3",
    "groundstate-GGA_PBE-electronic_structure-Al",
    "groundstate-GGA_PBE-lin-Al",
    "groundstate-GGA_PBE-Ar",
    "groundstate-GGA_PBE-He",
    "groundstate-LDA_PZ-wannier-SiC",
    "groundstate-HYB_PBE0-Si",
]


def _num(s):
    return float(s.replace("D", "E"))


def _rationalise(x):
    """Printed k-coordinates (10 digits) back to the exact fraction they print."""
    f = Fraction(x).limit_denominator(96)
    return float(f) if abs(float(f) - x) < 1e-9 else x


def parse_info(path):
    text = open(path).read()
    init = text.split("Ending initialization")[0]
    lines = init.splitlines()
    out = {}
    for i, ln in enumerate(lines):
        if ln.strip().startswith("Lattice vectors (cartesian)"):
            rows = [[_num(v) for v in lines[i + k].split()] for k in (1, 2, 3)]
            out["avec_rows"] = rows          # row j = lattice vector j
    out["omega"] = _num(re.search(r"Unit cell volume\s*:\s*(\S+)", init).group(1))
    species = []
    blocks = re.split(r"\n Species :", init)[1:]
    for b in blocks:
        rmt = _num(re.search(r"muffin-tin radius\s*:\s*(\S+)", b).group(1))
        atoms = []
        m = re.search(r"atomic positions \(lattice\) :\n((?:\s+\d+ :.*\n)+)", b)
        for ln in m.group(1).strip("\n").splitlines():
            atoms.append([_num(v) for v in ln.split(":")[1].split()[:3]])
        species.append({"rmt": rmt, "atoms": atoms})
    out["species"] = species
    out["spin"] = re.search(r"Spin treatment\s*:\s*(.+)", init).group(1).strip()
    out["rgkmax"] = _num(re.search(r"\(rgkmax\)\s*:\s*(\S+)", init).group(1))
    out["gkmax"] = _num(re.search(r"Maximum \|G\+k\| for APW functions\s*:\s*(\S+)", init).group(1))
    out["gmaxvr"] = _num(re.search(r"Maximum \|G\| for potential and density\s*:\s*(\S+)", init).group(1))
    out["ngrid"] = [int(v) for v in re.search(r"G-vector grid sizes\s*:\s*(\d+)\s+(\d+)\s+(\d+)", init).groups()]
    out["ngvec"] = int(re.search(r"Total number of G-vectors\s*:\s*(\d+)", init).group(1))
    out["nlotot"] = int(re.search(r"Total number of local-orbitals\s*:\s*(\d+)", init).group(1))
    out["nmatmax"] = int(re.search(r"Maximum Hamiltonian size\s*:\s*(\d+)", init).group(1))
    out["ngkmax"] = int(re.search(r"Maximum number of plane-waves\s*:\s*(\d+)", init).group(1))
    return out


def parse_kpoints(path):
    lines = open(path).read().splitlines()
    n = int(lines[0].split(":")[0])
    kp = []
    for ln in lines[1:1 + n]:
        v = ln.split()
        kp.append({"vkl": [_rationalise(_num(x)) for x in v[1:4]], "nmat": int(v[-1])})
    return kp


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <exciting source tree>")
    root = sys.argv[1]
    farm = os.path.join(root, "test", "test_farm")
    out = {}
    for case in CASES:
        ref = os.path.join(farm, case, "ref")
        info = parse_info(os.path.join(ref, "INFO.OUT"))
        if info["spin"] != "spin-unpolarised":
            continue
        info["kpoints"] = parse_kpoints(os.path.join(ref, "KPOINTS.OUT"))
        info["source"] = f"test/test_farm/{case}/ref/INFO.OUT, KPOINTS.OUT"
        out[case] = info
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_counts.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}: {len(out)} cases")


if __name__ == "__main__":
    main()
