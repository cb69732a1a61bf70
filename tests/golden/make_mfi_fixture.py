"""Generates tests/golden/mfi_framework.json: the MFI framework of the reference's known-answer tests.

Framework::makeMFI (src/raspakit/framework.cpp:1591-1660) lists the asymmetric unit of MFI (12 Si, 26 O, fractional
coordinates and charges), the cell lengths and the space group (Hall number 292, P n m a). This script reads those from
the reference source as text and stores them as data; the expansion to the unit cell is done by the tests
(reference_systems.mfi). It needs the RASPA3 source tree (argument or RASPA3_SRC) and runs here, not in the tests.

    python tests/golden/make_mfi_fixture.py /path/to/RASPA3
"""

import json
import os
import re
import sys


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RASPA3_SRC", "")
    src = open(os.path.join(root, "src", "raspakit", "framework.cpp")).read()
    body = src[src.index("Framework Framework::makeMFI"):src.index("Framework Framework::makeCHA")]
    hall = int(re.search(r"space_group_hall_number\s*=\s*(\d+)", body).group(1))
    cell = [float(v) for v in re.search(r"SimulationBox\(([\d.]+),\s*([\d.]+),\s*([\d.]+)\)", body).groups()]
    atoms = []
    for m in re.finditer(r"Atom\(double3\(([-\d.]+),\s*([-\d.]+),\s*([-\d.]+)\),\s*([-\d.]+),.*?type_(si|o)\.value",
                         body, re.S):
        x, y, z, q, t = m.groups()
        atoms.append([float(x), float(y), float(z), float(q), "Si" if t == "si" else "O"])
    out = {"source": "src/raspakit/framework.cpp:1591-1660 (Framework::makeMFI)", "hall_number": hall,
           "cell_lengths": cell, "asymmetric_atoms": atoms}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mfi_framework.json")
    json.dump(out, open(path, "w"), indent=1)
    print(path, len(atoms), "atoms")


if __name__ == "__main__":
    main()
