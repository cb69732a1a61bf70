"""Generates tests/golden/interpolants.json: values and d/ds of the reference's tricubic and triquintic cell
polynomials at seeded random corner data and local coordinates.

The reference evaluates InterpolationEnergyGrid::interpolate through computeCoefficients(X, a), an unrolled map from
the corner data X to the monomial coefficients a (interpolation_energy_grid.cpp:193-358 for 64 values, :2116-3500
for 216), then sums a[i + n*j + n*n*k] s_x^i s_y^j s_z^k (n = 4 or 6). This script reads those two functions from the
reference source as text, applies them to the random inputs and stores only inputs and outputs; it needs the RASPA3
source tree (argument or RASPA3_SRC) and runs here, not in the tests.

    python tests/golden/make_interpolant_fixtures.py /path/to/RASPA3
"""

import json
import os
import re
import sys

import numpy as np

SEED = 20240521
CASES = 12


def coefficient_maps(path):
    src = open(path).read()
    maps = {}
    for n, size in ((64, 4), (216, 6)):
        head = re.search(r"computeCoefficients\(const std::array<double, %d>& X,\s*std::array<double, %d>& a\)\s*\{"
                         % (n, n), src)
        body = src[head.end():src.index("return", head.end())]
        rows = {}
        for stmt in body.split(";"):
            m = re.match(r"\s*a\[(\d+)\]\s*=\s*(.*)", stmt, re.S)
            if not m:
                continue
            expr = re.sub(r"\s+", "", m.group(2)).replace("+-", "-").replace("--", "+")
            terms = re.findall(r"([+-]?)((?:\d+(?:\.\d*)?(?:e[+-]?\d+)?)\*)?X\[(\d+)\]", expr)
            consumed = "".join(s + (c or "") + "X[" + j + "]" for s, c, j in terms)
            assert consumed == expr.lstrip("+"), (m.group(1), expr[:80])
            row = {}
            for sign, coef, j in terms:
                v = float(coef[:-1]) if coef else 1.0
                row[int(j)] = row.get(int(j), 0.0) + (-v if sign == "-" else v)
            rows[int(m.group(1))] = row
        assert sorted(rows) == list(range(n)), n
        maps[n] = (size, rows)
    return maps


def evaluate(size, rows, X, s):
    a = np.array([sum(c * X[j] for j, c in rows[r].items()) for r in range(size ** 3)])
    v, ds = 0.0, np.zeros(3)
    for k in range(size):
        for j in range(size):
            for i in range(size):
                c = a[i + size * j + size * size * k]
                v += c * s[0] ** i * s[1] ** j * s[2] ** k
                if i:
                    ds[0] += i * c * s[0] ** (i - 1) * s[1] ** j * s[2] ** k
                if j:
                    ds[1] += j * c * s[0] ** i * s[1] ** (j - 1) * s[2] ** k
                if k:
                    ds[2] += k * c * s[0] ** i * s[1] ** j * s[2] ** (k - 1)
    return v, ds


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RASPA3_SRC", "")
    path = os.path.join(root, "src", "raspakit", "interpolation_energy_grid.cpp")
    maps = coefficient_maps(path)
    rng = np.random.default_rng(SEED)
    out = {"seed": SEED, "source": "src/raspakit/interpolation_energy_grid.cpp computeCoefficients", "cases": {}}
    for n, (size, rows) in maps.items():
        cases = []
        for _ in range(CASES):
            X = rng.normal(size=n)
            s = rng.random(3)
            v, ds = evaluate(size, rows, X, s)
            cases.append({"X": X.tolist(), "s": s.tolist(), "value": v, "ds": ds.tolist()})
        out["cases"][str(n // 8)] = cases
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "interpolants.json")
    with open(dst, "w") as f:
        json.dump(out, f)
    print("wrote", dst)


if __name__ == "__main__":
    main()
