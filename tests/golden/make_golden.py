"""Extract the bempp-cl golden matrices that pin bempp-rs's boundary assembly.

Source: tests/compare_to_bempp_cl.rs of bempp-rs (the eight active tests at lines
19-206).  Every test assembles on ``regular_sphere(0)`` (the unit octahedron, 8 cells,
6 vertices) with default options (37-point regular rule, order-4 Duffy rules) and
compares entry (i, j) of bempp-rs's matrix with ``from_cl[perm[i]][perm[j]]`` (perm is
the identity for DP0) within an absolute ``epsilon``.

Give the root of a bempp-rs checkout as the one argument:

    python tests/golden/make_golden.py <path to bempp-rs>

It writes tests/golden/bempp_cl_octahedron.json and, from the four potential-operator
tests that the file keeps commented out (lines 208-320: single and double layer
potentials of the Laplace and the k = 3 Helmholtz kernel, DP0, at the points (2, 0, 0),
(0, 2, 0), (0, 0, 2)), tests/golden/bempp_cl_octahedron_potentials.json.  The fixtures
are committed; the tests never read the reference tree.
"""

from __future__ import annotations

import json
import os
import re
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bempp_cl_octahedron.json")
OUT_POT = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "bempp_cl_octahedron_potentials.json")

# commented test name -> (kernel, operator)
POTENTIAL_TESTS = {
    "test_laplace_single_layer_potential_dp0": ("laplace", "single_layer"),
    "test_helmholtz_single_layer_potential_dp0": ("helmholtz", "single_layer"),
    "test_laplace_double_layer_potential_dp0": ("laplace", "double_layer"),
    "test_helmholtz_double_layer_potential_dp0": ("helmholtz", "double_layer"),
}

# test name -> (kernel, operator, space degree, continuous)
TESTS = {
    "test_laplace_single_layer_dp0_dp0": ("laplace", "single_layer", 0, False),
    "test_laplace_double_layer_dp0_dp0": ("laplace", "double_layer", 0, False),
    "test_laplace_adjoint_double_layer_dp0_dp0": ("laplace", "adjoint_double_layer", 0, False),
    "test_laplace_hypersingular_p1_p1": ("laplace", "hypersingular", 1, True),
    "test_helmholtz_single_layer_dp0_dp0": ("helmholtz", "single_layer", 0, False),
    "test_helmholtz_double_layer_dp0_dp0": ("helmholtz", "double_layer", 0, False),
    "test_helmholtz_adjoint_double_layer_dp0_dp0": ("helmholtz", "adjoint_double_layer", 0, False),
    "test_helmholtz_hypersingular_p1_p1": ("helmholtz", "hypersingular", 1, True),
}


def parse_matrix(text: str):
    text = text.strip()
    assert text.startswith("[[") and text.endswith("]]"), text[:40]
    rows = []
    for row in re.findall(r"\[([^\[\]]*)\]", text[1:-1]):
        if "c64::new" in row:
            vals = re.findall(r"c64::new\(\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*\)", row)
            rows.append([[float(a), float(b)] for a, b in vals])
        else:
            rows.append([float(v) for v in row.split(",") if v.strip()])
    return rows


def main(reference: str):
    src = open(os.path.join(reference, "tests", "compare_to_bempp_cl.rs")).read()
    # only the active (non-commented) tests
    active = "\n".join(line for line in src.splitlines() if not line.lstrip().startswith("//"))
    out = {"source": "bempp-rs tests/compare_to_bempp_cl.rs", "cases": []}
    for m in re.finditer(r"fn (test_\w+)\(\)\s*\{(.*?)\n\}", active, re.S):
        name, body = m.group(1), m.group(2)
        if name not in TESTS:
            continue
        kernel, op, degree, cont = TESTS[name]
        mat = parse_matrix(re.search(r"let from_cl = (\[\[.*?\]\]);", body, re.S).group(1))
        eps = float(re.search(r"epsilon = ([0-9.eE-]+)", body).group(1))
        perm_m = re.search(r"let perm = \[([0-9, ]+)\];", body)
        perm = [int(x) for x in perm_m.group(1).split(",")] if perm_m else list(range(len(mat)))
        k_m = re.search(r"helmholtz::assembler::\w+\(([0-9.]+),", body)
        line = src[: src.index("fn " + name + "()")].count("\n") + 1
        out["cases"].append(
            {
                "name": name,
                "line": line,
                "kernel": kernel,
                "operator": op,
                "degree": degree,
                "continuous": cont,
                "wavenumber": float(k_m.group(1)) if k_m else None,
                "epsilon": eps,
                "perm": perm,
                "matrix": mat,
            }
        )
    assert len(out["cases"]) == len(TESTS), [c["name"] for c in out["cases"]]
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out['cases'])} cases to {OUT}")
    potentials(src)


def potentials(src: str):
    """The commented potential tests: from_cl[dof][point], compared with matrix[point, dof]."""
    lines = src.splitlines()
    out = {"source": "bempp-rs tests/compare_to_bempp_cl.rs (commented tests)", "cases": []}
    for i, line in enumerate(lines):
        m = re.match(r"\s*//\s*fn (test_\w+_potential_dp0)\(\)", line)
        if not m or m.group(1) not in POTENTIAL_TESTS:
            continue
        body = []
        for line2 in lines[i + 1:]:
            t = re.sub(r"^\s*//\s?", "", line2)
            if t.startswith("}"):
                break
            body.append(t)
        body = "\n".join(body)
        kernel, op = POTENTIAL_TESTS[m.group(1)]
        mat = parse_matrix(re.search(r"let from_cl = (\[\[.*?\]\]);", body, re.S).group(1))
        eps = float(re.search(r"epsilon = ([0-9.eE-]+)", body).group(1))
        k_m = re.search(r"helmholtz::assembler::\w+\(([0-9.]+)\)", body)
        pts = [[0.0] * 3 for _ in range(3)]
        for a, b, v in re.findall(r"points\.get_mut\(\[(\d), (\d)\]\)\.unwrap\(\) = ([0-9.]+);", body):
            pts[int(b)][int(a)] = float(v)  # column b of the 3 x npoints array is point b
        out["cases"].append({"name": m.group(1), "line": i + 1, "kernel": kernel, "operator": op,
                             "wavenumber": float(k_m.group(1)) if k_m else None,
                             "epsilon": eps, "points": pts, "matrix": mat})
    assert len(out["cases"]) == len(POTENTIAL_TESTS), [c["name"] for c in out["cases"]]
    with open(OUT_POT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out['cases'])} cases to {OUT_POT}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to a bempp-rs checkout>")
    sys.exit(main(sys.argv[1]))
