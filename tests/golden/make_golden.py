"""Generate tests/golden/known_answers.json from the reference's own tests.

The reference (Tesserae.jl) is Julia and cannot run here, so its known answers
are taken from the literal expectations in its test files and doctests. For each
case this script checks that the cited reference line still says what the case
records (provenance), then writes the case. Run from the repository root:

    python tests/golden/make_golden.py path/to/Tesserae.jl

The JSON is committed; tests read only the JSON.
"""
from __future__ import annotations

import json
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent


def line(ref: pathlib.Path, rel: str, lineno: int) -> str:
    return (ref / rel).read_text().splitlines()[lineno - 1]


def require(ref, rel, lineno, *needles):
    text = line(ref, rel, lineno)
    for n in needles:
        if n not in text:
            raise SystemExit(f"{rel}:{lineno} no longer contains {n!r}: {text!r}")
    return f"{rel}:{lineno}"


def main(ref_root: str):
    ref = pathlib.Path(ref_root)
    cases = []

    # 1-D jets (test/basis.jl:311-312)
    cases.append({"kind": "jet_bspline_quadratic", "xi": 0.0, "value": 0.75, "deriv": 0.0,
                  "source": require(ref, "test/basis.jl", 311, "jet(Order(1), BSpline(Quadratic()), 0) == (0.75, 0.0)")})
    cases.append({"kind": "jet_ugimp", "xi": 0.0, "l": 1.0, "value": 0.75, "deriv": 0.0,
                  "source": require(ref, "test/basis.jl", 312, "jet(Order(1), gimp, 0, 1) == (0.75, 0.0)")})

    # uGIMP support sizes at l = h/2 on CartesianMesh(0.1, (0,1)) (test/basis.jl:337-339)
    require(ref, "test/basis.jl", 337, "l = 0.5spacing(mesh)")
    cases.append({"kind": "ugimp_support_size", "h": 0.1, "lims": [0.0, 1.0], "x": 0.40, "l": 0.05, "size": 3,
                  "source": require(ref, "test/basis.jl", 338, "x=Vec(0.40)", "== (3,)")})
    cases.append({"kind": "ugimp_support_size", "h": 0.1, "lims": [0.0, 1.0], "x": 0.44, "l": 0.05, "size": 2,
                  "source": require(ref, "test/basis.jl", 339, "x=Vec(0.44)", "== (2,)")})

    # Doctests of src/Mesh/cartesian.jl
    cases.append({"kind": "mesh_size", "h": 1.0, "lims": [[0, 3], [1, 4]], "size": [4, 4],
                  "source": require(ref, "src/Mesh/cartesian.jl", 31, "4×4 CartesianMesh")})
    cases.append({"kind": "supportnodes_radius", "h": 1.0, "lims": [[0, 5]], "x": [1.5], "r": 1, "range": [[2, 3]],
                  "source": require(ref, "src/Mesh/cartesian.jl", 184, "CartesianIndices((2:3,))")})
    cases.append({"kind": "supportnodes_radius", "h": 1.0, "lims": [[0, 5]], "x": [1.5], "r": 3, "range": [[1, 5]],
                  "source": require(ref, "src/Mesh/cartesian.jl", 187, "CartesianIndices((1:5,))")})
    cases.append({"kind": "findcell", "h": 1.0, "lims": [[0, 5], [0, 5]], "x": [1.5, 1.5], "cell": [2, 2],
                  "source": require(ref, "src/Mesh/cartesian.jl", 219, "CartesianIndex(2, 2)")})
    cases.append({"kind": "findblock", "h": 1.0, "lims": [[0, 10], [0, 10]], "x": [8.5, 1.5], "block": [3, 1],
                  "block_size_log2": 2,
                  "source": require(ref, "src/Mesh/cartesian.jl", 268, "CartesianIndex(3, 1)")})

    # Partition of unity / linear-field reproduction / truncation flags
    # (test/basis.jl:226-300, 309-346, 415-437). interior_point = 0.45 + 0.01 i,
    # boundary_point puts axis 1 at 0.02; meshes CartesianMesh(0.1, (0,1)^dim).
    require(ref, "test/basis.jl", 228, "0.45 + 0.01i")
    require(ref, "test/basis.jl", 229, "0.02")
    src_quad = require(ref, "test/basis.jl", 255, "BSpline(Quadratic())")
    src_quad_b = require(ref, "test/basis.jl", 266, "partition=false, reproduces_linear=false, truncated=true")
    src_gimp_i = require(ref, "test/basis.jl", 318, "partition=true, reproduces_linear=true")
    src_gimp_b = require(ref, "test/basis.jl", 320, "partition=false, reproduces_linear=false, truncated=true")
    src_gimp_full = require(ref, "test/basis.jl", 328, "partition=true, reproduces_linear=true")
    src_wls_i = require(ref, "test/basis.jl", 422, "partition=true, reproduces_linear=true, truncated=false")
    src_wls_b = require(ref, "test/basis.jl", 432, "partition=true, reproduces_linear=true, truncated=true")
    src_wls_g = require(ref, "test/basis.jl", 435, "partition=true, reproduces_linear=true, truncated=true")
    for dim in (2, 3):
        interior = [0.45 + 0.01 * (i + 1) for i in range(dim)]
        boundary = [0.02] + interior[1:]
        h = 0.1
        cases.append({"kind": "basis_props", "basis": "bspline_quadratic", "dim": dim, "h": h, "x": interior,
                      "l": 0.0, "pu": True, "lfr": True, "truncated": False, "source": src_quad})
        cases.append({"kind": "basis_props", "basis": "bspline_quadratic", "dim": dim, "h": h, "x": boundary,
                      "l": 0.0, "pu": False, "lfr": False, "truncated": True, "source": src_quad_b})
        cases.append({"kind": "basis_props", "basis": "ugimp", "dim": dim, "h": h, "x": interior,
                      "l": 0.5 * h, "pu": True, "lfr": True, "truncated": None, "source": src_gimp_i})
        cases.append({"kind": "basis_props", "basis": "ugimp", "dim": dim, "h": h, "x": boundary,
                      "l": 0.5 * h, "pu": False, "lfr": False, "truncated": True, "source": src_gimp_b})
        cases.append({"kind": "basis_props", "basis": "ugimp", "dim": dim, "h": h, "x": [0.44] * dim,
                      "l": h, "pu": True, "lfr": True, "truncated": None, "source": src_gimp_full})
        cases.append({"kind": "basis_props", "basis": "wls_bspline_quadratic", "dim": dim, "h": h, "x": interior,
                      "l": 0.0, "pu": True, "lfr": True, "truncated": False, "source": src_wls_i})
        cases.append({"kind": "basis_props", "basis": "wls_bspline_quadratic", "dim": dim, "h": h, "x": boundary,
                      "l": 0.0, "pu": True, "lfr": True, "truncated": True, "source": src_wls_b})
        cases.append({"kind": "basis_props", "basis": "wls_ugimp", "dim": dim, "h": h, "x": boundary,
                      "l": 0.5 * h / 2, "pu": True, "lfr": True, "truncated": True, "source": src_wls_g})

    # KernelCorrection restores both properties at the boundary (test/basis.jl:449-465)
    src_kc_i = require(ref, "test/basis.jl", 456, "partition=true, reproduces_linear=true, truncated=false")
    src_kc_b = require(ref, "test/basis.jl", 460, "partition=true, reproduces_linear=true, truncated=true")
    src_kc_g = require(ref, "test/basis.jl", 463, "partition=true, reproduces_linear=true, truncated=true")
    require(ref, "test/basis.jl", 455, "KernelCorrection(BSpline(Quadratic()))")
    require(ref, "test/basis.jl", 462, "KernelCorrection(uGIMP())")
    for dim in (2, 3):
        interior = [0.45 + 0.01 * (i + 1) for i in range(dim)]
        boundary = [0.02] + interior[1:]
        h = 0.1
        cases.append({"kind": "basis_props", "basis": "kc_bspline_quadratic", "dim": dim, "h": h, "x": interior,
                      "l": 0.0, "pu": True, "lfr": True, "truncated": False, "source": src_kc_i})
        cases.append({"kind": "basis_props", "basis": "kc_bspline_quadratic", "dim": dim, "h": h, "x": boundary,
                      "l": 0.0, "pu": True, "lfr": True, "truncated": True, "source": src_kc_b})
        cases.append({"kind": "basis_props", "basis": "kc_ugimp", "dim": dim, "h": h, "x": boundary,
                      "l": 0.5 * h / 2, "pu": True, "lfr": True, "truncated": True, "source": src_kc_g})

    # Positivity of KernelCorrection(BSpline(Quadratic()), MultiLinear) near the
    # boundary (test/basis.jl:566-614): the node's weight is > -sqrt(eps) for
    # particles on a 1/11 lattice over [max(x0, I - L - 1), min(x1, I + L - 1) - sqrt(eps)]
    # per axis (L = 1.5, 1-based node index I, unit spacing).
    require(ref, "test/basis.jl", 574, "step=1/11")
    require(ref, "test/basis.jl", 572, "BSpline{Quadratic} ? 1.5")
    for dim, node, lims, line_no in ((2, [2, 2], [[0, 10], [0, 10]], 596), (3, [2, 2, 1], [[0, 10]] * 3, 608)):
        cases.append({"kind": "kc_positive", "dim": dim, "h": 1.0, "lims": lims, "nodes": [node], "L": 1.5,
                      "source": require(ref, "test/basis.jl", line_no, "multilin, CartesianIndex(")})
    for dim, line_no in ((2, 601), (3, 613)):
        src = require(ref, "test/basis.jl", line_no, "all(i -> is_positive_everywhere(domain, kern, multilin, i)")
        for I in (([1, 1], [3, 2]) if dim == 2 else ([1, 1, 1], [3, 2, 1])):
            nodes = [list(t) for t in __import__("itertools").product(*[range(1, k + 1) for k in I])]
            cases.append({"kind": "kc_positive", "dim": dim, "h": 1.0, "lims": [[0, k] for k in I], "nodes": nodes,
                          "L": 1.5, "source": src})

    # generate_particles doctest (src/particles.jl:79-89): GridSampling() on
    # CartesianMesh(0.5, (0,3), (0,2)) gives 96 particles, the first at (0.125, 0.125)
    require(ref, "src/particles.jl", 79, "CartesianMesh(0.5, (0,3), (0,2))")
    require(ref, "src/particles.jl", 81, "alg=GridSampling()")
    require(ref, "src/particles.jl", 86, "(x = [0.125, 0.125]")
    cases.append({"kind": "grid_sampling", "h": 0.5, "lims": [[0, 3], [0, 2]], "spacing": 0.5, "n": 96,
                  "first": [0.125, 0.125], "source": require(ref, "src/particles.jl", 89, "96-element")})

    # Block-tile containment for 2D meshes of h = 0.02 (test/transfer.jl:941-957)
    cases.append({"kind": "tile_contains", "h": 0.02, "lims": [[0, 1], [0, 1]], "l": 0.01,
                  "bases": ["bspline_quadratic", "ugimp", "wls_bspline_quadratic"],
                  "source": require(ref, "test/transfer.jl", 942, "BSpline(Constant())")})

    # Partition lists equal findblock lists in ascending particle order (test/partition.jl:80-93)
    cases.append({"kind": "partition_lists", "source": require(ref, "test/partition.jl", 91, "actual == expected")})

    out = {"reference": "KeitaNakamura/Tesserae.jl", "generator": "tests/golden/make_golden.py", "cases": cases}
    (HERE / "known_answers.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {len(cases)} cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py path/to/Tesserae.jl")
    main(sys.argv[1])
