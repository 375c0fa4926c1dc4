"""Extracts the known answers of EtherParallelParticles.jl's own tests into reference_kat.json.

The reference is Julia and cannot run here, so its known-answer tests are read as text: every
value below is parsed out of the cited test file, and the script fails if a file no longer
contains the expression it expects.  Run it with the path of a checkout of the reference:

    python tests/golden/make_golden.py <path to EtherParallelParticles.jl>

The generated JSON is committed; the tests read only the JSON.
"""
import json
import os
import re
import sys

import numpy as np


def _read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def _line_of(text, needle):
    for k, line in enumerate(text.splitlines(), 1):
        if needle in line:
            return k
    raise SystemExit("expected text not found: %r" % needle)


def _ints(s):
    return [int(v) for v in re.findall(r"-?\d+", s)]


def neighbour_search(root):
    rel = "test/Algorithm/NeighbourSearchTest.jl"
    t = _read(root, rel)
    m = re.search(r"Domain2D\{IT, FT\}\(([^)]*)\)", t)
    dom = [float(v) for v in m.group(1).split(",")]
    pairs = re.search(r"active_pair = \[([^\]]*)\]", t).group(1)
    active = [tuple(_ints(p)) for p in pairs.split(",")]
    err = float(re.search(r"err = ([0-9.e-]+)", t).group(1))
    # The nine positions, NeighbourSearchTest.jl:49-59.  Julia evaluates them with start/gap in
    # Float32 and err in Float64; the Float64 intermediate is rounded when stored in zeros(FT, 9, 2).
    expr = [
        ("start_x + err", "start_y + err"),
        ("start_x + gap / 2", "start_y + err"),
        ("start_x + gap * 3 / 2 - err", "start_y + err"),
        ("start_x + err", "start_y + gap / 2"),
        ("start_x + gap / 2", "start_y + gap / 2"),
        ("start_x + gap * 3 / 2 - err", "start_y + gap / 2"),
        ("start_x + err", "start_y + gap - err"),
        ("start_x + gap / 2", "start_y + gap - err"),
        ("start_x + gap * 3 / 2 - err", "start_y + gap - err"),
    ]
    for k, (ex, ey) in enumerate(expr, 1):
        needle = "xy[%d, :] .= [%s, %s]" % (k, ex, ey)
        _line_of(t, needle)
    f32 = np.float32
    gap = f32(dom[0])
    sx, sy = f32(dom[1]), f32(dom[2])

    def ev(e, s):
        if e == "%s + err" % s[0]:
            return f32(np.float64(s[1]) + err)
        if e == "%s + gap / 2" % s[0]:
            return f32(s[1] + gap / f32(2))
        if e == "%s + gap * 3 / 2 - err" % s[0]:
            return f32(np.float64(s[1] + gap * f32(3) / f32(2)) - err)
        if e == "%s + gap - err" % s[0]:
            return f32(np.float64(s[1] + gap) - err)
        raise SystemExit("unknown expression " + e)

    xy = [[float(ev(ex, ("start_x", sx))), float(ev(ey, ("start_y", sy)))] for ex, ey in expr]
    ncount_line = _line_of(t, "nCount] ==")
    ncount = _ints(t.splitlines()[ncount_line])  # the vector is on the following line
    sets = [sorted(_ints(s)) for s in re.findall(r"\) == sort\(\[([^\]]*)\]\)", t)]
    if len(sets) != 9 or len(ncount) != 9:
        raise SystemExit("could not parse neighbour sets")
    return {
        "source": rel,
        "lines": {"domain": _line_of(t, "Domain2D{IT, FT}(0.15"), "positions": [49, 59],
                  "ncount": ncount_line, "sets": [72, 152]},
        "domain": {"gap": dom[0], "first": dom[1:3], "last": dom[3:5]},
        "active_pair": active,
        "max_neighbour_number": 50,
        "positions": xy,
        "tags": [1] * 9,
        "criterion": "default",
        "ncount": ncount,
        "neighbour_sets": sets,
    }


def action(root):
    rel = "test/Algorithm/ActionTest.jl"
    t = _read(root, rel)
    ln = _line_of(t, "float_properties_[1:9, 1] ≈ FT[")
    vals = _ints(t.splitlines()[ln - 1].split("FT[")[1])
    return {"source": rel, "line": ln, "counts": vals}


def neighbour_cells(root):
    rel = "test/Class/NeighbourSystem/NeighbourSystemBaseTest.jl"
    t = _read(root, rel)
    m = re.search(r"Domain2D\{IT, FT\}\(([^)]*)\)", t)
    dom = [float(v) for v in m.group(1).split(",")]
    ln = _line_of(t, "neighbour_cell_index_count_) ==")
    counts = _ints(t.splitlines()[ln])
    shape = _ints(re.search(r"neighbour_cell_index_list_\) == \((\d+, \d+)\)", t).group(1))
    return {"source": rel, "line": ln, "domain": {"gap": dom[0], "first": dom[1:3], "last": dom[3:5]},
            "counts": counts, "list_shape": shape}


def domain(root):
    rel = "test/Class/DomainTest.jl"
    t = _read(root, rel)
    g = lambda name: float(re.search(name + r" = (-?[0-9.]+)", t).group(1))
    out = {"source": rel, "gap": g("gap"), "first": [g("x_0"), g("y_0")], "last": [g("x_1"), g("y_1")]}
    out["n_x"] = _ints(re.search(r"get_n_x\(domain_2d\) == (\d+)", t).group(1))[0]
    out["n_y"] = _ints(re.search(r"get_n_y\(domain_2d\) == (\d+)", t).group(1))[0]
    m = re.search(r"indexCartesianFromPosition\(domain_2d, ([0-9.]+)f0, ([0-9.]+)f0\) == \(IT\((\d+)\), IT\((\d+)\)\)", t)
    out["point"] = [float(m.group(1)), float(m.group(2))]
    out["cartesian"] = [int(m.group(3)), int(m.group(4))]
    m = re.search(r"indexLinearFromPosition\(domain_2d, [0-9.]+f0, [0-9.]+f0\) == IT\((\d+) \+ \((\d+) - 1\) \* (\d+)\)", t)
    a, b, c = int(m.group(1)), int(m.group(2)), int(m.group(3))
    out["linear"] = a + (b - 1) * c
    m = re.search(r"indexCartesianToLinear\(domain_2d, IT\((\d+)\), IT\((\d+)\)\) == (\d+) \+ \((\d+) - 1\) \* (\d+)", t)
    out["to_linear"] = {"ij": [int(m.group(1)), int(m.group(2))],
                        "value": int(m.group(3)) + (int(m.group(4)) - 1) * int(m.group(5))}
    out["inside_point"] = out["point"]
    out["lines"] = [16, 39]
    return out


def adjacency(root):
    rel = "test/Class/NeighbourSystem/ActivePairTest.jl"
    t = _read(root, rel)
    pairs = [tuple(_ints(p)) for p in re.search(r"pair_vector = \[([^\]]*)\]", t).group(1).split(",")]
    body = t.split("adjacency_matrix_) == IT[")[1].split("]")[0]
    rows = [_ints(r) for r in body.strip().splitlines() if r.strip()]
    rel2 = "test/Class/NeighbourSystem/NeighbourSystemTest.jl"
    t2 = _read(root, rel2)
    pairs2 = [tuple(_ints(p)) for p in re.search(r"active_pair = \[([^\]]*)\]", t2).group(1).split(",")]
    body2 = t2.split("adjacency_matrix_) ==")[1].split("IT[")[1].split("]")[0]
    rows2 = [_ints(r) for r in body2.strip().splitlines() if r.strip()]
    return [{"source": rel, "pairs": pairs, "matrix": rows},
            {"source": rel2, "pairs": pairs2, "matrix": rows2}]


def columns(root):
    rel = "test/Class/ParticleSystem/ParticleSystemTest.jl"
    t = _read(root, rel)
    out = {"source": rel}
    for key in ["Tag", "IsMovable", "nCount", "nIndex", "nR", "PositionVec", "nRVec"]:
        out[key] = int(re.search(r"basic_index_\.%s == (\d+)" % key, t).group(1))
    body = re.search(r"float_named_tuple = \((.*?)\n        \)", t, re.S).group(1)
    out["float_named_tuple"] = [[k, v.strip()] for k, v in re.findall(r"(\w+) = ([^,\n]+)", body)]
    body = re.search(r"int_named_tuple = \(([^)]*)\)", t).group(1)
    out["int_named_tuple"] = [[k, v.strip()] for k, v in re.findall(r"(\w+) = ([^,]+)", body)]
    out["neighbour_count"] = 50
    out["dim"] = 2
    return out


def main():
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: make_golden.py <path to a checkout of EtherParallelParticles.jl>")
    root = sys.argv[1]
    kat = {
        "generated_by": "tests/golden/make_golden.py",
        "neighbour_search": neighbour_search(root),
        "action": action(root),
        "neighbour_cells": neighbour_cells(root),
        "domain": domain(root),
        "adjacency": adjacency(root),
        "columns": columns(root),
    }
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kat.json")
    with open(out, "w") as f:
        json.dump(kat, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
