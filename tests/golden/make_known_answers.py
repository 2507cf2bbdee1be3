"""Extract the reference's in-repository known answers for the multifrontal
hot path into known_answers.json (run in a container where the reference
checkout is mounted; the JSON is committed so tests never read the
reference at run time).

Sources (paths relative to the reference root):
  src/Multifrontal.jl/README.md   Cholesky example (A, factor L, F \\ b),
                                  LDLt example (A, unit L, D, F \\ b, signs=)
  src/AMFLib.jl/README.md         AMF order of the 8-vertex graph
  README.md                       clique tree of the 8-vertex graph (alg=MF())
  src/Multifrontal.jl/src/selinv.jl  selected inverse of the 5x5 example (docstring)
  src/Multifrontal.jl/src/regularization/dynamic_regularization.jl
                                  DynamicRegularization example: A and Matrix(F)
                                  (printed to 6 significant digits)
  test/core.jl                    the 17-vertex graph of Vandenberghe & Andersen
                                  (Figure 4.3) and its clique tree under the order
                                  1:17 with Maximal supernodes (Figure 4.7 left):
                                  parent indices, residuals and separators

The factor displays are in elimination order (P A P^T = L L^T).
"""
from __future__ import annotations

import json
import os
import re
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")


def _rows_after(lines, start, count):
    rows = []
    i = start
    while len(rows) < count:
        s = lines[i].strip()
        i += 1
        if not s:
            continue
        toks = s.replace("⋅", "nan").split()
        rows.append([float(t) for t in toks])
    return rows, i


def _matrix_literal(lines, i):
    """Parse 'julia> A = [' ... ']' starting at line i."""
    rows = []
    j = i + 1
    while not lines[j].strip().startswith("]"):
        rows.append([float(t) for t in lines[j].split()])
        j += 1
    return rows, j + 1


def _core_maximal(core):
    """The 17-vertex graph and its Maximal clique tree from test/core.jl."""
    i = next(k for k, l in enumerate(core) if l.strip().startswith("_graph = BipartiteGraph("))
    j = next(k for k in range(i, len(core)) if core[k].strip() == "[")
    G = []
    j += 1
    while core[j].strip() != "],":
        G.append([int(t) for t in core[j].split()])
        j += 1
    i = next(k for k in range(j, len(core)) if "cliquetree(graph; alg = 1:17, snd = Maximal())" in core[k])
    i = next(k for k in range(i, len(core)) if "map(i -> parentindex(tree, i), 1:8)" in core[k])
    par = re.search(r"\[(.*)\]", core[i + 1]).group(1)
    parent = [None if t.strip() == "nothing" else int(t) for t in par.split(",")]

    def label_lists(start_marker):
        k = next(q for q in range(i, len(core)) if start_marker in core[q])
        lists = []
        k += 1
        while len(lists) < 8:
            m = re.search(r"\[([\d, ]*)\]", core[k])
            if m:
                body = m.group(1).strip()
                lists.append([int(t) for t in body.split(",")] if body else [])
            k += 1
        return lists

    res = label_lists("map(i -> view(label, residual(tree, i)), 1:8)")
    sep = label_lists("map(i -> view(label, separator(tree, i)), 1:8)")
    return {"graph": G, "order": list(range(1, 18)), "parent": parent, "residual_labels": res,
            "separator_labels": sep}


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_known_answers.py <path of a CliqueTrees.jl checkout>")
    REF = sys.argv[1]
    mf = open(os.path.join(REF, "src/Multifrontal.jl/README.md")).read().splitlines()
    out = {"source": "AlgebraicJulia/CliqueTrees.jl READMEs (see make_known_answers.py)"}
    # --- Cholesky example
    i = next(k for k, l in enumerate(mf) if l.startswith("julia> A = ["))
    A, i = _matrix_literal(mf, i)
    i = next(k for k in range(i, len(mf)) if "cholesky!(ChordalCholesky(A))" in mf[k])
    L, i = _rows_after(mf, i + 2, 5)
    i = next(k for k in range(i, len(mf)) if mf[k].startswith("julia> b = ["))
    b = [float(t) for t in re.findall(r"-?\d+", mf[i].split("=")[1])]
    i = next(k for k in range(i, len(mf)) if mf[k].startswith("julia> F \\ b"))
    x = [float(mf[k].strip()) for k in range(i + 2, i + 7)]
    out["cholesky"] = {"A": A, "L": L, "b": b, "x": x}
    # --- LDLt example
    i = next(k for k in range(i, len(mf)) if mf[k].startswith("julia> A = ["))
    A2, i = _matrix_literal(mf, i)
    i = next(k for k in range(i, len(mf)) if "ldlt!(ChordalLDLt(A))" in mf[k])
    L2, i = _rows_after(mf, i + 2, 5)
    D2, i = _rows_after(mf, i, 5)
    d2 = [D2[r][r] if len(D2[r]) > r else D2[r][0] for r in range(5)]
    # D rows print as '4.0 ⋅ ⋅ ...' so the diagonal is the only number in each row
    d2 = [[v for v in row if v == v][0] for row in D2]
    i = next(k for k in range(i, len(mf)) if mf[k].startswith("julia> b = ["))
    b2 = [float(t) for t in re.findall(r"-?\d+", mf[i].split("=")[1])]
    i = next(k for k in range(i, len(mf)) if mf[k].startswith("julia> F \\ b"))
    x2 = [float(mf[k].strip()) for k in range(i + 2, i + 7)]
    i = next(k for k in range(i, len(mf)) if "signs=[" in mf[k])
    signs = [float(t) for t in re.findall(r"-?\d+", mf[i].split("signs=")[1])]
    L3, i = _rows_after(mf, i + 2, 5)
    D3, i = _rows_after(mf, i, 5)
    d3 = [[v for v in row if v == v][0] for row in D3]
    out["ldlt"] = {"A": A2, "L": L2, "d": d2, "b": b2, "x": x2, "signs": signs, "L_signs": L3, "d_signs": d3}
    # --- AMF order of the 8-vertex graph
    amf = open(os.path.join(REF, "src/AMFLib.jl/README.md")).read().splitlines()
    i = next(k for k, l in enumerate(amf) if "graph = sparse([" in l)
    G = []
    j = i + 1
    while not amf[j].strip().startswith("])"):
        G.append([int(t) for t in amf[j].split()])
        j += 1
    i = next(k for k in range(j, len(amf)) if amf[k].strip() == "julia> perm")
    perm = [int(amf[k].strip()) for k in range(i + 2, i + 10)]
    out["amf"] = {"graph": G, "perm": perm}
    # --- clique tree (alg = MF()) of the same graph
    rd = open(os.path.join(REF, "README.md")).read().splitlines()
    i = next(k for k, l in enumerate(rd) if "cliquetree(graph; alg=MF())" in l)
    i = next(k for k in range(i, len(rd)) if rd[k].startswith("julia> tree"))
    tree_lines = []
    k = i + 2
    while rd[k].strip() and not rd[k].startswith("```"):
        tree_lines.append(rd[k])
        k += 1
    # parse the printed tree: depth from the prefix width, bag from [..]
    nodes = []
    stack = []
    for line in tree_lines:
        m = re.search(r"\[([\d, ]+)\]", line)
        bag = [int(t) for t in m.group(1).split(",")]
        depth = m.start() // 3
        while len(stack) > depth:
            stack.pop()
        parent = stack[-1] if stack else None
        nodes.append({"bag": bag, "parent": parent})
        stack.append(bag)
    out["cliquetree_mf"] = nodes
    # --- selected inverse of the 5x5 example (selinv.jl docstring)
    sl = open(os.path.join(REF, "src/Multifrontal.jl/src/selinv.jl")).read().splitlines()
    i = next(k for k, l in enumerate(sl) if l.startswith("julia> A = ["))
    As, i = _matrix_literal(sl, i)
    i = next(k for k in range(i, len(sl)) if "selinv!(cholesky!(ChordalCholesky(A)))" in sl[k])
    Z, i = _rows_after(sl, i + 2, 5)
    out["selinv"] = {"A": As, "Z": Z}
    # --- DynamicRegularization example (docstring)
    dr = open(os.path.join(REF, "src/Multifrontal.jl/src/regularization/dynamic_regularization.jl")).read().splitlines()
    i = next(k for k, l in enumerate(dr) if l.startswith("julia> A = ["))
    Ad, i = _matrix_literal(dr, i)
    i = next(k for k in range(i, len(dr)) if dr[k].startswith("julia> B = Matrix(F)"))
    Bd, i = _rows_after(dr, i + 2, 3)
    out["dynamic_regularization"] = {"A": Ad, "B": Bd}
    # --- the 17-vertex graph and its Maximal clique tree (order 1:17)
    core = open(os.path.join(REF, "test/core.jl")).read().splitlines()
    out["maximal17"] = _core_maximal(core)
    json.dump(out, open(OUT, "w"), indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
