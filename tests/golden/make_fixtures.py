"""Generate the golden fixtures in this directory.

Run from the repository root, with the path of a reference checkout
(vaishna77/AIFMM_LS) as the only argument:

    python tests/golden/make_fixtures.py <reference checkout>

Outputs (small JSON files, committed):
  gauss_legendre_10.json   -- the reference's 10-point Gauss-Legendre table
                              (LS/Gauss_Legendre_Nodes_and_Weights.hpp, case 10)
  interaction_slots.json   -- the neighbour / inner / outer slot assignment of
                              FMM2DTree_find_error.hpp assign_Child{0..3}_Interaction
                              (which slot each child of each parent-neighbour gets)
  bessel_mpmath.json       -- J_n(x), Y_n(x), n = 0..60, from mpmath at 40 digits
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def gl_table(ref):
    src = open(os.path.join(ref, "LS", "Gauss_Legendre_Nodes_and_Weights.hpp")).read()
    start = src.index("case 10:")
    end = src.index("break;", start)
    body = src[start:end]
    nodes = dict(re.findall(r"nodes\[(\d+)\]\s*=\s*([-0-9.eE+]+);", body))
    weights = dict(re.findall(r"weights\[(\d+)\]\s*=\s*([-0-9.eE+]+);", body))
    n = 10
    return {"n": n,
            "nodes": [nodes[str(i)] for i in range(n)],
            "weights": [weights[str(i)] for i in range(n)],
            "source": "LS/Gauss_Legendre_Nodes_and_Weights.hpp case 10"}


def interaction_slots(ref):
    src = open(os.path.join(ref, "FMM2DTree_find_error.hpp")).read()
    out = []
    for c in range(4):
        m = re.search(r"void assign_Child%d_Interaction\(int j, int k\) \{(.*?)\n\t\}\n" % c, src, re.S)
        body = m.group(1)
        # siblings
        for kind, slot, off in re.findall(r"tree\[nL\]\[nC\]\.(neighborNumbers)\[(\d+)\]\s*=\s*nC([+-]\d+);", body):
            out.append({"child": c, "parent_neighbor": -1, "grandchild": c + int(off),
                        "kind": "neighbor", "slot": int(slot)})
        # blocks per parent neighbour
        parts = re.split(r"nN\s*=\s*tree\[j\]\[k\]\.neighborNumbers\[(\d+)\];", body)
        for i in range(1, len(parts), 2):
            pn = int(parts[i])
            blk = parts[i + 1]
            for kind, slot, g in re.findall(
                    r"tree\[nL\]\[nC\]\.(neighborNumbers|innerNumbers|outerNumbers)\[(\d+)\]\s*=\s*tree\[j\]\[nN\]\.childrenNumbers\[(\d+)\];", blk):
                out.append({"child": c, "parent_neighbor": pn, "grandchild": int(g),
                            "kind": {"neighborNumbers": "neighbor", "innerNumbers": "inner",
                                     "outerNumbers": "outer"}[kind], "slot": int(slot)})
    return {"source": "FMM2DTree_find_error.hpp assign_Child{0..3}_Interaction", "entries": out}


def bessel_fixture():
    import mpmath
    mpmath.mp.dps = 40
    xs = [0.05, 0.12, 0.3, 0.7, 0.94, 1.5, 2.7, 4.1, 7.3, 12.0, 19.5, 33.3, 47.9, 61.0, 75.2, 113.0, 180.4, 226.0]
    out = {"nmax": 60, "x": xs, "J": [], "Y": []}
    for x in xs:
        out["J"].append([mpmath.nstr(mpmath.besselj(n, x), 25) for n in range(61)])
        out["Y"].append([mpmath.nstr(mpmath.bessely(n, x), 25) for n in range(61)])
    return out


def main():
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: make_fixtures.py <path of the reference checkout>")
    ref = sys.argv[1]
    with open(os.path.join(HERE, "gauss_legendre_10.json"), "w") as f:
        json.dump(gl_table(ref), f, indent=1)
    with open(os.path.join(HERE, "interaction_slots.json"), "w") as f:
        json.dump(interaction_slots(ref), f, indent=0)
    with open(os.path.join(HERE, "bessel_mpmath.json"), "w") as f:
        json.dump(bessel_fixture(), f)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
