"""Writes tests/golden/stencil_orderings.json: lbmpy's 'walberla' and 'lehmann' direction orderings
of D2Q9, D3Q19 and D3Q27, read as literals from the reference's src/lbmpy/stencils.py (run where
the reference checkout is available; the fixture is committed so tests never read the reference).
EsoPull / EsoPush (fieldaccess.py:184-318) stream a direction on read or on write by the parity
of its position in the 'lehmann' ordering."""
import ast
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def orderings(reference_root):
    path = os.path.join(reference_root, "src", "lbmpy", "stencils.py")
    tree = ast.parse(open(path).read())
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "predefined_stencils" for t in node.targets):
            table = ast.literal_eval(node.value)
            return {name: {k: [list(d) for d in table[name][k]] for k in ("walberla", "lehmann")}
                    for name in ("D2Q9", "D3Q19", "D3Q27")}
    raise RuntimeError("predefined_stencils not found in " + path)


def main(reference_root):
    with open(os.path.join(HERE, "stencil_orderings.json"), "w") as fh:
        json.dump(orderings(reference_root), fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_orderings.py <path to the lbmpy checkout>")
    main(sys.argv[1])
