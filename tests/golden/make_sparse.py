"""Writes tests/golden/sparse_index.npz: cell lists and pull index arrays computed by lbmpy's own
``SparseLbMapper`` (src/lbmpy/sparse/mapping.py:13-156) on small 3-D flag fields.

Run where a checkout of mabau/lbmpy is available, giving its root as the argument:

    python tests/golden/make_sparse.py <path to the lbmpy checkout>

lbmpy's package needs pystencils to import; the mapper class itself needs only numpy, so this
script takes the class definition out of mapping.py with ``ast`` and executes it alone (the one
pystencils name it reads, the coordinate field names, is supplied).  The fixture is committed, so
the tests never read the reference.

Cases (flags: fluid 1, NoSlip 2, UBB 4; ghost layer of 1):
- ``channel``: D3Q19, 6 x 5 x 4 interior, NoSlip at y = 0 and y = max, x and z periodic
  (ghost cells flagged 0, reached through the periodic wrap).
- ``cavity``: D3Q19, 5 x 5 x 5 interior, NoSlip walls, UBB lid at z = max (listed boundary cells),
  a NoSlip block inside.
- ``periodic27``: D3Q27, 4 x 3 x 5 fully periodic box with a NoSlip cell in the middle.
"""
import ast
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FLUID, NOSLIP, UBB = 1, 2, 4


def load_mapper(reference_root):
    path = os.path.join(reference_root, "src", "lbmpy", "sparse", "mapping.py")
    tree = ast.parse(open(path).read())
    cls = next(n for n in tree.body if isinstance(n, ast.ClassDef) and n.name == "SparseLbMapper")
    mod = ast.Module(body=[cls], type_ignores=[])
    ns = {"np": np, "Tuple": tuple, "boundary_index_array_coordinate_names": ["x", "y", "z"]}
    exec(compile(mod, path, "exec"), ns)
    return ns["SparseLbMapper"]


def cases():
    orderings = json.load(open(os.path.join(HERE, "stencil_orderings.json")))
    q19 = [tuple(d) for d in orderings["D3Q19"]["walberla"]]
    q27 = [tuple(d) for d in orderings["D3Q27"]["walberla"]]

    ch = np.zeros((8, 7, 6), dtype=np.uint16)
    ch[1:-1, 1:-1, 1:-1] = FLUID
    ch[:, 0, :] = NOSLIP
    ch[:, -1, :] = NOSLIP

    cav = np.full((7, 7, 7), NOSLIP, dtype=np.uint16)
    cav[1:-1, 1:-1, 1:-1] = FLUID
    cav[:, :, -1] = UBB
    cav[2:4, 3, 2:4] = NOSLIP

    per = np.zeros((6, 5, 7), dtype=np.uint16)
    per[1:-1, 1:-1, 1:-1] = FLUID
    per[2, 2, 3] = NOSLIP
    return {"channel": (q19, ch, UBB), "cavity": (q19, cav, UBB), "periodic27": (q27, per, UBB)}


def main(reference_root):
    Mapper = load_mapper(reference_root)
    out = {}
    for name, (stencil, flags, other) in cases().items():
        m = Mapper(stencil, flags, FLUID, NOSLIP, other)
        idx = m.create_index_array(1)
        coords = m.coordinates
        out[f"{name}_flags"] = flags
        out[f"{name}_coords"] = np.stack([coords[c] for c in ("x", "y", "z")], axis=-1)
        out[f"{name}_num_fluid"] = np.array(m.num_fluid_cells)
        out[f"{name}_index"] = np.ascontiguousarray(idx)
    np.savez_compressed(os.path.join(HERE, "sparse_index.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
