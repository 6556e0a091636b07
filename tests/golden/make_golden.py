"""Builds tests/golden/*.npz from the reference's own regression data.

Run where a checkout of mabau/lbmpy is available, giving its root as the argument:

    python tests/golden/make_golden.py <path to the lbmpy checkout>

The fixtures are committed, so the tests never read the reference.  Source files are lbmpy's
``tests/reference_files/*.npz``: final PDF states written by lbmpy's own generated kernels.

- ``ldc_d3q19_*_slab.npz``: a slab of 4 x-planes of the D3Q19 lid-driven cavities with the
  density and velocity lbmpy's getter wrote for them.
- ``lbmpy_states.npz``: for every regression state, its shape and a seeded sample of flat
  indices into the PDF array with the values lbmpy stored there (every entry for the small
  2-D cavities, 4096 entries otherwise).  The run parameters that reproduce each state are
  stated by the test that uses it (tests/test_golden_states.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

STATES = [f"LidDrivenCavity_SRT_{fm}_{c}" for fm in ("guo", "luo", "simple")
          for c in ("compressible", "incompressible")]
STATES += [f"ForceDrivenChannel_{fm}_{c}" for fm in ("guo", "luo", "simple")
           for c in ("compressible", "incompressible")]
STATES += ["LidDrivenCavity_TRT_luo_compressible", "LidDrivenCavity_TRT_luo_incompressible",
           "LidDrivenCavity_MRT_incompressible"]
SAMPLE = 4096


def main(reference_root):
    files = os.path.join(reference_root, "tests", "reference_files")
    sl = slice(6, 10)
    d = np.load(os.path.join(files, "LidDrivenCavity_MRT_incompressible.npz"))
    np.savez_compressed(os.path.join(HERE, "ldc_d3q19_mrt_incompressible_slab.npz"),
                        pdfs=d["pdfs"][sl], rho=d["rho"][sl], vel=d["vel"][sl])
    d = np.load(os.path.join(files, "LidDrivenCavity_TRT_luo_compressible.npz"))
    np.savez_compressed(os.path.join(HERE, "ldc_d3q19_trt_compressible_slab.npz"),
                        pdfs=d["pdfs"][sl], rho=d["rho"][sl], vel=d["vel"][sl])
    out = {}
    rng = np.random.default_rng(2024)
    for name in STATES:
        pdfs = np.load(os.path.join(files, name + ".npz"))["pdfs"]
        flat = pdfs.reshape(-1)
        if flat.size <= SAMPLE:
            idx = np.arange(flat.size, dtype=np.int64)
        else:
            idx = np.sort(rng.choice(flat.size, SAMPLE, replace=False)).astype(np.int64)
        out[name + "__shape"] = np.array(pdfs.shape, np.int64)
        out[name + "__idx"] = idx
        out[name + "__val"] = flat[idx]
    np.savez_compressed(os.path.join(HERE, "lbmpy_states.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the lbmpy checkout>")
    main(sys.argv[1])
