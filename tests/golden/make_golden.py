"""Builds tests/golden/*.npz from the reference's own regression data (run where the reference
checkout is available; the fixtures are committed so tests never read the reference).

Source: lbmpy tests/reference_files/LidDrivenCavity_MRT_incompressible.npz (D3Q19, walberla
order, zero-centred incompressible storage, no force) -- a slab of 4 x-planes is kept, with the
density and velocity lbmpy's getter wrote for it.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(reference_root):
    src = os.path.join(reference_root, "tests", "reference_files", "LidDrivenCavity_MRT_incompressible.npz")
    d = np.load(src)
    sl = slice(6, 10)
    np.savez_compressed(os.path.join(HERE, "ldc_d3q19_mrt_incompressible_slab.npz"),
                        pdfs=d["pdfs"][sl], rho=d["rho"][sl], vel=d["vel"][sl])
    src = os.path.join(reference_root, "tests", "reference_files", "LidDrivenCavity_TRT_luo_compressible.npz")
    d = np.load(src)
    np.savez_compressed(os.path.join(HERE, "ldc_d3q19_trt_compressible_slab.npz"),
                        pdfs=d["pdfs"][sl], rho=d["rho"][sl], vel=d["vel"][sl])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
