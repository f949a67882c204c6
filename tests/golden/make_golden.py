"""Generates tests/golden/ref_small.npz from the reference library itself.

The reference (YRT-PET 2.0.7) CPU library is compiled from its own sources by
oracle/ref.mk; this script drives it through oracle/pyoracle.py on small,
seeded inputs and stores the inputs and outputs.  The fixture travels with
the repository, so parity tests can run where the reference is absent.

    make -f oracle/ref.mk -j8 && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import pyoracle as po  # noqa: E402


def main():
    rng = np.random.default_rng(20261203)
    sc = po.Scanner(64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
    ip = po.ImageParams(32, 32, 16, 128, 128, 64)
    lut = po.ref_scanner_lut(sc)
    n = 512
    d1 = rng.integers(0, sc.num_dets, 4 * n).astype(np.uint32)
    d2 = rng.integers(0, sc.num_dets, 4 * n).astype(np.uint32)
    bins = po.ref_histo3d_bins(sc, d1, d2)
    ok = (bins != np.iinfo(np.uint64).max) & (d1 != d2)
    d1, d2, bins = d1[ok][:n], d2[ok][:n], bins[ok][:n]
    lors, ori = po.lors_from_detpairs(lut, d1, d2)
    img = rng.random(ip.shape, dtype=np.float32)
    tof = rng.normal(0, 250, n).astype(np.float32)
    vals = rng.random(n, dtype=np.float32)
    out = dict(lut=lut, d1=d1, d2=d2, bins=bins, lors=lors, orients=ori,
               image=img, tof=tof, values=vals,
               scanner=np.array([64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1],
                                np.float64),
               image_params=np.array([32, 32, 16, 128, 128, 64], np.float64))
    out["siddon_fwd"] = po.ref_siddon(sc, ip, lors, image=img, threads=1)
    out["siddon_tof_fwd"] = po.ref_siddon(sc, ip, lors, image=img, tof=tof,
                                          tof_fwhm_ps=214.0, tof_n_std=5,
                                          threads=1)
    out["siddon_bwd"] = po.ref_siddon(sc, ip, lors, values=vals,
                                      forward=False, threads=1)
    out["siddon_tof_bwd"] = po.ref_siddon(sc, ip, lors, values=vals, tof=tof,
                                          tof_fwhm_ps=214.0, tof_n_std=5,
                                          forward=False, threads=1)
    out["dd_fwd"] = po.ref_dd(sc, ip, lors, ori, image=img, threads=1)
    out["dd_tof_fwd"] = po.ref_dd(sc, ip, lors, ori, image=img, tof=tof,
                                  tof_fwhm_ps=214.0, tof_n_std=5, threads=1)
    dims = po.ref_histo3d_dims(sc)
    out["histo_dims"] = np.array(dims, np.uint64)
    qb = rng.integers(0, int(np.prod(dims)), 256).astype(np.uint64)
    pd1, pd2 = po.ref_histo3d_detpairs(sc, qb)
    out["query_bins"], out["query_d1"], out["query_d2"] = qb, pd1, pd2
    np.savez_compressed(os.path.join(HERE, "ref_small.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_small.npz"))


if __name__ == "__main__":
    main()
