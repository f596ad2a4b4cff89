"""Golden vectors for the frame / sky-mode transforms (tests/golden/transform_golden.npz),
from the REFERENCE's own src/bbhx/utils/transform.py on seeded random inputs.

Runs only where the reference checkout exists (its location comes from oracle/build_ref.py);
the fixture it writes is what the tests read.  Usage: python tests/golden/make_transform_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)
from oracle.build_ref import REF_ROOT  # noqa: E402

REF_SRC = os.path.join(REF_ROOT, "src")
sys.path.insert(0, os.path.join(REPO, "oracle", "refenv"))
sys.path.insert(0, REPO)
sys.path.insert(0, REF_SRC)

from bbhx.utils import transform as T  # noqa: E402


def main():
    rng = np.random.default_rng(20261203)
    n = 64
    t = rng.uniform(0.0, 3.0e7, n)
    lam = rng.uniform(0.0, 2 * np.pi, n)
    beta = np.arcsin(rng.uniform(-1, 1, n))
    psi = rng.uniform(0.0, np.pi, n)
    t0 = 0.37
    out = dict(t=t, lam=lam, beta=beta, psi=psi, t0=np.array(t0))
    out["l2s"] = np.array(T.LISA_to_SSB(t, lam, beta, psi, t0))
    out["s2l"] = np.array(T.SSB_to_LISA(t, lam, beta, psi, t0))
    out["tssb"] = T.tSSBfromLframe(t, lam, beta, 0.0)
    out["tl"] = T.tLfromSSBframe(t, lam, beta, 0.0)
    out["modpi"] = T.modpi(rng.uniform(-20, 20, n))
    out["mod2pi_in"] = rng.uniform(-20, 20, n)
    out["mod2pi"] = T.mod2pi(out["mod2pi_in"])
    coords = rng.uniform(0.1, 3.0, (5, 12))
    out["coords"] = coords
    for kind in ("both", "long", "lat"):
        out[f"sky_{kind}"] = T.mbh_sky_mode_transform(coords.copy(), kind=kind)
        out[f"sky_{kind}_cosi"] = T.mbh_sky_mode_transform(coords.copy(), kind=kind, cos_i=True)
    out["modpi_in"] = rng.uniform(-20, 20, n)
    out["modpi"] = T.modpi(out["modpi_in"])
    np.savez_compressed(os.path.join(HERE, "transform_golden.npz"), **out)
    print("written", sorted(out))


if __name__ == "__main__":
    main()
