"""Extract the PhenomD QNM table (final spin -> 22-mode ringdown and damping frequency,
1001 points, spin step 0.002) that the reference ships as Python data
(src/bbhx/waveforms/ringdownphenomd.py:3-2016) into ``qnm_phenomd.npz``.

The table is part of the PhenomD model definition (the reference fits a cubic spline
through it, phenomhm.py:148-163); it is data, not code, and must be identical for parity.
Test-side recipe, run once where the reference checkout exists:  python oracle/make_qnm_table.py
"""
import ast
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle.build_ref import REF_ROOT  # noqa: E402

SRC = os.path.join(REF_ROOT, "src", "bbhx", "waveforms", "ringdownphenomd.py")


def main():
    tree = ast.parse(open(SRC).read())
    vals = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            v = node.value
            if isinstance(v, ast.Call):  # np.array([...])
                vals[name] = np.array(ast.literal_eval(v.args[0]), dtype=np.float64)
            else:
                vals[name] = np.float64(ast.literal_eval(v))
    out = os.path.join(os.path.dirname(HERE), "bbhx_b200", "data", "qnm_phenomd.npz")
    np.savez(out, dspin=vals["dspin"], a=vals["QNMData_a"], fring=vals["QNMData_fring"],
             fdamp=vals["QNMData_fdamp"])
    print(out, {k: np.shape(v) for k, v in vals.items()})


if __name__ == "__main__":
    sys.exit(main())
