"""PhenomD QNM table: final spin -> 22-mode ringdown / damping frequency (1001 points,
spin step ``dspin``), the model data the reference ships in
src/bbhx/waveforms/ringdownphenomd.py; loaded from ``bbhx_b200/data/qnm_phenomd.npz``
(written by the test-side recipe ``oracle/make_qnm_table.py``)."""
import os

import numpy as np

_d = np.load(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "data",
                          "qnm_phenomd.npz"))
dspin = float(_d["dspin"])
QNMData_a = _d["a"].copy()
QNMData_fring = _d["fring"].copy()
QNMData_fdamp = _d["fdamp"].copy()
