"""The autotuner's knob (GPU): the aggregation depth of the dense->band
reduction changes its schedule (how many Householder panels are applied per
rank-2K trailing update), not its result.  A 7^3 lens deck (N_H = 2744) is
solved at depths 64, 128 and 256 in both precisions: the FP64 eigenvalues
agree within 1e-9 eV, the mixed ones within 1 micro-eV."""

import numpy as np
import pytest

import qudos_b200 as q
from qudos_b200 import autotune, configs
from qudos_b200 import lib as L

pytestmark = pytest.mark.gpu


def test_aggregation_depth_changes_schedule_not_result(tmp_path):
    assert q.device_count() > 0, "no CUDA device visible"
    d = configs.write_deck(str(tmp_path / "lens"), *configs.lens_7(mg=3))
    pr = q.Problem(d)
    try:
        for prec, tol in ((q.QD_PREC_FP64, 1e-9), (q.QD_PREC_MIXED, 1e-6)):
            ws = []
            for depth in (64, 128, 256):
                L.check(L.lib.qd_tuning_set(0, 0, 0))
                L.check(L.lib.qd_tuning_set(prec, 1 << 62, depth))
                ws.append(pr.solve(prec)[0])
            for w in ws[1:]:
                assert np.abs(w - ws[0]).max() < tol, (prec, np.abs(w - ws[0]).max())
    finally:
        autotune.load()
