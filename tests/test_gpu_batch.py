"""Batched solves (GPU): eigenstates_batched over instances of different sizes
returns, for every instance, what a solve of that instance alone returns
(FP64: within 1e-10 eV; mixed: within 1 micro-eV of the FP64 solve)."""

import os

import numpy as np
import pytest

import qudos_b200 as q
from qudos_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


def _dirs(tmp, n):
    decks = configs.batch_lenses(n, seed=3)
    out = []
    for i, (p, c, desc) in enumerate(decks):
        # keep the test small: cutoffs 5^3 and 7^3 only
        mg = 2 + (desc["mg"] % 2)
        p = p.replace("M_Gx: %d" % desc["mg"], "M_Gx: %d" % mg).replace("M_Gy: %d" % desc["mg"], "M_Gy: %d" % mg)
        p = p.replace("M_Gz: %d" % desc["mg"], "M_Gz: %d" % mg).replace("M_S_Gx: %d" % desc["mg"], "M_S_Gx: %d" % mg)
        p = p.replace("M_S_Gy: %d" % desc["mg"], "M_S_Gy: %d" % mg).replace("M_S_Gz: %d" % desc["mg"], "M_S_Gz: %d" % mg)
        out.append(configs.write_deck(os.path.join(str(tmp), "b%d" % i), p, c))
    return out


@pytest.mark.parametrize("threads", [1, 4])
def test_batched_matches_single_solves(tmp_path, threads):
    dirs = _dirs(tmp_path, 6)
    ref = [q.Problem(d).solve(q.QD_PREC_FP64) for d in dirs]
    assert len({r[1].shape[0] for r in ref}) == 2  # both sizes present
    out64 = q.solve_batch([q.Problem(d) for d in dirs], q.QD_PREC_FP64, threads)
    outmx = q.solve_batch([q.Problem(d) for d in dirs], q.QD_PREC_MIXED, threads)
    for (w, v), (w64, _), (wmx, _) in zip(ref, out64, outmx):
        assert np.abs(w64 - w).max() < 1e-10
        assert np.abs(wmx - w).max() < 1e-6
