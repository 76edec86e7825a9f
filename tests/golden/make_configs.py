"""Oracle fixtures for the measured workloads at their full sizes.

    python tests/golden/make_configs.py [name ...]      (names: pyramid_11, molecule_15)

Runs the CPU oracle (numpy assembly + LAPACK zheevr from scipy's OpenBLAS)
once per deck and stores, in ``tests/golden/<name>/oracle.json``:

* the window's eigenvalues (eV), ascending;
* the Kramers-summed Bloch characters of every pair (8 bands);
* gauge-invariant projections of every Kramers pair's subspace: for the
  seeded probe vectors r_k (``probe_vectors``), ||V_P^H r_k||^2 / ||r_k||^2,
  which a rotation inside the pair leaves unchanged and which moves by about
  the subspace angle when the subspace moves;
* the oracle's wall times.

The decks are those of ``qudos_b200.configs``; ``molecule_15`` is solved with
16 e + 16 h Kramers pairs (64 states), whose window contains the 32-state
window of the metric.  The GPU tests compare against these numbers without
rerunning a 15^3 CPU solve.
"""

import json
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

N_PROBES = 4


def probe_vectors(n_h, n_probes=N_PROBES, seed=20261204):
    """Complex Gaussian probes, the same on every machine (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n_h, n_probes)) + 1j * rng.standard_normal((n_h, n_probes))


def pair_projections(v, probes):
    """(n_pairs, n_probes): ||V_P^H r_k||^2 / ||r_k||^2 for consecutive column pairs P."""
    c = np.abs(v.conj().T @ probes) ** 2
    c = c[0::2] + c[1::2]
    return c / (np.abs(probes) ** 2).sum(axis=0)[None, :]


DECKS = {
    "pyramid_11": lambda C: C.pyramid_11(mg=5, n_states=8),
    "molecule_15": lambda C: C.molecule_15(mg=7, n_states=16),
}


def make(name):
    from qudos_b200 import configs
    from oracle import eigen, inputs, pipeline

    params, cell = DECKS[name](configs)
    with tempfile.TemporaryDirectory() as d:
        configs.write_deck(d, params, cell)
        p, geo = inputs.load(d)
        t0 = time.time()
        pr = pipeline.prepare(p, geo)
        t1 = time.time()
        H = pipeline.assemble(pr)
        t2 = time.time()
        lo, hi = eigen.index_window(pr.n_pw, p["N_VB"], p["N_CB"])
        w, v = eigen.diagonalise(H, lo, hi)
        t3 = time.time()
    del H
    bloch = eigen.bloch_character(v, pr.n_pw)
    out = {
        "deck": name, "n_h": int(pr.n_h), "n_pw": int(pr.n_pw), "N_VB": int(p["N_VB"]), "N_CB": int(p["N_CB"]),
        "window": [int(lo), int(hi)], "eigenvalues_eV": w.tolist(),
        "bloch_pairs": (bloch[0::2] + bloch[1::2]).tolist(),
        "probe_seed": 20261204, "n_probes": N_PROBES,
        "pair_projections": pair_projections(v, probe_vectors(pr.n_h)).tolist(),
        "oracle_seconds": {"tables": t1 - t0, "assembly": t2 - t1, "zheevr": t3 - t2},
        "oracle": "numpy assembly + scipy.linalg.eigh(driver='evr', subset_by_index) on OpenBLAS",
        "threads": os.cpu_count(),
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), name)
    os.makedirs(dst, exist_ok=True)
    with open(os.path.join(dst, "oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(name, "N_H", pr.n_h, "seconds", out["oracle_seconds"])


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(DECKS)):
        make(n)
