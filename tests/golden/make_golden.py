"""Copy the reference's own example inputs and golden outputs used as fixtures.

Run once in a container where the reference checkout is available:

    python tests/golden/make_golden.py /path/to/qudos

It copies, per example, ``parameters.in`` and ``supercell.in`` (comment lines
removed) and the golden ``energies_vb.dat`` / ``energies_cb.dat`` from
``code/example/<name>/Electronic_structure``, and extracts from the golden
outputs the quantities that do not depend on the phase of each state or on
the rotation of the two states of a Kramers pair:
* ``coulomb_direct.json``: the direct terms between Kramers pairs
  (J_PQ = sum over the two states of each pair of V(i, i, k, k)) from
  ``coulomb_matrix_elements_{hh,ee,eh_direct}.dat``;
* ``momentum_pairs.json``: for each of the five polarisations of
  ``momentum_matrix_elements.dat`` ([100], [010], [001], [110], [-110]) the sums
  of |p|^2 over the four (CB state, VB state) combinations of a CB pair and a
  VB pair;
* ``probability_pairs.npz``: the probability densities of the example's line
  scans ([100], [001], [111] for Prism_111; [100], [010], [001] for
  Truncated_pyramid; ``probability_density_{vb,cb}_<k>_<dir>.dat``, columns
  total, SO, LH, HH, CB in nm^-3) summed over the two states of each pair.
The tests read only these fixtures, never the reference checkout.
"""

import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

# fixture directory -> (example, line scans in its golden outputs)
EXAMPLES = {"prism_111": ("Prism_111", ("100", "001", "111")),
            "truncated_pyramid": ("Truncated_pyramid", ("100", "010", "001"))}


def strip_comments(text):
    out = []
    for line in text.splitlines():
        s = line.split("#", 1)[0].rstrip() if line.lstrip().startswith("#") else line.rstrip()
        if s.strip():
            out.append(s)
    return "\n".join(out) + "\n"


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, (ex, scans) in EXAMPLES.items():
        src = os.path.join(ref, "code", "example", ex, "Electronic_structure")
        dst = os.path.join(here, name)
        os.makedirs(dst, exist_ok=True)
        for f in ("parameters.in", "supercell.in"):
            with open(os.path.join(src, f)) as fi, open(os.path.join(dst, f), "w") as fo:
                fo.write(strip_comments(fi.read()))
        for f in ("energies_vb.dat", "energies_cb.dat"):
            with open(os.path.join(src, "PWEM_test_ref", f)) as fi, open(os.path.join(dst, f), "w") as fo:
                fo.write(fi.read())
        from oracle import coulomb, inputs
        import numpy as np
        p, _ = inputs.load(dst)
        ref_dir = os.path.join(src, "PWEM_test_ref")
        # momentum matrix elements: |p| columns 5, 8, 11, 14, 17 (1-based) per polarisation
        mm = np.loadtxt(os.path.join(ref_dir, "momentum_matrix_elements.dat"), ndmin=2)
        ncs, nvs = 2 * p["N_CB"], 2 * p["N_VB"]
        absp = np.zeros((5, ncs, nvs))
        for row in mm:
            c, v = int(row[0]) - 1, int(row[1]) - 1
            absp[:, c, v] = row[[4, 7, 10, 13, 16]]
        sums = (absp ** 2).reshape(5, ncs // 2, 2, nvs // 2, 2).sum(axis=(2, 4))
        with open(os.path.join(dst, "momentum_pairs.json"), "w") as fo:
            json.dump({"source": "code/example/%s/Electronic_structure/PWEM_test_ref/momentum_matrix_elements.dat" % ex,
                       "polarisations": ["100", "010", "001", "110", "-110"],
                       "units": "eV (|p|^2 / (HBSQM / 2))", "pair_sums": sums.tolist()}, fo, indent=1)
        # probability densities of three line scans, summed over Kramers pairs
        arrays = {}
        for tag in scans:
            for band, n in (("vb", nvs), ("cb", ncs)):
                rows = [np.loadtxt(os.path.join(ref_dir, "probability_density_%s_%d_%s.dat" % (band, k + 1, tag)))
                        for k in range(n)]
                arrays["%s_%s" % (band, tag)] = np.stack(
                    [rows[2 * q][:, 4:9] + rows[2 * q + 1][:, 4:9] for q in range(n // 2)]).astype(np.float32)
                arrays["xyz_%s" % tag] = rows[0][:, 0:3]
        np.savez_compressed(os.path.join(dst, "probability_pairs.npz"), **arrays)
        nv, nc = 2 * p["N_VB"], 2 * p["N_CB"]
        J = coulomb.read_golden_direct(os.path.join(src, "PWEM_test_ref"), nv, nc)
        with open(os.path.join(dst, "coulomb_direct.json"), "w") as fo:
            json.dump({"source": "code/example/%s/Electronic_structure/PWEM_test_ref" % ex, "n_vb_states": nv,
                       "n_cb_states": nc, "CME": p["CME"], "ranks": 4,
                       **{k: v.tolist() for k, v in J.items()}}, fo, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/qudos-checkout")
    main(sys.argv[1])
