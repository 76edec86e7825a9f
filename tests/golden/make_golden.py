"""Copy the reference's own example inputs and golden outputs used as fixtures.

Run once in a container where the reference checkout is available:

    python tests/golden/make_golden.py /path/to/qudos

It copies, per example, ``parameters.in`` and ``supercell.in`` (comment lines
removed) and the golden ``energies_vb.dat`` / ``energies_cb.dat`` from
``code/example/<name>/Electronic_structure``, and extracts from the golden
``coulomb_matrix_elements_{hh,ee,eh_direct}.dat`` the gauge-invariant direct
terms between Kramers pairs (J_PQ = sum over the two states of each pair of
V(i, i, k, k)) into ``coulomb_direct.json``.  The tests read only these
fixtures, never the reference checkout.
"""

import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

EXAMPLES = {"prism_111": "Prism_111"}


def strip_comments(text):
    out = []
    for line in text.splitlines():
        s = line.split("#", 1)[0].rstrip() if line.lstrip().startswith("#") else line.rstrip()
        if s.strip():
            out.append(s)
    return "\n".join(out) + "\n"


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, ex in EXAMPLES.items():
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
        p, _ = inputs.load(dst)
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
