"""Copy the reference's own example inputs and golden outputs used as fixtures.

Run once in a container where the reference checkout is available:

    python tests/golden/make_golden.py /path/to/qudos

It copies, per example, ``parameters.in`` and ``supercell.in`` (comment lines
removed) and the golden ``energies_vb.dat`` / ``energies_cb.dat`` from
``code/example/<name>/Electronic_structure``.  The GPU tests read only these
fixtures, never the reference checkout.
"""

import os
import sys

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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
