"""Oracle restatement of the input readers (test infrastructure).

``parameters.in`` and ``supercell.in`` are flat YAML ``Key: value`` files.
The reference reads them with libyaml scalar events
(``code/source/8_band/read_parameters.c:26-509``,
``code/source/8_band/read_supercell.c:23-367``); this module restates the same
key handling and unit conversions with a line parser.
"""

import copy

# Keys of parameters.in in the order of the reference's input_check slots
# (read_parameters.c:111-505).  "Softening" and "Sigma_softening" are optional.
PARAMETER_KEYS = (
    "N_shape", "M_Gx", "M_Gy", "M_Gz", "Strain_supercell_type", "M_S_Gx", "M_S_Gy", "M_S_Gz",
    "N_VB", "N_CB", "T", "Fx", "Fy", "Fz", "Kx", "Ky", "Kz", "N_line", "Strain", "Isotropic",
    "Elastic_const", "Elastic_const_order", "Piezo", "Overlaps", "Localisation", "MME", "CME",
    "Coulomb_supercell_type", "M_C_Gx", "M_C_Gy", "M_C_Gz", "Softening", "Sigma_softening",
    "Linescan_100", "Linescan_010", "Linescan_001", "Linescan_110", "Linescan_101", "Linescan_011",
    "Linescan_111", "Cross_sections", "N_cross", "Cross_section_100", "Cross_section_010",
    "Cross_section_001", "Cross_section_m110", "Cross_section_110", "Cross_section_m101",
    "Cross_section_0m11", "Cross_section_111", "3D_output", "N_3D", "Eigensolver",
)
OPTIONAL_KEYS = ("Softening", "Sigma_softening")


class InputError(ValueError):
    pass


def scalar_pairs(text):
    """Yield (key, value) scalar pairs of a flat YAML mapping, in file order."""
    for raw in text.splitlines():
        line = raw
        # YAML comment: '#' at line start or preceded by whitespace
        for i, ch in enumerate(line):
            if ch == "#" and (i == 0 or line[i - 1] in " \t"):
                line = line[:i]
                break
        line = line.strip()
        if not line:
            continue
        if ":" not in line:
            raise InputError("malformed line (no ':'): %r" % raw)
        key, value = line.split(":", 1)
        yield key.strip(), value.strip()


def _int(v):
    return int(v.strip().split()[0], 10) if v.strip() else 0


def _float(v):
    return float(v)


def convert_parameter(p, key, value):
    """Apply one key (read_parameters.c:111-505; read_command_line_input.c:37-46)."""
    if key == "N_shape":
        p["N_shape"] = _int(value)
    elif key in ("M_Gx", "M_Gy", "M_Gz", "M_S_Gx", "M_S_Gy", "M_S_Gz", "M_C_Gx", "M_C_Gy", "M_C_Gz"):
        p["N" + key[1:]] = 2 * _int(value) + 1  # N = 2*M + 1 (read_parameters.c:126)
    elif key in ("Fx", "Fy", "Fz"):
        p[key] = 1.0e-05 * _float(value)  # kV/cm -> V/Angstrom (read_parameters.c:193-211)
    elif key in ("Kx", "Ky", "Kz"):
        p[key] = 0.1 * _float(value)  # nm^-1 -> Angstrom^-1
    elif key == "T":
        p["T"] = _float(value)
    elif key == "Sigma_softening":
        p["Sigma_softening"] = 10.0 * _float(value)  # nm -> Angstrom
    elif key in PARAMETER_KEYS:
        p[key] = _int(value)
    else:
        return False
    return True


def read_parameters(text, overrides=()):
    """Parse parameters.in text; ``overrides`` are CLI ``-Key=value`` strings."""
    p = {"Softening": 0, "Sigma_softening": 0.0}
    seen = set(OPTIONAL_KEYS)
    for key, value in scalar_pairs(text):
        if convert_parameter(p, key, value):
            seen.add(key)
    for arg in overrides:
        if not arg.startswith("-") or "=" not in arg:
            raise InputError("bad override %r" % arg)
        key, value = arg[1:].split("=", 1)
        if convert_parameter(p, key, value):
            seen.add(key)
    missing = [k for k in PARAMETER_KEYS if k not in seen]
    if missing:
        raise InputError("missing parameters: %s" % ", ".join(missing))
    return p


GEOMETRY_FIELDS = ("shape", "embedded", "material", "material_type", "RL1", "RL2", "RL3",
                   "RCL1", "RCL2", "RCL3", "x", "y", "Ox", "Oy", "Oz", "L1", "L2", "L3", "L4", "L5",
                   "SL1", "SL2", "SL3", "CL1", "CL2", "CL3", "alpha", "beta", "gamma")


def empty_geometry():
    g = {k: 0 for k in GEOMETRY_FIELDS}
    for k in ("x", "y", "Ox", "Oy", "Oz", "L1", "L2", "L3", "L4", "L5", "SL1", "SL2", "SL3",
              "CL1", "CL2", "CL3", "alpha", "beta", "gamma"):
        g[k] = 0.0
    return g


def read_supercell(text, n_shape, strain_region_type, coulomb_region_type):
    """Parse supercell.in (read_supercell.c:23-367).

    Record 0 (the supercell) ends at "Coulomb length 3"; every later shape record
    ends at "Euler gamma angle".  Lengths and centres are converted nm -> Angstrom.
    """
    geo = [empty_geometry() for _ in range(n_shape)]
    idx = 0
    for key, value in scalar_pairs(text):
        if idx >= n_shape:
            raise InputError("N_shape is less than the number of shapes given in supercell.in")
        g = geo[idx]
        if key == "Embedded":
            g["embedded"] = _int(value)
        elif key == "QD shape":
            g["shape"] = _int(value)
        elif key == "Material":
            g["material"] = _int(value)
        elif key == "Compos x":
            g["x"] = _float(value)
        elif key == "Compos y":
            g["y"] = _float(value)
        elif key in ("Centre x", "Centre y", "Centre z"):
            g["O" + key[-1]] = 10 * _float(value)
        elif key.startswith("Length "):
            g["L" + key[-1]] = 10 * _float(value)
        elif key.startswith("Strain length "):
            a = key[-1]
            if strain_region_type == 0:
                g["SL" + a] = 10 * _float(value)
            else:
                g["RL" + a] = _int(value)
                g["SL" + a] = g["L" + a] * g["RL" + a]
        elif key.startswith("Coulomb length "):
            a = key[-1]
            if coulomb_region_type == 0:
                g["CL" + a] = 10 * _float(value)
            else:
                g["RCL" + a] = _int(value)
                g["CL" + a] = g["L" + a] * g["RCL" + a]
            if a == "3":
                idx += 1
        elif key == "Euler alpha angle":
            g["alpha"] = _float(value)
        elif key == "Euler beta angle":
            g["beta"] = _float(value)
        elif key == "Euler gamma angle":
            g["gamma"] = _float(value)
            idx += 1
    if idx < n_shape:
        raise InputError("N_shape is greater than the number of shapes given in supercell.in")
    return geo


def effective_strain_region_type(p, geo):
    """8_band_main.c:195-200: a commensurate strain cell of relative size 1 with the
    same plane-wave counts is treated as the free-length (direct copy) case."""
    t = p["Strain_supercell_type"]
    g0 = geo[0]
    if (t == 1 and g0["RL1"] == 1 and g0["RL2"] == 1 and g0["RL3"] == 1
            and p["N_Gx"] == p["N_S_Gx"] and p["N_Gy"] == p["N_S_Gy"] and p["N_Gz"] == p["N_S_Gz"]):
        return 0
    return t


def load(directory, overrides=()):
    """Read ``parameters.in`` and ``supercell.in`` from ``directory``."""
    import os
    with open(os.path.join(directory, "parameters.in")) as f:
        p = read_parameters(f.read(), overrides)
    with open(os.path.join(directory, "supercell.in")) as f:
        geo = read_supercell(f.read(), p["N_shape"], p["Strain_supercell_type"], p["Coulomb_supercell_type"])
    return p, geo


def clone(geo):
    return copy.deepcopy(geo)
