"""Oracle restatement of the material-parameter interpolation (test infrastructure).

Follows ``code/source/8_band/material_parameters.c:22-1542`` and
``code/source/8_band/interpolate_quaternary.c:23-160``.
"""

import math

from .material_table import BINARY_COLUMNS, BINARY_ROWS, TERNARY_BOWING

HBSQM = 7.61996    # hbar^2/m0 [eV Angstrom^2] (8_band.h:51)
EPS = 1.0e-08      # 8_band.h:59

BINARY_NAMES = ("AlN", "AlP", "AlAs", "AlSb", "AlBi", "GaN", "GaP", "GaAs", "GaSb", "GaBi",
                "InN", "InP", "InAs", "InSb", "InBi")
TERNARY_NAMES = ("AlGaP", "AlGaAs", "AlGaSb", "GaInP", "GaInAs", "GaInSb", "AlInP", "AlInAs",
                 "AlInSb", "AlPAs", "AlPSb", "AlAsSb", "GaPAs", "GaPSb", "GaAsSb", "InPAs",
                 "InPSb", "InAsSb")

# Material systems (material_parameters.c:35-335): (material_type, binaries, ternaries).
# Type 0: A(x)B(1-x)C(y)D(1-y) with binaries (AC, AD, BC, BD), ternaries (ABC, ABD, ACD, BCD).
# Type 1: A(x)B(y)C(1-x-y)D with binaries (AD, BD, CD), ternaries (ABD, ACD, BCD).
# Type 2: AB(x)C(y)D(1-x-y) with binaries (AB, AC, AD), ternaries (ABC, ABD, ACD).
# System 10 uses ternary index 2 for its ACD slot exactly as the reference does
# (material_parameters.c:255-273).
MATERIAL_SYSTEMS = {
    0: (0, (1, 2, 6, 7), (0, 1, 9, 12)),
    1: (0, (1, 3, 6, 8), (0, 2, 10, 13)),
    2: (0, (2, 3, 7, 8), (1, 2, 11, 14)),
    3: (0, (6, 7, 11, 12), (3, 4, 12, 15)),
    4: (0, (6, 8, 11, 13), (3, 5, 13, 16)),
    5: (0, (7, 8, 12, 13), (4, 5, 14, 17)),
    6: (0, (1, 2, 11, 12), (6, 7, 9, 15)),
    7: (0, (1, 3, 11, 13), (6, 8, 10, 16)),
    8: (0, (2, 3, 12, 13), (7, 8, 11, 17)),
    9: (1, (1, 6, 11), (0, 6, 3)),
    10: (1, (2, 7, 12), (1, 2, 4)),
    11: (1, (3, 8, 13), (2, 8, 5)),
    12: (2, (1, 2, 3), (9, 10, 11)),
    13: (2, (6, 7, 8), (12, 13, 14)),
    14: (2, (11, 12, 13), (15, 16, 17)),
}

PARAM_FIELDS = ("a", "C11", "C12", "C44", "e14", "B114", "B124", "B156", "Eg", "Dso", "Ep", "P",
                "sc", "g1", "g2", "g3", "ac", "av", "b", "d", "Ev_avg", "E_so", "E_lh", "E_hh",
                "E_cb", "nr")


def binary_column(name):
    j = BINARY_COLUMNS.index(name)
    return [BINARY_ROWS[b][j] for b in BINARY_NAMES]


def interpolate(bowing, mtype, x, y, P, B=None):
    """interpolate_quaternary.c:23-160.  ``P`` maps slot names (AC, AD, ...) to binary
    values, ``B`` maps (ABC, ABD, ACD, BCD, ABCD) to bowing values."""
    if bowing == 0:
        if mtype == 0:
            return (x * y * P["AC"] + x * (1.0 - y) * P["AD"]
                    + (1.0 - x) * y * P["BC"] + (1.0 - x) * (1.0 - y) * P["BD"])
        if mtype == 1:
            return x * P["AD"] + y * P["BD"] + (1.0 - x - y) * P["CD"]
        return x * P["AB"] + y * P["AC"] + (1.0 - x - y) * P["AD"]
    if mtype == 0:
        if abs(x - 1.0) < EPS and abs(y - 1.0) < EPS:
            return P["AC"]
        if abs(x - 1.0) < EPS and abs(y) < EPS:
            return P["AD"]
        if abs(x) < EPS and abs(y - 1.0) < EPS:
            return P["BC"]
        if abs(x) < EPS and abs(y) < EPS:
            return P["BD"]
        P_ABC = x * P["AC"] + (1.0 - x) * P["BC"] - x * (1.0 - x) * B["ABC"]
        P_ABD = x * P["AD"] + (1.0 - x) * P["BD"] - x * (1.0 - x) * B["ABD"]
        P_ACD = y * P["AC"] + (1.0 - y) * P["AD"] - y * (1.0 - y) * B["ACD"]
        P_BCD = y * P["BC"] + (1.0 - y) * P["BD"] - y * (1.0 - y) * B["BCD"]
        r = (x * (1.0 - x) * (y * P_ABC + (1.0 - y) * P_ABD)
             + y * (1.0 - y) * (x * P_ACD + (1.0 - x) * P_BCD))
        r /= x * (1.0 - x) + y * (1.0 - y)
        r -= x * (1.0 - x) * y * (1.0 - y) * B["ABCD"]
        return r
    if mtype == 1:
        return (x * P["AD"] + y * P["BD"] + (1.0 - x - y) * P["CD"]
                - x * y * B["ABD"] - x * (1.0 - x - y) * B["ACD"] - y * (1.0 - x - y) * B["BCD"]
                - x * y * (1.0 - x - y) * B["ABCD"])
    return (x * P["AB"] + y * P["AC"] + (1.0 - x - y) * P["AD"]
            - x * y * B["ABC"] - x * (1.0 - x - y) * B["ABD"] - y * (1.0 - x - y) * B["ACD"]
            - x * y * (1.0 - x - y) * B["ABCD"])


BIN_SLOTS = {0: ("AC", "AD", "BC", "BD"), 1: ("AD", "BD", "CD"), 2: ("AB", "AC", "AD")}
TERN_SLOTS = {0: ("ABC", "ABD", "ACD", "BCD"), 1: ("ABD", "ACD", "BCD"), 2: ("ABC", "ABD", "ACD")}


def material_parameters(T, geo, include_piezo):
    """material_parameters.c:22-1542.  Returns one parameter dict per shape and sets
    ``material_type`` in ``geo``."""
    for g in geo:
        if g["material"] not in MATERIAL_SYSTEMS:
            raise ValueError("Requested material system not recognised")
        g["material_type"] = MATERIAL_SYSTEMS[g["material"]][0]

    col = {c: binary_column(c) for c in BINARY_COLUMNS}
    # Modified band parameters from T = 0 gaps (material_parameters.c:360-372)
    Eg0, Dso, Ep, mc = col["Eg"], col["Dso"], col["Ep"], col["mc"]
    sc = [1.0 / mc[i] - (Ep[i] / 3.0) * (2.0 / Eg0[i] + 1.0 / (Eg0[i] + Dso[i])) for i in range(15)]
    g1 = [col["gL1"][i] - Ep[i] / (3.0 * Eg0[i] + Dso[i]) for i in range(15)]
    g2 = [col["gL2"][i] - Ep[i] / (6.0 * Eg0[i] + 2.0 * Dso[i]) for i in range(15)]
    g3 = [col["gL3"][i] - Ep[i] / (6.0 * Eg0[i] + 2.0 * Dso[i]) for i in range(15)]
    # Varshni band gaps (material_parameters.c:378-392)
    Eg = list(Eg0)
    for i in range(15):
        alpha = col["alpha_T"][i] * 0.001
        if T > 0.001:
            if i != 6:
                Eg[i] -= (alpha * T * T) / (T + col["beta_T"][i])
            else:
                Eg[i] += 0.1081 * (1.0 - (math.cosh(164.0 / T) / math.sinh(164.0 / T)))
    tables = dict(col)
    tables.update(sc=sc, g1=g1, g2=g2, g3=g3, Eg=Eg)
    tables["e14_used"] = col["e14"] if include_piezo == 1 else col["e14_calc"]  # :604-646

    def lin(name, g):
        mtype, bins, _ = MATERIAL_SYSTEMS[g["material"]]
        P = {s: tables[name][b] for s, b in zip(BIN_SLOTS[mtype], bins)}
        return interpolate(0, mtype, g["x"], g["y"], P)

    params = []
    for g in geo:
        p = {}
        for name, src in (("a", "a"), ("C11", "C11"), ("C12", "C12"), ("C44", "C44"),
                          ("e14", "e14_used"), ("B114", "B114"), ("B124", "B124"),
                          ("B156", "B156"), ("ac", "ac"), ("av", "av"), ("b", "b"), ("d", "d"),
                          ("nr", "nr")):
            p[name] = lin(src, g)
        params.append(p)

    # Ternary Ev_avg bowing referenced to the matrix lattice constant (material_parameters.c:1060-1081)
    a, av = col["a"], col["av"]
    pairs = ((1, 6), (2, 7), (3, 8), (6, 11), (7, 12), (8, 13), (1, 11), (2, 12), (3, 13),
             (1, 2), (1, 3), (2, 3), (6, 7), (6, 8), (7, 8), (11, 12), (11, 13), (12, 13))
    bow_Ev = [(3.0 / params[0]["a"]) * (av[i] - av[j]) * (a[i] - a[j]) for i, j in pairs]
    bow_Eg = [TERNARY_BOWING[t][0] for t in TERNARY_NAMES]
    bow_Dso = [TERNARY_BOWING[t][1] for t in TERNARY_NAMES]

    def bow(name, bowtab, g):
        mtype, bins, terns = MATERIAL_SYSTEMS[g["material"]]
        P = {s: tables[name][b] for s, b in zip(BIN_SLOTS[mtype], bins)}
        B = {s: bowtab[t] for s, t in zip(TERN_SLOTS[mtype], terns)}
        B["ABCD"] = 0.0  # all quaternary bowing parameters are zero
        return interpolate(1, mtype, g["x"], g["y"], P, B)

    for g, p in zip(geo, params):
        p["Ev_avg"] = bow("Ev_avg", bow_Ev, g)
        p["Eg"] = bow("Eg", bow_Eg, g)
        p["Dso"] = bow("Dso", bow_Dso, g)
        p["sc"] = lin("sc", g)
        p["Ep"] = lin("Ep", g)
        p["P"] = math.sqrt(0.5 * HBSQM * p["Ep"])  # :1384
        p["g1"] = lin("g1", g)
        p["g2"] = lin("g2", g)
        p["g3"] = lin("g3", g)
    # Band edges, zero at the matrix VB edge (material_parameters.c:1529-1538)
    ref = params[0]["Ev_avg"] + params[0]["Dso"] / 3.0
    for p in params:
        p["E_hh"] = p["Ev_avg"] + p["Dso"] / 3.0 - ref
        p["E_so"] = p["E_hh"] - p["Dso"]
        p["E_lh"] = p["E_hh"]
        p["E_cb"] = p["E_hh"] + p["Eg"]
    return params
