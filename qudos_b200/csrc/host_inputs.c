/* Host side of the solve path: input readers, plane-wave grids and material
 * parameters.
 *
 *  - parameters.in / supercell.in are flat YAML "Key: value" files; the
 *    reference reads them with libyaml scalar events
 *    (code/source/8_band/read_parameters.c:26-509,
 *    read_command_line_input.c:23-513, read_supercell.c:23-367).  This reader
 *    keeps the same keys, units and record structure with a line parser.
 *  - basis grids follow basis_set.c:23-90.
 *  - material parameters follow material_parameters.c:22-1542 and
 *    interpolate_quaternary.c:23-160.
 */
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "qd_internal.h"

/* ---------------------------------------------------------------------- */
/* parameters.in                                                           */
/* ---------------------------------------------------------------------- */
enum { NKEYS = 53 };
static const char *const key_names[NKEYS] = {
    "N_shape", "M_Gx", "M_Gy", "M_Gz", "Strain_supercell_type", "M_S_Gx", "M_S_Gy", "M_S_Gz",
    "N_VB", "N_CB", "T", "Fx", "Fy", "Fz", "Kx", "Ky", "Kz", "N_line", "Strain", "Isotropic",
    "Elastic_const", "Elastic_const_order", "Piezo", "Overlaps", "Localisation", "MME", "CME",
    "Coulomb_supercell_type", "M_C_Gx", "M_C_Gy", "M_C_Gz", "Softening", "Sigma_softening",
    "Linescan_100", "Linescan_010", "Linescan_001", "Linescan_110", "Linescan_101", "Linescan_011",
    "Linescan_111", "Cross_sections", "N_cross", "Cross_section_100", "Cross_section_010",
    "Cross_section_001", "Cross_section_m110", "Cross_section_110", "Cross_section_m101",
    "Cross_section_0m11", "Cross_section_111", "3D_output", "N_3D", "Eigensolver"};

static int key_index(const char *k) {
    for (int i = 0; i < NKEYS; i++)
        if (strcmp(k, key_names[i]) == 0) return i;
    return -1;
}

static char *trim(char *s) {
    while (*s && isspace((unsigned char)*s)) s++;
    char *e = s + strlen(s);
    while (e > s && isspace((unsigned char)e[-1])) *--e = 0;
    return s;
}

/* Returns key index, or -1 for an unknown key (ignored, as by the reference). */
static int apply_key(qd_params *p, const char *key, const char *value, int *err) {
    int k = key_index(key);
    char *end = NULL;
    long iv = strtol(value, &end, 10);
    double dv = strtod(value, &end);
    *err = 0;
    switch (k) {
        case 0: p->n_shape = (int)iv; break;
        case 1: p->N[0] = 2 * (int)iv + 1; break;  /* N = 2 M + 1 (read_parameters.c:126) */
        case 2: p->N[1] = 2 * (int)iv + 1; break;
        case 3: p->N[2] = 2 * (int)iv + 1; break;
        case 4: p->strain_type = (int)iv; break;
        case 5: p->NS[0] = 2 * (int)iv + 1; break;
        case 6: p->NS[1] = 2 * (int)iv + 1; break;
        case 7: p->NS[2] = 2 * (int)iv + 1; break;
        case 8: p->n_vb = (int)iv; break;
        case 9: p->n_cb = (int)iv; break;
        case 10: p->T = dv; break;
        case 11: p->F[0] = 1.0e-05 * dv; break;    /* kV/cm -> V/Angstrom (read_parameters.c:193-211) */
        case 12: p->F[1] = 1.0e-05 * dv; break;
        case 13: p->F[2] = 1.0e-05 * dv; break;
        case 14: p->K[0] = 0.1 * dv; break;        /* nm^-1 -> Angstrom^-1 */
        case 15: p->K[1] = 0.1 * dv; break;
        case 16: p->K[2] = 0.1 * dv; break;
        case 18: p->strain = (int)iv; break;
        case 19: p->isotropic = (int)iv; break;
        case 20: p->elastic_const = (int)iv; break;
        case 21: p->elastic_order = (int)iv; break;
        case 22: p->piezo = (int)iv; break;
        case 26: p->cme = (int)iv; break;
        case 27: p->coulomb_type = (int)iv; break;
        case 28: p->NC[0] = 2 * (int)iv + 1; break;
        case 29: p->NC[1] = 2 * (int)iv + 1; break;
        case 30: p->NC[2] = 2 * (int)iv + 1; break;
        case 31: p->softening = (int)iv; break;
        case 32: p->sigma = 10.0 * dv; break;      /* nm -> Angstrom */
        case 52: p->eigensolver = (int)iv; break;
        default: break;                            /* output-only keys: accepted, unused here */
    }
    if (k >= 0 && value[0] == 0) *err = 1;
    return k;
}

/* Iterate "key: value" lines; calls fn for each pair.  '#' starts a comment at
 * line start or after whitespace (YAML rule). */
typedef int (*pair_fn)(void *ctx, const char *key, const char *value);

static int for_each_pair(const char *text, pair_fn fn, void *ctx) {
    const char *s = text;
    char line[1024];
    while (*s) {
        size_t n = strcspn(s, "\n");
        if (n >= sizeof(line)) return qd_set_error(QD_ERR_INPUT, "input line too long");
        memcpy(line, s, n);
        line[n] = 0;
        s += n + (s[n] == '\n');
        for (size_t i = 0; line[i]; i++)
            if (line[i] == '#' && (i == 0 || line[i - 1] == ' ' || line[i - 1] == '\t')) {
                line[i] = 0;
                break;
            }
        char *t = trim(line);
        if (!*t) continue;
        char *colon = strchr(t, ':');
        if (!colon) return qd_set_error(QD_ERR_INPUT, "malformed input line (no ':'): %s", t);
        *colon = 0;
        int rc = fn(ctx, trim(t), trim(colon + 1));
        if (rc) return rc;
    }
    return QD_OK;
}

struct param_ctx { qd_params *p; int seen[NKEYS]; };

static int param_pair(void *vctx, const char *key, const char *value) {
    struct param_ctx *c = (struct param_ctx *)vctx;
    int err = 0;
    int k = apply_key(c->p, key, value, &err);
    if (err) return qd_set_error(QD_ERR_INPUT, "empty value for parameter %s", key);
    if (k >= 0) c->seen[k] = 1;
    return QD_OK;
}

int qd_read_parameters_text(const char *text, qd_params *p, int *seen_all) {
    struct param_ctx c;
    memset(&c, 0, sizeof(c));
    memset(p, 0, sizeof(*p));
    c.p = p;
    c.seen[31] = c.seen[32] = 1; /* Softening / Sigma_softening are optional (read_parameters.c:71-74) */
    int rc = for_each_pair(text, param_pair, &c);
    if (rc) return rc;
    for (int k = 0; k < NKEYS; k++)
        if (!c.seen[k]) {
            if (seen_all) *seen_all = 0;
            return qd_set_error(QD_ERR_INPUT, "parameters.in: missing parameter %s", key_names[k]);
        }
    if (seen_all) *seen_all = 1;
    return QD_OK;
}

int qd_apply_override(qd_params *p, const char *arg) {
    /* read_command_line_input.c:37-46: "-Key=value" */
    char buf[256];
    if (!arg || arg[0] != '-' || strlen(arg) >= sizeof(buf))
        return qd_set_error(QD_ERR_INPUT, "bad command-line override: %s", arg ? arg : "(null)");
    strcpy(buf, arg + 1);
    char *eq = strchr(buf, '=');
    if (!eq) return qd_set_error(QD_ERR_INPUT, "bad command-line override: %s", arg);
    *eq = 0;
    int err = 0;
    apply_key(p, buf, eq + 1, &err);
    if (err) return qd_set_error(QD_ERR_INPUT, "empty override value: %s", arg);
    return QD_OK;
}

/* ---------------------------------------------------------------------- */
/* supercell.in                                                            */
/* ---------------------------------------------------------------------- */
struct cell_ctx {
    const qd_params *p;
    struct supercell_geometry *geo;
    int idx;
};

static int cell_pair(void *vctx, const char *key, const char *value) {
    struct cell_ctx *c = (struct cell_ctx *)vctx;
    if (c->idx >= c->p->n_shape)
        return qd_set_error(QD_ERR_INPUT,
                            "The parameter 'N_shape' is less than the number of shapes given in supercell.in");
    struct supercell_geometry *g = &c->geo[c->idx];
    char *end;
    double dv = strtod(value, &end);
    int iv = (int)strtol(value, &end, 10);
    if (!strcmp(key, "Embedded")) g->embedded = iv;
    else if (!strcmp(key, "QD shape")) g->shape = iv;
    else if (!strcmp(key, "Material")) g->material = iv;
    else if (!strcmp(key, "Compos x")) g->x = dv;
    else if (!strcmp(key, "Compos y")) g->y = dv;
    else if (!strcmp(key, "Centre x")) g->Ox = 10 * dv;   /* nm -> Angstrom (read_supercell.c:162-204) */
    else if (!strcmp(key, "Centre y")) g->Oy = 10 * dv;
    else if (!strcmp(key, "Centre z")) g->Oz = 10 * dv;
    else if (!strcmp(key, "Length 1")) g->L1 = 10 * dv;
    else if (!strcmp(key, "Length 2")) g->L2 = 10 * dv;
    else if (!strcmp(key, "Length 3")) g->L3 = 10 * dv;
    else if (!strcmp(key, "Length 4")) g->L4 = 10 * dv;
    else if (!strcmp(key, "Length 5")) g->L5 = 10 * dv;
    else if (!strncmp(key, "Strain length ", 14)) {
        int a = key[14] - '1';
        double *SL = a == 0 ? &g->SL1 : a == 1 ? &g->SL2 : &g->SL3;
        int *RL = a == 0 ? &g->RL1 : a == 1 ? &g->RL2 : &g->RL3;
        double L = a == 0 ? g->L1 : a == 1 ? g->L2 : g->L3;
        if (c->p->strain_type == 0) *SL = 10 * dv;
        else { *RL = iv; *SL = L * (*RL); }
    } else if (!strncmp(key, "Coulomb length ", 15)) {
        int a = key[15] - '1';
        double *CL = a == 0 ? &g->CL1 : a == 1 ? &g->CL2 : &g->CL3;
        int *RCL = a == 0 ? &g->RCL1 : a == 1 ? &g->RCL2 : &g->RCL3;
        double L = a == 0 ? g->L1 : a == 1 ? g->L2 : g->L3;
        if (c->p->coulomb_type == 0) *CL = 10 * dv;
        else { *RCL = iv; *CL = L * (*RCL); }
        if (a == 2) c->idx++;  /* record 0 ends at "Coulomb length 3" */
    } else if (!strcmp(key, "Euler alpha angle")) g->alpha = dv;
    else if (!strcmp(key, "Euler beta angle")) g->beta = dv;
    else if (!strcmp(key, "Euler gamma angle")) {
        g->gamma = dv;
        c->idx++;  /* shape records end at "Euler gamma angle" */
    }
    return QD_OK;
}

int qd_read_supercell_text(const char *text, const qd_params *p, struct supercell_geometry *geo) {
    memset(geo, 0, sizeof(*geo) * (size_t)p->n_shape);
    struct cell_ctx c = {p, geo, 0};
    int rc = for_each_pair(text, cell_pair, &c);
    if (rc) return rc;
    if (c.idx < p->n_shape)
        return qd_set_error(QD_ERR_INPUT,
                            "The parameter 'N_shape' is greater than the number of shapes given in supercell.in");
    return QD_OK;
}

/* ---------------------------------------------------------------------- */
/* basis grids                                                             */
/* ---------------------------------------------------------------------- */
void qd_basis_grid(int n_T, double L, double *out) {
    for (int i = 0; i < n_T; i++) out[i] = ((2.0 * M_PI) / L) * (0.5 * (1.0 - (double)n_T) + (double)i);
}

/* ---------------------------------------------------------------------- */
/* material parameters                                                     */
/* ---------------------------------------------------------------------- */
#define QD_N_BINARY 15
#define QD_N_BINARY_COLS 24
#define QD_N_TERNARY 18
/* Published III-V parameters (Vurgaftman, Meyer, Ram-Mohan, J. Appl. Phys. 89,
 * 5815 (2001); piezoelectric coefficients from Caro, Schulz, O'Reilly, PRB 91,
 * 075203 (2015)): the values of the reference's material_parameters.h, one row
 * per binary compound.  Columns: a C11 C12 C44 e14 e14_calc B114 B124 B156 ac
 * av b d Ev_avg Eg Dso mc Ep gL1 gL2 gL3 nr alpha_T beta_T. */
enum { C_a, C_C11, C_C12, C_C44, C_e14, C_e14c, C_B114, C_B124, C_B156, C_ac, C_av, C_b, C_d, C_Ev,
       C_Eg, C_Dso, C_mc, C_Ep, C_gL1, C_gL2, C_gL3, C_nr, C_aT, C_bT };
static const double qd_binary_rows[QD_N_BINARY][QD_N_BINARY_COLS] = {
    /* AlN  */ {4.38, 304.0, 160.0, 193.0, 0.548, 0.548, -6.81, -5.04, -4.15, -6.0, 3.4, -1.9, -10.0, -2.64, 4.9, 0.019, 0.25, 27.1, 1.92, 0.47, 0.85, 2.16, 0.593, 600.0},
    /* AlP  */ {5.4672, 133.0, 63.0, 61.5, 0.014, 0.014, -2.02, -2.76, -1.43, -5.7, 3.0, -1.5, -4.6, -0.94, 3.63, 0.07, 0.22, 17.7, 3.35, 0.71, 1.23, 2.75, 0.5771, 372.0},
    /* AlAs */ {5.6611, 125.0, 53.4, 54.2, -0.055, -0.055, -1.61, -2.59, -1.32, -5.64, 2.47, -2.3, -3.4, -0.53, 3.099, 0.28, 0.15, 21.1, 3.76, 0.82, 1.42, 3.0, 0.885, 530.0},
    /* AlSb */ {6.1355, 87.69, 43.41, 40.76, -0.094, -0.094, -0.76, -1.99, -0.82, -4.5, 1.4, -1.35, -4.3, 0.39, 2.386, 0.676, 0.14, 18.7, 5.18, 1.19, 1.97, 3.19, 0.42, 140.0},
    /* AlBi */ {6.3417, 72.2, 36.2, 33.4, -0.094, -0.094, -0.76, -1.99, -0.82, -4.5, 1.4, -1.35, -4.3, 1.1, 0.042, 2.124, 99.999, 99.999, 99.999, 99.999, 99.999, 3.19, 0.42, 140.0},
    /* GaN  */ {4.5, 293.0, 159.0, 155.0, 0.366, 0.366, -5.38, -6.73, -3.18, -2.2, 5.2, -2.2, -3.4, -1.84, 3.299, 0.017, 0.15, 25.0, 2.67, 0.75, 1.1, 2.4, 0.593, 600.0},
    /* GaP  */ {5.4505, 140.5, 62.03, 70.33, -0.121, -0.121, -1.23, -3.27, -1.38, -8.2, 1.7, -1.6, -4.6, -0.47, 2.886, 0.08, 0.13, 31.4, 4.05, 0.49, 2.93, 2.9, 0.0, 0.0},
    /* GaAs */ {5.6503, 118.8, 53.8, 59.4, -0.16, -0.23, -0.439, -3.765, -0.492, -8.013, 0.22, -1.824, -5.062, 0.0, 1.518, 0.34, 0.0667, 25.7, 7.1, 2.02, 2.91, 3.6304, 0.5405, 204.0},
    /* GaSb */ {6.0959, 88.42, 40.26, 43.22, -0.216, -0.216, -0.31, -2.77, -0.7, -7.5, 0.8, -2.0, -4.7, 0.77, 0.812, 0.76, 0.039, 27.0, 13.4, 4.7, 6.0, 3.79, 0.417, 140.0},
    /* GaBi */ {6.324, 73.0, 32.7, 36.3, -0.216, -0.216, -0.31, -2.77, -0.7, -7.5, 0.8, -2.0, -4.7, 1.1, -1.45, 2.15, 99.999, 99.999, 99.999, 99.999, 99.999, 3.79, 0.417, 140.0},
    /* InN  */ {4.98, 187.0, 125.0, 86.0, 0.593, 0.593, -5.96, -6.32, -2.0, -1.85, 1.5, -1.2, -9.3, -1.58, 1.94, 0.006, 0.12, 25.0, 3.72, 1.26, 1.63, 2.59, 0.245, 624.0},
    /* InP  */ {5.8697, 101.1, 56.1, 45.6, 0.016, 0.016, -1.54, -3.62, -1.02, -6.0, 0.6, -2.0, -5.0, -0.14, 1.424, 0.108, 0.0795, 20.7, 5.08, 1.6, 2.1, 3.1, 0.363, 162.0},
    /* InAs */ {6.0553, 83.3, 45.3, 39.6, -0.045, -0.115, -0.531, -4.076, -0.12, -5.08, 1.0, -1.8, -3.6, 0.173, 0.405, 0.38, 0.02226, 21.846, 19.67, 8.4, 9.3, 3.821, 0.276, 93.0},
    /* InSb */ {6.4794, 68.47, 37.35, 31.11, -0.161, -0.161, -0.62, -4.04, -0.16, -6.94, 0.36, -2.0, -4.7, 0.8, 0.235, 0.81, 0.0135, 23.3, 34.8, 15.0, 16.5, 3.95, 0.42, 170.0},
    /* InBi */ {6.686, 58.5, 30.4, 27.5, -0.161, -0.161, -0.62, -4.04, -0.16, -6.94, 0.36, -2.0, -4.7, 1.1, -1.63, 2.15, 99.999, 99.999, 99.999, 99.999, 99.999, 3.95, 0.42, 170.0},
};
static const double qd_ternary_bowing[QD_N_TERNARY][2] = {
    /* AlGaP  */ {0.0, 0.0},
    /* AlGaAs */ {0.528, 0.0},
    /* AlGaSb */ {0.566, 0.3},
    /* GaInP  */ {0.65, 0.0},
    /* GaInAs */ {0.477, 0.15},
    /* GaInSb */ {0.415, 0.1},
    /* AlInP  */ {-0.48, -0.19},
    /* AlInAs */ {0.7, 0.15},
    /* AlInSb */ {0.43, 0.25},
    /* AlPAs  */ {0.22, 0.0},
    /* AlPSb  */ {2.7, 0.0},
    /* AlAsSb */ {0.8, 0.15},
    /* GaPAs  */ {0.19, 0.0},
    /* GaPSb  */ {2.7, 0.0},
    /* GaAsSb */ {1.43, 0.6},
    /* InPAs  */ {0.1, 0.16},
    /* InPSb  */ {1.9, 0.75},
    /* InAsSb */ {0.67, 1.2},
};

/* Material systems (material_parameters.c:35-335): type, binaries, ternaries.
 * Type 0 A(x)B(1-x)C(y)D(1-y): binaries AC AD BC BD, ternaries ABC ABD ACD BCD.
 * Type 1 A(x)B(y)C(1-x-y)D: binaries AD BD CD, ternaries ABD ACD BCD.
 * Type 2 AB(x)C(y)D(1-x-y): binaries AB AC AD, ternaries ABC ABD ACD.
 * System 10 keeps the reference's ternary index 2 in its ACD slot
 * (material_parameters.c:255-273). */
static const int sys_type[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 2, 2, 2};
static const int sys_bin[15][4] = {{1, 2, 6, 7}, {1, 3, 6, 8}, {2, 3, 7, 8}, {6, 7, 11, 12},
                                   {6, 8, 11, 13}, {7, 8, 12, 13}, {1, 2, 11, 12}, {1, 3, 11, 13},
                                   {2, 3, 12, 13}, {1, 6, 11, -1}, {2, 7, 12, -1}, {3, 8, 13, -1},
                                   {1, 2, 3, -1}, {6, 7, 8, -1}, {11, 12, 13, -1}};
static const int sys_tern[15][4] = {{0, 1, 9, 12}, {0, 2, 10, 13}, {1, 2, 11, 14}, {3, 4, 12, 15},
                                    {3, 5, 13, 16}, {4, 5, 14, 17}, {6, 7, 9, 15}, {6, 8, 10, 16},
                                    {7, 8, 11, 17}, {0, 6, 3, -1}, {1, 2, 4, -1}, {2, 8, 5, -1},
                                    {9, 10, 11, -1}, {12, 13, 14, -1}, {15, 16, 17, -1}};

/* interpolate_quaternary.c:23-160.  P[] are the binary values in the system's
 * slot order, B[] the ternary bowings in slot order (quaternary bowing is 0). */
static double interp(int bowing, int type, double x, double y, const double P[4], const double B[4]) {
    const double eps = QD_EPS;
    if (bowing == 0) {
        if (type == 0)
            return x * y * P[0] + x * (1.0 - y) * P[1] + (1.0 - x) * y * P[2] +
                   (1.0 - x) * (1.0 - y) * P[3];
        return x * P[0] + y * P[1] + (1.0 - x - y) * P[2];
    }
    if (type == 0) {
        if (fabs(x - 1.0) < eps && fabs(y - 1.0) < eps) return P[0];
        if (fabs(x - 1.0) < eps && fabs(y) < eps) return P[1];
        if (fabs(x) < eps && fabs(y - 1.0) < eps) return P[2];
        if (fabs(x) < eps && fabs(y) < eps) return P[3];
        double P_ABC = x * P[0] + (1.0 - x) * P[2] - x * (1.0 - x) * B[0];
        double P_ABD = x * P[1] + (1.0 - x) * P[3] - x * (1.0 - x) * B[1];
        double P_ACD = y * P[0] + (1.0 - y) * P[1] - y * (1.0 - y) * B[2];
        double P_BCD = y * P[2] + (1.0 - y) * P[3] - y * (1.0 - y) * B[3];
        double r = x * (1.0 - x) * (y * P_ABC + (1.0 - y) * P_ABD) +
                   y * (1.0 - y) * (x * P_ACD + (1.0 - x) * P_BCD);
        r /= x * (1.0 - x) + y * (1.0 - y);
        return r;
    }
    /* types 1 and 2 share the form with their own slot meaning */
    return x * P[0] + y * P[1] + (1.0 - x - y) * P[2] - x * y * B[0] - x * (1.0 - x - y) * B[1] -
           y * (1.0 - x - y) * B[2];
}

/* Scale factors applied to the Ep and Luttinger gamma_1 columns of the binary
 * table before interpolation (1 = the table as published); the gradient
 * entry point differentiates with respect to them. */
double qd_scale_Ep = 1.0, qd_scale_gL1 = 1.0;

int qd_material_parameters(double T, int include_piezo, int n_shape, struct supercell_geometry *geo,
                           struct material_params *out) {
    double col[QD_N_BINARY_COLS][QD_N_BINARY];
    for (int i = 0; i < QD_N_BINARY; i++)
        for (int c = 0; c < QD_N_BINARY_COLS; c++) col[c][i] = qd_binary_rows[i][c];
    for (int i = 0; i < QD_N_BINARY; i++) {
        col[C_Ep][i] *= qd_scale_Ep;
        col[C_gL1][i] *= qd_scale_gL1;
    }
    for (int s = 0; s < n_shape; s++) {
        if (geo[s].material < 0 || geo[s].material > 14)
            return qd_set_error(QD_ERR_INPUT, "Requested material system not recognised");
        geo[s].material_type = sys_type[geo[s].material];
    }
    /* modified band parameters from the T = 0 gaps (material_parameters.c:360-372) */
    double sc[QD_N_BINARY], g1[QD_N_BINARY], g2[QD_N_BINARY], g3[QD_N_BINARY], Eg[QD_N_BINARY];
    for (int i = 0; i < QD_N_BINARY; i++) {
        double Eg0 = col[C_Eg][i], Dso = col[C_Dso][i], Ep = col[C_Ep][i];
        sc[i] = 1.0 / col[C_mc][i] - (Ep / 3.0) * (2.0 / Eg0 + 1.0 / (Eg0 + Dso));
        g1[i] = col[C_gL1][i] - Ep / (3.0 * Eg0 + Dso);
        g2[i] = col[C_gL2][i] - Ep / (6.0 * Eg0 + 2.0 * Dso);
        g3[i] = col[C_gL3][i] - Ep / (6.0 * Eg0 + 2.0 * Dso);
        /* Varshni (material_parameters.c:378-392) */
        double alpha = col[C_aT][i] * 0.001;
        Eg[i] = Eg0;
        if (T > 0.001) {
            if (i != 6) Eg[i] -= (alpha * T * T) / (T + col[C_bT][i]);
            else Eg[i] += 0.1081 * (1.0 - (cosh(164.0 / T) / sinh(164.0 / T)));
        }
    }
    const double *e14 = include_piezo == 1 ? col[C_e14] : col[C_e14c]; /* :604-646 */
    double P[4], B[4] = {0, 0, 0, 0};
#define LIN(dst, arr)                                                                             \
    do {                                                                                          \
        for (int q = 0; q < 4; q++) P[q] = sys_bin[m][q] >= 0 ? (arr)[sys_bin[m][q]] : 0.0;       \
        (dst) = interp(0, t, g->x, g->y, P, B);                                                   \
    } while (0)
    for (int s = 0; s < n_shape; s++) {
        struct supercell_geometry *g = &geo[s];
        struct material_params *o = &out[s];
        int m = g->material, t = sys_type[m];
        memset(o, 0, sizeof(*o));
        LIN(o->a, col[C_a]);
        LIN(o->C11, col[C_C11]);
        LIN(o->C12, col[C_C12]);
        LIN(o->C44, col[C_C44]);
        LIN(o->e14, e14);
        LIN(o->B114, col[C_B114]);
        LIN(o->B124, col[C_B124]);
        LIN(o->B156, col[C_B156]);
        LIN(o->ac, col[C_ac]);
        LIN(o->av, col[C_av]);
        LIN(o->b, col[C_b]);
        LIN(o->d, col[C_d]);
        LIN(o->nr, col[C_nr]);
    }
    /* ternary Ev_avg bowing referenced to the matrix lattice constant (material_parameters.c:1060-1081) */
    static const int pairs[QD_N_TERNARY][2] = {{1, 6}, {2, 7}, {3, 8}, {6, 11}, {7, 12}, {8, 13},
                                               {1, 11}, {2, 12}, {3, 13}, {1, 2}, {1, 3}, {2, 3},
                                               {6, 7}, {6, 8}, {7, 8}, {11, 12}, {11, 13}, {12, 13}};
    double bowEv[QD_N_TERNARY], bowEg[QD_N_TERNARY], bowDso[QD_N_TERNARY];
    for (int k = 0; k < QD_N_TERNARY; k++) {
        int i = pairs[k][0], j = pairs[k][1];
        bowEv[k] = (3.0 / out[0].a) * (col[C_av][i] - col[C_av][j]) * (col[C_a][i] - col[C_a][j]);
        bowEg[k] = qd_ternary_bowing[k][0];
        bowDso[k] = qd_ternary_bowing[k][1];
    }
#define BOW(dst, arr, btab)                                                                       \
    do {                                                                                          \
        for (int q = 0; q < 4; q++) {                                                             \
            P[q] = sys_bin[m][q] >= 0 ? (arr)[sys_bin[m][q]] : 0.0;                               \
            B[q] = sys_tern[m][q] >= 0 ? (btab)[sys_tern[m][q]] : 0.0;                            \
        }                                                                                         \
        (dst) = interp(1, t, g->x, g->y, P, B);                                                   \
        for (int q = 0; q < 4; q++) B[q] = 0.0;                                                   \
    } while (0)
    for (int s = 0; s < n_shape; s++) {
        struct supercell_geometry *g = &geo[s];
        struct material_params *o = &out[s];
        int m = g->material, t = sys_type[m];
        BOW(o->Ev_avg, col[C_Ev], bowEv);
        BOW(o->Eg, Eg, bowEg);
        BOW(o->Dso, col[C_Dso], bowDso);
        LIN(o->sc, sc);
        LIN(o->Ep, col[C_Ep]);
        o->P = sqrt(0.5 * QD_HBSQM * o->Ep); /* :1384 */
        LIN(o->g1, g1);
        LIN(o->g2, g2);
        LIN(o->g3, g3);
    }
#undef LIN
#undef BOW
    /* band edges, zero at the matrix VB edge (material_parameters.c:1529-1538) */
    double ref = out[0].Ev_avg + out[0].Dso / 3.0;
    for (int s = 0; s < n_shape; s++) {
        out[s].E_hh = out[s].Ev_avg + out[s].Dso / 3.0 - ref;
        out[s].E_so = out[s].E_hh - out[s].Dso;
        out[s].E_lh = out[s].E_hh;
        out[s].E_cb = out[s].E_hh + out[s].Eg;
    }
    return QD_OK;
}

/* Derivative of every shape's material parameters with respect to the scale
 * of the binary table's Ep column (which = 0) or Luttinger gamma_1 column
 * (which = 1), at the current scales.  Only sc, g1, g2, g3, Ep and P depend on
 * them: sc_i, g1_i, g2_i, g3_i are linear in the binary Ep_i, the
 * interpolation is linear in the binary values, and P = sqrt(HBSQM Ep / 2)
 * gives dP = HBSQM dEp / (4 P).  Every other field of dmat is zero. */
int qd_material_tangent(int which, int n_shape, const struct supercell_geometry *geo,
                        const struct material_params *mat, struct material_params *dmat) {
    double dsc[QD_N_BINARY], dg1[QD_N_BINARY], dg2[QD_N_BINARY], dEp[QD_N_BINARY];
    for (int i = 0; i < QD_N_BINARY; i++) {
        const double *row = qd_binary_rows[i];
        const double Eg0 = row[C_Eg], Dso = row[C_Dso];
        dsc[i] = dg1[i] = dg2[i] = dEp[i] = 0.0;
        if (which == 0) {
            dEp[i] = row[C_Ep];
            dsc[i] = -(dEp[i] / 3.0) * (2.0 / Eg0 + 1.0 / (Eg0 + Dso));
            dg1[i] = -dEp[i] / (3.0 * Eg0 + Dso);
            dg2[i] = -dEp[i] / (6.0 * Eg0 + 2.0 * Dso);
        } else {
            dg1[i] = row[C_gL1];
        }
    }
    double P[4], B[4] = {0, 0, 0, 0};
    for (int s = 0; s < n_shape; s++) {
        const struct supercell_geometry *g = &geo[s];
        struct material_params *o = &dmat[s];
        const int m = g->material, t = sys_type[m];
        memset(o, 0, sizeof(*o));
#define DLIN(dst, arr)                                                                            \
    do {                                                                                          \
        for (int q = 0; q < 4; q++) P[q] = sys_bin[m][q] >= 0 ? (arr)[sys_bin[m][q]] : 0.0;       \
        (dst) = interp(0, t, g->x, g->y, P, B);                                                   \
    } while (0)
        DLIN(o->sc, dsc);
        DLIN(o->g1, dg1);
        DLIN(o->g2, dg2);
        o->g3 = o->g2; /* g2 and g3 share the Ep correction and neither has a gamma_1 term */
        DLIN(o->Ep, dEp);
#undef DLIN
        o->P = mat[s].P > 0.0 ? QD_HBSQM * o->Ep / (4.0 * mat[s].P) : 0.0;
    }
    return QD_OK;
}
