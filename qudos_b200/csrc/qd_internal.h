/* Internal declarations shared by the host C code and the CUDA translation
 * units of libqdgpu.  Not part of the public ABI. */
#ifndef QD_INTERNAL_H
#define QD_INTERNAL_H

#include "../../include/qudos_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QD_N_BAND 8
#define QD_HBSQM 7.61996   /* hbar^2/m0 [eV Angstrom^2] (8_band.h:51) */
#define QD_ESQEPS 180.9513 /* e^2/eps0 [eV Angstrom] (8_band.h:52) */
#define QD_EPS 1.0e-08     /* 8_band.h:59 */
#define QD_N_COEF 28       /* fields of the fused per-difference coefficient table */

/* Everything the solve path needs from parameters.in / supercell.in. */
typedef struct {
    int n_shape;
    int N[3], NS[3], NC[3];      /* plane waves per axis: electronic, strain, Coulomb cells */
    int strain_type, coulomb_type;
    int n_vb, n_cb;
    double T, F[3], K[3];
    int strain, isotropic, elastic_const, elastic_order, piezo, cme, softening;
    double sigma;
    int eigensolver;
} qd_params;

struct qd_problem {
    qd_params p;
    struct supercell_geometry *geo;  /* n_shape (host) */
    struct material_params *mat;     /* n_shape (host) */
    double *G[3], *GS[3];            /* host grids: electronic (2N-1), strain (2NS-1) */
    int NT[3], NTS[3];
    int64_t nT, nTS, n_pw, n_h;
    int lo, hi;                      /* 0-based eigen window */
    int same_cells;                  /* strain cell == electronic cell */
    /* device state (owned) */
    void *d_geo, *d_mat;
    double *d_G[3], *d_GS[3];
    void *d_chi_s, *d_eps_s, *d_phi_s;   /* strain cell: chi [n_shape][nTS], eps [6][nTS], phi */
    void *d_chi, *d_eps, *d_phi, *d_conv; /* electronic cell: chi [n_shape][nT], eps[6], phi, conv [n_shape][8] */
    void *d_coef;                        /* fused coefficients [QD_N_COEF][nT] */
    int tables_ready;
    /* table builds for a directional derivative: chi of shape chi_dir_shape is
     * shifted by chi_dir_t times the direction arrays (strain cell [nTS],
     * electronic cell [nT]; device) when chi_dir_t != 0 */
    int chi_dir_shape;
    double chi_dir_t;
    void *d_chi_dir_s, *d_chi_dir;
};

/* host_inputs.c */
int qd_read_parameters_text(const char *text, qd_params *p, int *seen_all);
int qd_apply_override(qd_params *p, const char *arg);
int qd_read_supercell_text(const char *text, const qd_params *p, struct supercell_geometry *geo);
int qd_material_parameters(double T, int include_piezo, int n_shape, struct supercell_geometry *geo,
                           struct material_params *out);
void qd_basis_grid(int n_T, double L, double *out);
extern double qd_scale_Ep, qd_scale_gL1;

void qd_count_launch(int n);
/* SMs the calling host thread's solves may spread over: the device's count
 * nsm, or the thread's budget when one is set (qd_set_sm_budget; the batched
 * entry point gives each worker a share so that instances overlap). */
int qd_sm_budget(int nsm);
void qd_set_sm_budget(int n);

/* Stream-ordered device allocations of the solve path, served from the
 * device's default memory pool with its release threshold raised, so that
 * repeated solves reuse the same memory instead of mapping it anew.
 * Return cudaError_t values (0 = success). */
int qd_pool_alloc(void **p, size_t bytes, void *stream);
void qd_pool_free(void *p, void *stream);

/* error state (api.cu) */
int qd_set_error(int code, const char *fmt, ...);

/* device-side stages (tables.cu, assemble.cu) */
int qd_tables_build_dev(struct qd_problem *pr);
int qd_coef_from_host_tables(int n_shape, const int N[3], const double *Gx, const double *Gy,
                             const double *Gz, double Kx, double Ky, double Kz, const double F[3],
                             const struct supercell_geometry *geo, const struct material_params *mat,
                             int strain_on, int piezo_on, const qd_complex128 *const *chi,
                             const qd_complex128 *const *eps, const qd_complex128 *phi,
                             const qd_complex128 *const *conv8, void **d_coef_out, double **d_G_out);
int qd_assemble_launch(const void *d_coef, const double *d_Gx, const double *d_Gy, const double *d_Gz,
                       const int N[3], const double K[3], void *H, int64_t ld, int mode, int prec,
                       void *stream);

int qd_assemble_dk_launch(const void *d_coef, const double *d_Gx, const double *d_Gy, const double *d_Gz,
                          const int N[3], const double K[3], int axis, void *H, int64_t ld, int mode, void *stream);
int qd_hemm_lower_dev(int64_t n, const void *H, int64_t ld, const void *X, int64_t ldx, int k, void *Y, int64_t ldy,
                      double beta, void *stream);
int qd_gram_dev(int64_t n, const void *A, int64_t lda, int ka, const void *B, int64_t ldb, int kb, void *C, int ldc,
                void *stream);

/* eigensolver (eig.cu) */
int qd_eigh_window(int64_t n, void *H, int64_t ld, int lo, int hi, int prec, double *w_dev,
                   void *Z_dev, int64_t ldz, void *stream);

#ifdef __cplusplus
}
#endif
#endif
