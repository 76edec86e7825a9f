// Coulomb matrix elements (coulomb_matrix_elements.c:24-627, include_CME = 1).
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#include "qd_internal.h"

extern "C" int qd_coulomb(qd_problem *pr, int n_vb_states, int n_cb_states, const qd_complex128 *eigvec_host,
                          qd_complex128 *hh, qd_complex128 *ee, qd_complex128 *eh_direct,
                          qd_complex128 *eh_exchange) {
    (void)pr; (void)n_vb_states; (void)n_cb_states; (void)eigvec_host; (void)hh; (void)ee; (void)eh_direct;
    (void)eh_exchange;
    return qd_set_error(QD_ERR_UNSUPPORTED, "Coulomb matrix elements are not built yet");
}

extern "C" void coulomb_matrix_elements(struct wave_vectors basis, struct wave_vectors coulomb_basis,
                                        struct supercell_geometry *supercell, struct material_params *parameters,
                                        int *N_states, struct eigenstate *eigenstate_vb,
                                        struct eigenstate *eigenstate_cb, struct coulomb_matrix_element CME,
                                        int coulomb_region_type) {
    (void)basis; (void)coulomb_basis; (void)supercell; (void)parameters; (void)N_states; (void)eigenstate_vb;
    (void)eigenstate_cb; (void)CME; (void)coulomb_region_type;
    printf("coulomb_matrix_elements failed: not built yet\n");
    exit(1);
}
