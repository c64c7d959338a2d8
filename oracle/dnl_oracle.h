/*
 * dnl_oracle.h - CPU restatement of DynELA's per-increment explicit hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU engine is compared
 * with; it is never linked into, loaded by or called from the engine.  It is
 * a plain-C, FP64, single-threaded restatement of the reference algorithm, each
 * function citing the reference file:line it follows, on the same
 * `dnl_model_desc` and the same state layout as the engine (include/dnlgpu.h).
 * It is itself pinned against the reference compiled from its own sources
 * (oracle/_ref) by the tests.
 */
#ifndef DNL_ORACLE_H
#define DNL_ORACLE_H

#include "dnlgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model orc_model;

orc_model *orc_create(const dnl_model_desc *d);
void orc_destroy(orc_model *m);
const char *orc_last_error(void);
int orc_init(orc_model *m);
long orc_run(orc_model *m, double t_stop, long max_incs);
int orc_element_pass(orc_model *m, double time_step);
int orc_get_nodes(orc_model *m, int field, double *out);
int orc_set_nodes(orc_model *m, int field, const double *in);
int orc_get_ips(orc_model *m, double *out);
int orc_set_ips(orc_model *m, const double *in);
void orc_control(orc_model *m, double out[4]);
double orc_courant(orc_model *m);
int orc_element_lengths(orc_model *m, double *len, double *wave);
int orc_energies(orc_model *m, double out[3]);
long orc_abi_sizeof(int which);

/* Building blocks exposed for unit tests. */
void orc_sym_eigen3(const double a[6], double lambda[3], double vec[3][3]);
void orc_polar_lnU(const double F[9], double lnU[6], double R[9]);
/* One radial return (Element.C:407-622) on a single point; state is
 * [stress 6, plastic strain 6, epsp, depsp, gamma, gammaCum, yield, T, pressure, eint, einel]
 * (21 doubles, updated in place); returns the Newton iteration count or -1. */
int orc_radial_return(const dnl_material *mat, const double dE[6], double dt, double *state);
int orc_radial_return_method(const dnl_material *mat, const double dE[6], double dt, double *state, int direct);
double orc_jc_yield(const dnl_material *mat, double epsp, double depsp, double T);
double orc_jc_hardening(const dnl_material *mat, double epsp, double depsp, double T, double dt);

#ifdef __cplusplus
}
#endif

#endif
