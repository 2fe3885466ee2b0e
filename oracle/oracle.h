/*
 * oracle.h -- CPU restatement of the reference's forward dynamic-rupture
 * path.  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py load it as the checker.  The
 * product (libcgfd.so) never links or calls it.
 *
 * Same inputs as the product (cgfd_config from include/cgfd.h); the entry
 * points mirror include/cgfd.h with an oracle_ prefix.  Built twice by
 * oracle/build.py: liboracle.so (float, the reference's arithmetic) and
 * liboracle64.so (double, for error estimates).
 */
#ifndef CGFD_ORACLE_H
#define CGFD_ORACLE_H

#include "../include/cgfd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_solver oracle_solver;

int  oracle_create(const cgfd_config *cfg, oracle_solver **out);
int  oracle_run(oracle_solver *s, int nsteps);
int  oracle_get_fault(oracle_solver *s, int fault_id, int field, float *out);
int  oracle_get_stations(oracle_solver *s, float *out, int *nrec);
int  oracle_get_fault_stations(oracle_solver *s, float *out, int *nrec);
int  oracle_get_wavefield(oracle_solver *s, int cmp, float *out);
int  oracle_set_wavefield(oracle_solver *s, int cmp, const float *in);
/* metric (0 jac, 1..9 xi_x..zeta_z) at interior points [nk][nj][ni] */
int  oracle_get_metric(oracle_solver *s, int cmp, float *out);
/* surface peaks [15][nj][ni] as cgfd_get_surface_peaks */
int  oracle_get_surface_peaks(oracle_solver *s, float *out);
int  oracle_dt_max(oracle_solver *s, float *dtmax);
int  oracle_set_threads(int nthreads);
int  oracle_real_bytes(void);
void oracle_destroy(oracle_solver *s);
const char *oracle_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
