/* Minimal LAPACKE declaration so the reference's CPU branch
 * (src/few/cutils/interpolate.cu:14-17, 231-236) links against the LAPACK that
 * scipy bundles (OpenBLAS, symbols prefixed "scipy_").  Used only by the
 * oracle/_ref build recipe in oracle/Makefile. */
#ifndef FEW_ORACLE_LAPACKE_SHIM_H
#define FEW_ORACLE_LAPACKE_SHIM_H
#define LAPACK_COL_MAJOR 102
#ifdef __cplusplus
extern "C" {
#endif
int scipy_LAPACKE_dgtsv(int matrix_layout, int n, int nrhs, double *dl, double *d, double *du,
                        double *b, int ldb);
#ifdef __cplusplus
}
#endif
#define LAPACKE_dgtsv scipy_LAPACKE_dgtsv
#endif
