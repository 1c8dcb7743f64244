/* Stand-in for LAPACKE (LAPACK 3.8.0 in the reference's README.md:11).  The only
 * routine the reference calls is zpteqr (FAME_Main/Lanczos_Isotropic.cu:53); it is
 * bound to the LP64 LAPACKE build exported by scipy's bundled OpenBLAS. */
#ifndef FAME_REF_SHIM_LAPACKE_H
#define FAME_REF_SHIM_LAPACKE_H
typedef int lapack_int;
#define LAPACK_COL_MAJOR 102
extern "C" lapack_int scipy_LAPACKE_zpteqr(int layout, char compz, lapack_int n,
                                           double* d, double* e, void* z, lapack_int ldz);
#define LAPACKE_zpteqr(layout, compz, n, d, e, z, ldz) \
  scipy_LAPACKE_zpteqr((layout), (compz), (n), (d), (e), (void*)(z), (ldz))
#endif
