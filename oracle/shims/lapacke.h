/*
 * Test-infrastructure shim (oracle only): stands in for the LAPACKE header that the
 * reference CPU build of Interpolate.cu includes (Interpolate.cu:8, call at :236).
 * No LAPACK is installed in this image, so this header provides LAPACKE_dgtsv with
 * the algorithm LAPACK documents for DGTSV: Gaussian elimination of a tridiagonal
 * system with partial pivoting (row interchanges between neighbouring rows), which
 * creates one extra super-diagonal, followed by back substitution.
 *
 * Argument meaning follows the LAPACKE C interface for one right-hand side:
 *   n   order of the matrix, nrhs number of right-hand sides (only 1 is used),
 *   dl  (n-1) sub-diagonal, d (n) diagonal, du (n-1) super-diagonal,
 *   b   right-hand side, overwritten by the solution.
 * Returns 0 on success, i>0 if the i-th pivot is exactly zero.
 */
#ifndef ORACLE_SHIM_LAPACKE_H
#define ORACLE_SHIM_LAPACKE_H

#include <cmath>

#ifndef LAPACK_COL_MAJOR
#define LAPACK_COL_MAJOR 102
#endif

static inline int LAPACKE_dgtsv(int layout, int n, int nrhs, double *dl, double *d,
                                double *du, double *b, int ldb)
{
    (void)layout;
    (void)ldb;
    if (n <= 0 || nrhs != 1)
        return -1;
    /* extra second super-diagonal produced by interchanges */
    double *du2 = new double[n > 2 ? n - 2 : 1];
    for (int i = 0; i < n - 2; i++)
        du2[i] = 0.0;

    for (int i = 0; i < n - 1; i++)
    {
        if (std::fabs(d[i]) >= std::fabs(dl[i]))
        {
            /* keep row i as pivot row */
            if (d[i] == 0.0)
            {
                delete[] du2;
                return i + 1;
            }
            double m = dl[i] / d[i];
            d[i + 1] -= m * du[i];
            b[i + 1] -= m * b[i];
            dl[i] = 0.0;
        }
        else
        {
            /* swap rows i and i+1, row i+1 becomes the pivot row */
            double m = d[i] / dl[i];
            d[i] = dl[i];
            double old_d_next = d[i + 1];
            d[i + 1] = du[i] - m * old_d_next;
            if (i < n - 2)
            {
                du2[i] = du[i + 1];
                du[i + 1] = -m * du2[i];
            }
            du[i] = old_d_next;
            double bi = b[i];
            b[i] = b[i + 1];
            b[i + 1] = bi - m * b[i + 1];
            dl[i] = 0.0;
        }
    }
    if (d[n - 1] == 0.0)
    {
        delete[] du2;
        return n;
    }
    /* back substitution with the upper band (d, du, du2) */
    b[n - 1] /= d[n - 1];
    if (n > 1)
        b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
    for (int i = n - 3; i >= 0; i--)
        b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i];
    delete[] du2;
    return 0;
}

#endif
