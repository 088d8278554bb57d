/* Stand-in for the reference's src/inverse_matrix.c, which calls LAPACK
 * dgetrf_/dgetri_ (src/inverse_matrix.c:14-18) and needs lapacke.h, absent here.
 *
 * Same symbol and contract: invert the 3x3 matrix A in place.  The reference uses it
 * only once, at set-up, to invert per-ion polarisability tensors (src/config.c:171).
 * Gauss-Jordan elimination with partial pivoting: for a diagonal input every inverse
 * entry is exactly 1.0/a_ii, as LAPACK's triangular inverse gives.
 * Linked into the drop-in build of the reference program (Makefile target dropin) and
 * into the compiled-reference checker. */
#include <math.h>
#include <stdio.h>

void invertmatrix3x3(double A[3][3]) {
    double m[3][6];
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            m[i][j] = A[i][j];
            m[i][j + 3] = (i == j) ? 1.0 : 0.0;
        }
    }
    for (int c = 0; c < 3; c++) {
        int p = c;
        for (int r = c + 1; r < 3; r++)
            if (fabs(m[r][c]) > fabs(m[p][c])) p = r;
        if (m[p][c] == 0.0) {
            fprintf(stderr, "ERROR : singular matrix in invertmatrix3x3\n");
            return;
        }
        if (p != c) {
            for (int j = 0; j < 6; j++) {
                double t = m[c][j];
                m[c][j] = m[p][j];
                m[p][j] = t;
            }
        }
        double inv = 1.0 / m[c][c];
        for (int j = 0; j < 6; j++) m[c][j] = (j == c) ? 1.0 : m[c][j] * inv;
        /* the pivot row's identity part now holds 1/a_cc exactly for a diagonal input */
        for (int r = 0; r < 3; r++) {
            if (r == c) continue;
            double f = m[r][c];
            if (f == 0.0) continue;
            for (int j = 0; j < 6; j++) m[r][j] -= f * m[c][j];
        }
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = m[i][j + 3];
}
