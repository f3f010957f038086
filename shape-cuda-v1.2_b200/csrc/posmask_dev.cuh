// posmask's per-pixel arithmetic (src/shape/posmask.c:58-174), shared by
// the lightcurve kernel (core.cu) and the one-view posmask (posview.cu).
#pragma once

#include "shape_types.h"

namespace shape {

__device__ inline int iround_(double x) { return (x < 0.0) ? (int)(x - 0.5) : (int)(x + 0.5); }

// posmask's sun-view depth at the unrounded sun-view pixel (i0, j0), whose
// nearest pixel (im, jm) is covered (src/shape/posmask.c:101-160): bilinear
// between the four surrounding pixels when all are covered, else the
// nearest pixel's depth corrected along x and y by a one-sided difference
// with whichever neighbour is covered. ZI: the sun view's (2n+1)^2 depths.
__device__ inline double posmask_zill(const double *ZI, int n, int side, double i0, double j0, int im, int jm)
{
    const double bignum = 0.99 * SHAPE_HUGENUMBER;
#define ZILL(a_, b_) ((double)ZI[(long long)((a_) + n) * side + ((b_) + n)])
    const int i1 = (int)floor(i0), j1 = (int)floor(j0);
    double zill;
    if (ZILL(i1, j1) > -bignum && ZILL(i1 + 1, j1) > -bignum &&
        ZILL(i1, j1 + 1) > -bignum && ZILL(i1 + 1, j1 + 1) > -bignum) {
        double t = i0 - i1, u = j0 - j1;
        zill = (1 - t) * (1 - u) * ZILL(i1, j1) + t * (1 - u) * ZILL(i1 + 1, j1)
               + t * u * ZILL(i1 + 1, j1 + 1) + (1 - t) * u * ZILL(i1, j1 + 1);
    } else {
        zill = ZILL(im, jm);
        int i_sign = (i0 >= im) ? 1 : -1;
        int i2 = im + i_sign;
        if (abs(i2) <= n && ZILL(i2, jm) > -bignum) {
            zill += fabs(i0 - im) * (ZILL(i2, jm) - ZILL(im, jm));
        } else {
            i2 = im - i_sign;
            if (abs(i2) <= n && ZILL(i2, jm) > -bignum)
                zill -= fabs(i0 - im) * (ZILL(i2, jm) - ZILL(im, jm));
        }
        int j_sign = (j0 >= jm) ? 1 : -1;
        int j2 = jm + j_sign;
        if (abs(j2) <= n && ZILL(im, j2) > -bignum) {
            zill += fabs(j0 - jm) * (ZILL(im, j2) - ZILL(im, jm));
        } else {
            j2 = jm - j_sign;
            if (abs(j2) <= n && ZILL(im, j2) > -bignum)
                zill -= fabs(j0 - jm) * (ZILL(im, j2) - ZILL(im, jm));
        }
    }
#undef ZILL
    return zill;
}

}  // namespace shape
