/* Full-form RCD and AMaZE demosaics: CPU oracle (TEST INFRASTRUCTURE only;
 * imported by tests/ as the checker, never by the product library).
 *
 * The reference's demosaic.rcd and demosaic.amaze nodes compute reduced 5x5
 * stencils (src/cpipe/nodes/demosaic/demosaic_rcd_generator.cpp:8-77,
 * demosaic_amaze_generator.cpp:8-79).  This file restates the published
 * algorithms those nodes are named after, as this project defines them for
 * its "full" form (node parameter algorithm = "full"):
 *
 *  RCD -- Ratio Corrected Demosaicing, Luis Sanz Rodriguez (v2.3, as
 *  distributed with RawTherapee / librtprocess):
 *   1   vertical/horizontal discrimination VH = Sv / (Sv + Sh), S = max(1e-10,
 *       sum over the pixel and its two neighbours along the direction of the
 *       squared 7-tap high-pass (1, -3, -1, 6, -1, -3, 1) of the mosaic);
 *   2   low-pass of the mosaic (1/4 centre, 1/8 cross, 1/16 diagonals);
 *   3   green at red/blue sites: cardinal estimates c_n * 2 lpf / (eps + lpf +
 *       lpf_n2), each direction pair blended with the opposite gradients
 *       (eps + four absolute differences reaching 4 pixels), then
 *       VH' * H + (1 - VH') * V, VH' the centre VH or the mean of its four
 *       diagonal neighbours, whichever is further from 0.5;
 *   4.1 diagonal discrimination PQ the same way along the two diagonals;
 *   4.2 the other colour at red/blue sites: green plus the diagonal colour
 *       differences, blended by diagonal gradients and PQ';
 *   4.3 red and blue at green sites: green plus the cardinal colour
 *       differences, blended by cardinal gradients and VH'.
 *  Outputs are clamped below at 0; eps = 1e-5.
 *
 *  AMaZE -- Aliasing Minimization and Zipper Elimination, Emil Martinec
 *  (2010, as distributed with RawTherapee), in these stages:
 *   A   gradients delh, delv and the directional weights
 *       eps + |c(+2) - c| + |c - c(-2)| + del per axis;
 *   B   green-minus-colour differences vcd / hcd from the adaptive-ratio
 *       estimates (ratio used where |1 - ratio| < 0.75, else Hamilton-Adams),
 *       blended by the directional weights; Hamilton-Adams alone where the
 *       site or either estimate exceeds 0.8 (highlight protection);
 *       dgint = min of the squared up/down (left/right) estimate differences;
 *   C   the vertical weight hvwt from the variance of the colour differences
 *       over four samples each way (about their mean), or from the dgint
 *       fluctuation when the two measures disagree or the latter is more
 *       decisive;
 *   D   the Nyquist texture test at red/blue sites (Gaussian-weighted
 *       squared vcd - hcd over the 13-site quincunx minus 0.5 x the
 *       Gaussian-weighted squared gradients over the 5x5 window), then a
 *       majority vote of the eight same-lattice neighbours (ties keep the
 *       site's own flag);
 *   E   in Nyquist areas hvwt from the area statistics of the same-colour
 *       sites within +-6 that are Nyquist sites;
 *   F   hvwt replaced by the mean of its four diagonal neighbours' values
 *       (from E, so the result does not depend on a scan order) when that is
 *       more decisive; green = c + hcd (1 - hvwt) + vcd hvwt;
 *   G   in Nyquist areas green from the Gaussian-weighted squared green
 *       curvatures over the quincunx;
 *   H   the other colour's difference at red/blue sites from the four
 *       diagonal directions, each 1.325 d1 - 0.175 d3 - 0.075 (two side
 *       sites), weighted by 1 / (eps + three absolute differences);
 *   I   red and blue at green sites from the four cardinal neighbours'
 *       differences weighted by hvwt (vertical) and 1 - hvwt (horizontal).
 *  The Gaussian weights are computed from their definitions (not tabulated):
 *  exp(-d^2 / (2 s^2)) normalised over the stated support, s^2 = 2.88 for the
 *  quincunx and 5x5 tests of D (distances in pixels), s^2 = 2.25 for G's
 *  quincunx; 0.5 is the Nyquist threshold.  Inputs are the normalised mosaic
 *  (white = 1), so the highlight limit is 0.8.
 *
 * Both algorithms read the mosaic through reflect-101 extension (period
 * 2(n-1), which keeps the CFA phase), so every output pixel uses the same
 * formulas; every intermediate quantity outside the frame is evaluated from
 * that extension at its own position.  The kernels compute exactly these
 * expressions in binary32 in this operation order (no contraction), so the
 * R = float instantiation is their bit-exact checker; the R = double one is
 * the FP64 reference.  Parity with RawTherapee's own implementations is not
 * claimed (they are not part of the reference tree). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int dm_refl(int i, int n) {
    if (n <= 1) return 0;
    const int p = 2 * (n - 1);
    i %= p;
    if (i < 0) i += p;
    return i >= n ? p - i : i;
}

static inline int dm_color(const uint8_t cfa4[4], int x, int y) { return cfa4[((y & 1) << 1) | (x & 1)]; }

/* The Gaussian weight sets of the AMaZE restatement, in double. */
void oracle_amaze_weights(double odd[4], double grad[6], double quinc[4]) {
    /* quincunx of 13 sites: d^2 = 0 (1), 2 (4), 4 (4), 8 (4) */
    const double qd[4] = {0.0, 2.0, 4.0, 8.0}, qn[4] = {1.0, 4.0, 4.0, 4.0};
    /* 5x5 window: d^2 = 0 (1), 1 (4), 2 (4), 4 (4), 5 (8), 8 (4) */
    const double gd[6] = {0.0, 1.0, 2.0, 4.0, 5.0, 8.0}, gn[6] = {1.0, 4.0, 4.0, 4.0, 8.0, 4.0};
    double s = 0.0;
    for (int i = 0; i < 4; ++i) s += qn[i] * exp(-qd[i] / (2.0 * 2.88));
    for (int i = 0; i < 4; ++i) odd[i] = exp(-qd[i] / (2.0 * 2.88)) / s;
    s = 0.0;
    for (int i = 0; i < 6; ++i) s += gn[i] * exp(-gd[i] / (2.0 * 2.88));
    for (int i = 0; i < 6; ++i) grad[i] = 0.5 * exp(-gd[i] / (2.0 * 2.88)) / s;
    s = 0.0;
    for (int i = 0; i < 4; ++i) s += qn[i] * exp(-qd[i] / (2.0 * 2.25));
    for (int i = 0; i < 4; ++i) quinc[i] = exp(-qd[i] / (2.0 * 2.25)) / s;
}

static void amaze_weights_f(float o[4], float g[6], float q[4]) {
    double od[4], gd[6], qd[4];
    oracle_amaze_weights(od, gd, qd);
    for (int i = 0; i < 4; ++i) o[i] = (float)od[i], q[i] = (float)qd[i];
    for (int i = 0; i < 6; ++i) g[i] = (float)gd[i];
}
static void amaze_weights_d(double o[4], double g[6], double q[4]) { oracle_amaze_weights(o, g, q); }

#define R float
#define SFX _f
#include "oracle_demosaic_full.h"
#undef R
#undef SFX

#define R double
#define SFX _d
#include "oracle_demosaic_full.h"
#undef R
#undef SFX

/* algo: 1 RCD, 2 AMaZE.  prec: 0 binary32 (the kernels' arithmetic), 1 FP64.
 * out: w x h x 3 doubles (the binary32 results widened exactly). */
int oracle_demosaic_full(int algo, int prec, const float* in, int w, int h, const uint8_t cfa4[4], double* out) {
    if (w <= 0 || h <= 0) return -1;
    const size_t n = (size_t)w * h * 3;
    if (prec == 1) return algo == 1 ? oracle_rcd_full_d(in, w, h, cfa4, out) : oracle_amaze_full_d(in, w, h, cfa4, out);
    float* tmp = (float*)malloc(sizeof(float) * n);
    if (!tmp) return -1;
    const int st = algo == 1 ? oracle_rcd_full_f(in, w, h, cfa4, tmp) : oracle_amaze_full_f(in, w, h, cfa4, tmp);
    for (size_t i = 0; i < n; ++i) out[i] = tmp[i];
    free(tmp);
    return st;
}
