/* FP64 CPU oracle for two-stage colour BM3D (aot_id denoise_bm3d_spec).
 *
 * TEST INFRASTRUCTURE ONLY: tests and the benchmark's CPU-baseline leg load
 * this file as the checker; the product path never does.
 *
 * The reference's denoise.bm3d node is a 2x2 box blend
 * (reference src/cpipe/nodes/denoise/bm3d_step1_generator.cpp:33-61, restated
 * in oracle_nodes.c).  This file restates the published algorithm the node is
 * named after, so parity here is pinned to the publication, not to reference
 * output:
 *   Dabov, Foi, Katkovnik, Egiazarian, "Image denoising by sparse 3D
 *   transform-domain collaborative filtering", IEEE TIP 16(8), 2007;
 *   the colour form of the same authors (ICIP 2007): grouping on luminance,
 *   the same groups for the chrominance channels;
 *   parameter values from Lebrun, "An analysis and implementation of the BM3D
 *   image denoising method", IPOL 2 (2012).
 *
 * Definition (shared with the CUDA kernels, which compute it in FP32):
 *  - colour: orthonormal opponent transform Y=(R+G+B)/sqrt3, U=(R-B)/sqrt2,
 *    V=(R-2G+B)/sqrt6, so the per-channel noise sigma is unchanged;
 *  - reference blocks: 8x8 at x = min(i*nstep, W-8) for i = 0.. until W-8 is
 *    reached (same in y);
 *  - matching: integer squared distance over the block of the quantised
 *    luminance q = rint(clamp(L,0,1)*255), L = ((R+G)+B)*(1/3) in FP32 for
 *    step 1 and L = Y_basic*(1/sqrt3) in FP32 for step 2; candidates are all
 *    block positions within +-(ns-1)/2 of the reference (clipped to the
 *    image); accepted if d <= floor(64*tau); the group is the reference block
 *    followed by the accepted candidates in increasing (d, raster position),
 *    truncated to n2 and then to the largest power of two;
 *  - 3D transform: orthonormal 8x8 DCT-II per block, then the orthonormal Haar
 *    wavelet along the group (full decomposition, in place: the approximation
 *    of level s at index b (b % 2s == 0), the detail at b+s);
 *  - step 1: hard threshold |c| > lambda3d*sigma, weight 1/(sigma^2*N_kept)
 *    (1 when nothing is kept);
 *  - step 2: groups of the basic estimate and of the noisy image at the same
 *    positions; Wiener shrink W = B^2/(B^2+sigma^2) of the noisy coefficients,
 *    weight 1/(sigma^2*max(sum W^2, 1e-20)) (1 when the sum is 0);
 *  - aggregation: weight x 8x8 Kaiser window (beta) per block, numerator and
 *    denominator per channel; estimate = numerator / denominator;
 *  - alpha is copied; images smaller than 8x8, sigma <= 0 or a sigma whose
 *    FP32 square is 0 are copied.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/cpipe_b200_params.h"

#define ST_OK 0
#define ST_BAD_INDEX 5

static const double kS3 = 1.7320508075688772935; /* sqrt 3 */
static const double kS2 = 1.4142135623730950488;
static const double kS6 = 2.4494897427831780982;

int oracle_bm3d_ref_count(int n, int nstep) {
    if (n < 8 || nstep < 1) return 0;
    int m = (n - 8) / nstep + 1;
    if ((n - 8) % nstep) m++;
    return m;
}

static inline int ref_pos(int i, int n, int nstep) {
    int p = i * nstep;
    return p > n - 8 ? n - 8 : p;
}

static inline uint8_t quantise(float l) {
    if (!(l > 0.0f)) l = 0.0f;
    if (l > 1.0f) l = 1.0f;
    return (uint8_t)rintf(l * 255.0f);
}

/* Step-1 matching luminance of an RGBA float image. */
void oracle_bm3d_quantise_rgb(const float* rgba, int w, int h, uint8_t* q) {
    for (long i = 0; i < (long)w * h; ++i) {
        float s = (rgba[4 * i] + rgba[4 * i + 1]) + rgba[4 * i + 2];
        q[i] = quantise(s * (1.0f / 3.0f));
    }
}

/* Step-2 matching luminance from the basic estimate's Y channel (FP32 value). */
void oracle_bm3d_quantise_y(const float* y, int w, int h, uint8_t* q) {
    for (long i = 0; i < (long)w * h; ++i) q[i] = quantise(y[i] * 0.57735026918962576f);
}

uint32_t oracle_bm3d_dthr(float tau) { return (uint32_t)floor(64.0 * (double)tau); }

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y);
}

/* Group of the reference block at (x, y): pos[0] = the reference, then the
 * accepted candidates.  pos entries are (y << 16) | x.  Returns the number of
 * entries before the power-of-two truncation (1..n2).  scratch holds ns*ns
 * keys. */
int oracle_bm3d_match(const uint8_t* q, int w, int h, int x, int y, int ns, int n2,
                      uint32_t dthr, uint32_t* pos, uint64_t* scratch) {
    int R = (ns - 1) / 2, n = 0;
    int y0 = y - R < 0 ? 0 : y - R, y1 = y + R > h - 8 ? h - 8 : y + R;
    int x0 = x - R < 0 ? 0 : x - R, x1 = x + R > w - 8 ? w - 8 : x + R;
    pos[0] = ((uint32_t)y << 16) | (uint32_t)x;
    if (n2 <= 1) return 1;
    for (int yy = y0; yy <= y1; ++yy)
        for (int xx = x0; xx <= x1; ++xx) {
            if (xx == x && yy == y) continue;
            uint32_t d = 0;
            for (int v = 0; v < 8; ++v)
                for (int u = 0; u < 8; ++u) {
                    int e = (int)q[(long)(y + v) * w + x + u] - (int)q[(long)(yy + v) * w + xx + u];
                    d += (uint32_t)(e * e);
                }
            if (d > dthr) continue;
            uint32_t widx = (uint32_t)((yy - y + R) * ns + (xx - x + R));
            scratch[n++] = ((uint64_t)d << 11) | widx;
        }
    qsort(scratch, n, sizeof(uint64_t), cmp_u64);
    int take = n < n2 - 1 ? n : n2 - 1;
    for (int k = 0; k < take; ++k) {
        int widx = (int)(scratch[k] & 2047u);
        int yy = y + widx / ns - R, xx = x + widx % ns - R;
        pos[1 + k] = ((uint32_t)yy << 16) | (uint32_t)xx;
    }
    return 1 + take;
}

static int pow2_floor(int n) {
    int p = 1;
    while (p * 2 <= n) p *= 2;
    return p;
}

static double bessel_i0(double x) {
    double sum = 1.0, term = 1.0, hx = 0.5 * x;
    for (int k = 1; k < 64; ++k) {
        term *= (hx / k) * (hx / k);
        sum += term;
        if (term < 1e-18 * sum) break;
    }
    return sum;
}

/* 8x8 Kaiser window, row-major [v][u]. */
void oracle_bm3d_kaiser(double beta, double* k64) {
    double k1[8], i0b = bessel_i0(beta);
    for (int n = 0; n < 8; ++n) {
        double t = (2.0 * n - 7.0) / 7.0;
        k1[n] = bessel_i0(beta * sqrt(1.0 - t * t)) / i0b;
    }
    for (int v = 0; v < 8; ++v)
        for (int u = 0; u < 8; ++u) k64[v * 8 + u] = k1[v] * k1[u];
}

static double g_dct[8][8]; /* g_dct[k][n] = a(k) cos((2n+1) k pi / 16) */
static int g_dct_ready = 0;

static void dct_init(void) {
    if (g_dct_ready) return;
    for (int k = 0; k < 8; ++k)
        for (int n = 0; n < 8; ++n)
            g_dct[k][n] = (k == 0 ? sqrt(0.125) : 0.5) * cos((2 * n + 1) * k * M_PI / 16.0);
    g_dct_ready = 1;
}

static void dct2(double* b, int inverse) {
    double t[64];
    /* rows (along u) */
    for (int v = 0; v < 8; ++v)
        for (int k = 0; k < 8; ++k) {
            double s = 0.0;
            for (int n = 0; n < 8; ++n) s += (inverse ? g_dct[n][k] : g_dct[k][n]) * b[v * 8 + n];
            t[v * 8 + k] = s;
        }
    /* columns (along v) */
    for (int u = 0; u < 8; ++u)
        for (int k = 0; k < 8; ++k) {
            double s = 0.0;
            for (int n = 0; n < 8; ++n) s += (inverse ? g_dct[n][k] : g_dct[k][n]) * t[n * 8 + u];
            b[k * 8 + u] = s;
        }
}

static void haar(double* g, int N, int inverse) {
    const double r2 = 1.0 / kS2;
    if (!inverse) {
        for (int s = 1; s < N; s *= 2)
            for (int b = 0; b < N; b += 2 * s)
                for (int i = 0; i < 64; ++i) {
                    double a = g[b * 64 + i], o = g[(b + s) * 64 + i];
                    g[b * 64 + i] = (a + o) * r2;
                    g[(b + s) * 64 + i] = (a - o) * r2;
                }
    } else {
        for (int s = N / 2; s >= 1; s /= 2)
            for (int b = 0; b < N; b += 2 * s)
                for (int i = 0; i < 64; ++i) {
                    double a = g[b * 64 + i], d = g[(b + s) * 64 + i];
                    g[b * 64 + i] = (a + d) * r2;
                    g[(b + s) * 64 + i] = (a - d) * r2;
                }
    }
}

typedef struct {
    int w, h, nrx, nry, ns, n2, nstep;
    double sigma, thr, k64[64];
} Geo;

/* One stage over the whole image.  noisy/basic: 3 YUV planes (double); q:
 * matching luminance; est: 3 output planes.  basic == NULL selects step 1. */
static void run_stage(const Geo* g, const double* noisy, const double* basic, const uint8_t* q,
                      uint32_t dthr, double* est) {
    const int w = g->w, h = g->h;
    const long npx = (long)w * h;
    const int halo = (g->ns - 1) / 2 + 8;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    if (nthreads > g->nry) nthreads = g->nry;
    if (nthreads < 1) nthreads = 1;
    double* acc = (double*)calloc((size_t)6 * npx, sizeof(double));
#pragma omp parallel num_threads(nthreads)
    {
        int t = 0, nt = 1;
#ifdef _OPENMP
        t = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        int j0 = (int)((long)g->nry * t / nt), j1 = (int)((long)g->nry * (t + 1) / nt);
        int ylo = 0, yhi = 0;
        if (j1 > j0) {
            ylo = ref_pos(j0, h, g->nstep) - halo;
            yhi = ref_pos(j1 - 1, h, g->nstep) + halo;
            if (ylo < 0) ylo = 0;
            if (yhi > h) yhi = h;
        }
        long band = (long)(yhi - ylo) * w;
        double* loc = (double*)calloc((size_t)6 * (band > 0 ? band : 1), sizeof(double));
        uint64_t* scratch = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)g->ns * g->ns);
        double* gz = (double*)malloc(sizeof(double) * 16 * 64);
        double* gb = (double*)malloc(sizeof(double) * 16 * 64);
        uint32_t pos[16];
        for (int j = j0; j < j1; ++j)
            for (int i = 0; i < g->nrx; ++i) {
                int x = ref_pos(i, w, g->nstep), y = ref_pos(j, h, g->nstep);
                int cnt = oracle_bm3d_match(q, w, h, x, y, g->ns, g->n2, dthr, pos, scratch);
                int N = pow2_floor(cnt);
                for (int c = 0; c < 3; ++c) {
                    for (int b = 0; b < N; ++b) {
                        int bx = (int)(pos[b] & 0xFFFF), by = (int)(pos[b] >> 16);
                        for (int v = 0; v < 8; ++v)
                            for (int u = 0; u < 8; ++u) {
                                long o = (long)c * npx + (long)(by + v) * w + bx + u;
                                gz[b * 64 + v * 8 + u] = noisy[o];
                                if (basic) gb[b * 64 + v * 8 + u] = basic[o];
                            }
                        dct2(gz + b * 64, 0);
                        if (basic) dct2(gb + b * 64, 0);
                    }
                    haar(gz, N, 0);
                    if (basic) haar(gb, N, 0);
                    double wgt;
                    if (!basic) {
                        int kept = 0;
                        for (int k = 0; k < N * 64; ++k) {
                            if (fabs(gz[k]) > g->thr) kept++;
                            else gz[k] = 0.0;
                        }
                        wgt = kept ? 1.0 / (g->sigma * g->sigma * kept) : 1.0;
                    } else {
                        double sw2 = 0.0, s2 = g->sigma * g->sigma;
                        for (int k = 0; k < N * 64; ++k) {
                            double b2 = gb[k] * gb[k], W = b2 / (b2 + s2);
                            gz[k] *= W;
                            sw2 += W * W;
                        }
                        wgt = sw2 > 0.0 ? 1.0 / (s2 * (sw2 > 1e-20 ? sw2 : 1e-20)) : 1.0;
                    }
                    haar(gz, N, 1);
                    for (int b = 0; b < N; ++b) {
                        dct2(gz + b * 64, 1);
                        int bx = (int)(pos[b] & 0xFFFF), by = (int)(pos[b] >> 16);
                        for (int v = 0; v < 8; ++v)
                            for (int u = 0; u < 8; ++u) {
                                long o = (long)(by + v - ylo) * w + bx + u;
                                double kw = wgt * g->k64[v * 8 + u];
                                loc[(long)c * band + o] += kw * gz[b * 64 + v * 8 + u];
                                loc[(long)(3 + c) * band + o] += kw;
                            }
                    }
                }
            }
#pragma omp critical
        {
            for (int c = 0; c < 6; ++c)
                for (long o = 0; o < band; ++o) acc[(long)c * npx + (long)ylo * w + o] += loc[(long)c * band + o];
        }
        free(loc);
        free(scratch);
        free(gz);
        free(gb);
    }
    for (int c = 0; c < 3; ++c)
        for (long o = 0; o < npx; ++o) est[(long)c * npx + o] = acc[(long)c * npx + o] / acc[(long)(3 + c) * npx + o];
    free(acc);
}

static int check_params(const cpipe_Bm3dSpecParams* p) {
    int n2 = p->n2;
    if (!(n2 == 1 || n2 == 2 || n2 == 4 || n2 == 8 || n2 == 16)) return 0;
    if (p->ns < 1 || p->ns > 45 || (p->ns & 1) == 0) return 0;
    if (p->nstep < 1 || p->nstep > 8) return 0;
    if (!(p->tau_match1 >= 0.0f && p->tau_match1 <= 16000.0f)) return 0;
    if (!(p->tau_match2 >= 0.0f && p->tau_match2 <= 16000.0f)) return 0;
    if (p->stages != 1 && p->stages != 2) return 0;
    if (p->transform < 0 || p->transform > 2) return 0; /* precision forms of the GPU path; one definition */
    if (!(p->lambda3d >= 0.0f) || !(p->kaiser_beta >= 0.0f)) return 0;
    return 1;
}

/* rgba: HxWx4 float32 input.  out: HxWx4 double.  basic_yuv (optional): the
 * step-1 estimate, 3 planes of H*W doubles (Y, U, V). */
int oracle_bm3d_spec(const float* rgba, int w, int h, const cpipe_Bm3dSpecParams* p, double* out,
                     double* basic_yuv) {
    if (!check_params(p)) return ST_BAD_INDEX;
    const long npx = (long)w * h;
    if (w < 8 || h < 8 || !(p->sigma > 0.0f) || !(p->sigma * p->sigma > 0.0f)) {
        for (long i = 0; i < 4 * npx; ++i) out[i] = rgba[i];
        if (basic_yuv)
            for (long i = 0; i < npx; ++i) {
                double r = rgba[4 * i], gg = rgba[4 * i + 1], b = rgba[4 * i + 2];
                basic_yuv[i] = (r + gg + b) / kS3;
                basic_yuv[npx + i] = (r - b) / kS2;
                basic_yuv[2 * npx + i] = (r - 2.0 * gg + b) / kS6;
            }
        return ST_OK;
    }
    dct_init();
    Geo g;
    g.w = w; g.h = h; g.ns = p->ns; g.n2 = p->n2; g.nstep = p->nstep;
    g.nrx = oracle_bm3d_ref_count(w, p->nstep);
    g.nry = oracle_bm3d_ref_count(h, p->nstep);
    g.sigma = p->sigma;
    g.thr = (double)p->lambda3d * (double)p->sigma;
    oracle_bm3d_kaiser(p->kaiser_beta, g.k64);

    double* noisy = (double*)malloc(sizeof(double) * 3 * npx);
    double* est1 = (double*)malloc(sizeof(double) * 3 * npx);
    double* est2 = p->stages == 2 ? (double*)malloc(sizeof(double) * 3 * npx) : NULL;
    uint8_t* q = (uint8_t*)malloc((size_t)npx);
    for (long i = 0; i < npx; ++i) {
        double r = rgba[4 * i], gg = rgba[4 * i + 1], b = rgba[4 * i + 2];
        noisy[i] = (r + gg + b) / kS3;
        noisy[npx + i] = (r - b) / kS2;
        noisy[2 * npx + i] = (r - 2.0 * gg + b) / kS6;
    }
    oracle_bm3d_quantise_rgb(rgba, w, h, q);
    run_stage(&g, noisy, NULL, q, oracle_bm3d_dthr(p->tau_match1), est1);
    if (basic_yuv) memcpy(basic_yuv, est1, sizeof(double) * 3 * npx);
    const double* fin = est1;
    if (p->stages == 2) {
        float* yf = (float*)malloc(sizeof(float) * npx);
        for (long i = 0; i < npx; ++i) yf[i] = (float)est1[i];
        oracle_bm3d_quantise_y(yf, w, h, q);
        free(yf);
        run_stage(&g, noisy, est1, q, oracle_bm3d_dthr(p->tau_match2), est2);
        fin = est2;
    }
    for (long i = 0; i < npx; ++i) {
        double Y = fin[i] / kS3, U = fin[npx + i] / kS2, V = fin[2 * npx + i] / kS6;
        out[4 * i] = Y + U + V;
        out[4 * i + 1] = Y - 2.0 * V;
        out[4 * i + 2] = Y - U + V;
        out[4 * i + 3] = rgba[4 * i + 3];
    }
    free(noisy);
    free(est1);
    free(est2);
    free(q);
    return ST_OK;
}
