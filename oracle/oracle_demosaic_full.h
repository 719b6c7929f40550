/* Body of the full-form RCD and AMaZE demosaic oracle, instantiated twice by
 * oracle_demosaic_full.c: R = float (the kernels' arithmetic, operation for
 * operation, for bit-exact checks) and R = double (the FP64 reference the
 * kernels' error is reported against).  TEST INFRASTRUCTURE only.
 *
 * Needs: R, SFX (name suffix), and the helpers of oracle_demosaic_full.c.
 * See oracle_demosaic_full.c for the definition of both algorithms. */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define F(name) CAT(name, SFX)

/* The CFA plane extended by reflection (period 2(n-1), CFA phase kept) to a
 * margin of M pixels on each side: e[(y + M) * pw + (x + M)] = c(x, y). */
typedef struct {
    R* v;
    int pw, ph, M;
} F(ext_t);

static R F(absr)(R a) { return (R)fabs((double)a); }
static R F(maxr)(R a, R b) { return a > b ? a : b; }
static R F(minr)(R a, R b) { return a < b ? a : b; }

static int F(ext_make)(F(ext_t) * e, const float* in, int w, int h, int M) {
    e->M = M;
    e->pw = w + 2 * M;
    e->ph = h + 2 * M;
    e->v = (R*)malloc(sizeof(R) * (size_t)e->pw * (size_t)e->ph);
    if (!e->v) return -1;
    for (int y = 0; y < e->ph; ++y)
        for (int x = 0; x < e->pw; ++x)
            e->v[(size_t)y * e->pw + x] = (R)in[(size_t)dm_refl(y - M, h) * w + dm_refl(x - M, w)];
    return 0;
}

static R* F(plane)(const F(ext_t) * e) { return (R*)calloc((size_t)e->pw * (size_t)e->ph, sizeof(R)); }

/* ------------------------------------------------------------------ RCD */
#define AT(p, x, y) (p)[(size_t)((y) + M) * pw + ((x) + M)]
#define CC(x, y) AT(c, x, y)

/* Squared 7-tap high-pass (1, -3, -1, 6, -1, -3, 1) through (x, y) along
 * direction (dx, dy). */
static R F(rcd_hpf)(const R* c, int pw, int M, int x, int y, int dx, int dy) {
    const R t1 = ((CC(x - 3 * dx, y - 3 * dy) - CC(x - dx, y - dy)) - CC(x + dx, y + dy)) + CC(x + 3 * dx, y + 3 * dy);
    const R t2 = (R)3 * (CC(x - 2 * dx, y - 2 * dy) + CC(x + 2 * dx, y + 2 * dy));
    const R t = (t1 - t2) + (R)6 * CC(x, y);
    return t * t;
}

/* Discrimination between the directions (dx1, dy1) and (dx2, dy2): s1 / (s1 + s2),
 * s = max(epssq, three squared high-passes along the direction). */
static R F(rcd_dir)(const R* c, int pw, int M, int x, int y, int dx1, int dy1, int dx2, int dy2) {
    const R eps2 = (R)1e-10;
    const R s1 = F(maxr)(eps2, (F(rcd_hpf)(c, pw, M, x - dx1, y - dy1, dx1, dy1) + F(rcd_hpf)(c, pw, M, x, y, dx1, dy1)) +
                                   F(rcd_hpf)(c, pw, M, x + dx1, y + dy1, dx1, dy1));
    const R s2 = F(maxr)(eps2, (F(rcd_hpf)(c, pw, M, x - dx2, y - dy2, dx2, dy2) + F(rcd_hpf)(c, pw, M, x, y, dx2, dy2)) +
                                   F(rcd_hpf)(c, pw, M, x + dx2, y + dy2, dx2, dy2));
    return s1 / (s1 + s2);
}

/* The refined discrimination: the centre value, or the mean of the four
 * diagonal neighbours when that is further from 0.5. */
static R F(disc)(const R* d, int pw, int M, int x, int y) {
    const R ctr = AT(d, x, y);
    const R nb = (R)0.25 * (((AT(d, x - 1, y - 1) + AT(d, x + 1, y - 1)) + AT(d, x - 1, y + 1)) + AT(d, x + 1, y + 1));
    return F(absr)((R)0.5 - ctr) < F(absr)((R)0.5 - nb) ? nb : ctr;
}

static R F(intp)(R a, R b, R c) { return (a * b) + (((R)1 - a) * c); }

int F(oracle_rcd_full)(const float* in, int w, int h, const uint8_t cfa4[4], R* rgb) {
    const int M = 12;
    F(ext_t) e;
    if (F(ext_make)(&e, in, w, h, M)) return -1;
    const int pw = e.pw;
    const R* c = e.v;
    R *vh = F(plane)(&e), *lpf = F(plane)(&e), *pq = F(plane)(&e), *g = F(plane)(&e), *rb = F(plane)(&e);
    if (!vh || !lpf || !pq || !g || !rb) return -1;
    const R eps = (R)1e-5;
    /* 1: vertical / horizontal discrimination; 4.1: diagonal discrimination */
    for (int y = -7; y < h + 7; ++y)
        for (int x = -7; x < w + 7; ++x) {
            AT(vh, x, y) = F(rcd_dir)(c, pw, M, x, y, 0, 1, 1, 0);
            AT(pq, x, y) = F(rcd_dir)(c, pw, M, x, y, 1, 1, -1, 1);
        }
    /* 2: low-pass of the mosaic */
    for (int y = -9; y < h + 9; ++y)
        for (int x = -9; x < w + 9; ++x)
            AT(lpf, x, y) = (((R)0.25 * CC(x, y)) +
                             ((R)0.125 * (((CC(x, y - 1) + CC(x, y + 1)) + CC(x - 1, y)) + CC(x + 1, y)))) +
                            ((R)0.0625 * (((CC(x - 1, y - 1) + CC(x + 1, y - 1)) + CC(x - 1, y + 1)) + CC(x + 1, y + 1)));
    /* 3: green at red and blue sites */
    for (int y = -6; y < h + 6; ++y)
        for (int x = -6; x < w + 6; ++x) {
            if (dm_color(cfa4, x, y) == 1) {
                AT(g, x, y) = CC(x, y);
                continue;
            }
            const R l0 = AT(lpf, x, y);
            const R gn = (((eps + F(absr)(CC(x, y - 1) - CC(x, y + 1))) + F(absr)(CC(x, y) - CC(x, y - 2))) +
                          F(absr)(CC(x, y - 1) - CC(x, y - 3))) + F(absr)(CC(x, y - 2) - CC(x, y - 4));
            const R gs = (((eps + F(absr)(CC(x, y - 1) - CC(x, y + 1))) + F(absr)(CC(x, y) - CC(x, y + 2))) +
                          F(absr)(CC(x, y + 1) - CC(x, y + 3))) + F(absr)(CC(x, y + 2) - CC(x, y + 4));
            const R gw = (((eps + F(absr)(CC(x - 1, y) - CC(x + 1, y))) + F(absr)(CC(x, y) - CC(x - 2, y))) +
                          F(absr)(CC(x - 1, y) - CC(x - 3, y))) + F(absr)(CC(x - 2, y) - CC(x - 4, y));
            const R ge = (((eps + F(absr)(CC(x - 1, y) - CC(x + 1, y))) + F(absr)(CC(x, y) - CC(x + 2, y))) +
                          F(absr)(CC(x + 1, y) - CC(x + 3, y))) + F(absr)(CC(x + 2, y) - CC(x + 4, y));
            const R en = (CC(x, y - 1) * (l0 + l0)) / ((eps + l0) + AT(lpf, x, y - 2));
            const R es = (CC(x, y + 1) * (l0 + l0)) / ((eps + l0) + AT(lpf, x, y + 2));
            const R ew = (CC(x - 1, y) * (l0 + l0)) / ((eps + l0) + AT(lpf, x - 2, y));
            const R ee = (CC(x + 1, y) * (l0 + l0)) / ((eps + l0) + AT(lpf, x + 2, y));
            const R ve = ((gs * en) + (gn * es)) / (gn + gs);
            const R he = ((ge * ew) + (gw * ee)) / (gw + ge);
            AT(g, x, y) = F(intp)(F(disc)(vh, pw, M, x, y), he, ve);
        }
    /* 4.2: blue at red sites and red at blue sites */
    for (int y = -4; y < h + 4; ++y)
        for (int x = -4; x < w + 4; ++x) {
            if (dm_color(cfa4, x, y) == 1) continue;
            const R g0 = AT(g, x, y);
            const R gnw = ((eps + F(absr)(CC(x - 1, y - 1) - CC(x + 1, y + 1))) + F(absr)(CC(x - 1, y - 1) - CC(x - 3, y - 3))) +
                          F(absr)(g0 - AT(g, x - 2, y - 2));
            const R gne = ((eps + F(absr)(CC(x + 1, y - 1) - CC(x - 1, y + 1))) + F(absr)(CC(x + 1, y - 1) - CC(x + 3, y - 3))) +
                          F(absr)(g0 - AT(g, x + 2, y - 2));
            const R gsw = ((eps + F(absr)(CC(x + 1, y - 1) - CC(x - 1, y + 1))) + F(absr)(CC(x - 1, y + 1) - CC(x - 3, y + 3))) +
                          F(absr)(g0 - AT(g, x - 2, y + 2));
            const R gse = ((eps + F(absr)(CC(x - 1, y - 1) - CC(x + 1, y + 1))) + F(absr)(CC(x + 1, y + 1) - CC(x + 3, y + 3))) +
                          F(absr)(g0 - AT(g, x + 2, y + 2));
            const R enw = CC(x - 1, y - 1) - AT(g, x - 1, y - 1);
            const R ene = CC(x + 1, y - 1) - AT(g, x + 1, y - 1);
            const R esw = CC(x - 1, y + 1) - AT(g, x - 1, y + 1);
            const R ese = CC(x + 1, y + 1) - AT(g, x + 1, y + 1);
            const R pe = ((gse * enw) + (gnw * ese)) / (gnw + gse);
            const R qe = ((gsw * ene) + (gne * esw)) / (gne + gsw);
            AT(rb, x, y) = g0 + F(intp)(F(disc)(pq, pw, M, x, y), qe, pe);
        }
    /* 4.3: red and blue at green sites; assemble */
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const int site = dm_color(cfa4, x, y);
            R out[3];
            const R g0 = AT(g, x, y);
            out[1] = g0;
            if (site != 1) {
                out[site] = CC(x, y);
                out[2 - site] = AT(rb, x, y);
            } else {
                const R d = F(disc)(vh, pw, M, x, y);
                for (int k = 0; k <= 2; k += 2) {
                    /* k at a red/blue site (x + dx, y + dy): the CFA value there, or
                     * the step-4.2 value where that site holds the other colour */
#define XK(dx, dy) (dm_color(cfa4, x + (dx), y + (dy)) == k ? CC(x + (dx), y + (dy)) : AT(rb, x + (dx), y + (dy)))
                    const R gn = ((eps + F(absr)(g0 - AT(g, x, y - 2))) + F(absr)(XK(0, -1) - XK(0, 1))) +
                                 F(absr)(XK(0, -1) - XK(0, -3));
                    const R gs = ((eps + F(absr)(g0 - AT(g, x, y + 2))) + F(absr)(XK(0, 1) - XK(0, -1))) +
                                 F(absr)(XK(0, 1) - XK(0, 3));
                    const R gw = ((eps + F(absr)(g0 - AT(g, x - 2, y))) + F(absr)(XK(-1, 0) - XK(1, 0))) +
                                 F(absr)(XK(-1, 0) - XK(-3, 0));
                    const R ge = ((eps + F(absr)(g0 - AT(g, x + 2, y))) + F(absr)(XK(1, 0) - XK(-1, 0))) +
                                 F(absr)(XK(1, 0) - XK(3, 0));
                    const R en = XK(0, -1) - AT(g, x, y - 1);
                    const R es = XK(0, 1) - AT(g, x, y + 1);
                    const R ew = XK(-1, 0) - AT(g, x - 1, y);
                    const R ee = XK(1, 0) - AT(g, x + 1, y);
#undef XK
                    const R ve = ((gs * en) + (gn * es)) / (gn + gs);
                    const R he = ((ge * ew) + (gw * ee)) / (gw + ge);
                    out[k] = g0 + F(intp)(d, he, ve);
                }
            }
            for (int k = 0; k < 3; ++k) rgb[3 * ((size_t)y * w + x) + k] = F(maxr)((R)0, out[k]);
        }
    free(e.v);
    free(vh);
    free(lpf);
    free(pq);
    free(g);
    free(rb);
    return 0;
}

/* ---------------------------------------------------------------- AMaZE */
int F(oracle_amaze_full)(const float* in, int w, int h, const uint8_t cfa4[4], R* rgb) {
    const int M = 24;
    F(ext_t) e;
    if (F(ext_make)(&e, in, w, h, M)) return -1;
    const int pw = e.pw;
    const R* c = e.v;
    const R eps = (R)1e-5, eps2 = (R)1e-10, arthresh = (R)0.75, clip8 = (R)0.8;
    R *dw0 = F(plane)(&e), *dw1 = F(plane)(&e), *dhv = F(plane)(&e), *vcd = F(plane)(&e), *hcd = F(plane)(&e);
    R *dgv = F(plane)(&e), *dgh = F(plane)(&e), *hvw = F(plane)(&e), *hve = F(plane)(&e), *cdsq = F(plane)(&e);
    R *g = F(plane)(&e), *dg = F(plane)(&e), *cvh = F(plane)(&e), *cvv = F(plane)(&e), *hvf = F(plane)(&e);
    R* cdo = F(plane)(&e);
    unsigned char* nyq = (unsigned char*)calloc((size_t)e.pw * e.ph, 1);
    unsigned char* nyq2 = (unsigned char*)calloc((size_t)e.pw * e.ph, 1);
    if (!dw0 || !dw1 || !dhv || !vcd || !hcd || !dgv || !dgh || !hvw || !hve || !cdsq || !g || !dg || !cvh || !cvv ||
        !hvf || !cdo || !nyq || !nyq2)
        return -1;
    R wodd[4], wgrad[6], wquinc[4];
    F(amaze_weights)(wodd, wgrad, wquinc);
    /* A: gradients and directional weights */
    for (int y = -22; y < h + 22; ++y)
        for (int x = -22; x < w + 22; ++x) {
            const R dh = F(absr)(CC(x + 1, y) - CC(x - 1, y));
            const R dv = F(absr)(CC(x, y + 1) - CC(x, y - 1));
            AT(dw0, x, y) = ((eps + F(absr)(CC(x, y + 2) - CC(x, y))) + F(absr)(CC(x, y) - CC(x, y - 2))) + dv;
            AT(dw1, x, y) = ((eps + F(absr)(CC(x + 2, y) - CC(x, y))) + F(absr)(CC(x, y) - CC(x - 2, y))) + dh;
            AT(dhv, x, y) = (dh * dh) + (dv * dv);
        }
    /* B: colour differences (green minus the site's other colour) from
     * Hamilton-Adams and adaptive-ratio estimates, with highlight protection */
    for (int y = -20; y < h + 20; ++y)
        for (int x = -20; x < w + 20; ++x) {
            const R c0 = CC(x, y);
            const R sgn = dm_color(cfa4, x, y) == 1 ? (R)-1 : (R)1;
            const R d0 = AT(dw0, x, y), d1 = AT(dw1, x, y);
            const R cru = (CC(x, y - 1) * (AT(dw0, x, y - 2) + d0)) /
                          ((AT(dw0, x, y - 2) * (eps + c0)) + (d0 * (eps + CC(x, y - 2))));
            const R crd = (CC(x, y + 1) * (AT(dw0, x, y + 2) + d0)) /
                          ((AT(dw0, x, y + 2) * (eps + c0)) + (d0 * (eps + CC(x, y + 2))));
            const R crl = (CC(x - 1, y) * (AT(dw1, x - 2, y) + d1)) /
                          ((AT(dw1, x - 2, y) * (eps + c0)) + (d1 * (eps + CC(x - 2, y))));
            const R crr = (CC(x + 1, y) * (AT(dw1, x + 2, y) + d1)) /
                          ((AT(dw1, x + 2, y) * (eps + c0)) + (d1 * (eps + CC(x + 2, y))));
            const R guha = CC(x, y - 1) + ((R)0.5 * (c0 - CC(x, y - 2)));
            const R gdha = CC(x, y + 1) + ((R)0.5 * (c0 - CC(x, y + 2)));
            const R glha = CC(x - 1, y) + ((R)0.5 * (c0 - CC(x - 2, y)));
            const R grha = CC(x + 1, y) + ((R)0.5 * (c0 - CC(x + 2, y)));
            R guar = F(absr)((R)1 - cru) < arthresh ? c0 * cru : guha;
            R gdar = F(absr)((R)1 - crd) < arthresh ? c0 * crd : gdha;
            R glar = F(absr)((R)1 - crl) < arthresh ? c0 * crl : glha;
            R grar = F(absr)((R)1 - crr) < arthresh ? c0 * crr : grha;
            const R hwt = AT(dw1, x - 1, y) / (AT(dw1, x - 1, y) + AT(dw1, x + 1, y));
            const R vwt = AT(dw0, x, y - 1) / (AT(dw0, x, y + 1) + AT(dw0, x, y - 1));
            const R gvha = (vwt * gdha) + (((R)1 - vwt) * guha);
            const R ghha = (hwt * grha) + (((R)1 - hwt) * glha);
            R vc = sgn * (((vwt * gdar) + (((R)1 - vwt) * guar)) - c0);
            R hc = sgn * (((hwt * grar) + (((R)1 - hwt) * glar)) - c0);
            if (c0 > clip8 || gvha > clip8 || ghha > clip8) {
                guar = guha;
                gdar = gdha;
                glar = glha;
                grar = grha;
                vc = sgn * (gvha - c0);
                hc = sgn * (ghha - c0);
            }
            AT(vcd, x, y) = vc;
            AT(hcd, x, y) = hc;
            AT(dgv, x, y) = F(minr)((guha - gdha) * (guha - gdha), (guar - gdar) * (guar - gdar));
            AT(dgh, x, y) = F(minr)((glha - grha) * (glha - grha), (glar - grar) * (glar - grar));
            AT(cdsq, x, y) = (vc - hc) * (vc - hc);
        }
    /* C: vertical weight of the colour-difference interpolation, from the
     * colour-difference variances and the fluctuation of the estimates */
    for (int y = -10; y < h + 10; ++y)
        for (int x = -10; x < w + 10; ++x) {
            const R hwt = AT(dw1, x - 1, y) / (AT(dw1, x - 1, y) + AT(dw1, x + 1, y));
            const R vwt = AT(dw0, x, y - 1) / (AT(dw0, x, y + 1) + AT(dw0, x, y - 1));
            R su = (R)0, sd = (R)0, sl = (R)0, sr = (R)0;
            for (int k = 0; k < 4; ++k) {
                su = su + AT(vcd, x, y - k);
                sd = sd + AT(vcd, x, y + k);
                sl = sl + AT(hcd, x - k, y);
                sr = sr + AT(hcd, x + k, y);
            }
            const R mu = (R)0.25 * su, md = (R)0.25 * sd, ml = (R)0.25 * sl, mr = (R)0.25 * sr;
            R vu = (R)0, vd = (R)0, vl = (R)0, vr = (R)0;
            for (int k = 0; k < 4; ++k) {
                vu = vu + (AT(vcd, x, y - k) - mu) * (AT(vcd, x, y - k) - mu);
                vd = vd + (AT(vcd, x, y + k) - md) * (AT(vcd, x, y + k) - md);
                vl = vl + (AT(hcd, x - k, y) - ml) * (AT(hcd, x - k, y) - ml);
                vr = vr + (AT(hcd, x + k, y) - mr) * (AT(hcd, x + k, y) - mr);
            }
            const R vvar = (eps2 + (vwt * vd)) + (((R)1 - vwt) * vu);
            const R hvar = (eps2 + (hwt * vr)) + (((R)1 - hwt) * vl);
            const R fu = (AT(dgv, x, y) + AT(dgv, x, y - 1)) + AT(dgv, x, y - 2);
            const R fd = (AT(dgv, x, y) + AT(dgv, x, y + 1)) + AT(dgv, x, y + 2);
            const R fl = (AT(dgh, x, y) + AT(dgh, x - 1, y)) + AT(dgh, x - 2, y);
            const R fr = (AT(dgh, x, y) + AT(dgh, x + 1, y)) + AT(dgh, x + 2, y);
            const R vvar1 = (eps2 + (vwt * fd)) + (((R)1 - vwt) * fu);
            const R hvar1 = (eps2 + (hwt * fr)) + (((R)1 - hwt) * fl);
            const R varwt = hvar / (vvar + hvar);
            const R diffwt = hvar1 / (vvar1 + hvar1);
            AT(hvw, x, y) = (((R)0.5 - varwt) * ((R)0.5 - diffwt) > (R)0 &&
                             F(absr)((R)0.5 - diffwt) < F(absr)((R)0.5 - varwt))
                                ? varwt
                                : diffwt;
        }
    /* D: Nyquist texture test at red/blue sites, then a majority vote of the
     * eight same-lattice neighbours */
    for (int y = -15; y < h + 15; ++y)
        for (int x = -15; x < w + 15; ++x) {
            if (dm_color(cfa4, x, y) == 1) continue;
            R a = wodd[0] * AT(cdsq, x, y);
            a = a + wodd[1] * (((AT(cdsq, x - 1, y - 1) + AT(cdsq, x + 1, y - 1)) + AT(cdsq, x - 1, y + 1)) + AT(cdsq, x + 1, y + 1));
            a = a + wodd[2] * (((AT(cdsq, x, y - 2) + AT(cdsq, x - 2, y)) + AT(cdsq, x + 2, y)) + AT(cdsq, x, y + 2));
            a = a + wodd[3] * (((AT(cdsq, x - 2, y - 2) + AT(cdsq, x + 2, y - 2)) + AT(cdsq, x - 2, y + 2)) + AT(cdsq, x + 2, y + 2));
            R b = wgrad[0] * AT(dhv, x, y);
            b = b + wgrad[1] * (((AT(dhv, x, y - 1) + AT(dhv, x - 1, y)) + AT(dhv, x + 1, y)) + AT(dhv, x, y + 1));
            b = b + wgrad[2] * (((AT(dhv, x - 1, y - 1) + AT(dhv, x + 1, y - 1)) + AT(dhv, x - 1, y + 1)) + AT(dhv, x + 1, y + 1));
            b = b + wgrad[3] * (((AT(dhv, x, y - 2) + AT(dhv, x - 2, y)) + AT(dhv, x + 2, y)) + AT(dhv, x, y + 2));
            b = b + wgrad[4] * (((((((AT(dhv, x - 1, y - 2) + AT(dhv, x + 1, y - 2)) + AT(dhv, x - 2, y - 1)) +
                                    AT(dhv, x + 2, y - 1)) + AT(dhv, x - 2, y + 1)) + AT(dhv, x + 2, y + 1)) +
                                 AT(dhv, x - 1, y + 2)) + AT(dhv, x + 1, y + 2));
            b = b + wgrad[5] * (((AT(dhv, x - 2, y - 2) + AT(dhv, x + 2, y - 2)) + AT(dhv, x - 2, y + 2)) + AT(dhv, x + 2, y + 2));
            AT(nyq, x, y) = (a - b) > (R)0 ? 1 : 0;
        }
    for (int y = -13; y < h + 13; ++y)
        for (int x = -13; x < w + 13; ++x) {
            if (dm_color(cfa4, x, y) == 1) continue;
            const int s = AT(nyq, x - 1, y - 1) + AT(nyq, x + 1, y - 1) + AT(nyq, x - 1, y + 1) + AT(nyq, x + 1, y + 1) +
                          AT(nyq, x, y - 2) + AT(nyq, x - 2, y) + AT(nyq, x + 2, y) + AT(nyq, x, y + 2);
            AT(nyq2, x, y) = s > 4 ? 1 : (s < 4 ? 0 : AT(nyq, x, y));
        }
    /* E: in Nyquist areas, the weight from the same-colour sites' area statistics */
    for (int y = -7; y < h + 7; ++y)
        for (int x = -7; x < w + 7; ++x) {
            if (dm_color(cfa4, x, y) == 1) continue;
            R hv = AT(hvw, x, y);
            if (AT(nyq2, x, y)) {
                R sh = (R)0, sv = (R)0, qh = (R)0, qv = (R)0, n = (R)0;
                for (int i = -6; i <= 6; i += 2)
                    for (int j = -6; j <= 6; j += 2) {
                        const int qx = x + j, qy = y + i;
                        if (!AT(nyq2, qx, qy)) continue;
                        const R q0 = CC(qx, qy);
                        sh = sh + (q0 - (R)0.5 * (CC(qx - 1, qy) + CC(qx + 1, qy)));
                        sv = sv + (q0 - (R)0.5 * (CC(qx, qy - 1) + CC(qx, qy + 1)));
                        qh = qh + (R)0.5 * ((q0 - CC(qx - 1, qy)) * (q0 - CC(qx - 1, qy)) +
                                            (q0 - CC(qx + 1, qy)) * (q0 - CC(qx + 1, qy)));
                        qv = qv + (R)0.5 * ((q0 - CC(qx, qy - 1)) * (q0 - CC(qx, qy - 1)) +
                                            (q0 - CC(qx, qy + 1)) * (q0 - CC(qx, qy + 1)));
                        n = n + (R)1;
                    }
                const R hvar = eps2 + F(absr)((n * qh) - (sh * sh));
                const R vvar = eps2 + F(absr)((n * qv) - (sv * sv));
                hv = hvar / (vvar + hvar);
            }
            AT(hve, x, y) = hv;
        }
    /* F: the weight refined from the diagonal neighbours; green; curvatures */
    for (int y = -6; y < h + 6; ++y)
        for (int x = -6; x < w + 6; ++x) {
            if (dm_color(cfa4, x, y) == 1) {
                AT(g, x, y) = CC(x, y);
                continue;
            }
            const R hv0 = AT(hve, x, y);
            const R alt = (R)0.25 * (((AT(hve, x - 1, y - 1) + AT(hve, x + 1, y - 1)) + AT(hve, x - 1, y + 1)) + AT(hve, x + 1, y + 1));
            const R hv = F(absr)((R)0.5 - hv0) < F(absr)((R)0.5 - alt) ? alt : hv0;
            AT(hvf, x, y) = hv;
            const R d = (AT(hcd, x, y) * ((R)1 - hv)) + (AT(vcd, x, y) * hv);
            AT(dg, x, y) = d;
            AT(g, x, y) = CC(x, y) + d;
        }
    for (int y = -6; y < h + 6; ++y)
        for (int x = -6; x < w + 6; ++x) {
            if (dm_color(cfa4, x, y) == 1 || !AT(nyq2, x, y)) continue;
            const R g0 = AT(g, x, y);
            const R th = g0 - (R)0.5 * (CC(x - 1, y) + CC(x + 1, y));
            const R tv = g0 - (R)0.5 * (CC(x, y - 1) + CC(x, y + 1));
            AT(cvh, x, y) = th * th;
            AT(cvv, x, y) = tv * tv;
        }
    /* G: green refined in Nyquist areas from the green curvatures */
    for (int y = -4; y < h + 4; ++y)
        for (int x = -4; x < w + 4; ++x) {
            if (dm_color(cfa4, x, y) == 1 || !AT(nyq2, x, y)) continue;
            R gh = wquinc[0] * AT(cvh, x, y), gv = wquinc[0] * AT(cvv, x, y);
            gh = gh + wquinc[1] * (((AT(cvh, x - 1, y - 1) + AT(cvh, x + 1, y - 1)) + AT(cvh, x - 1, y + 1)) + AT(cvh, x + 1, y + 1));
            gv = gv + wquinc[1] * (((AT(cvv, x - 1, y - 1) + AT(cvv, x + 1, y - 1)) + AT(cvv, x - 1, y + 1)) + AT(cvv, x + 1, y + 1));
            gh = gh + wquinc[2] * (((AT(cvh, x, y - 2) + AT(cvh, x - 2, y)) + AT(cvh, x + 2, y)) + AT(cvh, x, y + 2));
            gv = gv + wquinc[2] * (((AT(cvv, x, y - 2) + AT(cvv, x - 2, y)) + AT(cvv, x + 2, y)) + AT(cvv, x, y + 2));
            gh = gh + wquinc[3] * (((AT(cvh, x - 2, y - 2) + AT(cvh, x + 2, y - 2)) + AT(cvh, x - 2, y + 2)) + AT(cvh, x + 2, y + 2));
            gv = gv + wquinc[3] * (((AT(cvv, x - 2, y - 2) + AT(cvv, x + 2, y - 2)) + AT(cvv, x - 2, y + 2)) + AT(cvv, x + 2, y + 2));
            gh = eps2 + gh;
            gv = eps2 + gv;
            const R d = ((AT(hcd, x, y) * gv) + (AT(vcd, x, y) * gh)) / (gv + gh);
            AT(dg, x, y) = d;
            AT(g, x, y) = CC(x, y) + d;
        }
    /* H: the other colour's difference at red/blue sites, from the four
     * diagonal directions */
    for (int y = -1; y < h + 1; ++y)
        for (int x = -1; x < w + 1; ++x) {
            if (dm_color(cfa4, x, y) == 1) continue;
            R num = (R)0, den = (R)0;
            for (int k = 0; k < 4; ++k) {
                const int dx = (k & 1) ? 1 : -1, dy = (k & 2) ? 1 : -1;
                const R d1 = AT(dg, x + dx, y + dy), dm = AT(dg, x - dx, y - dy), d3 = AT(dg, x + 3 * dx, y + 3 * dy);
                const R wt = (R)1 / (((eps + F(absr)(d1 - dm)) + F(absr)(d1 - d3)) + F(absr)(dm - d3));
                const R est = (((R)1.325 * d1) - ((R)0.175 * d3)) - ((R)0.075 * AT(dg, x + 3 * dx, y + dy)) -
                              ((R)0.075 * AT(dg, x + dx, y + 3 * dy));
                num = num + wt * est;
                den = den + wt;
            }
            AT(cdo, x, y) = num / den;
        }
    /* I: red and blue at green sites from the four cardinal neighbours, weighted
     * by their vertical weight; assemble */
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const int site = dm_color(cfa4, x, y);
            const R g0 = AT(g, x, y);
            R out[3];
            out[1] = g0;
            if (site != 1) {
                out[site] = CC(x, y);
                out[2 - site] = g0 - AT(cdo, x, y);
            } else {
                const R wn = AT(hvf, x, y - 1), ws = AT(hvf, x, y + 1);
                const R ww = (R)1 - AT(hvf, x - 1, y), we = (R)1 - AT(hvf, x + 1, y);
                const R t = (R)1 / (((wn + we) + ww) + ws);
                for (int k = 0; k <= 2; k += 2) {
#define CDK(dx, dy) (dm_color(cfa4, x + (dx), y + (dy)) == k ? AT(dg, x + (dx), y + (dy)) : AT(cdo, x + (dx), y + (dy)))
                    const R s = (((wn * CDK(0, -1)) + (we * CDK(1, 0))) + (ww * CDK(-1, 0))) + (ws * CDK(0, 1));
#undef CDK
                    out[k] = g0 - (s * t);
                }
            }
            for (int k = 0; k < 3; ++k) rgb[3 * ((size_t)y * w + x) + k] = F(maxr)((R)0, out[k]);
        }
    free(e.v);
    R* planes[] = {dw0, dw1, dhv, vcd, hcd, dgv, dgh, hvw, hve, cdsq, g, dg, cvh, cvv, hvf, cdo};
    for (size_t i = 0; i < sizeof(planes) / sizeof(planes[0]); ++i) free(planes[i]);
    free(nyq);
    free(nyq2);
    return 0;
}

#undef CC
#undef AT
#undef F
#undef CAT
#undef CAT2
