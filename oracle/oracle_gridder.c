/*
 * ORACLE — test infrastructure only.  Nothing in the product links or calls
 * this file; it is the CPU checker that the CUDA gridder is compared against,
 * and the CPU baseline that bench.py times beside it.
 *
 * A single-threaded C restatement of yandasoft's table-based visibility
 * gridder hot loop, with the same FP32/FP64 arithmetic as the reference:
 *
 *   - askap::nint (un-vendored base-askap 1.6.0): round half away from zero
 *     by adding +-0.5 in double and truncating.  Call sites:
 *     askap/gridding/TableVisGridder.cc:617-618,635-636,
 *     askap/gridding/WDependentGridderBase.cc:124,127.
 *   - uv-cell / oversample index block: TableVisGridder.cc:604-650.
 *   - w -> plane mapping (linear, power-law, gaussian sampling):
 *     WDependentGridderBase.cc:53-67,118-170; PowerWSampling.cc:60-80;
 *     GaussianWSampling.cc:70-167 (and GaussianWSampling.h:103-104).
 *   - the generic grid/degrid loop, including weights, sum of weights, the
 *     PSF branch, the strict on-grid test and the degrid write-back:
 *     TableVisGridder.cc:451-884.
 *   - GridKernel::grid / GridKernel::degrid pointer path:
 *     askap/gridding/GridKernel.cc:57-137.
 *
 * Complex arithmetic is written out component-wise exactly as
 * -fcx-limited-range evaluates it (CMakeLists.txt:181-183); compile with
 * -ffp-contract=off so that no product is fused into an FMA.
 *
 * Polarisation conversion is the identity (vis and image polarisation frames
 * equal), so scimath::PolConverter is not restated.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdio.h>
#include <stdlib.h>

#define ORC_C 299792458.0
#define ORC_PI 3.14159265358979323846

/* error codes shared with the python wrapper */
#define ORC_OK 0
#define ORC_ERR_FREQ 1
#define ORC_ERR_FRAC 2
#define ORC_ERR_WRANGE 3
#define ORC_ERR_CINDEX 4
#define ORC_ERR_GINDEX 5
#define ORC_ERR_WEIGHT 6
#define ORC_ERR_SUMW 7
#define ORC_ERR_CFSHAPE 8

static char orc_errmsg[512];
const char *orc_last_error(void) { return orc_errmsg; }

/* askap::nint(double): x>0 ? int(x+0.5) : int(x-0.5) */
int orc_nint(double x)
{
    return x > 0 ? (int)(x + 0.5) : (int)(x - 0.5);
}

/* ---------------------------------------------------------------------- */
/* w sampling                                                             */
/* ---------------------------------------------------------------------- */
enum { ORC_WS_LINEAR = 0, ORC_WS_POWER = 1, ORC_WS_GAUSS = 2 };

typedef struct {
    int nwplanes;
    double wscale;     /* wmax / ((n-1)/2), or 1 if n == 1 */
    int sampling;      /* ORC_WS_* */
    double exponent;   /* power law */
    double two_sigma2; /* gaussian */
    double amplitude;  /* gaussian */
    int wmaxclip;
} orc_wcfg;

/* Returns the index function of the non-linear sampling, FP64. */
static double orc_ws_index(const orc_wcfg *c, double wterm, int *err)
{
    if (c->sampling == ORC_WS_POWER) {
        if (wterm > 0) return pow(wterm, 1. / c->exponent);
        if (wterm < 0) return -pow(-wterm, 1. / c->exponent);
        return 0.;
    }
    /* gaussian */
    if (wterm == -1. || wterm == 1.) return wterm;
    {
        const double expterm = 1. - fabs(wterm) / c->amplitude;
        double plane2;
        if (!(expterm > 0.)) { *err = ORC_ERR_WRANGE; return 0.; }
        plane2 = -log(expterm) * c->two_sigma2;
        if (!(plane2 >= 0.)) { *err = ORC_ERR_WRANGE; return 0.; }
        if (wterm < 0) return -sqrt(plane2);
        if (wterm > 0) return sqrt(plane2);
        return 0.;
    }
}

double orc_ws_map(int sampling, double exponent, double two_sigma2, double amplitude, double plane)
{
    if (sampling == ORC_WS_POWER) {
        if (plane > 0) return pow(plane, exponent);
        if (plane < 0) return -pow(-plane, exponent);
        return 0.;
    } else {
        const double a = amplitude * (1 - exp(-plane * plane / two_sigma2));
        if (plane < 0) return -a;
        if (plane > 0) return a;
        return 0.;
    }
}

double orc_ws_index_pub(int sampling, double exponent, double two_sigma2, double amplitude, double wterm)
{
    orc_wcfg c;
    int err = 0;
    memset(&c, 0, sizeof(c));
    c.sampling = sampling; c.exponent = exponent; c.two_sigma2 = two_sigma2; c.amplitude = amplitude;
    return orc_ws_index(&c, wterm, &err);
}

/* GaussianWSampling::calculateDistributionParameters: bisection for 2 sigma^2 */
static double orc_gauss_target(double ts2)
{
    return sqrt(-ts2 * log(0.5 + 0.5 * exp(-1. / ts2)));
}

int orc_gauss_params(double wplanes50, double *two_sigma2, double *amplitude)
{
    double lo, hi, ts2 = 1.;
    size_t it;
    if (!(wplanes50 > 0) || !(wplanes50 * sqrt(2) < 1.)) return ORC_ERR_WRANGE;
    lo = wplanes50 * wplanes50 / log(2.) / 2.;
    hi = 0.2 / (1 / sqrt(2) - wplanes50);
    if (hi < lo) { lo = hi; hi = 5.; }
    for (it = 0; it < 100; ++it) {
        ts2 = (lo + hi) / 2.;
        if (orc_gauss_target(ts2) < wplanes50) lo = ts2; else hi = ts2;
        if (hi - lo < 1e-5) break;
    }
    *two_sigma2 = ts2;
    *amplitude = 1. / (1. - exp(-1. / ts2));
    return ORC_OK;
}

/* WDependentGridderBase::getWPlane. Returns plane, -1 when clipped, sets err
 * when the reference would throw. */
static int orc_get_wplane(const orc_wcfg *c, double w, int *err)
{
    int result;
    if (c->sampling != ORC_WS_LINEAR && c->nwplanes > 1) {
        const int half = (c->nwplanes - 1) / 2;
        const double wmaxv = c->wscale * half;
        const double scaled = orc_ws_index(c, w / wmaxv, err);
        if (*err) return -1;
        result = half + orc_nint(scaled * half);
    } else {
        result = c->nwplanes > 1 ? (c->nwplanes - 1) / 2 + orc_nint(w / c->wscale) : 0;
    }
    if (result < c->nwplanes && result > -1) return result;
    if (!c->wmaxclip) {
        *err = ORC_ERR_WRANGE;
        snprintf(orc_errmsg, sizeof orc_errmsg,
                 "W scaling error: recommend allowing larger range of w, you have w=%.17g wavelengths", w);
    }
    return -1;
}

double orc_get_wterm(int nwplanes, double wscale, int sampling, double exponent,
                     double two_sigma2, double amplitude, int plane)
{
    const int half = (nwplanes - 1) / 2;
    if (sampling != ORC_WS_LINEAR && nwplanes > 1) {
        const double scaled = (double)(plane - half) / (double)half;
        return orc_ws_map(sampling, exponent, two_sigma2, amplitude, scaled) * (wscale * half);
    }
    return (double)(plane - half) * wscale;
}

/* itsCMap / itsGMap for the W gridders: plane = getWPlane(uvw(2)/C * freq)
 * (WProjectVisGridder.cc:136-146, WStackVisGridder.cc:82-95,
 * AWProjectVisGridder.cc:140-170).  map is (row, chan), row fastest.
 * For AWProject the caller adds the (chan, feed, field) offset. */
int orc_wplane_map(int64_t nrow, int nchan, const double *uvw, const double *freq,
                   int nwplanes, double wscale, int sampling, double exponent,
                   double two_sigma2, double amplitude, int wmaxclip, int32_t *map)
{
    orc_wcfg c;
    int64_t i;
    int ch, err = 0;
    c.nwplanes = nwplanes; c.wscale = wscale; c.sampling = sampling; c.exponent = exponent;
    c.two_sigma2 = two_sigma2; c.amplitude = amplitude; c.wmaxclip = wmaxclip;
    for (i = 0; i < nrow; ++i) {
        const double w = uvw[3 * i + 2] / ORC_C;
        for (ch = 0; ch < nchan; ++ch) {
            map[i + nrow * ch] = orc_get_wplane(&c, w * freq[ch], &err);
            if (err) return err;
        }
    }
    return ORC_OK;
}

/* W-stacking + W-projection composition: the grid plane is the w-stack of
 * w (WDependentGridderBase::getWPlane over the stack sampling), the CF plane
 * is getWPlane of the residual w - wterm(stack) over the projection sampling
 * (half a stack spacing).  gmap/cmap are (row, chan), row fastest. */
int orc_wstack_wproj_map(int64_t nrow, int nchan, const double *uvw, const double *freq,
                         int nstacks, double sscale, int swmaxclip,
                         int nwplanes, double wscale, int32_t *gmap, int32_t *cmap)
{
    orc_wcfg cs, cp;
    int64_t i;
    int ch, err = 0;
    memset(&cs, 0, sizeof cs);
    memset(&cp, 0, sizeof cp);
    cs.nwplanes = nstacks; cs.wscale = sscale; cs.sampling = ORC_WS_LINEAR; cs.wmaxclip = swmaxclip;
    cp.nwplanes = nwplanes; cp.wscale = wscale; cp.sampling = ORC_WS_LINEAR; cp.wmaxclip = 0;
    for (i = 0; i < nrow; ++i) {
        const double w = uvw[3 * i + 2] / ORC_C;
        for (ch = 0; ch < nchan; ++ch) {
            const double wf = w * freq[ch];
            const int g = orc_get_wplane(&cs, wf, &err);
            int c = -1;
            if (err) return err;
            if (g >= 0) {
                const int half = (nstacks - 1) / 2;
                const double wst = (double)(g - half) * sscale;
                c = orc_get_wplane(&cp, wf - wst, &err);
                if (err) return err;
            }
            gmap[i + nrow * ch] = g;
            cmap[i + nrow * ch] = c;
        }
    }
    return ORC_OK;
}

/* ---------------------------------------------------------------------- */
/* index block of TableVisGridder::generic                                */
/* ---------------------------------------------------------------------- */
static int orc_axis_index(double f, double coord, double cell, int os, int n,
                          int *pi, int *pfrac)
{
    const double scaled = f * coord / (ORC_C * cell);
    int i = orc_nint(scaled);
    int frac = orc_nint(os * ((double)i - scaled));
    if (frac < 0) { i += 1; frac += os; }
    else if (frac >= os) { i -= 1; frac -= os; }
    if (frac < 0 || frac >= os) {
        snprintf(orc_errmsg, sizeof orc_errmsg, "Fractional offset out of range, scaled=%.17g", scaled);
        return ORC_ERR_FRAC;
    }
    *pi = i + n / 2;
    *pfrac = frac;
    return ORC_OK;
}

/* Bit-exact cell and oversample offsets for every (row, chan); outputs are
 * (row, chan) arrays, row fastest. */
int orc_indices(int64_t nrow, int nchan, const double *uvw, const double *freq,
                double cellu, double cellv, int os, int nx, int ny,
                int32_t *iu, int32_t *iv, int32_t *fu, int32_t *fv)
{
    int64_t i;
    int ch, e;
    for (i = 0; i < nrow; ++i) {
        for (ch = 0; ch < nchan; ++ch) {
            const int64_t k = i + nrow * ch;
            e = orc_axis_index(freq[ch], uvw[3 * i + 0], cellu, os, nx, &iu[k], &fu[k]);
            if (e) return e;
            e = orc_axis_index(freq[ch], uvw[3 * i + 1], cellv, os, ny, &iv[k], &fv[k]);
            if (e) return e;
        }
    }
    return ORC_OK;
}

/* ---------------------------------------------------------------------- */
/* GridKernel (pointer path)                                              */
/* ---------------------------------------------------------------------- */
static void orc_grid_kernel(float *grid, int nx, const float *cf, float rv, float iv,
                            int iu, int ivv, int support)
{
    int sv, su;
    const int w = 2 * support + 1;
    for (sv = -support; sv <= support; ++sv) {
        const float *c = cf + 2 * (size_t)w * (size_t)(sv + support);
        float *g = grid + 2 * ((size_t)(iu - support) + (size_t)nx * (size_t)(ivv + sv));
        for (su = -support; su <= support; ++su, c += 2, g += 2) {
            const float t0 = rv * c[0];
            const float t1 = iv * c[1];
            const float t2 = rv * c[1];
            const float t3 = iv * c[0];
            g[0] += t0 - t1;
            g[1] += t2 + t3;
        }
    }
}

static void orc_degrid_kernel(float *out, const float *grid, int nx, const float *cf,
                              int iu, int ivv, int support)
{
    int sv, su;
    const int w = 2 * support + 1;
    float re = 0.f, im = 0.f;
    for (sv = -support; sv <= support; ++sv) {
        const float *c = cf + 2 * (size_t)w * (size_t)(sv + support);
        const float *g = grid + 2 * ((size_t)(iu - support) + (size_t)nx * (size_t)(ivv + sv));
        for (su = -support; su <= support; ++su, c += 2, g += 2) {
            const float a = c[0] * g[0];
            const float b = c[1] * g[1];
            const float d = -c[0] * g[1];
            const float e = c[1] * g[0];
            re += a + b;
            im += d + e;
        }
    }
    out[0] = re;
    out[1] = im;
}

/* The tap loops the generic loop calls: the restatements above by default;
 * the checker may install the reference's own compiled GridKernel
 * (oracle/_ref) through orc_set_tap_kernels to pin them (NULL restores
 * the restatements). */
typedef void (*orc_grid_fn)(float *, int, const float *, float, float, int, int, int);
typedef void (*orc_degrid_fn)(float *, const float *, int, const float *, int, int, int);
static orc_grid_fn orc_grid_tap = orc_grid_kernel;
static orc_degrid_fn orc_degrid_tap = orc_degrid_kernel;

void orc_set_tap_kernels(orc_grid_fn g, orc_degrid_fn d)
{
    orc_grid_tap = g ? g : orc_grid_kernel;
    orc_degrid_tap = d ? d : orc_degrid_kernel;
}

/* ---------------------------------------------------------------------- */
/* TableVisGridder::generic                                               */
/* ---------------------------------------------------------------------- */
typedef struct {
    int nx, ny;              /* padded grid shape */
    int npol;                /* image = vis polarisations (identity conversion) */
    int nchan_img;           /* image channels */
    int ngrids;              /* itsGrid.size() */
    double cellu, cellv;     /* uv cell size in wavelengths */
    int os;                  /* oversampling */
    int ncf;                 /* itsConvFunc.size() */
    const int32_t *cf_size;  /* nrow of each CF matrix (odd), 0 = empty */
    const int64_t *cf_off;   /* offset of each CF in complex elements */
    const float *cf_data;    /* complex64 data, each CF column-major */
    int noffsets;            /* itsConvFuncOffsets.size() */
    const int32_t *cf_offsets; /* (offU, offV) per plane before oversampling */
    int forward;             /* 1: degrid */
    int psf;                 /* PSF gridder */
    int track_per_os;        /* gridder.oversampleweight */
    int nsumw_rows;          /* itsSumWeights.shape()(0) */
    int pcf;                 /* preconditioner-function (PCF) gridder */
} orc_cfg;

typedef struct {
    double samples;   /* itsSamplesGridded / itsSamplesDegridded */
    double taps;      /* itsNumberGridded / itsNumberDegridded */
    double vectors_flagged;
    double vectors_wflagged;
} orc_stats;

/*
 * grids:  ngrids x (nx, ny, npol, nchan_img) complex64, column-major.
 * sumw:   (nsumw_rows, npol, nchan_img) double, column-major.
 * vis/noise: (nrow, nchan, npol) complex64 cubes, column-major (row fastest).
 * flag:   (nrow, nchan, npol) bytes.
 * cmap, gmap: (nrow, nchan) plane indices (row fastest).
 * chan_map: accessor channel -> image channel, -1 when unmapped.
 * row_ok:  NULL or per-row mask (MaxPointingSeparation).
 * psf_ok:  NULL or per-row mask (representative feed/field of the PSF).
 * mfs:     NULL or per-channel multi-frequency weight.
 * delay:   NULL or per-row delay (m) for the phasor.
 * carry:   npol complex values (itsImagePolFrameVis) kept across calls.
 */
int orc_generic(const orc_cfg *cfg, int64_t nrow, int nchan, int npol,
                const double *uvw, const double *delay, const double *freq,
                const int32_t *chan_map, const uint8_t *flag,
                float *vis, const float *noise,
                const int32_t *cmap, const int32_t *gmap,
                const uint8_t *row_ok, const uint8_t *psf_ok, const float *mfs,
                float *grids, double *sumw, float *carry, orc_stats *st,
                int64_t row_offset)
{
    const int os = cfg->os;
    const int64_t plane_cells = (int64_t)cfg->nx * cfg->ny;
    const int64_t grid_elems = plane_cells * cfg->npol * cfg->nchan_img;
    int64_t i;
    int ch, pol, e;
    float noisev[8][2];
    /* conjugate CF of the PCF branch: a buffer per thread, reused by every call */
    static __thread float *conj_cf = NULL;
    static __thread int conj_cap = 0;
    if (npol != cfg->npol || npol > 8) {
        snprintf(orc_errmsg, sizeof orc_errmsg, "only identity polarisation conversion is restated");
        return ORC_ERR_CINDEX;
    }
    for (i = 0; i < nrow; ++i) {
        if (row_ok && !row_ok[i]) continue;
        for (ch = 0; ch < nchan; ++ch) {
            const double f = freq[ch];
            int iu, iv, fracu, fracv, all_good = 1, wgood = 1;
            double phase;
            float ph_re, ph_im;
            const int64_t rc = i + nrow * ch;
            if (ch == 0) {
                const double r = f / ORC_C;
                if (!(r > 0.1 && r < 30000)) {
                    snprintf(orc_errmsg, sizeof orc_errmsg, "Check frequencies in the input file");
                    return ORC_ERR_FREQ;
                }
            }
            e = orc_axis_index(f, uvw[3 * i + 0], cfg->cellu, os, cfg->nx, &iu, &fracu);
            if (e) return e;
            e = orc_axis_index(f, uvw[3 * i + 1], cfg->cellv, os, cfg->ny, &iv, &fracv);
            if (e) return e;
            /* phase = 2.0f * pi * f * delay / c, evaluated in double */
            phase = 2.0 * ORC_PI * f * (delay ? delay[i] : 0.0) / ORC_C;
            ph_re = (float)cos(phase);
            ph_im = (float)sin(phase);
            for (pol = 0; pol < npol; ++pol) {
                if (flag[rc + nrow * (int64_t)nchan * pol]) { all_good = 0; break; }
            }
            if (!(all_good && chan_map[ch] >= 0)) {
                if (!cfg->forward) st->vectors_flagged += 1;
                continue;
            }
            {
                const int img_chan = chan_map[ch];
                if (!cfg->forward) {
                    for (pol = 0; pol < npol; ++pol) {
                        const int64_t k = rc + nrow * (int64_t)nchan * pol;
                        if (!cfg->psf) {
                            carry[2 * pol] = vis[2 * k];
                            carry[2 * pol + 1] = vis[2 * k + 1];
                        }
                        noisev[pol][0] = noise[2 * k];
                        noisev[pol][1] = noise[2 * k + 1];
                    }
                }
                for (pol = 0; pol < npol; ++pol) {
                    const int g_ind = gmap ? gmap[rc] : 0;
                    int plane, c_ind, support;
                    int off_u = 0, off_v = 0, iuo, ivo;
                    const float *cf;
                    float *grid;
                    if (g_ind < 0) { wgood = 0; st->vectors_wflagged += 1; break; }
                    if (g_ind >= cfg->ngrids) return ORC_ERR_GINDEX;
                    plane = cmap ? cmap[rc] : 0;
                    if (plane < 0) { wgood = 0; st->vectors_wflagged += 1; break; }
                    c_ind = fracu + os * (fracv + os * plane);
                    if (c_ind < 0 || c_ind >= cfg->ncf) {
                        snprintf(orc_errmsg, sizeof orc_errmsg, "Index into convolution functions out of range %d", c_ind);
                        return ORC_ERR_CINDEX;
                    }
                    if (cfg->cf_size[c_ind] % 2 != 1) return ORC_ERR_CFSHAPE;
                    support = (cfg->cf_size[c_ind] - 1) / 2;
                    if (cfg->cf_offsets && plane < cfg->noffsets) {
                        off_u = cfg->cf_offsets[2 * plane];
                        off_v = cfg->cf_offsets[2 * plane + 1];
                    }
                    iuo = iu + off_u;
                    ivo = iv + off_v;
                    if (!((iuo - support) > 0 && (ivo - support) > 0 &&
                          (iuo + support) < cfg->nx && (ivo + support) < cfg->ny)) continue;
                    cf = cfg->cf_data + 2 * cfg->cf_off[c_ind];
                    grid = grids + 2 * ((int64_t)g_ind * grid_elems + plane_cells * (pol + (int64_t)cfg->npol * img_chan));
                    if (cfg->forward) {
                        float cv[2], re, im;
                        orc_degrid_tap(cv, grid, cfg->nx, cf, iuo, ivo, support);
                        st->samples += 1.0;
                        st->taps += (double)((2 * support + 1) * (2 * support + 1));
                        if (mfs) { cv[0] *= mfs[ch]; cv[1] *= mfs[ch]; }
                        re = cv[0] * ph_re - cv[1] * ph_im;
                        im = cv[0] * ph_im + cv[1] * ph_re;
                        carry[2 * pol] = re;
                        carry[2 * pol + 1] = im;
                    } else {
                        const float nre = noisev[pol][0];
                        const float vn = nre * nre;
                        const float wt = (vn > 0.) ? (float)(1. / vn) : 0.f;
                        const int srow = cfg->track_per_os ? c_ind : plane;
                        double *sw;
                        if (!(wt > 0.)) {
                            snprintf(orc_errmsg, sizeof orc_errmsg, "Weight is supposed to be a positive number");
                            return ORC_ERR_WEIGHT;
                        }
                        if (srow >= cfg->nsumw_rows) return ORC_ERR_SUMW;
                        sw = sumw + srow + (int64_t)cfg->nsumw_rows * (pol + (int64_t)cfg->npol * img_chan);
                        if (!cfg->psf && !cfg->pcf) {
                            /* rVis = phasor * conj(vis) * wt */
                            const float vr = carry[2 * pol], vi = -carry[2 * pol + 1];
                            float rr = ph_re * vr - ph_im * vi;
                            float ri = ph_re * vi + ph_im * vr;
                            rr *= wt; ri *= wt;
                            if (mfs) { rr *= mfs[ch]; ri *= mfs[ch]; }
                            orc_grid_tap(grid, cfg->nx, cf, rr, ri, iuo, ivo, support);
                            st->samples += 1.0;
                            st->taps += (double)((2 * support + 1) * (2 * support + 1));
                            *sw += wt;
                        }
                        if (cfg->psf && (!psf_ok || psf_ok[i])) {
                            float ur = 1.f * wt, ui = 0.f * wt;
                            if (mfs) { ur *= mfs[ch]; ui *= mfs[ch]; }
                            orc_grid_tap(grid, cfg->nx, cf, ur, ui, iuo, ivo, support);
                            st->samples += 1.0;
                            st->taps += (double)((2 * support + 1) * (2 * support + 1));
                            *sw += wt;
                        }
                        if (cfg->pcf) {
                            /* uVis = wt (no MFS weight); the conjugate CF on one
                             * half of the uv plane, so that the w information
                             * kept in the imaginary part adds with conjugate
                             * symmetry; no sum of weights */
                            const float ur = 1.f * wt, ui = 0.f * wt;
                            const int w = 2 * support + 1;
                            if ((ivo < cfg->ny / 2 && iuo >= cfg->nx / 2) || (ivo <= cfg->ny / 2 && iuo < cfg->nx / 2)) {
                                int k;
                                if (conj_cap < w * w) {
                                    free(conj_cf);
                                    conj_cap = w * w;
                                    conj_cf = (float *)malloc(sizeof(float) * 2 * (size_t)conj_cap);
                                    if (!conj_cf) { conj_cap = 0; return ORC_ERR_CINDEX; }
                                }
                                for (k = 0; k < w * w; ++k) {
                                    conj_cf[2 * k] = cf[2 * k];
                                    conj_cf[2 * k + 1] = -cf[2 * k + 1];
                                }
                                orc_grid_tap(grid, cfg->nx, conj_cf, ur, ui, iuo, ivo, support);
                            } else {
                                orc_grid_tap(grid, cfg->nx, cf, ur, ui, iuo, ivo, support);
                            }
                            st->samples += 1.0;
                            st->taps += (double)(w * w);
                        }
                    }
                }
                if (wgood) {
                    if (cfg->forward) {
                        for (pol = 0; pol < npol; ++pol) {
                            const int64_t k = (row_offset + i) + nrow * (ch + (int64_t)nchan * pol);
                            vis[2 * k] += carry[2 * pol];
                            vis[2 * k + 1] += carry[2 * pol + 1];
                        }
                    }
                } else if (!cfg->forward) {
                    st->vectors_wflagged += 1;
                }
            }
        }
    }
    return ORC_OK;
}
