/*
 * ORACLE — test infrastructure only.  FP64 direct-DFT measurement equation.
 *
 * V(row, chan) = sum_k S_k(f) * D_k(row, f) * exp(+i * 2 pi f / c *
 *                (l_k u + m_k v + (n_k - 1) w)),    n_k = sqrt(1 - l_k^2 - m_k^2)
 *
 * following UnpolarizedPointSource::calcPoint
 * (askap/measurementequation/UnpolarizedPointSource.cc:80-107) and, for
 * Gaussian components, the decorrelation factor of
 * UnpolarizedGaussianSource::calcGaussian
 * (askap/measurementequation/UnpolarizedGaussianSource.cc:126-160):
 *   D = exp(-r f^2), r = (bmaj^2 up^2 + bmin^2 vp^2) pi^2 / (4 ln 2),
 *   up = (cos(bpa) u + sin(bpa) v)/c,  vp = (-sin(bpa) u + cos(bpa) v)/c.
 * S_k(f) = flux0 (f/ref)^alpha.  An optional per-(row, component) gain
 * (e.g. a primary-beam attenuation) multiplies S.
 *
 * uvw in metres (row-major [u v w]); output column-major (row fastest) per
 * channel, complex double interleaved.  Threads split rows.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

#define DFT_C 299792458.0
#define DFT_2PI 6.28318530717958647692

typedef struct {
    int64_t r0, r1, nrow;
    int nchan, ncomp;
    const double *uvw, *freq, *comp; /* comp: ncomp x 8 (flux, l, m, bmaj, bmin, bpa, si, reffreq) */
    const double *gain;              /* NULL or (ncomp, nrow, nchan) multipliers, row fastest */
    double *out;
} dft_job;

static void *dft_worker(void *arg)
{
    const dft_job *j = (const dft_job *)arg;
    const double scale = M_PI * M_PI / (4 * log(2.0));
    int64_t i;
    for (i = j->r0; i < j->r1; ++i) {
        const double u = j->uvw[3 * i], v = j->uvw[3 * i + 1], w = j->uvw[3 * i + 2];
        int k, ch;
        for (ch = 0; ch < j->nchan; ++ch) {
            double *o = j->out + 2 * (i + j->nrow * ch);
            o[0] = 0.0;
            o[1] = 0.0;
        }
        for (k = 0; k < j->ncomp; ++k) {
            const double *p = j->comp + 8 * k;
            const double l = p[1], m = p[2];
            const double n = sqrt(1.0 - (l * l + m * m));
            const double delay = DFT_2PI * (l * u + m * v + (n - 1.0) * w) / DFT_C;
            double r = 0.0;
            if (p[3] > 0.0 || p[4] > 0.0) {
                const double up = (cos(p[5]) * u + sin(p[5]) * v) / DFT_C;
                const double vp = (-sin(p[5]) * u + cos(p[5]) * v) / DFT_C;
                r = (p[3] * p[3] * up * up + p[4] * p[4] * vp * vp) * scale;
            }
            for (ch = 0; ch < j->nchan; ++ch) {
                const double f = j->freq[ch];
                double flux = p[0];
                double *o = j->out + 2 * (i + j->nrow * ch);
                double ph;
                if (p[6] != 0.0) flux *= pow(f / p[7], p[6]);
                if (r != 0.0) flux *= exp(-r * f * f);
                if (j->gain) flux *= j->gain[(int64_t)k * j->nrow * j->nchan + i + j->nrow * ch];
                ph = delay * f;
                o[0] += flux * cos(ph);
                o[1] += flux * sin(ph);
            }
        }
    }
    return NULL;
}

int orc_dft(int64_t nrow, int nchan, const double *uvw, const double *freq,
            int ncomp, const double *comp, const double *gain, double *out, int nthreads)
{
    pthread_t th[256];
    dft_job jobs[256];
    int t;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    for (t = 0; t < nthreads; ++t) {
        jobs[t].r0 = nrow * t / nthreads;
        jobs[t].r1 = nrow * (t + 1) / nthreads;
        jobs[t].nrow = nrow;
        jobs[t].nchan = nchan;
        jobs[t].ncomp = ncomp;
        jobs[t].uvw = uvw;
        jobs[t].freq = freq;
        jobs[t].comp = comp;
        jobs[t].gain = gain;
        jobs[t].out = out;
        if (pthread_create(&th[t], NULL, dft_worker, &jobs[t]) != 0) return 1;
    }
    for (t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    return 0;
}
