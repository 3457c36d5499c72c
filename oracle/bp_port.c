/*
 * C restatement of algotom's CPU back-projector -- TEST INFRASTRUCTURE ONLY.
 *
 * Follows back_projection_cpu (algotom/rec/reconstruction.py:307-359): per
 * angle the reference takes cos/sin of the float32 value -angle in float32
 * (Numba types math.cos(float32) as float32), forms the detector position
 * in float64, interpolates with a float32 tap difference and adds the
 * float64 value into a float32 image.  With ref_arith = 1 this routine does
 * exactly that, so its output matches the single-threaded reference bit for
 * bit (built with -ffp-contract=off, as Numba does not contract).  The
 * reference runs prange over ANGLES and races on the shared image; here the
 * image rows are handed out to POSIX threads instead, which keeps each
 * pixel's additions in angle order and makes the result deterministic.
 *
 * With ref_arith = 0 it is an FP64 checker: float64 trig of the
 * float32-rounded angle, float64 tap difference and a float64 accumulator
 * (out is double*).
 *
 * Used as the timed CPU baseline (kind "port") and by the tests as a fast
 * FP64 oracle at sizes where the NumPy restatement is slow.  Never linked
 * into, or called by, the product library.
 */
#include <immintrin.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <unistd.h>

typedef struct {
    const float *sino;
    long long sino_stride;
    int nrow, ncol, edge_pad, ref_arith;
    const double *ct, *st;
    double cen;
    void *out;
    long long out_stride;
    int next_row;            /* shared row counter, taken under `lock` */
    pthread_mutex_t lock;
} bp_job;

/* Image row y of one sinogram: every angle in order, as the reference adds
 * them into pixel (y, x).  The inner loop is written branch-free (clamped
 * position, select on the in-range test) so that compilers vectorise it; the
 * arithmetic per in-range pixel is the reference's: when ceil == floor the
 * tap difference is multiplied by an exact zero, giving s[d] as the
 * reference's separate branch does for finite data.  gcc emits AVX-512,
 * AVX2 and baseline clones and picks one at load time. */
__attribute__((target_clones("avx512f", "avx2", "default")))
static void bp_row(bp_job *j, int y)
{
    const int ncol = j->ncol, w1 = ncol - 1;
    const double ic = 0.5 * (double)w1;
    const double yc = (double)y - ic;
    const double wmax = (double)w1;
    float *restrict of = j->ref_arith
        ? (float *)j->out + (long long)y * j->out_stride : 0;
    double *restrict od = j->ref_arith
        ? 0 : (double *)j->out + (long long)y * j->out_stride;
    for (int x = 0; x < ncol; ++x) {
        if (of) of[x] = 0.0f; else od[x] = 0.0;
    }
    for (int i = 0; i < j->nrow; ++i) {
        const float *restrict row = j->sino + (long long)i * j->sino_stride;
        const double c = j->ct[i], ys = yc * j->st[i], cen = j->cen;
        const float e0 = row[0], e1 = row[w1];
        if (of && !j->edge_pad) {
            for (int x = 0; x < ncol; ++x) {
                const double f = ((double)x - ic) * c + ys + cen;
                const int inr = (f >= 0.0) & (f <= wmax);
                const double fc = inr ? f : 0.0;
                const int d = (int)fc;
                const int u = d + (fc > (double)d);
                const float yd = row[d];
                const float dv = row[u] - yd;
                const double val = (double)yd + (double)dv * (fc - (double)d);
                const float upd = (float)((double)of[x] + val);
                of[x] = inr ? upd : of[x];
            }
        } else if (of) {
            for (int x = 0; x < ncol; ++x) {
                const double f = ((double)x - ic) * c + ys + cen;
                const int inr = (f >= 0.0) & (f <= wmax);
                const double fc = inr ? f : 0.0;
                const int d = (int)fc;
                const int u = d + (fc > (double)d);
                const float yd = row[d];
                const float dv = row[u] - yd;
                double val = (double)yd + (double)dv * (fc - (double)d);
                const double ev = (double)(f < 0.0 ? e0 : e1);
                val = inr ? val : ev;
                of[x] = (float)((double)of[x] + val);
            }
        } else {
            for (int x = 0; x < ncol; ++x) {
                const double f = ((double)x - ic) * c + ys + cen;
                const int inr = (f >= 0.0) & (f <= wmax);
                const double fc = inr ? f : 0.0;
                const int d = (int)fc;
                const int u = d + (fc > (double)d);
                const double yd = (double)row[d];
                const double dv = (double)row[u] - yd;
                const double val = yd + dv * (fc - (double)d);
                const double ev = j->edge_pad ? (double)(f < 0.0 ? e0 : e1)
                                              : 0.0;
                od[x] += inr ? val : ev;
            }
        }
    }
}

/* Same row as bp_row for the reference arithmetic without edge padding,
 * four pixels per step with AVX2: float64 positions, float32 tap gathers,
 * float32 tap difference, float64 value, float32 accumulator -- the same
 * operations in the same order (no contraction), hence the same bits. */
__attribute__((target("avx2")))
static void bp_row_avx2(bp_job *j, int y)
{
    const int ncol = j->ncol, w1 = ncol - 1;
    const double ic = 0.5 * (double)w1;
    const double yc = (double)y - ic;
    float *of = (float *)j->out + (long long)y * j->out_stride;
    for (int x = 0; x < ncol; ++x) of[x] = 0.0f;
    const __m256d wmax = _mm256_set1_pd((double)w1), zero = _mm256_setzero_pd();
    const __m256d lane = _mm256_set_pd(3.0, 2.0, 1.0, 0.0);
    const int n4 = ncol & ~3;
    for (int i = 0; i < j->nrow; ++i) {
        const float *row = j->sino + (long long)i * j->sino_stride;
        const double c = j->ct[i], ys = yc * j->st[i], cen = j->cen;
        const __m256d vc = _mm256_set1_pd(c), vys = _mm256_set1_pd(ys), vcen = _mm256_set1_pd(cen);
        for (int x = 0; x < n4; x += 4) {
            __m256d xd = _mm256_sub_pd(_mm256_add_pd(_mm256_set1_pd((double)x), lane), _mm256_set1_pd(ic));
            __m256d f = _mm256_add_pd(_mm256_add_pd(_mm256_mul_pd(xd, vc), vys), vcen);
            __m256d inr = _mm256_and_pd(_mm256_cmp_pd(f, zero, _CMP_GE_OQ), _mm256_cmp_pd(f, wmax, _CMP_LE_OQ));
            __m256d fc = _mm256_and_pd(f, inr);
            __m128i d = _mm256_cvttpd_epi32(fc);
            __m256d dd = _mm256_cvtepi32_pd(d);
            __m128i up = _mm256_cvtpd_epi32(_mm256_and_pd(_mm256_cmp_pd(fc, dd, _CMP_GT_OQ), _mm256_set1_pd(1.0)));
            __m128i u = _mm_add_epi32(d, up);
            __m128 yd = _mm_i32gather_ps(row, d, 4);
            __m128 yu = _mm_i32gather_ps(row, u, 4);
            __m128 dv = _mm_sub_ps(yu, yd);
            __m256d val = _mm256_add_pd(_mm256_cvtps_pd(yd),
                                        _mm256_mul_pd(_mm256_cvtps_pd(dv), _mm256_sub_pd(fc, dd)));
            __m128 acc = _mm_loadu_ps(of + x);
            __m128 upd = _mm256_cvtpd_ps(_mm256_add_pd(_mm256_cvtps_pd(acc), val));
            __m128 m = _mm256_cvtpd_ps(inr);  /* all-ones lanes stay all-ones (NaN bits) */
            _mm_storeu_ps(of + x, _mm_blendv_ps(acc, upd, m));
        }
        for (int x = n4; x < ncol; ++x) {
            const double f = ((double)x - ic) * c + ys + cen;
            if (f >= 0.0 && f <= (double)w1) {
                int d = (int)floor(f);
                int u = (int)ceil(f);
                double val;
                if (u != d) {
                    float yd = row[d];
                    float dv = row[u] - yd;
                    val = (double)yd + (double)dv * (f - (double)d);
                } else {
                    val = (double)row[d];
                }
                of[x] = (float)((double)of[x] + val);
            }
        }
    }
}

static int g_have_avx2 = -1;

static void *bp_worker(void *arg)
{
    bp_job *j = (bp_job *)arg;
    const int fast = j->ref_arith && !j->edge_pad && g_have_avx2 > 0;
    for (;;) {
        pthread_mutex_lock(&j->lock);
        int y0 = j->next_row;
        j->next_row += 4;
        pthread_mutex_unlock(&j->lock);
        if (y0 >= j->ncol) break;
        int y1 = y0 + 4 < j->ncol ? y0 + 4 : j->ncol;
        for (int y = y0; y < y1; ++y) {
            if (fast) bp_row_avx2(j, y);
            else bp_row(j, y);
        }
    }
    return 0;
}

/* One sinogram [nrow, ncol] (row stride `sino_stride` floats) to an image
 * [ncol, ncol] whose rows are `out_stride` elements apart. */
static void bp_one(const float *sino, long long sino_stride, int nrow,
                   int ncol, const float *angles, float center, int edge_pad,
                   int ref_arith, void *out, long long out_stride,
                   int nthreads)
{
    bp_job j;
    if (g_have_avx2 < 0) g_have_avx2 = __builtin_cpu_supports("avx2") ? 1 : 0;
    double *ct = (double *)malloc(sizeof(double) * (size_t)(nrow + 1));
    double *st = (double *)malloc(sizeof(double) * (size_t)(nrow + 1));
    for (int i = 0; i < nrow; ++i) {
        float th = -angles[i];
        if (ref_arith) {
            ct[i] = (double)cosf(th);
            st[i] = (double)sinf(th);
        } else {
            ct[i] = cos((double)th);
            st[i] = sin((double)th);
        }
    }
    j.sino = sino; j.sino_stride = sino_stride; j.nrow = nrow; j.ncol = ncol;
    j.edge_pad = edge_pad; j.ref_arith = ref_arith; j.ct = ct; j.st = st;
    j.cen = (double)center; j.out = out; j.out_stride = out_stride;
    j.next_row = 0;
    pthread_mutex_init(&j.lock, 0);
    if (nthreads > ncol) nthreads = ncol;
    if (nthreads <= 1) {
        bp_worker(&j);
    } else {
        pthread_t *t = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
        for (int k = 0; k < nthreads; ++k) pthread_create(&t[k], 0, bp_worker, &j);
        for (int k = 0; k < nthreads; ++k) pthread_join(t[k], 0);
        free(t);
    }
    pthread_mutex_destroy(&j.lock);
    free(ct);
    free(st);
}

/* Stack [nrow, nslice, ncol] -> [ncol, nslice, ncol]; nslice = 1 with a
 * plain 2-D sinogram.  Returns 0. */
int oracle_backproject(const float *sino, int nrow, int nslice, int ncol,
                       const float *angles, float center, int edge_pad,
                       int ref_arith, void *out, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    for (int k = 0; k < nslice; ++k) {
        const float *s = sino + (long long)k * ncol;
        if (ref_arith) {
            float *o = (float *)out + (long long)k * ncol;
            bp_one(s, (long long)nslice * ncol, nrow, ncol, angles, center,
                   edge_pad, 1, o, (long long)nslice * ncol, nthreads);
        } else {
            double *o = (double *)out + (long long)k * ncol;
            bp_one(s, (long long)nslice * ncol, nrow, ncol, angles, center,
                   edge_pad, 0, o, (long long)nslice * ncol, nthreads);
        }
    }
    return 0;
}

int oracle_max_threads(void)
{
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}
