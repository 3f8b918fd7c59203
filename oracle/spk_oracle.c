/* Test infrastructure: the float64 oracle of the spektralab render path (spk_oracle.h says what it is).
 * Each function names the reference source it restates. Compiled with -ffp-contract=off. */
#include "spk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../spektralab-engine_b200/csrc/grain_sampler.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static const double kTiny = 1e-10;

/* ---- the Gaussian machinery (reference src/fx/gaussian.cpp:19-53, :316-407) ---------------------- */

static int reflect(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * n;
    int m = i % period;
    if (m < 0) m += period;
    return m < n ? m : period - 1 - m;
}

static void fir_channel(const double* in, double* out, int w, int h, int c, double sigma) {
    const int r = (int)floor(3.0 * sigma + 0.5);
    if (r == 0) {
        for (size_t i = 0; i < (size_t)w * h; ++i) out[3 * i + c] = in[3 * i + c];
        return;
    }
    double* taps = (double*)malloc(sizeof(double) * (size_t)(2 * r + 1));
    double sum = 0.0;
    for (int k = -r; k <= r; ++k) {
        const double t = (double)k / sigma;
        taps[k + r] = exp(-0.5 * t * t);
        sum += taps[k + r];
    }
    for (int k = 0; k <= 2 * r; ++k) taps[k] /= sum;
    double* tmp = (double*)malloc(sizeof(double) * (size_t)w * h);
#pragma omp parallel for
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            double a = 0.0;
            for (int i = -r; i <= r; ++i) a += taps[i + r] * in[3 * ((size_t)reflect(y + i, h) * w + x) + c];
            tmp[(size_t)y * w + x] = a;
        }
#pragma omp parallel for
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            double a = 0.0;
            for (int i = -r; i <= r; ++i) a += taps[i + r] * tmp[(size_t)y * w + reflect(x + i, w)];
            out[3 * ((size_t)y * w + x) + c] = a;
        }
    free(tmp);
    free(taps);
}

/* Young and van Vliet (1995), third order, forward then backward, replicated-edge start */
static void iir_line(double* v, int n, size_t stride, const double k[4]) {
    double w1 = v[0], w2 = w1, w3 = w1;
    for (int i = 0; i < n; ++i) {
        const double t = ((k[0] * v[i * stride] + k[1] * w1) + k[2] * w2) + k[3] * w3;
        w3 = w2;
        w2 = w1;
        w1 = t;
        v[i * stride] = t;
    }
    double y1 = v[(size_t)(n - 1) * stride], y2 = y1, y3 = y1;
    for (int i = n - 1; i >= 0; --i) {
        const double t = ((k[0] * v[i * stride] + k[1] * y1) + k[2] * y2) + k[3] * y3;
        y3 = y2;
        y2 = y1;
        y1 = t;
        v[i * stride] = t;
    }
}

static void iir_channel(const double* in, double* out, int w, int h, int c, double sigma) {
    double q;
    if (sigma >= 2.5) q = 0.98711 * sigma - 0.96330;
    else q = 3.97156 - 4.14554 * sqrt(1.0 - 0.26891 * sigma);
    const double q2 = q * q, q3 = q2 * q;
    const double b0 = ((1.57825 + 2.44413 * q) + 1.4281 * q2) + 0.422205 * q3;
    const double b1 = (2.44413 * q + 2.85619 * q2) + 1.26661 * q3;
    const double b2 = -(1.4281 * q2 + 1.26661 * q3);
    const double b3 = 0.422205 * q3;
    const double k[4] = {1.0 - ((b1 + b2) + b3) / b0, b1 / b0, b2 / b0, b3 / b0};
    for (size_t i = 0; i < (size_t)w * h; ++i) out[3 * i + c] = in[3 * i + c];
#pragma omp parallel for
    for (int y = 0; y < h; ++y) iir_line(out + 3 * (size_t)y * w + c, w, 3, k);
#pragma omp parallel for
    for (int x = 0; x < w; ++x) iir_line(out + 3 * (size_t)x + c, h, 3 * (size_t)w, k);
}

void orc_gaussian(const double* in, double* out, int32_t w, int32_t h, const double sigma[3]) {
    for (int c = 0; c < 3; ++c) {
        if (!(sigma[c] > 0.0)) {
            for (size_t i = 0; i < (size_t)w * h; ++i) out[3 * i + c] = in[3 * i + c];
        } else if (sigma[c] < 3.0) {
            fir_channel(in, out, w, h, c, sigma[c]);
        } else {
            iir_channel(in, out, w, h, c, sigma[c]);
        }
    }
}

/* raw := a raw + b sum_k w_k G_k(raw)   (reference src/fx/halation.cpp:307-329) */
static void mixture_mix(double* raw, int w, int h, int n, const double wt[][3], const double sg[][3],
                        const double a[3], const double b[3]) {
    const size_t N = (size_t)w * h * 3;
    double* acc = (double*)calloc(N, sizeof(double));
    double* g = (double*)malloc(N * sizeof(double));
    for (int k = 0; k < n; ++k) {
        orc_gaussian(raw, g, w, h, sg[k]);
        for (size_t i = 0; i < N; ++i) acc[i] += wt[k][i % 3] * g[i];
    }
    for (size_t i = 0; i < N; ++i) raw[i] = a[i % 3] * raw[i] + b[i % 3] * acc[i];
    free(acc);
    free(g);
}

/* ---- expose (reference kernels/film.metal:50-99, :189-227) -------------------------------------- */

static double mitchell(double u) {
    const double a = fabs(u);
    if (a < 1.0) return (1.0 / 6.0) * (7.0 * a * a * a - 12.0 * a * a + 16.0 / 3.0);
    if (a < 2.0) return (1.0 / 6.0) * ((-7.0 / 3.0) * a * a * a + 12.0 * a * a - 20.0 * a + 32.0 / 3.0);
    return 0.0;
}

static void mitchell_axis(double t, int L, int idx[4], double wt[4]) {
    const double last = (double)(L - 1);
    double u = t * last, frac;
    int base;
    if (u <= 0.0) u = 0.0;
    if (u >= last) {
        base = L - 2;
        frac = 1.0;
    } else {
        base = (int)floor(u);
        frac = u - (double)base;
    }
    for (int k = 0; k < 4; ++k) {
        int i = base - 1 + k;
        if (i < 0) i = -i;
        if (i >= L) i = 2 * (L - 1) - i;
        idx[k] = i;
    }
    wt[0] = mitchell(frac + 1.0);
    wt[1] = mitchell(frac);
    wt[2] = mitchell(frac - 1.0);
    wt[3] = mitchell(frac - 2.0);
}

/* rgb (binary32) or rgb64 (binary64, when rgb is NULL) */
static void expose(const OracleSetup* s, const float* rgb, const double* rgb64, double* H, size_t n) {
#pragma omp parallel for
    for (size_t p = 0; p < n; ++p) {
        const double r = rgb ? rgb[3 * p] : rgb64[3 * p];
        const double g = rgb ? rgb[3 * p + 1] : rgb64[3 * p + 1];
        const double b = rgb ? rgb[3 * p + 2] : rgb64[3 * p + 2];
        const double* A = s->A;
        const double X = A[0] * r + A[1] * g + A[2] * b;
        const double Y = A[3] * r + A[4] * g + A[5] * b;
        const double Z = A[6] * r + A[7] * g + A[8] * b;
        const double bs = X + Y + Z;
        const double d = bs > 1e-10 ? bs : 1e-10;
        const double x = X / d, y = Y / d, o = 1.0 - x;
        const double t0 = fmin(fmax(o * o, 0.0), 1.0);
        const double t1 = fmin(fmax(y / (o > 1e-10 ? o : 1e-10), 0.0), 1.0);
        const double bp = isnan(bs) ? 0.0 : bs;
        int ia[4], ib[4];
        double wa[4], wb[4];
        mitchell_axis(t0, s->L, ia, wa);
        mitchell_axis(t1, s->L, ib, wb);
        double sum = 0.0, a[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                const double w = wa[i] * wb[j];
                const double* t = s->table + 3 * ((size_t)ia[i] * s->L + ib[j]);
                sum += w;
                for (int c = 0; c < 3; ++c) a[c] += w * t[c];
            }
        for (int c = 0; c < 3; ++c) H[3 * p + c] = bp * (sum != 0.0 ? a[c] / sum : a[c]) * s->gain;
    }
}

/* ---- curves and grain (reference kernels/film.metal:84-101, fx_grain.metal:39-97, fx_random.h) ---- */

static size_t search_right(const double* x, size_t K, size_t stride, double v) {
    size_t lo = 0, hi = K;
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        if (x[mid * stride] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static double curve_y(const OracleSetup* s, const double* table, int c, double v) {
    const double* x = s->cx;
    const double* y = table + (size_t)c * s->K;
    if (v <= x[0]) return y[0];
    if (v >= x[s->K - 1]) return y[s->K - 1];
    const size_t lo = search_right(x, (size_t)s->K, 1, v);
    const size_t l = lo == 0 ? 0 : lo - 1;
    const double t = (v - x[l]) * s->cinv[l];
    return y[l] + t * (y[l + 1] - y[l]);
}

static double curve(const OracleSetup* s, int c, double v) { return curve_y(s, s->cy, c, v); }

static double grain_value(const OracleSetup* s, double D, int c, uint32_t pixel, const float* counts) {
    const double v = s->positive ? -D : D;
    const size_t K = (size_t)s->gK;
    double dl[3];
    if (v <= s->gaxis[c]) {
        for (int l = 0; l < 3; ++l) dl[l] = s->glayers[l * 3 + c];
    } else if (v >= s->gaxis[3 * (K - 1) + c]) {
        for (int l = 0; l < 3; ++l) dl[l] = s->glayers[((K - 1) * 3 + l) * 3 + c];
    } else {
        const size_t lo = search_right(s->gaxis + c, K, 3, v);
        const size_t j = lo == 0 ? 0 : lo - 1;
        const double t = (v - s->gaxis[3 * j + c]) * s->ginv[3 * j + c];
        for (int l = 0; l < 3; ++l) {
            const double y0 = s->glayers[(j * 3 + l) * 3 + c], y1 = s->glayers[((j + 1) * 3 + l) * 3 + c];
            dl[l] = y0 + t * (y1 - y0);
        }
    }
    double G = 0.0;
    for (int l = 0; l < 3; ++l) {
        const int lc = l * 3 + c;
        const double d = dl[l] + s->dmin_l[lc];
        const double Dl = s->sat_d[lc], n = s->count[lc];
        double q = d / Dl;
        q = q < 1e-6 ? 1e-6 : (q > 0.999999 ? 0.999999 : q);
        const double sat = 1.0 - q * s->uniformity[c] * 0.999999;
        const double lam = (n / sat) * q;
        const double k = counts ? (double)counts[(size_t)pixel * 9 + c * 3 + l]
                                : (double)spk_poisson((float)lam, pixel, SPK_STREAM_GRAIN((uint32_t)c, (uint32_t)l),
                                                      s->seed);
        G += k * (Dl / n) * sat;
    }
    return G - s->dmin_c[c];
}

static double smooth01d(double t) {
    const double u = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    return u * u * (3.0 - 2.0 * u);
}

/* the frame maximum of the exposure's values, NaN skipped (reference src/film/geometry.cpp:210-217) */
static double frame_max(const double* H, size_t N) {
    double m = -INFINITY;
    for (size_t i = 0; i < N; ++i)
        if (H[i] > m) m = H[i];
    return m;
}

/* the highlight boost (reference src/film/develop.cpp:32-62) and the back-reflection headroom
 * (src/fx/halation.cpp:68-86, kernels/fx_halation.metal:18-39), in binary64 */
static void highlights(const OracleSetup* s, double* H, size_t n) {
    const size_t N = 3 * n;
    if (s->boost_ev != 0.0) {
        const double M = frame_max(H, N);
        if (M == 0.0) {
            for (size_t i = 0; i < N; ++i) H[i] *= 0.0;
        } else {
            double x0 = 0.184 * pow(2.0, 4.0);
            x0 = x0 < M ? x0 : M;
            if (x0 != M) {
                const double a = pow(28.0, 1.0 - 0.3), q = a * (1.0 - x0 / M);
                const double k = (pow(2.0, s->boost_ev) - 1.0) / (exp(q) - q - 1.0);
                for (size_t i = 0; i < N; ++i)
                    if (H[i] > x0) {
                        const double z = a * (H[i] - x0) / M;
                        H[i] += k * M * (exp(z) - z - 1.0);
                    }
            }
        }
    }
    if (s->headroom_ev > 0.0) {
        const double clip = frame_max(H, N);
        if (clip > 0.0 && isfinite(clip)) {
            for (size_t p = 0; p < n; ++p) {
                double* v = H + 3 * p;
                const double m = fmax(fmax(v[0], v[1]), v[2]);
                if (!(m > 0.0)) continue;
                const double lm = log2(m);
                const double s1 = smooth01d((lm - log2(clip) + 1.0) / 0.75);
                const double s2 = smooth01d(lm - log2(0.184) - 1.5);
                const double g = exp2(s->headroom_ev * s1 * s2);
                for (int c = 0; c < 3; ++c) v[c] *= g;
            }
        }
    }
}

static int develop_impl(const OracleSetup* s, const float* rgb, const double* rgb64, int32_t w, int32_t h,
                        const float* counts, double* neg) {
    const size_t n = (size_t)w * h, N = 3 * n;
    double* H = (double*)malloc(N * sizeof(double));
    expose(s, rgb, rgb64, H, n);
    if (s->boost_ev != 0.0 || s->headroom_ev > 0.0) highlights(s, H, n);
    if (s->lens_blur_px > 0.0) {
        double* t = (double*)malloc(N * sizeof(double));
        const double sg[3] = {s->lens_blur_px, s->lens_blur_px, s->lens_blur_px};
        orc_gaussian(H, t, w, h, sg);
        memcpy(H, t, N * sizeof(double));
        free(t);
    }
    if (s->n_scatter > 0) mixture_mix(H, w, h, s->n_scatter, s->scatter_w, s->scatter_s, s->scatter_a, s->scatter_b);
    if (s->n_bounce > 0) mixture_mix(H, w, h, s->n_bounce, s->bounce_w, s->bounce_s, s->mix_a, s->mix_b);
    double* D = (double*)malloc(N * sizeof(double));
#pragma omp parallel for
    for (size_t i = 0; i < N; ++i) D[i] = curve(s, (int)(i % 3), log10(fmax(H[i], 0.0) + 1e-10));
    if (s->couplers) {
        /* the correction from the first development, its diffusion, then the pre-inverted curve */
        double* chi = (double*)malloc(N * sizeof(double));
#pragma omp parallel for
        for (size_t p = 0; p < n; ++p) {
            double sv[3];
            for (int c = 0; c < 3; ++c) sv[c] = s->positive ? s->dmax[c] - D[3 * p + c] : D[3 * p + c];
            for (int m = 0; m < 3; ++m)
                chi[3 * p + m] = (sv[0] * s->coupler_m[m] + sv[1] * s->coupler_m[3 + m]) + sv[2] * s->coupler_m[6 + m];
        }
        const double zero[3] = {0.0, 0.0, 0.0}, one[3] = {1.0, 1.0, 1.0};
        if (s->n_dir > 0) mixture_mix(chi, w, h, s->n_dir, s->dir_w, s->dir_s, zero, one);
#pragma omp parallel for
        for (size_t i = 0; i < N; ++i)
            D[i] = curve_y(s, s->cy0, (int)(i % 3), log10(fmax(H[i], 0.0) + 1e-10) - chi[i]);
        free(chi);
    }
    if (!s->grain) {
        memcpy(neg, D, N * sizeof(double));
    } else {
        double* G = (double*)malloc(N * sizeof(double));
#pragma omp parallel for
        for (size_t i = 0; i < N; ++i) G[i] = grain_value(s, D[i], (int)(i % 3), (uint32_t)(i / 3), counts);
        if (s->final_blur > 0.0) {
            const double sg[3] = {s->final_blur, s->final_blur, s->final_blur};
            orc_gaussian(G, H, w, h, sg);
            memcpy(G, H, N * sizeof(double));
        }
        for (size_t i = 0; i < N; ++i) neg[i] = s->amount == 1.0 ? G[i] : (1.0 - s->amount) * D[i] + s->amount * G[i];
        free(G);
    }
    free(D);
    free(H);
    return 0;
}

int orc_develop(const OracleSetup* s, const float* rgb, int32_t w, int32_t h, const float* counts, double* neg) {
    return develop_impl(s, rgb, NULL, w, h, counts, neg);
}

/* ---- print (reference kernels/print.metal:29-127, :165-317) -------------------------------------- */

static void spectral_n(const double* eps, const double* beta, const double* wt, int32_t nl, const double d[3],
                       double r[3]) {
    r[0] = r[1] = r[2] = 0.0;
    for (int32_t l = 0; l < nl; ++l) {
        const double D = ((d[0] * eps[3 * l] + d[1] * eps[3 * l + 1]) + d[2] * eps[3 * l + 2]) + beta[l];
        const double T = pow(10.0, -D);
        for (int k = 0; k < 3; ++k) r[k] += T * wt[3 * l + k];
    }
}

static void spectral(const double* eps, const double* beta, const double* wt, const double d[3], double r[3]) {
    spectral_n(eps, beta, wt, 81, d, r);
}

void orc_spectral(const double* eps, const double* beta, const double* wt, int32_t nl, const double* d, int64_t n,
                  double* out) {
    for (int64_t p = 0; p < n; ++p) spectral_n(eps, beta, wt, nl, d + 3 * p, out + 3 * p);
}

static double paper(const OracleSetup* s, int c, double v) {
    if (isnan(v)) return v;
    const size_t K = (size_t)s->pK;
    if (v <= s->px[0]) return s->py[c];
    if (v >= s->px[K - 1]) return s->py[3 * (K - 1) + c];
    const size_t j = search_right(s->px, K, 1, v) - 1;
    const double y0 = s->py[3 * j + c];
    return y0 + ((v - s->px[j]) * s->pr[j]) * (s->py[3 * (j + 1) + c] - y0);
}

static double sgn(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }

static double knee(double d, double tau, double lim, double p) {
    if (d <= tau) return d;
    const double x = (d - tau) / (lim - tau);
    return tau + (lim - tau) * (x / pow(1.0 + pow(x, p), 1.0 / p));
}

static double post_adapt(double v, double f_l) {
    const double f = pow((f_l * fabs(v)) / 100.0, 0.42);
    return ((400.0 * sgn(v)) * f) / (27.13 + f) + 0.1;
}

static void mat(const double* m, const double v[3], double o[3]) {
    o[0] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    o[1] = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    o[2] = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
}

static void gamut(const OracleSetup* s, double rgb[3]) {
    const double* k = s->cam_k;
    const double f_l = k[0], n_bb = k[1], n_cb = k[2], nn = k[3], z = k[4], a_w = k[5], cc = k[6], n_c = k[7];
    const double j_first = k[8], j_last = k[9], h_first = k[10], h_step = k[11];
    const double kn[3] = {k[12], k[13], k[14]}, lc[3] = {k[15], k[16], k[17]}, j_white = k[18];
    const double d_rgb[3] = {k[19], k[20], k[21]};
    const double cz = cc * z, inv_cz = 1.0 / cz, f_l_qrt = pow(f_l, 0.25);
    const double chroma_k = pow(1.64 - pow(0.29, nn), 0.73), hundred_over_f_l = 100.0 / f_l;
    double xyz[3], x100[3], r16[3];
    mat(s->m_to_xyz, rgb, xyz);
    for (int i = 0; i < 3; ++i) x100[i] = 100.0 * xyz[i];
    mat(s->m16, x100, r16);
    const double ra = post_adapt(d_rgb[0] * r16[0], f_l), ga = post_adapt(d_rgb[1] * r16[1], f_l),
                 ba = post_adapt(d_rgb[2] * r16[2], f_l);
    const double a = (ra - (12.0 * ga) / 11.0) + ba / 11.0;
    const double b = ((ra + ga) - 2.0 * ba) / 9.0;
    const double h = atan2(b, a);
    const double et = 0.25 * (cos(h + 2.0) + 3.8);
    const double A = (((2.0 * ra + ga) + ba / 20.0) - 0.305) * n_bb;
    const double ratio = A / a_w;
    const double J = (100.0 * sgn(ratio)) * pow(fabs(ratio), cz);
    const double den = (ra + ga) + (21.0 * ba) / 20.0;
    const double t = den != 0.0 ? (((((50000.0 / 13.0) * n_c) * n_cb) * et) * sqrt(a * a + b * b)) / den : 0.0;
    const double C = t > 0.0 ? (pow(t, 0.9) * sqrt(fabs(J) / 100.0)) * chroma_k : 0.0;
    const double M = C * f_l_qrt;
    const double Mp = log(1.0 + 0.0228 * M) / 0.0228;
    double Jp = (1.7 * J) / (1.0 + 0.007 * J);
    if (s->lc_active) {
        double Ln = Jp / j_white;
        if (Ln > lc[0]) {
            Ln = knee(Ln, lc[0], lc[1], lc[2]);
            Jp = Ln * j_white;
        }
    }
    const int rows = 64, cols = 720;
    const double Jc = fmin(fmax(Jp, j_first), j_last);
    const double u = ((Jc - j_first) / (j_last - j_first)) * (double)(rows - 1);
    int l0 = (int)floor(u);
    l0 = l0 < 0 ? 0 : (l0 > rows - 2 ? rows - 2 : l0);
    const double fl = u - (double)l0;
    const double v = (h - h_first) / h_step;
    const double vf = floor(v);
    int h0 = ((int)vf) % cols;
    if (h0 < 0) h0 += cols;
    const int h1 = h0 == cols - 1 ? 0 : h0 + 1;
    const double fh = v - vf;
    const double* cm = s->cmax;
    const double cmv = (1.0 - fl) * ((1.0 - fh) * cm[l0 * cols + h0] + fh * cm[l0 * cols + h1]) +
                       fl * ((1.0 - fh) * cm[(l0 + 1) * cols + h0] + fh * cm[(l0 + 1) * cols + h1]);
    const double cs = fmax(cmv, 1e-9);
    double dch = Mp / cs;
    if (dch > 0.0) dch = knee(dch, kn[0], kn[1], kn[2]);
    const double Mn = dch * cs;
    const double Mi = (exp(0.0228 * Mn) - 1.0) / 0.0228;
    const double Ji = Jp / (1.7 - 0.007 * Jp);
    const double Ci = Mi / f_l_qrt;
    const double Ai = (a_w * sgn(Ji)) * pow(fabs(Ji / 100.0), inv_cz);
    const double sq = sqrt(fabs(Ji) / 100.0);
    const double ti = (sq > 0.0 && Ci > 0.0) ? pow(Ci / (sq * chroma_k), 1.0 / 0.9) : 0.0;
    const double p2 = Ai / n_bb + 0.305, p3 = 21.0 / 20.0;
    double ai = 0.0, bi = 0.0;
    if (ti != 0.0) {
        const double p1 = ((((50000.0 / 13.0) * n_c) * n_cb) * et) / ti;
        const double sh = sin(h), ch = cos(h);
        if (fabs(sh) >= fabs(ch)) {
            const double p4 = p1 / sh;
            bi = ((p2 * (2.0 + p3)) * (460.0 / 1403.0)) /
                 (((p4 + ((2.0 + p3) * (220.0 / 1403.0)) * (ch / sh)) - 27.0 / 1403.0) + p3 * (6300.0 / 1403.0));
            ai = (bi * ch) / sh;
        } else {
            const double p5 = p1 / ch;
            ai = ((p2 * (2.0 + p3)) * (460.0 / 1403.0)) /
                 ((p5 + (2.0 + p3) * (220.0 / 1403.0)) - (27.0 / 1403.0 - p3 * (6300.0 / 1403.0)) * (sh / ch));
            bi = (ai * sh) / ch;
        }
    }
    const double xa[3] = {((460.0 * p2 + 451.0 * ai) + 288.0 * bi) / 1403.0,
                          ((460.0 * p2 - 891.0 * ai) - 261.0 * bi) / 1403.0,
                          ((460.0 * p2 - 220.0 * ai) - 6300.0 * bi) / 1403.0};
    double rc[3], xo[3];
    for (int i = 0; i < 3; ++i) {
        const double vv = xa[i] - 0.1, av = fabs(vv);
        const double beta = av >= 400.0 ? 0.0 : (27.13 * av) / (400.0 - av);
        rc[i] = ((hundred_over_f_l * sgn(vv)) * pow(beta, 1.0 / 0.42)) / d_rgb[i];
    }
    mat(s->m16_inv, rc, xo);
    for (int i = 0; i < 3; ++i) xo[i] /= 100.0;
    mat(s->m_to_rgb, xo, rgb);
}

static double cctf(double v, int mode) {
    switch (mode) {
        case 0: return v <= 0.0031308 ? 12.92 * v : 1.055 * sgn(v) * pow(fabs(v), 1.0 / 2.4) - 0.055;
        case 1: return v < 1.0 / 512.0 ? 16.0 * v : pow(v, 1.0 / 1.8);
        case 2: return pow(v, 256.0 / 563.0);
        case 3: return v < 0.018 ? 4.5 * v : 1.099 * sgn(v) * pow(fabs(v), 0.45) - 0.099;
        default: return v;
    }
}

static uint16_t enc16(double v) {
    if (isnan(v)) return 0;
    const double c = fmin(fmax(v, 0.0), 1.0);
    return (uint16_t)floor(c * 65535.0 + 0.5);
}

int orc_print(const OracleSetup* s, const double* neg, int32_t w, int32_t h, uint16_t* out, double* lin) {
    const size_t n = (size_t)w * h, N = 3 * n;
    double* rgb = (double*)malloc(N * sizeof(double));
    double* field = NULL;
    if (s->glare && s->printed) {
        /* one lognormal value per pixel on all channels, then its blur */
        double* f = (double*)malloc(N * sizeof(double));
        field = (double*)malloc(N * sizeof(double));
#pragma omp parallel for
        for (size_t p = 0; p < n; ++p) {
            const double v = (double)spk_lognormal(s->glare_mean, s->glare_sd, (uint32_t)p, 200u, s->print_seed);
            f[3 * p] = f[3 * p + 1] = f[3 * p + 2] = v;
        }
        const double sg[3] = {s->glare_sigma, s->glare_sigma, s->glare_sigma};
        if (s->glare_sigma > 0.0)
            orc_gaussian(f, field, w, h, sg);
        else
            memcpy(field, f, N * sizeof(double));
        free(f);
    }
#pragma omp parallel for
    for (size_t p = 0; p < n; ++p) {
        double d[3] = {neg[3 * p], neg[3 * p + 1], neg[3 * p + 2]}, r[3];
        if (s->printed) {
            spectral(s->enl_eps, s->enl_beta, s->enl_wt, d, r);
            for (int c = 0; c < 3; ++c) {
                double l = log10(fmax(r[c] * s->g[c] + s->o[c], 0.0) + kTiny);
                l = log10(fmax(pow(10.0, l) * s->k_gain, 0.0) + kTiny);
                d[c] = paper(s, c, l);
            }
        }
        spectral(s->scan_eps, s->scan_beta, s->scan_wt, d, r);
        for (int c = 0; c < 3; ++c) r[c] = fmax(r[c], 0.0) + kTiny;
        if (s->levels) {
            double Yp = s->levels_m * r[1] + s->levels_q;
            Yp = Yp < 0.0 ? 0.0 : (Yp > 1.0 ? 1.0 : Yp);
            const double sc = Yp / (r[1] + kTiny);
            for (int c = 0; c < 3; ++c) r[c] *= sc;
        }
        if (field)
            for (int c = 0; c < 3; ++c) r[c] += (field[3 * p + c] / 100.0) * s->glare_tint[c];
        double o[3];
        mat(s->to_rgb, r, o);
        gamut(s, o);
        for (int c = 0; c < 3; ++c) rgb[3 * p + c] = o[c];
    }
    if (s->scanner_lens_blur > 0.0) {
        double* t = (double*)malloc(N * sizeof(double));
        const double sg[3] = {s->scanner_lens_blur, s->scanner_lens_blur, s->scanner_lens_blur};
        orc_gaussian(rgb, t, w, h, sg);
        memcpy(rgb, t, N * sizeof(double));
        free(t);
    }
    if (s->unsharp_sigma > 0.0 && s->unsharp_amount > 0.0) {
        double* g = (double*)malloc(N * sizeof(double));
        const double sg[3] = {s->unsharp_sigma, s->unsharp_sigma, s->unsharp_sigma};
        orc_gaussian(rgb, g, w, h, sg);
        const double a = s->unsharp_amount;
        for (size_t i = 0; i < N; ++i) rgb[i] = (1.0 + a) * rgb[i] - a * g[i];
        free(g);
    }
    free(field);
    if (s->edr && s->printed) {
#pragma omp parallel for
        for (size_t p = 0; p < n; ++p) {
            double* v = rgb + 3 * p;
            double y = (s->edr_r_y[0] * v[0] + s->edr_r_y[1] * v[1]) + s->edr_r_y[2] * v[2];
            y = y > 0.0 ? y : 0.0;
            double yp = y;
            if (y > 0.0 && (y < s->edr_toe || y > s->edr_shoulder)) {
                const int N = s->edr_n > 2 ? s->edr_n : 2;
                double u = (log2(y) - s->edr_lo) / (s->edr_hi - s->edr_lo);
                u = (u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u)) * (N - 1);
                int i0 = (int)floor(u);
                i0 = i0 < N - 2 ? i0 : N - 2;
                const double t = u - i0;
                yp = exp2((1.0 - t) * s->edr_tab[i0] + t * s->edr_tab[i0 + 1]);
            }
            for (int c = 0; c < 3; ++c) v[c] = v[c] * yp / (y + kTiny);
        }
    }
    if (lin) memcpy(lin, rgb, N * sizeof(double));
#pragma omp parallel for
    for (size_t p = 0; p < n; ++p) {
        double v[3] = {rgb[3 * p], rgb[3 * p + 1], rgb[3 * p + 2]};
        if (s->cctf_active) {
            double m[3];
            mat(s->m_nid, v, m);
            for (int c = 0; c < 3; ++c) v[c] = cctf(m[c], s->cctf_mode);
        }
        for (int c = 0; c < 3; ++c) out[4 * p + c] = enc16(v[c]);
        out[4 * p + 3] = 65535;
    }
    free(rgb);
    return 0;
}

int orc_render(const OracleSetup* s, const float* rgb, int32_t w, int32_t h, const float* counts, uint16_t* out,
               double* out_negative) {
    const size_t N = (size_t)w * h * 3;
    double* neg = (double*)malloc(N * sizeof(double));
    orc_develop(s, rgb, w, h, counts, neg);
    orc_print(s, neg, w, h, out, NULL);
    if (out_negative) memcpy(out_negative, neg, N * sizeof(double));
    free(neg);
    return 0;
}

int orc_render64(const OracleSetup* s, const double* rgb, int32_t w, int32_t h, const float* counts,
                 uint16_t* out, double* out_negative) {
    const size_t N = (size_t)w * h * 3;
    double* neg = (double*)malloc(N * sizeof(double));
    develop_impl(s, NULL, rgb, w, h, counts, neg);
    orc_print(s, neg, w, h, out, NULL);
    if (out_negative) memcpy(out_negative, neg, N * sizeof(double));
    free(neg);
    return 0;
}

/* ---- before the film path: tier downscale, decode, geometry ---- */

/* "c b | a b c d | c b": period 2 (n - 1) (reference src/util/numeric.cpp:134-140) */
static int64_t mirror_i(int64_t i, int64_t n) {
    if (n <= 1) return 0;
    const int64_t period = 2 * (n - 1);
    int64_t m = i % period;
    if (m < 0) m += period;
    return m < n ? m : period - m;
}

/* gaussian taps with sigma = max(0, (n / m - 1) / 2), radius floor(4 sigma + 0.5), binary64 normalised
 * in ascending k and narrowed; returns the radius (taps holds 2 r + 1 values) */
static int tier_taps(int32_t n, int32_t m, float** taps) {
    const double sigma = fmax(0.0, ((double)n / (double)m - 1.0) / 2.0);
    const int r = sigma > 0.0 ? (int)floor(4.0 * sigma + 0.5) : 0;
    *taps = (float*)malloc((size_t)(2 * r + 1) * sizeof(float));
    if (r == 0) {
        (*taps)[0] = 1.0f;
        return 0;
    }
    double* w = (double*)malloc((size_t)(2 * r + 1) * sizeof(double));
    double sum = 0.0;
    for (int k = -r; k <= r; ++k) {
        const double t = (double)k / sigma;
        w[k + r] = exp(-0.5 * t * t);
        sum += w[k + r];
    }
    for (int k = 0; k <= 2 * r; ++k) (*taps)[k] = (float)(w[k] / sum);
    free(w);
    return r;
}

/* output o -> the source coordinate (o + 1/2) n / m - 1/2 as num / den, mirrored into [0, n - 1] */
static void tier_sample(int64_t N, int64_t M, int64_t o, uint32_t* i0, uint32_t* i1, float* t) {
    const int64_t den = 2 * M;
    int64_t num = (2 * o + 1) * N - M;
    if (num > den * (N - 1)) num = 2 * den * (N - 1) - num;
    if (num < 0) num = -num;
    int64_t a = num / den;
    if (a > N - 1) a = N - 1;
    *i0 = (uint32_t)a;
    *i1 = (uint32_t)(a + 1 < N - 1 ? a + 1 : N - 1);
    *t = (float)(num - a * den) / (float)den;
}

int orc_downscale(const float* src, int32_t w, int32_t h, int32_t ow, int32_t oh, float* dst) {
    const size_t N = (size_t)w * h * 3;
    float* a = (float*)malloc(N * sizeof(float));
    float* b = (float*)malloc(N * sizeof(float));
    memcpy(a, src, N * sizeof(float));
    float *ty, *tx;
    const int ry = tier_taps(h, oh, &ty), rx = tier_taps(w, ow, &tx);
    if (ry > 0) {
#pragma omp parallel for
        for (int32_t y = 0; y < h; ++y)
            for (int32_t x = 0; x < w; ++x)
                for (int c = 0; c < 3; ++c) {
                    float acc = 0.0f;
                    for (int k = -ry; k <= ry; ++k)
                        acc = fmaf(ty[k + ry], a[3 * ((size_t)mirror_i(y + k, h) * w + x) + c], acc);
                    b[3 * ((size_t)y * w + x) + c] = acc;
                }
        float* t = a;
        a = b;
        b = t;
    }
    if (rx > 0) {
#pragma omp parallel for
        for (int32_t y = 0; y < h; ++y)
            for (int32_t x = 0; x < w; ++x)
                for (int c = 0; c < 3; ++c) {
                    float acc = 0.0f;
                    for (int k = -rx; k <= rx; ++k)
                        acc = fmaf(tx[k + rx], a[3 * ((size_t)y * w + mirror_i(x + k, w)) + c], acc);
                    b[3 * ((size_t)y * w + x) + c] = acc;
                }
        float* t = a;
        a = b;
        b = t;
    }
#pragma omp parallel for
    for (int32_t oy = 0; oy < oh; ++oy) {
        uint32_t y0, y1;
        float tyv;
        tier_sample(h, oh, oy, &y0, &y1, &tyv);
        for (int32_t ox = 0; ox < ow; ++ox) {
            uint32_t x0, x1;
            float txv;
            tier_sample(w, ow, ox, &x0, &x1, &txv);
            for (int c = 0; c < 3; ++c) {
                const float pa = a[3 * ((size_t)y0 * w + x0) + c], pb = a[3 * ((size_t)y0 * w + x1) + c];
                const float pd = a[3 * ((size_t)y1 * w + x0) + c], pe = a[3 * ((size_t)y1 * w + x1) + c];
                const float top = fmaf(txv, pb - pa, pa), bot = fmaf(txv, pe - pd, pd);
                dst[3 * ((size_t)oy * ow + ox) + c] = fmaf(tyv, bot - top, top);
            }
        }
    }
    free(tx);
    free(ty);
    free(a);
    free(b);
    return 0;
}

/* the inverse transfer functions in binary64 */
static double decode64(double v, int mode) {
    switch (mode) {
        case 0:
            return v <= 0.040449936 ? v / 12.92 : pow((v + 0.055) / 1.055, 2.4);
        case 1:
            return v < 16.0 / 512.0 ? v / 16.0 : pow(v, 1.8);
        case 2:
            return pow(v, 563.0 / 256.0);
        case 3: {
            const double bp = 1.099 * pow(0.018, 0.45) - 0.099;
            return v < bp ? v / 4.5 : pow((v + 0.099) / 1.099, 1.0 / 0.45);
        }
        default:
            return v;
    }
}

/* the clamped bilinear axis of geometry_cpu: f <= 0 or f >= n - 1 clamps with t = 0 */
static void geo_axis(double f, int32_t n, int32_t* i0, int32_t* i1, double* t) {
    if (f <= 0.0) {
        *i0 = 0;
        *t = 0.0;
    } else if (f >= (double)(n - 1)) {
        *i0 = n - 1;
        *t = 0.0;
    } else {
        const double fl = floor(f);
        *i0 = (int32_t)fl;
        *t = f - fl;
    }
    *i1 = *i0 + 1 < n - 1 ? *i0 + 1 : n - 1;
}

int orc_prepare(const float* src, int32_t w, int32_t h, int32_t decode, int32_t mode, const double geo[8],
                double* dst, int32_t* out_w, int32_t* out_h) {
    const size_t N = (size_t)w * h * 3;
    double* d = (double*)malloc(N * sizeof(double));
    for (size_t i = 0; i < N; ++i) d[i] = decode ? decode64((double)src[i], mode) : (double)src[i];
    const double cx = geo[0], cy = geo[1], cw = geo[2], ch = geo[3], deg = geo[4];
    const int q = (((int)geo[5] % 4) + 4) % 4;
    const int fh = geo[6] != 0.0, fv = geo[7] != 0.0;
    if (cx == 0.0 && cy == 0.0 && cw == 1.0 && ch == 1.0 && deg == 0.0 && q == 0 && !fh && !fv) {
        memcpy(dst, d, N * sizeof(double));
        *out_w = w;
        *out_h = h;
        free(d);
        return 0;
    }
    /* the output size is the rounded crop (sides exchanged by an odd quarter turn); output pixel centres
     * (u, v) map through the turn and flips, scale to the crop, rotate about its centre */
    const double CW = fmax(1.0, round(cw * w)), CH = fmax(1.0, round(ch * h));
    const double OW = (q & 1) ? CH : CW, OH = (q & 1) ? CW : CH;
    const double sx = cw * w / CW, sy = ch * h / CH, hx = cw * w / 2.0, hy = ch * h / 2.0;
    const double ccx = (cx + cw / 2.0) * w - 0.5, ccy = (cy + ch / 2.0) * h - 0.5;
    const double th = deg * 3.14159265358979323846 / 180.0, ca = cos(th), sa = sin(th);
    const int32_t ow = (int32_t)OW, oh = (int32_t)OH;
#pragma omp parallel for
    for (int32_t oy = 0; oy < oh; ++oy)
        for (int32_t ox = 0; ox < ow; ++ox) {
            double U0 = ox + 0.5, V0 = oy + 0.5;
            if (fh) U0 = OW - U0;
            if (fv) V0 = OH - V0;
            double u, v;
            switch (q) {
                case 0: u = U0; v = V0; break;
                case 1: v = OW - U0; u = V0; break;
                case 2: u = OW - U0; v = OH - V0; break;
                default: v = U0; u = OH - V0; break;
            }
            const double P = sx * u - hx, Q = sy * v - hy;
            const double fx = ccx + (P * ca - Q * sa), fy = ccy + (P * sa + Q * ca);
            int32_t x0, x1, y0, y1;
            double tx, ty;
            geo_axis(fx, w, &x0, &x1, &tx);
            geo_axis(fy, h, &y0, &y1, &ty);
            for (int c = 0; c < 3; ++c) {
                const double a = d[3 * ((size_t)y0 * w + x0) + c], b = d[3 * ((size_t)y0 * w + x1) + c];
                const double e0 = d[3 * ((size_t)y1 * w + x0) + c], e1 = d[3 * ((size_t)y1 * w + x1) + c];
                const double top = a * (1.0 - tx) + b * tx, bot = e0 * (1.0 - tx) + e1 * tx;
                dst[3 * ((size_t)oy * ow + ox) + c] = top * (1.0 - ty) + bot * ty;
            }
        }
    *out_w = ow;
    *out_h = oh;
    free(d);
    return 0;
}

/* ---- the auto-exposure meter ---- */

/* ascending, NaN last */
static int cmp_nan_last(const void* pa, const void* pb) {
    const double a = *(const double*)pa, b = *(const double*)pb;
    const int na = isnan(a), nb = isnan(b);
    if (na || nb) return na - nb;
    return (a > b) - (a < b);
}

static double meter_legacy(double e) {
    const double ev = -log2(e);
    return isfinite(ev) ? ev : 0.0;
}

static double clamp3(double v, double lo, double hi) {
    v = v < lo ? lo : v;
    return hi < v ? hi : v;
}

int orc_meter(const double* rgb, int32_t sw, int32_t sh, const double m[9], double out[7]) {
    const double mid = 0.184, floor_y = 0.184 / 4096.0, two_s2 = 2.0 * (0.2 * 0.2);
    const size_t n = (size_t)sw * sh;
    for (int i = 0; i < 7; ++i) out[i] = 0.0;
    if (n == 0) return 0;
    double* Y = (double*)malloc(n * sizeof(double));
    double* W = (double*)malloc(n * sizeof(double));
    double* S = (double*)malloc(n * sizeof(double));
    const double M = (double)(sw > sh ? sw : sh);
    for (size_t k = 0; k < n; ++k) {
        Y[k] = (m[3] * rgb[3 * k] + m[4] * rgb[3 * k + 1]) + m[5] * rgb[3 * k + 2];
        const double x = ((double)(k % sw) / sw - 0.5) * (sw / M), y = ((double)(k / sw) / sh - 0.5) * (sh / M);
        W[k] = exp(-(x * x + y * y) / two_s2);
    }
    double s = 0.0, swy = 0.0, sw_ = 0.0;
    for (size_t k = 0; k < n; ++k) {
        s += Y[k];
        swy += W[k] * Y[k];
        sw_ += W[k];
    }
    memcpy(S, Y, n * sizeof(double));
    qsort(S, n, sizeof(double), cmp_nan_last);
    const double med = (n % 2) ? S[n / 2] : (S[n / 2 - 1] + S[n / 2]) / 2.0;
    out[0] = meter_legacy((swy / sw_) / mid);
    out[1] = meter_legacy((s / n) / mid);
    out[2] = meter_legacy(med / mid);
    /* y = max(Y, floor) keeps the order (a NaN stays NaN, last) */
    for (size_t k = 0; k < n; ++k) S[k] = S[k] < floor_y ? floor_y : S[k];
#define PCT(q) S[(size_t)((uint64_t)(q) * (uint64_t)(n - 1) / 1000u)]
    const double p1 = PCT(10), p5 = PCT(50), p99 = PCT(990), p995 = PCT(995);
#undef PCT
    double sl = 0.0, swl = 0.0, sw2 = 0.0;
    size_t cnt = 0;
    for (size_t k = 0; k < n; ++k) {
        const double y = Y[k] < floor_y ? floor_y : Y[k];
        if (!(y >= p1 && y <= p99)) continue;
        const double l = log(y);
        sl += l;
        swl += W[k] * l;
        sw2 += W[k];
        ++cnt;
    }
    const double bal = -log2(exp(sl / (double)cnt) / mid);
    out[3] = bal;
    out[4] = -log2(exp(swl / sw2) / mid);
    out[5] = clamp3(log2(mid * pow(2.0, 2.5) / p995), bal - 3.0, bal);
    out[6] = clamp3(log2(mid * pow(2.0, -3.5) / p5), bal, bal + 2.0);
    free(Y);
    free(W);
    free(S);
    return 0;
}

/* ---- the shared binary32 sampler ---- */

void orc_poisson(const float* lam, float* counts, uint32_t n, uint32_t stream, uint32_t seed) {
#pragma omp parallel for
    for (int64_t i = 0; i < (int64_t)n; ++i) counts[i] = spk_poisson(lam[i], (uint32_t)i, stream, seed);
}

void orc_lognormal(float* out, uint32_t n, float mean, float sd, uint32_t stream, uint32_t seed) {
#pragma omp parallel for
    for (int64_t i = 0; i < (int64_t)n; ++i) out[i] = spk_lognormal(mean, sd, (uint32_t)i, stream, seed);
}

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) {
        spk_u4 c = {ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]};
        const spk_u4 r = spk_philox(c, key[2 * i], key[2 * i + 1]);
        out[4 * i] = r.x;
        out[4 * i + 1] = r.y;
        out[4 * i + 2] = r.z;
        out[4 * i + 3] = r.w;
    }
}

float orc_uniform(uint32_t word) { return spk_uniform(word); }
float orc_logf(float x) { return spk_logf(x); }
float orc_expf(float x) { return spk_expf(x); }
float orc_cosf(float x) { return spk_cosf(x); }

/* splitmix64 (Steele, Lea and Flood, OOPSLA 2014) as the reference's seed sequence draws it
 * (src/fx/rng.hpp:17-41): state += golden gamma, then the 30/27/31 mix, low 32 bits */
uint32_t orc_splitmix_next(uint64_t* state) {
    *state += 0x9E3779B97F4A7C15ull;
    uint64_t z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (uint32_t)z;
}

int orc_render_linear(const OracleSetup* s, const double* rgb, int32_t w, int32_t h, const float* counts,
                      double* out_linear) {
    const size_t n = (size_t)w * h;
    double* neg = (double*)malloc(3 * n * sizeof(double));
    uint16_t* out = (uint16_t*)malloc(4 * n * sizeof(uint16_t));
    develop_impl(s, NULL, rgb, w, h, counts, neg);
    orc_print(s, neg, w, h, out, out_linear);
    free(out);
    free(neg);
    return 0;
}
