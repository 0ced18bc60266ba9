/* CPU oracle for the BRiDCT hot path: TEST INFRASTRUCTURE ONLY (the checker).
 *
 * Restates, in scalar float32 C, the algorithm of the reference's rectangular
 * route (src/generated/rect.c via src/plan.c):
 *   - sj_scale and the plan's normalization/correction tables  (src/plan.c:40-47, 92-108)
 *   - the 1D scaled DCT-II core col_fN: Makhoul reorder (idx tables), a real
 *     split-radix FFT whose sub-transforms carry Johnson-Frigo scale factors
 *     (the leaf and comb functions, tangent twiddle tables tab), and the tangent post rotation
 *     post*_body                              (src/generated/rect_generated.inc:5-109, 660-834)
 *   - col_tN as the exact transpose of col_fN (leafT, combT, post_tbody)
 *   - the 2D driver: vertical (columns) then bands (rows) with x norm on output
 *     for FORWARD, x norm on input then bands/vertical with col_t for INVERSE,
 *     and fwd -> x corr -> inv for ROUNDTRIP         (src/generated/rect.c:5-23)
 * The recursion is written out by hand (not generated) so that it checks the
 * CUDA path's generated arithmetic independently.  Nothing in the product links it.
 */
#include "sj_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI 3.14159265358979323846

double oracle_sj_scale(int n, int k)
{
    if (n <= 4)
        return 1.0;
    k %= n / 4;
    double angle = 2 * PI * k / n;
    return oracle_sj_scale(n / 4, k) * (k <= n / 8 ? cos(angle) : sin(angle));
}

/* Variant scale: 0 = S (s(n,k)), 1 = S2 (s(2n,k)), 2 = S4 (s(4n,k)). */
static double vscale(int variant, int n, int k)
{
    return oracle_sj_scale((1 << variant) * n, k);
}

static int sub_variant(int variant)
{
    return variant == 0 ? 1 : variant == 1 ? 2 : 1;
}

typedef struct { float re, im; } cpx;

static cpx cmul(cpx a, double cr, double ci)
{
    float r = (float)cr, i = (float)ci;
    cpx o = {a.re * r - a.im * i, a.re * i + a.im * r};
    return o;
}
static cpx cscale(cpx a, double s) { cpx o = {a.re * (float)s, a.im * (float)s}; return o; }
static cpx cadd(cpx a, cpx b) { cpx o = {a.re + b.re, a.im + b.im}; return o; }
static cpx csub(cpx a, cpx b) { cpx o = {a.re - b.re, a.im - b.im}; return o; }
static cpx cconj(cpx a) { cpx o = {a.re, -a.im}; return o; }
static cpx cmul_mi(cpx a) { cpx o = {a.im, -a.re}; return o; }  /* * (-i) */
static cpx cmul_i(cpx a) { cpx o = {-a.im, a.re}; return o; }   /* * (+i) */

/* Per-k combine coefficients shared by the forward comb and its transpose. */
typedef struct {
    double tr, ti;              /* t_k = w^k s_Z(k) / s(n,k) */
    double a1, a2, a3, a4;      /* X_k, X_{n/2-k} multipliers on U_k and A */
    double a5, a6, a7, a8;      /* X_{k+n/4}, X_{n/4-k} multipliers on U_{k+n/4} and B */
} comb_coef;

static comb_coef comb_coefficients(int n, int variant, int k)
{
    int uv = sub_variant(variant);
    comb_coef c;
    double base = oracle_sj_scale(n, k);
    double sz = vscale(0, n / 4, k);
    double ang = 2 * PI * k / n;
    c.tr = cos(ang) * sz / base;
    c.ti = -sin(ang) * sz / base;
    double su_k = vscale(uv, n / 2, k), su_q = vscale(uv, n / 2, n / 4 - k);
    c.a1 = su_k / vscale(variant, n, k);
    c.a2 = base / vscale(variant, n, k);
    c.a3 = su_k / vscale(variant, n, n / 2 - k);
    c.a4 = base / vscale(variant, n, n / 2 - k);
    c.a5 = su_q / vscale(variant, n, k + n / 4);
    c.a6 = base / vscale(variant, n, k + n / 4);
    c.a7 = su_q / vscale(variant, n, n / 4 - k);
    c.a8 = base / vscale(variant, n, n / 4 - k);
    return c;
}

/* Half spectrum X[0..n/2] / scale of a real sequence x[0], x[s], ... (length n). */
static void rfft(const float *x, ptrdiff_t s, int n, int variant, cpx *X)
{
    if (n == 1) {
        X[0].re = x[0];
        X[0].im = 0;
        return;
    }
    if (n == 2) {
        X[0].re = (x[0] + x[s]) * (float)(1.0 / vscale(variant, 2, 0));
        X[1].re = (x[0] - x[s]) * (float)(1.0 / vscale(variant, 2, 1));
        X[0].im = X[1].im = 0;
        return;
    }
    cpx *U = malloc(sizeof(cpx) * (size_t)(n / 4 + 1));
    cpx *Z = malloc(sizeof(cpx) * (size_t)(n / 8 + 1));
    cpx *Zp = malloc(sizeof(cpx) * (size_t)(n / 8 + 1));
    float *xm = malloc(sizeof(float) * (size_t)(n / 4));
    rfft(x, 2 * s, n / 2, sub_variant(variant), U);
    rfft(x + s, 4 * s, n / 4, 0, Z);
    for (int m = 0; m < n / 4; m++)                     /* x[4m-1], indices mod n */
        xm[m] = x[(ptrdiff_t)((4 * m - 1 + n) % n) * s];
    rfft(xm, 1, n / 4, 0, Zp);
    char *done = calloc((size_t)n / 2 + 1, 1);
    for (int k = 0; k <= n / 8; k++) {
        comb_coef c = comb_coefficients(n, variant, k);
        cpx tz = cmul(Z[k], c.tr, c.ti);
        cpx tzp = cmul(Zp[k], c.tr, -c.ti);
        cpx A = cadd(tz, tzp), B = csub(tz, tzp);
        cpx uk = U[k], uq = cconj(U[n / 4 - k]);
        int idx[4] = {k, n / 2 - k, k + n / 4, n / 4 - k};
        cpx val[4];
        val[0] = cadd(cscale(uk, c.a1), cscale(A, c.a2));
        val[1] = cconj(csub(cscale(uk, c.a3), cscale(A, c.a4)));
        val[2] = cadd(cscale(uq, c.a5), cmul_mi(cscale(B, c.a6)));
        val[3] = cconj(cadd(cscale(uq, c.a7), cmul_i(cscale(B, c.a8))));
        for (int j = 0; j < 4; j++)
            if (!done[idx[j]]) {
                done[idx[j]] = 1;
                X[idx[j]] = val[j];
            }
    }
    X[0].im = 0;
    X[n / 2].im = 0;
    free(done); free(xm); free(Zp); free(Z); free(U);
}

/* Transpose of rfft: adjoint half spectrum Xb[0..n/2] -> xb[0], xb[s], ... */
static void rfft_t(const cpx *Xb, int n, int variant, float *xb, ptrdiff_t s)
{
    if (n == 1) {
        xb[0] = Xb[0].re;
        return;
    }
    if (n == 2) {
        float a = Xb[0].re * (float)(1.0 / vscale(variant, 2, 0));
        float b = Xb[1].re * (float)(1.0 / vscale(variant, 2, 1));
        xb[0] = a + b;
        xb[s] = a - b;
        return;
    }
    cpx *Ub = calloc((size_t)(n / 4 + 1), sizeof(cpx));
    cpx *Zb = calloc((size_t)(n / 8 + 1), sizeof(cpx));
    cpx *Zpb = calloc((size_t)(n / 8 + 1), sizeof(cpx));
    float *xm = malloc(sizeof(float) * (size_t)(n / 4));
    char *done = calloc((size_t)n / 2 + 1, 1);
    for (int k = 0; k <= n / 8; k++) {
        comb_coef c = comb_coefficients(n, variant, k);
        int idx[4] = {k, n / 2 - k, k + n / 4, n / 4 - k};
        int own[4];
        for (int j = 0; j < 4; j++) {
            own[j] = !done[idx[j]];
            done[idx[j]] = 1;
        }
        cpx zero = {0, 0}, ukb = zero, uqb = zero, Ab = zero, Bb = zero;
        cpx xb_[4];
        for (int j = 0; j < 4; j++) {
            xb_[j] = own[j] ? Xb[idx[j]] : zero;
            if (idx[j] == 0 || idx[j] == n / 2)
                xb_[j].im = 0;                   /* structurally real outputs */
        }
        ukb = cadd(ukb, cscale(xb_[0], c.a1));
        Ab = cadd(Ab, cscale(xb_[0], c.a2));
        cpx w = cconj(xb_[1]);
        ukb = cadd(ukb, cscale(w, c.a3));
        Ab = csub(Ab, cscale(w, c.a4));
        uqb = cadd(uqb, cscale(xb_[2], c.a5));
        Bb = cadd(Bb, cmul_i(cscale(xb_[2], c.a6)));
        w = cconj(xb_[3]);
        uqb = cadd(uqb, cscale(w, c.a7));
        Bb = cadd(Bb, cmul_mi(cscale(w, c.a8)));
        cpx tzb = cadd(Ab, Bb), tzpb = csub(Ab, Bb);
        Zb[k] = cadd(Zb[k], cmul(tzb, c.tr, -c.ti));
        Zpb[k] = cadd(Zpb[k], cmul(tzpb, c.tr, c.ti));
        Ub[k] = cadd(Ub[k], ukb);
        Ub[n / 4 - k] = cadd(Ub[n / 4 - k], cconj(uqb));
    }
    Ub[0].im = 0; Ub[n / 4].im = 0;
    Zb[0].im = 0; Zb[n / 8].im = 0;
    Zpb[0].im = 0; Zpb[n / 8].im = 0;
    rfft_t(Ub, n / 2, sub_variant(variant), xb, 2 * s);
    rfft_t(Zb, n / 4, 0, xb + s, 4 * s);
    rfft_t(Zpb, n / 4, 0, xm, 1);
    for (int m = 0; m < n / 4; m++)
        xb[(ptrdiff_t)((4 * m - 1 + n) % n) * s] = xm[m];
    free(done); free(xm); free(Zpb); free(Zb); free(Ub);
}

static int makhoul(int n, int j)
{
    return j < n / 2 ? 2 * j : 2 * (n - 1 - j) + 1;
}

void oracle_core_f(int n, const float *x, ptrdiff_t xs, float *y, ptrdiff_t ys)
{
    float *v = malloc(sizeof(float) * (size_t)n);
    cpx *X = malloc(sizeof(cpx) * (size_t)(n / 2 + 1));
    for (int j = 0; j < n; j++)
        v[j] = x[(ptrdiff_t)makhoul(n, j) * xs];
    rfft(v, 1, n, 0, X);
    y[0] = X[0].re;
    y[(ptrdiff_t)(n / 2) * ys] = X[n / 2].re;
    for (int k = 1; k < n / 2; k++) {              /* post*_body, t = -tan(pi k / 2n) */
        float t = (float)(-tan(PI * k / (2.0 * n)));
        y[(ptrdiff_t)k * ys] = X[k].re - t * X[k].im;
        y[(ptrdiff_t)(n - k) * ys] = -(X[k].im + t * X[k].re);
    }
    free(X); free(v);
}

void oracle_core_t(int n, const float *x, ptrdiff_t xs, float *y, ptrdiff_t ys)
{
    float *v = malloc(sizeof(float) * (size_t)n);
    cpx *X = malloc(sizeof(cpx) * (size_t)(n / 2 + 1));
    X[0].re = x[0]; X[0].im = 0;
    X[n / 2].re = x[(ptrdiff_t)(n / 2) * xs]; X[n / 2].im = 0;
    for (int k = 1; k < n / 2; k++) {              /* post*_tbody */
        float t = (float)(-tan(PI * k / (2.0 * n)));
        float ok = x[(ptrdiff_t)k * xs], onk = x[(ptrdiff_t)(n - k) * xs];
        X[k].re = ok - onk * t;
        X[k].im = -(onk + ok * t);
    }
    rfft_t(X, n, 0, v, 1);
    for (int j = 0; j < n; j++)
        y[(ptrdiff_t)makhoul(n, j) * ys] = v[j];
    free(X); free(v);
}

int oracle_plan_tables(int h, int w, float *norm, float *corr)
{
    double *inv[2];
    for (int axis = 0; axis < 2; axis++) {
        int n = axis ? w : h;
        inv[axis] = malloc(sizeof(double) * (size_t)n);
        for (int k = 0; k < n; k++)
            inv[axis][k] = 1.0 / (oracle_sj_scale(4 * n, k) * sqrt((k ? 2.0 : 1.0) / n));
    }
    for (int r = 0; r < h; r++)
        for (int c = 0; c < w; c++) {
            double s = 1.0 / (inv[0][r] * inv[1][c]);
            norm[(size_t)r * w + c] = (float)s;
            corr[(size_t)r * w + c] = (float)(s * s);
        }
    free(inv[0]); free(inv[1]);
    return 0;
}

static int supported(int h, int w)
{
    return h >= 8 && h <= 1024 && w >= 8 && w <= 1024 && !(h & (h - 1)) && !(w & (w - 1));
}

/* vertical(): 1D core down every column (rect.c:5-7). */
static void vertical(int h, int w, int inv, const float *a, float *b)
{
    for (int c = 0; c < w; c++)
        (inv ? oracle_core_t : oracle_core_f)(h, a + c, w, b + c, w);
}

/* bands(): 1D core along every row, times an optional table (rect.c:8-15). */
static void bands(int h, int w, int inv, const float *a, float *b, const float *tab)
{
    for (int r = 0; r < h; r++) {
        (inv ? oracle_core_t : oracle_core_f)(w, a + (size_t)r * w, 1, b + (size_t)r * w, 1);
        if (tab)
            for (int c = 0; c < w; c++)
                b[(size_t)r * w + c] *= tab[(size_t)r * w + c];
    }
}

int oracle_apply_batch(int h, int w, int mode, size_t batch, const float *x, float *y)
{
    if (!supported(h, w) || mode < 0 || mode > 2)
        return -1;
    size_t e = (size_t)h * w;
    float *norm = malloc(sizeof(float) * e), *corr = malloc(sizeof(float) * e);
    float *a = malloc(sizeof(float) * e), *b = malloc(sizeof(float) * e);
    oracle_plan_tables(h, w, norm, corr);
    for (size_t i = 0; i < batch; i++) {
        const float *xi = x + i * e;
        float *yi = y + i * e;
        if (mode == 0) {
            vertical(h, w, 0, xi, a);
            bands(h, w, 0, a, yi, norm);
        } else {
            if (mode == 1) {
                for (size_t j = 0; j < e; j++)
                    a[j] = xi[j] * norm[j];
            } else {
                vertical(h, w, 0, xi, b);
                bands(h, w, 0, b, a, corr);
            }
            bands(h, w, 1, a, b, NULL);
            vertical(h, w, 1, b, yi);
        }
    }
    free(b); free(a); free(corr); free(norm);
    return 0;
}
