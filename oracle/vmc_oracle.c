/* vmc_oracle.c — CPU restatement of VMaChine's Metropolis/E_L hot path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY (see vmc_oracle.h).  Never linked into the product.
 * Each function cites the reference file:line (paths inside evenmn/VMaChine) whose
 * arithmetic it restates.  Pinned against the compiled reference by
 * tests/test_oracle_pin.py (golden vectors from oracle/_ref).
 */
#include "vmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXN 128
#define MAXD (MAXN * 3)
#define MAXORB 64
#define MAXDEG 24

/* ---------------------------------------------------------------- orbitals */

static long binom(int n, int k)
{
    long r = 1;
    for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
    return r;
}

/* Closed-shell Hermite orbital quantum numbers, in the order of
 * basis.cpp:81-116 (2D: (i-j, j); 3D: (i-j-k, j, k) for shells i).
 * Returns the orbital count, or -1 for an open shell (basis.cpp:62-79). */
static int hermite_orbitals(int N, int d, int q[][3])
{
    int shells = 0;
    for (int c = 0;; c++) {
        long orb = 2 * binom(c + d, d);
        if (orb == N) { shells = c + 1; break; }
        if (orb > N) return -1;
    }
    int cnt = 0;
    for (int i = 0; i < shells; i++) {
        if (d == 2) {
            for (int j = 0; j <= i; j++) { q[cnt][0] = i - j; q[cnt][1] = j; q[cnt][2] = 0; cnt++; }
        } else {
            for (int j = 0; j <= i; j++)
                for (int k = 0; k <= i - j; k++) {
                    q[cnt][0] = i - j - k; q[cnt][1] = j; q[cnt][2] = k; cnt++;
                }
        }
    }
    return cnt;
}

/* Normalised Hermite functions h_m = H_m / sqrt(2^m m!) and their first and second
 * derivatives, for m <= mmax.  The reference evaluates the same functions from
 * hard-coded polynomials times 1/sqrt(2^m m!) (hermite.cpp:12-17, 334-508, argument
 * not scaled by sqrt(omega)); here the physicists' three-term recurrence
 * H_{m+1} = 2x H_m - 2m H_{m-1} with H'_m = 2m H_{m-1} is used instead. */
static void hermite_table(double x, int mmax, double *h, double *h1, double *h2)
{
    h[0] = 1.0;
    if (mmax >= 1) h[1] = sqrt(2.0) * x;
    for (int m = 1; m < mmax; m++)
        h[m + 1] = sqrt(2.0 / (m + 1)) * x * h[m] - sqrt((double)m / (m + 1)) * h[m - 1];
    for (int m = 0; m <= mmax; m++) {
        h1[m] = m >= 1 ? sqrt(2.0 * m) * h[m - 1] : 0.0;
        h2[m] = m >= 2 ? 2.0 * sqrt((double)m * (m - 1)) * h[m - 2] : 0.0;
    }
}

/* phi_k(r) and derivatives along dim a (hermite.cpp:35-72: product over dims). */
typedef struct {
    int n, d, mmax, basis, horb3;
    double Z;
    int q[MAXORB][3]; /* Hermite degrees, or hydrogen (n, l, m) */
} orbset;

/* Hydrogen orbitals of hydrogenorbital.cpp:108-394 (alpha fixed at 1, k = Z),
 * n <= 3 and l <= 1: phi = A(r) f(r) exp(-k r / n) with A = 1 (s) or one
 * coordinate (p: m = 1 -> x, -1 -> y, 0 -> z) and f = 1 (1s, 2p), 2 - k r (2s),
 * 2 k^2 r^2 - 18 k r + 27 (3s), k r - 6 (3p).  With R = f exp(-k r / n):
 *   d_a phi   = (d_a A) R + A R' x_a / r
 *   d_a^2 phi = 2 (d_a A) R' x_a / r + A (R'' x_a^2 / r^2 + R' (1 / r - x_a^2 / r^3)). */
static void hydrogen_eval(const orbset *o, const double *r, double *phi, double *dphi, double *d2phi)
{
    double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]), k = o->Z;
    for (int q = 0; q < o->n; q++) {
        int nq = o->q[q][0], l = o->q[q][1], m = o->q[q][2];
        double f = 1.0, fp = 0.0, fpp = 0.0;
        if (nq == 2 && l == 0) { f = 2.0 - k * rr; fp = -k; }
        if (nq == 3 && l == 0) { f = 2.0 * k * k * rr * rr - 18.0 * k * rr + 27.0; fp = 4.0 * k * k * rr - 18.0 * k; fpp = 4.0 * k * k; }
        if (nq == 3 && l == 1) { f = k * rr - 6.0; fp = k; }
        double a = k / nq, ex = exp(-a * rr);
        double R = f * ex, R1 = (fp - a * f) * ex, R2 = (fpp - 2.0 * a * fp + a * a * f) * ex;
        int ca = l == 1 ? (m == 1 ? 0 : m == -1 ? 1 : 2) : -1;
        double A = ca >= 0 ? r[ca] : 1.0;
        if (phi) phi[q] = A * R;
        for (int c = 0; c < 3; c++) {
            double u = r[c] / rr, dA = c == ca ? 1.0 : 0.0;
            if (dphi) dphi[c * o->n + q] = dA * R + A * R1 * u;
            double d2 = 2.0 * dA * R1 * u + A * (R2 * u * u + R1 * (1.0 / rr - u * u / rr));
            if (nq == 3 && o->horb3) {
                /* the reference's n = 3 "second derivatives" (hydrogenorbital.cpp:351-364),
                 * which are not d^2/dx_c^2: reproduced under the quirk */
                double kr = k * rr, pre = k * ex / (81.0 * rr * rr * rr);
                d2 = l == 0 ? pre * (rr * rr * (2.0 * kr * (5.0 - 3.0 * kr) - 27.0) +
                                     r[c] * r[c] * (kr * (2.0 * kr * (kr - 18.0) + 9.0) + 27.0))
                            : pre * A * (kr - 18.0) * (kr - 6.0) / rr;
            }
            if (d2phi) d2phi[c * o->n + q] = d2;
        }
    }
}

static void orb_eval(const orbset *o, const double *r, double *phi, double *dphi /*d x n*/,
                     double *d2phi /*d x n*/)
{
    if (o->basis == VMO_BASIS_HYDROGEN) {
        hydrogen_eval(o, r, phi, dphi, d2phi);
        return;
    }
    double h[3][MAXDEG], h1[3][MAXDEG], h2[3][MAXDEG];
    for (int a = 0; a < o->d; a++) hermite_table(r[a], o->mmax, h[a], h1[a], h2[a]);
    for (int k = 0; k < o->n; k++) {
        double v = 1.0;
        for (int a = 0; a < o->d; a++) v *= h[a][o->q[k][a]];
        if (phi) phi[k] = v;
        for (int a = 0; a < o->d; a++) {
            double p1 = h1[a][o->q[k][a]], p2 = h2[a][o->q[k][a]];
            for (int b = 0; b < o->d; b++)
                if (b != a) { p1 *= h[b][o->q[k][b]]; p2 *= h[b][o->q[k][b]]; }
            if (dphi) dphi[a * o->n + k] = p1;
            if (d2phi) d2phi[a * o->n + k] = p2;
        }
    }
}

static int orb_setup(const vmo_system *s, orbset *o)
{
    o->d = s->d;
    o->basis = s->basis;
    o->Z = s->Z;
    o->horb3 = (s->quirks & VMO_Q_HORB3) != 0;
    if (s->basis == VMO_BASIS_HYDROGEN) {
        /* closed-shell atoms (hydrogenorbital.cpp:28-58); orbitals (n, l, m) in the
         * order of generateLOS (hydrogenorbital.cpp:60-76), l <= 1 here */
        if (s->d != 3 || (s->N != 2 && s->N != 4 && s->N != 10 && s->N != 12 && s->N != 18)) return -1;
        int cnt = 0;
        for (int nq = 1; nq <= 3 && cnt < s->N / 2; nq++)
            for (int l = 0; l < nq && l <= 1 && cnt < s->N / 2; l++)
                for (int m = -l; m <= l && cnt < s->N / 2; m++) {
                    o->q[cnt][0] = nq; o->q[cnt][1] = l; o->q[cnt][2] = m;
                    cnt++;
                }
        o->n = cnt;
        o->mmax = 0;
        return 0;
    }
    int n = hermite_orbitals(s->N, s->d, o->q);
    if (n < 0 || n > MAXORB) return -1;
    o->n = n;
    int mmax = 0;
    for (int k = 0; k < n; k++)
        for (int a = 0; a < s->d; a++)
            if (o->q[k][a] > mmax) mmax = o->q[k][a];
    o->mmax = mmax + 2;
    return 0;
}

/* In-place Gauss-Jordan inverse with partial pivoting of an n x n row-major
 * matrix.  The reference inverts each spin block with Eigen's PartialPivLU
 * (slaterdeterminant.cpp:112-119); the inverse is the same matrix up to rounding. */
static int invert(double *a, int n)
{
    int piv[MAXORB];
    double b[MAXORB * MAXORB];
    for (int i = 0; i < n * n; i++) b[i] = 0.0;
    for (int i = 0; i < n; i++) b[i * n + i] = 1.0;
    for (int c = 0; c < n; c++) {
        int p = c;
        double best = fabs(a[c * n + c]);
        for (int r = c + 1; r < n; r++)
            if (fabs(a[r * n + c]) > best) { best = fabs(a[r * n + c]); p = r; }
        if (best == 0.0) return -1;
        piv[c] = p;
        if (p != c)
            for (int j = 0; j < n; j++) {
                double t = a[c * n + j]; a[c * n + j] = a[p * n + j]; a[p * n + j] = t;
                t = b[c * n + j]; b[c * n + j] = b[p * n + j]; b[p * n + j] = t;
            }
        double inv = 1.0 / a[c * n + c];
        for (int j = 0; j < n; j++) { a[c * n + j] *= inv; b[c * n + j] *= inv; }
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            double f = a[r * n + c];
            if (f == 0.0) continue;
            for (int j = 0; j < n; j++) { a[r * n + j] -= f * a[c * n + j]; b[r * n + j] -= f * b[c * n + j]; }
        }
    }
    (void)piv;
    memcpy(a, b, sizeof(double) * n * n);
    return 0;
}

/* ------------------------------------------------------------ helpers */

static double dist(const double *x, int d, int i, int j)
{
    double acc = 0.0;
    for (int a = 0; a < d; a++) {
        double t = x[d * i + a] - x[d * j + a];
        acc += t * t;
    }
    return sqrt(acc); /* metropolis.cpp:9-19 */
}

static double radius(const double *x, int d, int i)
{
    double acc = 0.0;
    for (int a = 0; a < d; a++) acc += x[d * i + a] * x[d * i + a];
    return sqrt(acc); /* metropolis.cpp:31-39 */
}

/* Pade-Jastrow spin coefficients (padejastrow.cpp:140-170). */
static double pade_beta(int N, int d, int i, int j)
{
    double sym = d == 2 ? 1.0 / 3 : d == 3 ? 1.0 / 4 : 1.0 / 5;
    double anti = d == 2 ? 1.0 : d == 3 ? 1.0 / 2 : 1.0 / 3;
    int h = N / 2;
    return ((i < h && j < h) || (i >= h && j >= h)) ? sym : anti;
}

int vmo_num_parameters(const vmo_system *s, int e)
{
    int D = s->N * s->d;
    switch (s->elem[e]) {
    case VMO_SLATER: return 0;
    case VMO_SIMPLEJASTROW: return s->N * s->N;          /* simplejastrow.cpp:15 */
    case VMO_RBMGAUSSIAN: return D;                      /* rbmgaussian.cpp:12 */
    case VMO_RBMPRODUCT: return s->hidden * D + s->hidden; /* rbmproduct.cpp:101 */
    default: return 1;
    }
}

/* hidden-unit activations of RBMProduct (rbmproduct.cpp:191-197);
 * with the sort quirk the visible vector is the sorted coordinate list
 * (wavefunction.cpp:40-55 sorts m_positions in place). */
static void rbm_hidden(const vmo_system *s, const double *th, const double *x, double *v,
                       double *pn, double *nn, double *xs_out)
{
    int D = s->N * s->d, H = s->hidden;
    double sig2 = 100.0 * s->sigma * s->sigma; /* sigma = 10 * width (rbmproduct.cpp:102) */
    double xs[MAXD];
    memcpy(xs, x, sizeof(double) * D);
    if (s->quirks & VMO_Q_RBM_SORT) {
        for (int i = 1; i < D; i++) { /* insertion sort, ascending */
            double t = xs[i];
            int j = i - 1;
            while (j >= 0 && xs[j] > t) { xs[j + 1] = xs[j]; j--; }
            xs[j + 1] = t;
        }
    }
    for (int j = 0; j < H; j++) {
        double acc = 0.0;
        for (int i = 0; i < D; i++) acc += th[H + i + D * j] * xs[i]; /* W(i,j), col-major */
        v[j] = th[j] + acc / sig2;
        double e = exp(v[j]);
        pn[j] = 1.0 / (e + 1.0);
        nn[j] = e * pn[j];
    }
    if (xs_out) memcpy(xs_out, xs, sizeof(double) * D);
}

/* ------------------------------------------------------------ evaluation */

/* gpair (N x N, row-major, i < j used) holds, per Pade pair, the gamma its cached
 * f and h were last computed with; NULL means the current gamma for every pair. */
static int eval_impl(const vmo_system *s, const double *theta, const double *x,
                     const double *gpair, double *grad, double *lap, double *pgrad,
                     double *energies)
{
    const int N = s->N, d = s->d, D = N * d, P = s->p_max;
    double gsum[MAXD];
    for (int k = 0; k < D; k++) gsum[k] = 0.0;
    double lapsum = 0.0;
    for (int e = 0; e < s->n_elem; e++) {
        const double *th = theta + (size_t)e * P;
        double *g = grad + (size_t)e * D, *pg = pgrad + (size_t)e * P;
        for (int k = 0; k < D; k++) g[k] = 0.0;
        for (int j = 0; j < P; j++) pg[j] = 0.0;
        double L = 0.0;
        switch (s->elem[e]) {
        case VMO_GAUSSIAN: { /* gaussian.cpp:62-78 */
            double wa = s->omega * th[0], x2 = 0.0;
            for (int k = 0; k < D; k++) { g[k] = -wa * x[k]; x2 += x[k] * x[k]; }
            L = -wa * D;
            pg[0] = -0.5 * s->omega * x2;
            break;
        }
        case VMO_SLATER: { /* slaterdeterminant.cpp:155-191 */
            orbset o;
            if (orb_setup(s, &o)) return -2;
            int n = o.n;
            double sdd_sum = 0.0, dd2 = 0.0;
            for (int b = 0; b < 2; b++) {
                double A[MAXORB * MAXORB], phi[MAXORB];
                for (int i = 0; i < n; i++) {
                    orb_eval(&o, x + d * (b * n + i), phi, NULL, NULL);
                    for (int k = 0; k < n; k++) A[i * n + k] = phi[k];
                }
                if (invert(A, n)) return -1; /* A now holds inv: inv[k*n + i] = Ainv(k, i) */
                for (int i = 0; i < n; i++) {
                    int q = b * n + i;
                    double dphi[3 * MAXORB], d2phi[3 * MAXORB];
                    orb_eval(&o, x + d * q, NULL, dphi, d2phi);
                    for (int a = 0; a < d; a++) {
                        double dd = 0.0, sdd = 0.0;
                        for (int k = 0; k < n; k++) {
                            dd += dphi[a * n + k] * A[k * n + i];
                            sdd += d2phi[a * n + k] * A[k * n + i];
                        }
                        g[q * d + a] = dd;
                        sdd_sum += sdd;
                        dd2 += dd * dd;
                    }
                }
            }
            L = sdd_sum - dd2;
            break;
        }
        case VMO_PADE: { /* padejastrow.cpp:75-116 */
            double gam = th[0], dg = 0.0;
            for (int i = 0; i < N; i++)
                for (int j = i + 1; j < N; j++) {
                    /* f, h come from the cached arrays (gamma of their last update,
                     * padejastrow.cpp:192-209); the Laplacian's (1 + 2 gamma h) uses
                     * the current gamma (padejastrow.cpp:101-105). */
                    double gp = gpair ? gpair[i * N + j] : gam;
                    double r = dist(x, d, i, j), beta = pade_beta(N, d, i, j);
                    double f1 = 1.0 / (1.0 + gp * r), f = beta * f1 * f1, h = r * f1;
                    for (int a = 0; a < d; a++) {
                        double c = (x[d * i + a] - x[d * j + a]) / r;
                        g[d * i + a] += f * c;
                        g[d * j + a] -= f * c;
                        L += 2.0 * f * (1.0 - (1.0 + 2.0 * gam * h) * c * c) / r;
                    }
                    dg += beta * h * h;
                }
            pg[0] = (s->quirks & VMO_Q_PADE_DGAMMA) ? -0.5 * dg : -dg;
            break;
        }
        case VMO_SIMPLEJASTROW: { /* simplejastrow.cpp:67-111 */
            for (int i = 0; i < N; i++)
                for (int j = i + 1; j < N; j++) {
                    double r = dist(x, d, i, j), beta = th[i + N * j];
                    for (int a = 0; a < d; a++) {
                        double c = (x[d * i + a] - x[d * j + a]) / r;
                        g[d * i + a] += beta * c;
                        g[d * j + a] -= beta * c;
                        L += 2.0 * beta * (1.0 - c * c) / r;
                    }
                    pg[i + N * j] = r;
                }
            break;
        }
        case VMO_RBMGAUSSIAN: { /* rbmgaussian.cpp:67-87 */
            double s2 = s->sigma * s->sigma;
            for (int k = 0; k < D; k++) {
                g[k] = -(x[k] - th[k]) / s2;
                pg[k] = (x[k] - th[k]) / s2;
            }
            L = -D / s2;
            break;
        }
        case VMO_RBMPRODUCT: { /* rbmproduct.cpp:167-189 */
            int H = s->hidden;
            double s2 = 100.0 * s->sigma * s->sigma, s4 = s2 * s2;
            double v[256], pn[256], nn[256], xs[MAXD];
            rbm_hidden(s, th, x, v, pn, nn, xs);
            for (int k = 0; k < D; k++) {
                double acc = 0.0, acc2 = 0.0;
                for (int j = 0; j < H; j++) {
                    double w = th[H + k + D * j];
                    acc += w * nn[j];
                    acc2 += w * w * pn[j] * nn[j];
                }
                g[k] = acc / s2;
                L += acc2 / s4;
            }
            for (int j = 0; j < H; j++) {
                pg[j] = nn[j];
                for (int i = 0; i < D; i++) pg[H + i + D * j] = xs[i] * nn[j];
            }
            break;
        }
        case VMO_HYDROGENLIKE: { /* hydrogenlike.cpp:268-286 */
            double az = th[0] * s->Z, rs = 0.0;
            for (int i = 0; i < N; i++) {
                double r = radius(x, d, i);
                rs += r;
                for (int a = 0; a < d; a++) g[d * i + a] = -az * x[d * i + a] / r;
                L -= 2.0 / r;
            }
            L *= az;
            pg[0] = -s->Z * rs;
            break;
        }
        default: return -3;
        }
        lap[e] = L;
        lapsum += L;
        for (int k = 0; k < D; k++) gsum[k] += g[k];
    }
    /* System::getKineticEnergy (elementoperation.cpp:95-109) */
    double g2 = 0.0;
    for (int k = 0; k < D; k++) g2 += gsum[k] * gsum[k];
    energies[0] = -0.5 * (lapsum + g2);
    double vext = 0.0;
    if (s->hamiltonian == VMO_HAM_HO) { /* harmonicoscillator.cpp:16-20 */
        for (int k = 0; k < D; k++) vext += x[k] * x[k];
        vext *= 0.5 * s->omega * s->omega;
    } else { /* atomicnucleus.cpp:35-45 (l = 0) */
        for (int i = 0; i < N; i++) vext += 1.0 / radius(x, d, i);
        vext *= -s->Z;
    }
    energies[1] = vext;
    double vint = 0.0;
    if (s->coulomb) /* coulomb.cpp:17-48, no screening */
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++) vint += 1.0 / dist(x, d, i, j);
    energies[2] = vint;
    return 0;
}

int vmo_eval(const vmo_system *s, const double *theta, const double *x, double *grad,
             double *lap, double *pgrad, double *energies)
{
    return eval_impl(s, theta, x, NULL, grad, lap, pgrad, energies);
}

static int ratio_impl(const vmo_system *s, const double *theta, const double *x,
                      const double *gpair, int k, double xnew, double *ratios)
{
    const int N = s->N, d = s->d, D = N * d, P = s->p_max;
    const int p = k / d;
    double y[MAXD];
    memcpy(y, x, sizeof(double) * D);
    y[k] = xnew;
    for (int e = 0; e < s->n_elem; e++) {
        const double *th = theta + (size_t)e * P;
        double r = 1.0;
        switch (s->elem[e]) {
        case VMO_GAUSSIAN: /* gaussian.cpp:23-28 */
            r = exp(s->omega * th[0] * (x[k] * x[k] - y[k] * y[k]));
            break;
        case VMO_SLATER: { /* slaterdeterminant.cpp:150-153, 177-180 */
            orbset o;
            if (orb_setup(s, &o)) return -2;
            int n = o.n, b = p / n;
            double A[MAXORB * MAXORB], phi[MAXORB];
            for (int i = 0; i < n; i++) {
                orb_eval(&o, x + d * (b * n + i), phi, NULL, NULL);
                for (int kk = 0; kk < n; kk++) A[i * n + kk] = phi[kk];
            }
            if (invert(A, n)) return -1;
            orb_eval(&o, y + d * p, phi, NULL, NULL);
            double R = 0.0;
            for (int kk = 0; kk < n; kk++) R += phi[kk] * A[kk * n + (p - b * n)];
            r = R * R;
            break;
        }
        case VMO_PADE: { /* padejastrow.cpp:211-218 */
            double gam = th[0], acc = 0.0;
            int j0 = (s->quirks & VMO_Q_PADE_RATIO) ? p + 1 : 0;
            for (int j = j0; j < N; j++) {
                if (j == p) continue;
                int lo = p < j ? p : j, hi = p < j ? j : p;
                double gp = gpair ? gpair[lo * N + hi] : gam;
                double ro = dist(x, d, p, j), rn = dist(y, d, p, j);
                acc += pade_beta(N, d, p, j) * (rn / (1.0 + gam * rn) - ro / (1.0 + gp * ro));
            }
            r = exp(2.0 * acc);
            break;
        }
        case VMO_SIMPLEJASTROW: { /* simplejastrow.cpp:145-156 */
            double acc = 0.0;
            int j0 = (s->quirks & VMO_Q_SJ_RATIO) ? p + 1 : 0;
            for (int j = j0; j < N; j++) {
                if (j == p) continue;
                int lo = p < j ? p : j, hi = p < j ? j : p;
                acc += th[lo + N * hi] * (dist(y, d, p, j) - dist(x, d, p, j));
            }
            r = exp(2.0 * acc);
            break;
        }
        case VMO_RBMGAUSSIAN: { /* rbmgaussian.cpp:34-46 */
            double s2 = s->sigma * s->sigma;
            double xo = x[k] - th[k], xn = y[k] - th[k];
            r = exp((xo * xo - xn * xn) / (2.0 * s2));
            break;
        }
        case VMO_RBMPRODUCT: { /* rbmproduct.cpp:199-203 */
            double v[256], po[256], pn2[256], nn[256];
            rbm_hidden(s, th, x, v, po, nn, NULL);
            rbm_hidden(s, th, y, v, pn2, nn, NULL);
            double prod = 1.0;
            for (int j = 0; j < s->hidden; j++) prod *= po[j] / pn2[j];
            r = prod * prod;
            break;
        }
        case VMO_HYDROGENLIKE: /* hydrogenlike.cpp:231-242 */
            r = exp(2.0 * s->Z * th[0] * (radius(x, d, p) - radius(y, d, p)));
            break;
        default: return -3;
        }
        ratios[e] = r;
    }
    return 0;
}

int vmo_ratio(const vmo_system *s, const double *theta, const double *x, int k, double xnew,
              double *ratios)
{
    return ratio_impl(s, theta, x, NULL, k, xnew, ratios);
}

int vmo_quantum_force(const vmo_system *s, const double *theta, const double *x, double *f)
{
    const int D = s->N * s->d;
    double grad[VMO_MAX_ELEM * MAXD], lap[VMO_MAX_ELEM], pg[VMO_MAX_ELEM * 1024], en[3];
    if (s->p_max > 1024) return -4;
    int rc = vmo_eval(s, theta, x, grad, lap, pg, en);
    if (rc) return rc;
    for (int k = 0; k < D; k++) {
        double acc = 0.0;
        for (int e = 0; e < s->n_elem; e++) acc += grad[e * D + k];
        f[k] = 2.0 * acc;
    }
    return 0;
}

/* ------------------------------------------------------------ RNG */

void vmo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static const double TWO_M32 = 2.3283064365386963e-10; /* 2^-32 */

void vmo_step_randoms(uint64_t seed, uint32_t walker, uint64_t step, int sampling, double out[3])
{
    uint32_t ctr[4] = {(uint32_t)step, (uint32_t)(step >> 32), walker, 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t w[4];
    vmo_philox(ctr, key, w);
    out[0] = w[0] * TWO_M32;
    if (sampling == VMO_IS) {
        double u1 = ((double)w[1] + 1.0) * TWO_M32, u2 = w[2] * TWO_M32;
        out[1] = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    } else {
        out[1] = w[1] * TWO_M32;
    }
    out[2] = w[3] * TWO_M32;
}

void vmo_initial_positions(uint64_t seed, uint32_t walker, int D, int normal, double sd,
                           double *pos)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (int c = 0; c < D; c++) {
        uint32_t ctr[4] = {(uint32_t)c, 0u, walker, 1u}, w[4];
        vmo_philox(ctr, key, w);
        if (normal) {
            double u1 = ((double)w[0] + 1.0) * TWO_M32, u2 = w[1] * TWO_M32;
            pos[c] = sd * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        } else {
            pos[c] = w[0] * TWO_M32;
        }
    }
}

/* ------------------------------------------------------------ sampling loop */

/* The drift limiter of the corrected mode (Umrigar, Nightingale and Runge, J. Chem.
 * Phys. 99, 2865 (1993)): v (-1 + sqrt(1 + 2 a dt v^2)) / (a dt v^2), written as
 * 2 v / (1 + sqrt(1 + 2 a dt v^2)); a = 0 leaves v alone. */
static double drift_limited(const vmo_system *s, double v)
{
    if (!(s->drift_limit > 0.0) || (s->quirks & VMO_Q_IS_GREEN)) return v;
    return 2.0 * v / (1.0 + sqrt(1.0 + 2.0 * s->drift_limit * s->step * v * v));
}

int vmo_run(const vmo_system *s, const double *theta, int W, double *pos, double *fcache,
            double *gpair, int steps, int burn_in, int iter, int batches, const double *stream, uint64_t seed,
            uint64_t *counter, unsigned char *accepted, double *energies, double *sums)
{
    const int N = s->N, d = s->d, D = N * d, E = s->n_elem, P = s->p_max;
    const int EP = E * P, NS = 9 + 2 * EP;
    if (D > MAXD || E > VMO_MAX_ELEM || P > 1024) return -4;
    const int bs = (steps - burn_in) / batches;
    const int wlo = bs * (iter % batches), whi = bs * (iter % batches + 1);
    const double dt = s->step, sqdt = sqrt(s->step);
    double *grad = malloc(sizeof(double) * VMO_MAX_ELEM * MAXD);
    double *pg = malloc(sizeof(double) * VMO_MAX_ELEM * 1024);
    int rc = 0;
    for (int w = 0; w < W && !rc; w++) {
        double *x = pos + (size_t)w * D, *fc = fcache + (size_t)w * D, *acc = sums + (size_t)w * NS;
        double *gp = gpair ? gpair + (size_t)w * N * N : NULL;
        for (int j = 0; j < NS; j++) acc[j] = 0.0;
        for (int i = 0; i < steps; i++) {
            double rnd[3];
            if (stream) memcpy(rnd, stream + ((size_t)w * steps + i) * 3, sizeof rnd);
            else vmo_step_randoms(seed, (uint32_t)w, counter[w]++, s->sampling, rnd);
            int k = (int)floor(rnd[0] * D);
            double lap[VMO_MAX_ELEM], en[3], ratios[VMO_MAX_ELEM];
            double dx, fo = 0.0, fn = 0.0;
            if (s->sampling == VMO_IS) { /* importancesampling.cpp:49-60 */
                if ((rc = eval_impl(s, theta, x, gp, grad, lap, pg, en))) break;
                double gk = 0.0;
                for (int e = 0; e < E; e++) gk += grad[e * D + k];
                fn = 2.0 * drift_limited(s, gk);
                fo = (s->quirks & VMO_Q_IS_GREEN) ? fc[k] : fn;
                dx = 0.5 * dt * fn + rnd[1] * sqdt;
            } else { /* bruteforce.cpp:34 */
                dx = 10.0 * (rnd[1] - 0.5) * s->step;
            }
            if ((rc = ratio_impl(s, theta, x, gp, k, x[k] + dx, ratios))) break;
            double p = 1.0;
            for (int e = 0; e < E; e++) p *= ratios[e]; /* elementoperation.cpp:80-87 */
            double wgt = p;
            if (s->sampling == VMO_IS) {
                if (s->quirks & VMO_Q_IS_GREEN) {
                    wgt = (exp(0.5 * (fo - fn) * dx) + 1.0) * p; /* importancesampling.cpp:43-47,70-71 */
                } else { /* Fokker-Planck Green's function ratio for a one-coordinate move */
                    double y[MAXD];
                    memcpy(y, x, sizeof(double) * D);
                    y[k] += dx;
                    if ((rc = eval_impl(s, theta, y, gp, grad, lap, pg, en))) break;
                    double gk = 0.0;
                    for (int e = 0; e < E; e++) gk += grad[e * D + k];
                    double fy = 2.0 * drift_limited(s, gk);
                    wgt = p * exp(0.5 * (fo + fy) * (0.25 * dt * (fo - fy) - dx));
                }
            }
            int acc_move = !(wgt < rnd[2]);
            if (acc_move) {
                x[k] += dx;
                if (s->sampling == VMO_IS) fc[k] = fn;
                if (gp) /* the moved particle's Pade pairs now hold the current gamma */
                    for (int e = 0; e < E; e++)
                        if (s->elem[e] == VMO_PADE) {
                            int pp = k / d;
                            for (int j = 0; j < N; j++) {
                                gp[pp * N + j] = theta[(size_t)e * P];
                                gp[j * N + pp] = theta[(size_t)e * P];
                            }
                        }
            }
            if (accepted) accepted[(size_t)w * steps + i] = (unsigned char)acc_move;
            if (i >= burn_in || energies) {
                if ((rc = eval_impl(s, theta, x, gp, grad, lap, pg, en))) break;
                if (energies) memcpy(energies + ((size_t)w * steps + i) * 3, en, sizeof en);
            }
            if (i >= burn_in) { /* sampler.cpp:52-90 */
                double el = en[0] + en[1] + en[2];
                acc[0] += el; acc[1] += el * el;
                acc[2] += en[0]; acc[3] += en[0] * en[0];
                acc[4] += en[1]; acc[5] += en[1] * en[1];
                acc[6] += en[2]; acc[7] += en[2] * en[2];
                acc[8] += acc_move;
                if (i > wlo && i < whi)
                    for (int j = 0; j < EP; j++) { acc[9 + j] += pg[j]; acc[9 + EP + j] += pg[j] * el; }
            }
        }
    }
    free(grad);
    free(pg);
    return rc;
}

/* ------------------------------------------------------------ blocking */

/* chi-square 95% quantiles for 1..64 degrees of freedom (the test statistic of the
 * automatic blocking method, Jonsson, Phys. Rev. E 98, 043304 (2018)). */
static const double CHI2_95[64] = {
    3.841459, 5.991465, 7.814728, 9.487729, 11.070498, 12.591587, 14.067140, 15.507313, 16.918978,
    18.307038, 19.675138, 21.026070, 22.362032, 23.684791, 24.995790, 26.296228, 27.587112,
    28.869299, 30.143527, 31.410433, 32.670573, 33.924438, 35.172462, 36.415029, 37.652484,
    38.885139, 40.113272, 41.337138, 42.556968, 43.772972, 44.985343, 46.194260, 47.399884,
    48.602367, 49.801850, 50.998460, 52.192320, 53.383541, 54.572228, 55.758479, 56.942387,
    58.124038, 59.303512, 60.480887, 61.656233, 62.829620, 64.001112, 65.170769, 66.338649,
    67.504807, 68.669294, 69.832160, 70.993453, 72.153216, 73.311493, 74.468324, 75.623748,
    76.777803, 77.930524, 79.081944, 80.232098, 81.381015, 82.528727, 83.675261};

/* blocker.cpp:15-71: blocking transforms, lag-1 autocovariance test statistic. */
double vmo_blocking(const double *x, long n, double *mean_out)
{
    if (n <= 1 || (n & (n - 1))) return -1.0;
    int dd = 0;
    while ((1L << dd) < n) dd++;
    double *v = malloc(sizeof(double) * n);
    double mean = 0.0;
    for (long i = 0; i < n; i++) mean += x[i];
    mean /= (double)n;
    memcpy(v, x, sizeof(double) * n);
    double gam[64], var[64], M[64];
    long m = n;
    for (int k = 0; k < dd; k++) {
        double g = 0.0, s2 = 0.0;
        for (long i = 0; i + 1 < m; i++) g += (v[i] - mean) * (v[i + 1] - mean);
        for (long i = 0; i < m; i++) s2 += (v[i] - mean) * (v[i] - mean);
        gam[k] = g / m;
        var[k] = s2 / m;
        for (long i = 0; i < m / 2; i++) v[i] = 0.5 * (v[2 * i] + v[2 * i + 1]);
        m /= 2;
    }
    for (int j = 0; j < dd; j++) M[j] = pow(gam[j] / var[j], 2) * pow(2.0, dd - j);
    /* reverse cumulative sum: C[i] = sum_{j >= dd-1-i} M[j] */
    double C[64];
    for (int i = 0; i < dd; i++) {
        double acc = 0.0;
        for (int j = dd - 1 - i; j < dd; j++) acc += M[j];
        C[i] = acc;
    }
    int k;
    for (k = dd - 1; k >= 0; k--)
        if (C[k] < CHI2_95[k]) break;
    int K = dd - (k + 1);
    double nK = pow(2.0, dd - K);
    free(v);
    if (mean_out) *mean_out = mean;
    return var[K] / nK;
}
