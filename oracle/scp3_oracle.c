/*
 * TEST INFRASTRUCTURE ONLY -- the oracle.  This file is the CPU restatement of
 * the reference's Hamiltonian-build hot path, in plain C, FP64, scalar.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it,
 * and only as the checker; the product never links or calls it.
 *
 * Every function cites the reference file:line it restates.  It is pinned
 * against the reference's own sources compiled unchanged (oracle/_ref, see
 * tests/golden/make_golden.py and tests/test_oracle_golden.py).
 *
 * Two deliberate, documented differences from the reference:
 *  - TTM3-F: the induced-field accumulator is zeroed before the first Jacobi
 *    sweep.  The reference's fill (ttm3f.cpp:108-109) starts at Efq, so its Efd
 *    starts from whatever the heap held (garbage on a first call, the previous
 *    call's field afterwards).  Both converge to the same fixed point to the
 *    1e-15 dipole tolerance.
 *  - Sobol points are addressed directly through the Gray code instead of the
 *    reference's stateful walk (sobol.cpp:27796-27836); the points are equal.
 */
#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../scp3_b200/csrc/sobol_dirnum.h"
#include "../scp3_b200/csrc/ps_coeffs.h"

#define LOG_MAX 62

/* ------------------------------------------------------------------------- */
/* Sobol: Bratley-Fox direction numbers (sobol.cpp:27684-27752).              */
/* v is dims x 62, row-major: v[i*62 + j] is the j-th direction number of     */
/* dimension i, already scaled by 2^(61-j) as i8_sobol does.                  */
/* ------------------------------------------------------------------------- */
int or_sobol_dirnums(int dims, int64_t* v)
{
    if (dims < 1 || dims > SCP3_SOBOL_MAX_DIMS) return -1;
    for (int i = 0; i < dims; i++)
        for (int j = 0; j < LOG_MAX; j++) v[i * LOG_MAX + j] = 0;
    for (int j = 0; j < LOG_MAX; j++) v[j] = 1;             /* dimension 0 */
    for (int i = 1; i < dims; i++) {
        int poly = scp3_sobol_poly[i];
        int m = 0;
        for (int t = poly; t > 1; t >>= 1) m++;              /* degree */
        int includ[LOG_MAX];
        for (int k = m - 1, t = poly; k >= 0; k--, t >>= 1) includ[k] = t & 1;
        for (int j = 0; j < m; j++) v[i * LOG_MAX + j] = scp3_sobol_vinit[i][j];
        for (int j = m; j < LOG_MAX; j++) {
            int64_t nv = v[i * LOG_MAX + j - m];
            int64_t l = 1;
            for (int k = 0; k < m; k++) {
                l *= 2;
                if (includ[k]) nv ^= l * v[i * LOG_MAX + j - k - 1];
            }
            v[i * LOG_MAX + j] = nv;
        }
    }
    int64_t l = 1;
    for (int j = LOG_MAX - 2; j >= 0; j--) {
        l *= 2;
        for (int i = 0; i < dims; i++) v[i * LOG_MAX + j] *= l;
    }
    return 0;
}

/* The 62-bit integer state of point `index` (the reference's lastq before its
 * update, sobol.cpp:27851-27856): XOR of the direction numbers selected by the
 * Gray code of the index. */
static int64_t sobol_state(const int64_t* vrow, int64_t index)
{
    uint64_t g = (uint64_t)index ^ ((uint64_t)index >> 1);
    int64_t x = 0;
    for (int b = 0; g; b++, g >>= 1)
        if (g & 1) x ^= vrow[b];
    return x;
}

/* Project-defined seeded scramble (the reference only takes scrambled points as
 * text through -r, SCP3.cpp:188-194; its generator is MATLAB's
 * scramble(sobolset,'MatousekAffineOwen'), matlab/MatousekAffineOwen.m:1-5, which
 * is a random linear matrix scramble plus a random digital shift).  For each
 * dimension: a lower-triangular GF(2) matrix with unit diagonal acting on the
 * 62 binary digits (output digit p depends on input digits of equal or higher
 * significance) and a 62-bit digital shift, drawn from splitmix64. */
static uint64_t splitmix64(uint64_t* s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void or_scramble_params(int dims, uint64_t seed, uint64_t* masks /* dims x 62 */, uint64_t* shift)
{
    const uint64_t low62 = (1ull << 62) - 1;
    for (int d = 0; d < dims; d++) {
        uint64_t s = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(d + 1));
        for (int p = 0; p < LOG_MAX; p++) {
            uint64_t above = low62 & ~((2ull << p) - 1);      /* bits p+1..61 */
            masks[d * LOG_MAX + p] = (1ull << p) | (splitmix64(&s) & above);
        }
        shift[d] = splitmix64(&s) & low62;
    }
}

static int64_t scramble_bits(const uint64_t* mrow, uint64_t shift, int64_t x)
{
    uint64_t y = 0;
    for (int p = 0; p < LOG_MAX; p++)
        y |= (uint64_t)(__builtin_popcountll((uint64_t)x & mrow[p]) & 1) << p;
    return (int64_t)(y ^ shift);
}

/* Uniforms of points index0 .. index0+n-1, out is n x dims sample-major.
 * masks/shift NULL: the reference's unscrambled points (quasi = lastq*recipd,
 * recipd = 2^-62, sobol.cpp:27752 and 27853). */
void or_sobol_uniforms(int dims, const int64_t* v, const uint64_t* masks, const uint64_t* shift,
                       int64_t index0, int64_t n, double* out)
{
    const double recipd = 1.0 / (double)(1ull << 62);
    for (int64_t s = 0; s < n; s++)
        for (int d = 0; d < dims; d++) {
            int64_t x = sobol_state(v + d * LOG_MAX, index0 + s);
            if (masks) x = scramble_bits(masks + d * LOG_MAX, shift[d], x);
            out[s * dims + d] = (double)x * recipd;
        }
}

/* Beasley-Springer-Moro inverse normal CDF (beasley_springer_moro.cpp:14-46). */
void or_bsm(int64_t n, const double* u, double* x)
{
    static const double a[4] = {2.50662823884, -18.61500062529, 41.39119773534, -25.44106049637};
    static const double b[4] = {-8.47351093090, 23.08336743743, -21.06224101826, 3.13082909833};
    static const double c[9] = {0.3374754822726147, 0.9761690190917186, 0.1607979714918209,
                                0.0276438810333863, 0.0038405729373609, 0.0003951896511919,
                                0.0000321767881768, 0.0000002888167364, 0.0000003960315187};
    for (int64_t j = 0; j < n; j++) {
        double y = u[j] - 0.5;
        if (fabs(y) < 0.42) {
            double r = y * y;
            x[j] = y * (((a[3] * r + a[2]) * r + a[1]) * r + a[0]) /
                   ((((b[3] * r + b[2]) * r + b[1]) * r + b[0]) * r + 1);
        } else {
            double r = (y > 0) ? log(-log(1 - u[j])) : log(-log(u[j]));
            double t = c[0] + r * (c[1] + r * (c[2] + r * (c[3] + r * (c[4] + r * (c[5] +
                       r * (c[6] + r * (c[7] + r * c[8])))))));
            x[j] = (y < 0) ? -t : t;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* qTIP4P/f energy (qtip4pf.cpp:57-145 monomer, 190-286 pair terms), kcal/mol, */
/* coordinates in Angstrom, order O H H per water.                            */
/* ------------------------------------------------------------------------- */
#define QT_CHARGECON 18.22234397655801030455
static const double qt_qM = -1.1128 * QT_CHARGECON;
#define QT_QH (-qt_qM / 2)
#define QT_ROHEQ 0.9419
#define QT_AHOHEQ 107.4
#define QT_EPS 0.1852
#define QT_SIGMA 3.1589
#define QT_ALPHAR 2.287
#define QT_DR 116.09
#define QT_KTHETA 87.85
#define QT_GAMMAM 0.73612
#define QT_GAMMA1 ((1.0 - QT_GAMMAM) / 2)

static double dist2(const double* a, const double* b)
{
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return dx * dx + dy * dy + dz * dz;
}

static double qt_monomer(const double* w)
{
    double d1[3], d2[3], r1 = 0, r2 = 0, c = 0;
    for (int k = 0; k < 3; k++) {
        d1[k] = w[3 + k] - w[k];
        d2[k] = w[6 + k] - w[k];
        r1 += d1[k] * d1[k];
        r2 += d2[k] * d2[k];
        c += d1[k] * d2[k];
    }
    r1 = sqrt(r1);
    r2 = sqrt(r2);
    double x1 = QT_ALPHAR * (r1 - QT_ROHEQ), x2 = QT_ALPHAR * (r2 - QT_ROHEQ);
    double v1 = x1 * x1 * (1.0 - x1 * (1.0 - (7.0 / 12.0) * x1)) * QT_DR;
    double v2 = x2 * x2 * (1.0 - x2 * (1.0 - (7.0 / 12.0) * x2)) * QT_DR;
    double th = acos(c * (1.0 / r1 / r2));
    double dth = th - QT_AHOHEQ * M_PI / 180.0;
    return v1 + v2 + 0.5 * QT_KTHETA * dth * dth;
}

double or_qtip4pf(int nw, const double* crd)
{
    double msite[3 * 64];
    if (nw > 64) return NAN;
    double e_int = 0, e_vdw = 0, e_el = 0;
    for (int i = 0; i < nw; i++) {
        const double* w = crd + 9 * i;
        for (int k = 0; k < 3; k++) msite[3 * i + k] = QT_GAMMAM * w[k] + QT_GAMMA1 * (w[3 + k] + w[6 + k]);
        e_int += qt_monomer(w);
    }
    for (int i = 0; i < nw; i++) {
        for (int j = 0; j < nw; j++) {          /* M(i) - H(j), i != j */
            if (i == j) continue;
            for (int l = 1; l < 3; l++)
                e_el += QT_QH * qt_qM / sqrt(dist2(msite + 3 * i, crd + 9 * j + 3 * l));
        }
        for (int j = i + 1; j < nw; j++) {
            for (int a = 1; a < 3; a++)
                for (int b = 1; b < 3; b++)
                    e_el += QT_QH * QT_QH / sqrt(dist2(crd + 9 * i + 3 * a, crd + 9 * j + 3 * b));
            double s2 = QT_SIGMA * QT_SIGMA / dist2(crd + 9 * i, crd + 9 * j);
            double s6 = s2 * s2 * s2;
            e_vdw += 4 * QT_EPS * s6 * (s6 - 1.0);
            e_el += qt_qM * qt_qM / sqrt(dist2(msite + 3 * i, msite + 3 * j));
        }
    }
    return e_int + e_vdw + e_el;
}

/* ------------------------------------------------------------------------- */
/* Partridge-Schwenke monomer energy and TTM3-F dipole-moment-surface charges */
/* (ps.cpp:470-603 pot_nasa, ps.cpp:605-836 dms_nasa with ttm3=true, energy/  */
/* charges only).                                                             */
/* ------------------------------------------------------------------------- */
static double ps_c5z[245];
static int ps_ready = 0;

static void ps_init(void)
{
    if (ps_ready) return;
    for (int i = 0; i < 245; i++)          /* ps.cpp:508-511 */
        ps_c5z[i] = 0.999677885 * scp3_ps_c5zA[i] + 0.15860145369897 * scp3_ps_cbasis[i] +
                    -1.6351695982132 * scp3_ps_ccore[i] + 1.0 * scp3_ps_crest[i];
    ps_ready = 1;
}

#define PS_REOH 0.958649
#define PS_B1 2.0
#define PS_ROH 0.9519607159623009
#define PS_ALPHAOH 2.587949757553683
#define PS_DEOHA 42290.92019288289
#define PS_PHH1A 16.94879431193463
#define PS_PHH2 12.66426998162947
#define PS_F5Z 0.999677885
#define PS_COSTHE (-.24780227221366464506)

static void ps_geom(const double* rr, double* roh1, double* roh2, double* d1, double* d2, double* dhh,
                    double* costh)
{
    double rhh[3], a = 0, b = 0, c = 0;
    for (int i = 0; i < 3; i++) {
        roh1[i] = rr[3 + i] - rr[i];
        roh2[i] = rr[6 + i] - rr[i];
        rhh[i] = rr[3 + i] - rr[6 + i];
        a += roh1[i] * roh1[i];
        b += roh2[i] * roh2[i];
        c += rhh[i] * rhh[i];
    }
    *d1 = sqrt(a);
    *d2 = sqrt(b);
    *dhh = sqrt(c);
    *costh = (roh1[0] * roh2[0] + roh1[1] * roh2[1] + roh1[2] * roh2[2]) / (*d1 * *d2);
}

static void ps_powers(double x1, double x2, double x3, double f[3][16])
{
    for (int i = 0; i < 3; i++) {
        f[i][0] = 0.0;
        f[i][1] = 1.0;
    }
    for (int j = 2; j < 16; j++) {
        f[0][j] = f[0][j - 1] * x1;
        f[1][j] = f[1][j - 1] * x2;
        f[2][j] = f[2][j - 1] * x3;
    }
}

double or_ps_pot(const double* rr)
{
    ps_init();
    double roh1[3], roh2[3], d1, d2, dhh, costh, f[3][16];
    ps_geom(rr, roh1, roh2, &d1, &d2, &dhh, &costh);
    const double deoh = PS_F5Z * PS_DEOHA;
    const double phh1 = PS_F5Z * PS_PHH1A * exp(PS_PHH2);
    double e1x = exp(-PS_ALPHAOH * (d1 - PS_ROH)), e2x = exp(-PS_ALPHAOH * (d2 - PS_ROH));
    double va = deoh * (e1x * (e1x - 2.0) + e2x * (e2x - 2.0));
    double vb = phh1 * exp(-PS_PHH2 * dhh);
    ps_powers((d1 - PS_REOH) / PS_REOH, (d2 - PS_REOH) / PS_REOH, costh - PS_COSTHE, f);
    double efac = exp(-PS_B1 * (pow(d1 - PS_REOH, 2) + pow(d2 - PS_REOH, 2)));
    double sum0 = 0;
    for (int j = 1; j < 245; j++) {
        int I = scp3_ps_idx1[j], J = scp3_ps_idx2[j], K = scp3_ps_idx3[j];
        sum0 += ps_c5z[j] * (f[0][I] * f[1][J] + f[0][J] * f[1][I]) * f[2][K];
    }
    double e = va + vb + (2 * ps_c5z[0] + efac * sum0);
    e += 0.44739574026257;
    e *= 0.00285914375100642899;
    return e;
}

void or_ps_dms(const double* rr, double* q3)
{
    const double ath0 = 1.82400520401572996557;
    double roh1[3], roh2[3], d1, d2, dhh, costh, f[3][16];
    ps_geom(rr, roh1, roh2, &d1, &d2, &dhh, &costh);
    double efac = exp(-1.0 * (pow(d1 - PS_REOH, 2) + pow(d2 - PS_REOH, 2)));
    ps_powers((d1 - PS_REOH) / PS_REOH, (d2 - PS_REOH) / PS_REOH, costh - PS_COSTHE, f);
    double p1 = 0, p2 = 0, pl1 = costh, pl2 = 0.5 * (3 * pl1 * pl1 - 1.0);
    for (int j = 1; j < 84; j++) {
        int I = scp3_ps_idxD0[j], J = scp3_ps_idxD1[j], K = scp3_ps_idxD2[j];
        p1 += scp3_ps_coefD[j] * f[0][I] * f[1][J] * f[2][K];
        p2 += scp3_ps_coefD[j] * f[0][J] * f[1][I] * f[2][K];
    }
    const double xx = 0.529177249;
    double pc0 = 0.2999e0 * (pow(d1, -0.6932e0) + pow(d2, -0.6932e0)) *
                 (1.0099e0 + pl1 * -0.1801e0 + pl2 * 0.0892e0);
    p1 = scp3_ps_coefD[0] + p1 * efac + pc0 * xx;
    p2 = scp3_ps_coefD[0] + p2 * efac + pc0 * xx;
    q3[0] = -(p1 + p2);
    q3[1] = p1;
    q3[2] = p2;
    /* TTM3-F modification of the gas-phase surface (ps.cpp:760-790) */
    double axb[3] = {roh1[1] * roh2[2] - roh1[2] * roh2[1], -roh1[0] * roh2[2] + roh1[2] * roh2[0],
                     roh1[0] * roh2[1] - roh1[1] * roh2[0]};
    double s0 = 0;
    for (int i = 0; i < 3; i++) s0 += pow(axb[i], 2);
    double sinth = sqrt(s0) / (d1 * d2);
    double ang = atan2(sinth, costh);
    p1 = 0.5 * (d1 - 0.9578) + 0.012 * (ang - ath0);
    p2 = 0.5 * (d2 - 0.9578) + 0.012 * (ang - ath0);
    q3[0] = q3[0] - (p1 + p2);
    q3[1] = q3[1] + p1;
    q3[2] = q3[2] + p2;
}

/* ------------------------------------------------------------------------- */
/* TTM3-F smeared interactions (ttm3f-bits-smear.cpp:17-80, 97-287).          */
/* ------------------------------------------------------------------------- */
static double gammq23(double x)
{
    const double a = 2.0 / 3.0, eps = 2.220446049250313e-16;
    const double fpmin = 2.2250738585072014e-308 / 2.220446049250313e-16;
    if (x < 5.0 / 3.0) {                                    /* series */
        double ap = a, sum = 1.0 / a, del = sum;
        for (;;) {
            ++ap;
            del *= x / ap;
            sum += del;
            if (fabs(del) < fabs(sum) * eps) break;
        }
        return 1.354117939426400e+00 - sum * exp(-x + a * log(x));
    }
    double b = x + 1.0 - a, c = 1.0 / fpmin, d = 1.0 / b, h = d;   /* continued fraction */
    for (int i = 1;; ++i) {
        double an = -i * (i - a);
        b += 2.0;
        d = an * d + b;
        if (fabs(d) < fpmin) d = fpmin;
        c = b + an / c;
        if (fabs(c) < fpmin) c = fpmin;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (fabs(del - 1.0) <= eps) break;
    }
    return exp(-x + a * log(x)) * h;
}

#define A_XX 0.175
static void smear(double r, double AA, int want0, double* ts0, double* ts1, double* ts2)
{
    const double a13 = pow(A_XX, 1.0 / 3.0);
    double dri = 1.0 / r, drsqi = dri * dri;
    double rA = r / AA, rA3 = rA * rA * rA;
    double e1 = exp(-A_XX * rA3);
    if (want0) *ts0 = (1.0 - e1 + a13 * rA * gammq23(A_XX * rA3)) * dri;
    *ts1 = (1.0 - e1) * dri * drsqi;
    if (ts2) *ts2 = (*ts1 - e1 * A_XX / (AA * AA * AA)) * drsqi;
}

/* TTM3-F energy (ttm3f.cpp:92-321), kcal/mol.  Returns the energy; *iters gets
 * the number of Jacobi sweeps (maxiter+1 if not converged). */
double or_ttm3f(int nw, const double* crd, int maxiter, int* iters)
{
    ps_init();
    const double polarM = 1.444, polfacH = 0.496, polfacM = 0.837;
    const double AA_HH = pow(polfacH * polfacH, 1.0 / 6.0);
    const double AA_HM = pow(polfacH * polfacM, 1.0 / 6.0);
    const double AA_MM = pow(polfacM * polfacM, 1.0 / 6.0);
    const double gammaM = 0.46, gamma1 = 1.0 - gammaM, gamma2 = gammaM / 2;
    const double CHARGECON = 18.22234397655801030455, DEBYE = 4.8033324;
    const double vdwC = -0.72298855E+03, vdwD = 0.10211829E+06, vdwE = 0.37170376E+01;
    const int n3 = 3 * nw;
    double* mem = (double*)calloc((size_t)(9 * n3 + n3 * n3), sizeof(double));
    double *ms = mem, *q = ms + n3, *dip = q + n3, *dipp = dip + n3, *efd = dipp + n3, *efq = efd + n3,
           *phi = efq + n3, *ddt = phi + n3;
    double e_int = 0;
    for (int i = 0; i < nw; i++) {
        const double* w = crd + 9 * i;
        for (int k = 0; k < 3; k++) ms[3 * i + k] = gamma1 * w[k] + gamma2 * (w[3 + k] + w[6 + k]);
        e_int += or_ps_pot(w);
        double q3[3];
        or_ps_dms(w, q3);
        double t = gamma2 / gamma1;
        q[3 * i + 0] = CHARGECON * q3[0] / gamma1;
        q[3 * i + 1] = CHARGECON * (q3[1] + t * (q3[1] + q3[2]));
        q[3 * i + 2] = CHARGECON * (q3[2] + t * (q3[1] + q3[2]));
    }
    double e_vdw = 0;
    for (int i = 0; i < nw; i++) {
        int i3 = 3 * i;
        for (int j = 0; j < nw; j++) {                       /* M(i) - H(j) */
            if (i == j) continue;
            for (int l = 1; l < 3; l++) {
                int jl = 3 * j + l;
                double R[3];
                for (int k = 0; k < 3; k++) R[k] = ms[i3 + k] - crd[3 * jl + k];
                double ts0, ts1;
                smear(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), AA_HM, 1, &ts0, &ts1, NULL);
                phi[i3] += ts0 * q[jl];
                phi[jl] += ts0 * q[i3];
                for (int k = 0; k < 3; k++) efq[i3 + k] += q[jl] * ts1 * R[k];
            }
        }
        for (int j = i + 1; j < nw; j++) {
            int j3 = 3 * j;
            for (int a = 1; a < 3; a++)
                for (int b = 1; b < 3; b++) {
                    double ts0, ts1;
                    smear(sqrt(dist2(crd + 3 * (i3 + a), crd + 3 * (j3 + b))), AA_HH, 1, &ts0, &ts1, NULL);
                    phi[i3 + a] += q[j3 + b] * ts0;
                    phi[j3 + b] += q[i3 + a] * ts0;
                }
            double r2 = dist2(crd + 9 * i, crd + 9 * j), r = sqrt(r2);
            e_vdw += vdwC / (r2 * r2 * r2) + vdwD * exp(-vdwE * r);
            double R[3];
            for (int k = 0; k < 3; k++) R[k] = ms[i3 + k] - ms[j3 + k];
            double ts0, ts1, ts2;
            smear(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), AA_MM, 1, &ts0, &ts1, &ts2);
            phi[i3] += ts0 * q[j3];
            phi[j3] += ts0 * q[i3];
            for (int k = 0; k < 3; k++) {
                efq[i3 + k] += q[j3] * ts1 * R[k];
                efq[j3 + k] -= q[i3] * ts1 * R[k];
            }
            double dd3[3][3];                                /* ttm3f.cpp:239-249 */
            for (int k = 0; k < 3; k++) {
                dd3[k][k] = 3.0 * ts2 * R[k] * R[k] - ts1;
                for (int l = k + 1; l < 3; l++) dd3[k][l] = dd3[l][k] = 3.0 * ts2 * R[k] * R[l];
            }
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) {
                    ddt[n3 * (i3 + k) + j3 + l] = dd3[k][l];
                    ddt[n3 * (j3 + k) + i3 + l] = dd3[k][l];
                }
        }
    }
    for (int i = 0; i < n3; i++) dipp[i] = dip[i] = polarM * efq[i];
    const double stath = DEBYE / CHARGECON / sqrt((double)nw);
    int it;
    for (it = 0; it < maxiter; it++) {
        for (int k = 0; k < n3; k++)
            for (int l = 0; l < n3; l++) efd[k] += ddt[n3 * k + l] * dip[l];
        double dd = 0;
        for (int i = 0; i < n3; i++) {
            dip[i] = polarM * (efq[i] + efd[i]);
            dip[i] = 0.7 * dip[i] + (1.0 - 0.7) * dipp[i];
            double del = dip[i] - dipp[i];
            dd += del * del;
        }
        if (sqrt(dd) * stath < 1.0e-15) break;
        memcpy(dipp, dip, sizeof(double) * n3);
        memset(efd, 0, sizeof(double) * n3);
    }
    if (iters) *iters = (it < maxiter) ? it + 1 : maxiter + 1;
    double e_el = 0, e_ind = 0;
    for (int i = 0; i < n3; i++) {
        e_el += phi[i] * q[i];
        e_ind -= dip[i] * efq[i];
    }
    free(mem);
    return e_int + e_vdw + e_el / 2 + e_ind / 2;
}

/* ------------------------------------------------------------------------- */
/* Basis (HarmonicOscillatorBasis.cpp:16-44, ScaledMatrixElements.cpp:870-930) */
/* ------------------------------------------------------------------------- */
static double ho1(double y) { return sqrt(2.0) * y; }
static double ho2(double y) { return (2.0 * y * y - 1.0) / sqrt(2.0); }
static double ho3(double y) { return (2.0 * y * y - 3.0) * y / sqrt(3.0); }

size_t or_basis_size(int nm, int n2, int n3)   /* ScaledMatrixElements.cpp:73-78 */
{
    return 1 + (size_t)nm + (size_t)n2 * (n2 + 1) / 2 + (size_t)n3 * (1 + n3) * (2 + n3) / 6;
}

void or_get_bra(int nm, int n2, int n3, const double* q, double* bra)
{
    size_t R = 0;
    bra[R++] = 1.0;
    for (int m = 0; m < nm; m++) bra[R++] = ho1(q[m]);
    for (int m = 0; m < n2; m++) bra[R++] = ho2(q[m]);
    for (int m = 0; m < n2; m++)
        for (int n = m + 1; n < n2; n++) bra[R++] = ho1(q[m]) * ho1(q[n]);
    for (int m = 0; m < n3; m++) bra[R++] = ho3(q[m]);
    for (int m = 0; m < n3; m++)
        for (int n = m + 1; n < n3; n++) {
            bra[R++] = ho2(q[m]) * ho1(q[n]);
            bra[R++] = ho1(q[m]) * ho2(q[n]);
        }
    for (int m = 0; m < n3; m++)
        for (int n = m + 1; n < n3; n++)
            for (int p = n + 1; p < n3; p++) bra[R++] = ho1(q[m]) * ho1(q[n]) * ho1(q[p]);
}

/* HO diagonal (ScaledMatrixElements.cpp:735-784) plus the inactive-mode
 * zero-point term of SCP3.cpp:239.  M is column-major with leading dim ld. */
void or_add_ho_diagonal(int nm, const double* omega_sel, int n2, int n3, double zpe_inactive, double* M,
                        int64_t ld)
{
    double e0 = 0;
    for (int k = 0; k < nm; k++) e0 += omega_sel[k];
    e0 *= 0.5;
    size_t C = 0;
#define DIAG(c) M[(size_t)(c) * ld + (c)]
    DIAG(C) += e0;
    C++;
    for (int k = 0; k < nm; k++, C++) DIAG(C) += e0 + omega_sel[k];
    for (int k = 0; k < n2; k++, C++) DIAG(C) += e0 + 2 * omega_sel[k];
    for (int k = 0; k < n2; k++)
        for (int l = k + 1; l < n2; l++, C++) DIAG(C) += e0 + omega_sel[k] + omega_sel[l];
    for (int k = 0; k < n3; k++, C++) DIAG(C) += e0 + 3.0 * omega_sel[k];
    for (int k = 0; k < n3; k++)
        for (int l = k + 1; l < n3; l++) {
            DIAG(C) += e0 + 2.0 * omega_sel[k] + omega_sel[l];
            C++;
            DIAG(C) += e0 + omega_sel[k] + 2.0 * omega_sel[l];
            C++;
        }
    for (int k = 0; k < n3; k++)
        for (int l = k + 1; l < n3; l++)
            for (int j = l + 1; j < n3; j++, C++)
                DIAG(C) += e0 + omega_sel[k] + omega_sel[l] + omega_sel[j];
    for (size_t c = 0; c < C; c++) DIAG(c) += zpe_inactive;   /* SCP3.cpp:239, a separate add */
#undef DIAG
}

/* ------------------------------------------------------------------------- */
/* Per-sample stage of SCP3_a (SCP3.cpp:196-223): normals -> q -> r -> V_anh. */
/* normals: n x nm0 sample-major.  q_out: n x nm0.  v_out: n.                 */
/* pes_id 0 = qTIP4P/f, 1 = TTM3-F.                                           */
/* ------------------------------------------------------------------------- */
void or_samples(int pes_id, int nw, const double* x0, const double* MUa, const double* omega, int nm0,
                const double* normals, int64_t n, double* q_out, double* v_out)
{
    const double bohr = 0.52917721092, kcal = 627.509474277194;
    const int N3 = 9 * nw;
    double* r = (double*)malloc(sizeof(double) * N3);
    for (int64_t s = 0; s < n; s++) {
        double* q = q_out + s * nm0;
        for (int k = 0; k < nm0; k++) q[k] = normals[s * nm0 + k] / sqrt(2.0);
        for (int a = 0; a < N3; a++) {
            double acc = 0.0;
            for (int k = 0; k < nm0; k++) acc += MUa[(size_t)k * N3 + a] * q[k];
            r[a] = bohr * (x0[a] + acc);
        }
        double V = (pes_id == 0 ? or_qtip4pf(nw, r) : or_ttm3f(nw, r, 500, NULL)) / kcal;
        double h = 0.0;
        for (int k = 0; k < nm0; k++) h += q[k] * (omega[k] * q[k]);
        v_out[s] = V - 0.5 * h;
    }
    free(r);
}

/* Accumulation of the -G path (ScaledMatrixElements.cpp:951-971) restated as
 * the plain sum it computes: M_upper[i,j] += sum_s bra_i(s) V(s) bra_j(s), i<=j.
 * q_sel: n x nm (the selected modes), M column-major nb x nb. */
void or_accumulate(int nm, int n2, int n3, const double* q_sel, const double* v, int64_t n, double* M)
{
    size_t nb = or_basis_size(nm, n2, n3);
    double* bra = (double*)malloc(sizeof(double) * nb);
    for (int64_t s = 0; s < n; s++) {
        or_get_bra(nm, n2, n3, q_sel + s * nm, bra);
        for (size_t j = 0; j < nb; j++) {
            double bj = bra[j] * v[s];
            double* col = M + j * nb;
            for (size_t i = 0; i <= j; i++) col[i] += bra[i] * bj;
        }
    }
    free(bra);
}

/* |bra_i| |V| |bra_j| summed over samples: the scale against which an
 * element's rounding error is measured (near-cancelling elements). */
void or_accumulate_abs(int nm, int n2, int n3, const double* q_sel, const double* v, int64_t n, double* M)
{
    size_t nb = or_basis_size(nm, n2, n3);
    double* bra = (double*)malloc(sizeof(double) * nb);
    for (int64_t s = 0; s < n; s++) {
        or_get_bra(nm, n2, n3, q_sel + s * nm, bra);
        for (size_t j = 0; j < nb; j++) {
            double bj = fabs(bra[j] * v[s]);
            double* col = M + j * nb;
            for (size_t i = 0; i <= j; i++) col[i] += fabs(bra[i]) * bj;
        }
    }
    free(bra);
}

/* ------------------------------------------------------------------------- */
/* The gradient (default) path.                                               */
/* ------------------------------------------------------------------------- */

/* qTIP4P/f energy and gradient (qtip4pf.cpp:252-397): kcal/mol and kcal/mol/A.
 * The M site is a fixed linear combination of O, H, H, so a force on it goes to
 * the three atoms with the weights gammaM, gamma1, gamma1. */
static void qt_monomer_grad(const double* w, double* g, double* e)
{
    double d1[3], d2[3], r1 = 0, r2 = 0, c = 0;
    for (int k = 0; k < 3; k++) {
        d1[k] = w[3 + k] - w[k];
        d2[k] = w[6 + k] - w[k];
        r1 += d1[k] * d1[k];
        r2 += d2[k] * d2[k];
        c += d1[k] * d2[k];
    }
    r1 = sqrt(r1);
    r2 = sqrt(r2);
    const double x1 = QT_ALPHAR * (r1 - QT_ROHEQ), x2 = QT_ALPHAR * (r2 - QT_ROHEQ);
    const double v1 = x1 * x1 * (1.0 - x1 * (1.0 - (7.0 / 12.0) * x1)) * QT_DR;
    const double v2 = x2 * x2 * (1.0 - x2 * (1.0 - (7.0 / 12.0) * x2)) * QT_DR;
    /* d/dx of x^2 - x^3 + 7/12 x^4 */
    const double dv1 = QT_DR * QT_ALPHAR * x1 * (2.0 - x1 * (3.0 - (7.0 / 3.0) * x1));
    const double dv2 = QT_DR * QT_ALPHAR * x2 * (2.0 - x2 * (3.0 - (7.0 / 3.0) * x2));
    const double cs = c / (r1 * r2);
    const double th = acos(cs);
    const double dth = th - QT_AHOHEQ * M_PI / 180.0;
    *e += v1 + v2 + 0.5 * QT_KTHETA * dth * dth;
    /* dE/dcos = k dth * dth/dcos = -k dth / sin(th) */
    const double de_dc = -QT_KTHETA * dth / sqrt(1.0 - cs * cs);
    for (int k = 0; k < 3; k++) {
        const double u1 = d1[k] / r1, u2 = d2[k] / r2;
        const double gh1 = dv1 * u1 + de_dc * (u2 - cs * u1) / r1;
        const double gh2 = dv2 * u2 + de_dc * (u1 - cs * u2) / r2;
        g[3 + k] += gh1;
        g[6 + k] += gh2;
        g[k] -= gh1 + gh2;
    }
}

/* charge-charge term q_a q_b / r between points a and b: energy, and the
 * gradient added into ga (at a) and gb (at b) */
static double qt_coulomb(double qq, const double* a, const double* b, double* ga, double* gb)
{
    double d[3], r2 = 0;
    for (int k = 0; k < 3; k++) {
        d[k] = a[k] - b[k];
        r2 += d[k] * d[k];
    }
    const double ir = 1.0 / sqrt(r2), e = qq * ir, f = -e * ir * ir;
    for (int k = 0; k < 3; k++) {
        ga[k] += f * d[k];
        gb[k] -= f * d[k];
    }
    return e;
}

double or_qtip4pf_grad(int nw, const double* crd, double* grad)
{
    double msite[3 * 64], gm[3 * 64];
    if (nw > 64) return NAN;
    double e = 0;
    for (int i = 0; i < 9 * nw; i++) grad[i] = 0.0;
    for (int i = 0; i < 3 * nw; i++) gm[i] = 0.0;
    for (int i = 0; i < nw; i++) {
        const double* w = crd + 9 * i;
        for (int k = 0; k < 3; k++) msite[3 * i + k] = QT_GAMMAM * w[k] + QT_GAMMA1 * (w[3 + k] + w[6 + k]);
        qt_monomer_grad(w, grad + 9 * i, &e);
    }
    for (int i = 0; i < nw; i++) {
        for (int j = 0; j < nw; j++) {
            if (i == j) continue;
            for (int l = 1; l < 3; l++)
                e += qt_coulomb(QT_QH * qt_qM, msite + 3 * i, crd + 9 * j + 3 * l, gm + 3 * i, grad + 9 * j + 3 * l);
        }
        for (int j = i + 1; j < nw; j++) {
            for (int a = 1; a < 3; a++)
                for (int b = 1; b < 3; b++)
                    e += qt_coulomb(QT_QH * QT_QH, crd + 9 * i + 3 * a, crd + 9 * j + 3 * b, grad + 9 * i + 3 * a,
                                    grad + 9 * j + 3 * b);
            double d[3], r2 = 0;
            for (int k = 0; k < 3; k++) {
                d[k] = crd[9 * i + k] - crd[9 * j + k];
                r2 += d[k] * d[k];
            }
            const double s2 = QT_SIGMA * QT_SIGMA / r2, s6 = s2 * s2 * s2;
            e += 4 * QT_EPS * s6 * (s6 - 1.0);
            /* dE/dx_i = 2 dE/dr2 d, dE/dr2 = 4 eps (3 s6 - 6 s12) / r2 */
            const double f = 2.0 * 4 * QT_EPS * (3.0 * s6 - 6.0 * s6 * s6) / r2;
            for (int k = 0; k < 3; k++) {
                grad[9 * i + k] += f * d[k];
                grad[9 * j + k] -= f * d[k];
            }
            e += qt_coulomb(qt_qM * qt_qM, msite + 3 * i, msite + 3 * j, gm + 3 * i, gm + 3 * j);
        }
    }
    for (int i = 0; i < nw; i++)
        for (int k = 0; k < 3; k++) {
            grad[9 * i + k] += QT_GAMMAM * gm[3 * i + k];
            grad[9 * i + 3 + k] += QT_GAMMA1 * gm[3 * i + k];
            grad[9 * i + 6 + k] += QT_GAMMA1 * gm[3 * i + k];
        }
    return e;
}

/* Per-sample stage of the gradient path (SCP3.cpp:205-223, use_gradient):
 * V_anh as or_samples, and Vq = MUa^T (bohr dV/dr / autokcal) - omega % q for
 * all nm0 modes (n x nm0, sample-major).  qTIP4P/f only. */
void or_samples_grad(int nw, const double* x0, const double* MUa, const double* omega, int nm0,
                     const double* normals, int64_t n, double* q_out, double* v_out, double* vq_out)
{
    const double bohr = 0.52917721092, kcal = 627.509474277194;
    const int N3 = 9 * nw;
    double* r = (double*)malloc(sizeof(double) * N3);
    double* g = (double*)malloc(sizeof(double) * N3);
    for (int64_t s = 0; s < n; s++) {
        double* q = q_out + s * nm0;
        for (int k = 0; k < nm0; k++) q[k] = normals[s * nm0 + k] / sqrt(2.0);
        for (int a = 0; a < N3; a++) {
            double acc = 0.0;
            for (int k = 0; k < nm0; k++) acc += MUa[(size_t)k * N3 + a] * q[k];
            r[a] = bohr * (x0[a] + acc);
        }
        const double V = or_qtip4pf_grad(nw, r, g) / kcal;
        for (int a = 0; a < N3; a++) g[a] *= bohr / kcal;
        double h = 0.0;
        for (int k = 0; k < nm0; k++) h += q[k] * (omega[k] * q[k]);
        v_out[s] = V - 0.5 * h;
        for (int k = 0; k < nm0; k++) {
            double acc = 0.0;
            for (int a = 0; a < N3; a++) acc += MUa[(size_t)k * N3 + a] * g[a];
            vq_out[s * nm0 + k] = acc - omega[k] * q[k];
        }
    }
    free(r);
    free(g);
}

/* The gradient (Stein) estimator of <i|V|j> (ScaledMatrixElements.cpp:102-725,
 * TripleExcitations.h), restated by the rule its formulas follow: with
 * phi_i phi_j = prod_m p_m(q_m) over the set S of modes either function
 * excites, every mode m in S contributes the Stein identity
 * E[q g(q)] = 1/2 E[g'(q)] (q ~ N(0, 1/2)) applied to the factor q_m of
 * p_m = p_m(0) + q_m r_m(q_m):
 *     T_m = R_m [ (p_m(0) + r_m'/2) V + (r_m/2) dV/dq_m ],  R_m = prod_{m' != m} p_m',
 * and the estimate is the mean of T_m over S (V itself for <0|V|0>).  One
 * exception reproduces the reference as written: see <3_m|V|3_m> below.
 * Per mode, with h_0..h_3 the oscillator functions (levels a, b):
 *     r_ab = d_a h_b + h_a(0) d_b,  d_a = (h_a(q) - h_a(0)) / q. */
static void ho_parts(int a, double q, double* h, double* h0, double* dh, double* d, double* dd)
{
    const double s2 = sqrt(2.0), s3 = sqrt(3.0);
    switch (a) {
        case 0: *h = 1, *h0 = 1, *dh = 0, *d = 0, *dd = 0; break;
        case 1: *h = s2 * q, *h0 = 0, *dh = s2, *d = s2, *dd = 0; break;
        case 2: *h = (2 * q * q - 1) / s2, *h0 = -1 / s2, *dh = 2 * s2 * q, *d = s2 * q, *dd = s2; break;
        default: *h = (2 * q * q - 3) * q / s3, *h0 = 0, *dh = (6 * q * q - 3) / s3, *d = (2 * q * q - 3) / s3,
                 *dd = 4 * q / s3; break;
    }
}

/* One sample's estimate for the pair of functions given as (mode, level) lists. */
double or_stein_term(const double* q, double V, const double* vq, int ni, const int* mi, const int* li, int nj,
                     const int* mj, const int* lj)
{
    int S[8], A[8], B[8], ns = 0;
    for (int k = 0; k < ni; k++) S[ns] = mi[k], A[ns] = li[k], B[ns] = 0, ns++;
    for (int k = 0; k < nj; k++) {
        int f = -1;
        for (int t = 0; t < ns; t++)
            if (S[t] == mj[k]) f = t;
        if (f >= 0) B[f] = lj[k];
        else S[ns] = mj[k], A[ns] = 0, B[ns] = lj[k], ns++;
    }
    if (ns == 0) return V;
    double p[8], u[8], w[8];
    for (int t = 0; t < ns; t++) {
        double ha, ha0, dha, da, dda, hb, hb0, dhb, db, ddb;
        const double x = q[S[t]];
        ho_parts(A[t], x, &ha, &ha0, &dha, &da, &dda);
        ho_parts(B[t], x, &hb, &hb0, &dhb, &db, &ddb);
        const double r = da * hb + ha0 * db;
        const double dr = dda * hb + da * dhb + ha0 * ddb;
        p[t] = ha * hb;
        u[t] = ha0 * hb0 + 0.5 * dr;
        w[t] = 0.5 * r;
        /* <3_m|V|3_m>: the reference's formula (TripleExcitations.h:763-773) has
         * (q^2 - 3) V where the identity gives (10 q^2 - 3) V; kept for parity */
        if (A[t] == 3 && B[t] == 3) u[t] = (2 * x * x - 3) * (x * x - 3) / 6.0;
    }
    double sum = 0.0;
    for (int t = 0; t < ns; t++) {
        double R = 1.0;
        for (int o = 0; o < ns; o++)
            if (o != t) R *= p[o];
        sum += R * (u[t] * V + w[t] * vq[S[t]]);
    }
    return sum / ns;
}

/* (mode, level) list of basis function R in the order of or_get_bra */
static int basis_modes(int nm, int n2, int n3, size_t R, int* m, int* l)
{
    size_t k = 0;
    if (R == k) return 0;
    k++;
    if (R < k + (size_t)nm) { m[0] = (int)(R - k), l[0] = 1; return 1; }
    k += nm;
    if (R < k + (size_t)n2) { m[0] = (int)(R - k), l[0] = 2; return 1; }
    k += n2;
    for (int a = 0; a < n2; a++)
        for (int b = a + 1; b < n2; b++, k++)
            if (R == k) { m[0] = a, l[0] = 1, m[1] = b, l[1] = 1; return 2; }
    if (R < k + (size_t)n3) { m[0] = (int)(R - k), l[0] = 3; return 1; }
    k += n3;
    for (int a = 0; a < n3; a++)
        for (int b = a + 1; b < n3; b++) {
            if (R == k) { m[0] = a, l[0] = 2, m[1] = b, l[1] = 1; return 2; }
            k++;
            if (R == k) { m[0] = a, l[0] = 1, m[1] = b, l[1] = 2; return 2; }
            k++;
        }
    for (int a = 0; a < n3; a++)
        for (int b = a + 1; b < n3; b++)
            for (int c = b + 1; c < n3; c++, k++)
                if (R == k) { m[0] = a, l[0] = 1, m[1] = b, l[1] = 1, m[2] = c, l[2] = 1; return 3; }
    return -1;
}

int or_basis_modes(int nm, int n2, int n3, int64_t R, int* m, int* l) { return basis_modes(nm, n2, n3, (size_t)R, m, l); }

/* addEpot(q, V, Vq, M) (ScaledMatrixElements.cpp:704-719): M_upper[i,j] += sum_s
 * estimate_ij(s), i <= j.  q_sel, vq_sel: n x nm (selected modes), M nb x nb. */
void or_accumulate_stein(int nm, int n2, int n3, const double* q_sel, const double* v, const double* vq_sel, int64_t n,
                         double* M)
{
    const size_t nb = or_basis_size(nm, n2, n3);
    int* mm = (int*)malloc(sizeof(int) * 3 * nb);
    int* ll = (int*)malloc(sizeof(int) * 3 * nb);
    int* cnt = (int*)malloc(sizeof(int) * nb);
    for (size_t R = 0; R < nb; R++) cnt[R] = basis_modes(nm, n2, n3, R, mm + 3 * R, ll + 3 * R);
    for (size_t j = 0; j < nb; j++)
        for (size_t i = 0; i <= j; i++) {
            double acc = 0.0;
            for (int64_t s = 0; s < n; s++)
                acc += or_stein_term(q_sel + s * nm, v[s], vq_sel + s * nm, cnt[i], mm + 3 * i, ll + 3 * i, cnt[j],
                                     mm + 3 * j, ll + 3 * j);
            M[j * nb + i] += acc;
        }
    free(mm), free(ll), free(cnt);
}
