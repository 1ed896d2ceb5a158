// TTM3-F energy, warp-cooperative: one warp per geometry.  Same model and
// constants as the reference (ttm3f.cpp:92-321; Partridge-Schwenke monomer and
// dipole-moment surface ps.cpp:470-836; smeared interactions
// ttm3f-bits-smear.cpp:17-287):
//   lanes 0..nw-1   one water each: M site, PS monomer energy, DMS charges
//   all lanes       strided over the pair tasks: smeared potentials, fields,
//                   the 3nw x 3nw dipole tensor (shared-memory atomics for the
//                   per-site sums)
//   lanes 0..3nw-1  one row each of the Jacobi sweep for the induced dipoles
// The induced field is zeroed before the first sweep (the reference's fill at
// ttm3f.cpp:108-109 starts at Efq and leaves Efd to whatever the heap held).
// Every data-dependent loop is bounded: the incomplete-gamma series and
// continued fraction at 1000 terms, the dipole iteration at 500 sweeps
// (ttm3f.cpp:31), after which *iters reports 501 and the caller counts the
// sample as not converged (the reference only asserts, and not under NDEBUG,
// ttm3f.cpp:309).
#pragma once
#include "common.cuh"

namespace scp3 {
namespace ttm {

struct Consts {
    double AA_HH, AA_HM, AA_MM;   // pow(polfac*polfac, 1/6), ttm3f.cpp:25-27
    double aXX13;                 // pow(0.175, 1/3), ttm3f-bits-smear.cpp:201
    double c5z[245];              // combined monomer coefficients, ps.cpp:508-511
    double phh1;                  // f5z*phh1A*exp(phh2), ps.cpp:514
    double coefD[84];
    unsigned char idx1[245], idx2[245], idx3[245];
    unsigned char idxD0[84], idxD1[84], idxD2[84];
};

// Defined here: only sampling.cu includes this header (whole-program compilation).
__constant__ Consts kC;

constexpr double kPolarM = 1.444;
constexpr double kDebye = 4.8033324;
constexpr double kChargeCon = 18.22234397655801030455;
constexpr double kGammaM = 0.46, kGamma1 = 1.0 - kGammaM, kGamma2 = kGammaM / 2;  // ttm3f-bits.h:21-23
constexpr double kVdwC = -0.72298855E+03, kVdwD = 0.10211829E+06, kVdwE = 0.37170376E+01;
constexpr double kAXX = 0.175;
constexpr int kSeriesCap = 1000;

// scratch per warp, in elements of T: charge, phi, efq, dip, dipp, efd (3nw each),
// ddt (3nw x 3nw), power tables (48 per water); with the gradient also the
// charge derivatives (27 per water) and the M-site forces (3nw)
__host__ __device__ inline size_t scratch_elems(int nw, bool grad = false)
{
    return (size_t)18 * nw + (size_t)9 * nw * nw + 48 * nw + (grad ? (size_t)30 * nw : 0);
}

template <typename T> struct Eps;
template <> struct Eps<double> { static constexpr double v = 2.220446049250313e-16; static constexpr double fpmin = 2.2250738585072014e-308 / 2.220446049250313e-16; };
template <> struct Eps<float> { static constexpr float v = 1.1920929e-07f; static constexpr float fpmin = 1.1754944e-38f / 1.1920929e-07f; };

// gammq(2/3, x) * Gamma(2/3): series below 5/3, continued fraction above
// (ttm3f-bits-smear.cpp:17-80).
template <typename T>
__device__ T gammq23(T x)
{
    const T a = T(2.0 / 3.0), eps = Eps<T>::v, fpmin = Eps<T>::fpmin;
    if (x < T(5.0 / 3.0)) {
        T ap = a, sum = T(1) / a, del = sum;
        for (int it = 0; it < kSeriesCap; it++) {
            ++ap;
            del *= x / ap;
            sum += del;
            if (fabs(del) < fabs(sum) * eps) break;
        }
        return T(1.354117939426400e+00) - sum * exp(-x + a * log(x));
    }
    T b = x + T(1) - a, c = T(1) / fpmin, d = T(1) / b, h = d;
    for (int i = 1; i <= kSeriesCap; ++i) {
        const T an = -i * (i - a);
        b += T(2);
        d = an * d + b;
        if (fabs(d) < fpmin) d = fpmin;
        c = b + an / c;
        if (fabs(c) < fpmin) c = fpmin;
        d = T(1) / d;
        const T del = d * c;
        h *= del;
        if (fabs(del - T(1)) <= eps) break;
    }
    return exp(-x + a * log(x)) * h;
}

// smear0/01/012 (ttm3f-bits-smear.cpp:213-287): ts0 always, ts1/ts2 on request.
template <typename T>
__device__ __forceinline__ void smear(T r, T AA, T& ts0, T& ts1, T* ts2)
{
    const T dri = T(1) / r, drsqi = dri * dri;
    const T rA = r / AA, rA3 = rA * rA * rA;
    const T e1 = exp(-T(kAXX) * rA3);
    ts0 = (T(1) - e1 + T(kC.aXX13) * rA * gammq23(T(kAXX) * rA3)) * dri;
    ts1 = (T(1) - e1) * dri * drsqi;
    if (ts2) *ts2 = (ts1 - e1 * T(kAXX) / (AA * AA * AA)) * drsqi;
}

template <typename T>
__device__ __forceinline__ void powers(T x1, T x2, T x3, T* f /* [3][16] */)
{
    f[0] = f[16] = f[32] = T(0);
    f[1] = f[17] = f[33] = T(1);
    for (int j = 2; j < 16; j++) {
        f[j] = f[j - 1] * x1;
        f[16 + j] = f[16 + j - 1] * x2;
        f[32 + j] = f[32 + j - 1] * x3;
    }
}

// Monomer energy (pot_nasa, energy part) and charges (dms_nasa with ttm3=true),
// kcal/mol and elementary charges, for the water at w[9].  f: 48 scratch.
template <typename T>
__device__ void monomer(const T* w, T* f, T& e, T q3[3])
{
    constexpr double reoh = 0.958649, b1 = 2.0, roh = 0.9519607159623009, alphaoh = 2.587949757553683;
    constexpr double deohA = 42290.92019288289, phh2 = 12.66426998162947, f5z = 0.999677885;
    constexpr double costhe = -.24780227221366464506;
    T roh1[3], roh2[3], rhh[3], d1 = 0, d2 = 0, dhh = 0;
    for (int i = 0; i < 3; i++) {
        roh1[i] = w[3 + i] - w[i];
        roh2[i] = w[6 + i] - w[i];
        rhh[i] = w[3 + i] - w[6 + i];
        d1 += roh1[i] * roh1[i];
        d2 += roh2[i] * roh2[i];
        dhh += rhh[i] * rhh[i];
    }
    d1 = sqrt(d1);
    d2 = sqrt(d2);
    dhh = sqrt(dhh);
    const T costh = (roh1[0] * roh2[0] + roh1[1] * roh2[1] + roh1[2] * roh2[2]) / (d1 * d2);
    // --- pot_nasa (ps.cpp:486-570)
    const T deoh = T(f5z * deohA);
    const T e1x = exp(-T(alphaoh) * (d1 - T(roh))), e2x = exp(-T(alphaoh) * (d2 - T(roh)));
    const T va = deoh * (e1x * (e1x - T(2)) + e2x * (e2x - T(2)));
    const T vb = T(kC.phh1) * exp(-T(phh2) * dhh);
    const T x1 = (d1 - T(reoh)) / T(reoh), x2 = (d2 - T(reoh)) / T(reoh);
    powers(x1, x2, costh - T(costhe), f);
    const T dr1 = d1 - T(reoh), dr2 = d2 - T(reoh);
    const T efac = exp(-T(b1) * (dr1 * dr1 + dr2 * dr2));
    T sum0 = 0;
    for (int j = 1; j < 245; j++) {
        const int I = kC.idx1[j], J = kC.idx2[j], K = kC.idx3[j];
        sum0 += T(kC.c5z[j]) * (f[I] * f[16 + J] + f[J] * f[16 + I]) * f[32 + K];
    }
    e = (va + vb + (T(2) * T(kC.c5z[0]) + efac * sum0) + T(0.44739574026257)) * T(0.00285914375100642899);
    // --- dms_nasa (ps.cpp:605-790), charges only
    const T efacD = exp(-(dr1 * dr1 + dr2 * dr2));   // b1D = 1
    T p1 = 0, p2 = 0;
    const T pl1 = costh, pl2 = T(0.5) * (T(3) * pl1 * pl1 - T(1));
    for (int j = 1; j < 84; j++) {
        const int I = kC.idxD0[j], J = kC.idxD1[j], K = kC.idxD2[j];
        p1 += T(kC.coefD[j]) * f[I] * f[16 + J] * f[32 + K];
        p2 += T(kC.coefD[j]) * f[J] * f[16 + I] * f[32 + K];
    }
    const T xx = T(0.529177249);
    const T pc0 = T(0.2999) * (pow(d1, T(-0.6932)) + pow(d2, T(-0.6932))) *
                  (T(1.0099) + pl1 * T(-0.1801) + pl2 * T(0.0892));
    p1 = T(kC.coefD[0]) + p1 * efacD + pc0 * xx;
    p2 = T(kC.coefD[0]) + p2 * efacD + pc0 * xx;
    T axb[3] = {roh1[1] * roh2[2] - roh1[2] * roh2[1], -roh1[0] * roh2[2] + roh1[2] * roh2[0],
                roh1[0] * roh2[1] - roh1[1] * roh2[0]};
    const T sinth = sqrt(axb[0] * axb[0] + axb[1] * axb[1] + axb[2] * axb[2]) / (d1 * d2);
    const T ang = atan2(sinth, costh);
    const T m1 = T(0.5) * (d1 - T(0.9578)) + T(0.012) * (ang - T(1.82400520401572996557));
    const T m2 = T(0.5) * (d2 - T(0.9578)) + T(0.012) * (ang - T(1.82400520401572996557));
    q3[0] = -(p1 + p2) - (m1 + m2);
    q3[1] = p1 + m1;
    q3[2] = p2 + m2;
}

// Energy (kcal/mol) of crd[9nw] (shared, T); ms: 3nw shared; sc: scratch_elems(nw).
// Returns the sum on all lanes; *iters = Jacobi sweeps (kTtmMaxIter+1 if capped).
template <typename T>
__device__ double energy_warp(const T* crd, T* ms, T* sc, int nw, const uint32_t* __restrict__ tasks, int ntasks,
                              int lane, int* iters)
{
    const int n3 = 3 * nw;
    T *chg = sc, *phi = chg + n3, *efq = phi + n3, *dip = efq + n3, *dipp = dip + n3, *efd = dipp + n3,
      *ddt = efd + n3, *fpow = ddt + n3 * n3;
    for (int i = lane; i < n3 * n3; i += 32) ddt[i] = T(0);
    for (int i = lane; i < n3; i += 32) phi[i] = efq[i] = efd[i] = T(0);
    double part = 0;
    for (int i = lane; i < nw; i += 32) {
        const T* w = crd + 9 * i;
        for (int k = 0; k < 3; k++) ms[3 * i + k] = T(kGamma1) * w[k] + T(kGamma2) * (w[3 + k] + w[6 + k]);
        T e, q3[3];
        monomer(w, fpow + 48 * i, e, q3);
        part += (double)e;
        const T t = T(kGamma2 / kGamma1);
        chg[3 * i + 0] = T(kChargeCon) * q3[0] / T(kGamma1);
        chg[3 * i + 1] = T(kChargeCon) * (q3[1] + t * (q3[1] + q3[2]));
        chg[3 * i + 2] = T(kChargeCon) * (q3[2] + t * (q3[1] + q3[2]));
    }
    __syncwarp();
    for (int t = lane; t < ntasks; t += 32) {
        const uint32_t task = __ldg(tasks + t), type = task & 3u, a = (task >> 2) & 0x7fffu, b = task >> 17;
        if (type == 0) {            // M site of water a, H atom b  (ttm3f.cpp:149-174)
            const int ia = 3 * a;
            T R[3];
            for (int k = 0; k < 3; k++) R[k] = ms[ia + k] - crd[3 * b + k];
            T ts0, ts1;
            smear<T>(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), T(kC.AA_HM), ts0, ts1, nullptr);
            const int jb = b;        // charge index of atom b = 3*water + l
            atomicAdd(phi + ia, ts0 * chg[jb]);
            atomicAdd(phi + jb, ts0 * chg[ia]);
            for (int k = 0; k < 3; k++) atomicAdd(efq + ia + k, chg[jb] * ts1 * R[k]);
        } else if (type == 1) {     // H/H  (ttm3f.cpp:183-200)
            T ts0, ts1;
            smear<T>(sqrt(dist2(crd + 3 * a, crd + 3 * b)), T(kC.AA_HH), ts0, ts1, nullptr);
            atomicAdd(phi + a, chg[b] * ts0);
            atomicAdd(phi + b, chg[a] * ts0);
        } else if (type == 2) {     // O/O van der Waals  (ttm3f.cpp:204-219)
            const T r2 = dist2(crd + 3 * a, crd + 3 * b);
            part += (double)(T(kVdwC) / (r2 * r2 * r2) + T(kVdwD) * exp(-T(kVdwE) * sqrt(r2)));
        } else {                    // M/M  (ttm3f.cpp:222-256)
            const int i3 = 3 * a, j3 = 3 * b;
            T R[3];
            for (int k = 0; k < 3; k++) R[k] = ms[i3 + k] - ms[j3 + k];
            T ts0, ts1, ts2;
            smear<T>(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), T(kC.AA_MM), ts0, ts1, &ts2);
            atomicAdd(phi + i3, ts0 * chg[j3]);
            atomicAdd(phi + j3, ts0 * chg[i3]);
            for (int k = 0; k < 3; k++) {
                atomicAdd(efq + i3 + k, chg[j3] * ts1 * R[k]);
                atomicAdd(efq + j3 + k, -(chg[i3] * ts1 * R[k]));
            }
            for (int k = 0; k < 3; k++)
                for (int l = k; l < 3; l++) {
                    const T d = T(3) * ts2 * R[k] * R[l] - (k == l ? ts1 : T(0));
                    ddt[n3 * (i3 + k) + j3 + l] = d;
                    ddt[n3 * (j3 + k) + i3 + l] = d;
                    ddt[n3 * (i3 + l) + j3 + k] = d;
                    ddt[n3 * (j3 + l) + i3 + k] = d;
                }
        }
    }
    __syncwarp();
    // induced dipoles (ttm3f.cpp:268-307); the iterate is carried in FP64 so the
    // FP32 form can still reach its residual target
    const double tol = sizeof(T) == 8 ? 1.0e-15 : 1.0e-8;
    const double stath = kDebye / kChargeCon / sqrt((double)nw);
    double dcur = 0.0, dprev = 0.0, efqk = 0.0;
    if (lane < n3) {
        efqk = (double)efq[lane];
        dcur = dprev = kPolarM * efqk;
        dip[lane] = (T)dcur;
    }
    __syncwarp();
    int it = 0;
    for (; it < kTtmMaxIter; it++) {
        double ef = 0.0, del2 = 0.0;
        if (lane < n3) {
            const T* row = ddt + n3 * lane;
            for (int l = 0; l < n3; l++) ef += (double)row[l] * (double)dip[l];
            double d = kPolarM * (efqk + ef);
            d = 0.7 * d + (1.0 - 0.7) * dprev;
            const double del = d - dprev;
            del2 = del * del;
            dcur = d;
        }
        del2 = warp_sum(del2);
        __syncwarp();
        if (lane < n3) dip[lane] = (T)dcur;
        __syncwarp();
        if (sqrt(del2) * stath < tol) break;
        dprev = dcur;
    }
    *iters = (it < kTtmMaxIter) ? it + 1 : kTtmMaxIter + 1;
    double el = 0.0, ind = 0.0;
    if (lane < n3) {
        el = (double)phi[lane] * (double)chg[lane];
        ind = -dcur * efqk;
    }
    const double tot = warp_sum(part) + warp_sum(el) / 2 + warp_sum(ind) / 2;
    __syncwarp();
    return tot;
}

// ---------------------------------------------------------------- energy + gradient
// The E+g operator (ttm3f.cpp:325-720), FP64: the monomer energy with its
// gradient (pot_nasa with dr, ps.cpp:486-603), the charges with their
// derivatives (dms_nasa with dq3, ps.cpp:605-836), the smeared pair terms with
// their forces, the induced dipoles as in energy_warp, then the charge-dipole
// and dipole-dipole forces, the M-site forces spread over O, H, H, and the
// terms of the geometry-dependent charges.

__device__ __forceinline__ void smear123(double r, double AA, double& ts1, double& ts2, double& ts3)
{
    const double dri = 1.0 / r, drsqi = dri * dri;
    const double rA = r / AA, rA3 = rA * rA * rA;
    const double e1 = exp(-kAXX * rA3);
    const double AA3 = AA * AA * AA;
    ts1 = (1.0 - e1) * dri * drsqi;
    ts2 = (ts1 - e1 * kAXX / AA3) * drsqi;
    ts3 = (ts2 - 0.6 * e1 * r * kAXX * kAXX / (AA3 * AA3)) * drsqi;
}

// Monomer at w[9]: energy e (kcal/mol), its gradient g9 (written), the charges
// q3 and the derivatives of the scaled site charges grdq[27] (GRDQ layout of
// ttm3f.cpp:371-393: [atom H1, H2, O][charge H1, H2, M][xyz], times CHARGECON).
__device__ inline void monomer_grad(const double* w, double* f, double& e, double q3[3], double* g9, double* grdq)
{
    constexpr double reoh = 0.958649, b1 = 2.0, roh = 0.9519607159623009, alphaoh = 2.587949757553683;
    constexpr double deohA = 42290.92019288289, phh2 = 12.66426998162947, f5z = 0.999677885;
    constexpr double costhe = -.24780227221366464506, tocal = 0.00285914375100642899;
    constexpr double ath0 = 1.82400520401572996557, dms1 = 0.5, dms2 = 0.9578, dms3 = 0.012;
    double roh1[3], roh2[3], rhh[3], d1 = 0, d2 = 0, dhh = 0;
    for (int i = 0; i < 3; i++) {
        roh1[i] = w[3 + i] - w[i];
        roh2[i] = w[6 + i] - w[i];
        rhh[i] = w[3 + i] - w[6 + i];
        d1 += roh1[i] * roh1[i];
        d2 += roh2[i] * roh2[i];
        dhh += rhh[i] * rhh[i];
    }
    d1 = sqrt(d1);
    d2 = sqrt(d2);
    dhh = sqrt(dhh);
    const double costh = (roh1[0] * roh2[0] + roh1[1] * roh2[1] + roh1[2] * roh2[2]) / (d1 * d2);
    // --- pot_nasa with its derivatives
    const double deoh = f5z * deohA;
    const double e1x = exp(-alphaoh * (d1 - roh)), e2x = exp(-alphaoh * (d2 - roh));
    const double va = deoh * (e1x * (e1x - 2.0) + e2x * (e2x - 2.0));
    const double vb = kC.phh1 * exp(-phh2 * dhh);
    const double dva1 = 2.0 * alphaoh * deoh * e1x * (1.0 - e1x) / d1;
    const double dva2 = 2.0 * alphaoh * deoh * e2x * (1.0 - e2x) / d2;
    const double dvb = -phh2 * vb / dhh;
    const double x1 = (d1 - reoh) / reoh, x2 = (d2 - reoh) / reoh;
    powers(x1, x2, costh - costhe, f);
    const double dr1 = d1 - reoh, dr2 = d2 - reoh;
    const double efac = exp(-b1 * (dr1 * dr1 + dr2 * dr2));
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int j = 1; j < 245; j++) {
        const int I = kC.idx1[j], J = kC.idx2[j], K = kC.idx3[j];
        const double c = kC.c5z[j];
        const double sym = f[I] * f[16 + J] + f[J] * f[16 + I];
        s0 += c * sym * f[32 + K];
        s1 += c * ((I - 1) * f[I - 1] * f[16 + J] + (J - 1) * f[J - 1] * f[16 + I]) * f[32 + K];
        s2 += c * ((J - 1) * f[I] * f[16 + J - 1] + (I - 1) * f[J] * f[16 + I - 1]) * f[32 + K];
        s3 += c * sym * (K - 1) * f[32 + K - 1];
    }
    e = (va + vb + (2.0 * kC.c5z[0] + efac * s0) + 0.44739574026257) * tocal;
    const double dvc1 = (-2 * b1 * efac * dr1 * s0 + efac * s1 / reoh) / d1;
    const double dvc2 = (-2 * b1 * efac * dr2 * s0 + efac * s2 / reoh) / d2;
    const double dvcc = efac * s3;
    for (int i = 0; i < 3; i++) {
        const double h1 = dva1 * roh1[i] + dvb * rhh[i] + dvc1 * roh1[i] +
                          dvcc * (roh2[i] / (d1 * d2) - costh * roh1[i] / (d1 * d1));
        const double h2 = dva2 * roh2[i] - dvb * rhh[i] + dvc2 * roh2[i] +
                          dvcc * (roh1[i] / (d1 * d2) - costh * roh2[i] / (d2 * d2));
        g9[3 + i] = h1 * tocal;
        g9[6 + i] = h2 * tocal;
        g9[i] = -(h1 + h2) * tocal;
    }
    // --- dms_nasa with dq3
    const double efacD = exp(-(dr1 * dr1 + dr2 * dr2));   // b1D = 1
    double p1 = 0, p2 = 0, dp1r1 = 0, dp1r2 = 0, dp1c = 0, dp2r1 = 0, dp2r2 = 0, dp2c = 0;
    const double pl1 = costh, pl2 = 0.5 * (3 * pl1 * pl1 - 1.0);
    for (int j = 1; j < 84; j++) {
        const int I = kC.idxD0[j], J = kC.idxD1[j], K = kC.idxD2[j];
        const double c = kC.coefD[j];
        p1 += c * f[I] * f[16 + J] * f[32 + K];
        p2 += c * f[J] * f[16 + I] * f[32 + K];
        dp1r1 += c * (I - 1) * f[I - 1] * f[16 + J] * f[32 + K];
        dp1r2 += c * (J - 1) * f[I] * f[16 + J - 1] * f[32 + K];
        dp1c += c * (K - 1) * f[I] * f[16 + J] * f[32 + K - 1];
        dp2r1 += c * (J - 1) * f[J - 1] * f[16 + I] * f[32 + K];
        dp2r2 += c * (I - 1) * f[J] * f[16 + I - 1] * f[32 + K];
        dp2c += c * (K - 1) * f[J] * f[16 + I] * f[32 + K - 1];
    }
    const double xx = 0.529177249, xx2 = xx * xx;
    dp1r1 /= reoh / xx;
    dp1r2 /= reoh / xx;
    dp2r1 /= reoh / xx;
    dp2r2 /= reoh / xx;
    const double pa = 0.2999, pb = -0.6932, pc0c = 1.0099, pc1 = -0.1801, pc2 = 0.0892;
    const double ang_f = pc0c + pl1 * pc1 + pl2 * pc2;
    const double pc0 = pa * (pow(d1, pb) + pow(d2, pb)) * ang_f;
    const double dpc0r1 = pa * pb * pow(d1, pb - 1) * ang_f * xx2;
    const double dpc0r2 = pa * pb * pow(d2, pb - 1) * ang_f * xx2;
    const double dpc0c = pa * (pow(d1, pb) + pow(d2, pb)) * (pc1 + 0.5 * (6.0 * pl1) * pc2) * xx;
    const double defr1 = -2.0 * dr1 * efacD * xx, defr2 = -2.0 * dr2 * efacD * xx;
    dp1r1 = dp1r1 * efacD + p1 * defr1 + dpc0r1;
    dp1r2 = dp1r2 * efacD + p1 * defr2 + dpc0r2;
    dp1c = dp1c * efacD + dpc0c;
    dp2r1 = dp2r1 * efacD + p2 * defr1 + dpc0r1;
    dp2r2 = dp2r2 * efacD + p2 * defr2 + dpc0r2;
    dp2c = dp2c * efacD + dpc0c;
    p1 = kC.coefD[0] + p1 * efacD + pc0 * xx;
    p2 = kC.coefD[0] + p2 * efacD + pc0 * xx;
    dp1r1 /= xx;
    dp1r2 /= xx;
    dp2r1 /= xx;
    dp2r2 /= xx;
    const double axb[3] = {roh1[1] * roh2[2] - roh1[2] * roh2[1], -roh1[0] * roh2[2] + roh1[2] * roh2[0],
                           roh1[0] * roh2[1] - roh1[1] * roh2[0]};
    const double sinth = sqrt(axb[0] * axb[0] + axb[1] * axb[1] + axb[2] * axb[2]) / (d1 * d2);
    const double ang = atan2(sinth, costh);
    const double m1 = dms1 * (d1 - dms2) + dms3 * (ang - ath0);
    const double m2 = dms1 * (d2 - dms2) + dms3 * (ang - ath0);
    q3[0] = -(p1 + p2) - (m1 + m2);
    q3[1] = p1 + m1;
    q3[2] = p2 + m2;
    dp1r1 += dms1;
    dp2r2 += dms1;
    dp1c -= dms3 / sinth;
    dp2c -= dms3 / sinth;
    const double f1q1r13 = (dp1r1 - dp1c * costh / d1) / d1, f1q1r23 = dp1c / (d1 * d2);
    const double f2q1r23 = (dp1r2 - dp1c * costh / d2) / d2, f2q1r13 = dp1c / (d2 * d1);
    const double f1q2r13 = (dp2r1 - dp2c * costh / d1) / d1, f1q2r23 = dp2c / (d1 * d2);
    const double f2q2r23 = (dp2r2 - dp2c * costh / d2) / d2, f2q2r13 = dp2c / (d2 * d1);
    double dq[27];   // [atom H1, H2, O][charge h1, h2, O][xyz]
    for (int k = 0; k < 3; k++) {
        dq[0 * 9 + 0 * 3 + k] = f1q1r13 * roh1[k] + f1q1r23 * roh2[k];
        dq[1 * 9 + 0 * 3 + k] = f2q1r13 * roh1[k] + f2q1r23 * roh2[k];
        dq[2 * 9 + 0 * 3 + k] = -(dq[k] + dq[9 + k]);
        dq[0 * 9 + 1 * 3 + k] = f1q2r13 * roh1[k] + f1q2r23 * roh2[k];
        dq[1 * 9 + 1 * 3 + k] = f2q2r13 * roh1[k] + f2q2r23 * roh2[k];
        dq[2 * 9 + 1 * 3 + k] = -(dq[3 + k] + dq[9 + 3 + k]);
        dq[0 * 9 + 2 * 3 + k] = -(dq[k] + dq[3 + k]);
        dq[1 * 9 + 2 * 3 + k] = -(dq[9 + k] + dq[9 + 3 + k]);
        dq[2 * 9 + 2 * 3 + k] = -(dq[18 + k] + dq[18 + 3 + k]);
    }
    const double t = kGamma2 / kGamma1;
    for (int a = 0; a < 3; a++)
        for (int k = 0; k < 3; k++) {
            const double h1 = dq[9 * a + k], h2 = dq[9 * a + 3 + k], o = dq[9 * a + 6 + k];
            grdq[9 * a + 0 + k] = kChargeCon * (h1 + t * (h1 + h2));
            grdq[9 * a + 3 + k] = kChargeCon * (h2 + t * (h2 + h1));
            grdq[9 * a + 6 + k] = kChargeCon * (o - 2 * t * (h1 + h2));
        }
}

// Energy (kcal/mol, all lanes) and gradient g[9nw] (kcal/mol/A, shared, complete
// after the call) of crd[9nw] (shared); ms 3nw shared; sc: scratch_elems(nw, true).
__device__ inline double energy_grad_warp(const double* crd, double* ms, double* sc, double* g, int nw,
                                          const uint32_t* __restrict__ tasks, int ntasks, int lane, int* iters)
{
    const int n3 = 3 * nw;
    double *chg = sc, *phi = chg + n3, *efq = phi + n3, *dip = efq + n3, *dipp = dip + n3, *efd = dipp + n3,
           *ddt = efd + n3, *fpow = ddt + n3 * n3, *grdq = fpow + 48 * nw, *dM = grdq + 27 * nw;
    for (int i = lane; i < n3 * n3; i += 32) ddt[i] = 0.0;
    for (int i = lane; i < n3; i += 32) phi[i] = efq[i] = efd[i] = dM[i] = 0.0;
    double part = 0;
    for (int i = lane; i < nw; i += 32) {
        const double* w = crd + 9 * i;
        for (int k = 0; k < 3; k++) ms[3 * i + k] = kGamma1 * w[k] + kGamma2 * (w[3 + k] + w[6 + k]);
        double e, q3[3];
        monomer_grad(w, fpow + 48 * i, e, q3, g + 9 * i, grdq + 27 * i);
        part += e;
        const double t = kGamma2 / kGamma1;
        chg[3 * i + 0] = kChargeCon * q3[0] / kGamma1;
        chg[3 * i + 1] = kChargeCon * (q3[1] + t * (q3[1] + q3[2]));
        chg[3 * i + 2] = kChargeCon * (q3[2] + t * (q3[1] + q3[2]));
    }
    __syncwarp();
    // pair terms with their forces (ttm3f.cpp:403-520)
    for (int t = lane; t < ntasks; t += 32) {
        const uint32_t task = __ldg(tasks + t), type = task & 3u, a = (task >> 2) & 0x7fffu, b = task >> 17;
        if (type == 0) {            // M site of water a, H atom b
            const int ia = 3 * a;
            double R[3];
            for (int k = 0; k < 3; k++) R[k] = ms[ia + k] - crd[3 * b + k];
            double ts0, ts1;
            smear<double>(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), kC.AA_HM, ts0, ts1, nullptr);
            atomicAdd(phi + ia, ts0 * chg[b]);
            atomicAdd(phi + b, ts0 * chg[ia]);
            const double tmp1 = chg[b] * ts1, tmp2 = chg[ia] * tmp1;
            for (int k = 0; k < 3; k++) {
                atomicAdd(efq + ia + k, tmp1 * R[k]);
                atomicAdd(g + 3 * b + k, tmp2 * R[k]);
            }
        } else if (type == 1) {     // H/H
            double R[3];
            for (int k = 0; k < 3; k++) R[k] = crd[3 * a + k] - crd[3 * b + k];
            double ts0, ts1;
            smear<double>(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), kC.AA_HH, ts0, ts1, nullptr);
            atomicAdd(phi + a, chg[b] * ts0);
            atomicAdd(phi + b, chg[a] * ts0);
            const double qq = chg[a] * chg[b] * ts1;
            for (int k = 0; k < 3; k++) {
                atomicAdd(g + 3 * a + k, -qq * R[k]);
                atomicAdd(g + 3 * b + k, qq * R[k]);
            }
        } else if (type == 2) {     // O/O van der Waals
            double R[3];
            for (int k = 0; k < 3; k++) R[k] = crd[3 * a + k] - crd[3 * b + k];
            const double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2], r = sqrt(r2), r6 = r2 * r2 * r2;
            const double expon = kVdwD * exp(-kVdwE * r);
            part += kVdwC / r6 + expon;
            const double tmp = -(6.0 * kVdwC / r6) / r2 - kVdwE * expon / r;
            for (int k = 0; k < 3; k++) {
                atomicAdd(g + 3 * a + k, tmp * R[k]);
                atomicAdd(g + 3 * b + k, -tmp * R[k]);
            }
        } else {                    // M/M
            const int i3 = 3 * a, j3 = 3 * b;
            double R[3];
            for (int k = 0; k < 3; k++) R[k] = ms[i3 + k] - ms[j3 + k];
            double ts0, ts1, ts2;
            smear<double>(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), kC.AA_MM, ts0, ts1, &ts2);
            atomicAdd(phi + i3, ts0 * chg[j3]);
            atomicAdd(phi + j3, ts0 * chg[i3]);
            for (int k = 0; k < 3; k++) {
                atomicAdd(efq + i3 + k, chg[j3] * ts1 * R[k]);
                atomicAdd(efq + j3 + k, -(chg[i3] * ts1 * R[k]));
            }
            for (int k = 0; k < 3; k++)
                for (int l = k; l < 3; l++) {
                    const double d = 3.0 * ts2 * R[k] * R[l] - (k == l ? ts1 : 0.0);
                    ddt[n3 * (i3 + k) + j3 + l] = d;
                    ddt[n3 * (j3 + k) + i3 + l] = d;
                    ddt[n3 * (i3 + l) + j3 + k] = d;
                    ddt[n3 * (j3 + l) + i3 + k] = d;
                }
        }
    }
    __syncwarp();
    // induced dipoles (ttm3f.cpp:528-581)
    const double stath = kDebye / kChargeCon / sqrt((double)nw);
    double dcur = 0.0, dprev = 0.0, efqk = 0.0;
    if (lane < n3) {
        efqk = efq[lane];
        dcur = dprev = kPolarM * efqk;
        dip[lane] = dcur;
    }
    __syncwarp();
    int it = 0;
    for (; it < kTtmMaxIter; it++) {
        double ef = 0.0, del2 = 0.0;
        if (lane < n3) {
            const double* row = ddt + n3 * lane;
            for (int l = 0; l < n3; l++) ef += row[l] * dip[l];
            double d = kPolarM * (efqk + ef);
            d = 0.7 * d + (1.0 - 0.7) * dprev;
            const double del = d - dprev;
            del2 = del * del;
            dcur = d;
        }
        del2 = warp_sum(del2);
        __syncwarp();
        if (lane < n3) dip[lane] = dcur;
        __syncwarp();
        if (sqrt(del2) * stath < 1.0e-15) break;
        dprev = dcur;
    }
    *iters = (it < kTtmMaxIter) ? it + 1 : kTtmMaxIter + 1;
    double el = 0.0, ind = 0.0;
    if (lane < n3) {
        el = phi[lane] * chg[lane];
        ind = -dcur * efqk;
    }
    const double tot = warp_sum(part) + warp_sum(el) / 2 + warp_sum(ind) / 2;
    __syncwarp();
    // charge-dipole and dipole-dipole forces (ttm3f.cpp:594-676)
    for (int t = lane; t < ntasks; t += 32) {
        const uint32_t task = __ldg(tasks + t), type = task & 3u, a = (task >> 2) & 0x7fffu, b = task >> 17;
        if (type == 0) {            // dipole of M(a), charge of H atom b
            const int i3 = 3 * a;
            double R[3], diR = 0;
            for (int k = 0; k < 3; k++) {
                R[k] = ms[i3 + k] - crd[3 * b + k];
                diR += dip[i3 + k] * R[k];
            }
            const double r = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
            const double dri = 1.0 / r, drsqi = dri * dri, rA = r / kC.AA_HM, e1 = exp(-kAXX * rA * rA * rA);
            const double ts1 = (1.0 - e1) * dri * drsqi;
            const double ts2 = (ts1 - e1 * kAXX / (kC.AA_HM * kC.AA_HM * kC.AA_HM)) * drsqi;   // smear12
            for (int k = 0; k < 3; k++) {
                const double derij = chg[b] * (3 * ts2 * diR * R[k] - ts1 * dip[i3 + k]);
                atomicAdd(dM + i3 + k, derij);
                atomicAdd(g + 3 * b + k, -derij);
            }
            atomicAdd(phi + b, -ts1 * diR);
        } else if (type == 3) {     // M(a), M(b): both charge-dipole directions, dipole-dipole once
            const int i3 = 3 * a, j3 = 3 * b;
            double R[3], diR = 0, djR = 0, didj = 0;
            for (int k = 0; k < 3; k++) {
                R[k] = ms[i3 + k] - ms[j3 + k];
                diR += dip[i3 + k] * R[k];
                djR += dip[j3 + k] * R[k];
                didj += dip[i3 + k] * dip[j3 + k];
            }
            double ts1, ts2, ts3;
            smear123(sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]), kC.AA_MM, ts1, ts2, ts3);
            for (int k = 0; k < 3; k++) {
                // (i, j): dipole of i, charge of j, added to i and taken from j;
                // (j, i): R and dip_j.R change sign together, added to j and taken from i
                const double dij = chg[j3] * (3 * ts2 * diR * R[k] - ts1 * dip[i3 + k]);
                const double dji = chg[i3] * (3 * ts2 * djR * R[k] - ts1 * dip[j3 + k]);
                const double dd = -3 * ts2 * (didj * R[k] + djR * dip[i3 + k] + diR * dip[j3 + k]) +
                                  15 * ts3 * diR * djR * R[k];
                atomicAdd(dM + i3 + k, dij - dji + dd);
                atomicAdd(dM + j3 + k, -(dij - dji + dd));
            }
            atomicAdd(phi + j3, -ts1 * diR);
            atomicAdd(phi + i3, ts1 * djR);
        }
    }
    __syncwarp();
    // M-site forces onto O, H, H, and the charges' geometry dependence (ttm3f.cpp:680-716)
    for (int i = lane; i < nw; i += 32) {
        const int i3 = 3 * i;
        const double* gq = grdq + 27 * i;
        for (int k = 0; k < 3; k++) {
            const double tmp = dM[i3 + k] - chg[i3] * efq[i3 + k];
            g[9 * i + k] += kGamma1 * tmp + gq[18 + 0 + k] * phi[i3 + 1] + gq[18 + 3 + k] * phi[i3 + 2] +
                            gq[18 + 6 + k] * phi[i3];
            g[9 * i + 3 + k] += kGamma2 * tmp + gq[0 + k] * phi[i3 + 1] + gq[3 + k] * phi[i3 + 2] +
                                gq[6 + k] * phi[i3];
            g[9 * i + 6 + k] += kGamma2 * tmp + gq[9 + k] * phi[i3 + 1] + gq[9 + 3 + k] * phi[i3 + 2] +
                                gq[9 + 6 + k] * phi[i3];
        }
    }
    __syncwarp();
    return tot;
}

}  // namespace ttm
}  // namespace scp3
