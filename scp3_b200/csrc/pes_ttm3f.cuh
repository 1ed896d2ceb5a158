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
// ddt (3nw x 3nw), power tables (48 per water)
__host__ __device__ inline size_t scratch_elems(int nw) { return (size_t)18 * nw + (size_t)9 * nw * nw + 48 * nw; }

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

}  // namespace ttm
}  // namespace scp3
