// TEST INFRASTRUCTURE ONLY (the oracle / CPU baseline): never linked into the product.
//
// The reference's Hamiltonian build on the CPU, the -G (no-gradient) path of
// SCP3_a (SCP3.cpp:154-272), with the parts that need armadillo restated in
// plain C++ and everything else taken from the reference's own sources:
//
//   per sample   sobol::std_normal (reference source) or caller-given normals
//                (the -r path, SCP3.cpp:188-194); q = y / sqrt(2) (SCP3.cpp:201);
//                r = bohr*(x0 + MUa q) (SCP3.cpp:208); V = pot(nw, r)/autokcalpmol
//                (SCP3.cpp:219, reference PES source); V_anh = V - q.(omega%q)/2
//                (SCP3.cpp:222-223)
//   per block    get_bra (restated from ScaledMatrixElements.cpp:870-930),
//                ket = bra*V (ScaledMatrixElements.cpp:964-967), dsyr2k('U','N',
//                0.5, bra, ket, 1, M) (ScaledMatrixElements.cpp:942-949, 970) from
//                the BLAS that scipy bundles, with OpenMP as in the reference.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <string>
#include <vector>
using namespace std;

#include "qtip4pf.h"
#include "ttm3f.h"
#include "sobol.hpp"
#include "HarmonicOscillatorBasis.h"

extern "C" void scipy_dsyr2k_(const char* uplo, const char* trans, const int* n, const int* k,
                              const double* alpha, const double* a, const int* lda,
                              const double* b, const int* ldb, const double* beta,
                              double* c, const int* ldc);

namespace {

const double kBohr = 0.52917721092;                 // Constants.cpp:12
const double kAuToKcalPerMol = 627.509474277194;    // Constants.h:21

size_t basis_size(int nm, int n2, int n3)           // ScaledMatrixElements.cpp:73-78
{
    size_t s2 = 1 + nm + (size_t)n2 * (n2 + 1) / 2;
    return s2 + (size_t)n3 * (1 + n3) * (2 + n3) / 6;
}

// Restatement of ScaledMatrixElements::get_bra (ScaledMatrixElements.cpp:870-930).
void get_bra(int nm, int n2, int n3, const double* q, double* bra)
{
    size_t R = 0;
    bra[R++] = 1.0;
    for (int m = 0; m < nm; m++) bra[R++] = ho_basis[1](q[m]);
    for (int m = 0; m < n2; m++) bra[R++] = ho_basis[2](q[m]);
    for (int m = 0; m < n2; m++) {
        double bm = ho_basis[1](q[m]);
        for (int n = m + 1; n < n2; n++) bra[R++] = bm * ho_basis[1](q[n]);
    }
    for (int m = 0; m < n3; m++) bra[R++] = ho_basis[3](q[m]);
    for (int m = 0; m < n3; m++) {
        double bm = ho_basis[1](q[m]);
        double bm2 = ho_basis[2](q[m]);
        for (int n = m + 1; n < n3; n++) {
            bra[R++] = bm2 * ho_basis[1](q[n]);
            bra[R++] = bm * ho_basis[2](q[n]);
        }
    }
    for (int m = 0; m < n3; m++) {
        double bm = ho_basis[1](q[m]);
        for (int n = m + 1; n < n3; n++) {
            double bmn = bm * ho_basis[1](q[n]);
            for (int p = n + 1; p < n3; p++) bra[R++] = bmn * ho_basis[1](q[p]);
        }
    }
}

}  // namespace

extern "C" {

size_t ref_basis_size(int nm, int n2, int n3) { return basis_size(nm, n2, n3); }

void ref_get_bra(int nm, int n2, int n3, const double* q, double* bra) { get_bra(nm, n2, n3, q, bra); }

// Runs `nsamples` (a multiple of `block`) samples of the -G sample loop and
// accumulates into the upper triangle of the column-major Nb x Nb matrix M
// (M is not divided by the sample count, exactly as in SCP3_a before its
// periodic readout).  pes_id: 0 = qTIP4P/f, 1 = TTM3-F.  If `normals` is not
// NULL it holds nsamples x nm0 standard normals, sample-major (the -r text file
// order, SCP3.cpp:189-193); otherwise the reference's Sobol stream continues
// from *seed.  timings[0..2] receive seconds spent in sampling+PES, in
// get_bra+ket and in dsyr2k.  Returns 0, or -1 on bad arguments.
int ref_hbuild(int pes_id, int nw, const double* x0, const double* MUa, const double* omega,
               int nm0, const int* modes, int nm, int n2, int n3, long long* seed,
               const double* normals, long long nsamples, int block, double* M, double* timings)
{
    if (nw <= 0 || nm0 != 9 * nw - 6 || nm <= 0 || nm > nm0 || n2 > nm || n3 > nm || block <= 0 ||
        nsamples % block != 0)
        return -1;
    h2o::PES* pot = nullptr;
    h2o::qtip4pf qt;
    h2o::ttm3f tt;
    if (pes_id == 0) pot = &qt;
    else if (pes_id == 1) pot = &tt;
    else return -1;

    const int N3 = 9 * nw;
    const size_t nb = basis_size(nm, n2, n3);
    vector<double> by((size_t)nm0 * block), bV(block), r(N3), qsel(nm);
    vector<double> bra(nb * block), ket(nb * block);
    double t_pes = 0, t_bra = 0, t_syr = 0;

    for (long long i = 0; i < nsamples; i += block) {
        auto t0 = chrono::steady_clock::now();
        for (int j = 0; j < block; j++) {
            double* col = &by[(size_t)nm0 * j];
            if (normals) memcpy(col, normals + (size_t)(i + j) * nm0, sizeof(double) * nm0);
            else sobol::std_normal(nm0, seed, col);
        }
        for (size_t k = 0; k < by.size(); k++) by[k] /= sqrt(2.0);
        for (int j = 0; j < block; j++) {
            const double* q = &by[(size_t)nm0 * j];
            for (int a = 0; a < N3; a++) {
                double s = 0.0;
                for (int k = 0; k < nm0; k++) s += MUa[(size_t)k * N3 + a] * q[k];
                r[a] = kBohr * (x0[a] + s);
            }
            double V = (*pot)(nw, r.data()) / kAuToKcalPerMol;
            double h = 0.0;
            for (int k = 0; k < nm0; k++) h += q[k] * (omega[k] * q[k]);
            bV[j] = V - 0.5 * h;
        }
        auto t1 = chrono::steady_clock::now();
#pragma omp parallel
        {
            vector<double> qs(nm);
#pragma omp for schedule(static)
            for (int j = 0; j < block; j++) {
                for (int k = 0; k < nm; k++) qs[k] = by[(size_t)nm0 * j + modes[k]];
                get_bra(nm, n2, n3, qs.data(), &bra[nb * j]);
            }
#pragma omp for schedule(static)
            for (int j = 0; j < block; j++)
                for (size_t k = 0; k < nb; k++) ket[nb * j + k] = bra[nb * j + k] * bV[j];
        }
        auto t2 = chrono::steady_clock::now();
        const char U = 'U', Nt = 'N';
        const int n = (int)nb, kk = block;
        const double alpha = 0.5, beta = 1.0;
        scipy_dsyr2k_(&U, &Nt, &n, &kk, &alpha, bra.data(), &n, ket.data(), &n, &beta, M, &n);
        auto t3 = chrono::steady_clock::now();
        t_pes += chrono::duration<double>(t1 - t0).count();
        t_bra += chrono::duration<double>(t2 - t1).count();
        t_syr += chrono::duration<double>(t3 - t2).count();
    }
    if (timings) {
        timings[0] = t_pes;
        timings[1] = t_bra;
        timings[2] = t_syr;
    }
    return 0;
}

}  // extern "C"
