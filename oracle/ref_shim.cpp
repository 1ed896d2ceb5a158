// TEST INFRASTRUCTURE ONLY (the oracle): never linked into the product.
//
// extern "C" entry points over the reference's own, unmodified sources, which
// the recipe in oracle/Makefile compiles from the reference tree into
// oracle/_ref/libscp3ref.so.  Used to pin the C restatement (scp3_oracle.c)
// and as the timed CPU baseline.
//
//   qTIP4P/f     h2o::qtip4pf::operator()   qtip4pf.cpp:190-286 (E), 290-435 (E+grad)
//   TTM3-F       h2o::ttm3f::operator()     ttm3f.cpp:92-321 (E), 325-720 (E+grad)
//   Sobol        sobol::i8_sobol            sobol.cpp:14198-27868
//   std_normal   sobol::std_normal          sobol.cpp:28706-28713
//   BSM          beasley_springer_moro      beasley_springer_moro.cpp:14-46
//   Hermite      ho_basis[]                 HarmonicOscillatorBasis.cpp:16-44
//   SCP1 loop    SCP1::average sample loop  SCP1.cpp:49-69 (restated over the above)
#include <cmath>
#include <cstddef>
#include <string>
#include <vector>
using namespace std;

#include "qtip4pf.h"
#include "ttm3f.h"
#include "sobol.hpp"
#include "beasley_springer_moro.h"
#include "HarmonicOscillatorBasis.h"
#include "Constants.h"

static h2o::qtip4pf g_qtip4pf;
static h2o::ttm3f g_ttm3f;

extern "C" {

double ref_qtip4pf_energy(int nw, const double* crd) { return g_qtip4pf(nw, crd); }

double ref_qtip4pf_energy_grad(int nw, const double* crd, double* grad)
{
    return g_qtip4pf(nw, crd, grad);
}

double ref_ttm3f_energy(int nw, const double* crd) { return g_ttm3f(nw, crd); }

double ref_ttm3f_energy_grad(int nw, const double* crd, double* grad)
{
    return g_ttm3f(nw, crd, grad);
}

// One call of i8_sobol: uniforms of point *seed, then *seed advances.
void ref_i8_sobol(int dims, long long* seed, double* quasi) { sobol::i8_sobol(dims, seed, quasi); }

// One call of std_normal: i8_sobol followed by BSM (the per-sample draw of SCP3.cpp:197).
void ref_std_normal(int dims, long long* seed, double* out) { sobol::std_normal(dims, seed, out); }

void ref_bsm(int n, double* u, double* x) { beasley_springer_moro(n, u, x); }

double ref_ho(int n, double y) { return ho_basis[n](y); }

// The sample loop of SCP1::average (SCP1.cpp:49-69) for points i0 <= i < i1,
// written with plain loops over the reference's own std_normal and potential
// (SCP1.cpp itself needs Armadillo and MPI): sums of V, UX and UX dq^T, UX_q
// column-major.  isqrtM_U is column-major dim x dim; dq = isqrtM_U y summed over
// k in order.  Single-threaded (i8_sobol keeps static state), as one MPI rank.
void ref_scp1_average(int pes, int nw, const double* q, const double* d, const double* isqrtM_U,
                      long long skip, long long i0, long long i1, double* Upot, double* UX, double* UX_q)
{
    const int dim = 9 * nw;
    std::vector<double> y(dim), dq(dim), r(dim), g(dim);
    h2o::PES* pot = pes == 0 ? (h2o::PES*)&g_qtip4pf : (h2o::PES*)&g_ttm3f;
    *Upot = 0.0;
    for (int i = 0; i < dim; i++) UX[i] = 0.0;
    for (int i = 0; i < dim * dim; i++) UX_q[i] = 0.0;
    for (long long i = i0; i < i1; i++) {
        long long current_skip = skip + i;
        sobol::std_normal(dim, &current_skip, y.data());
        for (int k = 0; k < dim; k++) y[k] *= std::sqrt(d[k]);
        for (int c = 0; c < dim; c++) {
            double acc = 0.0;
            for (int k = 0; k < dim; k++) acc += isqrtM_U[(size_t)k * dim + c] * y[k];
            dq[c] = acc;
            r[c] = bohr * (q[c] + acc);
        }
        *Upot += (*pot)(nw, r.data(), g.data()) / autokcalpmol;
        for (int c = 0; c < dim; c++) g[c] *= bohr / autokcalpmol;
        for (int c = 0; c < dim; c++) UX[c] += g[c];
        for (int j = 0; j < dim; j++)
            for (int c = 0; c < dim; c++) UX_q[(size_t)j * dim + c] += g[c] * dq[j];
    }
}

}  // extern "C"
