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
#include <cstddef>
#include <string>
using namespace std;

#include "qtip4pf.h"
#include "ttm3f.h"
#include "sobol.hpp"
#include "beasley_springer_moro.h"
#include "HarmonicOscillatorBasis.h"

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

}  // extern "C"
