// Host-side tables of the build: Sobol direction numbers (+ scramble), basis
// descriptors and pair tasks of the water potentials.
#include <cstring>

#include "internal.h"
#include "sobol_dirnum.h"

namespace scp3 {

namespace {

// Bratley-Fox recurrence of i8_sobol (sobol.cpp:27700-27752): row i of the
// direction numbers from the primitive polynomial poly[i] of degree m and the
// m initial numbers, then column j scaled by 2^(61-j).
void dirnums(int dims, std::vector<int64_t>& v /* dims x 62 */)
{
    v.assign((size_t)dims * kLogMax, 0);
    for (int j = 0; j < kLogMax; j++) v[j] = 1;
    for (int i = 1; i < dims; i++) {
        const unsigned poly = scp3_sobol_poly[i];
        const int m = 31 - __builtin_clz(poly);
        int64_t* row = &v[(size_t)i * kLogMax];
        for (int j = 0; j < m; j++) row[j] = scp3_sobol_vinit[i][j];
        for (int j = m; j < kLogMax; j++) {
            int64_t nv = row[j - m];
            for (int k = 0; k < m; k++)
                if ((poly >> (m - 1 - k)) & 1u) nv ^= (int64_t(2) << k) * row[j - k - 1];
            row[j] = nv;
        }
    }
    for (int j = 0; j < kLogMax - 1; j++) {
        const int64_t scale = int64_t(1) << (kLogMax - 1 - j);
        for (int i = 0; i < dims; i++) v[(size_t)i * kLogMax + j] *= scale;
    }
}

uint64_t splitmix64(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

// The scramble of dimension d: output digit p (bit p of the 62-bit state) is the
// parity of (state & mask_p), mask_p = bit p plus seeded bits above p; then XOR
// a seeded 62-bit shift.  Masks and shift come from one splitmix64 stream per
// dimension started at seed ^ (0xD1B54A32D192ED03 * (d+1)).
int sobol_tables(int dims, int scramble, uint64_t seed, std::vector<int64_t>& vbm, std::vector<uint64_t>& shift)
{
    if (dims < 1 || dims > SCP3_SOBOL_MAX_DIMS) return fail(SCP3GPU_ERR_ARG, "sobol: dims must be 1..1111");
    std::vector<int64_t> v;
    dirnums(dims, v);
    shift.assign(dims, 0);
    if (scramble) {
        const uint64_t low62 = (1ull << 62) - 1;
        for (int d = 0; d < dims; d++) {
            uint64_t s = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(d + 1));
            uint64_t mask[kLogMax];
            for (int p = 0; p < kLogMax; p++) mask[p] = (1ull << p) | (splitmix64(s) & low62 & ~((2ull << p) - 1));
            shift[d] = splitmix64(s) & low62;
            for (int b = 0; b < kLogMax; b++) {
                const uint64_t x = (uint64_t)v[(size_t)d * kLogMax + b];
                uint64_t y = 0;
                for (int p = 0; p < kLogMax; p++) y |= (uint64_t)(__builtin_popcountll(x & mask[p]) & 1) << p;
                v[(size_t)d * kLogMax + b] = (int64_t)y;
            }
        }
    }
    vbm.assign((size_t)kLogMax * dims, 0);
    for (int d = 0; d < dims; d++)
        for (int b = 0; b < kLogMax; b++) vbm[(size_t)b * dims + d] = v[(size_t)d * kLogMax + b];
    return SCP3GPU_OK;
}

std::vector<uint32_t> basis_descriptors(int nm, int n2, int n3)
{
    std::vector<uint32_t> d;
    auto put = [&](uint32_t kind, int m, int n, int p) {
        d.push_back(kind | ((uint32_t)m << 3) | ((uint32_t)n << 11) | ((uint32_t)p << 19));
    };
    put(kGround, 0, 0, 0);
    for (int m = 0; m < nm; m++) put(kHo1, m, 0, 0);
    for (int m = 0; m < n2; m++) put(kHo2, m, 0, 0);
    for (int m = 0; m < n2; m++)
        for (int n = m + 1; n < n2; n++) put(kHo1Ho1, m, n, 0);
    for (int m = 0; m < n3; m++) put(kHo3, m, 0, 0);
    for (int m = 0; m < n3; m++)
        for (int n = m + 1; n < n3; n++) {
            put(kHo2Ho1, m, n, 0);
            put(kHo1Ho2, m, n, 0);
        }
    for (int m = 0; m < n3; m++)
        for (int n = m + 1; n < n3; n++)
            for (int p = n + 1; p < n3; p++) put(kHo1Ho1Ho1, m, n, p);
    return d;
}

// Same pair set as the reference's loops (qtip4pf.cpp:213-283, ttm3f.cpp:144-257):
// for every ordered i != j the two H of j against the M site of i, and for i < j
// the four H/H pairs, O/O and M/M.
std::vector<uint32_t> pair_tasks(int nw)
{
    std::vector<uint32_t> t;
    auto put = [&](uint32_t type, int a, int b) { t.push_back(type | ((uint32_t)a << 2) | ((uint32_t)b << 17)); };
    // grouped by type so that the lanes of a warp mostly take the same branch
    for (int i = 0; i < nw; i++)
        for (int j = 0; j < nw; j++)
            if (i != j)
                for (int l = 1; l < 3; l++) put(0, i, 3 * j + l);
    for (int i = 0; i < nw; i++)
        for (int j = i + 1; j < nw; j++)
            for (int a = 1; a < 3; a++)
                for (int b = 1; b < 3; b++) put(1, 3 * i + a, 3 * j + b);
    for (int i = 0; i < nw; i++)
        for (int j = i + 1; j < nw; j++) put(2, 3 * i, 3 * j);
    for (int i = 0; i < nw; i++)
        for (int j = i + 1; j < nw; j++) put(3, i, j);
    return t;
}

// Each basis function as a product of three entries of a per-sample table
// [1, h1(q_0..), h2(q_0..), h3(q_0..)]: entry indices a, b, c in bits 0..9,
// 10..19, 20..29 (0 is the constant 1).
std::vector<uint32_t> basis_factor_table(int nm, int n2, int n3)
{
    std::vector<uint32_t> d;
    auto h1 = [&](int m) { return 1 + m; };
    auto h2 = [&](int m) { return 1 + nm + m; };
    auto h3 = [&](int m) { return 1 + 2 * nm + m; };
    auto put = [&](int a, int b, int c) { d.push_back((uint32_t)a | ((uint32_t)b << 10) | ((uint32_t)c << 20)); };
    put(0, 0, 0);
    for (int m = 0; m < nm; m++) put(h1(m), 0, 0);
    for (int m = 0; m < n2; m++) put(h2(m), 0, 0);
    for (int m = 0; m < n2; m++)
        for (int n = m + 1; n < n2; n++) put(h1(m), h1(n), 0);
    for (int m = 0; m < n3; m++) put(h3(m), 0, 0);
    for (int m = 0; m < n3; m++)
        for (int n = m + 1; n < n3; n++) {
            put(h2(m), h1(n), 0);
            put(h1(m), h2(n), 0);
        }
    for (int m = 0; m < n3; m++)
        for (int n = m + 1; n < n3; n++)
            for (int p = n + 1; p < n3; p++) put(h1(m), h1(n), h1(p));
    return d;
}

// addHODiagonal (ScaledMatrixElements.cpp:735-784): the harmonic energy of
// every basis function, in basis order, from the selected modes' frequencies.
std::vector<double> ho_diagonal(const std::vector<double>& w, int n2, int n3)
{
    const int nm = (int)w.size();
    std::vector<double> d;
    double e0 = 0;
    for (double x : w) e0 += x;
    e0 *= 0.5;
    d.push_back(e0);
    for (int k = 0; k < nm; k++) d.push_back(e0 + w[k]);
    for (int k = 0; k < n2; k++) d.push_back(e0 + 2 * w[k]);
    for (int k = 0; k < n2; k++)
        for (int l = k + 1; l < n2; l++) d.push_back(e0 + w[k] + w[l]);
    for (int k = 0; k < n3; k++) d.push_back(e0 + 3.0 * w[k]);
    for (int k = 0; k < n3; k++)
        for (int l = k + 1; l < n3; l++) {
            d.push_back(e0 + 2.0 * w[k] + w[l]);
            d.push_back(e0 + w[k] + 2.0 * w[l]);
        }
    for (int k = 0; k < n3; k++)
        for (int l = k + 1; l < n3; l++)
            for (int j = l + 1; j < n3; j++) d.push_back(e0 + w[k] + w[l] + w[j]);
    return d;
}

}  // namespace scp3
