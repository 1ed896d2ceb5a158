// scp3: the SCP3 driver (SCP3.cpp) over libscp3gpu.so.
//
// Same command line as the reference (SCP3.cpp:33-44, 92-151):
//   scp3 [-N p] [-S p] [-r file] [-2 N2] [-3 N3] [-p pes] [-m modes] [-G] [-B block] input.dat
// plus --precision fp64|bf16x3|f16x3, --scramble-seed S (seeded scramble of the
// device Sobol points), --device d, --write-modes file (x0 and the normal modes
// the run samples: the eigenvector signs are the eigensolver's choice, so the
// file is what another program needs to reproduce the run's points).  Reads the input file (load_from_vladimir,
// DiskIO.cpp:72-116), reorders O H H (DiskIO.cpp:142-195), builds the normal
// modes (SCP3.cpp:296-314), and runs the sample loop of SCP3_a (SCP3.cpp:154-272)
// on the GPU: E0_sd.dat every 2^14 samples (SCP3.cpp:234-250), sM_%07d.h5 every
// 2^17 (SCP3.cpp:252-255), omega0.dat at start (SCP3.cpp:300-302).
//
// Without -G the reference's default gradient estimator runs
// (ScaledMatrixElements.cpp:102-725): on the GPU with the potential and its
// gradient in FP64, its products in FP64 (--precision fp64) or BF16x3 on the
// tensor cores (--precision bf16x3); f16x3 needs -G (ScaledMatrixElements.cpp:951-971).
#include <getopt.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/scp3gpu.h"

using namespace std;

namespace {

const double kBohr = 0.52917721092, kAutocm = 2.194746313e5;   // Constants.cpp:12-13
const double kHmass = 1837.15137, kDmass = 2.0 * kHmass, kCmass = 21891.6543;
const double kOmass = kCmass * 15.9994 / 12.0107;

struct Options {
    int64_t nsobol = 1 << 20;
    int64_t skip = 1 << 30;
    string rng_file, input, pes = "qtip4pf", precision = "fp64", modes_file;
    int n2 = 0, n3 = 0, block = 1024, device = 0;
    bool use_gradient = true, scramble = false;
    uint64_t scramble_seed = 0;
    vector<int> modes;
};

[[noreturn]] void die(const string& m)
{
    cerr << m << "\n";
    exit(EXIT_FAILURE);
}

vector<int> parse_modes(const string& desc)    // SCP3.cpp:63-89
{
    vector<int> out;
    istringstream iss(desc);
    while (iss.good()) {
        if (iss.peek() == ',') iss.get();
        int a, b;
        if (!(iss >> a)) break;
        b = a;
        if (iss.peek() == '-') {
            iss.get();
            iss >> b;
        }
        for (; a <= b; a++) out.push_back(a);
    }
    return out;
}

Options parse(int argc, char** argv)
{
    static struct option opts[] = {{"NSobol", required_argument, nullptr, 'N'},
                                   {"skip", required_argument, nullptr, 'S'},
                                   {"rng-file", required_argument, nullptr, 'r'},
                                   {"doubles", required_argument, nullptr, '2'},
                                   {"triples", required_argument, nullptr, '3'},
                                   {"PES", required_argument, nullptr, 'p'},
                                   {"select-modes", required_argument, nullptr, 'm'},
                                   {"no-gradient", no_argument, nullptr, 'G'},
                                   {"block-width", required_argument, nullptr, 'B'},
                                   {"precision", required_argument, nullptr, 1000},
                                   {"scramble-seed", required_argument, nullptr, 1001},
                                   {"device", required_argument, nullptr, 1002},
                                   {"write-modes", required_argument, nullptr, 1003},
                                   {nullptr, 0, nullptr, 0}};
    Options o;
    int ch;
    while ((ch = getopt_long(argc, argv, "S:N:2:3:r:p:m:GB:", opts, nullptr)) != -1) {
        switch (ch) {
            case 'N': {
                const int p2 = atoi(optarg);
                if (p2 > 40) die("-N <N>: <N>is too large, NSobol = 2^<N>");
                o.nsobol = int64_t(1) << p2;
                break;
            }
            case 'S': {
                const int p2 = atoi(optarg);
                if (p2 > 60) die("-S <N>: <N>is too large, sobol_skip = 2^<N>");
                o.skip = int64_t(1) << p2;
                break;
            }
            case '2': o.n2 = atoi(optarg); break;
            case '3': o.n3 = atoi(optarg); break;
            case 'r': o.rng_file = optarg; break;
            case 'p': o.pes = optarg; break;
            case 'm': o.modes = parse_modes(optarg); break;
            case 'G': o.use_gradient = false; break;
            case 'B': o.block = atoi(optarg); break;
            case 1000: o.precision = optarg; break;
            case 1001:
                o.scramble = true;
                o.scramble_seed = strtoull(optarg, nullptr, 0);
                break;
            case 1002: o.device = atoi(optarg); break;
            case 1003: o.modes_file = optarg; break;
            default: die("Unknown option: " + to_string(ch));
        }
    }
    if (argc - optind < 1) die("No input file supplied");
    o.input = argv[optind];
    if (o.block <= 0) die("-B must be positive");
    return o;
}

double nuclear_mass(const string& s)   // DiskIO.cpp:22-40
{
    if (s == "H") return kHmass;
    if (s == "D") return kDmass;
    if (s == "C") return kCmass;
    if (s == "O") return kOmass;
    die("Unknown species " + s);
}

// load_from_vladimir (DiskIO.cpp:72-116): x0 in bohr, H upper triangle by columns.
void load_input(const string& name, vector<double>& mass, vector<double>& x0, vector<double>& H)
{
    ifstream fin(name);
    if (!fin.good()) die("File not found: " + name);
    int N;
    fin >> N;
    string skip;
    getline(fin, skip);
    getline(fin, skip);
    mass.assign(3 * N, 0.0);
    x0.assign(3 * N, 0.0);
    for (int i = 0; i < N; i++) {
        string sp;
        fin >> sp;
        for (int k = 0; k < 3; k++) mass[3 * i + k] = nuclear_mass(sp);
        fin >> x0[3 * i] >> x0[3 * i + 1] >> x0[3 * i + 2];
    }
    for (double& v : x0) v /= kBohr;
    const int n = 3 * N;
    H.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = 0; j <= i; j++) {
            double v;
            if (!(fin >> v)) die("Hessian in " + name + " is truncated");
            H[(size_t)i * n + j] = H[(size_t)j * n + i] = v;
        }
}

// OHHOHH (DiskIO.cpp:142-195)
void ohhohh(vector<double>& mass, vector<double>& x0, vector<double>& H)
{
    const int n = (int)mass.size();
    vector<int> p(n);
    int iO = 0, iH = 3;
    for (int i = 0; i < n; i += 3) {
        if (mass[i] == kOmass) {
            for (int j = 0; j < 3; j++) p[iO + j] = i + j;
            iO += 9;
        } else if (mass[i] == kHmass || mass[i] == kDmass) {
            for (int j = 0; j < 3; j++) p[iH + j] = i + j;
            iH += 3;
            iH += 3 * (iH % 9 == 0);
        } else {
            die("Uknown mass at i = " + to_string(i));
        }
    }
    vector<double> m2(n), x2(n), H2((size_t)n * n);
    for (int i = 0; i < n; i++) {
        m2[i] = mass[p[i]];
        x2[i] = x0[p[i]];
        for (int j = 0; j < n; j++) H2[(size_t)i * n + j] = H[(size_t)p[i] * n + p[j]];
    }
    mass.swap(m2), x0.swap(x2), H.swap(H2);
}

// Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major A,
// destroyed): ascending eigenvalues w, eigenvectors as the columns of V
// (column-major n x n).  Stands in for armadillo's eig_sym (SCP3.cpp:298).
void eig_sym(int n, vector<double> A, vector<double>& w, vector<double>& V)
{
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
    auto a = [&](int i, int j) -> double& { return A[(size_t)i * n + j]; };
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) (i == j ? tot : off) += a(i, j) * a(i, j);
        if (off <= 1e-30 * (tot + off)) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                if (a(p, q) == 0.0) continue;
                const double theta = (a(q, q) - a(p, p)) / (2 * a(p, q));
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                const double c = 1 / sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; k++) {   // columns p, q
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {   // rows p, q
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    const double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
                    V[(size_t)p * n + k] = c * vkp - s * vkq;
                    V[(size_t)q * n + k] = s * vkp + c * vkq;
                }
            }
    }
    vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
    w.resize(n);
    vector<double> V2((size_t)n * n);
    for (int k = 0; k < n; k++) {
        w[k] = a(order[k], order[k]);
        for (int i = 0; i < n; i++) V2[(size_t)k * n + i] = V[(size_t)order[k] * n + i];
    }
    V.swap(V2);
}

void check(int rc, const char* what)
{
    if (rc != SCP3GPU_OK) die(string(what) + ": " + scp3gpu_last_error());
}

}  // namespace

int main(int argc, char** argv)
{
    Options o = parse(argc, argv);
    if (o.use_gradient && o.precision == "f16x3")
        die("The gradient estimator runs its products in FP64 or BF16x3; run f16x3 with -G.");
    vector<double> mass, x0, H;
    load_input(o.input, mass, x0, H);
    ohhohh(mass, x0, H);
    const int n = (int)x0.size(), N = n / 3, nm0 = n - 6;
    vector<double> w2, U;
    eig_sym(n, H, w2, U);
    {
        ofstream sout("omega0.dat");                    // SCP3.cpp:300-302
        for (double v : w2) sout << sqrt(fabs(v)) * kAutocm << "\n";
    }
    if (o.n2 == 0) o.n2 = 3 * N - 6;                   // SCP3.cpp:305
    vector<double> omega(nm0), MUa((size_t)n * nm0);
    for (int k = 0; k < nm0; k++) {
        omega[k] = sqrt(w2[6 + k]);
        const double alpha = sqrt(omega[k]);
        for (int i = 0; i < n; i++) MUa[(size_t)k * n + i] = U[(size_t)(6 + k) * n + i] / (sqrt(mass[i]) * alpha);
    }
    if (!o.modes_file.empty()) {
        // line 1: x0 (bohr, O H H order); line 2 + k: omega_k, then column k of MUa
        FILE* f = fopen(o.modes_file.c_str(), "w");
        if (!f) die("cannot write " + o.modes_file);
        for (int i = 0; i < n; i++) fprintf(f, "%.17g%c", x0[i], i + 1 < n ? ' ' : '\n');
        for (int k = 0; k < nm0; k++) {
            fprintf(f, "%.17g", omega[k]);
            for (int i = 0; i < n; i++) fprintf(f, " %.17g", MUa[(size_t)k * n + i]);
            fprintf(f, "\n");
        }
        fclose(f);
    }
    if (o.modes.empty())
        for (int k = 0; k < nm0; k++) o.modes.push_back(k);
    if (o.n2 > (int)o.modes.size() || o.n3 > (int)o.modes.size())
        die("Number of double or triple excitations exceed number of modes.");

    scp3gpu_config c = {};
    c.nw = n / 9;
    c.nmodes0 = nm0;
    c.x0 = x0.data();
    c.MUa = MUa.data();
    c.omega = omega.data();
    c.nmodes = (int)o.modes.size();
    c.modes = o.modes.data();
    c.n2 = o.n2;
    c.n3 = o.n3;
    if (o.pes == "qtip4pf") c.pes = SCP3GPU_PES_QTIP4PF;
    else if (o.pes == "ttm3f") c.pes = SCP3GPU_PES_TTM3F;
    else die("Unknown H2O potential: " + o.pes);
    if (o.precision == "fp64") c.precision = SCP3GPU_PREC_FP64;
    else if (o.precision == "bf16x3") c.precision = SCP3GPU_PREC_BF16X3;
    else if (o.precision == "f16x3") c.precision = SCP3GPU_PREC_F16X3;
    else die("Unknown precision " + o.precision);
    c.scramble = o.scramble ? SCP3GPU_SOBOL_SCRAMBLED : SCP3GPU_SOBOL_REFERENCE;
    c.scramble_seed = o.scramble_seed;
    c.device = o.device;
    c.estimator = o.use_gradient ? SCP3GPU_ESTIMATOR_GRADIENT : SCP3GPU_ESTIMATOR_DIRECT;
    scp3gpu_hbuild* h = nullptr;
    check(scp3gpu_hbuild_create(&c, &h), "create");
    const int64_t nb = scp3gpu_hbuild_basis_size(h);
    const int64_t n1 = scp3gpu_sub_basis_size(c.nmodes, c.n2, c.n3, 1);
    const int64_t n2s = scp3gpu_sub_basis_size(c.nmodes, c.n2, c.n3, 2);

    ifstream rng_in;
    if (!o.rng_file.empty()) {
        rng_in.open(o.rng_file);
        if (!rng_in.good()) die("cannot open " + o.rng_file);
    }
    ofstream e0("E0_sd.dat");
    e0.setf(ios::fixed);
    e0.precision(10);
    vector<double> by;
    vector<double> Mout;
    int64_t sobol_index = o.skip;
    for (int64_t i = 0; i < o.nsobol; i += o.block) {
        if (rng_in.is_open()) {                        // SCP3.cpp:188-194
            by.resize((size_t)o.block * nm0);
            for (double& v : by)
                if (!(rng_in >> v)) die("-r file ended before " + to_string(o.nsobol) + " samples");
            check(scp3gpu_hbuild_accumulate_normals(h, by.data(), o.block), "accumulate_normals");
        } else {
            check(scp3gpu_hbuild_accumulate(h, sobol_index, o.block), "accumulate");
            sobol_index += o.block;
        }
        if ((i + o.block) % (1 << 14) == 0) {          // SCP3.cpp:234-250
            double E0[2];
            check(scp3gpu_hbuild_eigvals(h, n1, 1, &E0[0]), "eigvals singles");
            check(scp3gpu_hbuild_eigvals(h, n2s, 1, &E0[1]), "eigvals doubles");
            e0 << i + o.block << " " << E0[0] * kAutocm << " " << E0[1] * kAutocm << " "
               << (E0[1] - E0[0]) * kAutocm << endl;
            if ((i + o.block) % (1 << 17) == 0) {      // SCP3.cpp:252-255
                Mout.resize((size_t)nb * nb);
                check(scp3gpu_hbuild_read(h, Mout.data(), nb, 1), "read");
                // The reference's M holds the upper triangle only (dsyr2k 'U' into a zero
                // matrix, ScaledMatrixElements.cpp:970; the gradient path fills upper
                // elements, :709-725), so its sM files hold zeros below the diagonal.
                for (int64_t j = 0; j < nb; j++)
                    for (int64_t r = j + 1; r < nb; r++) Mout[(size_t)j * nb + r] = 0.0;
                char s[128];
                snprintf(s, sizeof s, "sM_%07lld.h5", (long long)(i + o.block));
                check(scp3gpu_save_h5(s, Mout.data(), nb, nb), "save_h5");
            }
        }
    }
    int64_t nonfinite = 0, notconv = 0;
    const int rc = scp3gpu_hbuild_status(h, &nonfinite, &notconv);
    if (rc != SCP3GPU_OK)
        cerr << "warning: " << nonfinite << " non-finite samples, " << notconv << " unconverged TTM3-F samples\n";
    scp3gpu_hbuild_destroy(h);
    return 0;
}
