// eigensolver: the reference's eigensolver tool (eigensolver.cpp:87-111) over
// libscp3gpu.so -- read dataset "M" of an sM_*.h5 file, compute its lowest
// n eigenpairs on the GPU, and write eigenpairs<name>.dat in the reference's
// format (15 significant digits; eigenvalues one per line, then one
// eigenvector per line).
//
//   eigensolver <sM_*.h5> <n_eigenpairs> [--device D]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/scp3gpu.h"

int main(int argc, char* argv[])
{
    if (argc < 3) {
        std::cerr << "usage: eigensolver <sM_*.h5> <n_eigenpairs> [--device D]\n";
        return EXIT_FAILURE;
    }
    const std::string fin_name(argv[1]);
    const int k = std::atoi(argv[2]);
    int device = 0;
    for (int i = 3; i + 1 < argc; i++)
        if (!std::strcmp(argv[i], "--device")) device = std::atoi(argv[++i]);
    int64_t nr = 0, nc = 0;
    if (scp3gpu_load_h5(fin_name.c_str(), nullptr, &nr, &nc) != SCP3GPU_OK) {
        std::cerr << scp3gpu_last_error() << "\n";
        return EXIT_FAILURE;
    }
    if (nr != nc) std::cerr << "HDF5 dataset \"M\" has wrong shape. ndims = 2, dims = " << nc << "x" << nr << "\n";
    std::vector<double> M((size_t)nr * nc);
    if (scp3gpu_load_h5(fin_name.c_str(), M.data(), &nr, &nc) != SCP3GPU_OK) {
        std::cerr << scp3gpu_last_error() << "\n";
        return EXIT_FAILURE;
    }
    if (k < 1 || k > nr) {
        std::cerr << "n_eigenpairs must be 1.." << nr << "\n";
        return EXIT_FAILURE;
    }
    std::vector<double> W(k), Z((size_t)nr * k);
    if (scp3gpu_syevr_lowest(M.data(), nr, nr, k, W.data(), Z.data(), nr, device) != SCP3GPU_OK) {
        std::cerr << scp3gpu_last_error() << "\n";
        return EXIT_FAILURE;
    }
    // eigenpairs + fin_name.substr(2, length - 5) + .dat (eigensolver.cpp:97-99)
    const std::string base = fin_name.size() > 5 ? fin_name.substr(2, fin_name.size() - 5) : fin_name;
    const std::string fout_name = "eigenpairs" + base + ".dat";
    std::ofstream fout(fout_name.c_str());
    fout.precision(15);
    fout << "# Lowest " << k << " eigenvalues\n";
    for (int i = 0; i < k; i++) fout << W[i] << "\n";
    fout << "# Corresponding eigenvectors, one per line." << std::endl;
    for (int i = 0; i < k; i++) {
        for (int64_t r = 0; r < nr; r++) fout << (r ? " " : "") << Z[(size_t)i * nr + r];
        fout << "\n";
    }
    return fout.good() ? EXIT_SUCCESS : EXIT_FAILURE;
}
