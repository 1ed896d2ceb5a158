// Internal declarations shared by the translation units of libscp3gpu.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/scp3gpu.h"

namespace scp3 {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define SCP3_STR2(x) #x
#define SCP3_STR(x) SCP3_STR2(x)
#define SCP3_CUDA(call)                                                                         \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return ::scp3::cuda_fail(e_, __FILE__ ":" SCP3_STR(__LINE__) " " #call); \
    } while (0)

// ---------------------------------------------------------------- device helpers
template <typename T>
inline int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) return SCP3GPU_OK;
    SCP3_CUDA(cudaMalloc((void**)p, count * sizeof(T)));
    return SCP3GPU_OK;
}

template <typename T>
inline int upload(T** p, const T* host, size_t count)
{
    int rc = dalloc(p, count);
    if (rc) return rc;
    if (count) SCP3_CUDA(cudaMemcpy(*p, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return SCP3GPU_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

inline int check_device(int dev)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(SCP3GPU_ERR_UNSUPPORTED, "no CUDA device");
    if (dev < 0 || dev >= n) return fail(SCP3GPU_ERR_ARG, "device ordinal out of range");
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return fail(SCP3GPU_ERR_UNSUPPORTED, "libscp3gpu is built for sm_100a (B200) only");
    return SCP3GPU_OK;
}


constexpr int kLogMax = 62;           // bits of the Sobol state (sobol.cpp:27700)
constexpr int kMaxModes = 255;        // modes fit the 8-bit fields of a basis descriptor
constexpr int kMaxWaters = 16;        // per-sample kernels keep one geometry per warp in smem
constexpr int kTtmMaxIter = 500;      // ttm3f.cpp:31
constexpr double kBohr = 0.52917721092;              // Constants.cpp:12
constexpr double kAuToKcalPerMol = 627.509474277194; // Constants.h:21

// ---------------------------------------------------------------- host tables
// Sobol direction numbers, [bit][dim] layout (bit-major, dims contiguous), each
// scaled by 2^(61-bit) as i8_sobol does (sobol.cpp:27684-27752).  With a
// scramble seed, every direction number is pushed through the dimension's
// linear scramble matrix (scrambling commutes with the Gray-code XOR) and the
// digital shifts are returned separately.
int sobol_tables(int dims, int scramble, uint64_t seed, std::vector<int64_t>& v_bit_major,
                 std::vector<uint64_t>& shift);

// Basis descriptors in getBasisSize order (ScaledMatrixElements.cpp:870-930):
// kind in bits 0..2, modes m, n, p in bits 3..10, 11..18, 19..26.
enum BasisKind : uint32_t {
    kGround = 0, kHo1 = 1, kHo2 = 2, kHo1Ho1 = 3, kHo3 = 4, kHo2Ho1 = 5, kHo1Ho2 = 6, kHo1Ho1Ho1 = 7
};
std::vector<uint32_t> basis_descriptors(int nm, int n2, int n3);

// The same basis as products of entries of a per-sample Hermite table
// [1, h1(q_m), h2(q_m), h3(q_m)] (indices a, b, c in 10-bit fields).
std::vector<double> ho_diagonal(const std::vector<double>& omega_sel, int n2, int n3);
std::vector<uint32_t> basis_factor_table(int nm, int n2, int n3);

// Pair tasks of the water potentials, in one list per cluster size: type in
// bits 0..1 (0: M-site(i)/H(j), 1: H/H, 2: O/O, 3: M/M) and the two atom or
// site indices in bits 2..16 and 17..31 (atoms index 3*water+{0,1,2}; M sites
// index the water).
std::vector<uint32_t> pair_tasks(int nw);

// ---------------------------------------------------------------- launches
struct SampleArgs {
    int nw, nm0, nm;              // waters, all modes, selected modes
    const double* x0;             // [9nw] bohr
    const double* MUa;            // [9nw x nm0] column-major
    const double* omega;          // [nm0]
    const int* modes;             // [nm]
    const int64_t* vdir;          // [62 x nm0] bit-major direction numbers
    const uint64_t* shift;        // [nm0] or nullptr
    const uint32_t* tasks;        // pair tasks
    int ntasks;
    const double* normals;        // [n x nm0] sample-major, or nullptr to draw Sobol points
    const float* normals32;       // the same in FP32 (read when normals is nullptr), or nullptr
    int64_t index0;               // first Sobol index
    int64_t n;                    // samples this launch
    int64_t nvalid;               // samples beyond this are padding (q = 0, V = 0)
    double* q64;                  // [n x nm] selected q, FP64 (may be nullptr)
    float* q32;                   // [n x nm] selected q, FP32 (may be nullptr)
    double* v;                    // [n] V_anh (hartree)
    unsigned long long* counters; // [2] non-finite, not converged
    int skip_pes;                 // 1: q only, V_anh = 0 (the surrogate supplies V)
    double* vq;                   // [n x nm] dV_anh/dq of the selected modes, FP64 (gradient path; FP64
                                  // potential), or nullptr
};
// pes: SCP3GPU_PES_*, fp32: run the potential in FP32.
int launch_samples(int pes, bool fp32, const SampleArgs& a, cudaStream_t s);

// All clusters of a batch in one launch: cluster c (grid.y) runs args_dev[c]
// (args_host: a host copy of the same array, for the launch shape), n samples
// each.
int launch_samples_batch(int pes, bool fp32, const SampleArgs* args_host, const SampleArgs* args_dev, int ncl,
                         int64_t n, cudaStream_t s);

// Energies (kcal/mol) and gradients (kcal/mol/A, [n][9nw]) of n geometries, FP64;
// iters (may be null): TTM3-F dipole sweeps per geometry
int launch_pes_energy_grad(int pes, int nw, int64_t n, const double* crd, double* E, double* G, int* iters,
                           const uint32_t* tasks, int ntasks, cudaStream_t s);

int launch_pes_energy(int pes, int nw, int64_t n, const double* crd, double* E, int* iters,
                      const uint32_t* tasks, int ntasks, cudaStream_t s);

int launch_std_normal(int dims, int64_t index0, int64_t n, const int64_t* vdir, const uint64_t* shift,
                      double* out, cudaStream_t s);

// FP64 plain form: Phi[i][s] and W[i][s] = V_s Phi[i][s], rows i < nb_pad, K = ldk.
int launch_expand_fp64(const uint32_t* desc, int nb, int nb_pad, int nm, const double* q, const double* v,
                       int64_t n, int64_t ldk, double* phi, double* w, cudaStream_t s);

// Gradient (Stein) estimator, FP64, as products of reduced basis functions
// (stein.cu).  Virtual rows (m, i): basis function i that excites mode m, ordered
// by m then i, plus one last row for <0|V|0>.
struct SteinPlan {
    int nb = 0, nb_pad = 0, nm = 0;
    int nv = 0, nv_pad = 0;          // virtual rows (with the ground row), padded to 128
    int rt = 0, ct = 0;              // 128-row tiles of the virtual rows and of the basis
    int nsplit = 1;                  // sample ranges of the products (C)
    int dsplit = 1;                  // sample ranges of the same-mode pair sums (D), a multiple of nsplit
    int64_t chunk = 0;               // samples per pass
    int64_t dsize = 0;               // doubles of the same-mode pair sums per split
    int ndtasks = 0;
    uint32_t* vrdesc = nullptr;      // [nv] mode, level, the other factors of the row's function
    int* rank3 = nullptr;            // [nb * 3] rank of function i in E_m for its k-th mode
    int* voff = nullptr;             // [nm + 1] first virtual row of mode m
    int64_t* doff = nullptr;         // [nm] first same-mode pair sum of mode m
    int4* dtasks = nullptr;          // [ndtasks] (m, row tile, column tile) of the tiled pair kernel
    int nftasks = 0;
    int* ftasks = nullptr;           // [nftasks] modes of the triangle-blocked pair kernel
    double* W = nullptr;             // [chunk][nv_pad]  reduced function x Stein weight
    double* Phi = nullptr;           // [chunk][nb_pad]  basis functions
    double* C = nullptr;             // [nsplit][rt * ct][128 * 128]
    double* D = nullptr;             // [dsplit][dsize]
    // Split form (BF16x3 products on the tensor cores): W and Phi as one operand of
    // 32-slot boxes, W rows [0, nv_pad), Phi rows from nv_pad; C is then the
    // 128 x 256 tiles' unit partials P.
    bool split = false;
    int bpairs = 0;                  // Phi panel pairs (the last a one-panel tile when ct is odd)
    int ntiles2 = 0;                 // tiles (W panel, Phi pair): rt * bpairs
    int64_t slots = 0;               // K slots of a whole pass (4160 per 4096 samples)
    uint16_t* xop = nullptr;         // [row block][k-block][hi, lo][128 x 32]
    uint32_t* xdesc = nullptr;       // [rows] the expansion's table indices of each row
    // Same-mode pair sums on the tensor cores too (when every function without
    // one of its factors is again a basis function): rows W_b(m, i) =
    // R_i^m K^m_{a_i b} from row nv_pad, one block of e_m rows per (mode m, level
    // b present in m), against the Phi columns of the reduced functions.
    bool tcpairs = false;
    int nwb_pad = 0;                 // W_b rows, padded to 128; Phi rows start at nv_pad + nwb_pad
    int trows = 0;                   // rows of the expansion's table (1, h_l(q_m), K^m_a0, V, K^m_ab)
    uint32_t* tspec = nullptr;       // [trows] kind | a << 4 | b << 6 | mode << 8 of each table row
    int* tile_of = nullptr;          // [row panels][bpairs] tile of (W panel, Phi pair), -1 = none
    int* red3 = nullptr;             // [nb * 3] function i without its k-th factor (basis index)
    int* wb_off = nullptr;           // [nm * 4] first operand row of block (m, b), -1 = none
    // Blocks (m, b) whose functions all reduce to the constant (red = the ground
    // function: for the doubles basis, level 2 = h2(q_m) alone) need only sum_s of
    // each row: they are summed in the expansion instead of multiplied.
    int nsum = 0;                    // rows summed
    int* sum_off = nullptr;          // [nm * 4] first summed row of block (m, b), -1 = none
    float* spart = nullptr;          // [chunk / 4096 * 130][nsum] per-32-slot-block sums of a pass
    double* sums = nullptr;          // [nsum] sum over the samples so far
    int4* tiles2 = nullptr;          // (W row, Phi row, 0, second Phi row)
    int* nosign = nullptr;           // [chunk / 4096] first negative 16-group: never
    double* P = nullptr;             // [nsplit][ntiles2][128 x 256] tile-local column-major
    int* err = nullptr;              // a bounded wait of the contraction expired
};
// split: BF16x3 products (tcgen05) instead of FP64 ones.
int stein_create(SteinPlan& p, const std::vector<uint32_t>& desc, int nm, int64_t chunk, int sms,
                 bool split = false);
// Samples of a pass holding nvalid samples (padding samples carry V = 0 and dV/dq = 0).
int64_t stein_pass_samples(const SteinPlan& p, int64_t nvalid);
void stein_destroy(SteinPlan& p);
int stein_zero(const SteinPlan& p, cudaStream_t s);
// One pass of k samples (k = stein_pass_samples(); q, vq: [k][nm], v: [k]).
int stein_pass(const SteinPlan& p, const uint32_t* desc, const double* q, const double* v, const double* vq,
               int64_t k, cudaStream_t s);
// The dense column-major nb x nb estimate (both triangles), divided by `divisor`;
// with `diag` the diagonal becomes (v + diag[i]) + zpe, as launch_unpack.
int stein_unpack(const SteinPlan& p, const uint32_t* desc, double divisor, const double* diag, double zpe,
                 double* M, int64_t ld, cudaStream_t s);

struct TileMap {
    int tile;          // tile edge (64 FP64, 128 tensor-core)
    int nt;            // tiles per side
    int ntiles;        // upper tiles nt(nt+1)/2
};
// P[split][tile][tile*tile] += sum over this split's sample range of Phi_i W_j.
int launch_contract_fp64(const double* phi, const double* w, int64_t ldk, int64_t k, int nb_pad,
                         const TileMap& tm, int nsplit, double* partial, cudaStream_t s);

// The plain build's form: Phi and W sample-major ([k][ld], ld = tm.nt * 128),
// P[split][tile][128*128] += sum over this split's sample range of Phi_i W_j.
int launch_expand_fp64_sm(const uint32_t* desc, int nb, int nm, const double* q, const double* v, int64_t n,
                          int64_t ld, double* phi, double* w, cudaStream_t s);
int launch_contract_fp64_t128(const double* phi, const double* w, int64_t ld, int64_t k, const TileMap& tm,
                              int nsplit, double* partial, cudaStream_t s);

// P[split][ti * ct + tj][128*128] += sum over this split's sample range of
// A[k][ti*128 + r] B[k][tj*128 + c] (sample-major operands, every tile of the
// rt x ct rectangle).
int launch_gemm_fp64_rect(const double* A, int64_t lda, const double* B, int64_t ldb, int64_t k, int rt, int ct,
                          int nsplit, double* partial, cudaStream_t s);

// Sum the splits of P into a dense column-major nb x nb matrix (upper triangle
// mirrored to the lower), divided by `divisor`; with `diag` (length nb) the
// diagonal becomes (v + diag[i]) + zpe, the order of SCP3.cpp:237-239.
int launch_unpack(const double* partial, const TileMap& tm, int nsplit, int nb, double divisor, const double* diag,
                  double zpe, double* M, int64_t ld, cudaStream_t s);

// Upload the TTM3-F constants (combined monomer coefficients, damping widths)
// to the current device once.
int ttm_init_device();

// SCP1 per-sample stage (SCP1.cpp:52-63): for points index0 + s, s < n, of the
// unscrambled Sobol sequence in dim = 9 nw dimensions, y = std_normal % sqrt(d),
// dq = isqrtM_U y, V = pes(bohr (q + dq)) / autokcal, G = dV/dr bohr / autokcal;
// writes V[n], G[n][dim], D[n][dim] = dq (and the TTM3-F sweep counts).
struct Scp1Args {
    int nw, dim;
    const double* q;          // [dim] bohr
    const double* sqd;        // [dim] sqrt(d)
    const double* U;          // [dim x dim] isqrtM_U, column-major
    const int64_t* vdir;      // [62][dim]
    int64_t index0, n;
    const uint32_t* tasks;
    int ntasks;
    double* V;
    double* G;
    double* D;
    int* iters;               // may be null
};
int launch_scp1_samples(int pes, const Scp1Args& a, cudaStream_t s);

}  // namespace scp3
