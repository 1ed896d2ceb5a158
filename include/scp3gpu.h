/*
 * scp3gpu.h -- C ABI of the B200 Hamiltonian build (libscp3gpu.so).
 *
 * Plain C types only: host pointers unless a name says "_dev".  Every function
 * returns an int status (SCP3GPU_OK == 0) and never exits or traps; the last
 * error's text is available from scp3gpu_last_error().  One handle belongs to
 * one host thread; all of a handle's device work is ordered on its own stream.
 *
 * The reference (SCP3) has no plugin API; the hot path sits behind three C++
 * seams, each of which an entry point below replaces (citations are
 * file:line in the reference tree):
 *
 *   h2o::PES::operator()(nw, crd)              PES.h:14-22, qtip4pf.cpp:190-286,
 *                                              ttm3f.cpp:92-321
 *   sobol::std_normal(dims, &seed, u)          sobol.hpp:31, sobol.cpp:28706-28713
 *   ScaledMatrixElements(omega, N2, N3),       ScaledMatrixElements.h:75-96,
 *     getBasisSize, getSubBasisSize,           ScaledMatrixElements.cpp:73-99,
 *     addEpot(q, V, M)  (-G path),             ScaledMatrixElements.cpp:951-971,
 *     addHODiagonal(M)                         ScaledMatrixElements.cpp:735-784
 *
 * and the fused sample loop of SCP3_a (SCP3.cpp:154-272) that drives them.
 */
#ifndef SCP3GPU_H
#define SCP3GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference calls exit(EXIT_FAILURE) instead,
 *      e.g. SCP3.cpp:156-160, ScaledMatrixElements.cpp:202-205) ---- */
#define SCP3GPU_OK 0
#define SCP3GPU_ERR_ARG 1           /* bad shape, option or pointer            */
#define SCP3GPU_ERR_CUDA 2          /* a CUDA runtime/driver call failed       */
#define SCP3GPU_ERR_NOMEM 3         /* device allocation failed                */
#define SCP3GPU_ERR_NOT_CONVERGED 4 /* TTM3-F dipoles hit the iteration cap    */
#define SCP3GPU_ERR_NONFINITE 5     /* a sample produced a non-finite V        */
#define SCP3GPU_ERR_TIMEOUT 6       /* a bounded device-side wait gave up      */
#define SCP3GPU_ERR_UNSUPPORTED 7   /* no sm_100 device / feature missing      */

/* potentials (h2o.h:20-47 knows "qtip4pf"; TTM3-F added, ttm3f.cpp) */
#define SCP3GPU_PES_QTIP4PF 0
#define SCP3GPU_PES_TTM3F 1

/* arithmetic of the build */
#define SCP3GPU_PREC_FP64 0   /* plain: everything FP64 (parity form)                  */
#define SCP3GPU_PREC_BF16X3 1 /* split: potential FP32, contraction BF16x3 on tcgen05,
                                 FP32 accumulation flushed to FP64 every 4096 samples */
#define SCP3GPU_PREC_BF16X3_PES64 2 /* split contraction as above, potential in FP64       */
#define SCP3GPU_PREC_F16X3 3  /* as BF16X3 with FP16 halves (11-bit significands, operand
                                 scaled by 2^6): same tensor rate, ~2^-22 products      */
#define SCP3GPU_PREC_F16X3_PES64 4 /* FP16x3 contraction, potential in FP64             */

/* sampling */
#define SCP3GPU_SOBOL_REFERENCE 0 /* i8_sobol points, unscrambled (sobol.cpp:14198-27868) */
#define SCP3GPU_SOBOL_SCRAMBLED 1 /* seeded linear matrix scramble + digital shift         */

const char* scp3gpu_last_error(void);
int scp3gpu_version(void);

/* ------------------------------------------------------------------ PES
 * Energies of n geometries, each 9*nw doubles in Angstrom, O H H per water;
 * E[k] in kcal/mol.  Replaces h2o::PES::operator()(nw, crd) (PES.h:14-22).
 * Host buffers; `iters` (may be NULL) receives the TTM3-F Jacobi sweep count
 * per geometry (0 for qTIP4P/f).  Returns SCP3GPU_ERR_NOT_CONVERGED if any
 * TTM3-F geometry hit the 500-sweep cap (its energy is still written). */
int scp3gpu_pes_energy(int pes, int nw, int64_t n, const double* crd, double* E, int* iters);

/* Energies and gradients (kcal/mol/Angstrom, n x 9*nw), FP64 -- h2o::PES::operator()(nw,
 * crd, grad) (PES.h:14-22): qtip4pf.cpp:252-397, ttm3f.cpp:325-720.
 * SCP3GPU_ERR_NOT_CONVERGED if a TTM3-F geometry hit the dipole sweep cap. */
int scp3gpu_pes_energy_grad(int pes, int nw, int64_t n, const double* crd, double* E, double* grad);

/* Device-buffer variant (crd_dev, E_dev on `device`), ordered on the legacy
 * default stream of that device. */
int scp3gpu_pes_energy_dev(int pes, int nw, int64_t n, const double* crd_dev, double* E_dev, int device);

/* ------------------------------------------------------------------ sampling
 * n x dims standard normals of points index0 .. index0+n-1, sample-major,
 * into host memory.  SCP3GPU_SOBOL_REFERENCE reproduces the reference's
 * sobol::std_normal stream: call k of std_normal(dims, &seed) with seed
 * starting at S returns row (S + k) - index0 when index0 = S (sobol.hpp:31).
 * Uniform bit patterns are exact; BSM uses the device log (<= 2 ulp). */
int scp3gpu_sobol_std_normal(int dims, int64_t index0, int64_t n, int scramble, uint64_t scramble_seed,
                             double* out);

/* ------------------------------------------------------------------ basis
 * getBasisSize / getSubBasisSize (ScaledMatrixElements.cpp:73-99). */
int64_t scp3gpu_basis_size(int nmodes, int n2, int n3);
int64_t scp3gpu_sub_basis_size(int nmodes, int n2, int n3, int level);

/* ------------------------------------------------------------------ the build
 * One handle = one ScaledMatrixElements + the SCP3_a sample loop around it. */
typedef struct scp3gpu_hbuild scp3gpu_hbuild;

typedef struct scp3gpu_config {
    int nw;                 /* waters; coordinates = 9*nw                              */
    int nmodes0;            /* internal modes 9*nw-6 (rows of `by`, SCP3.cpp:183)      */
    const double* x0;       /* [9*nw] reference geometry, bohr, O H H (SCP3.cpp:292)   */
    const double* MUa;      /* [9*nw x nmodes0] column-major (SCP3.cpp:309-314)        */
    const double* omega;    /* [nmodes0] harmonic frequencies, hartree (SCP3.cpp:307)  */
    int nmodes;             /* selected modes (-m, SCP3.cpp:316-318)                   */
    const int* modes;       /* [nmodes] indices into 0..nmodes0-1                      */
    int n2;                 /* modes with double excitations (-2)                      */
    int n3;                 /* modes with triple excitations (-3)                      */
    int pes;                /* SCP3GPU_PES_*  (-p)                                     */
    int precision;          /* SCP3GPU_PREC_*                                          */
    int scramble;           /* SCP3GPU_SOBOL_*                                         */
    uint64_t scramble_seed;
    int chunk;              /* samples per device pass; multiple of 4096, 0 = auto:
                               2^18 for the split forms (halved while one pass's
                               operand would exceed ~6 GB); 2^16 for the FP64 form
                               (halved while its Phi and W would exceed ~4 GB); for
                               the gradient estimator 2^14 (FP64 products) or 2^16
                               (BF16x3 products), halved while a pass's operands
                               would exceed ~4 GB                                     */
    int device;             /* CUDA device ordinal                                     */
    int estimator;          /* SCP3GPU_ESTIMATOR_*                                     */
} scp3gpu_config;

/* matrix-element estimator (SCP3.cpp:226-231) */
#define SCP3GPU_ESTIMATOR_DIRECT 0   /* -G: sum_s Phi V Phi^T (ScaledMatrixElements.cpp:951-971)         */
#define SCP3GPU_ESTIMATOR_GRADIENT 1 /* the default: Stein estimator from V and dV/dq
                                        (ScaledMatrixElements.cpp:102-725, TripleExcitations.h); its
                                        products in FP64 (SCP3GPU_PREC_FP64) or BF16x3 on tcgen05
                                        (SCP3GPU_PREC_BF16X3, _BF16X3_PES64); the potential and its
                                        gradient (qtip4pf.cpp:252-397, ttm3f.cpp:325-720) in FP64, or
                                        FP32 for qTIP4P/f with SCP3GPU_PREC_BF16X3; FP16 forms are
                                        SCP3GPU_ERR_UNSUPPORTED                                      */

/* Replaces ScaledMatrixElements(omega(modes), N2, N3) + M.zeros (SCP3.cpp:164-169). */
int scp3gpu_hbuild_create(const scp3gpu_config* cfg, scp3gpu_hbuild** out);
int scp3gpu_hbuild_destroy(scp3gpu_hbuild* h);
/* Zero the accumulated sums and the sample count. */
int scp3gpu_hbuild_reset(scp3gpu_hbuild* h);
int64_t scp3gpu_hbuild_basis_size(const scp3gpu_hbuild* h);
/* The cudaStream_t all of the handle's work is ordered on. */
void* scp3gpu_hbuild_stream(const scp3gpu_hbuild* h);

/* Samples index0 .. index0+n-1 of the handle's Sobol stream, generated on the
 * device: Sobol -> BSM -> q = y/sqrt(2) -> r = bohr(x0 + MUa q) -> V/autokcal
 * -> V_anh = V - q.(omega%q)/2 -> M += sum Phi V_anh Phi^T (upper).  The
 * fused form of SCP3.cpp:187-232 with use_gradient = false (-G).  Asynchronous
 * on the handle's stream. */
int scp3gpu_hbuild_accumulate(scp3gpu_hbuild* h, int64_t index0, int64_t n);

/* The -r path (SCP3.cpp:188-194): n x nmodes0 standard normals, sample-major,
 * in host memory (copied in, overlapped with compute).  Blocks until the host
 * buffer may be reused. */
int scp3gpu_hbuild_accumulate_normals(scp3gpu_hbuild* h, const double* normals, int64_t n);
/* As scp3gpu_hbuild_accumulate_normals with the normals in FP32 (half the
 * host-to-device bytes): the build equals scp3gpu_hbuild_accumulate_normals on
 * the same values widened to double.  The split forms compute q in FP32, so
 * for them the FP32 input loses nothing but the normals' own rounding. */
int scp3gpu_hbuild_accumulate_normals_f32(scp3gpu_hbuild* h, const float* normals, int64_t n);

/* addEpot(q, V, M) of the -G path on caller data (ScaledMatrixElements.cpp:951-971):
 * q is n x nmodes (selected modes, sample-major), V is n; both host buffers. */
int scp3gpu_hbuild_add_epot(scp3gpu_hbuild* h, const double* q, const double* V, int64_t n);

/* Samples accumulated so far. */
int64_t scp3gpu_hbuild_sample_count(const scp3gpu_hbuild* h);

/* Synchronise, then write the accumulated matrix into host memory M
 * (column-major, leading dimension ld >= Nb), upper triangle plus the mirrored
 * lower triangle.  mode 0: the raw FP64 sum (M of SCP3_a before dividing);
 * mode 1: Mout = sum/count + HO diagonal + inactive-mode zero-point energy
 * (SCP3.cpp:237-239 with addHODiagonal, ScaledMatrixElements.cpp:735-784). */
int scp3gpu_hbuild_read(scp3gpu_hbuild* h, double* M, int64_t ld, int mode);

/* As scp3gpu_hbuild_read, into device memory M_dev (on the handle's device),
 * ordered on the handle's stream without a host synchronisation. */
int scp3gpu_hbuild_read_dev(scp3gpu_hbuild* h, double* M_dev, int64_t ld, int mode);

/* The k lowest eigenvalues (hartree, ascending) of the leading `nsub` x `nsub`
 * block of Mout (nsub = Nb for the whole basis; getSubBasisSize for the
 * singles/doubles readouts of SCP3.cpp:241-247), FP64 on the device. */
int scp3gpu_hbuild_eigvals(scp3gpu_hbuild* h, int64_t nsub, int k, double* evals);

/* The k lowest eigenvalues (ascending) and, with Z != NULL, their eigenvectors
 * (columns of Z, leading dimension ldz) of the symmetric n x n host matrix A
 * (column-major, leading dimension lda), FP64 on the device -- replaces
 * dsyevr(A, IU = k, &C) of the eigensolver tool (eigensolver.cpp:20-84): the
 * upper triangle is read unless A(0, n-1) == 0, then the lower one. */
int scp3gpu_syevr_lowest(const double* A, int64_t n, int64_t lda, int k, double* W, double* Z, int64_t ldz,
                         int device);

/* addEpot(q, V, Vq, M) of the gradient path (ScaledMatrixElements.cpp:704-719):
 * n samples of the selected modes' q and dV_anh/dq (n x nmodes, sample-major)
 * and V_anh into the sums of a SCP3GPU_ESTIMATOR_GRADIENT handle. */
int scp3gpu_hbuild_add_epot_grad(scp3gpu_hbuild* h, const double* q, const double* V, const double* Vq, int64_t n);

/* Per-sample status counters since create/reset: samples with a non-finite
 * V, TTM3-F samples that hit the sweep cap. */
int scp3gpu_hbuild_status(scp3gpu_hbuild* h, int64_t* nonfinite, int64_t* not_converged);

/* ------------------------------------------------------------------ batch
 * Several clusters of uneven size and basis built together (no counterpart in
 * the reference, which builds one cluster per SCP3 run, SCP3.cpp:154-272).
 * Every cluster has its own config (geometry, modes, N2/N3, Sobol seed); all
 * share one potential, one split precision (FP64 is rejected with
 * SCP3GPU_ERR_UNSUPPORTED) and one device.  Each pass runs one launch per
 * stage for all clusters; an accumulate call is one CUDA graph replay.  At
 * creation the contraction's work shape is chosen by timing (unless
 * SCP3GPU_BATCH_NO_AUTOTUNE).  Every cluster sees the same Sobol index range,
 * as separate scp3gpu_hbuild handles given the same calls would. */
typedef struct scp3gpu_batch scp3gpu_batch;
#define SCP3GPU_BATCH_NO_GRAPH 1    /* launch the passes directly instead of replaying a graph */
#define SCP3GPU_BATCH_NO_AUTOTUNE 2 /* keep the default work shape                          */
/* chunk: samples per pass (multiple of 4096; 0 = sized for ~3 GB of operand per pass buffer) */
int scp3gpu_batch_create(const scp3gpu_config* cfgs, int ncl, int64_t chunk, int flags, scp3gpu_batch** out);
int scp3gpu_batch_destroy(scp3gpu_batch* b);
int scp3gpu_batch_reset(scp3gpu_batch* b);
int scp3gpu_batch_size(const scp3gpu_batch* b);
int64_t scp3gpu_batch_basis_size(const scp3gpu_batch* b, int cluster);
int64_t scp3gpu_batch_sample_count(const scp3gpu_batch* b);
void* scp3gpu_batch_stream(const scp3gpu_batch* b);
/* the chosen work shape: sample ranges per tile and pass, CTAs of the
 * contraction launch (0 = one per work unit), samples per pass, and the timed
 * contraction of one pass in ms (0 without autotuning); pointers may be NULL */
int scp3gpu_batch_shape(const scp3gpu_batch* b, int* nsplit, int* ctas, int64_t* chunk, double* ms);
/* Sobol points index0 .. index0+n-1 for every cluster (asynchronous) */
int scp3gpu_batch_accumulate(scp3gpu_batch* b, int64_t index0, int64_t n);
/* as scp3gpu_hbuild_read for one cluster */
int scp3gpu_batch_read(scp3gpu_batch* b, int cluster, double* M, int64_t ld, int mode);
int scp3gpu_batch_status(scp3gpu_batch* b, int cluster, int64_t* nonfinite, int64_t* not_converged);

/* addEpot of the -G path without any device allocation, for callers that
 * cannot call cudaMalloc (a host framework that owns all device memory and hands
 * out only its own buffers, a locked-down allocator, an allocation-free hot
 * loop).  No counterpart in the reference: it exists for those callers.
 * q_dev (n x nmodes, sample-major), V_dev (n) and M_dev (column-major, leading
 * dimension ld >= Nb) are device buffers of the current device; adds
 * sum_s Phi(q_s) V_s Phi(q_s)^T into M_dev (both triangles), FP64, ordered on
 * `stream` (a cudaStream_t; NULL = the legacy default stream).  Working space
 * comes from one static 64 MiB device array; bases over 4032 functions are
 * rejected with SCP3GPU_ERR_ARG.  Throughput falls as the basis nears that
 * limit: samples go through in chunks of 4096 up to 832 functions, and the
 * chunk halves as the tile sums take more of the array (1024 at 1217-1536
 * functions, 512 at 1985-2368, 16 from 3969), each chunk costing two kernel
 * launches.  The first call
 * on a device looks up that array's address (make it before any stream
 * capture); all calls share the array, so calls that overlap on the GPU race --
 * order them on one stream. */
int scp3gpu_add_epot_static(int nmodes, int n2, int n3, const double* q_dev, const double* V_dev, int64_t n,
                            double* M_dev, int64_t ld, void* stream);

/* Write M (n_rows x n_cols, column-major, host memory) as an sM_*.h5 file:
 * dataset "M", dims {n_cols, n_rows}, float32 -- replaces save_hdf5(mat&, char*)
 * (DiskIO.cpp:201-227), which SCP3 calls every 2^17 samples (SCP3.cpp:252-255).
 * Stored contiguous rather than chunked + deflate. */
int scp3gpu_save_h5(const char* path, const double* M, int64_t n_rows, int64_t n_cols);
/* As scp3gpu_save_h5 with the storage chosen: deflate = 0..9 writes the
 * reference's chunked layout (chunks of min(n_cols, ceil(131072 / n_rows))
 * whole columns, each deflated at that level -- 6 in DiskIO.cpp:214-216,
 * compressed on all host threads); deflate = -1 writes it contiguous. */
int scp3gpu_save_h5_layout(const char* path, const double* M, int64_t n_rows, int64_t n_cols, int deflate);
/* load_hdf5(name, M) (DiskIO.cpp:267-289): dataset "M" (dims {n_cols, n_rows},
 * float32 or float64, contiguous or chunked with deflate) into column-major M
 * (leading dimension n_rows).  M == NULL returns the shape only. */
int scp3gpu_load_h5(const char* path, double* M, int64_t* n_rows, int64_t* n_cols);

/* ------------------------------------------------------------------ surrogate
 * The learned control variate (no counterpart in the reference, which always
 * evaluates the exact potential, SCP3.cpp:205-225): an n_in -> hidden -> hidden
 * -> hidden -> 1 GELU network with BF16 weights and FP32 accumulation, trained
 * and evaluated by this library's kernels (the forward layers on the tcgen05
 * tensor cores: n_in 1..256, hidden 64, 128, 192 or 256).  Host buffers; q is
 * n x n_in (sample-major), t and y are n targets/outputs in the units of V_anh. */
typedef struct scp3gpu_mlp scp3gpu_mlp;
int scp3gpu_mlp_create(int n_in, int hidden, int max_batch, uint64_t seed, int device, scp3gpu_mlp** out);
int scp3gpu_mlp_destroy(scp3gpu_mlp* m);
int64_t scp3gpu_mlp_num_params(const scp3gpu_mlp* m);
/* flat parameters: for each layer l = 0..3, W_l (out x in, row-major) then b_l */
int scp3gpu_mlp_get_params(scp3gpu_mlp* m, float* p, int64_t n);
int scp3gpu_mlp_set_params(scp3gpu_mlp* m, const float* p, int64_t n);
/* output = raw * scale + shift (targets are fitted in raw units) */
int scp3gpu_mlp_set_output(scp3gpu_mlp* m, float scale, float shift);
int scp3gpu_mlp_forward(scp3gpu_mlp* m, const float* q, int64_t n, float* y);
/* mean-squared-error loss (raw units) of one batch (n a multiple of 64) and its
 * gradient in the flat parameter order */
int scp3gpu_mlp_grad(scp3gpu_mlp* m, const float* q, const float* t, int n, float* loss, float* grad);
int scp3gpu_mlp_train(scp3gpu_mlp* m, const float* q, const float* t, int64_t n, int epochs, int batch, float lr,
                      uint64_t seed, float* final_loss);

#define SCP3GPU_SURROGATE_NONE 0
#define SCP3GPU_SURROGATE_REPLACE 1  /* V_anh := V_nn(q); the potential is not evaluated */
#define SCP3GPU_SURROGATE_RESIDUAL 2 /* V_anh := V_anh - V_nn(q)                         */
/* Attach a surrogate to a split-form build (its input is the selected modes'
 * q; max_batch >= the build's pass size); the control-variate estimate is
 * M_replace / N_replace + M_residual / N_residual over two builds. */
int scp3gpu_hbuild_set_surrogate(scp3gpu_hbuild* h, scp3gpu_mlp* m, int mode);
/* The per-sample stage alone for points index0..index0+n-1: q of the selected
 * modes (n x nmodes, FP32) and V_anh (n, FP64) into host buffers -- training
 * data for the surrogate. */
int scp3gpu_hbuild_sample(scp3gpu_hbuild* h, int64_t index0, int64_t n, float* q, double* v);

/* ------------------------------------------------------------------ SCP1
 * The thermal averages of the SCP1 effective-Hessian iteration: the sample
 * loop of SCP1::average (SCP1.cpp:34-90) for one rank's share of the points.
 * A handle holds the device buffers (pes: SCP3GPU_PES_*, 1 <= nw <= 8, chunk:
 * samples per device pass, 0 = 65536). */
typedef struct scp3gpu_scp1 scp3gpu_scp1;
int scp3gpu_scp1_create(int pes, int nw, int64_t chunk, int device, scp3gpu_scp1** out);
/* Points i0 <= i < i1 of the unscrambled Sobol sequence at offset `skip`
 * (dimension 9*nw; the reference's current_skip = sobol_skip + i), with
 * q[9nw] (bohr), d[9nw] (displacement variances, >= 0) and isqrtM_U (9nw x 9nw,
 * column-major): returns the SUMS over those points of V (hartree), UX[9nw] =
 * dV/dr (hartree/bohr) and UX_q (9nw x 9nw, column-major) = sum UX dq^T -- the
 * per-rank partials that SCP1.cpp:71-78 all-reduces before dividing by NSobol.
 * Host buffers.  Replaces SCP1::average's loop (SCP1.cpp:49-69). */
int scp3gpu_scp1_average(scp3gpu_scp1* h, const double* q, const double* d, const double* isqrtM_U, int64_t skip,
                         int64_t i0, int64_t i1, double* Upot, double* UX, double* UX_q);
/* TTM3-F samples whose dipoles hit the 500-sweep cap so far (the reference
 * uses their energies and gradients as they are). */
int scp3gpu_scp1_status(const scp3gpu_scp1* h, int64_t* not_converged);
void scp3gpu_scp1_destroy(scp3gpu_scp1* h);

/* Kernel timing (no counterpart in the reference, which has no in-code timing;
 * only a VTune build profile, config/vtune.mk:1-4).  enable = 1 clears and starts
 * recording CUDA events around every kernel the handle launches on its stream;
 * enable = 0 stops, synchronises and returns, per kernel kind (0 per-sample,
 * 1 basis expansion / sign partition, 2 contraction, 3 read-out), the summed
 * device milliseconds and the launch counts (arrays of 4; may be NULL). */
int scp3gpu_hbuild_profile(scp3gpu_hbuild* h, int enable, double* ms, int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif /* SCP3GPU_H */
