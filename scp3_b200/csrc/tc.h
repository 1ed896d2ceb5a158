// Split-precision (BF16x3) contraction on the tcgen05 tensor cores.
#pragma once
#include "internal.h"

namespace scp3 {
namespace tc {

// One CTA's share of the contraction: the A and B row bases (128-row panels of
// the operand, which may hold several clusters' bases one after another), the
// offset of its cluster's per-block sign-group table, and the offset of its
// FP64 partial tile (per sample-range split, after split * nitems tiles).
struct WorkItem {
    int arow, brow;     // first operand rows of the tile's A and B panels
    int neg_off;        // index of the cluster's first entry in the sign-group table
    int pad;
    long long poff;     // partial offset in doubles (tile index * 128 * 128)
};

// Per-cluster inputs of the split-operand expansion.
struct ExpandDesc {
    const uint32_t* factors;   // [nb] basis factor table
    int nb, nb_pad, nm;
    int row0;                  // first operand row of this cluster
    const float* q;            // [samples][nm]
    const double* v;           // [samples]
    const int* slot_of;        // [slots] K slot -> sample
};

// The single build's contraction (128 x 256 tiles, contract_tc.cu).
struct Plan {
    int nb = 0, nb_pad = 0, nm = 0;   // nb_pad: whole 256-row panel pairs
    int nt = 0, ntiles = 0;       // 128-row panels per side; 128 x 256 tiles
    int nsplit = 1;               // sample ranges per pass (each unit (split, tile) owns an FP64 partial)
    int grid = 0;                 // CTAs of the contraction (one per SM at most)
    int64_t chunk = 0;            // samples per pass (multiple of kFlush)
    int products = 3;             // 3: hi*hi + hi*lo + lo*hi; 4: + lo*lo
    bool f16 = false;             // halves in FP16 (operand scaled by 2^6) instead of BF16
    int64_t slots = 0;            // K slots per pass after sign partition and padding
    // device buffers
    // two pass buffers, so one pass can be prepared while the previous contracts
    // [row block][k-block][hi, lo][128 x 64] 16-bit sqrt|V| Phi, each box in the swizzled MMA order
    uint16_t* x[2] = {nullptr, nullptr};
    int* slot_of[2] = {nullptr, nullptr};    // [slots] K slot -> sample (-1: zero padding)
    int* group_meta[2] = {nullptr, nullptr}; // per 4096-sample block: first negative 16-group
    int2* tiles2 = nullptr;       // [ntiles] (first A row, first B row) of each 128 x 256 tile
    int* tile_index = nullptr;    // [nt*nt] owner of block (ti, tj): 2 * tile + column half
    uint32_t* factors = nullptr;  // [nb] basis functions as products of Hermite-table entries
    ExpandDesc* desc_dev = nullptr;   // [2] expansion descriptors of the two pass buffers
    ExpandDesc desc_host[2] = {};     // what desc_dev holds (uploaded again only when it changes)
    double* partial = nullptr;    // [nsplit][ntiles][128 x 256] FP64, tile-local column-major
    int* err_flag = nullptr;      // bounded-wait failures
};

constexpr int kTile = 128;        // UMMA M = N = 128
constexpr int kFlush = 4096;      // samples per sign-partition block (the FP64 flush is finer, see contract_tc.cu)
constexpr int kSlotsPerFlush = kFlush + 64;  // sign partition pads each sign group to 16

int create(Plan& p, int nb, int nm, int n2, int n3, int chunk_req, int sms, bool f16);
void destroy(Plan& p);
int64_t pass_samples(const Plan& p, int64_t nvalid);
int zero(Plan& p, cudaStream_t s);
// pev/pkind (may be null): when given, an event pair is recorded around every
// launch with its kind (1 preparation, 2 contraction) for the handle's timing.
// prepare: sign partition + expansion of n samples (q32, v) into pass buffer buf.
int prepare(Plan& p, int buf, int nb, int nm, const float* q32, const double* v, int64_t n, cudaStream_t s,
            std::vector<cudaEvent_t>* pev, std::vector<int>* pkind);
// contract: the tensor-core accumulation of pass buffer buf into the partials.
int contract(Plan& p, int buf, int64_t n, cudaStream_t s, std::vector<cudaEvent_t>* pev, std::vector<int>* pkind);
// both, on one stream, buffer 0
int accumulate_pass(Plan& p, const uint32_t* desc, int nb, int nm, const float* q32, const double* v, int64_t n,
                    cudaStream_t s, std::vector<cudaEvent_t>* pev, std::vector<int>* pkind);
int unpack(Plan& p, int nb, double divisor, const double* diag, double zpe, double* M, int64_t ld, cudaStream_t s);

// Launchers shared by the single build and the batch (several clusters in one launch).
int launch_partition(const double* v, int64_t v_stride, int* slot_of, int64_t slot_stride, int* neg, int neg_stride,
                     int nflush, int nclusters, cudaStream_t s);
// slots: K slots of this pass (k-blocks of 64); nkb: k-blocks per row block in the operand's allocation
// sw64: 32-slot boxes in the 64-byte swizzle (the single build's 128 x 256 contraction;
// nkb then counts 32-slot k-blocks); otherwise 64-slot boxes in the 128-byte swizzle.
int launch_expand(const ExpandDesc* descs_dev, int nclusters, int max_nb_pad, int max_nm, int64_t slots, int64_t nkb,
                  uint16_t* x, bool f16, cudaStream_t s, bool sw64 = false);
// max_ctas > 0: at most that many CTAs, each looping over work units (persistent); 0: one CTA per unit.
int launch_contract(const uint16_t* x, int64_t nkb, const WorkItem* items, int nitems, const int* neg, int nflush,
                    int nsplit, int products, bool f16, double* partial, int* err_flag, cudaStream_t s,
                    int max_ctas = 0);
int launch_unpack(const double* partial, const int* tile_index, int nt, int nitems_total, int nsplit, int64_t item0,
                  int nb, double divisor, const double* diag, double zpe, double* M, int64_t ld, cudaStream_t s);

}  // namespace tc
}  // namespace scp3
