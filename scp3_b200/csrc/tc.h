// Split-precision (BF16x3 / FP16x3) contraction on the tcgen05 tensor cores.
#pragma once
#include "internal.h"

namespace scp3 {
namespace tc {

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
    bool f16 = false;             // halves in FP16 (operand scaled by 2^6) instead of BF16
    int64_t slots = 0;            // K slots per pass after sign partition and padding
    // device buffers
    // two pass buffers, so one pass can be prepared while the previous contracts
    // [row block][32-slot k-block][hi, lo][128 x 32] 16-bit sqrt|V| Phi, each box in the swizzled MMA order
    uint16_t* x[2] = {nullptr, nullptr};
    int* slot_of[2] = {nullptr, nullptr};    // [slots] K slot -> sample (-1: zero padding)
    int* group_meta[2] = {nullptr, nullptr}; // per 4096-sample block: first negative 16-group
    int4* tiles2 = nullptr;       // [ntiles] (A row, B rows 0..127, sign-table offset, B rows 128..255) of each 128 x 256 tile
    int* tile_index = nullptr;    // [nt*nt] owner of block (ti <= tj): 4 * tile + 2 * transposed + column half
    uint32_t* factors = nullptr;  // [nb] basis functions as products of Hermite-table entries
    ExpandDesc* desc_dev = nullptr;   // [2] expansion descriptors of the two pass buffers
    ExpandDesc desc_host[2] = {};     // what desc_dev holds (uploaded again only when it changes)
    double* partial = nullptr;    // [nsplit][ntiles][128 x 256] FP64, tile-local column-major
    int* err_flag = nullptr;      // bounded-wait failures
};

constexpr int kTile = 128;        // UMMA M; a tile is 128 x 256 (two panels of B)
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
// contract: the tensor-core accumulation of pass buffer buf into the partials;
// head_done (may be null) is recorded once every whole wave of work units is queued.
int contract(Plan& p, int buf, int64_t n, cudaStream_t s, std::vector<cudaEvent_t>* pev, std::vector<int>* pkind,
             cudaEvent_t head_done = nullptr);
// both, on one stream, buffer 0
int accumulate_pass(Plan& p, const uint32_t* desc, int nb, int nm, const float* q32, const double* v, int64_t n,
                    cudaStream_t s, std::vector<cudaEvent_t>* pev, std::vector<int>* pkind);
int unpack(Plan& p, int nb, double divisor, const double* diag, double zpe, double* M, int64_t ld, cudaStream_t s);

// Launchers shared by the single build and the batch (several clusters in one launch).
int launch_partition(const double* v, int64_t v_stride, int* slot_of, int64_t slot_stride, int* neg, int neg_stride,
                     int nflush, int nclusters, cudaStream_t s);
// slots: K slots of this pass; nkb: 32-slot k-blocks per row block in the operand's allocation
int launch_expand(const ExpandDesc* descs_dev, int nclusters, int max_nb_pad, int max_nm, int64_t slots, int64_t nkb,
                  uint16_t* x, bool f16, cudaStream_t s);
// 128 x 256 tiling shared by the single build and the batch (contract_tc.cu).
struct BaseTile {
    int cluster, ti;              // A panel
    int s0, s1, halves;           // B panels; halves owned (bit 0: s0, bit 1: s1)
    int tr;                       // bit h: half h yields the transpose of needed block (s_h, ti)
    int row0, neg_off;            // the cluster's first operand row and sign-group table offset
};
void add_cluster_tiles(std::vector<BaseTile>& base, int cluster, int nt, int nt_need, int row0, int neg_off);
void finish_tiling(const std::vector<BaseTile>& base, const std::vector<int>& cluster_nt, int sms,
                   std::vector<int4>& tiles, std::vector<std::vector<int>>& owner, int& nsplit);
// grid CTAs loop over units (split, tile); nkb_* count 32-slot k-blocks
// units [u_begin, u_end) (u_end < 0: all)
int launch_contract(const uint16_t* x, int64_t nkb_alloc, const int4* tiles, int ntiles, int nsplit, int nkb_pass,
                    const int* neg, bool f16, double* partial, int* err_flag, int grid, cudaStream_t s,
                    int u_begin = 0, int u_end = -1);
// dense column-major nb x nb of one cluster (its block-owner table) from the unit partials
int launch_unpack(const double* partial, const int* owner, int nt, int ntiles, int nsplit, int nb, double divisor,
                  const double* diag, double zpe, double* M, int64_t ld, cudaStream_t s);
constexpr int kKBlock2 = 32;      // K slots per k-block of the 128 x 256 contraction's operand

}  // namespace tc
}  // namespace scp3
