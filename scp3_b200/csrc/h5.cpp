// The sM_*.h5 matrix file (save_hdf5 / load_hdf5, DiskIO.cpp:201-227 and
// DiskIO.cpp:267-289), written without the HDF5 library: one dataset "M" in the
// root group, dims {n_cols, n_rows} filled from column-major memory, stored as
// little-endian IEEE float32 -- the reference's layout and element type.
//
// The file uses the HDF5 format's most widely read structures: superblock
// version 0, a root group held by a symbol table (version-1 B-tree + local heap
// + symbol-table node), and a version-1 object header for the dataset with
// dataspace, datatype, fill-value (v2) and contiguous layout (v3) messages.
// Unlike the reference (chunked, deflate level 6) the data is stored contiguous
// and uncompressed; readers see the same dataset.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace {

constexpr uint64_t kUndef = ~0ull;

struct Buf {
    std::vector<unsigned char> b;
    size_t pos() const { return b.size(); }
    void u8(unsigned v) { b.push_back((unsigned char)v); }
    void u16(unsigned v) { u8(v & 255), u8((v >> 8) & 255); }
    void u32(uint32_t v)
    {
        for (int i = 0; i < 4; i++) u8((v >> (8 * i)) & 255);
    }
    void u64(uint64_t v)
    {
        for (int i = 0; i < 8; i++) u8((unsigned)((v >> (8 * i)) & 255));
    }
    void bytes(const char* s, size_t n) { b.insert(b.end(), s, s + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad8()
    {
        while (b.size() % 8) b.push_back(0);
    }
    void put64(size_t at, uint64_t v)
    {
        for (int i = 0; i < 8; i++) b[at + i] = (unsigned char)((v >> (8 * i)) & 255);
    }
};

// One version-1 object header message: type, size (data padded to 8), flags.
void message(Buf& o, unsigned type, unsigned flags, const std::vector<unsigned char>& data)
{
    const size_t size = (data.size() + 7) & ~(size_t)7;
    o.u16(type);
    o.u16((unsigned)size);
    o.u8(flags);
    o.zeros(3);
    o.b.insert(o.b.end(), data.begin(), data.end());
    o.zeros(size - data.size());
}

std::vector<unsigned char> le(uint64_t v, int n)
{
    std::vector<unsigned char> r(n);
    for (int i = 0; i < n; i++) r[i] = (unsigned char)((v >> (8 * i)) & 255);
    return r;
}

void append(std::vector<unsigned char>& a, const std::vector<unsigned char>& b) { a.insert(a.end(), b.begin(), b.end()); }

}  // namespace

using namespace scp3;

extern "C" int scp3gpu_save_h5(const char* path, const double* M, int64_t n_rows, int64_t n_cols)
{
    if (!path || !M || n_rows < 1 || n_cols < 1) return fail(SCP3GPU_ERR_ARG, "save_h5: bad arguments");
    const int group_leaf_k = 4, group_internal_k = 16;
    Buf o;
    // ---- superblock v0 (96 bytes)
    const char sig[8] = {'\x89', 'H', 'D', 'F', '\r', '\n', '\x1a', '\n'};
    o.bytes(sig, 8);
    o.u8(0), o.u8(0), o.u8(0), o.u8(0), o.u8(0);   // versions: superblock, free space, root entry, reserved, shared msg
    o.u8(8), o.u8(8), o.u8(0);                     // sizes of offsets and lengths
    o.u16(group_leaf_k), o.u16(group_internal_k);
    o.u32(0);                                      // consistency flags
    o.u64(0);                                      // base address
    o.u64(kUndef);                                 // free-space info
    const size_t eof_at = o.pos();
    o.u64(0);                                      // end of file, patched below
    o.u64(kUndef);                                 // driver information block
    // root group symbol table entry
    o.u64(0);                                      // link name offset
    const size_t root_oh_at = o.pos();
    o.u64(0);                                      // object header address, patched
    o.u32(1), o.u32(0);                            // cache type 1: B-tree and heap addresses follow
    const size_t root_scratch_at = o.pos();
    o.u64(0), o.u64(0);                            // B-tree, heap (patched)
    // ---- root group object header (v1) with one symbol-table message
    const size_t root_oh = o.pos();
    o.u8(1), o.u8(0), o.u16(1), o.u32(1), o.u32(24), o.u32(0);
    const size_t symtab_msg_at = o.pos() + 8;
    message(o, 0x0011, 0, std::vector<unsigned char>(16, 0));
    // ---- local heap: "" at 0, "M" at 8
    o.pad8();
    const size_t heap = o.pos();
    o.bytes("HEAP", 4), o.u8(0), o.zeros(3);
    o.u64(16);                                     // data segment size
    o.u64(kUndef);                                 // no free block
    const size_t heap_data_at = o.pos();
    o.u64(0);                                      // data segment address, patched
    const size_t heap_data = o.pos();
    o.zeros(8);
    o.bytes("M", 1), o.zeros(7);
    // ---- v1 B-tree, group node, one child
    const size_t btree = o.pos();
    o.bytes("TREE", 4), o.u8(0), o.u8(0), o.u16(1);
    o.u64(kUndef), o.u64(kUndef);
    o.u64(0);                                      // key 0: ""
    const size_t child_at = o.pos();
    o.u64(0);                                      // child 0: symbol table node, patched
    o.u64(8);                                      // key 1: "M"
    o.zeros((size_t)(2 * group_internal_k - 1) * 16);   // room for 2K children + 2K+1 keys
    // ---- symbol table node with the dataset's entry
    const size_t snod = o.pos();
    o.bytes("SNOD", 4), o.u8(1), o.u8(0), o.u16(1);
    o.u64(8);                                      // link name offset of "M"
    const size_t dset_oh_at = o.pos();
    o.u64(0);                                      // object header address, patched
    o.u32(0), o.u32(0), o.zeros(16);
    o.zeros((size_t)(2 * group_leaf_k - 1) * 40);
    // ---- dataset object header (v1)
    o.pad8();
    const size_t dset_oh = o.pos();
    std::vector<unsigned char> space = {1, 2, 0, 0, 0, 0, 0, 0};   // v1, rank 2, no max dims
    append(space, le((uint64_t)n_cols, 8));
    append(space, le((uint64_t)n_rows, 8));
    std::vector<unsigned char> dtype = {0x11, 0x20, 31, 0};         // v1 float, LE, implied msb, sign bit 31
    append(dtype, le(4, 4));                                        // size
    append(dtype, le(0, 2)), append(dtype, le(32, 2));              // bit offset, precision
    dtype.push_back(23), dtype.push_back(8), dtype.push_back(0), dtype.push_back(23);   // exp loc/size, mant loc/size
    append(dtype, le(127, 4));                                      // exponent bias
    std::vector<unsigned char> fill = {2, 1, 0, 0};                 // v2, early allocation, write on alloc, undefined
    const uint64_t nbytes = (uint64_t)n_rows * n_cols * 4;
    std::vector<unsigned char> layout = {3, 1};                     // v3, contiguous
    const size_t hdr_size = 4 * 8 + 24 + 24 + 8 + 24;
    o.u8(1), o.u8(0), o.u16(4), o.u32(1), o.u32((uint32_t)hdr_size), o.u32(0);
    message(o, 0x0001, 0, space);
    message(o, 0x0003, 1, dtype);
    message(o, 0x0005, 1, fill);
    const size_t layout_addr_at = o.pos() + 8 + 2;
    append(layout, le(0, 8)), append(layout, le(nbytes, 8));
    message(o, 0x0008, 0, layout);
    o.pad8();
    const size_t data = o.pos();
    // ---- patch addresses
    o.put64(eof_at, data + nbytes);
    o.put64(root_oh_at, root_oh);
    o.put64(root_scratch_at, btree);
    o.put64(root_scratch_at + 8, heap);
    o.put64(symtab_msg_at, btree);
    o.put64(symtab_msg_at + 8, heap);
    o.put64(heap_data_at, heap_data);
    o.put64(child_at, snod);
    o.put64(dset_oh_at, dset_oh);
    o.put64(layout_addr_at, data);

    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(SCP3GPU_ERR_ARG, std::string("save_h5: cannot open ") + path);
    bool ok = std::fwrite(o.b.data(), 1, o.b.size(), f) == o.b.size();
    std::vector<float> row(4096);
    const uint64_t total = (uint64_t)n_rows * n_cols;
    for (uint64_t k = 0; ok && k < total; k += row.size()) {
        const size_t m = (size_t)std::min<uint64_t>(row.size(), total - k);
        for (size_t i = 0; i < m; i++) row[i] = (float)M[k + i];   // column-major memory order
        ok = std::fwrite(row.data(), sizeof(float), m, f) == m;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? SCP3GPU_OK : fail(SCP3GPU_ERR_ARG, std::string("save_h5: write failed for ") + path);
}
