// The sM_*.h5 matrix file (save_hdf5 / load_hdf5, DiskIO.cpp:201-227 and
// DiskIO.cpp:267-289), written and read without the HDF5 library: one dataset
// "M" in the root group, dims {n_cols, n_rows} filled from column-major memory,
// stored as little-endian IEEE float32 -- the reference's layout and element
// type.
//
// Two storage layouts:
//   chunked  the reference's: chunks of whole columns, chunk dims
//            {min(n_cols, ceil(131072 / n_rows)), n_rows}, each deflated at
//            level 6 (zlib stream, HDF5 filter 1), indexed by a version-1
//            B-tree of raw-data chunks.  Chunks compress in parallel.
//   contiguous  uncompressed, one block (fast; what a dump inside a timed loop uses).
// The file uses the format's most widely read structures: superblock version 0,
// a root group held by a symbol table (version-1 B-tree + local heap +
// symbol-table node), and a version-1 object header for the dataset.
//
// The reader takes either layout, float32 or float64 data, and the object-header
// forms the HDF5 library writes by default (continuation and NIL messages,
// attributes and timestamps skipped; a root group of several symbol-table
// nodes).
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kChunkK = 32;               // indexed-storage B-tree K (superblock v0 default)
constexpr size_t kChunkElems = 128 * 1024;

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

struct Chunk {
    std::vector<unsigned char> z;   // deflated bytes
    uint64_t col0 = 0;              // first column (offset in dims[0])
    uint64_t addr = 0;
};

// The superblock, root group and dataset header.  `layout` and `filters` are the
// dataset's layout and (optional) filter pipeline messages; `layout_addr_off`
// is where the data/B-tree address sits inside `layout`.  Returns the offset of
// that address in the buffer.
size_t header(Buf& o, int64_t n_rows, int64_t n_cols, const std::vector<unsigned char>& layout, size_t layout_addr_off,
              const std::vector<unsigned char>* filters, size_t* eof_at)
{
    const int group_leaf_k = 4, group_internal_k = 16;
    // ---- superblock v0 (96 bytes)
    const char sig[8] = {'\x89', 'H', 'D', 'F', '\r', '\n', '\x1a', '\n'};
    o.bytes(sig, 8);
    o.u8(0), o.u8(0), o.u8(0), o.u8(0), o.u8(0);   // versions: superblock, free space, root entry, reserved, shared msg
    o.u8(8), o.u8(8), o.u8(0);                     // sizes of offsets and lengths
    o.u16(group_leaf_k), o.u16(group_internal_k);
    o.u32(0);                                      // consistency flags
    o.u64(0);                                      // base address
    o.u64(kUndef);                                 // free-space info
    *eof_at = o.pos();
    o.u64(0);                                      // end of file, patched by the caller
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
    // fill value v2: allocation early (contiguous) / incremental (chunked), write on allocation, undefined
    const std::vector<unsigned char> fill = {2, (unsigned char)(filters ? 3 : 1), 0, 0};
    auto msize = [](size_t n) { return 8 + ((n + 7) & ~(size_t)7); };
    const size_t hdr_size = msize(space.size()) + msize(dtype.size()) + msize(fill.size()) + msize(layout.size()) +
                            (filters ? msize(filters->size()) : 0);
    o.u8(1), o.u8(0), o.u16(filters ? 5 : 4), o.u32(1), o.u32((uint32_t)hdr_size), o.u32(0);
    message(o, 0x0001, 0, space);
    message(o, 0x0003, 1, dtype);
    message(o, 0x0005, 1, fill);
    if (filters) message(o, 0x000B, 0, *filters);
    const size_t layout_addr_at = o.pos() + 8 + layout_addr_off;
    message(o, 0x0008, 0, layout);
    o.pad8();
    // ---- patch addresses
    o.put64(root_oh_at, root_oh);
    o.put64(root_scratch_at, btree);
    o.put64(root_scratch_at + 8, heap);
    o.put64(symtab_msg_at, btree);
    o.put64(symtab_msg_at + 8, heap);
    o.put64(heap_data_at, heap_data);
    o.put64(child_at, snod);
    o.put64(dset_oh_at, dset_oh);
    return layout_addr_at;
}

// Version-1 B-tree of raw-data chunks (node type 1) over `chunks` (in column
// order), every node written at full size (2K entries).  Returns the root address.
uint64_t chunk_btree(Buf& o, const std::vector<Chunk>& chunks, uint64_t c0, uint64_t n_rows, uint64_t n_cols)
{
    struct Key {
        uint32_t size, mask;
        uint64_t col, row;
    };
    const size_t key_bytes = 4 + 4 + 3 * 8;
    const size_t node_bytes = 24 + 2 * kChunkK * 8 + (2 * kChunkK + 1) * key_bytes;
    auto put_key = [&](const Key& k) {
        o.u32(k.size), o.u32(k.mask);
        o.u64(k.col), o.u64(k.row), o.u64(0);
    };
    // level 0: children are chunks
    struct Entry {
        Key left;
        uint64_t child;
    };
    std::vector<Entry> level;
    for (const Chunk& c : chunks) level.push_back(Entry{Key{(uint32_t)c.z.size(), 0, c.col0, 0}, c.addr});
    // the right key of the last chunk: its offset plus the chunk dims, as the HDF5 library writes it
    const Key end_key{0, 0, chunks.back().col0 + c0, n_rows};
    (void)n_cols;
    int lvl = 0;
    while (true) {
        std::vector<Entry> up;
        const size_t nn = (level.size() + 2 * kChunkK - 1) / (2 * kChunkK);
        std::vector<size_t> addr(nn);
        for (size_t n = 0; n < nn; n++) addr[n] = o.pos() + n * node_bytes;
        for (size_t n = 0; n < nn; n++) {
            const size_t e0 = n * 2 * kChunkK, e1 = std::min(level.size(), e0 + 2 * kChunkK);
            const size_t start = o.pos();
            o.bytes("TREE", 4), o.u8(1), o.u8((unsigned)lvl), o.u16((unsigned)(e1 - e0));
            o.u64(n > 0 ? addr[n - 1] : kUndef), o.u64(n + 1 < nn ? addr[n + 1] : kUndef);
            for (size_t e = e0; e < e1; e++) {
                put_key(level[e].left);
                o.u64(level[e].child);
            }
            put_key(e1 < level.size() ? level[e1].left : end_key);
            o.zeros(node_bytes - (o.pos() - start));
            up.push_back(Entry{level[e0].left, addr[n]});
        }
        if (nn == 1) return addr[0];
        level.swap(up);
        lvl++;
    }
}

bool write_all(const char* path, const Buf& o, const std::vector<Chunk>* chunks, const double* M, uint64_t total)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    bool ok = std::fwrite(o.b.data(), 1, o.b.size(), f) == o.b.size();
    if (chunks) {
        for (const Chunk& c : *chunks)
            if (ok) ok = std::fwrite(c.z.data(), 1, c.z.size(), f) == c.z.size();
    } else {
        std::vector<float> row(4096);
        for (uint64_t k = 0; ok && k < total; k += row.size()) {
            const size_t m = (size_t)std::min<uint64_t>(row.size(), total - k);
            for (size_t i = 0; i < m; i++) row[i] = (float)M[k + i];   // column-major memory order
            ok = std::fwrite(row.data(), sizeof(float), m, f) == m;
        }
    }
    return (std::fclose(f) == 0) && ok;
}

}  // namespace

using namespace scp3;

extern "C" int scp3gpu_save_h5_layout(const char* path, const double* M, int64_t n_rows, int64_t n_cols, int deflate)
{
    if (!path || !M || n_rows < 1 || n_cols < 1 || deflate < -1 || deflate > 9)
        return fail(SCP3GPU_ERR_ARG, "save_h5: bad arguments");
    Buf o;
    size_t eof_at = 0;
    const uint64_t total = (uint64_t)n_rows * n_cols;
    if (deflate < 0) {
        std::vector<unsigned char> layout = {3, 1};                 // v3, contiguous
        append(layout, le(0, 8)), append(layout, le(total * 4, 8));
        const size_t addr_at = header(o, n_rows, n_cols, layout, 2, nullptr, &eof_at);
        o.put64(addr_at, o.pos());
        o.put64(eof_at, o.pos() + total * 4);
        if (!write_all(path, o, nullptr, M, total))
            return fail(SCP3GPU_ERR_ARG, std::string("save_h5: write failed for ") + path);
        return SCP3GPU_OK;
    }
    // chunks of whole columns, DiskIO.cpp:211-213
    const uint64_t c0 = std::min<uint64_t>((uint64_t)n_cols, (kChunkElems + n_rows - 1) / n_rows);
    const uint64_t nch = ((uint64_t)n_cols + c0 - 1) / c0;
    std::vector<Chunk> chunks(nch);
    std::atomic<uint64_t> next{0};
    std::atomic<bool> bad{false};
    auto work = [&]() {
        std::vector<float> buf((size_t)(c0 * n_rows));
        for (uint64_t k; (k = next.fetch_add(1)) < nch && !bad;) {
            const uint64_t col0 = k * c0, ncols = std::min<uint64_t>(c0, (uint64_t)n_cols - col0);
            std::fill(buf.begin(), buf.end(), 0.0f);   // an edge chunk is stored at full size
            for (uint64_t i = 0; i < ncols * n_rows; i++) buf[i] = (float)M[col0 * n_rows + i];
            uLongf zn = compressBound((uLong)(buf.size() * 4));
            chunks[k].z.resize(zn);
            if (compress2(chunks[k].z.data(), &zn, reinterpret_cast<const Bytef*>(buf.data()), (uLong)(buf.size() * 4),
                          deflate) != Z_OK)
                bad = true;
            chunks[k].z.resize(zn);
            chunks[k].col0 = col0;
        }
    };
    const int nth = (int)std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)nch));
    std::vector<std::thread> pool;
    for (int t = 1; t < nth; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    if (bad) return fail(SCP3GPU_ERR_ARG, "save_h5: deflate failed");
    // filter pipeline v1: deflate (id 1), one client value (the level) + 4 bytes padding
    std::vector<unsigned char> filters = {1, 1, 0, 0, 0, 0, 0, 0};
    append(filters, le(1, 2)), append(filters, le(0, 2)), append(filters, le(0, 2)), append(filters, le(1, 2));
    append(filters, le((uint64_t)deflate, 4)), append(filters, le(0, 4));
    // layout v3, chunked: rank + 1 dims (the last is the element size), B-tree address
    std::vector<unsigned char> layout = {3, 2, 3};
    append(layout, le(0, 8));
    append(layout, le(c0, 4)), append(layout, le((uint64_t)n_rows, 4)), append(layout, le(4, 4));
    const size_t addr_at = header(o, n_rows, n_cols, layout, 3, &filters, &eof_at);
    uint64_t at = o.pos();
    const size_t key_bytes = 32, node_bytes = 24 + 2 * kChunkK * 8 + (2 * kChunkK + 1) * key_bytes;
    // B-tree nodes go after the header, chunks after the nodes: count the nodes first
    uint64_t nodes = 0;
    for (uint64_t l = nch; ; ) {
        const uint64_t nn = (l + 2 * kChunkK - 1) / (2 * kChunkK);
        nodes += nn;
        if (nn == 1) break;
        l = nn;
    }
    uint64_t data = at + nodes * node_bytes;
    for (Chunk& c : chunks) {
        c.addr = data;
        data += c.z.size();
    }
    const uint64_t root = chunk_btree(o, chunks, c0, (uint64_t)n_rows, (uint64_t)n_cols);
    if (o.pos() != at + nodes * node_bytes) return fail(SCP3GPU_ERR_ARG, "save_h5: B-tree size mismatch");
    o.put64(addr_at, root);
    o.put64(eof_at, data);
    if (!write_all(path, o, &chunks, M, total))
        return fail(SCP3GPU_ERR_ARG, std::string("save_h5: write failed for ") + path);
    return SCP3GPU_OK;
}

extern "C" int scp3gpu_save_h5(const char* path, const double* M, int64_t n_rows, int64_t n_cols)
{
    return scp3gpu_save_h5_layout(path, M, n_rows, n_cols, -1);
}

// ------------------------------------------------------------------ reader
namespace {

struct File {
    std::vector<unsigned char> b;
    bool ok(uint64_t at, uint64_t n) const { return at <= b.size() && n <= b.size() - at; }
    uint64_t u(uint64_t at, int n) const
    {
        uint64_t v = 0;
        for (int i = n - 1; i >= 0; i--) v = (v << 8) | b[at + i];
        return v;
    }
};

struct Msg {
    unsigned type;
    uint64_t at, size;
};

// Messages of a version-1 object header, following continuation messages.
bool header_messages(const File& f, uint64_t oh, std::vector<Msg>& out)
{
    if (!f.ok(oh, 16) || f.b[oh] != 1) return false;
    const unsigned nmsg = (unsigned)f.u(oh + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks = {{oh + 16, f.u(oh + 8, 4)}};
    for (size_t bi = 0; bi < blocks.size() && out.size() < nmsg; bi++) {
        uint64_t p = blocks[bi].first;
        const uint64_t end = p + blocks[bi].second;
        while (p + 8 <= end && out.size() < nmsg) {
            if (!f.ok(p, 8)) return false;
            const unsigned type = (unsigned)f.u(p, 2);
            const uint64_t size = f.u(p + 2, 2);
            if (!f.ok(p + 8, size)) return false;
            if (type == 0x0010 && size >= 16) blocks.push_back({f.u(p + 8, 8), f.u(p + 16, 8)});
            out.push_back(Msg{type, p + 8, size});
            p += 8 + size;
        }
        if (blocks.size() > 64) return false;
    }
    return true;
}

// Object header address of `name` in the group whose symbol table is (btree, heap).
bool find_in_group(const File& f, uint64_t btree, uint64_t heap, const char* name, uint64_t& oh, int depth = 0)
{
    if (depth > 16 || !f.ok(heap, 32) || std::memcmp(&f.b[heap], "HEAP", 4) != 0) return false;
    const uint64_t heap_data = f.u(heap + 24, 8);
    if (!f.ok(btree, 24) || std::memcmp(&f.b[btree], "TREE", 4) != 0 || f.b[btree + 4] != 0) return false;
    const unsigned level = f.b[btree + 5], used = (unsigned)f.u(btree + 6, 2);
    for (unsigned e = 0; e < used; e++) {
        const uint64_t child = f.u(btree + 24 + 8 + 16 * e, 8);
        if (level > 0) {
            if (find_in_group(f, child, heap, name, oh, depth + 1)) return true;
            continue;
        }
        if (!f.ok(child, 8) || std::memcmp(&f.b[child], "SNOD", 4) != 0) return false;
        const unsigned nsym = (unsigned)f.u(child + 6, 2);
        for (unsigned k = 0; k < nsym; k++) {
            const uint64_t ent = child + 8 + 40 * (uint64_t)k;
            if (!f.ok(ent, 40)) return false;
            const uint64_t name_at = heap_data + f.u(ent, 8);
            if (!f.ok(name_at, std::strlen(name) + 1)) continue;
            if (std::memcmp(&f.b[name_at], name, std::strlen(name) + 1) == 0) {
                oh = f.u(ent + 8, 8);
                return true;
            }
        }
    }
    return false;
}

struct ChunkRef {
    uint64_t addr, size, col;
    uint32_t mask;
};

bool collect_chunks(const File& f, uint64_t node, int rank, std::vector<ChunkRef>& out, int depth = 0)
{
    if (depth > 32 || !f.ok(node, 24) || std::memcmp(&f.b[node], "TREE", 4) != 0 || f.b[node + 4] != 1) return false;
    const unsigned level = f.b[node + 5], used = (unsigned)f.u(node + 6, 2);
    const uint64_t key_bytes = 8 + 8 * (uint64_t)(rank + 1);
    for (unsigned e = 0; e < used; e++) {
        const uint64_t key = node + 24 + e * (key_bytes + 8);
        if (!f.ok(key, key_bytes + 8)) return false;
        const uint64_t child = f.u(key + key_bytes, 8);
        if (level > 0) {
            if (!collect_chunks(f, child, rank, out, depth + 1)) return false;
        } else {
            out.push_back(ChunkRef{child, f.u(key, 4), f.u(key + 8, 8), (uint32_t)f.u(key + 4, 4)});
        }
    }
    return true;
}

}  // namespace

// Reads dataset "M": with M == NULL only the shape.  M: column-major n_rows x n_cols, leading dimension n_rows.
extern "C" int scp3gpu_load_h5(const char* path, double* M, int64_t* n_rows, int64_t* n_cols)
{
    if (!path || !n_rows || !n_cols) return fail(SCP3GPU_ERR_ARG, "load_h5: bad arguments");
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(SCP3GPU_ERR_ARG, std::string("load_h5: cannot open ") + path);
    File f;
    std::fseek(fp, 0, SEEK_END);
    const long len = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    f.b.resize(len > 0 ? (size_t)len : 0);
    const bool rd = std::fread(f.b.data(), 1, f.b.size(), fp) == f.b.size();
    std::fclose(fp);
    auto bad = [&](const char* why) { return fail(SCP3GPU_ERR_ARG, std::string("load_h5: ") + why + " in " + path); };
    static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    if (!rd || f.b.size() < 96 || std::memcmp(f.b.data(), sig, 8) != 0) return bad("not an HDF5 file");
    if (f.b[8] != 0 || f.b[13] != 8 || f.b[14] != 8) return bad("superblock version 0 with 8-byte offsets expected");
    const uint64_t root_oh = f.u(64, 8);
    std::vector<Msg> msgs;
    if (!header_messages(f, root_oh, msgs)) return bad("unreadable root group header");
    uint64_t btree = kUndef, heap = kUndef;
    for (const Msg& m : msgs)
        if (m.type == 0x0011) btree = f.u(m.at, 8), heap = f.u(m.at + 8, 8);
    uint64_t oh = 0;
    if (btree == kUndef || !find_in_group(f, btree, heap, "M", oh)) return bad("dataset \"M\" not found");
    msgs.clear();
    if (!header_messages(f, oh, msgs)) return bad("unreadable dataset header");
    const Msg *space = nullptr, *dtype = nullptr, *layout = nullptr, *filt = nullptr;
    for (const Msg& m : msgs) {
        if (m.type == 0x0001) space = &m;
        if (m.type == 0x0003) dtype = &m;
        if (m.type == 0x0008) layout = &m;
        if (m.type == 0x000B) filt = &m;
    }
    if (!space || !dtype || !layout) return bad("dataspace, datatype or layout message missing");
    const unsigned sver = f.b[space->at], rank = f.b[space->at + 1];
    const uint64_t dims_at = space->at + (sver == 1 ? 8 : 4);
    if (rank != 2) return bad("rank-2 dataset expected (DiskIO.cpp:275-280)");
    const uint64_t d0 = f.u(dims_at, 8), d1 = f.u(dims_at + 8, 8);   // {n_cols, n_rows}
    *n_cols = (int64_t)d0;
    *n_rows = (int64_t)d1;
    if (!M) return SCP3GPU_OK;
    if ((f.b[dtype->at] & 0x0F) != 1 || (f.b[dtype->at + 1] & 1)) return bad("little-endian IEEE float data expected");
    const uint64_t esize = f.u(dtype->at + 4, 4);
    if (esize != 4 && esize != 8) return bad("float32 or float64 data expected");
    auto convert = [&](const unsigned char* src, uint64_t n, double* dst) {
        for (uint64_t i = 0; i < n; i++) {
            if (esize == 4) {
                float x;
                std::memcpy(&x, src + 4 * i, 4);
                dst[i] = x;
            } else {
                std::memcpy(dst + i, src + 8 * i, 8);
            }
        }
    };
    const uint64_t total = d0 * d1;
    if (f.b[layout->at] != 3) return bad("layout message version 3 expected");
    const unsigned cls = f.b[layout->at + 1];
    if (cls == 1) {   // contiguous
        const uint64_t addr = f.u(layout->at + 2, 8);
        if (!f.ok(addr, total * esize)) return bad("data beyond the end of the file");
        convert(&f.b[addr], total, M);
        return SCP3GPU_OK;
    }
    if (cls != 2) return bad("contiguous or chunked layout expected");
    if (f.b[layout->at + 2] != 3) return bad("chunk dimensionality 3 expected");
    const uint64_t root = f.u(layout->at + 3, 8);
    const uint64_t c0 = f.u(layout->at + 11, 4), c1 = f.u(layout->at + 15, 4);
    if (c1 != d1 || c0 == 0) return bad("chunks of whole columns expected");
    // filters: deflate only
    unsigned nfilt = 0;
    if (filt) {
        const unsigned fver = f.b[filt->at];
        nfilt = f.b[filt->at + 1];
        uint64_t p = filt->at + (fver == 1 ? 8 : 2);
        for (unsigned k = 0; k < nfilt; k++) {
            const unsigned id = (unsigned)f.u(p, 2);
            if (id != 1) return bad("filters other than deflate are not supported");
            uint64_t name_len = (fver == 1 || id >= 256) ? f.u(p + 2, 2) : 0;
            const unsigned ncv = (unsigned)f.u(p + (fver == 1 || id >= 256 ? 6 : 4), 2);
            p += (fver == 1 || id >= 256) ? 8 : 6;
            p += name_len + 4ull * ncv + ((fver == 1 && (ncv & 1)) ? 4 : 0);
        }
    }
    std::vector<ChunkRef> ch;
    if (!collect_chunks(f, root, 2, ch)) return bad("unreadable chunk B-tree");
    std::vector<unsigned char> raw((size_t)(c0 * c1 * esize));
    uint64_t covered = 0;
    for (const ChunkRef& c : ch) {
        if (!f.ok(c.addr, c.size) || c.col % c0 != 0 || c.col >= d0) return bad("chunk out of range");
        const unsigned char* src = &f.b[c.addr];
        if (nfilt && !(c.mask & 1)) {
            uLongf n = (uLongf)raw.size();
            if (uncompress(raw.data(), &n, src, (uLong)c.size) != Z_OK || n != raw.size()) return bad("inflate failed");
            src = raw.data();
        } else if (c.size < raw.size()) {
            return bad("short unfiltered chunk");
        }
        const uint64_t ncols = std::min<uint64_t>(c0, d0 - c.col);
        convert(src, ncols * d1, M + c.col * d1);
        covered += ncols;
    }
    if (covered != d0) return bad("chunks do not cover the dataset");
    return SCP3GPU_OK;
}
