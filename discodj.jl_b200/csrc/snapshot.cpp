// Snapshot files of the particle state: (Psi, Pi = dPsi/dD) as HDF5.
//
// Writes what the study driver's snapshot writer writes
// (studies/eft_shell_crossing/scripts/run_jobs.jl:41-48, called from
// studies/eft_shell_crossing/src/runners.jl:154-156): the datasets "Psi" and "Pi", each a
// (n,n,n,3) Float32 column-major array, and the float64 attributes "D" and "L" of the root
// group. HDF5 lists a column-major array's dimensions in reverse, so a C-order reader sees
// (3,n,n,n) and a Julia reader (n,n,n,3), as with the reference's files.
//
// The file uses the oldest HDF5 format, which every HDF5 library reads: superblock
// version 0, version-1 object headers, and a root group held by a symbol table (a
// version-1 B-tree over one symbol-table node, names in a local heap). Every structure
// follows the HDF5 File Format Specification version 2.0 and carries the same messages,
// in the same versions, as the files the HDF5 library itself writes in this format
// (dataspace 1 with maximum dimensions, floating-point datatype 1, fill value 2, layout 3
// contiguous, attribute 1). All addresses are known before the first byte is written,
// so the metadata goes out first and the array payloads stream after it.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"
#include "snapshot.h"

namespace djb {
namespace {

constexpr uint64_t kUndef = ~uint64_t(0);
constexpr int kLeafK = 4;        // group leaf node K: a symbol-table node holds 2K entries
constexpr int kInternalK = 16;   // group internal node K: a B-tree node holds 2K children
constexpr uint64_t kSuperblock = 96;
constexpr uint64_t kSnodSize = 8 + 2 * kLeafK * 40;
constexpr uint64_t kBtreeSize = 24 + 2 * kInternalK * 8 + (2 * kInternalK + 1) * 8;
constexpr uint64_t kHeapFreeNone = 1;  // "no free block" in a local heap's free-list field

uint64_t pad8(uint64_t v) { return (v + 7) & ~uint64_t(7); }

struct Buf {
    std::vector<uint8_t> b;
    void u8(unsigned v) { b.push_back(uint8_t(v)); }
    void u16(unsigned v) { u8(v & 0xff); u8((v >> 8) & 0xff); }
    void u32(uint32_t v) { for (int i = 0; i < 4; ++i) u8((v >> (8 * i)) & 0xff); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) u8(unsigned((v >> (8 * i)) & 0xff)); }
    void bytes(const void* p, size_t n) { const uint8_t* c = static_cast<const uint8_t*>(p); b.insert(b.end(), c, c + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void align8() { zeros(pad8(b.size()) - b.size()); }
    size_t size() const { return b.size(); }
};

// IEEE little-endian floating-point datatype message body (class 1, version 1), 20 bytes.
void float_type(Buf& o, int bytes) {
    const bool f64 = bytes == 8;
    o.u8(0x11);                        // version 1, class 1 (floating point)
    o.u8(0x20);                        // little endian, no padding bits, implied mantissa MSB
    o.u8(f64 ? 63 : 31);               // sign bit position
    o.u8(0);
    o.u32(uint32_t(bytes));
    o.u16(0);                          // bit offset
    o.u16(f64 ? 64 : 32);              // precision
    o.u8(f64 ? 52 : 23);               // exponent location
    o.u8(f64 ? 11 : 8);                // exponent size
    o.u8(0);                           // mantissa location
    o.u8(f64 ? 52 : 23);               // mantissa size
    o.u32(f64 ? 1023u : 127u);         // exponent bias
}

void msg_header(Buf& o, unsigned type, size_t size, unsigned flags) {
    o.u16(type);
    o.u16(unsigned(size));
    o.u8(flags);
    o.zeros(3);
}

// Version-1 object header prefix (12 bytes, padded to 16).
void object_prefix(Buf& o, unsigned nmsg, uint64_t chunk) {
    o.u8(1);
    o.u8(0);
    o.u16(nmsg);
    o.u32(1);                          // reference count
    o.u32(uint32_t(chunk));
    o.zeros(4);
}

size_t attribute_msg_size(const std::string& name) { return 8 + pad8(name.size() + 1) + 24 + 8 + 8; }

void attribute_f64(Buf& o, const std::string& name, double v) {
    msg_header(o, 0x0C, attribute_msg_size(name), 0);
    o.u8(1);
    o.u8(0);
    o.u16(unsigned(name.size() + 1));
    o.u16(20);                         // datatype message size
    o.u16(8);                          // scalar dataspace message size
    o.bytes(name.c_str(), name.size() + 1);
    o.zeros(pad8(name.size() + 1) - (name.size() + 1));
    float_type(o, 8);
    o.zeros(4);
    o.u8(1); o.u8(0); o.u8(0); o.u8(0); o.u32(0);  // dataspace version 1, rank 0
    o.bytes(&v, 8);
}

size_t dataset_chunk(size_t rank) { return (8 + 8 + 16 * rank) + (8 + 24) + (8 + 8) + (8 + 24); }

void dataset_header(Buf& o, const std::vector<uint64_t>& dims, int elem, uint64_t addr, uint64_t bytes) {
    object_prefix(o, 4, dataset_chunk(dims.size()));
    msg_header(o, 0x01, 8 + 16 * dims.size(), 0);   // dataspace, version 1, with maximum dims
    o.u8(1); o.u8(uint8_t(dims.size())); o.u8(1); o.u8(0); o.u32(0);
    for (uint64_t d : dims) o.u64(d);
    for (uint64_t d : dims) o.u64(d);
    msg_header(o, 0x03, 24, 1);                     // datatype (constant)
    float_type(o, elem);
    o.zeros(4);
    msg_header(o, 0x05, 8, 1);                      // fill value, version 2: late allocation, default value
    o.u8(2); o.u8(2); o.u8(2); o.u8(1); o.u32(0);
    msg_header(o, 0x08, 24, 0);                     // layout, version 3, contiguous
    o.u8(3); o.u8(1); o.u64(addr); o.u64(bytes);
    o.zeros(6);
}

}  // namespace

int h5_write_arrays(const char* path, const std::vector<H5Array>& arrays, const std::vector<H5Attr>& attrs,
                    const H5Payload& payload) {
    if (!path || !*path) return fail(DJB_ERR_INVALID, "snapshot path is empty");
    if (arrays.empty() || arrays.size() > size_t(2 * kLeafK))
        return fail(DJB_ERR_INVALID, "a snapshot holds 1 to %d datasets", 2 * kLeafK);
    // names sorted as the symbol-table node keeps them (byte order)
    std::vector<size_t> order(arrays.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    for (size_t i = 1; i < order.size(); ++i)
        for (size_t j = i; j > 0 && arrays[order[j]].name < arrays[order[j - 1]].name; --j) std::swap(order[j], order[j - 1]);
    for (size_t i = 1; i < order.size(); ++i)
        if (arrays[order[i]].name == arrays[order[i - 1]].name) return fail(DJB_ERR_INVALID, "duplicate dataset name");
    for (const auto& a : arrays)
        if (a.name.empty() || a.dims.empty() || a.dims.size() > 32 || (a.elem != 4 && a.elem != 8))
            return fail(DJB_ERR_INVALID, "bad dataset description");

    // local heap data: the empty name at 0, then each dataset name, 8-byte aligned
    std::vector<uint64_t> name_off(arrays.size());
    uint64_t heap_data = 8;
    for (size_t i = 0; i < arrays.size(); ++i) {
        name_off[i] = heap_data;
        heap_data += pad8(arrays[i].name.size() + 1);
    }
    uint64_t root_chunk = 8 + 16;
    for (const auto& at : attrs) root_chunk += 8 + attribute_msg_size(at.name);

    const uint64_t a_root = kSuperblock;
    const uint64_t a_heap = a_root + 16 + root_chunk;
    const uint64_t a_heapdata = a_heap + 32;
    const uint64_t a_btree = a_heapdata + heap_data;
    const uint64_t a_snod = a_btree + kBtreeSize;
    std::vector<uint64_t> a_obj(arrays.size()), a_raw(arrays.size()), nbytes(arrays.size());
    uint64_t p = a_snod + kSnodSize;
    for (size_t i = 0; i < arrays.size(); ++i) {
        a_obj[i] = p;
        p += 16 + dataset_chunk(arrays[i].dims.size());
    }
    p = (p + 4095) & ~uint64_t(4095);     // payloads start on a page boundary
    for (size_t i = 0; i < arrays.size(); ++i) {
        uint64_t cnt = 1;
        for (uint64_t d : arrays[i].dims) cnt *= d;
        nbytes[i] = cnt * uint64_t(arrays[i].elem);
        a_raw[i] = p;
        p = pad8(p + nbytes[i]);
    }
    const uint64_t eof = p;

    Buf o;
    // superblock version 0
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    o.bytes(sig, 8);
    o.u8(0); o.u8(0); o.u8(0); o.u8(0); o.u8(0); o.u8(8); o.u8(8); o.u8(0);
    o.u16(kLeafK);
    o.u16(kInternalK);
    o.u32(0);
    o.u64(0);            // base address
    o.u64(kUndef);       // free-space info
    o.u64(eof);
    o.u64(kUndef);       // driver information block
    o.u64(0);            // root symbol-table entry: name offset
    o.u64(a_root);
    o.u32(1);            // cache type 1: B-tree and heap addresses in the scratch pad
    o.u32(0);
    o.u64(a_btree);
    o.u64(a_heap);
    // root group object header: symbol table message, then the attributes
    object_prefix(o, unsigned(1 + attrs.size()), root_chunk);
    msg_header(o, 0x11, 16, 0);
    o.u64(a_btree);
    o.u64(a_heap);
    for (const auto& at : attrs) attribute_f64(o, at.name, at.value);
    // local heap
    o.bytes("HEAP", 4);
    o.u8(0); o.zeros(3);
    o.u64(heap_data);
    o.u64(kHeapFreeNone);
    o.u64(a_heapdata);
    o.zeros(8);
    for (const auto& a : arrays) {
        o.bytes(a.name.c_str(), a.name.size() + 1);
        o.align8();
    }
    // B-tree node (type 0, leaf level) with one child: the symbol-table node
    o.bytes("TREE", 4);
    o.u8(0); o.u8(0); o.u16(1);
    o.u64(kUndef); o.u64(kUndef);
    o.u64(0);                                  // left key: the empty name
    o.u64(a_snod);
    o.u64(name_off[order.back()]);             // right key: the last name in the child
    o.zeros(kBtreeSize - (24 + 3 * 8));
    // symbol-table node
    o.bytes("SNOD", 4);
    o.u8(1); o.u8(0); o.u16(unsigned(arrays.size()));
    for (size_t i : order) {
        o.u64(name_off[i]);
        o.u64(a_obj[i]);
        o.u32(0); o.u32(0);
        o.zeros(16);
    }
    o.zeros(size_t(2 * kLeafK - arrays.size()) * 40);
    for (size_t i = 0; i < arrays.size(); ++i) {
        if (o.size() != a_obj[i]) return fail(DJB_ERR_INVALID, "snapshot layout mismatch");
        dataset_header(o, arrays[i].dims, arrays[i].elem, a_raw[i], nbytes[i]);
    }
    o.zeros(a_raw[0] - o.size());

    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(DJB_ERR_IO, "cannot open %s for writing", path);
    int rc = DJB_OK;
    if (std::fwrite(o.b.data(), 1, o.size(), fp) != o.size()) rc = fail(DJB_ERR_IO, "write failed: %s", path);
    uint64_t at = o.size();
    for (size_t i = 0; i < arrays.size() && rc == DJB_OK; ++i) {
        if (at != a_raw[i]) {
            const std::vector<uint8_t> z(a_raw[i] - at, 0);
            if (std::fwrite(z.data(), 1, z.size(), fp) != z.size()) { rc = fail(DJB_ERR_IO, "write failed: %s", path); break; }
        }
        rc = payload(i, fp);
        at = a_raw[i] + nbytes[i];
    }
    if (rc == DJB_OK && at != eof) {
        const std::vector<uint8_t> z(eof - at, 0);
        if (std::fwrite(z.data(), 1, z.size(), fp) != z.size()) rc = fail(DJB_ERR_IO, "write failed: %s", path);
    }
    if (std::fclose(fp) != 0 && rc == DJB_OK) rc = fail(DJB_ERR_IO, "closing %s failed", path);
    if (rc != DJB_OK) std::remove(path);
    return rc;
}

int h5_write_floats(FILE* fp, const float* p, size_t count) {
    if (std::fwrite(p, sizeof(float), count, fp) != count) return fail(DJB_ERR_IO, "snapshot write failed");
    return DJB_OK;
}

}  // namespace djb

int djb_write_snapshot_h5(const char* path, const float* psi, const float* pi, int32_t n, double D, double L) {
    djb::clear_error();
    if (n <= 0) return djb::fail(DJB_ERR_INVALID, "n must be positive");
    if (!psi || !pi) return djb::fail(DJB_ERR_INVALID, "null array");
    const uint64_t nn = uint64_t(n);
    const std::vector<uint64_t> dims = {3, nn, nn, nn};
    const size_t count = size_t(3 * nn * nn * nn);
    const std::vector<djb::H5Array> arrays = {{"Psi", dims, 4}, {"Pi", dims, 4}};
    return djb::h5_write_arrays(path, arrays, {{"D", D}, {"L", L}}, [&](size_t i, FILE* fp) {
        return djb::h5_write_floats(fp, i == 0 ? psi : pi, count);
    });
}
