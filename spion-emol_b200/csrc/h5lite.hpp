// h5lite.hpp -- the subset of the HDF5 file format that the scattering
// path's input (preprocessing file) and output (dipole scan files) use,
// written from the public HDF5 file-format specification; no libhdf5.
//
// Writer: superblock version 0, symbol-table groups (version-1 B-tree of
// group nodes, symbol-table nodes, local heap), version-1 object headers,
// contiguous or chunked (deflate) datasets of little-endian f64 / i64 / i32,
// scalar attributes of f64 / i64 / fixed-length strings.  This is the layout
// libhdf5 writes with its default (earliest) file-format settings, which is
// what the reference's writers get.
//
// Reader: superblock versions 0 and 1, symbol-table groups, version-1
// object headers with continuation blocks, dataspace versions 1 and 2,
// datatypes fixed-point / floating-point / string, layout version 3
// (compact, contiguous, chunked with version-1 chunk B-trees), filters
// deflate, shuffle and fletcher32, attribute message versions 1 to 3.
// Anything else (version-2 object headers, new-style link groups, other
// filters or layouts) is reported as unsupported, never misread.
#pragma once

#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace h5lite {

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

enum class Kind { F64 = 0, I64 = 1, I32 = 2, STR = 3 };

// ------------------------------------------------------------------ writer
class Writer {
public:
    explicit Writer(std::string path);
    ~Writer();
    Writer(const Writer&) = delete;
    Writer& operator=(const Writer&) = delete;

    // Creates the group and any missing parents ("/a/b").
    void group(const std::string& path);
    // Row-major data of the given shape (dims empty: scalar).  gzip in 1..9
    // stores it chunked along the first dimension and deflated.
    void dataset(const std::string& path, Kind kind, const std::vector<uint64_t>& dims, const void* data,
                 int gzip = 0);
    void attr_f64(const std::string& obj, const std::string& name, double v);
    void attr_i64(const std::string& obj, const std::string& name, long long v);
    void attr_str(const std::string& obj, const std::string& name, const std::string& v);
    // Lays the file out and writes it; the writer is spent afterwards.
    void close();

    struct Attr {
        std::string name;
        Kind kind;
        std::vector<uint8_t> value;
    };
    struct Node {
        bool is_group = true;
        std::map<std::string, std::unique_ptr<Node>> children;   // byte order = strcmp order
        std::vector<Attr> attrs;
        Kind kind = Kind::F64;
        std::vector<uint64_t> dims;
        std::vector<uint8_t> data;
        int gzip = 0;
    };

private:
    Node* find(const std::string& path, bool create_groups, bool want_group);
    uint64_t emit(Node& n, std::vector<uint8_t>& out);

    std::string path_;
    Node root_;
    uint64_t root_btree_ = 0, root_heap_ = 0;   // cached in the superblock's root entry
    bool closed_ = false;
};

// ------------------------------------------------------------------ reader
struct DataInfo {
    Kind kind = Kind::F64;     // F64 for floating types, I64 for integers, STR
    int elem = 8;              // element size in bytes
    bool is_signed = true;
    bool is_float = true;
    std::vector<uint64_t> dims;
};

class Reader {
public:
    explicit Reader(const std::string& path);
    ~Reader();
    Reader(const Reader&) = delete;
    Reader& operator=(const Reader&) = delete;

    bool exists(const std::string& path) const;
    bool is_group(const std::string& path) const;
    std::vector<std::string> list(const std::string& group) const;
    DataInfo info(const std::string& path) const;
    std::vector<uint64_t> shape(const std::string& path) const { return info(path).dims; }
    // The block [start, start + count) of a dataset, converted, row-major.
    // Empty start/count: the whole dataset.
    void read_f64(const std::string& path, double* out, const std::vector<uint64_t>& start = {},
                  const std::vector<uint64_t>& count = {}) const;
    void read_i64(const std::string& path, long long* out, const std::vector<uint64_t>& start = {},
                  const std::vector<uint64_t>& count = {}) const;
    double scalar_f64(const std::string& path) const;
    long long scalar_i64(const std::string& path) const;

    bool has_attr(const std::string& obj, const std::string& name) const;
    double attr_f64(const std::string& obj, const std::string& name) const;
    long long attr_i64(const std::string& obj, const std::string& name) const;
    std::string attr_str(const std::string& obj, const std::string& name) const;

    // parsed object header (public for the implementation's helpers)
    struct Msg {
        uint16_t type;
        std::vector<uint8_t> body;
    };
    struct Object {
        std::vector<Msg> msgs;
    };
    struct Link {
        std::string name;
        uint64_t header;
    };

private:
    uint64_t resolve(const std::string& path) const;   // object header address; throws if absent
    bool try_resolve(const std::string& path, uint64_t* addr) const;
    Object object_at(uint64_t addr) const;
    std::vector<Link> group_links(const Object& o) const;
    void read_raw(uint64_t addr, void* dst, uint64_t n) const;
    void read_block(const std::string& path, void* out, bool as_float, const std::vector<uint64_t>& start,
                    const std::vector<uint64_t>& count) const;

    std::FILE* f_ = nullptr;
    uint64_t root_ = 0;
    uint64_t base_ = 0;
    std::string path_;
    mutable std::map<uint64_t, Object> cache_;
};

}  // namespace h5lite
