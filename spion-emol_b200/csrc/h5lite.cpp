// h5lite.cpp -- see h5lite.hpp.  Structure layouts follow the public HDF5
// file-format specification (superblock v0/v1, object header v1, local heap,
// B-tree v1, symbol-table node, the header messages named below).
#include "h5lite.hpp"

#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <functional>

namespace h5lite {

namespace {

constexpr uint64_t UNDEF = ~0ull;
constexpr int GROUP_LEAF_K = 4;        // symbol-table nodes hold 2K = 8 links
constexpr int GROUP_NODE_K = 16;       // group B-tree nodes hold 2K = 32 children
constexpr int CHUNK_K = 32;            // chunk B-tree nodes hold 2K = 64 chunks
const uint8_t SIGNATURE[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

// message types
constexpr uint16_t M_NIL = 0x0000, M_DATASPACE = 0x0001, M_LINFO = 0x0002, M_DTYPE = 0x0003,
                   M_LINK = 0x0006, M_LAYOUT = 0x0008, M_FILTER = 0x000B, M_ATTR = 0x000C,
                   M_CONT = 0x0010, M_STAB = 0x0011, M_FILL = 0x0005;

void put(std::vector<uint8_t>& b, uint64_t v, int n) {
    for (int i = 0; i < n; ++i) b.push_back(static_cast<uint8_t>(v >> (8 * i)));
}
void pad8(std::vector<uint8_t>& b) {
    while (b.size() % 8) b.push_back(0);
}
uint64_t get(const uint8_t* p, int n) {
    uint64_t v = 0;
    for (int i = 0; i < n; ++i) v |= static_cast<uint64_t>(p[i]) << (8 * i);
    return v;
}
size_t elem_size(Kind k) { return k == Kind::I32 ? 4 : k == Kind::STR ? 1 : 8; }

std::vector<uint8_t> dtype_body(Kind k, size_t str_len = 0) {
    std::vector<uint8_t> b;
    switch (k) {
        case Kind::F64:
            // class 1 (floating point), version 1; little endian, implied msb
            // mantissa normalisation, sign at bit 63; IEEE double layout
            b = {0x11, 0x20, 0x3f, 0x00};
            put(b, 8, 4);
            put(b, 0, 2);
            put(b, 64, 2);
            b.push_back(52);
            b.push_back(11);
            b.push_back(0);
            b.push_back(52);
            put(b, 1023, 4);
            break;
        case Kind::I64:
        case Kind::I32:
            // class 0 (fixed point), version 1; little endian, signed
            b = {0x10, 0x08, 0x00, 0x00};
            put(b, elem_size(k), 4);
            put(b, 0, 2);
            put(b, 8 * elem_size(k), 2);
            break;
        case Kind::STR:
            // class 3 (string), version 1; null padded, ASCII
            b = {0x13, 0x01, 0x00, 0x00};
            put(b, str_len, 4);
            break;
    }
    return b;
}

std::vector<uint8_t> dspace_body(const std::vector<uint64_t>& dims) {
    std::vector<uint8_t> b = {1, static_cast<uint8_t>(dims.size()), 0, 0, 0, 0, 0, 0};
    for (uint64_t d : dims) put(b, d, 8);
    return b;
}

struct MsgOut {
    uint16_t type;
    std::vector<uint8_t> body;
};

// Appends a version-1 object header holding `msgs`; returns its address.
uint64_t put_header(std::vector<uint8_t>& out, std::vector<MsgOut> msgs) {
    pad8(out);
    const uint64_t at = out.size();
    uint64_t size = 0;
    for (auto& m : msgs) {
        pad8(m.body);
        size += 8 + m.body.size();
    }
    out.push_back(1);                      // version
    out.push_back(0);
    put(out, msgs.size(), 2);
    put(out, 1, 4);                        // reference count
    put(out, size, 4);
    put(out, 0, 4);                        // messages start 8-byte aligned
    for (auto& m : msgs) {
        put(out, m.type, 2);
        put(out, m.body.size(), 2);
        put(out, 0, 4);                    // flags + reserved
        out.insert(out.end(), m.body.begin(), m.body.end());
    }
    return at;
}

MsgOut attr_msg(const Writer::Attr& a) {
    const std::vector<uint8_t> dt = dtype_body(a.kind, a.kind == Kind::STR ? a.value.size() : 0);
    const std::vector<uint8_t> ds = dspace_body({});
    std::vector<uint8_t> b = {1, 0};
    put(b, a.name.size() + 1, 2);
    put(b, dt.size(), 2);
    put(b, ds.size(), 2);
    b.insert(b.end(), a.name.begin(), a.name.end());
    b.push_back(0);
    pad8(b);
    b.insert(b.end(), dt.begin(), dt.end());
    pad8(b);
    b.insert(b.end(), ds.begin(), ds.end());
    pad8(b);
    b.insert(b.end(), a.value.begin(), a.value.end());
    return MsgOut{M_ATTR, b};
}

std::vector<std::string> split_path(const std::string& p) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < p.size()) {
        while (i < p.size() && p[i] == '/') ++i;
        size_t j = i;
        while (j < p.size() && p[j] != '/') ++j;
        if (j > i) out.push_back(p.substr(i, j - i));
        i = j;
    }
    return out;
}

}  // namespace

// ================================================================== Writer
Writer::Writer(std::string path) : path_(std::move(path)) {}

Writer::~Writer() = default;

Writer::Node* Writer::find(const std::string& path, bool create_groups, bool want_group) {
    Node* cur = &root_;
    const auto parts = split_path(path);
    for (size_t i = 0; i < parts.size(); ++i) {
        if (!cur->is_group) throw Error("h5: " + path + ": a dataset cannot hold links");
        auto it = cur->children.find(parts[i]);
        if (it == cur->children.end()) {
            if (!create_groups) throw Error("h5: " + path + " does not exist");
            it = cur->children.emplace(parts[i], std::make_unique<Node>()).first;
        }
        cur = it->second.get();
    }
    if (want_group && !cur->is_group) throw Error("h5: " + path + " is a dataset");
    return cur;
}

void Writer::group(const std::string& path) {
    if (closed_) throw Error("h5: writer closed");
    find(path, true, true);
}

void Writer::dataset(const std::string& path, Kind kind, const std::vector<uint64_t>& dims, const void* data,
                     int gzip) {
    if (closed_) throw Error("h5: writer closed");
    if (kind == Kind::STR) throw Error("h5: string datasets are not written");
    const auto parts = split_path(path);
    if (parts.empty()) throw Error("h5: empty dataset path");
    std::string parent;
    for (size_t i = 0; i + 1 < parts.size(); ++i) parent += "/" + parts[i];
    Node* g = find(parent, true, true);
    if (g->children.count(parts.back())) throw Error("h5: " + path + " exists");
    auto n = std::make_unique<Node>();
    n->is_group = false;
    n->kind = kind;
    n->dims = dims;
    uint64_t count = 1;
    for (uint64_t d : dims) count *= d;
    const size_t bytes = count * elem_size(kind);
    n->data.resize(bytes);
    if (bytes) std::memcpy(n->data.data(), data, bytes);
    n->gzip = (gzip >= 1 && gzip <= 9 && !dims.empty() && count > 0) ? gzip : 0;
    g->children.emplace(parts.back(), std::move(n));
}

void Writer::attr_f64(const std::string& obj, const std::string& name, double v) {
    Attr a{name, Kind::F64, std::vector<uint8_t>(8)};
    std::memcpy(a.value.data(), &v, 8);
    find(obj, false, false)->attrs.push_back(std::move(a));
}

void Writer::attr_i64(const std::string& obj, const std::string& name, long long v) {
    Attr a{name, Kind::I64, std::vector<uint8_t>(8)};
    std::memcpy(a.value.data(), &v, 8);
    find(obj, false, false)->attrs.push_back(std::move(a));
}

void Writer::attr_str(const std::string& obj, const std::string& name, const std::string& v) {
    // fixed-length, null padded; an empty string is stored as one null byte
    Attr a{name, Kind::STR, std::vector<uint8_t>(v.begin(), v.end())};
    if (a.value.empty()) a.value.push_back(0);
    find(obj, false, false)->attrs.push_back(std::move(a));
}

uint64_t Writer::emit(Node& n, std::vector<uint8_t>& out) {
    std::vector<MsgOut> msgs;
    if (!n.is_group) {
        const size_t esz = elem_size(n.kind);
        msgs.push_back({M_DATASPACE, dspace_body(n.dims)});
        msgs.push_back({M_DTYPE, dtype_body(n.kind)});
        if (!n.gzip) {
            pad8(out);
            const uint64_t addr = out.size();
            out.insert(out.end(), n.data.begin(), n.data.end());
            msgs.push_back({M_FILL, {2, 2, 2, 0}});     // late allocation, write if set, undefined
            std::vector<uint8_t> lay = {3, 1};          // version 3, contiguous
            put(lay, n.data.empty() ? UNDEF : addr, 8);
            put(lay, n.data.size(), 8);
            msgs.push_back({M_LAYOUT, lay});
        } else {
            // chunks of whole rows along the first dimension, at most 2K chunks
            const uint64_t rows = n.dims[0];
            const uint64_t row_bytes = n.data.size() / rows;
            uint64_t cr = std::min<uint64_t>(rows, std::max<uint64_t>(1, (1u << 20) / std::max<uint64_t>(row_bytes, 1)));
            cr = std::max<uint64_t>(cr, (rows + 2 * CHUNK_K - 1) / (2 * CHUNK_K));
            if (cr * row_bytes / esz > 0xffffffffull) throw Error("h5: chunk too large");
            const uint64_t nchunks = (rows + cr - 1) / cr;
            const int nd = static_cast<int>(n.dims.size()) + 1;
            std::vector<uint64_t> sizes(nchunks), addrs(nchunks);
            std::vector<uint8_t> chunk(cr * row_bytes), z;
            for (uint64_t c = 0; c < nchunks; ++c) {
                const uint64_t r0 = c * cr, r1 = std::min(rows, r0 + cr);
                std::fill(chunk.begin(), chunk.end(), 0);   // edge chunks are stored whole
                std::memcpy(chunk.data(), n.data.data() + r0 * row_bytes, (r1 - r0) * row_bytes);
                uLongf zl = compressBound(chunk.size());
                z.resize(zl);
                if (compress2(z.data(), &zl, chunk.data(), chunk.size(), n.gzip) != Z_OK)
                    throw Error("h5: deflate failed");
                pad8(out);
                addrs[c] = out.size();
                sizes[c] = zl;
                out.insert(out.end(), z.begin(), z.begin() + zl);
            }
            // one leaf node of the chunk B-tree (type 1)
            pad8(out);
            const uint64_t bt = out.size();
            const size_t key = 8 + 8 * nd;
            const size_t node_size = 24 + 2 * CHUNK_K * 8 + (2 * CHUNK_K + 1) * key;
            std::vector<uint8_t> node = {'T', 'R', 'E', 'E', 1, 0};
            put(node, nchunks, 2);
            put(node, UNDEF, 8);
            put(node, UNDEF, 8);
            for (uint64_t c = 0; c <= nchunks; ++c) {
                put(node, c < nchunks ? sizes[c] : 0, 4);
                put(node, 0, 4);                          // filter mask: every filter applied
                put(node, c * cr, 8);                     // chunk origin (rows)
                for (int d = 1; d < nd; ++d) put(node, 0, 8);
                if (c < nchunks) put(node, addrs[c], 8);
            }
            node.resize(node_size, 0);
            out.insert(out.end(), node.begin(), node.end());
            msgs.push_back({M_FILL, {2, 3, 2, 0}});     // incremental allocation
            std::vector<uint8_t> lay = {3, 2, static_cast<uint8_t>(nd)};
            put(lay, bt, 8);
            put(lay, cr, 4);
            for (size_t d = 1; d < n.dims.size(); ++d) put(lay, n.dims[d], 4);
            put(lay, esz, 4);
            msgs.push_back({M_LAYOUT, lay});
            // filter pipeline v1: deflate with the level as its one parameter
            std::vector<uint8_t> fp = {1, 1, 0, 0, 0, 0, 0, 0};
            put(fp, 1, 2);
            put(fp, 0, 2);
            put(fp, 0, 2);
            put(fp, 1, 2);
            put(fp, n.gzip, 4);
            put(fp, 0, 4);
            msgs.push_back({M_FILTER, fp});
        }
        for (auto& a : n.attrs) msgs.push_back(attr_msg(a));
        return put_header(out, std::move(msgs));
    }
    // group: children first, then the local heap, symbol-table nodes and B-tree
    std::vector<std::pair<const std::string*, uint64_t>> kids;
    for (auto& kv : n.children) kids.push_back({&kv.first, emit(*kv.second, out)});
    const size_t per_node = 2 * GROUP_LEAF_K;
    const size_t nsnod = std::max<size_t>(1, (kids.size() + per_node - 1) / per_node);
    if (nsnod > 2 * GROUP_NODE_K) throw Error("h5: more than 256 links in one group");
    std::vector<uint8_t> heap_data(8, 0);            // offset 0: the empty name
    std::vector<uint64_t> name_off(kids.size());
    for (size_t i = 0; i < kids.size(); ++i) {
        name_off[i] = heap_data.size();
        heap_data.insert(heap_data.end(), kids[i].first->begin(), kids[i].first->end());
        heap_data.push_back(0);
        pad8(heap_data);
    }
    pad8(out);
    const uint64_t heap = out.size();
    out.insert(out.end(), {'H', 'E', 'A', 'P', 0, 0, 0, 0});
    put(out, heap_data.size(), 8);
    put(out, 1, 8);                                   // free list: none
    put(out, heap + 32, 8);
    out.insert(out.end(), heap_data.begin(), heap_data.end());
    std::vector<uint64_t> snod_addr(nsnod), snod_last(nsnod, 0);
    for (size_t s = 0; s < nsnod; ++s) {
        pad8(out);
        snod_addr[s] = out.size();
        const size_t lo = s * per_node, hi = std::min(kids.size(), lo + per_node);
        std::vector<uint8_t> sn = {'S', 'N', 'O', 'D', 1, 0};
        put(sn, hi - lo, 2);
        for (size_t i = lo; i < hi; ++i) {
            put(sn, name_off[i], 8);
            put(sn, kids[i].second, 8);
            put(sn, 0, 4);                            // no cached scratch data
            put(sn, 0, 4);
            put(sn, 0, 8);
            put(sn, 0, 8);
        }
        sn.resize(8 + per_node * 40, 0);
        out.insert(out.end(), sn.begin(), sn.end());
        if (hi > lo) snod_last[s] = name_off[hi - 1];
    }
    pad8(out);
    const uint64_t bt = out.size();
    std::vector<uint8_t> node = {'T', 'R', 'E', 'E', 0, 0};
    const size_t used = kids.empty() ? 0 : nsnod;
    put(node, used, 2);
    put(node, UNDEF, 8);
    put(node, UNDEF, 8);
    put(node, 0, 8);                                  // key 0: the empty name
    for (size_t s = 0; s < used; ++s) {
        put(node, snod_addr[s], 8);
        put(node, snod_last[s], 8);                   // largest name in child s
    }
    node.resize(24 + 2 * GROUP_NODE_K * 8 + (2 * GROUP_NODE_K + 1) * 8, 0);
    out.insert(out.end(), node.begin(), node.end());
    std::vector<uint8_t> st;
    put(st, bt, 8);
    put(st, heap, 8);
    msgs.push_back({M_STAB, st});
    for (auto& a : n.attrs) msgs.push_back(attr_msg(a));
    const uint64_t hdr = put_header(out, std::move(msgs));
    if (&n == &root_) {
        root_btree_ = bt;
        root_heap_ = heap;
    }
    return hdr;
}

void Writer::close() {
    if (closed_) return;
    closed_ = true;
    std::vector<uint8_t> out(96, 0);
    const uint64_t root = emit(root_, out);
    pad8(out);
    std::vector<uint8_t> sb(SIGNATURE, SIGNATURE + 8);
    sb.insert(sb.end(), {0, 0, 0, 0, 0, 8, 8, 0});
    put(sb, GROUP_LEAF_K, 2);
    put(sb, GROUP_NODE_K, 2);
    put(sb, 0, 4);
    put(sb, 0, 8);                                    // base address
    put(sb, UNDEF, 8);                                // free-space info
    put(sb, out.size(), 8);                           // end of file
    put(sb, UNDEF, 8);                                // driver info
    put(sb, 0, 8);                                    // root entry: name offset
    put(sb, root, 8);
    put(sb, 1, 4);                                    // cached symbol table
    put(sb, 0, 4);
    put(sb, root_btree_, 8);
    put(sb, root_heap_, 8);
    std::copy(sb.begin(), sb.end(), out.begin());
    std::FILE* f = std::fopen(path_.c_str(), "wb");
    if (!f) throw Error("h5: cannot create " + path_);
    const size_t w = std::fwrite(out.data(), 1, out.size(), f);
    const int c = std::fclose(f);
    if (w != out.size() || c != 0) throw Error("h5: short write to " + path_);
}

// ================================================================== Reader
namespace {

struct Layout {
    int cls = 1;                       // 0 compact, 1 contiguous, 2 chunked
    uint64_t addr = UNDEF, size = 0;
    std::vector<uint8_t> compact;
    std::vector<uint64_t> chunk;       // chunk dims (rank entries)
};
struct Filter {
    int id;
    unsigned flags;
    std::vector<uint32_t> cv;
};

DataInfo parse_dtype(const std::vector<uint8_t>& b, const std::string& what) {
    if (b.size() < 8) throw Error("h5: " + what + ": short datatype");
    DataInfo d;
    const int cls = b[0] & 0x0f;
    d.elem = static_cast<int>(get(&b[4], 4));
    if (cls == 0) {
        if (b[1] & 0x01) throw Error("h5: " + what + ": big-endian integers unsupported");
        d.kind = Kind::I64;
        d.is_float = false;
        d.is_signed = (b[1] & 0x08) != 0;
        if (d.elem != 1 && d.elem != 2 && d.elem != 4 && d.elem != 8)
            throw Error("h5: " + what + ": integer size unsupported");
    } else if (cls == 1) {
        if (b[1] & 0x41) throw Error("h5: " + what + ": non little-endian floats unsupported");
        d.kind = Kind::F64;
        d.is_float = true;
        if (d.elem != 4 && d.elem != 8) throw Error("h5: " + what + ": float size unsupported");
    } else if (cls == 3) {
        d.kind = Kind::STR;
        d.is_float = false;
    } else {
        throw Error("h5: " + what + ": datatype class " + std::to_string(cls) + " unsupported");
    }
    return d;
}

std::vector<uint64_t> parse_dspace(const std::vector<uint8_t>& b, const std::string& what) {
    if (b.size() < 4) throw Error("h5: " + what + ": short dataspace");
    const int ver = b[0], rank = b[1];
    size_t at;
    if (ver == 1) at = 8;
    else if (ver == 2) {
        if (b[3] == 2) throw Error("h5: " + what + ": null dataspace");
        at = 4;
    } else throw Error("h5: " + what + ": dataspace version unsupported");
    if (b.size() < at + 8 * (size_t)rank) throw Error("h5: " + what + ": short dataspace");
    std::vector<uint64_t> dims(rank);
    for (int i = 0; i < rank; ++i) dims[i] = get(&b[at + 8 * i], 8);
    return dims;
}

// raw element -> double / int64
double to_f64(const uint8_t* p, const DataInfo& d) {
    if (d.is_float) {
        if (d.elem == 8) {
            double v;
            std::memcpy(&v, p, 8);
            return v;
        }
        float v;
        std::memcpy(&v, p, 4);
        return v;
    }
    const uint64_t u = get(p, d.elem);
    if (d.is_signed && d.elem < 8 && (u >> (8 * d.elem - 1)) & 1) return static_cast<double>(static_cast<int64_t>(u | (~0ull << (8 * d.elem))));
    return d.is_signed ? static_cast<double>(static_cast<int64_t>(u)) : static_cast<double>(u);
}
long long to_i64(const uint8_t* p, const DataInfo& d) {
    if (d.is_float) return static_cast<long long>(to_f64(p, d));
    const uint64_t u = get(p, d.elem);
    if (d.is_signed && d.elem < 8 && (u >> (8 * d.elem - 1)) & 1) return static_cast<long long>(u | (~0ull << (8 * d.elem)));
    return static_cast<long long>(u);
}

}  // namespace

Reader::Reader(const std::string& path) : path_(path) {
    f_ = std::fopen(path.c_str(), "rb");
    if (!f_) throw Error("h5: cannot open " + path);
    std::fseek(f_, 0, SEEK_END);
    const long long fsize = std::ftell(f_);
    // the superblock sits at 0 or after a user block of 512 * 2^k bytes
    uint64_t sb = UNDEF;
    for (uint64_t at = 0; at + 8 <= (uint64_t)fsize; at = at ? at * 2 : 512) {
        uint8_t sig[8];
        std::fseek(f_, (long)at, SEEK_SET);
        if (std::fread(sig, 1, 8, f_) == 8 && std::memcmp(sig, SIGNATURE, 8) == 0) {
            sb = at;
            break;
        }
    }
    if (sb == UNDEF) {
        std::fclose(f_);
        f_ = nullptr;
        throw Error("h5: " + path + " is not an HDF5 file");
    }
    uint8_t h[128];
    std::fseek(f_, (long)sb, SEEK_SET);
    const size_t got = std::fread(h, 1, sizeof(h), f_);
    const int ver = h[8];
    if (got < 100 || (ver != 0 && ver != 1) || h[13] != 8 || h[14] != 8) {
        std::fclose(f_);
        f_ = nullptr;
        throw Error("h5: " + path + ": superblock version " + std::to_string(ver) +
                    " or non-64-bit offsets unsupported");
    }
    const size_t a0 = ver == 0 ? 24 : 28;            // version 1 adds indexed-storage K + reserved
    base_ = get(&h[a0], 8);
    root_ = get(&h[a0 + 32 + 8], 8);                 // root entry: name offset, then header address
}

Reader::~Reader() {
    if (f_) std::fclose(f_);
}

void Reader::read_raw(uint64_t addr, void* dst, uint64_t n) const {
    if (n == 0) return;
    if (std::fseek(f_, (long)(base_ + addr), SEEK_SET) != 0 || std::fread(dst, 1, n, f_) != n)
        throw Error("h5: " + path_ + ": read past the end of the file");
}

Reader::Object Reader::object_at(uint64_t addr) const {
    auto it = cache_.find(addr);
    if (it != cache_.end()) return it->second;
    uint8_t pre[16];
    read_raw(addr, pre, 16);
    if (std::memcmp(pre, "OHDR", 4) == 0) throw Error("h5: " + path_ + ": version-2 object headers unsupported");
    if (pre[0] != 1) throw Error("h5: " + path_ + ": object header version unsupported");
    const int nmsgs = static_cast<int>(get(&pre[2], 2));
    Object o;
    std::vector<std::pair<uint64_t, uint64_t>> blocks = {{addr + 16, get(&pre[8], 4)}};
    int seen = 0;
    for (size_t bi = 0; bi < blocks.size() && seen < nmsgs; ++bi) {
        std::vector<uint8_t> buf(blocks[bi].second);
        read_raw(blocks[bi].first, buf.data(), buf.size());
        size_t p = 0;
        while (p + 8 <= buf.size() && seen < nmsgs) {
            const uint16_t type = static_cast<uint16_t>(get(&buf[p], 2));
            const size_t sz = get(&buf[p + 2], 2);
            if (p + 8 + sz > buf.size()) throw Error("h5: " + path_ + ": corrupt object header");
            std::vector<uint8_t> body(buf.begin() + p + 8, buf.begin() + p + 8 + sz);
            ++seen;
            if (type == M_CONT) blocks.push_back({get(&body[0], 8), get(&body[8], 8)});
            else if (type != M_NIL) o.msgs.push_back(Msg{type, std::move(body)});
            p += 8 + sz;
        }
    }
    cache_[addr] = o;
    return o;
}

std::vector<Reader::Link> Reader::group_links(const Object& o) const {
    const Msg* st = nullptr;
    for (auto& m : o.msgs) {
        if (m.type == M_STAB) st = &m;
        if (m.type == M_LINK || m.type == M_LINFO)
            throw Error("h5: " + path_ + ": link-message groups unsupported");
    }
    if (!st) throw Error("h5: not a group");
    const uint64_t bt = get(&st->body[0], 8), heap = get(&st->body[8], 8);
    uint8_t hh[32];
    read_raw(heap, hh, 32);
    if (std::memcmp(hh, "HEAP", 4) != 0) throw Error("h5: " + path_ + ": corrupt local heap");
    std::vector<uint8_t> names(get(&hh[8], 8));
    read_raw(get(&hh[24], 8), names.data(), names.size());
    std::vector<Link> out;
    std::function<void(uint64_t)> walk = [&](uint64_t node) {
        uint8_t nh[24];
        read_raw(node, nh, 24);
        if (std::memcmp(nh, "TREE", 4) != 0 || nh[4] != 0) throw Error("h5: " + path_ + ": corrupt group B-tree");
        const int level = nh[5], used = static_cast<int>(get(&nh[6], 2));
        std::vector<uint8_t> body(8 + 16 * (size_t)used);
        read_raw(node + 24, body.data(), body.size());
        for (int i = 0; i < used; ++i) {
            const uint64_t child = get(&body[8 + 16 * i], 8);
            if (level > 0) {
                walk(child);
                continue;
            }
            uint8_t sh[8];
            read_raw(child, sh, 8);
            if (std::memcmp(sh, "SNOD", 4) != 0) throw Error("h5: " + path_ + ": corrupt symbol-table node");
            const int n = static_cast<int>(get(&sh[6], 2));
            std::vector<uint8_t> ent(40 * (size_t)n);
            read_raw(child + 8, ent.data(), ent.size());
            for (int k = 0; k < n; ++k) {
                const uint64_t off = get(&ent[40 * k], 8);
                if (off >= names.size()) throw Error("h5: " + path_ + ": corrupt link name");
                out.push_back(Link{std::string(reinterpret_cast<const char*>(&names[off])), get(&ent[40 * k + 8], 8)});
            }
        }
    };
    walk(bt);
    return out;
}

bool Reader::try_resolve(const std::string& path, uint64_t* addr) const {
    uint64_t cur = root_;
    for (const auto& part : split_path(path)) {
        const Object o = object_at(cur);
        bool is_grp = false;
        for (auto& m : o.msgs) is_grp |= m.type == M_STAB;
        if (!is_grp) return false;
        bool found = false;
        for (const auto& l : group_links(o))
            if (l.name == part) {
                cur = l.header;
                found = true;
                break;
            }
        if (!found) return false;
    }
    *addr = cur;
    return true;
}

uint64_t Reader::resolve(const std::string& path) const {
    uint64_t a = 0;
    if (!try_resolve(path, &a)) throw Error("h5: " + path_ + ": no object " + path);
    return a;
}

bool Reader::exists(const std::string& path) const {
    uint64_t a;
    return try_resolve(path, &a);
}

bool Reader::is_group(const std::string& path) const {
    uint64_t a;
    if (!try_resolve(path, &a)) return false;
    for (auto& m : object_at(a).msgs)
        if (m.type == M_STAB) return true;
    return false;
}

std::vector<std::string> Reader::list(const std::string& group) const {
    std::vector<std::string> out;
    for (const auto& l : group_links(object_at(resolve(group)))) out.push_back(l.name);
    std::sort(out.begin(), out.end());
    return out;
}

DataInfo Reader::info(const std::string& path) const {
    const Object o = object_at(resolve(path));
    const Msg *ds = nullptr, *dt = nullptr;
    for (auto& m : o.msgs) {
        if (m.type == M_DATASPACE) ds = &m;
        if (m.type == M_DTYPE) dt = &m;
    }
    if (!ds || !dt) throw Error("h5: " + path + " is not a dataset");
    DataInfo d = parse_dtype(dt->body, path);
    d.dims = parse_dspace(ds->body, path);
    return d;
}

void Reader::read_block(const std::string& path, void* out, bool as_float, const std::vector<uint64_t>& start_in,
                        const std::vector<uint64_t>& count_in) const {
    const Object o = object_at(resolve(path));
    DataInfo d;
    Layout lay;
    std::vector<Filter> filters;
    bool have_ds = false, have_dt = false, have_lay = false;
    for (auto& m : o.msgs) {
        const auto& b = m.body;
        if (m.type == M_DATASPACE) { d.dims = parse_dspace(b, path); have_ds = true; }
        if (m.type == M_DTYPE) {
            auto dims = d.dims;
            d = parse_dtype(b, path);
            d.dims = dims;
            have_dt = true;
        }
        if (m.type == M_LAYOUT) {
            if (b.empty() || b[0] != 3) throw Error("h5: " + path + ": layout version unsupported");
            lay.cls = b[1];
            if (lay.cls == 0) {
                const size_t n = get(&b[2], 2);
                lay.compact.assign(b.begin() + 4, b.begin() + 4 + n);
            } else if (lay.cls == 1) {
                lay.addr = get(&b[2], 8);
                lay.size = get(&b[10], 8);
            } else if (lay.cls == 2) {
                const int nd = b[2];
                lay.addr = get(&b[3], 8);
                for (int i = 0; i + 1 < nd; ++i) lay.chunk.push_back(get(&b[11 + 4 * i], 4));
            } else {
                throw Error("h5: " + path + ": layout class unsupported");
            }
            have_lay = true;
        }
        if (m.type == M_FILTER) {
            const int ver = b[0], nf = b[1];
            size_t p = ver == 1 ? 8 : 2;
            for (int i = 0; i < nf; ++i) {
                Filter fl;
                fl.id = static_cast<int>(get(&b[p], 2));
                size_t name_len = 0;
                if (ver == 1 || fl.id >= 256) {
                    name_len = get(&b[p + 2], 2);
                    p += 4;
                } else {
                    p += 2;
                }
                fl.flags = static_cast<unsigned>(get(&b[p], 2));
                const int ncv = static_cast<int>(get(&b[p + 2], 2));
                p += 4;
                p += ver == 1 ? (name_len + 7) / 8 * 8 : name_len;
                for (int k = 0; k < ncv; ++k) fl.cv.push_back(static_cast<uint32_t>(get(&b[p + 4 * k], 4)));
                p += 4 * (size_t)ncv;
                if (ver == 1 && ncv % 2) p += 4;
                filters.push_back(fl);
            }
        }
    }
    if (!have_ds || !have_dt || !have_lay) throw Error("h5: " + path + " is not a dataset");
    if (d.kind == Kind::STR) throw Error("h5: " + path + ": string datasets are not read");
    for (const auto& fl : filters)
        if (fl.id != 1 && fl.id != 2 && fl.id != 3)
            throw Error("h5: " + path + ": filter " + std::to_string(fl.id) + " unsupported");
    const int rank = static_cast<int>(d.dims.size());
    std::vector<uint64_t> start = start_in, count = count_in;
    if (start.empty()) start.assign(rank, 0);
    if (count.empty()) count = d.dims;
    if ((int)start.size() != rank || (int)count.size() != rank) throw Error("h5: " + path + ": block rank mismatch");
    uint64_t total = 1;
    for (int i = 0; i < rank; ++i) {
        if (start[i] + count[i] > d.dims[i]) throw Error("h5: " + path + ": block outside the dataset");
        total *= count[i];
    }
    double* of = static_cast<double*>(out);
    long long* oi = static_cast<long long*>(out);
    auto put_elems = [&](uint64_t dst, const uint8_t* src, uint64_t n) {
        for (uint64_t k = 0; k < n; ++k) {
            if (as_float) of[dst + k] = to_f64(src + k * d.elem, d);
            else oi[dst + k] = to_i64(src + k * d.elem, d);
        }
    };
    if (total == 0) return;
    // row-major strides of the output block
    std::vector<uint64_t> ost(rank, 1);
    for (int i = rank - 2; i >= 0; --i) ost[i] = ost[i + 1] * count[i + 1];
    // copies the intersection of the block with the box [org, org + ext)
    // whose elements `fetch(offset_in_box, n, dst)` provides
    auto copy_box = [&](const std::vector<uint64_t>& org, const std::vector<uint64_t>& ext,
                        const std::function<void(uint64_t, uint64_t, uint8_t*)>& fetch) {
        if (rank == 0) {
            std::vector<uint8_t> e(d.elem);
            fetch(0, 1, e.data());
            put_elems(0, e.data(), 1);
            return;
        }
        std::vector<uint64_t> lo(rank), hi(rank), bst(rank, 1);
        for (int i = 0; i < rank; ++i) {
            lo[i] = std::max(start[i], org[i]);
            hi[i] = std::min({start[i] + count[i], org[i] + ext[i], d.dims[i]});
            if (lo[i] >= hi[i]) return;
        }
        for (int i = rank - 2; i >= 0; --i) bst[i] = bst[i + 1] * ext[i + 1];
        const uint64_t run = hi[rank - 1] - lo[rank - 1];
        std::vector<uint8_t> tmp(run * d.elem);
        std::vector<uint64_t> idx(lo);
        for (;;) {
            uint64_t src = 0, dst = 0;
            for (int i = 0; i < rank; ++i) {
                src += (idx[i] - org[i]) * bst[i];
                dst += (idx[i] - start[i]) * ost[i];
            }
            fetch(src, run, tmp.data());
            put_elems(dst, tmp.data(), run);
            int i = rank - 2;
            for (; i >= 0; --i) {
                if (++idx[i] < hi[i]) break;
                idx[i] = lo[i];
            }
            if (i < 0) break;
        }
    };
    const std::vector<uint64_t> zero(rank, 0);
    if (lay.cls == 0) {
        copy_box(zero, d.dims, [&](uint64_t off, uint64_t n, uint8_t* dst) {
            if ((off + n) * d.elem > lay.compact.size()) throw Error("h5: " + path + ": short compact data");
            std::memcpy(dst, lay.compact.data() + off * d.elem, n * d.elem);
        });
        return;
    }
    if (lay.cls == 1) {
        if (lay.addr == UNDEF) {            // never written: the fill value (zero)
            if (as_float) std::fill(of, of + total, 0.0);
            else std::fill(oi, oi + total, 0LL);
            return;
        }
        copy_box(zero, d.dims, [&](uint64_t off, uint64_t n, uint8_t* dst) {
            read_raw(lay.addr + off * d.elem, dst, n * d.elem);
        });
        return;
    }
    // chunked: chunks missing from the tree read as zero
    if (as_float) std::fill(of, of + total, 0.0);
    else std::fill(oi, oi + total, 0LL);
    if (lay.addr == UNDEF) return;
    if ((int)lay.chunk.size() != rank) throw Error("h5: " + path + ": chunk rank mismatch");
    uint64_t chunk_elems = 1;
    for (uint64_t c : lay.chunk) chunk_elems *= c;
    const uint64_t chunk_bytes = chunk_elems * d.elem;
    const size_t key = 8 + 8 * (size_t)(rank + 1);
    std::function<void(uint64_t)> walk = [&](uint64_t node) {
        uint8_t nh[24];
        read_raw(node, nh, 24);
        if (std::memcmp(nh, "TREE", 4) != 0 || nh[4] != 1) throw Error("h5: " + path + ": corrupt chunk B-tree");
        const int level = nh[5], used = static_cast<int>(get(&nh[6], 2));
        std::vector<uint8_t> body((size_t)used * (key + 8) + key);
        read_raw(node + 24, body.data(), body.size());
        for (int c = 0; c < used; ++c) {
            const uint8_t* k = &body[(size_t)c * (key + 8)];
            const uint64_t child = get(k + key, 8);
            if (level > 0) {
                walk(child);
                continue;
            }
            const uint64_t stored = get(k, 4);
            const uint32_t mask = static_cast<uint32_t>(get(k + 4, 4));
            std::vector<uint64_t> org(rank);
            bool hit = true;
            for (int i = 0; i < rank; ++i) {
                org[i] = get(k + 8 + 8 * i, 8);
                if (org[i] >= start[i] + count[i] || org[i] + lay.chunk[i] <= start[i]) hit = false;
            }
            if (!hit) continue;
            std::vector<uint8_t> raw(stored);
            read_raw(child, raw.data(), stored);
            for (int fi = (int)filters.size() - 1; fi >= 0; --fi) {
                if (mask & (1u << fi)) continue;
                const Filter& fl = filters[fi];
                if (fl.id == 3) {                 // fletcher32: drop the trailing checksum
                    if (raw.size() < 4) throw Error("h5: " + path + ": short chunk");
                    raw.resize(raw.size() - 4);
                } else if (fl.id == 1) {          // deflate
                    std::vector<uint8_t> z(chunk_bytes);
                    uLongf zl = chunk_bytes;
                    if (uncompress(z.data(), &zl, raw.data(), raw.size()) != Z_OK || zl != chunk_bytes)
                        throw Error("h5: " + path + ": inflate failed");
                    raw.swap(z);
                } else if (fl.id == 2) {          // shuffle: byte planes back to elements
                    const size_t es = fl.cv.empty() ? d.elem : fl.cv[0];
                    const size_t ne = raw.size() / es;
                    std::vector<uint8_t> z(raw.size());
                    for (size_t b = 0; b < es; ++b)
                        for (size_t e = 0; e < ne; ++e) z[e * es + b] = raw[b * ne + e];
                    std::copy(raw.begin() + ne * es, raw.end(), z.begin() + ne * es);
                    raw.swap(z);
                }
            }
            if (raw.size() < chunk_bytes) throw Error("h5: " + path + ": short chunk");
            copy_box(org, lay.chunk, [&](uint64_t off, uint64_t n, uint8_t* dst) {
                std::memcpy(dst, raw.data() + off * d.elem, n * d.elem);
            });
        }
    };
    walk(lay.addr);
}

void Reader::read_f64(const std::string& path, double* out, const std::vector<uint64_t>& start,
                      const std::vector<uint64_t>& count) const {
    read_block(path, out, true, start, count);
}

void Reader::read_i64(const std::string& path, long long* out, const std::vector<uint64_t>& start,
                      const std::vector<uint64_t>& count) const {
    read_block(path, out, false, start, count);
}

double Reader::scalar_f64(const std::string& path) const {
    const DataInfo d = info(path);
    uint64_t n = 1;
    for (uint64_t x : d.dims) n *= x;
    if (n != 1) throw Error("h5: " + path + " is not a scalar");
    double v = 0.0;
    read_f64(path, &v);
    return v;
}

long long Reader::scalar_i64(const std::string& path) const {
    const DataInfo d = info(path);
    uint64_t n = 1;
    for (uint64_t x : d.dims) n *= x;
    if (n != 1) throw Error("h5: " + path + " is not a scalar");
    long long v = 0;
    read_i64(path, &v);
    return v;
}

namespace {

struct AttrData {
    DataInfo dt;
    std::vector<uint8_t> value;
};

bool find_attr(const Reader::Object& o, const std::string& name, AttrData* out) {
    for (auto& m : o.msgs) {
        if (m.type != M_ATTR) continue;
        const auto& b = m.body;
        const int ver = b[0];
        const size_t nsz = get(&b[2], 2), tsz = get(&b[4], 2), ssz = get(&b[6], 2);
        size_t p = ver == 3 ? 9 : 8;
        auto adv = [&](size_t n) { return ver == 1 ? (n + 7) / 8 * 8 : n; };
        if (ver < 1 || ver > 3 || p + nsz > b.size()) continue;
        std::string nm(reinterpret_cast<const char*>(&b[p]), nsz ? nsz - 1 : 0);
        nm = nm.c_str();
        p += adv(nsz);
        if (nm != name) continue;
        std::vector<uint8_t> dt(b.begin() + p, b.begin() + p + tsz);
        p += adv(tsz);
        std::vector<uint8_t> ds(b.begin() + p, b.begin() + p + ssz);
        p += adv(ssz);
        out->dt = parse_dtype(dt, name);
        out->dt.dims = parse_dspace(ds, name);
        out->value.assign(b.begin() + std::min(p, b.size()), b.end());
        return true;
    }
    return false;
}

}  // namespace

bool Reader::has_attr(const std::string& obj, const std::string& name) const {
    AttrData a;
    return find_attr(object_at(resolve(obj)), name, &a);
}

double Reader::attr_f64(const std::string& obj, const std::string& name) const {
    AttrData a;
    if (!find_attr(object_at(resolve(obj)), name, &a)) throw Error("h5: no attribute " + obj + ":" + name);
    if (a.dt.kind == Kind::STR || a.value.size() < (size_t)a.dt.elem)
        throw Error("h5: attribute " + name + " is not numeric");
    return to_f64(a.value.data(), a.dt);
}

long long Reader::attr_i64(const std::string& obj, const std::string& name) const {
    AttrData a;
    if (!find_attr(object_at(resolve(obj)), name, &a)) throw Error("h5: no attribute " + obj + ":" + name);
    if (a.dt.kind == Kind::STR || a.value.size() < (size_t)a.dt.elem)
        throw Error("h5: attribute " + name + " is not numeric");
    return to_i64(a.value.data(), a.dt);
}

std::string Reader::attr_str(const std::string& obj, const std::string& name) const {
    AttrData a;
    if (!find_attr(object_at(resolve(obj)), name, &a)) throw Error("h5: no attribute " + obj + ":" + name);
    if (a.dt.kind != Kind::STR) throw Error("h5: attribute " + name + " is not a string");
    std::string s(a.value.begin(), a.value.begin() + std::min<size_t>(a.dt.elem, a.value.size()));
    while (!s.empty() && (s.back() == '\0' || s.back() == ' ')) s.pop_back();
    return s.c_str();
}

}  // namespace h5lite
