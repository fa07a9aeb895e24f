// psi_store.cpp -- the on-disk psi store of the reference's back-propagation,
// the files the continuum-continuum dipole driver reads
// (src/scatt/BackPropagator.cpp:27-101, :255-283, :700-745 with the
// PotentialStorage layout of src/scatt/PotentialStorage.cpp:31-35,
// :556-631, :1542-1566), written from psi(n) as scatt_psi_sweep returns it
// and read back.  Host-only.
//
// A store is a directory holding
//   pot_chunk_<c>.bin  int32 count, then count psi matrices (N_psi x N_psi,
//                      column-major doubles), chunk_size per file but the last
//   metadata.bin       the unversioned layout of full (not symmetric-packed)
//                      stores: size_t n_points, int32 N_psi, int32 chunk_size,
//                      int32 chunks
//   psi_asym.bin       (when n_asym > 0) 'PSI_ASYM', int32 version 1, int32
//                      n_asym, int32 asym_offset, int32 N_psi, 8 reserved
//                      bytes, then n_asym matrices
//   manifest.txt       the reference's manifest line ("kind=psi energy=...")
//   __SUCCESS__        empty, written last: its presence certifies the store
// Files are written under a temporary name and renamed into place.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"

namespace fs = std::filesystem;

namespace scatt {
namespace {

struct StoreError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

std::string fmt6(double v) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.6f", v);
    return b;
}

std::string manifest_of(const scatt_psi_store_meta& m) {
    return "kind=psi energy=" + fmt6(m.energy) + " Nr=" + std::to_string(m.n_grid) + " dr=" + fmt6(m.dr) +
           " Npsi=" + std::to_string(m.n_psi) + " Nf=" + std::to_string(m.n_f) + " l_cont=" +
           std::to_string(m.l_cont) + " l_exch=" + std::to_string(m.l_exch) + " n_occ=" + std::to_string(m.n_occ) +
           " n_trans=" + std::to_string(m.n_transition) + " keep=" + std::to_string(m.keep_lo) + ".." +
           std::to_string(m.keep_hi);
}

void put(std::ofstream& f, const void* p, size_t n) {
    f.write(static_cast<const char*>(p), (std::streamsize)n);
}

// write through a temporary name, then rename into place
template <class F>
void atomic_write(const fs::path& path, F body) {
    const fs::path tmp = path.string() + ".tmp";
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f) throw StoreError("cannot write " + tmp.string());
        body(f);
        if (!f) throw StoreError("short write to " + tmp.string());
    }
    fs::rename(tmp, path);
}

template <class F>
int store_guarded(const char* who, F f) {
    try {
        return f();
    } catch (const StoreError& e) {
        set_last_error(std::string(who) + ": " + e.what());
        return SCATT_ERR_IO;
    } catch (const fs::filesystem_error& e) {
        set_last_error(std::string(who) + ": " + e.what());
        return SCATT_ERR_IO;
    } catch (const std::bad_alloc&) {
        set_last_error(std::string(who) + ": host allocation failed");
        return SCATT_ERR_OOM;
    }
}

}  // namespace
}  // namespace scatt

using namespace scatt;

struct scatt_psi_store {
    fs::path dir;
    uint64_t n_points = 0;
    int32_t n_psi = 0, chunk_size = 0, chunks = 0;
    int32_t n_asym = 0, asym_offset = 0;
    std::string manifest;
};

extern "C" {

int scatt_psi_store_dirname(const scatt_psi_store_meta* m, char* buf, int cap) {
    if (!m || !buf || cap < 1) return SCATT_ERR_ARG;
    const std::string s = "psi_Nr" + std::to_string(m->n_grid) + "_Npsi" + std::to_string(m->n_psi) + "_E" +
                          fmt6(m->energy) + "_lc" + std::to_string(m->l_cont) + "_keep" + std::to_string(m->keep_lo) +
                          "-" + std::to_string(m->keep_hi);
    if ((int)s.size() + 1 > cap) {
        set_last_error("scatt_psi_store_dirname: buffer too small");
        return SCATT_ERR_ARG;
    }
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return SCATT_OK;
}

int scatt_psi_store_write(const char* dir, const scatt_psi_store_meta* m, const double* psi, int ld,
                          const double* psi_asym, int ld_asym) {
    if (!dir || !m || !psi || m->n_psi < 1 || ld < m->n_psi || m->keep_hi < m->keep_lo || m->keep_lo < 0 ||
        m->chunk_size < 1 || m->n_asym < 0 || (m->n_asym > 0 && (!psi_asym || ld_asym < m->n_psi))) {
        set_last_error("scatt_psi_store_write: need a directory, N_psi >= 1, ld >= N_psi, keep_lo <= keep_hi, "
                       "chunk_size >= 1 and the asymptotic matrices when n_asym > 0");
        return SCATT_ERR_ARG;
    }
    return store_guarded("scatt_psi_store_write", [&]() {
        const fs::path d(dir);
        fs::create_directories(d);
        fs::remove(d / "__SUCCESS__");              // an unfinished rewrite is no store
        const int np = m->n_psi;
        const int64_t n_points = (int64_t)m->keep_hi - m->keep_lo + 1;
        const int32_t chunks = (int32_t)((n_points + m->chunk_size - 1) / m->chunk_size);
        std::vector<double> mat((size_t)np * np);
        auto pack = [&](const double* src, int l) {
            for (int c = 0; c < np; ++c) std::memcpy(mat.data() + (size_t)c * np, src + (size_t)c * l, np * sizeof(double));
        };
        for (int32_t c = 0; c < chunks; ++c) {
            const int64_t first = (int64_t)c * m->chunk_size;
            const int32_t count = (int32_t)std::min<int64_t>(m->chunk_size, n_points - first);
            atomic_write(d / ("pot_chunk_" + std::to_string(c) + ".bin"), [&](std::ofstream& f) {
                put(f, &count, sizeof(count));
                for (int32_t i = 0; i < count; ++i) {
                    pack(psi + (size_t)(first + i) * ld * ld, ld);
                    put(f, mat.data(), mat.size() * sizeof(double));
                }
            });
        }
        atomic_write(d / "metadata.bin", [&](std::ofstream& f) {
            const uint64_t n = (uint64_t)n_points;
            const int32_t ch = np, cs = m->chunk_size;
            put(f, &n, sizeof(n));
            put(f, &ch, sizeof(ch));
            put(f, &cs, sizeof(cs));
            put(f, &chunks, sizeof(chunks));
        });
        if (m->n_asym > 0) {
            atomic_write(d / "psi_asym.bin", [&](std::ofstream& f) {
                const char magic[8] = {'P', 'S', 'I', '_', 'A', 'S', 'Y', 'M'};
                const int32_t head[4] = {1, m->n_asym, m->asym_offset, np};
                const int64_t reserved = 0;
                put(f, magic, 8);
                put(f, head, sizeof(head));
                put(f, &reserved, sizeof(reserved));
                for (int i = 0; i < m->n_asym; ++i) {
                    pack(psi_asym + (size_t)i * ld_asym * ld_asym, ld_asym);
                    put(f, mat.data(), mat.size() * sizeof(double));
                }
            });
        }
        atomic_write(d / "manifest.txt", [&](std::ofstream& f) { f << manifest_of(*m); });
        atomic_write(d / "__SUCCESS__", [](std::ofstream&) {});
        return SCATT_OK;
    });
}

int scatt_psi_store_open(const char* dir, scatt_psi_store** out) {
    if (!dir || !out) return SCATT_ERR_ARG;
    *out = nullptr;
    return store_guarded("scatt_psi_store_open", [&]() {
        auto h = std::make_unique<scatt_psi_store>();
        h->dir = dir;
        if (!fs::exists(h->dir / "__SUCCESS__")) throw StoreError("no __SUCCESS__ marker in " + h->dir.string());
        std::ifstream f(h->dir / "metadata.bin", std::ios::binary);
        if (!f) throw StoreError("no metadata.bin in " + h->dir.string());
        int32_t first = 0;
        f.read(reinterpret_cast<char*>(&first), 4);
        if (first == 0x53594D4D) throw StoreError("symmetric-packed store: not a psi store");
        f.seekg(0);
        f.read(reinterpret_cast<char*>(&h->n_points), 8);
        f.read(reinterpret_cast<char*>(&h->n_psi), 4);
        f.read(reinterpret_cast<char*>(&h->chunk_size), 4);
        f.read(reinterpret_cast<char*>(&h->chunks), 4);
        if (!f || h->n_psi < 1 || h->chunk_size < 1) throw StoreError("bad metadata.bin in " + h->dir.string());
        std::ifstream mf(h->dir / "manifest.txt");
        std::stringstream ss;
        ss << mf.rdbuf();
        h->manifest = ss.str();
        std::ifstream a(h->dir / "psi_asym.bin", std::ios::binary);
        if (a) {
            char magic[8];
            int32_t head[4];
            a.read(magic, 8);
            a.read(reinterpret_cast<char*>(head), sizeof(head));
            if (!a || std::memcmp(magic, "PSI_ASYM", 8) != 0 || head[0] != 1 || head[3] != h->n_psi)
                throw StoreError("bad psi_asym.bin in " + h->dir.string());
            h->n_asym = head[1];
            h->asym_offset = head[2];
        }
        *out = h.release();
        return SCATT_OK;
    });
}

int scatt_psi_store_info(scatt_psi_store* h, long long* out6) {
    if (!h || !out6) return SCATT_ERR_ARG;
    out6[0] = (long long)h->n_points;
    out6[1] = h->n_psi;
    out6[2] = h->chunk_size;
    out6[3] = h->chunks;
    out6[4] = h->n_asym;
    out6[5] = h->asym_offset;
    return SCATT_OK;
}

int scatt_psi_store_manifest(scatt_psi_store* h, char* buf, int cap) {
    if (!h || !buf || cap < (int)h->manifest.size() + 1) return SCATT_ERR_ARG;
    std::memcpy(buf, h->manifest.c_str(), h->manifest.size() + 1);
    return SCATT_OK;
}

int scatt_psi_store_read(scatt_psi_store* h, long long first, long long count, double* out) {
    if (!h || !out || first < 0 || count < 0 || (uint64_t)(first + count) > h->n_points) return SCATT_ERR_ARG;
    return store_guarded("scatt_psi_store_read", [&]() {
        const size_t mb = (size_t)h->n_psi * h->n_psi * sizeof(double);
        for (long long i = 0; i < count;) {
            const long long n = first + i;
            const int c = (int)(n / h->chunk_size);
            const long long in_chunk = n - (long long)c * h->chunk_size;
            std::ifstream f(h->dir / ("pot_chunk_" + std::to_string(c) + ".bin"), std::ios::binary);
            int32_t cnt = 0;
            f.read(reinterpret_cast<char*>(&cnt), 4);
            if (!f || in_chunk >= cnt) throw StoreError("chunk " + std::to_string(c) + " is short");
            const long long take = std::min<long long>(count - i, cnt - in_chunk);
            f.seekg((std::streamoff)(4 + in_chunk * (long long)mb));
            f.read(reinterpret_cast<char*>(out + (size_t)i * h->n_psi * h->n_psi), (std::streamsize)(take * mb));
            if (!f) throw StoreError("chunk " + std::to_string(c) + " is short");
            i += take;
        }
        return SCATT_OK;
    });
}

int scatt_psi_store_read_asym(scatt_psi_store* h, double* out) {
    if (!h || !out) return SCATT_ERR_ARG;
    return store_guarded("scatt_psi_store_read_asym", [&]() {
        if (h->n_asym <= 0) return SCATT_OK;
        std::ifstream a(h->dir / "psi_asym.bin", std::ios::binary);
        a.seekg(32);
        a.read(reinterpret_cast<char*>(out), (std::streamsize)((size_t)h->n_asym * h->n_psi * h->n_psi * sizeof(double)));
        if (!a) throw StoreError("psi_asym.bin is short");
        return SCATT_OK;
    });
}

int scatt_psi_store_close(scatt_psi_store* h) {
    delete h;
    return SCATT_OK;
}

}  // extern "C"
