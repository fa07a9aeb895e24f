// io_capi.cpp -- extern "C" entry points of the file formats around the
// path: the HDF5 subset (h5lite), the dipole scan output of the reference's
// DipoleWriter (src/scatt/DipoleIO.cpp) and the preprocessing input of its
// HDF5Reader (src/io/HDF5Reader.hpp).  Host code only; no device work.
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "h5lite.hpp"
#include "scatt_b200.h"

namespace scatt {
void set_last_error(const std::string& msg);   // capi.cu
}

namespace fs = std::filesystem;
using scatt::set_last_error;

struct scatt_h5w {
    std::string path;
    std::unique_ptr<h5lite::Writer> w;
};

struct scatt_h5r {
    std::unique_ptr<h5lite::Reader> r;
};

struct scatt_preproc {
    std::unique_ptr<h5lite::Reader> orb;        // orbitals side (the one file when combined)
    std::unique_ptr<h5lite::Reader> pot_own;    // potentials side of the split layout
    bool split = false;
    int Nr = 0, Lmax_sce = 0, n_alpha = 0, n_occ_alpha = 0, n_sce = 0;
    int Lmax_orb_store = 0, Nlm_orb_store = 0, Nr_orb_store = 0;
    bool has_init = false, has_pol = false;
    double rmin = 0.0, dr = 0.0, E_init = 0.0, alpha_iso = 0.0;
    std::vector<double> orb_energies;
    std::vector<double> atoms;                  // n_atoms x 4: Z, x, y, z
    // buffers a desc points into
    std::vector<double> psi, vh;
};

namespace {

// runs f, turning exceptions into SCATT_ERR_IO (h5lite / filesystem) or
// SCATT_ERR_ARG with the message kept for scatt_last_error
template <class F>
int guarded(const char* who, F f) {
    try {
        return f();
    } catch (const h5lite::Error& e) {
        set_last_error(std::string(who) + ": " + e.what());
        return SCATT_ERR_IO;
    } catch (const fs::filesystem_error& e) {
        set_last_error(std::string(who) + ": " + e.what());
        return SCATT_ERR_IO;
    } catch (const std::bad_alloc&) {
        set_last_error(std::string(who) + ": host allocation failed");
        return SCATT_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(std::string(who) + ": " + e.what());
        return SCATT_ERR_ARG;
    }
}

std::vector<uint64_t> dims_of(int rank, const long long* d) {
    std::vector<uint64_t> v;
    for (int i = 0; i < rank; ++i) {
        if (d[i] < 0) throw std::invalid_argument("negative dimension");
        v.push_back(static_cast<uint64_t>(d[i]));
    }
    return v;
}

std::string pid_tmp(const std::string& path) {
    return path + ".tmp.pid" + std::to_string(static_cast<long long>(::getpid()));
}

// rename(tmp, path); success also when another process already put `path`
// in place (every writer of a scan writes the same content for a path)
void publish(const std::string& tmp, const std::string& path) {
    std::error_code ec;
    fs::rename(tmp, path, ec);
    if (ec) {
        std::error_code rm;
        fs::remove(tmp, rm);
        if (!fs::exists(path))
            throw h5lite::Error("cannot rename " + tmp + " -> " + path + ": " + ec.message());
    }
}

std::string tag_of(int ik) {
    std::string s = std::to_string(ik);
    while (s.size() < 4) s = "0" + s;
    return "ik" + s;
}

void check_meta(const scatt_dipole_meta* m) {
    if (!m) throw std::invalid_argument("meta is NULL");
    if (!(m->dk > 0.0)) throw std::invalid_argument("dk must be > 0");
    if (m->ik_min < 0) throw std::invalid_argument("ik_min < 0");
    if (m->ik_max <= m->ik_min) throw std::invalid_argument("ik_max <= ik_min");
    if (m->n_occ < 0 || m->n_atoms < 0) throw std::invalid_argument("negative count");
    if ((m->n_occ > 0 && (!m->occ_energies || !m->occ_spin_factors)) ||
        (m->n_atoms > 0 && (!m->Z || !m->xyz_bohr)))
        throw std::invalid_argument("NULL array with a positive count");
}

const char* str_or_empty(const char* s) { return s ? s : ""; }

void write_manifest(const std::string& dir, const scatt_dipole_meta* m) {
    const std::string path = dir + "/manifest.h5", tmp = pid_tmp(path);
    h5lite::Writer w(tmp);
    w.group("/grid");
    w.attr_f64("/grid", "r_min", m->r_min);
    w.attr_f64("/grid", "dr", m->dr);
    w.attr_i64("/grid", "N_grid", m->N_grid);
    w.attr_i64("/grid", "l_max_continuum", m->l_max_continuum);
    w.attr_f64("/grid", "E_HOMO", m->E_HOMO);
    w.group("/kgrid");
    w.attr_f64("/kgrid", "dk", m->dk);
    w.attr_i64("/kgrid", "ik_min", m->ik_min);
    w.attr_i64("/kgrid", "ik_max", m->ik_max);
    if (m->n_occ > 0) {
        w.dataset("/occ/energies", h5lite::Kind::F64, {(uint64_t)m->n_occ}, m->occ_energies);
        w.dataset("/occ/spin_factors", h5lite::Kind::F64, {(uint64_t)m->n_occ}, m->occ_spin_factors);
    }
    if (m->n_atoms > 0) {
        w.dataset("/atoms/Z", h5lite::Kind::I32, {(uint64_t)m->n_atoms}, m->Z);
        w.dataset("/atoms/xyz_bohr", h5lite::Kind::F64, {(uint64_t)m->n_atoms, 3}, m->xyz_bohr);
    }
    w.group("/conventions");
    w.attr_str("/conventions", "real_Ylm_q_map", "x=+1, y=-1, z=0");
    w.attr_str("/conventions", "psi_norm", "incoming-wave Psi- = (A - iB)^(-dagger)");
    w.attr_str("/conventions", "u_convention", "chi_lm(r) = r * F_lm(r)");
    w.attr_str("/conventions", "gauge_cross_section",
               "sigma^L = (4 pi^2 / c) omega Sum_mu |D^L|^2;  "
               "sigma^V = (4 pi^2 / c) (1/omega) Sum_mu |D^V|^2");
    w.group("/run");
    w.attr_str("/run", "molecule_name", str_or_empty(m->molecule_name));
    w.attr_str("/run", "git_hash", str_or_empty(m->git_hash));
    w.attr_str("/run", "iso_date_utc", str_or_empty(m->iso_date_utc));
    w.attr_str("/run", "psi_dir_prefix", str_or_empty(m->psi_dir_prefix));
    w.close();
    publish(tmp, path);
}

}  // namespace

extern "C" {

// ------------------------------------------------------------ HDF5 writer
int scatt_h5w_open(const char* path, scatt_h5w** out) {
    if (!path || !out) return SCATT_ERR_ARG;
    return guarded("scatt_h5w_open", [&]() {
        auto w = std::make_unique<h5lite::Writer>(pid_tmp(path));
        auto* h = new scatt_h5w();
        h->path = path;
        h->w = std::move(w);
        *out = h;
        return SCATT_OK;
    });
}

int scatt_h5w_group(scatt_h5w* h, const char* path) {
    if (!h || !path) return SCATT_ERR_ARG;
    return guarded("scatt_h5w_group", [&]() {
        h->w->group(path);
        return SCATT_OK;
    });
}

int scatt_h5w_dataset(scatt_h5w* h, const char* path, int kind, int rank, const long long* dims, const void* data,
                      int gzip) {
    if (!h || !path || kind < 0 || kind > 2 || rank < 0 || rank > 8 || (rank > 0 && !dims)) return SCATT_ERR_ARG;
    return guarded("scatt_h5w_dataset", [&]() {
        const auto d = dims_of(rank, dims);
        uint64_t n = 1;
        for (uint64_t x : d) n *= x;
        if (n > 0 && !data) throw std::invalid_argument("data is NULL");
        h->w->dataset(path, static_cast<h5lite::Kind>(kind), d, data, gzip);
        return SCATT_OK;
    });
}

int scatt_h5w_attr_f64(scatt_h5w* h, const char* obj, const char* name, double v) {
    if (!h || !obj || !name) return SCATT_ERR_ARG;
    return guarded("scatt_h5w_attr_f64", [&]() {
        h->w->attr_f64(obj, name, v);
        return SCATT_OK;
    });
}

int scatt_h5w_attr_i64(scatt_h5w* h, const char* obj, const char* name, long long v) {
    if (!h || !obj || !name) return SCATT_ERR_ARG;
    return guarded("scatt_h5w_attr_i64", [&]() {
        h->w->attr_i64(obj, name, v);
        return SCATT_OK;
    });
}

int scatt_h5w_attr_str(scatt_h5w* h, const char* obj, const char* name, const char* v) {
    if (!h || !obj || !name || !v) return SCATT_ERR_ARG;
    return guarded("scatt_h5w_attr_str", [&]() {
        h->w->attr_str(obj, name, v);
        return SCATT_OK;
    });
}

int scatt_h5w_close(scatt_h5w* h, int keep) {
    if (!h) return SCATT_ERR_ARG;
    const int st = guarded("scatt_h5w_close", [&]() {
        if (keep) {
            h->w->close();
            publish(pid_tmp(h->path), h->path);
        }
        return SCATT_OK;
    });
    delete h;
    return st;
}

// ------------------------------------------------------------ HDF5 reader
int scatt_h5r_open(const char* path, scatt_h5r** out) {
    if (!path || !out) return SCATT_ERR_ARG;
    return guarded("scatt_h5r_open", [&]() {
        auto r = std::make_unique<h5lite::Reader>(path);
        auto* h = new scatt_h5r();
        h->r = std::move(r);
        *out = h;
        return SCATT_OK;
    });
}

int scatt_h5r_kind(scatt_h5r* h, const char* path, int* kind) {
    if (!h || !path || !kind) return SCATT_ERR_ARG;
    return guarded("scatt_h5r_kind", [&]() {
        *kind = !h->r->exists(path) ? 0 : h->r->is_group(path) ? 1 : 2;
        return SCATT_OK;
    });
}

int scatt_h5r_shape(scatt_h5r* h, const char* path, int* rank, long long* dims8, int* elem_kind) {
    if (!h || !path || !rank) return SCATT_ERR_ARG;
    return guarded("scatt_h5r_shape", [&]() {
        const h5lite::DataInfo d = h->r->info(path);
        if (d.dims.size() > 8) throw h5lite::Error(std::string(path) + ": rank above 8");
        *rank = static_cast<int>(d.dims.size());
        for (size_t i = 0; i < d.dims.size() && dims8; ++i) dims8[i] = static_cast<long long>(d.dims[i]);
        if (elem_kind) *elem_kind = d.kind == h5lite::Kind::STR ? 3 : d.is_float ? 0 : 1;
        return SCATT_OK;
    });
}

int scatt_h5r_read(scatt_h5r* h, const char* path, int as_int, int rank, const long long* start,
                   const long long* count, void* out) {
    if (!h || !path || !out || rank < 0 || rank > 8) return SCATT_ERR_ARG;
    return guarded("scatt_h5r_read", [&]() {
        std::vector<uint64_t> s, c;
        if (start && count) {
            s = dims_of(rank, start);
            c = dims_of(rank, count);
        }
        if (as_int) h->r->read_i64(path, static_cast<long long*>(out), s, c);
        else h->r->read_f64(path, static_cast<double*>(out), s, c);
        return SCATT_OK;
    });
}

int scatt_h5r_list(scatt_h5r* h, const char* group, char* buf, long long cap, long long* needed) {
    if (!h || !group) return SCATT_ERR_ARG;
    return guarded("scatt_h5r_list", [&]() {
        std::string s;
        for (const auto& n : h->r->list(group)) s += n + "\n";
        if (needed) *needed = static_cast<long long>(s.size() + 1);
        if (buf && cap > 0) {
            const size_t n = std::min<size_t>(s.size(), static_cast<size_t>(cap - 1));
            std::memcpy(buf, s.data(), n);
            buf[n] = 0;
        }
        return SCATT_OK;
    });
}

int scatt_h5r_attr(scatt_h5r* h, const char* obj, const char* name, int* kind, double* f, long long* i, char* s,
                   long long cap) {
    if (!h || !obj || !name || !kind) return SCATT_ERR_ARG;
    return guarded("scatt_h5r_attr", [&]() {
        *kind = 0;
        if (!h->r->exists(obj) || !h->r->has_attr(obj, name)) return SCATT_OK;
        try {
            const std::string v = h->r->attr_str(obj, name);
            *kind = 3;
            if (s && cap > 0) {
                const size_t n = std::min<size_t>(v.size(), static_cast<size_t>(cap - 1));
                std::memcpy(s, v.data(), n);
                s[n] = 0;
            }
            return SCATT_OK;
        } catch (const h5lite::Error&) {
        }
        const double fv = h->r->attr_f64(obj, name);
        const long long iv = h->r->attr_i64(obj, name);
        *kind = (static_cast<double>(iv) == fv && std::floor(fv) == fv) ? 2 : 1;
        if (f) *f = fv;
        if (i) *i = iv;
        return SCATT_OK;
    });
}

int scatt_h5r_close(scatt_h5r* h) {
    delete h;
    return SCATT_OK;
}

// ------------------------------------------------------------ dipole scan output
int scatt_dipole_open(const char* scan_dir, const scatt_dipole_meta* meta) {
    if (!scan_dir) return SCATT_ERR_ARG;
    return guarded("scatt_dipole_open", [&]() {
        check_meta(meta);
        fs::create_directories(scan_dir);
        // an existing manifest is a resumed scan: kept as it is
        if (!fs::exists(std::string(scan_dir) + "/manifest.h5")) write_manifest(scan_dir, meta);
        return SCATT_OK;
    });
}

int scatt_dipole_has_energy(const char* scan_dir, int ik, int* has) {
    if (!scan_dir || !has || ik < 0) return SCATT_ERR_ARG;
    *has = fs::exists(std::string(scan_dir) + "/" + tag_of(ik) + ".h5") ? 1 : 0;
    return SCATT_OK;
}

int scatt_dipole_write_energy(const char* scan_dir, const scatt_dipole_meta* meta, const scatt_dipole_energy* e) {
    if (!scan_dir || !e) return SCATT_ERR_ARG;
    return guarded("scatt_dipole_write_energy", [&]() {
        check_meta(meta);
        if (e->ik < 0 || e->n_ch <= 0 || e->n_occ < 0) throw std::invalid_argument("bad ik / sizes");
        if (!e->A || !e->B || !e->D_re || !e->D_im || !e->Draw_re || !e->Draw_im || !e->d_raw ||
            !e->partial_sigma || (e->n_occ > 0 && (!e->b_overlap || !e->d_corr)))
            throw std::invalid_argument("NULL payload array");
        const uint64_t n = e->n_ch, no = e->n_occ;
        const std::string path = std::string(scan_dir) + "/" + tag_of(e->ik) + ".h5", tmp = pid_tmp(path);
        const double k = e->ik * meta->dk, E = 0.5 * k * k;
        h5lite::Writer w(tmp);
        w.group("/meta");
        w.attr_i64("/meta", "ik", e->ik);
        w.attr_f64("/meta", "k", k);
        w.attr_f64("/meta", "E", E);
        w.attr_f64("/meta", "omega", E - meta->E_HOMO);
        w.attr_f64("/meta", "fit_residual_rel", e->fit_residual_rel);
        w.attr_f64("/meta", "K_symmetry_err", e->K_symmetry_err);
        w.dataset("/A", h5lite::Kind::F64, {n, n}, e->A);
        w.dataset("/B", h5lite::Kind::F64, {n, n}, e->B);
        std::vector<double> empty;
        w.dataset("/b_overlap", h5lite::Kind::F64, {n, no}, no ? e->b_overlap : empty.data());
        const char* gauges[2] = {"length", "velocity"};
        const char* pols[3] = {"x", "y", "z"};
        w.group("/dipole");
        for (int s = 0; s < 6; ++s) {
            const std::string g = std::string("/dipole/") + gauges[s / 3] + "/" + pols[s % 3];
            w.group(g);
            w.dataset(g + "/D_ortho_re", h5lite::Kind::F64, {n}, e->D_re + s * n);
            w.dataset(g + "/D_ortho_im", h5lite::Kind::F64, {n}, e->D_im + s * n);
            w.dataset(g + "/D_raw_re", h5lite::Kind::F64, {n}, e->Draw_re + s * n);
            w.dataset(g + "/D_raw_im", h5lite::Kind::F64, {n}, e->Draw_im + s * n);
            w.dataset(g + "/d_raw", h5lite::Kind::F64, {n}, e->d_raw + s * n);
            w.dataset(g + "/d_correction", h5lite::Kind::F64, {no}, no ? e->d_corr + s * no : empty.data());
            w.attr_f64(g, "partial_sigma", e->partial_sigma[s]);
        }
        w.close();
        publish(tmp, path);
        return SCATT_OK;
    });
}

int scatt_dipole_finalize(const char* scan_dir) {
    if (!scan_dir) return SCATT_ERR_ARG;
    return guarded("scatt_dipole_finalize", [&]() {
        std::ofstream f(std::string(scan_dir) + "/__SUCCESS__");
        if (!f) throw h5lite::Error(std::string("cannot write ") + scan_dir + "/__SUCCESS__");
        return SCATT_OK;
    });
}

// ------------------------------------------------------------ preprocessing input
int scatt_preproc_open(const char* path, scatt_preproc** out) {
    if (!path || !out) return SCATT_ERR_ARG;
    return guarded("scatt_preproc_open", [&]() {
        auto p = std::make_unique<scatt_preproc>();
        const std::string s = path, ORB = ".orbitals.h5", POT = ".potentials.h5";
        auto ends = [&](const std::string& suf) {
            return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
        };
        std::string orb, pot;
        if (ends(ORB)) {
            orb = s;
            pot = s.substr(0, s.size() - ORB.size()) + POT;
        } else if (ends(POT)) {
            pot = s;
            orb = s.substr(0, s.size() - POT.size()) + ORB;
        }
        // split layout when both siblings open as HDF5; else one combined file
        if (!orb.empty() && fs::exists(orb) && fs::exists(pot)) {
            try {
                auto a = std::make_unique<h5lite::Reader>(orb);
                auto b = std::make_unique<h5lite::Reader>(pot);
                p->orb = std::move(a);
                p->pot_own = std::move(b);
                p->split = true;
            } catch (const h5lite::Error&) {
                p->orb.reset();
                p->pot_own.reset();
            }
        }
        if (!p->split) p->orb = std::make_unique<h5lite::Reader>(s);
        const h5lite::Reader& O = *p->orb;
        const h5lite::Reader& P = p->split ? *p->pot_own : O;
        p->rmin = O.scalar_f64("/grid/rmin");
        p->dr = O.scalar_f64("/grid/dr");
        p->Nr = static_cast<int>(O.scalar_i64("/grid/N"));
        p->Lmax_sce = static_cast<int>(O.scalar_i64("/angular/Lmax"));
        const auto zs = O.shape("/geometry/Z");
        const uint64_t na = zs.empty() ? 0 : zs[0];
        std::vector<long long> Z(na);
        std::vector<double> xyz(na * 3);
        if (na) {
            O.read_i64("/geometry/Z", Z.data());
            O.read_f64("/geometry/xyz_bohr", xyz.data());
        }
        for (uint64_t i = 0; i < na; ++i) {
            p->atoms.push_back(static_cast<double>(Z[i]));
            for (int c = 0; c < 3; ++c) p->atoms.push_back(xyz[3 * i + c]);
        }
        p->n_alpha = static_cast<int>(O.scalar_i64("/orbitals/n_alpha"));
        p->n_occ_alpha = static_cast<int>(O.scalar_i64("/orbitals/n_occ_alpha"));
        p->n_sce = O.exists("/orbitals/n_sce") ? static_cast<int>(O.scalar_i64("/orbitals/n_sce")) : p->n_alpha;
        p->Lmax_orb_store = O.exists("/orbitals/Lmax_orb_store")
                                ? static_cast<int>(O.scalar_i64("/orbitals/Lmax_orb_store")) : p->Lmax_sce;
        p->Nlm_orb_store = O.exists("/orbitals/Nlm_orb_store")
                               ? static_cast<int>(O.scalar_i64("/orbitals/Nlm_orb_store"))
                               : (p->Lmax_sce + 1) * (p->Lmax_sce + 1);
        p->Nr_orb_store = O.exists("/orbitals/Nr_orb_store")
                              ? static_cast<int>(O.scalar_i64("/orbitals/Nr_orb_store")) : p->Nr;
        const auto ne = O.shape("/orbitals/energies_hartree");
        p->orb_energies.resize(ne.empty() ? 1 : ne[0]);
        O.read_f64("/orbitals/energies_hartree", p->orb_energies.data());
        p->has_init = O.exists("/initial_state/psi_lm");
        if (p->has_init) p->E_init = O.scalar_f64("/initial_state/energy_hartree");
        p->has_pol = P.exists("/polarizability/alpha_iso_au");
        if (p->has_pol) p->alpha_iso = P.scalar_f64("/polarizability/alpha_iso_au");
        if (!P.exists("/potential/V_H")) throw h5lite::Error("no /potential/V_H");
        *out = p.release();
        return SCATT_OK;
    });
}

int scatt_preproc_info(scatt_preproc* p, int* out_i8, double* out_d4) {
    if (!p || !out_i8 || !out_d4) return SCATT_ERR_ARG;
    const int iv[8] = {p->Nr, p->Lmax_sce, p->n_alpha, p->n_occ_alpha,
                       p->n_sce, p->Nlm_orb_store, p->Nr_orb_store, p->has_init ? 1 : 0};
    std::copy(iv, iv + 8, out_i8);
    out_d4[0] = p->rmin;
    out_d4[1] = p->dr;
    out_d4[2] = p->E_init;
    out_d4[3] = p->alpha_iso;
    return SCATT_OK;
}

int scatt_preproc_orbital_energies(scatt_preproc* p, double* out, int n) {
    if (!p || !out || n < 0) return SCATT_ERR_ARG;
    const int m = std::min<int>(n, static_cast<int>(p->orb_energies.size()));
    std::copy(p->orb_energies.begin(), p->orb_energies.begin() + m, out);
    return SCATT_OK;
}

int scatt_preproc_atoms(scatt_preproc* p, double* out4, int n) {
    if (!p || !out4 || n < 0) return SCATT_ERR_ARG;
    const int m = std::min<int>(n, static_cast<int>(p->atoms.size() / 4));
    std::copy(p->atoms.begin(), p->atoms.begin() + 4 * m, out4);
    return SCATT_OK;
}

int scatt_preproc_desc(scatt_preproc* p, int l_cont_max, scatt_scan_desc* d, double* E_init) {
    if (!p || !d || l_cont_max < 0) return SCATT_ERR_ARG;
    return guarded("scatt_preproc_desc", [&]() {
        if (p->rmin != 0.0) throw std::invalid_argument("the solver's grid is r = ir * dr: /grid/rmin must be 0");
        const h5lite::Reader& O = *p->orb;
        const h5lite::Reader& P = p->split ? *p->pot_own : O;
        // the rows the reference reads: V_H's first (2 l_cont + 1)^2 multipoles
        // (main.cpp:365) and, per orbital, the first (l_cont + l_exch + 1)^2
        // channels with l_exch = min(l_cont, 10) (main.cpp:700-721)
        const auto vs = P.shape("/potential/V_H");
        if (vs.size() != 2 || (int)vs[1] < p->Nr) throw h5lite::Error("/potential/V_H shape");
        const uint64_t nH = std::min<uint64_t>(vs[0], (uint64_t)(2 * l_cont_max + 1) * (2 * l_cont_max + 1));
        p->vh.assign(nH * p->Nr, 0.0);
        P.read_f64("/potential/V_H", p->vh.data(), {0, 0}, {nH, (uint64_t)p->Nr});
        const int l_orb = l_cont_max + std::min(l_cont_max, 10);
        const int cut = (l_orb + 1) * (l_orb + 1);
        const auto ps = O.shape("/orbitals/psi_lm");
        const int Nlm_file = p->Nlm_orb_store;
        if (ps.size() != 2 || ps[0] < (uint64_t)p->n_sce * Nlm_file) throw h5lite::Error("/orbitals/psi_lm shape");
        const int Nr_store = static_cast<int>(std::min<uint64_t>(ps[1], (uint64_t)p->Nr_orb_store));
        const int take = std::min(cut, Nlm_file);
        int take_init = 0;
        if (p->has_init) {
            const auto is = O.shape("/initial_state/psi_lm");
            if (is.size() != 2) throw h5lite::Error("/initial_state/psi_lm shape");
            take_init = static_cast<int>(std::min<uint64_t>(is[0], (uint64_t)cut));
        }
        const int Nlm = std::max(take, take_init);
        const int n_orb = p->n_sce + (p->has_init ? 1 : 0);
        p->psi.assign((size_t)n_orb * Nlm * Nr_store, 0.0);
        std::vector<double> blk((size_t)take * Nr_store);
        for (int i = 0; i < p->n_sce; ++i) {
            O.read_f64("/orbitals/psi_lm", blk.data(), {(uint64_t)i * Nlm_file, 0}, {(uint64_t)take, (uint64_t)Nr_store});
            for (int l = 0; l < take; ++l)
                std::copy(blk.begin() + (size_t)l * Nr_store, blk.begin() + (size_t)(l + 1) * Nr_store,
                          p->psi.begin() + ((size_t)i * Nlm + l) * Nr_store);
        }
        if (p->has_init) {
            const auto is = O.shape("/initial_state/psi_lm");
            const int nr = static_cast<int>(std::min<uint64_t>(is[1], (uint64_t)Nr_store));
            std::vector<double> ib((size_t)take_init * nr);
            O.read_f64("/initial_state/psi_lm", ib.data(), {0, 0}, {(uint64_t)take_init, (uint64_t)nr});
            for (int l = 0; l < take_init; ++l)
                std::copy(ib.begin() + (size_t)l * nr, ib.begin() + (size_t)(l + 1) * nr,
                          p->psi.begin() + ((size_t)p->n_sce * Nlm + l) * Nr_store);
        }
        std::memset(d, 0, sizeof(*d));
        d->Nr = p->Nr;
        d->dr = p->dr;
        d->l_cont_max = l_cont_max;
        d->n_occ = p->n_occ_alpha;
        d->n_orb = n_orb;
        d->Nlm_store = Nlm;
        d->Nr_store = Nr_store;
        d->psi_lm = p->psi.data();
        d->init_state = p->has_init ? p->n_sce : -1;
        d->n_H = static_cast<int>(nH);
        d->V_H = p->vh.data();
        d->n_atoms = static_cast<int>(p->atoms.size() / 4);
        d->atoms = p->atoms.data();
        d->alpha_pol = p->has_pol ? p->alpha_iso : 0.0;
        d->pol_form = 0;
        d->r_c = 1.5;
        d->n_transition = 0;
        d->chi_cutoff = 1e-15;
        if (E_init) {
            const int homo = p->n_occ_alpha - 1;
            *E_init = p->has_init ? p->E_init
                                  : (homo >= 0 && homo < (int)p->orb_energies.size() ? p->orb_energies[homo] : 0.0);
        }
        return SCATT_OK;
    });
}

int scatt_preproc_close(scatt_preproc* p) {
    delete p;
    return SCATT_OK;
}

}  // extern "C"
