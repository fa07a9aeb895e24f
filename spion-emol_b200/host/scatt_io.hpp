// scatt_io.hpp -- C++ host interface of the file formats around the path,
// over the C ABI of libscatt_b200 (HDF5 subset, no libhdf5).
//
// Keeps the reference's names and behaviour for C++ callers: EnergyGrid
// (src/scatt/EnergyGrid.hpp:23-45), DipoleScanMeta / DipoleSlice /
// DipoleEnergyPayload / DipoleWriter / DipoleEnergyReadback / DipoleReader
// (src/scatt/DipoleIO.hpp:40-176) and the preprocessing reader
// (src/io/HDF5Reader.hpp:42-144: PreprocData, HDF5Reader with its split-
// layout detection).  Failures throw std::runtime_error with the library's
// message, as the reference's _check helper does.  Matrices use the
// column-major scatt_b200::Matrix of scatt_b200.hpp.
#pragma once

#include <algorithm>
#include <array>
#include <complex>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <vector>

#include "scatt_b200.h"
#include "scatt_b200.hpp"

namespace scatt_b200 {

struct EnergyGrid {
    double dk = 0.01;
    int ik_min = 1;
    int ik_max = 101;              // exclusive
    double k(int ik) const { return ik * dk; }
    double E(int ik) const {
        const double kv = k(ik);
        return 0.5 * kv * kv;
    }
    int size() const { return ik_max - ik_min; }
    std::string tag(int ik, int pad = 4) const {
        if (ik < 0) throw std::invalid_argument("EnergyGrid::tag: ik < 0");
        std::string s = std::to_string(ik);
        while (static_cast<int>(s.size()) < pad) s = "0" + s;
        return "ik" + s;
    }
    void validate() const {
        if (!(dk > 0.0)) throw std::invalid_argument("EnergyGrid: dk must be > 0");
        if (ik_min < 0) throw std::invalid_argument("EnergyGrid: ik_min < 0");
        if (ik_max <= ik_min) throw std::invalid_argument("EnergyGrid: ik_max <= ik_min");
    }
};

struct DipoleScanMeta {
    double r_min = 0.0, dr = 0.0;
    std::size_t N_grid = 0;
    int l_max_continuum = 0;
    EnergyGrid kgrid;
    double E_HOMO = 0.0;
    std::vector<double> occ_energies, occ_spin_factors;
    struct Atom {
        int Z;
        double x, y, z;
    };
    std::vector<Atom> atoms;
    std::string psi_dir_prefix, molecule_name, git_hash, iso_date_utc;
};

enum class DipoleGauge { Length = 0, Velocity = 1 };
enum class Polarization { X = 0, Y = 1, Z = 2 };

struct DipoleSlice {
    DipoleGauge gauge = DipoleGauge::Length;
    Polarization pol = Polarization::X;
    std::vector<std::complex<double>> D_reduced, D_reduced_raw;   // n_ch
    std::vector<double> d_raw;                                    // n_ch
    std::vector<double> d_correction;                             // n_occ
    double partial_sigma = 0.0;
};

struct DipoleEnergyPayload {
    int ik = 0;
    Matrix A, B;                   // n_ch x n_ch
    Matrix b_overlap;              // n_ch x n_occ
    std::array<DipoleSlice, 6> slices;
    double fit_residual_rel = 0.0, K_symmetry_err = 0.0;
};

struct DipoleEnergyReadback {
    int ik = 0;
    double k = 0.0, E = 0.0;
    Matrix A, B, b_overlap;
    std::array<DipoleSlice, 6> slices;
    double fit_residual_rel = 0.0, K_symmetry_err = 0.0;
};

namespace detail {

// the C struct of a meta, pointing into `m` and the two vectors it fills
inline scatt_dipole_meta c_meta(const DipoleScanMeta& m, std::vector<int>& Z, std::vector<double>& xyz) {
    Z.clear();
    xyz.clear();
    for (const auto& a : m.atoms) {
        Z.push_back(a.Z);
        xyz.insert(xyz.end(), {a.x, a.y, a.z});
    }
    scatt_dipole_meta c{};
    c.r_min = m.r_min;
    c.dr = m.dr;
    c.N_grid = static_cast<long long>(m.N_grid);
    c.l_max_continuum = m.l_max_continuum;
    c.dk = m.kgrid.dk;
    c.ik_min = m.kgrid.ik_min;
    c.ik_max = m.kgrid.ik_max;
    c.E_HOMO = m.E_HOMO;
    c.n_occ = static_cast<int>(m.occ_energies.size());
    c.occ_energies = m.occ_energies.data();
    c.occ_spin_factors = m.occ_spin_factors.data();
    c.n_atoms = static_cast<int>(Z.size());
    c.Z = Z.data();
    c.xyz_bohr = xyz.data();
    c.molecule_name = m.molecule_name.c_str();
    c.git_hash = m.git_hash.c_str();
    c.iso_date_utc = m.iso_date_utc.c_str();
    c.psi_dir_prefix = m.psi_dir_prefix.c_str();
    return c;
}

// column-major Matrix <-> row-major buffer
inline std::vector<double> row_major(const Matrix& M) {
    std::vector<double> out((size_t)M.rows * M.cols);
    for (int i = 0; i < M.rows; ++i)
        for (int j = 0; j < M.cols; ++j) out[(size_t)i * M.cols + j] = M(i, j);
    return out;
}

}  // namespace detail

// Generic reader over scatt_h5r_* (RAII).
class H5File {
public:
    explicit H5File(const std::string& path) { check(scatt_h5r_open(path.c_str(), &h_)); }
    ~H5File() { scatt_h5r_close(h_); }
    H5File(const H5File&) = delete;
    H5File& operator=(const H5File&) = delete;

    bool exists(const std::string& p) const {
        int k = 0;
        check(scatt_h5r_kind(h_, p.c_str(), &k));
        return k != 0;
    }
    std::vector<long long> shape(const std::string& p) const {
        int rank = 0, ek = 0;
        long long d[8] = {};
        check(scatt_h5r_shape(h_, p.c_str(), &rank, d, &ek));
        return std::vector<long long>(d, d + rank);
    }
    std::vector<double> read(const std::string& p) const {
        long long n = 1;
        for (long long x : shape(p)) n *= x;
        std::vector<double> v((size_t)n);
        check(scatt_h5r_read(h_, p.c_str(), 0, 0, nullptr, nullptr, v.data()));
        return v;
    }
    std::vector<long long> read_int(const std::string& p) const {
        long long n = 1;
        for (long long x : shape(p)) n *= x;
        std::vector<long long> v((size_t)n);
        check(scatt_h5r_read(h_, p.c_str(), 1, 0, nullptr, nullptr, v.data()));
        return v;
    }
    Matrix read_matrix(const std::string& p) const {   // 2-D row-major on disk
        const auto s = shape(p);
        if (s.size() != 2) throw std::runtime_error(p + " is not 2-D");
        const auto v = read(p);
        Matrix M((int)s[0], (int)s[1]);
        for (int i = 0; i < M.rows; ++i)
            for (int j = 0; j < M.cols; ++j) M(i, j) = v[(size_t)i * M.cols + j];
        return M;
    }
    double attr_double(const std::string& obj, const std::string& name) const {
        int k = 0;
        double f = 0.0;
        long long i = 0;
        check(scatt_h5r_attr(h_, obj.c_str(), name.c_str(), &k, &f, &i, nullptr, 0));
        if (k != 1 && k != 2) throw std::runtime_error("no numeric attribute " + obj + ":" + name);
        return f;
    }
    long long attr_int(const std::string& obj, const std::string& name) const {
        int k = 0;
        double f = 0.0;
        long long i = 0;
        check(scatt_h5r_attr(h_, obj.c_str(), name.c_str(), &k, &f, &i, nullptr, 0));
        if (k != 1 && k != 2) throw std::runtime_error("no numeric attribute " + obj + ":" + name);
        return i;
    }
    std::string attr_string(const std::string& obj, const std::string& name) const {
        int k = 0;
        std::vector<char> buf(4096, 0);
        check(scatt_h5r_attr(h_, obj.c_str(), name.c_str(), &k, nullptr, nullptr, buf.data(), (long long)buf.size()));
        if (k != 3) throw std::runtime_error("no string attribute " + obj + ":" + name);
        return std::string(buf.data());
    }

private:
    scatt_h5r* h_ = nullptr;
};

class DipoleWriter {
public:
    DipoleWriter(const std::string& scan_dir, const DipoleScanMeta& meta) : scan_dir_(scan_dir), meta_(meta) {
        meta_.kgrid.validate();
        const scatt_dipole_meta c = detail::c_meta(meta_, Z_, xyz_);
        check(scatt_dipole_open(scan_dir_.c_str(), &c));
    }
    bool has_energy(int ik) const {
        int has = 0;
        check(scatt_dipole_has_energy(scan_dir_.c_str(), ik, &has));
        return has != 0;
    }
    void write_energy(const DipoleEnergyPayload& p) {
        const int n = p.A.rows, no = p.b_overlap.cols;
        if (p.A.cols != n) throw std::runtime_error("DipoleWriter: A not square");
        if (p.B.rows != n || p.B.cols != n) throw std::runtime_error("DipoleWriter: B shape mismatch");
        if (p.b_overlap.rows != n) throw std::runtime_error("DipoleWriter: b_overlap row count != n_ch");
        // each slice goes where its own (gauge, polarization) puts it
        std::vector<double> Dre(6 * (size_t)n), Dim(6 * (size_t)n), Rre(6 * (size_t)n), Rim(6 * (size_t)n),
            draw(6 * (size_t)n), dcorr(6 * (size_t)no), sig(6);
        std::array<bool, 6> seen{};
        for (const DipoleSlice& sl : p.slices) {
            if ((int)sl.D_reduced.size() != n || (int)sl.D_reduced_raw.size() != n || (int)sl.d_raw.size() != n ||
                (int)sl.d_correction.size() != no)
                throw std::runtime_error("DipoleWriter: per-slice size mismatch");
            const int s = slice_index(sl.gauge, sl.pol);
            if (seen[s]) throw std::runtime_error("DipoleWriter: two slices of one gauge and polarization");
            seen[s] = true;
            for (int i = 0; i < n; ++i) {
                Dre[(size_t)s * n + i] = sl.D_reduced[i].real();
                Dim[(size_t)s * n + i] = sl.D_reduced[i].imag();
                Rre[(size_t)s * n + i] = sl.D_reduced_raw[i].real();
                Rim[(size_t)s * n + i] = sl.D_reduced_raw[i].imag();
                draw[(size_t)s * n + i] = sl.d_raw[i];
            }
            std::copy(sl.d_correction.begin(), sl.d_correction.end(), dcorr.begin() + (size_t)s * no);
            sig[s] = sl.partial_sigma;
        }
        const auto A = detail::row_major(p.A), B = detail::row_major(p.B), bo = detail::row_major(p.b_overlap);
        scatt_dipole_energy e{};
        e.ik = p.ik;
        e.n_ch = n;
        e.n_occ = no;
        e.A = A.data();
        e.B = B.data();
        e.b_overlap = bo.data();
        e.D_re = Dre.data();
        e.D_im = Dim.data();
        e.Draw_re = Rre.data();
        e.Draw_im = Rim.data();
        e.d_raw = draw.data();
        e.d_corr = dcorr.data();
        e.partial_sigma = sig.data();
        e.fit_residual_rel = p.fit_residual_rel;
        e.K_symmetry_err = p.K_symmetry_err;
        const scatt_dipole_meta c = detail::c_meta(meta_, Z_, xyz_);
        check(scatt_dipole_write_energy(scan_dir_.c_str(), &c, &e));
    }
    void finalize() { check(scatt_dipole_finalize(scan_dir_.c_str())); }
    const std::string& scan_dir() const { return scan_dir_; }

    // Canonical order {L,X}, {L,Y}, {L,Z}, {V,X}, {V,Y}, {V,Z}.
    static int slice_index(DipoleGauge g, Polarization p) {
        return (g == DipoleGauge::Length ? 0 : 3) + static_cast<int>(p);
    }

private:
    std::string scan_dir_;
    DipoleScanMeta meta_;
    std::vector<int> Z_;
    std::vector<double> xyz_;
};

class DipoleReader {
public:
    explicit DipoleReader(const std::string& scan_dir) : scan_dir_(scan_dir) {
        H5File f(scan_dir_ + "/manifest.h5");
        meta_.r_min = f.attr_double("/grid", "r_min");
        meta_.dr = f.attr_double("/grid", "dr");
        meta_.N_grid = static_cast<std::size_t>(f.attr_int("/grid", "N_grid"));
        meta_.l_max_continuum = static_cast<int>(f.attr_int("/grid", "l_max_continuum"));
        meta_.E_HOMO = f.attr_double("/grid", "E_HOMO");
        meta_.kgrid.dk = f.attr_double("/kgrid", "dk");
        meta_.kgrid.ik_min = static_cast<int>(f.attr_int("/kgrid", "ik_min"));
        meta_.kgrid.ik_max = static_cast<int>(f.attr_int("/kgrid", "ik_max"));
        if (f.exists("/occ")) {
            meta_.occ_energies = f.read("/occ/energies");
            meta_.occ_spin_factors = f.read("/occ/spin_factors");
        }
        if (f.exists("/atoms")) {
            const auto Z = f.read_int("/atoms/Z");
            const auto xyz = f.read("/atoms/xyz_bohr");
            for (size_t i = 0; i < Z.size(); ++i)
                meta_.atoms.push_back({(int)Z[i], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]});
        }
        meta_.molecule_name = f.attr_string("/run", "molecule_name");
        meta_.git_hash = f.attr_string("/run", "git_hash");
        meta_.iso_date_utc = f.attr_string("/run", "iso_date_utc");
        meta_.psi_dir_prefix = f.attr_string("/run", "psi_dir_prefix");
    }
    const DipoleScanMeta& meta() const { return meta_; }

    std::vector<int> available_ik() const {
        std::vector<int> out;
        for (const auto& e : std::filesystem::directory_iterator(scan_dir_)) {
            const std::string n = e.path().filename().string();
            if (n.size() > 5 && n.rfind("ik", 0) == 0 && n.substr(n.size() - 3) == ".h5") {
                const std::string num = n.substr(2, n.size() - 5);
                if (!num.empty() && std::all_of(num.begin(), num.end(), ::isdigit)) out.push_back(std::stoi(num));
            }
        }
        std::sort(out.begin(), out.end());
        return out;
    }

    DipoleEnergyReadback read_energy(int ik) const {
        H5File f(scan_dir_ + "/" + meta_.kgrid.tag(ik) + ".h5");
        DipoleEnergyReadback r;
        r.ik = static_cast<int>(f.attr_int("/meta", "ik"));
        r.k = f.attr_double("/meta", "k");
        r.E = f.attr_double("/meta", "E");
        r.fit_residual_rel = f.attr_double("/meta", "fit_residual_rel");
        r.K_symmetry_err = f.attr_double("/meta", "K_symmetry_err");
        r.A = f.read_matrix("/A");
        r.B = f.read_matrix("/B");
        r.b_overlap = f.read_matrix("/b_overlap");
        const char* gauges[2] = {"length", "velocity"};
        const char* pols[3] = {"x", "y", "z"};
        for (int s = 0; s < 6; ++s) {
            const std::string g = std::string("/dipole/") + gauges[s / 3] + "/" + pols[s % 3];
            DipoleSlice& sl = r.slices[s];
            sl.gauge = static_cast<DipoleGauge>(s / 3);
            sl.pol = static_cast<Polarization>(s % 3);
            const auto re = f.read(g + "/D_ortho_re"), im = f.read(g + "/D_ortho_im");
            const auto rre = f.read(g + "/D_raw_re"), rim = f.read(g + "/D_raw_im");
            for (size_t i = 0; i < re.size(); ++i) {
                sl.D_reduced.emplace_back(re[i], im[i]);
                sl.D_reduced_raw.emplace_back(rre[i], rim[i]);
            }
            sl.d_raw = f.read(g + "/d_raw");
            sl.d_correction = f.read(g + "/d_correction");
            sl.partial_sigma = f.attr_double(g, "partial_sigma");
        }
        return r;
    }

private:
    std::string scan_dir_;
    DipoleScanMeta meta_;
};

// The header fields of a preprocessing file (src/io/HDF5Reader.hpp:42-86);
// the large arrays stay in the reader and reach the solver through
// scan_desc.
struct PreprocData {
    double rmin = 0.0, dr = 0.0;
    std::size_t Nr = 0;
    int Lmax_sce = 0;
    int n_alpha = 0, n_occ_alpha = 0, n_sce = 0;
    int Nlm_orb_store = 0, Nr_orb_store = 0;
    std::vector<double> orb_energies;
    bool has_initial_state = false;
    double init_state_energy = 0.0;
    double alpha_iso = 0.0;
};

class HDF5Reader {
public:
    // path ending in .orbitals.h5 / .potentials.h5 with an existing sibling:
    // the split layout; anything else: one combined file
    explicit HDF5Reader(const std::string& path) { check(scatt_preproc_open(path.c_str(), &p_)); }
    ~HDF5Reader() { scatt_preproc_close(p_); }
    HDF5Reader(const HDF5Reader&) = delete;
    HDF5Reader& operator=(const HDF5Reader&) = delete;

    PreprocData load_header() const {
        int iv[8];
        double dv[4];
        check(scatt_preproc_info(p_, iv, dv));
        PreprocData d;
        d.Nr = static_cast<std::size_t>(iv[0]);
        d.Lmax_sce = iv[1];
        d.n_alpha = iv[2];
        d.n_occ_alpha = iv[3];
        d.n_sce = iv[4];
        d.Nlm_orb_store = iv[5];
        d.Nr_orb_store = iv[6];
        d.has_initial_state = iv[7] != 0;
        d.rmin = dv[0];
        d.dr = dv[1];
        d.init_state_energy = dv[2];
        d.alpha_iso = dv[3];
        d.orb_energies.assign(d.n_sce, 0.0);
        check(scatt_preproc_orbital_energies(p_, d.orb_energies.data(), d.n_sce));
        return d;
    }

    // The solver's scan description for continuum cutoff l_cont_max (valid
    // until the next call or the reader's end) and the initial state's energy.
    scatt_scan_desc scan_desc(int l_cont_max, double* E_init = nullptr) {
        scatt_scan_desc d{};
        check(scatt_preproc_desc(p_, l_cont_max, &d, E_init));
        return d;
    }

private:
    scatt_preproc* p_ = nullptr;
};

}  // namespace scatt_b200
