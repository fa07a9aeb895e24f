// molden.cpp -- reader of the Molden files the preprocessing step starts
// from (preprocessing/src/molden/Molden.hpp: [Atoms], [GTO], [MO] and the
// spherical-function flags), host-only, behind the C ABI (scatt_molden_*).
//
// What the file says is kept as written: atoms in bohr (an [Atoms] block
// marked Angs, or with no unit, is converted with the factor the reference
// uses), shells in file order with their raw exponents and contraction
// coefficients, MO coefficients in AO order.  Flags [5D], [5D7F], [5D10F],
// [7F], [9G] make d / f / g shells spherical (s, p, h and above always
// are); Fortran exponents (1.0D-3) are read.  Malformed input -- a missing
// section, a short line, an atom or AO index out of range, a combined sp
// shell, no alpha orbital -- is an SCATT_ERR_IO with the line.  The basis
// of scatt_molden_shells is the spherical one the expansion evaluates:
// a Cartesian shell of l >= 2 is an error there, as in the reference's
// build_basis (MoldenBasis.hpp:129-150).
#include <cctype>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"

namespace scatt {
namespace {

constexpr double BOHR_PER_ANGSTROM = 1.8897261245650618;

struct MoldenError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

std::string lowered(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// 1.0D-3 -> 1.0E-3: a D between a digit and a digit or sign
std::string fortran_exponents(std::string s) {
    for (size_t i = 1; i + 1 < s.size(); ++i)
        if ((s[i] == 'D' || s[i] == 'd') && std::isdigit((unsigned char)s[i - 1]) &&
            (std::isdigit((unsigned char)s[i + 1]) || s[i + 1] == '+' || s[i + 1] == '-'))
            s[i] = 'E';
    return s;
}

// "[Name] rest" -> lowered Name; false when the line opens no section
bool section_name(const std::string& line, std::string* name) {
    const std::string t = trim(line);
    if (t.size() < 3 || t[0] != '[') return false;
    const size_t c = t.find(']');
    if (c == std::string::npos) return false;
    *name = lowered(t.substr(1, c - 1));
    return true;
}

int element_z(const std::string& sym) {
    static const char* const table[] = {"h",  "he", "li", "be", "b",  "c",  "n",  "o",  "f",  "ne",
                                        "na", "mg", "al", "si", "p",  "s",  "cl", "ar", "k",  "ca"};
    const std::string s = lowered(sym);
    for (int z = 0; z < 20; ++z)
        if (s == table[z]) return z + 1;
    throw MoldenError("molden: unknown element '" + sym + "'");
}

int shell_l(const std::string& letter) {
    const std::string s = lowered(letter);
    if (s == "sp") throw MoldenError("molden: combined 'sp' shell not supported");
    static const char order[] = "spdfghi";
    for (int l = 0; l < 7; ++l)
        if (s.size() == 1 && s[0] == order[l]) return l;
    throw MoldenError("molden: unknown shell letter '" + letter + "'");
}

}  // namespace
}  // namespace scatt

using namespace scatt;

struct scatt_molden {
    struct Shell {
        int atom, l;
        bool pure;
        std::vector<double> exps, coefs;
    };
    struct Orbital {
        double energy = 0.0, occ = 0.0;
        bool beta = false;
        std::vector<double> C;
    };
    std::vector<double> atoms;               // Z, x, y, z (bohr) per atom
    std::vector<Shell> shells;
    std::vector<Orbital> alpha, beta;
    int nbf = 0, n_prim = 0;
    bool sph_d = false, sph_f = false, sph_g = false;

    void parse(const std::string& path) {
        std::ifstream f(path);
        if (!f) throw MoldenError("molden: cannot open '" + path + "'");
        std::vector<std::string> lines;
        for (std::string ln; std::getline(f, ln);) lines.push_back(ln);
        for (const auto& ln : lines) {            // the flags may stand anywhere
            std::string n;
            if (!section_name(ln, &n)) continue;
            if (n.find("5d10f") != std::string::npos) { sph_d = true; sph_f = false; }
            else if (n.find("5d7f") != std::string::npos) { sph_d = true; sph_f = true; }
            else if (n == "5d") sph_d = true;
            else if (n == "7f") sph_f = true;
            else if (n == "9g") sph_g = true;
        }
        parse_atoms(lines);
        parse_gto(lines);
        parse_mo(lines);
        if (alpha.empty()) throw MoldenError("molden: no alpha orbital in [MO]");
    }

    static int find(const std::vector<std::string>& lines, const char* want) {
        for (int i = 0; i < (int)lines.size(); ++i) {
            std::string n;
            if (section_name(lines[i], &n) && n == want) return i;
        }
        throw MoldenError(std::string("molden: [") + want + "] section missing");
    }
    static bool opens_section(const std::string& ln) {
        const std::string t = trim(ln);
        return !t.empty() && t[0] == '[';
    }

    void parse_atoms(const std::vector<std::string>& lines) {
        const int at = find(lines, "atoms");
        const std::string head = lowered(lines[at]);
        const bool au = head.find("au") != std::string::npos && head.find("angs") == std::string::npos;
        const double scale = au ? 1.0 : BOHR_PER_ANGSTROM;
        for (int i = at + 1; i < (int)lines.size() && !opens_section(lines[i]); ++i) {
            const std::string t = trim(lines[i]);
            if (t.empty()) continue;
            std::istringstream is(fortran_exponents(t));
            std::string sym;
            int idx = 0, z = 0;
            double x = 0, y = 0, w = 0;
            if (!(is >> sym >> idx >> z >> x >> y >> w)) throw MoldenError("molden: bad [Atoms] line: '" + t + "'");
            atoms.insert(atoms.end(), {(double)(z > 0 ? z : element_z(sym)), x * scale, y * scale, w * scale});
        }
        if (atoms.empty()) throw MoldenError("molden: [Atoms] holds no atom");
    }

    void parse_gto(const std::vector<std::string>& lines) {
        int i = find(lines, "gto") + 1;
        const int N = (int)lines.size(), n_atoms = (int)(atoms.size() / 4);
        while (i < N) {
            while (i < N && trim(lines[i]).empty()) ++i;
            if (i >= N || opens_section(lines[i])) break;
            std::istringstream ah(fortran_exponents(trim(lines[i])));
            int a1 = 0, zero = 0;
            if (!(ah >> a1 >> zero)) throw MoldenError("molden: bad [GTO] atom line: '" + trim(lines[i]) + "'");
            if (a1 < 1 || a1 > n_atoms) throw MoldenError("molden: [GTO] atom index out of range: '" + trim(lines[i]) + "'");
            ++i;
            while (i < N) {
                const std::string t = trim(lines[i]);
                if (t.empty()) { ++i; break; }
                if (opens_section(lines[i])) break;
                std::istringstream sh(fortran_exponents(t));
                std::string letter;
                int np = 0;
                double unused_scale = 0.0;
                if (!(sh >> letter >> np >> unused_scale) || np < 1)
                    throw MoldenError("molden: bad shell line: '" + t + "'");
                Shell s;
                s.atom = a1 - 1;
                s.l = shell_l(letter);
                s.pure = s.l <= 1 || (s.l == 2 && sph_d) || (s.l == 3 && sph_f) || (s.l == 4 && sph_g) || s.l >= 5;
                ++i;
                for (int p = 0; p < np; ++p, ++i) {
                    if (i >= N) throw MoldenError("molden: the file ends inside a shell");
                    std::istringstream pl(fortran_exponents(trim(lines[i])));
                    double a = 0, c = 0;
                    if (!(pl >> a >> c)) throw MoldenError("molden: bad primitive line: '" + trim(lines[i]) + "'");
                    s.exps.push_back(a);
                    s.coefs.push_back(c);
                }
                nbf += s.pure ? 2 * s.l + 1 : (s.l + 1) * (s.l + 2) / 2;
                n_prim += np;
                shells.push_back(std::move(s));
            }
        }
        if (shells.empty()) throw MoldenError("molden: [GTO] holds no shell");
    }

    void parse_mo(const std::vector<std::string>& lines) {
        int i = find(lines, "mo") + 1;
        const int N = (int)lines.size();
        auto key = [](const std::string& u, const char* k) {
            const size_t n = std::strlen(k);
            return u.size() >= n && lowered(u.substr(0, n)) == k;
        };
        auto value = [](const std::string& u) { return trim(u.substr(u.find('=') + 1)); };
        while (i < N) {
            if (trim(lines[i]).empty()) { ++i; continue; }
            if (opens_section(lines[i])) break;
            Orbital o;
            for (; i < N; ++i) {                  // Sym= Ene= Spin= Occup=, any order
                const std::string u = trim(lines[i]);
                if (u.empty()) continue;
                if (key(u, "sym=")) continue;
                if (key(u, "ene=")) o.energy = std::stod(fortran_exponents(value(u)));
                else if (key(u, "spin=")) o.beta = lowered(value(u)).rfind("b", 0) == 0;
                else if (key(u, "occup=")) o.occ = std::stod(fortran_exponents(value(u)));
                else break;
            }
            o.C.assign(nbf, 0.0);
            for (; i < N; ++i) {
                const std::string u = trim(lines[i]);
                if (u.empty()) { ++i; break; }
                if (opens_section(lines[i]) || key(u, "sym=") || key(u, "ene=") || key(u, "spin=") ||
                    key(u, "occup="))
                    break;
                std::istringstream cl(fortran_exponents(u));
                int k = 0;
                double c = 0;
                if (!(cl >> k >> c)) throw MoldenError("molden: bad MO coefficient line: '" + u + "'");
                if (k < 1 || k > nbf) throw MoldenError("molden: MO coefficient index out of range: '" + u + "'");
                o.C[k - 1] = c;
            }
            (o.beta ? beta : alpha).push_back(std::move(o));
        }
    }
};

namespace {

template <class F>
int molden_guarded(const char* who, F f) {
    try {
        return f();
    } catch (const MoldenError& e) {
        set_last_error(std::string(who) + ": " + e.what());
        return SCATT_ERR_IO;
    } catch (const std::invalid_argument& e) {
        set_last_error(std::string(who) + ": molden: a number does not parse (" + e.what() + ")");
        return SCATT_ERR_IO;
    } catch (const std::out_of_range& e) {
        set_last_error(std::string(who) + ": molden: a number is out of range (" + e.what() + ")");
        return SCATT_ERR_IO;
    } catch (const std::bad_alloc&) {
        set_last_error(std::string(who) + ": host allocation failed");
        return SCATT_ERR_OOM;
    }
}

}  // namespace

extern "C" {

int scatt_molden_open(const char* path, scatt_molden** out) {
    if (!path || !out) return SCATT_ERR_ARG;
    *out = nullptr;
    return molden_guarded("scatt_molden_open", [&]() {
        auto m = std::make_unique<scatt_molden>();
        m->parse(path);
        *out = m.release();
        return SCATT_OK;
    });
}

int scatt_molden_info(scatt_molden* m, int* out7) {
    if (!m || !out7) return SCATT_ERR_ARG;
    out7[0] = (int)(m->atoms.size() / 4);
    out7[1] = (int)m->shells.size();
    out7[2] = m->nbf;
    out7[3] = (int)m->alpha.size();
    out7[4] = (int)m->beta.size();
    out7[5] = m->n_prim;
    int cart = 0;
    for (const auto& s : m->shells) cart += (!s.pure && s.l >= 2) ? 1 : 0;
    out7[6] = cart;
    return SCATT_OK;
}

int scatt_molden_atoms(scatt_molden* m, double* zxyz) {
    if (!m || !zxyz) return SCATT_ERR_ARG;
    std::memcpy(zxyz, m->atoms.data(), m->atoms.size() * sizeof(double));
    return SCATT_OK;
}

int scatt_molden_shells(scatt_molden* m, int* l, int* nprim, double* center, double* exps, double* coefs) {
    if (!m || !l || !nprim || !center || !exps || !coefs) return SCATT_ERR_ARG;
    size_t p = 0;
    for (size_t i = 0; i < m->shells.size(); ++i) {
        const auto& s = m->shells[i];
        if (!s.pure && s.l >= 2) {
            set_last_error("scatt_molden_shells: shell " + std::to_string(i) + " (l = " + std::to_string(s.l) +
                           ") is Cartesian; the file needs the [5D] / [5D7F] / [9G] flags for spherical functions");
            return SCATT_ERR_ARG;
        }
        l[i] = s.l;
        nprim[i] = (int)s.exps.size();
        for (int k = 0; k < 3; ++k) center[3 * i + k] = m->atoms[4 * s.atom + 1 + k];
        std::memcpy(exps + p, s.exps.data(), s.exps.size() * sizeof(double));
        std::memcpy(coefs + p, s.coefs.data(), s.coefs.size() * sizeof(double));
        p += s.exps.size();
    }
    return SCATT_OK;
}

int scatt_molden_mos(scatt_molden* m, int beta, double* C, double* occ, double* energy) {
    if (!m || !C || !occ || !energy) return SCATT_ERR_ARG;
    const auto& v = beta ? m->beta : m->alpha;
    for (size_t i = 0; i < v.size(); ++i) {
        std::memcpy(C + i * (size_t)m->nbf, v[i].C.data(), (size_t)m->nbf * sizeof(double));
        occ[i] = v[i].occ;
        energy[i] = v[i].energy;
    }
    return SCATT_OK;
}

int scatt_molden_close(scatt_molden* m) {
    delete m;
    return SCATT_OK;
}

}  // extern "C"
