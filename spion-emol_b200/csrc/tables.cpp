// tables.cpp -- host-side construction of the energy-independent tables of a
// scan (angular coupling lists, nuclear multipoles, quadrature weights).
//
// Each builder restates the table the reference computes once per scan (or,
// in the reference, once per energy; WavefunctionSetup::prepare recomputes
// its G list for every energy, src/main.cpp:1124-1127):
//   * V_sigma(r) ........ Potentials::compute_V_sigma_total (Potentials.cpp:40-88)
//   * Gaunt pair list ... GauntSparseMatrix::build (GauntSparse.hpp:130-180)
//   * G_combined ........ ExchangeCoupling ctor (ExchangeCoupling.cpp:13-54) over
//                         build_G_vector (WavefunctionSetup.cpp:21-81)
//   * dipole tables ..... DipoleMatrixElement::compute_six (DipoleMatrixElement.cpp:628-645)
//   * Simpson weights ... DipoleMatrixElement::simpson_ (DipoleMatrixElement.cpp:142-192)
//   * chi' .............. five_point_derivative (DipoleMatrixElement.cpp:49-74)
#include "tables.hpp"

#include <algorithm>
#include <cmath>
#include <thread>

#include "angular.hpp"

namespace scatt {

namespace {
// real-Gaunt m selection: |m3| must be |m1| + |m2| or ||m1| - |m2||
void m_candidates(int m1, int m2, int l3, std::vector<int>& out) {
    out.clear();
    const int a = std::abs(m1) + std::abs(m2), b = std::abs(std::abs(m1) - std::abs(m2));
    const int cand[4] = {-a, -b, b, a};
    for (int c : cand) {
        if (c < -l3 || c > l3) continue;
        if (std::find(out.begin(), out.end(), c) == out.end()) out.push_back(c);
    }
    std::sort(out.begin(), out.end());
}

template <class F>
void parallel_for(int n, F f) {
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (int i = (int)t; i < n; i += (int)nt) f(i);
        });
    for (auto& x : th) x.join();
}
}  // namespace

std::vector<double> build_vsigma(int Nr, double dr, int l_max, int n_H, const double* V_H,
                                 int n_atoms, const double* atoms) {
    const int l_exp = 2 * l_max;
    const int n_exp = (l_exp + 1) * (l_exp + 1);
    std::vector<double> T((size_t)Nr * n_exp, 0.0);    // [ir][sigma]
    // Y_lm(R_hat) per atom
    std::vector<double> Y((size_t)n_atoms * n_exp, 0.0);
    std::vector<double> Ra(n_atoms);
    for (int a = 0; a < n_atoms; ++a) {
        const double x = atoms[4 * a + 1], y = atoms[4 * a + 2], z = atoms[4 * a + 3];
        const double R = std::sqrt(x * x + y * y + z * z);
        Ra[a] = R;
        double th = 0.0, ph = 0.0;
        if (R > 1e-14) {
            th = std::acos(std::clamp(z / R, -1.0, 1.0));
            ph = std::atan2(y, x);
        }
        for (int l = 0; l <= l_exp; ++l)
            for (int m = -l; m <= l; ++m) {
                double v;
                if (R < 1e-14) v = (l == 0) ? (1.0 / (2.0 * std::sqrt(M_PI))) : 0.0;
                else v = real_Ylm(l, m, th, ph);
                Y[(size_t)a * n_exp + lm_to_idx(l, m)] = v;
            }
    }
    parallel_for(Nr, [&](int ir) {
        const double r = ir * dr;
        if (!(r > 1e-14)) return;     // V(0) is the zero matrix (Potentials.cpp:327)
        double* row = &T[(size_t)ir * n_exp];
        const int nmax = std::min(n_exp, n_H);
        for (int s = 0; s < nmax; ++s) row[s] += V_H[(size_t)s * Nr + ir];
        for (int a = 0; a < n_atoms; ++a) {
            const double Z = atoms[4 * a];
            const double rl = std::min(r, Ra[a]), rg = std::max(r, Ra[a]);
            for (int l = 0; l <= l_exp; ++l) {
                const double radial = (4.0 * M_PI / (2.0 * l + 1.0)) * std::pow(rl, l) / std::pow(rg, l + 1);
                for (int m = -l; m <= l; ++m) {
                    const double Yv = Y[(size_t)a * n_exp + lm_to_idx(l, m)];
                    if (std::abs(Yv) > 1e-15) row[lm_to_idx(l, m)] += -Z * radial * Yv;
                }
            }
        }
    });
    return T;
}

PairCSR build_gaunt_pairs(int l_max) {
    const int ch = (l_max + 1) * (l_max + 1);
    const int l_exp = 2 * l_max;
    PairCSR P;
    const int np = ch * (ch + 1) / 2;
    P.row.resize(np);
    P.col.resize(np);
    std::vector<std::vector<std::pair<int, double>>> per(np);
    // pair index (mu_p, mu), mu >= mu_p, row-major upper triangle (GauntSparse.hpp:74-79)
    std::vector<int> base(ch);
    int idx = 0;
    for (int mp = 0; mp < ch; ++mp) {
        base[mp] = idx;
        for (int mu = mp; mu < ch; ++mu, ++idx) { P.row[idx] = mp; P.col[idx] = mu; }
    }
    parallel_for(ch, [&](int mp) {
        int l2, m2;
        idx_to_lm(mp, l2, m2);
        std::vector<int> mc;
        for (int mu = mp; mu < ch; ++mu) {
            int l1, m1;
            idx_to_lm(mu, l1, m1);
            auto& lst = per[base[mp] + (mu - mp)];
            for (int ls = std::abs(l1 - l2); ls <= std::min(l1 + l2, l_exp); ++ls) {
                if ((l1 + ls + l2) & 1) continue;
                m_candidates(m1, m2, ls, mc);
                for (int ms : mc) {
                    const double G = gaunt_real(l2, m2, ls, ms, l1, m1);
                    if (std::abs(G) > 1e-15) lst.emplace_back(lm_to_idx(ls, ms), G);
                }
            }
            std::sort(lst.begin(), lst.end());
        }
    });
    P.ptr.assign(np + 1, 0);
    for (int i = 0; i < np; ++i) P.ptr[i + 1] = P.ptr[i] + (int)per[i].size();
    P.sig.resize(P.ptr[np]);
    P.G.resize(P.ptr[np]);
    for (int i = 0; i < np; ++i)
        for (size_t k = 0; k < per[i].size(); ++k) {
            P.sig[P.ptr[i] + k] = per[i][k].first;
            P.G[P.ptr[i] + k] = per[i][k].second;
        }
    return P;
}

ExchCSR build_exchange(int n_mu, int n_sigma, int n_lambda) {
    ExchCSR X;
    const int rows = n_mu * n_sigma;
    std::vector<std::vector<std::pair<int, double>>> per(rows);
    parallel_for(n_mu, [&](int mu) {
        int lm, mm;
        idx_to_lm(mu, lm, mm);
        std::vector<int> mc;
        for (int s = 0; s < n_sigma; ++s) {
            int ls, ms;
            idx_to_lm(s, ls, ms);
            auto& lst = per[mu * n_sigma + s];
            for (int ll = std::abs(lm - ls); ll <= lm + ls; ++ll) {
                if ((lm + ll + ls) & 1) continue;
                m_candidates(mm, ms, ll, mc);
                for (int ml : mc) {
                    const int lam = lm_to_idx(ll, ml);
                    if (lam >= n_lambda) continue;
                    // build_G_vector keeps |gaunt_real(l_mu, m_mu, l_lambda, m_lambda, l_sigma, m_sigma)| > 1e-14
                    const double v = gaunt_real(lm, mm, ll, ml, ls, ms);
                    if (std::abs(v) > 1e-14) lst.emplace_back(lam, v);
                }
            }
            std::sort(lst.begin(), lst.end());
        }
    });
    X.ptr.assign(rows + 1, 0);
    for (int i = 0; i < rows; ++i) X.ptr[i + 1] = X.ptr[i] + (int)per[i].size();
    X.lam.resize(X.ptr[rows]);
    X.G.resize(X.ptr[rows]);
    X.n_lambda_max = 0;
    for (int i = 0; i < rows; ++i)
        for (size_t k = 0; k < per[i].size(); ++k) {
            X.lam[X.ptr[i] + k] = per[i][k].first;
            X.G[X.ptr[i] + k] = per[i][k].second;
            X.n_lambda_max = std::max(X.n_lambda_max, per[i][k].first + 1);
        }
    return X;
}

DipCSR build_dipole_tables(int n_mu, int n_lambda) {
    DipCSR D;
    const int qs[3] = {+1, -1, 0};       // x, y, z
    for (int qi = 0; qi < 3; ++qi) {
        auto& ptr = D.ptr[qi];
        auto& nu = D.nu[qi];
        auto& a = D.a[qi];
        auto& c = D.c[qi];
        ptr.assign(n_mu + 1, 0);
        for (int mu = 0; mu < n_mu; ++mu) {
            int lmu, mmu;
            idx_to_lm(mu, lmu, mmu);
            for (int lnu = std::max(0, lmu - 1); lnu <= lmu + 1; ++lnu) {
                if (std::abs(lmu - lnu) != 1) continue;
                for (int mnu = -lnu; mnu <= lnu; ++mnu) {
                    const int v = lm_to_idx(lnu, mnu);
                    if (v >= n_lambda) continue;
                    const double av = angular_dipole(lmu, mmu, qs[qi], lnu, mnu);
                    if (av != 0.0) {
                        nu.push_back(v);
                        a.push_back(av);
                        c.push_back(velocity_coef(lmu, lnu));
                    }
                }
            }
            ptr[mu + 1] = (int)nu.size();
        }
    }
    return D;
}

std::vector<double> simpson_weights(int n, double h) {
    std::vector<double> w(std::max(n, 0), 0.0);
    if (n < 2) return w;
    if (n == 2) { w[0] = w[1] = 0.5 * h; return w; }
    auto one_third = [&](int m) {
        w[0] += h / 3.0;
        w[m - 1] += h / 3.0;
        for (int i = 1; i < m - 1; i += 2) w[i] += 4.0 * h / 3.0;
        for (int i = 2; i < m - 2; i += 2) w[i] += 2.0 * h / 3.0;
    };
    if (n % 2 == 1) { one_third(n); return w; }
    if (n < 4) {
        for (int i = 0; i < n; ++i) w[i] = h * ((i == 0 || i == n - 1) ? 0.5 : 1.0);
        return w;
    }
    one_third(n - 3);
    w[n - 4] += 3.0 * h / 8.0;
    w[n - 3] += 9.0 * h / 8.0;
    w[n - 2] += 9.0 * h / 8.0;
    w[n - 1] += 3.0 * h / 8.0;
    return w;
}

void five_point_derivative(const double* f, int n, double dr, double* df) {
    if (n < 5) {
        if (n >= 2) {
            df[0] = (f[1] - f[0]) / dr;
            for (int i = 1; i < n - 1; ++i) df[i] = (f[i + 1] - f[i - 1]) / (2.0 * dr);
            df[n - 1] = (f[n - 1] - f[n - 2]) / dr;
        } else if (n == 1) {
            df[0] = 0.0;
        }
        return;
    }
    const double c = 1.0 / (12.0 * dr);
    for (int i = 2; i < n - 2; ++i) df[i] = (-f[i + 2] + 8.0 * f[i + 1] - 8.0 * f[i - 1] + f[i - 2]) * c;
    df[0] = (-25.0 * f[0] + 48.0 * f[1] - 36.0 * f[2] + 16.0 * f[3] - 3.0 * f[4]) * c;
    df[1] = (-3.0 * f[0] - 10.0 * f[1] + 18.0 * f[2] - 6.0 * f[3] + 1.0 * f[4]) * c;
    df[n - 2] = (-1.0 * f[n - 5] + 6.0 * f[n - 4] - 18.0 * f[n - 3] + 10.0 * f[n - 2] + 3.0 * f[n - 1]) * c;
    df[n - 1] = (3.0 * f[n - 5] - 16.0 * f[n - 4] + 36.0 * f[n - 3] - 48.0 * f[n - 2] + 25.0 * f[n - 1]) * c;
}

}  // namespace scatt
