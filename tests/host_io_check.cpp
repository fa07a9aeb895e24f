// Exercises the C++ I/O interface (host/scatt_io.hpp): a dipole scan written
// by DipoleWriter and read back by DipoleReader must match bit for bit; with
// a preprocessing file as argv[2], HDF5Reader's header and scan description
// are printed for the calling test to compare.
#include <cmath>
#include <cstdio>
#include <random>

#include "scatt_io.hpp"

using namespace scatt_b200;

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    try {
        std::mt19937_64 g(7);
        std::normal_distribution<double> nd;
        const int n = 9, no = 2;
        DipoleScanMeta m;
        m.dr = 0.01;
        m.N_grid = 4001;
        m.l_max_continuum = 2;
        m.kgrid = EnergyGrid{0.1, 1, 21};
        m.E_HOMO = -0.6;
        m.occ_energies = {-1.1, -0.6};
        m.occ_spin_factors = {2.0, 2.0};
        m.atoms = {{1, 0.0, 0.0, 0.7}, {1, 0.0, 0.0, -0.7}};
        m.molecule_name = "h2_like";
        DipoleWriter w(argv[1], m);
        DipoleEnergyPayload p;
        p.ik = 3;
        p.A = Matrix(n, n);
        p.B = Matrix(n, n);
        p.b_overlap = Matrix(n, no);
        for (auto& x : p.A.data) x = nd(g);
        for (auto& x : p.B.data) x = nd(g);
        for (auto& x : p.b_overlap.data) x = nd(g);
        for (int s = 5; s >= 0; --s) {          // slices in reverse: placed by their own labels
            DipoleSlice& sl = p.slices[5 - s];
            sl.gauge = static_cast<DipoleGauge>(s / 3);
            sl.pol = static_cast<Polarization>(s % 3);
            for (int i = 0; i < n; ++i) {
                sl.D_reduced.emplace_back(nd(g), nd(g));
                sl.D_reduced_raw.emplace_back(nd(g), nd(g));
                sl.d_raw.push_back(nd(g));
            }
            for (int i = 0; i < no; ++i) sl.d_correction.push_back(nd(g));
            sl.partial_sigma = std::fabs(nd(g));
        }
        p.fit_residual_rel = 1e-11;
        p.K_symmetry_err = 2e-13;
        if (w.has_energy(3)) return 3;
        w.write_energy(p);
        if (!w.has_energy(3)) return 4;
        w.finalize();
        DipoleReader r(argv[1]);
        const auto back = r.read_energy(3);
        bool ok = r.available_ik() == std::vector<int>{3} && back.A.data == p.A.data && back.B.data == p.B.data &&
                  back.b_overlap.data == p.b_overlap.data && back.k == 3 * 0.1 && back.E == 0.5 * (3 * 0.1) * (3 * 0.1) &&
                  back.fit_residual_rel == 1e-11 && r.meta().molecule_name == "h2_like" &&
                  r.meta().atoms.size() == 2 && r.meta().kgrid.ik_max == 21;
        for (const auto& sl : p.slices) {
            const auto& b = back.slices[DipoleWriter::slice_index(sl.gauge, sl.pol)];
            ok = ok && b.D_reduced == sl.D_reduced && b.D_reduced_raw == sl.D_reduced_raw && b.d_raw == sl.d_raw &&
                 b.d_correction == sl.d_correction && b.partial_sigma == sl.partial_sigma;
        }
        std::printf("dipole %s\n", ok ? "ok" : "MISMATCH");
        if (!ok) return 1;
        if (argc > 2) {
            HDF5Reader h(argv[2]);
            const PreprocData d = h.load_header();
            double E_init = 0.0;
            const scatt_scan_desc s = h.scan_desc(3, &E_init);
            std::printf("preproc %zu %d %d %d %d %d %d %d %.17g %.17g %.17g\n", d.Nr, d.Lmax_sce, d.n_alpha,
                        d.n_occ_alpha, d.n_sce, d.Nlm_orb_store, d.Nr_orb_store, d.has_initial_state ? 1 : 0, d.rmin,
                        d.dr, d.orb_energies.empty() ? 0.0 : d.orb_energies.back());
            std::printf("desc %d %d %d %d %d %d %d %.17g %.17g\n", s.n_orb, s.Nlm_store, s.Nr_store, s.init_state,
                        s.n_H, s.n_occ, s.n_atoms, s.psi_lm[1], E_init);
        }
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
        return 5;
    }
    return 0;
}
