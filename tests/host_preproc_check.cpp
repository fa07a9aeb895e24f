// The C++ preprocessing interface (host/scatt_preproc.hpp) as the
// reference's preprocessing driver would call it: the Molden reader on a
// small file (host-only, checked), and the device steps -- which without a
// device throw the library's no-device message.
#include <cmath>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>

#include "scatt_preproc.hpp"

namespace pp = scatt_b200::preproc;

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string path = std::string(argv[1]) + "/h.molden";
    {
        std::ofstream f(path);
        f << "[Molden Format]\n[Atoms] AU\nH 1 1 0.0 0.0 0.7\nH 2 1 0.0 0.0 -0.7\n[GTO]\n"
             "  1 0\n s 2 1.0\n  1.3D+00 0.6\n  0.2D+00 0.5\n p 1 1.0\n  0.8 1.0\n\n"
             "  2 0\n s 2 1.0\n  1.3D+00 0.6\n  0.2D+00 0.5\n p 1 1.0\n  0.8 1.0\n\n"
             "[MO]\n Sym= Ag\n Ene= -0.59\n Spin= Alpha\n Occup= 2.0\n 1 0.5\n 2 0.1\n 5 0.5\n 6 0.1\n";
    }
    const pp::MoldenFile m = pp::read_molden(path);
    if (m.nbf != 8 || m.shells.size() != 4 || m.alpha.C.rows != 1 || m.beta.C.rows != 0) return 10;
    if (m.atoms[0] != 1.0 || m.atoms[3] != 0.7 || m.shells[3].center[2] != -0.7) return 11;
    if (std::fabs(m.shells[0].exponents[0] - 1.3) > 1e-15 || m.alpha.C(0, 4) != 0.5 || m.alpha.occ[0] != 2.0) return 12;
    int n = 0;
    scatt_device_count(&n);
    if (n > 0) {
        std::cout << "compiled; a device is visible, the no-device checks do not apply\n";
        return 0;
    }
    const double origin[3] = {0.0, 0.0, 0.0};
    try {
        pp::project_basis(m, m.alpha, 4, 11, 0.0, 0.2, origin, 1);
        return 13;
    } catch (const std::runtime_error& e) {
        if (std::string(e.what()).find("no CUDA device") == std::string::npos) return 14;
    }
    try {
        pp::build_V_H(scatt_b200::Matrix(25, 11), 0.2, 4);
        return 15;
    } catch (const std::runtime_error& e) {
        if (std::string(e.what()).find("no CUDA device") == std::string::npos) return 16;
    }
    std::cout << "ok\n";
    return 0;
}
