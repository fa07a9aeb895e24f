// The C++ host interface's psi store and continuum-continuum dipole calls
// (ScanSolver::psi / psi_into, compute_cc_dipole), compiled as a caller
// writes them.  Without a device every call throws the library's no-device
// message; with one, the GPU tests cover the numbers.
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "scatt_b200.hpp"

namespace {

bool throws_no_device(void (*f)()) {
    try {
        f();
    } catch (const std::runtime_error& e) {
        return std::string(e.what()).find("no CUDA device") != std::string::npos;
    }
    return false;
}

void cc_call() {
    std::vector<scatt_b200::Matrix> a(6, scatt_b200::Matrix(4, 4)), b(6, scatt_b200::Matrix(4, 4));
    scatt_b200::Matrix cc = scatt_b200::compute_cc_dipole(a, b, 0, 0.05, 'z');
    std::cout << cc.rows << "\n";
}

void psi_call() {
    scatt_b200::ScanInputs in;
    in.Nr = 101;
    in.dr = 0.05;
    in.l_cont = 1;
    scatt_b200::ScanSolver sol(in);
    std::vector<std::vector<scatt_b200::Matrix>> psi = sol.psi({0.5}, 0, 50, 16, true);
    std::vector<double> flat;
    sol.psi_into({0.5}, 0, 50, 16, true, flat);
    std::cout << psi.size() << " " << flat.size() << "\n";
}

}  // namespace

int main() {
    int n = 0;
    scatt_device_count(&n);
    if (n > 0) {
        std::cout << "compiled; a device is visible, the no-device checks do not apply\n";
        return 0;
    }
    if (!throws_no_device(cc_call)) return 10;
    if (!throws_no_device(psi_call)) return 11;
    std::cout << "ok\n";
    return 0;
}
