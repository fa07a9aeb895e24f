// scatt/GpuDipoleEngine.hpp -- libscatt_b200 in place of the reference's
// src/scatt/GpuDipoleEngine.hpp: the per-radial-point dipole GEMM of
// DipoleMatrixElement.cpp:751-827, as scatt_b200::GpuDipoleEngine (one
// device GEMM per call on the calling thread's current device).
#pragma once

#include "scatt/GpuPropagate.hpp"

namespace scatt {

class GpuDipoleEngine : public scatt_b200::GpuDipoleEngine {
public:
    using scatt_b200::GpuDipoleEngine::GpuDipoleEngine;
};

}  // namespace scatt
