// scatt/GpuPropagate.hpp -- libscatt_b200 in place of the reference's
// src/scatt/GpuPropagate.hpp.  The same classes, in namespace scatt, with
// the constructors and methods the reference's stage classes call
// (SchurInverter.cpp:191-313, ForwardRPropagator.cpp:261-312,
// BackPropagator.cpp:559-645); the implementation is scatt_b200.hpp over the
// library's per-step entry points.  Build the reference with
// spion-emol_b200/host/seam ahead of its src/ on the include path, and with
// its own GpuPropagate and GpuDipoleEngine sources left out.
#pragma once

#include "scatt_b200.hpp"

namespace scatt {

class GpuContext : public scatt_b200::GpuContext {
public:
    using scatt_b200::GpuContext::GpuContext;
};

class GpuForwardStepper : public scatt_b200::GpuForwardStepper {
public:
    using scatt_b200::GpuForwardStepper::GpuForwardStepper;
};

class GpuSinvStepper : public scatt_b200::GpuSinvStepper {
public:
    using scatt_b200::GpuSinvStepper::GpuSinvStepper;
};

class GpuBackStepper : public scatt_b200::GpuBackStepper {
public:
    using scatt_b200::GpuBackStepper::GpuBackStepper;
};

}  // namespace scatt
