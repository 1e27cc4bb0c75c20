// Reference-side binding of librsgpu: declarations of the explicit
// specialisations that move RockSeis's float hot path onto the GPU.
//
// Compile lib/modelling.cpp and lib/fwi.cpp of the reference with this header
// force-included (`-include rockseis_gpu.h`): the declarations then precede the
// libraries' own `template class ModellingAcoustic2D<float>;` (and the other
// explicit instantiations), which therefore leave these members to the
// definitions in rockseis_gpu.cpp.  Every other member, and every double
// instantiation, keeps the reference's CPU code.
#pragma once
#include "modelling.h"
#include "fwi.h"

namespace rockseis {
template <> int ModellingAcoustic2D<float>::run();     // lib/modelling.cpp:197-291
template <> int ModellingElastic2D<float>::run();      // lib/modelling.cpp:545-645
template <> int FwiAcoustic2D<float>::run_optimal();   // lib/fwi.cpp:1159-1332
}  // namespace rockseis
