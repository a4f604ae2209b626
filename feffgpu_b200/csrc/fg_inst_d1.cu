// Explicit instantiation: precision double, initial-state class 1.
#include "fg_adjoint.cuh"
template struct fg::Launch<double, 1>;
template struct fg::LaunchCommon<double>;
