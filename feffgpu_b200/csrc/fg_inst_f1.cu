// Explicit instantiation: precision float, initial-state class 1.
#include "fg_adjoint.cuh"
template struct fg::Launch<float, 1>;
template struct fg::LaunchCommon<float>;
