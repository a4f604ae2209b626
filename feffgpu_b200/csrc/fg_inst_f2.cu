// Explicit instantiation: precision float, initial-state class 2.
#include "fg_adjoint.cuh"
template struct fg::Launch<float, 2>;
