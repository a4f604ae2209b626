// Explicit instantiation: precision float, initial-state class 3.
#include "fg_adjoint.cuh"
template struct fg::Launch<float, 3>;
