// Explicit instantiation: precision float, initial-state class 3 at lambda order 3.
#include "fg_adjoint.cuh"
template struct fg::Launch<float, 6>;
