// Explicit instantiation: precision float, initial-state class 2 at lambda order 3.
#include "fg_adjoint.cuh"
template struct fg::Launch<float, 5>;
