// Explicit instantiation: precision double, initial-state class 2.
#include "fg_adjoint.cuh"
template struct fg::Launch<double, 2>;
