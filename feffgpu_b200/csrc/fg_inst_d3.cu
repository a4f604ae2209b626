// Explicit instantiation: precision double, initial-state class 3.
#include "fg_adjoint.cuh"
template struct fg::Launch<double, 3>;
