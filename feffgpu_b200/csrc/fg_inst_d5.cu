// Explicit instantiation: precision double, initial-state class 2 at lambda order 3.
#include "fg_adjoint.cuh"
template struct fg::Launch<double, 5>;
