// Scalar type of the solver build (float: FP32 sweeps; double: the FP64 build).
#ifndef TYPES_H
#define TYPES_H
using scalar = float;
#endif
