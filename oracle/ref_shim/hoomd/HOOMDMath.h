// Minimal stand-in for HOOMD-blue's hoomd/HOOMDMath.h (HOOMD is not
// installed): the reference evaluator only needs the Scalar type. Double
// precision, as in a HOOMD double build.
#pragma once
#include <cmath>
typedef double Scalar;
