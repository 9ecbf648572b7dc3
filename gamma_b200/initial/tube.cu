// Problem module: planar relativistic shock tubes after
// src/Initial/Tests/1DST.cpp, run with cartesian + rel_cart.  1DST has no
// kinematics, boundary, source or regrid hooks (1DST.cpp:81-128), so this
// module keeps every default.  The tubes are set up on the host in Python
// (gamma_b200/problems.py, TubeSetup).
#include "problem_module.cuh"

namespace {
struct Tube : gamma_problem::Problem {};
}  // namespace

GAMMA_PROBLEM_MODULE("tube", Tube, gamma_problem::MODULES_CARTESIAN, GAMMA_PROBLEM_TUBE)
