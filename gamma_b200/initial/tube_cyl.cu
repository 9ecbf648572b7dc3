// Problem module: planar shock tubes (as tube.cu, src/Initial/Tests/1DST.cpp's
// hooks, all defaults) run with cartesian + rel_cyl, the reference's
// Hydro/rel_cyl.cpp module: its source term p/r acts on S_r with r the cell
// centre, so tubes are laid on x > 0.  Set up on the host in Python
// (gamma_b200/problems.py, TubeSetup).
#include "problem_module.cuh"

namespace {
struct TubeCyl : gamma_problem::Problem {};
}  // namespace

GAMMA_PROBLEM_MODULE("tube_cyl", TubeCyl, gamma_problem::MODULES_CARTESIAN_REL_CYL, -1)
