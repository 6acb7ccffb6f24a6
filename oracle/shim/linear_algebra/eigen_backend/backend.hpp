#pragma once
// ORACLE SHIM (test infrastructure only): mirrors the reference's
// src/linear_algebra/eigen_backend/backend.hpp, which also makes the saddle
// preconditioner dispatch specialisation visible.
#include "backend_types.hpp"
#include "preconditioners/solve_saddle_system.hpp"
