#pragma once
// ORACLE SHIM: see shim_dense.hpp.
#include "shim_dense.hpp"
