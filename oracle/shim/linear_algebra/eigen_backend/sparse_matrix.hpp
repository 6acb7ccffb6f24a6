#pragma once
// ORACLE SHIM: see shim_sparse.hpp.
#include "shim_sparse.hpp"
