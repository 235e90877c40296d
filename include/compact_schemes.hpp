// compact_schemes.hpp -- all drop-in headers of libcompact_b200.
#pragma once
#include "compact_schemes/common.hpp"
#include "compact_schemes/numerics_pc.hpp"
#include "compact_schemes/physics_pc.hpp"
#include "compact_schemes/gcbc.hpp"
