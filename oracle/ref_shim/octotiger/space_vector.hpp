// TEST INFRASTRUCTURE ONLY. Stand-in for octotiger/space_vector.hpp (HPX and
// Vc types) when oracle/build_ref.sh compiles the reference's
// octotiger/taylor.hpp, which only needs the definitions of defs.hpp.
#pragma once
#include "octotiger/defs.hpp"
