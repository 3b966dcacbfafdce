// TEST INFRASTRUCTURE ONLY. Stand-in for octotiger/profiler.hpp (HPX timers)
// when oracle/build_ref.sh compiles the reference's octotiger/taylor.hpp.
#pragma once
#define PROFILE()
