// TEST INFRASTRUCTURE ONLY. Stand-in for the reference's options header when
// its stencil generators are compiled by oracle/build_ref.sh: the generators
// read only opts().theta.
#pragma once
#include <iostream>
#include <sstream>
struct otfmm_ref_opts {
    double theta;
};
otfmm_ref_opts& opts();
