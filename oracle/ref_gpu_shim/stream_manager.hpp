// TEST INFRASTRUCTURE ONLY. Stand-in for CPPuddle's stream_manager.hpp (the
// stream pools of the reference's CUDA backend); see cuda_helper.hpp here.
#pragma once
