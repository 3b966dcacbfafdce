// TEST INFRASTRUCTURE ONLY. Stand-in for octotiger/config.hpp (which pulls in
// HPX) when oracle/build_ref.sh compiles the reference's octotiger/taylor.hpp:
// only the serialization trait that taylor.hpp specialises is needed.
#pragma once
namespace hpx {
namespace traits {
template <class T>
struct is_bitwise_serializable {};
}   // namespace traits
}   // namespace hpx
