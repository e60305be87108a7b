// TEST INFRASTRUCTURE ONLY (oracle/_ref build).  Stands in for yomm2's
// "yorel/yomm2/cute.hpp" (absent here) when the reference's own sources are
// compiled into the CPU oracle: the macros declare_method / define_method /
// register_class and the marker virtual_ come from the engine's C++
// multimethod layer, which implements the same resolution rule.
#ifndef FRANK_ORACLE_YOMM2_SHIM_HPP
#define FRANK_ORACLE_YOMM2_SHIM_HPP

#include "frank_b200/multimethod.hpp"

namespace yorel {
namespace yomm2 {
using ::frank_mm::virtual_;
inline void update_methods() { ::frank_mm::update_methods(); }
}  // namespace yomm2
}  // namespace yorel

#endif
