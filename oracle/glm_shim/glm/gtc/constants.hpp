// glm-subset shim, constants: TEST INFRASTRUCTURE ONLY (see ../glm.hpp).
#ifndef PXB_GLM_SHIM_CONSTANTS_HPP
#define PXB_GLM_SHIM_CONSTANTS_HPP

#include <limits>

#include "../glm.hpp"

namespace glm {
template <typename T> constexpr T pi() { return static_cast<T>(3.14159265358979323846264338327950288); }
template <typename T> constexpr T epsilon() { return std::numeric_limits<T>::epsilon(); }
}  // namespace glm

#endif  // PXB_GLM_SHIM_CONSTANTS_HPP
