// glm-subset shim: TEST INFRASTRUCTURE ONLY (see ../glm.hpp). The reference includes this
// header but its cloth/hair closure calls none of its transforms.
#ifndef PXB_GLM_SHIM_MATRIX_TRANSFORM_HPP
#define PXB_GLM_SHIM_MATRIX_TRANSFORM_HPP
#include "../glm.hpp"
#endif
