// precision.cuh -- arithmetic forms of the kernels (values of gx_precision in include/gx.h).
#pragma once

namespace gx {

enum Precision : int { kF64 = 0, kMixed = 1, kF64Exact = 2 };

}  // namespace gx
