// Kernel instantiations of one arithmetic form (SCL_FP64): the 2-D stage kernels.
#define SCL_PREC_VALUE SCL_FP64
#define SCL_PREC_NS prec_fp64_2d
#define SCL_PREC_GETTER_2D get_launchers_fp64_2d
#define SCL_PART 2
#include "scl_dispatch.cuh"
