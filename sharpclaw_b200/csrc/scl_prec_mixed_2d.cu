// Kernel instantiations of one arithmetic form (SCL_MIXED): the 2-D stage kernels.
#define SCL_PREC_VALUE SCL_MIXED
#define SCL_PREC_NS prec_mixed_2d
#define SCL_PREC_GETTER_2D get_launchers_mixed_2d
#define SCL_PART 2
#include "scl_dispatch.cuh"
