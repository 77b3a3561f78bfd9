// Kernel instantiations of one arithmetic form (SCL_FP64_STRICT).
#define SCL_PREC_VALUE SCL_FP64_STRICT
#define SCL_PREC_NS prec_fp64s
#define SCL_PREC_GETTER get_launchers_fp64s
#define SCL_BATCH_GETTER get_batch_launchers_fp64s
#include "scl_dispatch.cuh"
