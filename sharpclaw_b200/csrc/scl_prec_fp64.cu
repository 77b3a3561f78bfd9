// Kernel instantiations of one arithmetic form (SCL_FP64).
#define SCL_PREC_VALUE SCL_FP64
#define SCL_PREC_NS prec_fp64
#define SCL_PREC_GETTER get_launchers_fp64
#define SCL_BATCH_GETTER get_batch_launchers_fp64
#include "scl_dispatch.cuh"
