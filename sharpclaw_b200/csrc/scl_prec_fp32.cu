// Kernel instantiations of one arithmetic form (SCL_FP32).
#define SCL_PREC_VALUE SCL_FP32
#define SCL_PREC_NS prec_fp32
#define SCL_PREC_GETTER get_launchers_fp32
#define SCL_BATCH_GETTER get_batch_launchers_fp32
#include "scl_dispatch.cuh"
