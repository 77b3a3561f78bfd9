// Kernel instantiations of one arithmetic form (SCL_MIXED).
#define SCL_PREC_VALUE SCL_MIXED
#define SCL_PREC_NS prec_mixed
#define SCL_PREC_GETTER get_launchers_mixed
#define SCL_BATCH_GETTER get_batch_launchers_mixed
#include "scl_dispatch.cuh"
