// Kernel instantiations of one arithmetic form (SCL_FP64_STRICT): the 1-D and batched
// stage kernels (the 2-D ones are in scl_prec_fp64s_2d.cu).
#define SCL_PREC_VALUE SCL_FP64_STRICT
#define SCL_PREC_NS prec_fp64s
#define SCL_PREC_GETTER get_launchers_fp64s
#define SCL_PREC_GETTER_2D get_launchers_fp64s_2d
#define SCL_BATCH_GETTER get_batch_launchers_fp64s
#define SCL_PART 1
#include "scl_dispatch.cuh"
