// fvt_kernels_f32.cu -- the FP32 (mixed-precision) instantiations of the stage and
// output kernels: fvt_kernels.cu compiled a second time with STORM_FVT_F32_TU, which
// leaves out everything but the templates and the *_f32 entry points, and built with
// FMA contraction allowed (storm_b200/build.py).  The FP64 path, whose results must
// round exactly as the reference's expressions, is compiled only in fvt_kernels.cu
// with --fmad=false.
#define STORM_FVT_F32_TU 1
#include "fvt_kernels.cu"
