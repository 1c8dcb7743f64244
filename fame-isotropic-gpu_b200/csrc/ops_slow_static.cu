// Pencil stage kernels of runtime-geometry General lattices whose slow axis has a
// static plan (DynGeomSlow): the slow-axis lengths 48, 64 and 128, FP32 and FP64.
#include "op_kernels.cuh"

namespace fame {
#define FAME_SLOW_PENCILS(LS)                                                                 \
  template __global__ void k_pencil<float, true, PEN_QBQ, 0, DynGeomSlow<LS>>(PencilArgs<float>);      \
  template __global__ void k_pencil<float, true, PEN_QBQ_CG, 0, DynGeomSlow<LS>>(PencilArgs<float>);   \
  template __global__ void k_pencil<float, true, PEN_QR_OUT, 0, DynGeomSlow<LS>>(PencilArgs<float>);   \
  template __global__ void k_pencil<float, true, PEN_QRS_IN, 0, DynGeomSlow<LS>>(PencilArgs<float>);   \
  template __global__ void k_pencil<double, true, PEN_QBQ, 0, DynGeomSlow<LS>>(PencilArgs<double>);    \
  template __global__ void k_pencil<double, true, PEN_QR_OUT, 0, DynGeomSlow<LS>>(PencilArgs<double>); \
  template __global__ void k_pencil<double, true, PEN_QRS_IN, 0, DynGeomSlow<LS>>(PencilArgs<double>);
FAME_SLOW_PENCILS(48)
FAME_SLOW_PENCILS(64)
FAME_SLOW_PENCILS(128)
#undef FAME_SLOW_PENCILS
FAME_DEFINE_LAUNCH_GETTER(launches_ops_slow_static)
}  // namespace fame
