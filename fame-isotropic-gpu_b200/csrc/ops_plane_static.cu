// Plane stage kernels of runtime-geometry General lattices whose plane axes have
// static plans (DynGeomPlane): FCC 64x55x52 (fast 52, mid 55), BCC 48x45x39 (fast 39,
// mid 45) and the hexagonal 128x107x92 grid (fast 92, mid 107), FP32 and FP64.
#include "op_kernels.cuh"

namespace fame {
#define FAME_PLANES_F32(GP)                                                                            \
  template __global__ void k_plane_inv<float, true, IN_CG, false, 0, GP>(PlaneInArgs<float>);         \
  template __global__ void k_plane_inv<float, true, IN_VEC, false, 0, GP>(PlaneInArgs<float>);        \
  template __global__ void k_plane_inv<float, true, IN_VEC, true, 0, GP>(PlaneInArgs<float>);         \
  template __global__ void k_plane_fwd<float, true, EPI_CGR, false, 0, GP>(PlaneOutArgs<float>);      \
  template __global__ void k_plane_fwd<float, true, EPI_OUT, false, 0, GP>(PlaneOutArgs<float>);      \
  template __global__ void k_plane_fwd<float, true, EPI_OUT, true, 0, GP>(PlaneOutArgs<float>);
#define FAME_PLANES_F64(GP)                                                                            \
  template __global__ void k_plane_inv<double, true, IN_CG, false, 0, GP>(PlaneInArgs<double>);       \
  template __global__ void k_plane_inv<double, true, IN_VEC, false, 0, GP>(PlaneInArgs<double>);      \
  template __global__ void k_plane_inv<double, true, IN_VEC, true, 0, GP>(PlaneInArgs<double>);       \
  template __global__ void k_plane_inv<double, true, IN_REFINE, false, 0, GP>(PlaneInArgs<double>);   \
  template __global__ void k_plane_fwd<double, true, EPI_CG, false, 0, GP>(PlaneOutArgs<double>);     \
  template __global__ void k_plane_fwd<double, true, EPI_OUT, false, 0, GP>(PlaneOutArgs<double>);    \
  template __global__ void k_plane_fwd<double, true, EPI_OUT, true, 0, GP>(PlaneOutArgs<double>);     \
  template __global__ void k_plane_fwd<double, true, EPI_RESID, false, 0, GP>(PlaneOutArgs<double>);
FAME_PLANES_F32(PlaneFcc64)
FAME_PLANES_F64(PlaneFcc64)
FAME_PLANES_F32(PlaneBcc48)
FAME_PLANES_F64(PlaneBcc48)
FAME_PLANES_F32(PlaneHex128f)
FAME_PLANES_F64(PlaneHex128d)
#undef FAME_PLANES_F32
#undef FAME_PLANES_F64
FAME_DEFINE_LAUNCH_GETTER(launches_ops_plane_static)
}  // namespace fame
