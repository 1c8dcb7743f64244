// Operator stage kernels, FP32, Simple lattices, radices 2, 3, 4, 5, 8.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<float, false, IN_CG, false, 0, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, false, 0, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, true, 0, DynGeom>(PlaneInArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ, 0, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ_CG, 0, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QR_OUT, 0, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QRS_IN, 0, DynGeom>(PencilArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_CGR, false, 0, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, false, 0, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, true, 0, DynGeom>(PlaneOutArgs<float>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f32_simple)
}  // namespace fame
