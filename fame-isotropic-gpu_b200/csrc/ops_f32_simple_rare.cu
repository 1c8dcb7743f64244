// Operator stage kernels, FP32, Simple lattices, all radices (7, 11, 13, large primes).
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<float, false, IN_CG, false, true, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, false, true, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, true, true, DynGeom>(PlaneInArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ, true, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QR_OUT, true, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QRS_IN, true, DynGeom>(PencilArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_CG, false, true, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, false, true, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, true, true, DynGeom>(PlaneOutArgs<float>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f32_simple_rare)
}  // namespace fame
