// Operator stage kernels, FP32, General lattices, radix 7, 11, 13 (no passes for primes >= 17).
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<float, true, IN_CG, false, 1, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, true, IN_VEC, false, 1, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, true, IN_VEC, true, 1, DynGeom>(PlaneInArgs<float>);
template __global__ void k_pencil<float, true, PEN_QBQ, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, true, PEN_QBQ_CG, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, true, PEN_QR_OUT, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, true, PEN_QRS_IN, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_plane_fwd<float, true, EPI_CGR, false, 1, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, true, EPI_OUT, false, 1, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, true, EPI_OUT, true, 1, DynGeom>(PlaneOutArgs<float>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f32_general_rare)
}  // namespace fame
