// Operator stage kernels, FP32, General lattices, radix 7, 11, 13 and primes >= 17.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<float, true, IN_CG, false, 2, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, true, IN_VEC, false, 2, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, true, IN_VEC, true, 2, DynGeom>(PlaneInArgs<float>);
template __global__ void k_pencil<float, true, PEN_QBQ, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, true, PEN_QBQ_CG, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, true, PEN_QR_OUT, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, true, PEN_QRS_IN, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_plane_fwd<float, true, EPI_CGR, false, 2, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, true, EPI_OUT, false, 2, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, true, EPI_OUT, true, 2, DynGeom>(PlaneOutArgs<float>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f32_general_prime)
}  // namespace fame
