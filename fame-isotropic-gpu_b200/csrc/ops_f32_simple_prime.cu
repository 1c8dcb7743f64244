// Operator stage kernels, FP32, Simple lattices, radix 7, 11, 13 and primes >= 17.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<float, false, IN_CG, false, 2, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, false, 2, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, true, 2, DynGeom>(PlaneInArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ_CG, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QR_OUT, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QRS_IN, 2, DynGeom>(PencilArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_CGR, false, 2, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, false, 2, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, true, 2, DynGeom>(PlaneOutArgs<float>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f32_simple_prime)
}  // namespace fame
