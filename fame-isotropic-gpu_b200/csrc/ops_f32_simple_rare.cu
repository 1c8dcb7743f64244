// Operator stage kernels, FP32, Simple lattices, radix 7, 11, 13 (no passes for primes >= 17).
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<float, false, IN_CG, false, 1, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, false, 1, DynGeom>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, true, 1, DynGeom>(PlaneInArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ_CG, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QR_OUT, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QRS_IN, 1, DynGeom>(PencilArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_CGR, false, 1, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, false, 1, DynGeom>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, true, 1, DynGeom>(PlaneOutArgs<float>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f32_simple_rare)
}  // namespace fame
