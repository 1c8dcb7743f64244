// Operator stage kernels, FP64, General lattices, radix 7, 11, 13 and primes >= 17.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, true, IN_CG, false, 2, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, false, 2, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, true, 2, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_REFINE, false, 2, DynGeom>(PlaneInArgs<double>);
template __global__ void k_pencil<double, true, PEN_QBQ, 2, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QR_OUT, 2, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QRS_IN, 2, DynGeom>(PencilArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_CG, false, 2, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, false, 2, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, true, 2, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_RESID, false, 2, DynGeom>(PlaneOutArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f64_general_prime)
}  // namespace fame
