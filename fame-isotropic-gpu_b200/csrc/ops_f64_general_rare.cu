// Operator stage kernels, FP64, General lattices, radix 7, 11, 13 (no passes for primes >= 17).
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, true, IN_CG, false, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, false, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, true, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_REFINE, false, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_pencil<double, true, PEN_QBQ, 1, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QR_OUT, 1, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QRS_IN, 1, DynGeom>(PencilArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_CG, false, 1, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, false, 1, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, true, 1, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_RESID, false, 1, DynGeom>(PlaneOutArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f64_general_rare)
}  // namespace fame
