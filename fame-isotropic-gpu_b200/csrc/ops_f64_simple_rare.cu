// Operator stage kernels, FP64, Simple lattices, radix 7, 11, 13 (no passes for primes >= 17).
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, false, IN_CG, false, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_VEC, false, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_VEC, true, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_REFINE, false, 1, DynGeom>(PlaneInArgs<double>);
template __global__ void k_pencil<double, false, PEN_QBQ, 1, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, false, PEN_QR_OUT, 1, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, false, PEN_QRS_IN, 1, DynGeom>(PencilArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_CG, false, 1, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_OUT, false, 1, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_OUT, true, 1, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_RESID, false, 1, DynGeom>(PlaneOutArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f64_simple_rare)
}  // namespace fame
