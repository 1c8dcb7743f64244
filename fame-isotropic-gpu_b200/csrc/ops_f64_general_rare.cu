// Operator stage kernels, FP64, General lattices, all radices (7, 11, 13, large primes).
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, true, IN_CG, false, true, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, false, true, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, true, true, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_REFINE, false, true, DynGeom>(PlaneInArgs<double>);
template __global__ void k_pencil<double, true, PEN_QBQ, true, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QR_OUT, true, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QRS_IN, true, DynGeom>(PencilArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_CG, false, true, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, false, true, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, true, true, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_RESID, false, true, DynGeom>(PlaneOutArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f64_general_rare)
}  // namespace fame
