// Operator stage kernels, FP64, General lattices, radices 2, 3, 4, 5, 8.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, true, IN_CG, false, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, false, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_VEC, true, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, true, IN_REFINE, false, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_pencil<double, true, PEN_QBQ, false, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QR_OUT, false, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, true, PEN_QRS_IN, false, DynGeom>(PencilArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_CG, false, false, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, false, false, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_OUT, true, false, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, true, EPI_RESID, false, false, DynGeom>(PlaneOutArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f64_general)
}  // namespace fame
