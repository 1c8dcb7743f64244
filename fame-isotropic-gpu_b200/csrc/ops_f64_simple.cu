// Operator stage kernels, FP64, Simple lattices, radices 2, 3, 4, 5, 8.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, false, IN_CG, false, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_VEC, false, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_VEC, true, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_REFINE, false, false, DynGeom>(PlaneInArgs<double>);
template __global__ void k_pencil<double, false, PEN_QBQ, false, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, false, PEN_QR_OUT, false, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, false, PEN_QRS_IN, false, DynGeom>(PencilArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_CG, false, false, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_OUT, false, false, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_OUT, true, false, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_RESID, false, false, DynGeom>(PlaneOutArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f64_simple)
}  // namespace fame
