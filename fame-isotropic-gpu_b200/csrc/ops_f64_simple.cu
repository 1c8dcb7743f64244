// Operator stage kernels, FP64, Simple lattices, radices 2, 3, 4, 5, 8.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, false, IN_CG, false, 0, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_VEC, false, 0, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_VEC, true, 0, DynGeom>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_REFINE, false, 0, DynGeom>(PlaneInArgs<double>);
template __global__ void k_pencil<double, false, PEN_QBQ, 0, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, false, PEN_QR_OUT, 0, DynGeom>(PencilArgs<double>);
template __global__ void k_pencil<double, false, PEN_QRS_IN, 0, DynGeom>(PencilArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_CG, false, 0, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_OUT, false, 0, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_OUT, true, 0, DynGeom>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_RESID, false, 0, DynGeom>(PlaneOutArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_f64_simple)
}  // namespace fame
