// Operator stage kernels with the compile-time 96 x 96 x 96 geometry (cubic Simple
// lattice at Nx = 96), FP64: the CG and refinement hot path and the operator benchmark.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<double, false, IN_CG, false, 0, Stat96>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_VEC, false, 0, Stat96>(PlaneInArgs<double>);
template __global__ void k_plane_inv<double, false, IN_REFINE, false, 0, Stat96>(PlaneInArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_CG, false, 0, Stat96>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_OUT, false, 0, Stat96>(PlaneOutArgs<double>);
template __global__ void k_plane_fwd<double, false, EPI_RESID, false, 0, Stat96>(PlaneOutArgs<double>);
template __global__ void k_pencil_pipe<double>(PencilArgs<double>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_stat96_f64)
}  // namespace fame
