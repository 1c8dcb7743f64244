// Declarations of the operator stage kernels; the definitions are in
// op_kernels.cuh and instantiated in ops_*.cu.
#pragma once
#include "geom_policy.cuh"

namespace fame {
// shared memory of a plane CTA: plane [Lm x S] | twf [Lf] | twm [Lm] | lx [Lf] | ly [Lm]
template <typename R>
__host__ __device__ inline size_t plane_smem_bytes(int Lf, int Lm, int S) {
  return sizeof(cplx<R>) * ((size_t)Lm * S + 2 * (size_t)Lf + 2 * (size_t)Lm);
}

// shared memory of a pencil CTA: tile [Ls x TW] | 1/eps tile [Ls x TW] | twiddles [Ls]
template <typename R>
__host__ __device__ inline size_t pencil_smem_bytes(int Ls) {
  return (sizeof(cplx<R>) + sizeof(R)) * (size_t)Ls * PencilTW<R>::v + sizeof(cplx<R>) * (size_t)Ls;
}

// shared memory of a pipelined pencil CTA: two (tile, 1/eps tile) buffers | twiddles [Ls]
template <typename R>
__host__ __device__ inline size_t pencil_pipe_smem_bytes(int Ls) {
  return 2 * (sizeof(cplx<R>) + sizeof(R)) * (size_t)Ls * PencilTW<R>::v + sizeof(cplx<R>) * (size_t)Ls;
}

template <typename R, bool GEN, int IN, bool PR, int RARE, class GP> __global__ void k_plane_inv(PlaneInArgs<R> a);
template <typename R> __global__ void k_pencil_pipe(PencilArgs<R> a);
template <typename R, bool GEN, int MODE, int RARE, class GP> __global__ void k_pencil(PencilArgs<R> a);
template <typename R, bool GEN, int EPI, bool PR, int RARE, class GP> __global__ void k_plane_fwd(PlaneOutArgs<R> a);

// combinations instantiated with a static geometry (the CG / refinement hot path
// and the operator benchmark)
template <typename R, int IN, bool PR>
constexpr bool kStatInv = !PR && (IN == IN_CG || IN == IN_VEC || (IN == IN_REFINE && sizeof(R) == 8));
template <typename R, int MODE> constexpr bool kStatPen = MODE == PEN_QBQ || (MODE == PEN_QBQ_CG && sizeof(R) == 4);
// combinations instantiated with static plane plans on runtime geometries
// (ops_plane_static.cu)
template <typename R, int IN, bool PR>
constexpr bool kPlanInv = (IN == IN_CG && !PR) || IN == IN_VEC || (IN == IN_REFINE && !PR && sizeof(R) == 8);
template <typename R, int EPI, bool PR>
constexpr bool kPlanFwd = EPI == EPI_OUT || (!PR && ((EPI == EPI_CGR && sizeof(R) == 4) ||
                                                      ((EPI == EPI_CG || EPI == EPI_RESID) && sizeof(R) == 8)));
template <typename R, int EPI, bool PR>
constexpr bool kStatFwd = !PR && ((EPI == EPI_CG && sizeof(R) == 8) || (EPI == EPI_CGR && sizeof(R) == 4) || EPI == EPI_OUT ||
                                  (EPI == EPI_RESID && sizeof(R) == 8));
}  // namespace fame
