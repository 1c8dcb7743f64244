// Shared device/host definitions for the FAME B200 band-structure library.
//
// Complex values are stored interleaved (re, im) as float2 / double2, the same
// memory layout as cuDoubleComplex and the reference's `double _Complex` vectors,
// so host buffers from the reference (FAME_Main/FAME_Main_Code.cu:53-54) can be
// copied in and out unchanged.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fame {

template <typename R> struct C2;
template <> struct C2<float> { using T = float2; };
template <> struct C2<double> { using T = double2; };
template <typename R> using cplx = typename C2<R>::T;

template <typename R> __host__ __device__ __forceinline__ cplx<R> mk(R a, R b) {
  cplx<R> z;
  z.x = a;
  z.y = b;
  return z;
}
template <typename T> __host__ __device__ __forceinline__ T cadd(T a, T b) {
  T z;
  z.x = a.x + b.x;
  z.y = a.y + b.y;
  return z;
}
template <typename T> __host__ __device__ __forceinline__ T csub(T a, T b) {
  T z;
  z.x = a.x - b.x;
  z.y = a.y - b.y;
  return z;
}
template <typename T> __host__ __device__ __forceinline__ T cmul(T a, T b) {
  T z;
  z.x = a.x * b.x - a.y * b.y;
  z.y = a.x * b.y + a.y * b.x;
  return z;
}
// conj(a) * b
template <typename T> __host__ __device__ __forceinline__ T cmulc(T a, T b) {
  T z;
  z.x = a.x * b.x + a.y * b.y;
  z.y = a.x * b.y - a.y * b.x;
  return z;
}
template <typename T, typename S> __host__ __device__ __forceinline__ T cscale(T a, S s) {
  T z;
  z.x = a.x * s;
  z.y = a.y * s;
  return z;
}
template <typename T> __host__ __device__ __forceinline__ T cconj(T a) {
  T z;
  z.x = a.x;
  z.y = -a.y;
  return z;
}
template <typename T> __host__ __device__ __forceinline__ auto cabs2(T a) -> decltype(a.x) {
  return a.x * a.x + a.y * a.y;
}
__host__ __device__ __forceinline__ float2 to_f(double2 a) {
  return make_float2((float)a.x, (float)a.y);
}
__host__ __device__ __forceinline__ double2 to_d(float2 a) {
  return make_double2((double)a.x, (double)a.y);
}
template <typename R> __device__ __forceinline__ cplx<R> cvt(double2 a);
template <> __device__ __forceinline__ float2 cvt<float>(double2 a) { return to_f(a); }
template <> __device__ __forceinline__ double2 cvt<double>(double2 a) { return a; }

// e^{i*pi*x} evaluated with the CUDA math library's sincospi (argument in units of pi).
__device__ __forceinline__ double2 expipi(double x) {
  double s, c;
  sincospi(x, &s, &c);
  return make_double2(c, s);
}
__device__ __forceinline__ float2 expipi(float x) {
  float s, c;
  sincospif(x, &s, &c);
  return make_float2(c, s);
}

// Asynchronous global -> shared copies (cp.async, sm_80+): the data never passes
// through registers, so a thread keeps all its copies in flight at once.
// cp_async_wait_all waits for this thread's copies; a __syncthreads() after it
// publishes them to the CTA.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
// one element of 8 or 16 bytes
template <typename T> __device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  static_assert(sizeof(T) == 8 || sizeof(T) == 16, "8- or 16-byte elements");
  if constexpr (sizeof(T) == 16)
    cp_async16(smem, gmem);
  else
    cp_async8(smem, gmem);
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
// close this thread's current group of copies (possibly empty)
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's most recent groups are still in flight
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Bulk prefetch into L2 (cp.async.bulk.prefetch.L2, sm_90+) of the 16-byte-aligned
// part of [p, p + bytes): the start is rounded up and the end down to 16 bytes, so
// nothing outside the range is touched.  A hint only: no data reaches the thread.
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes) {
  const uintptr_t a = ((uintptr_t)p + 15) & ~(uintptr_t)15;
  const uintptr_t e = ((uintptr_t)p + bytes) & ~(uintptr_t)15;
  if (e <= a) return;
  const unsigned n = (unsigned)(e - a);
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a), "r"(n) : "memory");
}

// Shared-memory exchange between the CTAs of a cluster with an mbarrier (sm_90+).
// A CTA initialises its barrier, announces the bytes it expects, and waits for them;
// the other CTAs write into its shared memory with st.async, whose completion is
// counted on that barrier.  Unlike a cluster barrier with release semantics, nothing
// waits for the writers' outstanding global stores.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
// the address of this CTA's shared-memory location `local` in the CTA of cluster rank `rank`
__device__ __forceinline__ unsigned mapa_u32(unsigned local, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
// makes an initialised barrier visible to the cluster's other CTAs (before a cluster barrier)
__device__ __forceinline__ void mbar_init_fence_cluster() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(bar),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of the barrier for at most `max_cycles` SM clock cycles;
// false if it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, long long max_cycles) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > max_cycles) return false;
  return true;
}
// one complex value into cluster shared memory, counted on the destination's barrier
__device__ __forceinline__ void st_async(unsigned addr, float2 v, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];\n" ::"r"(addr),
               "f"(v.x), "f"(v.y), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void st_async(unsigned addr, double2 v, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];\n" ::"r"(addr),
               "d"(v.x), "d"(v.y), "r"(bar)
               : "memory");
}

// Kernels launched on the device, counted by each kernel's first thread.  Every
// translation unit has its own counter; FAME_DEFINE_LAUNCH_GETTER exposes it.
static __device__ unsigned long long g_launches;
#define FAME_DEFINE_LAUNCH_GETTER(fn)                                              \
  unsigned long long fn() {                                                        \
    unsigned long long v = 0;                                                      \
    if (cudaMemcpyFromSymbol(&v, ::fame::g_launches, sizeof(v)) != cudaSuccess) v = 0; \
    return v;                                                                      \
  }
#define FAME_COUNT_LAUNCH()                                                              \
  do {                                                                                   \
    if ((threadIdx.x | threadIdx.y | blockIdx.x | blockIdx.y | blockIdx.z) == 0) atomicAdd(&::fame::g_launches, 1ull); \
  } while (0)

// Status codes returned through the C ABI (include/fame_b200.h).
enum Status : int {
  kOk = 0,
  kBadInput = 1,
  kNoConvergence = 2,
  kWatchdog = 3,
  kCudaError = 4,
  kNoDevice = 5,
  kUnsupported = 6,
};

}  // namespace fame
