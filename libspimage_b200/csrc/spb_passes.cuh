// Helpers shared by the register-resident pass kernels (spb_fast.cu: 16
// points per thread; spb_split.cu: 8 points per thread): asynchronous copies,
// programmatic dependent launch, stage twiddles in shared memory, the
// Fourier projection with its operands at hand, the layout of the
// line-major projection operands in shared memory, and the launch helpers.
#pragma once
#include <math.h>

#include "spb_internal.h"
#include "spb_pointwise.cuh"

namespace spb {

// ------------------------------------------------------ async copy helpers
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Programmatic dependent launch.  What a pass kernel does before this point
// reads only data written two or more kernels earlier in the stream (twiddles,
// the previous iterate, flags, line-major operands) and writes only shared
// memory; the predecessor's output is read after the wait.  The successor may
// start its own prologue once this kernel's predecessor has completed, which
// keeps that two-kernel distance for every prologue; the release comes just
// before the final stores, so that the successor's blocks do not take SM
// residency from this kernel's.  Without the launch attribute both
// instructions return at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
// called before the final stores: the successor launches during this kernel's tail
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

template <typename K, typename... Args>
inline cudaError_t launch_maybe_pdl(K k, dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                                    Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

// stage-twiddle table of an N-point line into shared memory (N-1 entries)
template <int N>
__device__ __forceinline__ void stage_twiddles(float2 *tw_s, const float2 *__restrict__ stw) {
  for (int i = threadIdx.x; i < N - 1; i += blockDim.x) cp_async8(tw_s + i, stw + i);
}

// Fourier projection with the amplitude and measured bit already at hand
__device__ __forceinline__ float2 project_with(float2 G, float amp, bool measured, long long idx, const PassArgs &a,
                                               bool fourier_constraints) {
  if (fourier_constraints && (a.constraints & C_CENTROSYM)) G.y = 0.0f;
  if (!measured) return G;
  if (a.objective != 0) return a.phased_amp[idx % a.n_start];
  float m = 1.0f;
  if (!(a.constraints & C_MARGIN)) {
    m = __fdiv_rn(amp, cabs_ref(G));
  } else {
    const float av = cabs_ref(G);
    const float lo = a.amp_min[idx % a.n_start], hi = a.amp_max[idx % a.n_start];
    if (av < lo) m = __fdiv_rn(lo, av);
    else if (av > hi) m = __fdiv_rn(hi, av);
  }
  if (isfinite(m)) return make_float2(fmul(G.x, m), fmul(G.y, m));
  return make_float2(amp, 0.0f);
}

// words per line of the measured-bit bitmap (a multiple of 4 words)
__host__ __device__ constexpr int proj_words(int n) { return ((n + 127) / 128) * 4; }
template <int N, int C>
__host__ __device__ constexpr int amp_stride() {
  return N + (C == 1 ? 0 : (C <= 8 ? 32 / C : 4));
}
template <int N, int C>
__host__ __device__ constexpr int bits_stride() {
  return C == 1 ? proj_words(N) : proj_words(N) + ((((C <= 8 ? 32 / C : 4) - proj_words(N) % 32) + 32) % 32);
}

// dynamic shared memory limit of kernel K raised to at least smem (once per size)
template <auto K>
static cudaError_t ensure_smem(size_t smem) {
  static size_t have = 0;
  if (smem <= have) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) have = smem;
  return e;
}

}  // namespace spb
