// The persistent team kernel, one instantiation per grid size (N, M).
// A launch runs every active instance of a plan: CTA -> instance via cta_inst,
// rank within the team = blockIdx.x - team_first. Instances whose size is not
// the kernel's raise kDevBadSize and stop.
#pragma once
#include "bgp_programs.cuh"

BGP_NS_BEGIN

template <int N, int M>
__device__ void run_prog(Ctx& C, Ctl& S) {
#if defined(BGP_ONLY_API)
  prog_api<N, M>(C, S);
#elif defined(BGP_ONLY_SOLVE)
  prog_solve<N, M>(C, S);
#else
  if (C.I.prog == kProgSolve) prog_solve<N, M>(C, S);
  else prog_api<N, M>(C, S);
#endif
}

// Kernel body shared by the single-size and two-size kernels.
#define BGP_KERNEL_PROLOGUE                                                    \
  extern __shared__ double2 dyn_sm[];                                          \
  __shared__ Inst sI;                                                          \
  __shared__ Ctl S;                                                            \
  __shared__ double sred[kSredDoubles];                                        \
  __shared__ double tot[kNRec];                                                \
  __shared__ PassArgs Qs;                                                      \
  const int inst_ = L.cta_inst[blockIdx.x];                                    \
  if (threadIdx.x == 0) sI = L.insts[inst_];                                   \
  __syncthreads();                                                             \
  Team T{(int)blockIdx.x - sI.team_first, sI.team_size, sI.bar, L.abort_flag}; \
  Ctx C{sI, T, dyn_sm, sred, tot, Qs, 0, 0ull};                                \
  BGP_PROF_START(C)

#if defined(BGP_PROF)
#define BGP_PROF_START(C) (C).t_last = gtimer_ns();
#else
#define BGP_PROF_START(C)
#endif

// 16 warps per SM (128 registers a thread) while the longest line fits without
// spilling, else 8
template <int N, int M>
constexpr int min_blocks() { return (((N > M ? N : M) <= 512) ? 16 : 8) / kWarps; }

template <int N, int M>
__global__ void __launch_bounds__(kThreads, min_blocks<N, M>()) bgp_kernel_t(Launch L) {
  BGP_KERNEL_PROLOGUE
  if (sI.N == N && sI.M == M) { run_prog<N, M>(C, S); return; }
  if (threadIdx.x == 0) atomicCAS(L.abort_flag, 0, (int)kDevBadSize);
}

template <int N1, int M1, int N2, int M2>
__global__ void __launch_bounds__(kThreads, (min_blocks<N1, M1>() < min_blocks<N2, M2>() ? min_blocks<N1, M1>()
                                                                                         : min_blocks<N2, M2>()))
    bgp_kernel_t2(Launch L) {
  BGP_KERNEL_PROLOGUE
  if (sI.N == N1 && sI.M == M1) { run_prog<N1, M1>(C, S); return; }
  if (sI.N == N2 && sI.M == M2) { run_prog<N2, M2>(C, S); return; }
  if (threadIdx.x == 0) atomicCAS(L.abort_flag, 0, (int)kDevBadSize);
}

BGP_NS_END  // namespace bgp
