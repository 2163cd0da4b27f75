/*
 * peak.cu - the integer-ALU roof the stage report divides by.
 *
 * Every stage of the path is integer arithmetic (butterflies and filters with
 * rounding between steps), so beside its bytes against the HBM copy
 * bandwidth each stage reports its operations against what the SMs can issue.
 * That peak is measured, not assumed: a kernel of independent 32-bit adds
 * (kind 0) or multiply-adds (kind 1) in eight-register rings, enough warps on
 * every SM to hide the pipeline latency, timed with CUDA events.
 *
 * Each ring step is one source operation (a + b, or a * b + c, which the
 * hardware issues as one instruction); the result counts steps per second.
 *
 * The dependency-scheduled phase is bound by neither: each step of its
 * critical path is a block published on one SM and seen by a waiter on
 * another. Its floor is measured too: the one-way time of a flag handed
 * between warps on two SMs with the phase's own release store and acquire
 * polls, nothing else in the step.
 */
#include <cuda_runtime.h>

#include "../../include/av1b.h"

namespace av1b {
namespace {

template <int KIND>
__global__ void __launch_bounds__(256) k_int_peak(int* out, int iters, int seed) {
  int a0 = threadIdx.x ^ seed, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 5, a5 = a0 + 7,
      a6 = a0 + 11, a7 = a0 + 13;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (KIND == 0) {
        a0 += a1; a1 += a2; a2 += a3; a3 += a4; a4 += a5; a5 += a6; a6 += a7; a7 += a0;
      } else {
        a0 = a0 * a1 + a2; a1 = a1 * a2 + a3; a2 = a2 * a3 + a4; a3 = a3 * a4 + a5;
        a4 = a4 * a5 + a6; a5 = a5 * a6 + a7; a6 = a6 * a7 + a0; a7 = a7 * a0 + a1;
      }
    }
  }
  const int r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
  if (r == 0x7fffffff) out[0] = r;  /* keeps the work live; practically never stores */
}

__device__ __forceinline__ unsigned handoff_ld(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void handoff_st(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long handoff_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* CTA 0 hands a flag back and forth with CTA j = 1 .. partners in turn,
 * `rounds` round trips each, with the flags at each of `places` places in
 * memory (`place_stride` words apart: the L2 slice that holds a flag, against
 * where the two SMs sit, changes the time); ns[place * (partners + 1) + j] =
 * the round trips' total time. The ping and reply of partner j sit 128 bytes
 * apart at place + 64 j and place + 64 j + 32. Every wait gives up after
 * `limit` polls and sets *err; the launch is cooperative, so the partners are
 * resident while CTA 0 waits for them. */
__global__ void k_handoff(unsigned* flags, unsigned long long* ns, int partners, int rounds,
                          int places, int place_stride, unsigned limit, int* err) {
  if (threadIdx.x != 0) return;
  const int me = blockIdx.x;
  for (int pl = 0; pl < places; ++pl)
    for (int j = 1; j <= partners; ++j) {
      unsigned* ping = flags + static_cast<size_t>(pl) * place_stride + 64 * j;
      unsigned* reply = ping + 32;
      if (me == 0) {
        const unsigned long long t0 = handoff_ns();
        for (int k = 0; k < rounds; ++k) {
          handoff_st(ping, 2u * k + 1u);
          unsigned it = 0;
          while (handoff_ld(reply) != 2u * k + 2u)
            if (++it > limit) {
              atomicExch(err, 1);
              return;
            }
        }
        ns[pl * (partners + 1) + j] = handoff_ns() - t0;
      } else if (me == j) {
        for (int k = 0; k < rounds; ++k) {
          unsigned it = 0;
          while (handoff_ld(ping) != 2u * k + 1u)
            if (++it > limit) {
              atomicExch(err, 1);
              return;
            }
          handoff_st(reply, 2u * k + 2u);
        }
      }
      if (*reinterpret_cast<volatile int*>(err)) return;
    }
}

}  // namespace
}  // namespace av1b

/* The median one-way time, in ns, of a flag handed between warps on two SMs
 * with release stores and acquire polls: CTA 0 against up to 16 partners,
 * the flags at 8 places in memory, 32 round trips each. */
extern "C" AV1B_API int av1b_handoff_peak(int device, double* one_way_ns) {
  if (!one_way_ns) return AV1B_ERR_ARG;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return AV1B_ERR_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return AV1B_ERR_NO_DEVICE;
  int n_sm = 0, coop = 0;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  int rc = AV1B_ERR_CUDA;
  constexpr int kPlaces = 8;
  const int partners = n_sm - 1 < 16 ? n_sm - 1 : 16, rounds = 32;
  /* places 16 KB + 384 bytes apart (different address bits each), each
   * holding 64 words a partner */
  const int place_stride = 4096 + 96;
  const size_t words = static_cast<size_t>(kPlaces) * place_stride;
  const size_t n_ns = static_cast<size_t>(kPlaces) * (partners + 1);
  unsigned* flags = nullptr;
  unsigned long long* ns = nullptr;
  int* err = nullptr;
  if (coop && partners >= 1 && 64 * (partners + 1) <= place_stride &&
      cudaMalloc(&flags, words * sizeof(unsigned)) == cudaSuccess &&
      cudaMalloc(&ns, n_ns * sizeof(unsigned long long)) == cudaSuccess &&
      cudaMalloc(&err, sizeof(int)) == cudaSuccess &&
      cudaMemset(flags, 0, words * sizeof(unsigned)) == cudaSuccess &&
      cudaMemset(ns, 0, n_ns * sizeof(unsigned long long)) == cudaSuccess &&
      cudaMemset(err, 0, sizeof(int)) == cudaSuccess) {
    int np = partners, nr = rounds, npl = kPlaces, ps = place_stride;
    unsigned limit = 1u << 22;
    void* args[] = {&flags, &ns, &np, &nr, &npl, &ps, &limit, &err};
    /* one CTA of one warp on each SM */
    if (cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(av1b::k_handoff), dim3(n_sm), dim3(32),
                                    args, 0, nullptr) == cudaSuccess &&
        cudaDeviceSynchronize() == cudaSuccess) {
      unsigned long long h[kPlaces * 17] = {0};
      int herr = 0;
      if (cudaMemcpy(h, ns, n_ns * sizeof(unsigned long long), cudaMemcpyDeviceToHost) == cudaSuccess &&
          cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && !herr) {
        /* the median over every place and partner (slot 0 of each place is
         * CTA 0's own, unused) */
        unsigned long long v[kPlaces * 16];
        int m = 0;
        for (int pl = 0; pl < kPlaces; ++pl)
          for (int j = 1; j <= partners; ++j) v[m++] = h[pl * (partners + 1) + j];
        for (int a = 0; a < m; ++a)
          for (int b = a + 1; b < m; ++b)
            if (v[b] < v[a]) {
              const unsigned long long t = v[a];
              v[a] = v[b];
              v[b] = t;
            }
        *one_way_ns = static_cast<double>(v[(m - 1) / 2]) / (2.0 * rounds);
        rc = AV1B_OK;
      } else if (herr) {
        rc = AV1B_ERR_TIMEOUT;
      }
    }
  }
  if (flags) cudaFree(flags);
  if (ns) cudaFree(ns);
  if (err) cudaFree(err);
  cudaSetDevice(prev);
  return rc;
}

/* Ring steps per second of `kind` (0: add, 1: multiply-add) on `device`. */
extern "C" AV1B_API int av1b_int_peak(int device, int kind, double* ops_per_s) {
  if (!ops_per_s || kind < 0 || kind > 1) return AV1B_ERR_ARG;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return AV1B_ERR_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return AV1B_ERR_NO_DEVICE;
  int n_sm = 0;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
  int* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = AV1B_ERR_CUDA;
  if (cudaMalloc(&out, sizeof(int)) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
      cudaEventCreate(&e1) == cudaSuccess) {
    const int blocks = n_sm * 8, threads = 256, iters = 1 << 14;
    auto launch = [&]() {
      if (kind == 0) av1b::k_int_peak<0><<<blocks, threads>>>(out, iters, 1);
      else av1b::k_int_peak<1><<<blocks, threads>>>(out, iters, 1);
    };
    launch();  /* warm-up (module load, clocks) */
    float best = 0.f;
    for (int rep = 0; rep < 3 && cudaGetLastError() == cudaSuccess; ++rep) {
      cudaEventRecord(e0);
      launch();
      cudaEventRecord(e1);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        break;
      if (best == 0.f || ms < best) best = ms;
    }
    if (best > 0.f && cudaGetLastError() == cudaSuccess) {
      const double steps = static_cast<double>(blocks) * threads * iters * 4.0 * 8.0;
      *ops_per_s = steps / (best * 1e-3);
      rc = AV1B_OK;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (out) cudaFree(out);
  cudaSetDevice(prev);
  return rc;
}
