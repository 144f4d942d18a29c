// Shared device helpers for the ladder-DGA kernels: complex arithmetic on interleaved (re, im) pairs,
// error/status codes and launch geometry.
//
// Complex numbers are stored as double2 / float2 (re in .x, im in .y), the memory layout of numpy's
// complex128 / complex64, so host arrays and torch views cross the C ABI without repacking.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define DGA_OK 0
#define DGA_ERR_ARG 1        // invalid argument (null pointer, size out of range)
#define DGA_ERR_SCRATCH 2    // scratch buffer too small
#define DGA_ERR_LAUNCH 3     // CUDA launch error
#define DGA_ERR_CUDA 4       // other CUDA runtime error

// per-item status words written by the batched solvers
#define DGA_ITEM_OK 0
#define DGA_ITEM_SINGULAR 1    // exact zero pivot (numpy raises LinAlgError("Singular matrix"))
#define DGA_ITEM_NONFINITE 2   // NaN or Inf in the result
#define DGA_ITEM_NOCONVERGE 4  // iterative refinement did not reach its tolerance
#define DGA_ITEM_WAIT_TIMEOUT 8  // a bounded wait on an asynchronous copy or tensor-core tile ran out
// items a mixed-precision launch leaves for the FP64 re-solve
#define DGA_ITEM_REDO (DGA_ITEM_NOCONVERGE | DGA_ITEM_NONFINITE | DGA_ITEM_WAIT_TIMEOUT)

// largest matrix of the dense batched LU / solves (pivot and permutation arrays in shared memory)
#define DGA_DENSE_MAX_N 8192

// One problem (request) of a heterogeneous BSE batch; the layout is part of the C ABI (include/dga_b200.h).
typedef struct {
  const void* gamma_cm;  // [2][W][N][N] column-major compound Gamma_r
  const void* chi0_inv;  // [Q][W][nv][n2][n2]
  const void* uv;        // [2][Q][n2][n2]
  void* out;             // [2][Q][W][N][n2]
  int n_orb, niv, niw_half, n_q;
  double beta, inv_beta2;
} dga_bse_problem;

// Launch choices of the BSE solvers (the search space of the autotuner); layout is part of the C ABI.
typedef struct {
  int kernel;       // 0 = default, 1 = shared-memory-panel kernel (mixed form only), 2 = 128-thread kernel,
                    // 3 = shared-memory-panel kernel with tensor-core (tcgen05) trailing tiles (mixed form only)
  int ctas_per_sm;  // CTAs per SM of the 128-thread kernels (0 = as many as fit)
  long long wait_limit;  // polls of each bounded wait on a copy or tile inside an item (0 = the default limit)
} dga_bse_tuning;

namespace dga {

template <typename R>
struct cplx_t;
template <>
struct cplx_t<double> {
  using type = double2;
};
template <>
struct cplx_t<float> {
  using type = float2;
};

template <typename R>
using cplx = typename cplx_t<R>::type;

template <typename C>
__host__ __device__ __forceinline__ C cmake(decltype(C::x) re, decltype(C::x) im) {
  C z;
  z.x = re;
  z.y = im;
  return z;
}

template <typename C>
__host__ __device__ __forceinline__ C cadd(C a, C b) {
  return cmake<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
__host__ __device__ __forceinline__ C csub(C a, C b) {
  return cmake<C>(a.x - b.x, a.y - b.y);
}
template <typename C>
__host__ __device__ __forceinline__ C cmul(C a, C b) {
  return cmake<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__host__ __device__ __forceinline__ C cscale(C a, decltype(C::x) s) {
  return cmake<C>(a.x * s, a.y * s);
}
template <typename C>
__host__ __device__ __forceinline__ C cconj(C a) {
  return cmake<C>(a.x, -a.y);
}
// acc += a * b  (four real fused multiply-adds)
template <typename C>
__host__ __device__ __forceinline__ void cfma(C& acc, C a, C b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc -= a * b
template <typename C>
__host__ __device__ __forceinline__ void cfms(C& acc, C a, C b) {
  acc.x = fma(-a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
// |re| + |im|, the pivot measure of LAPACK's izamax / dcabs1
template <typename C>
__host__ __device__ __forceinline__ decltype(C::x) cabs1(C a) {
  return fabs(a.x) + fabs(a.y);
}
// 1 / z by Smith's algorithm (R. L. Smith, CACM 5(8):435, 1962): scales by the larger component so that
// neither |z|^2 nor the quotient overflows.
template <typename C>
__host__ __device__ __forceinline__ C crecip(C z) {
  using R = decltype(C::x);
  if (fabs(z.x) >= fabs(z.y)) {
    R r = z.y / z.x;
    R d = z.x + z.y * r;
    return cmake<C>(R(1) / d, -r / d);
  }
  R r = z.x / z.y;
  R d = z.y + z.x * r;
  return cmake<C>(r / d, R(-1) / d);
}
// a / b (Smith's algorithm)
template <typename C>
__host__ __device__ __forceinline__ C cdiv(C a, C b) {
  using R = decltype(C::x);
  if (fabs(b.x) >= fabs(b.y)) {
    R r = b.y / b.x;
    R d = b.x + b.y * r;
    return cmake<C>((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  R r = b.x / b.y;
  R d = b.y + b.x * r;
  return cmake<C>((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

template <typename C>
__device__ __forceinline__ bool cfinite(C a) {
  return isfinite(a.x) && isfinite(a.y);
}

// widen / narrow between precisions
__device__ __forceinline__ double2 to_c64(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_c64(double2 a) { return a; }
template <typename C>
__device__ __forceinline__ C from_c64(double2 a);
template <>
__device__ __forceinline__ double2 from_c64<double2>(double2 a) {
  return a;
}
template <>
__device__ __forceinline__ float2 from_c64<float2>(double2 a) {
  return make_float2((float)a.x, (float)a.y);
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// SMs of the current device (cached per device; 148 on B200).
int device_sm_count();

}  // namespace dga

// Records the last error message of the library (thread-local on the host side).
extern "C" const char* dga_last_error_string(void);
void dga_set_error(const char* fmt, ...);
