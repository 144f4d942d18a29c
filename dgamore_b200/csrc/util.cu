// Library-wide utilities: the last-error string and a generic strided complex copy (layout conversions
// between the upstream array layouts and the device layouts of this library).
#include "dga_common.cuh"

#include <stdarg.h>
#include <stdio.h>
#include <string.h>

static thread_local char g_last_error[512] = "";

void dga_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

extern "C" const char* dga_last_error_string(void) { return g_last_error; }

namespace dga {

// Streaming multiprocessors of the current device, read once per device (grid sizes of the streaming kernels
// are multiples of it).
int device_sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
  if (dev < 64 && cache[dev] > 0) return cache[dev];
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  if (dev < 64) cache[dev] = sms;
  return sms;
}

}  // namespace dga

extern "C" int dga_device_sm_count(void) { return dga::device_sm_count(); }

namespace dga {

constexpr int PERM_MAX_DIMS = 8;

struct PermDesc {
  int ndim;
  long long shape[PERM_MAX_DIMS];
  long long src_stride[PERM_MAX_DIMS];
  long long dst_stride[PERM_MAX_DIMS];
};

template <typename C>
__global__ void strided_copy_kernel(const C* __restrict__ src, C* __restrict__ dst, PermDesc d, long long total,
                                    double scale) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long rem = e, so = 0, doff = 0;
    for (int k = d.ndim - 1; k >= 0; --k) {
      const long long idx = rem % d.shape[k];
      rem /= d.shape[k];
      so += idx * d.src_stride[k];
      doff += idx * d.dst_stride[k];
    }
    C v = src[so];
    if (scale != 1.0) {
      v.x *= scale;
      v.y *= scale;
    }
    dst[doff] = v;
  }
}

}  // namespace dga

using namespace dga;

extern "C" {

// dst[sum_k idx_k * dst_stride_k] = scale * src[sum_k idx_k * src_stride_k] over the index box `shape`
// (strides in complex elements).  Used to move arrays between the upstream layouts (e.g. FourPoint
// [q,a,b,c,d,w,nu]) and the device layouts (e.g. the column-major compound matrices of the BSE).
int dga_strided_copy_c128(const void* src, void* dst, int ndim, const long long* shape, const long long* src_stride,
                          const long long* dst_stride, double scale, cudaStream_t stream) {
  if (!src || !dst || ndim <= 0 || ndim > PERM_MAX_DIMS || !shape || !src_stride || !dst_stride) {
    dga_set_error("dga_strided_copy_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  PermDesc d;
  d.ndim = ndim;
  long long total = 1;
  for (int k = 0; k < ndim; ++k) {
    if (shape[k] <= 0) return DGA_OK;
    d.shape[k] = shape[k];
    d.src_stride[k] = src_stride[k];
    d.dst_stride[k] = dst_stride[k];
    total *= shape[k];
  }
  const int threads = 256;
  long long blocks = (total + threads - 1) / threads;
  const long long cap = 32LL * device_sm_count();
  if (blocks > cap) blocks = cap;
  strided_copy_kernel<double2><<<(int)blocks, threads, 0, stream>>>((const double2*)src, (double2*)dst, d, total,
                                                                    scale);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_strided_copy_c128: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

// Library version: major * 10000 + minor * 100 + patch.
int dga_version(void) { return 100; }

}  // extern "C"
