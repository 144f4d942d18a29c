// Self-consistency glue on the device: the lattice Green's function and the frequency sums behind the filling,
// the occupations and the chemical-potential search (dgamore/greens_function.py:20-142, 212-292), and the
// k-average of the self-energy's tail for its moment fit (dgamore/self_energy.py:51-75).
//
//   G(k, nu) = [i nu + mu - e_k - Sigma(k, nu)]^-1            n x n per (k, nu), n <= 4
//   S(k)     = sum_nu Re G(k, nu),   T(k) = sum_nu Re G_model(k, nu),   G_model(k, nu) = [i nu + mu - e_k - s0]^-1
//
// The filling and the occupations follow from S, T and the n x n density matrices on the host
// (dgamore_b200/selfconsistency.py), as the upstream's get_total_fill and get_fill_nonlocal combine them.
// Layouts: Sigma [Nk][n][n][2 niv] (compressed k, nu = (2m + 1) pi / beta for m = -niv .. niv - 1), e_k [Nk][n][n],
// s0 [n][n] (real), all complex128 except s0, S and T (float64).
#include "dga_common.cuh"

namespace dga {

// Inverse of an n x n complex matrix by Gauss-Jordan elimination with partial pivoting (largest |re| + |im|, first
// index on ties, the pivot order of LAPACK's getrf that numpy.linalg.inv uses); a singular matrix gives NaN.
template <int NB>
__device__ __forceinline__ void inv_small(double2 (&a)[NB][NB], double2 (&x)[NB][NB]) {
#pragma unroll
  for (int i = 0; i < NB; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) x[i][j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    int p = c;
    double best = fabs(a[c][c].x) + fabs(a[c][c].y);
#pragma unroll
    for (int r = c + 1; r < NB; ++r) {
      const double v = fabs(a[r][c].x) + fabs(a[r][c].y);
      if (v > best) {
        best = v;
        p = r;
      }
    }
#pragma unroll
    for (int r = 0; r < NB; ++r)
      if (r == p && p != c) {
#pragma unroll
        for (int j = 0; j < NB; ++j) {
          const double2 t = a[c][j];
          a[c][j] = a[r][j];
          a[r][j] = t;
          const double2 u = x[c][j];
          x[c][j] = x[r][j];
          x[r][j] = u;
        }
      }
    const double2 piv = crecip(a[c][c]);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      a[c][j] = cmul(a[c][j], piv);
      x[c][j] = cmul(x[c][j], piv);
    }
#pragma unroll
    for (int r = 0; r < NB; ++r) {
      if (r == c) continue;
      const double2 f = a[r][c];
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        a[r][j] = csub(a[r][j], cmul(f, a[c][j]));
        x[r][j] = csub(x[r][j], cmul(f, x[c][j]));
      }
    }
  }
}

__device__ __forceinline__ double matsubara_nu(int m, double beta) { return (2.0 * m + 1.0) * M_PI / beta; }

// [i nu + mu - e_k - D] for an n x n D (complex), into a.
template <int NB>
__device__ __forceinline__ void g_matrix(double2 (&a)[NB][NB], const double2* __restrict__ ek, double nu, double mu,
                                         const double2* __restrict__ d, long long d_stride) {
#pragma unroll
  for (int i = 0; i < NB; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const double2 e = ek[i * NB + j], s = d[(i * NB + j) * d_stride];
      a[i][j] = make_double2((i == j ? mu : 0.0) - e.x - s.x, (i == j ? nu : 0.0) - e.y - s.y);
    }
}

template <int NB>
__global__ void g_full_kernel(const double2* __restrict__ sigma, const double2* __restrict__ ek, int nk, int nv,
                              double mu, double beta, double2* __restrict__ g) {
  const long long n = (long long)nk * nv;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / nv), v = (int)(e - (long long)k * nv);
    const double nu = matsubara_nu(v - nv / 2, beta);
    double2 a[NB][NB], x[NB][NB];
    g_matrix<NB>(a, ek + (size_t)k * NB * NB, nu, mu, sigma + (size_t)k * NB * NB * nv + v, nv);
    inv_small<NB>(a, x);
    double2* o = g + (size_t)k * NB * NB * nv + v;
#pragma unroll
    for (int i = 0; i < NB; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) o[(size_t)(i * NB + j) * nv] = x[i][j];
  }
}

// One block per k: S(k) and T(k), the frequency sums of Re G and Re G_model (threads over nu, then a block sum).
template <int NB>
__global__ void fill_sums_kernel(const double2* __restrict__ sigma, const double2* __restrict__ ek,
                                 const double* __restrict__ s0, int nk, int nv, double mu, double beta,
                                 double* __restrict__ s_out, double* __restrict__ t_out) {
  __shared__ double red[2 * NB * NB][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double2 s0c[NB * NB];
#pragma unroll
  for (int e = 0; e < NB * NB; ++e) s0c[e] = make_double2(s0[e], 0.0);
  for (int k = blockIdx.x; k < nk; k += gridDim.x) {
    double accs[NB * NB], acct[NB * NB];
#pragma unroll
    for (int e = 0; e < NB * NB; ++e) accs[e] = acct[e] = 0.0;
    const double2* ekk = ek + (size_t)k * NB * NB;
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
      const double nu = matsubara_nu(v - nv / 2, beta);
      double2 a[NB][NB], x[NB][NB];
      g_matrix<NB>(a, ekk, nu, mu, sigma + (size_t)k * NB * NB * nv + v, nv);
      inv_small<NB>(a, x);
#pragma unroll
      for (int i = 0; i < NB; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) accs[i * NB + j] += x[i][j].x;
      g_matrix<NB>(a, ekk, nu, mu, s0c, 1);
      inv_small<NB>(a, x);
#pragma unroll
      for (int i = 0; i < NB; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) acct[i * NB + j] += x[i][j].x;
    }
#pragma unroll
    for (int e = 0; e < NB * NB; ++e) {
      double s = accs[e], t = acct[e];
      for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        t += __shfl_down_sync(0xffffffffu, t, off);
      }
      if (lane == 0) {
        red[e][warp] = s;
        red[NB * NB + e][warp] = t;
      }
    }
    __syncthreads();
    if (threadIdx.x < 2 * NB * NB) {
      double sum = 0.0;
      for (int w = 0; w < nw; ++w) sum += red[threadIdx.x][w];
      if (threadIdx.x < NB * NB) s_out[(size_t)k * NB * NB + threadIdx.x] = sum;
      else t_out[(size_t)k * NB * NB + threadIdx.x - NB * NB] = sum;
    }
    __syncthreads();
  }
}

// out[e][v'] = mean_k Sigma[k][e][v0 + v'] for the n^2 orbital pairs e and nvs frequencies (one thread each,
// summing k in order).
__global__ void sigma_kmean_kernel(const double2* __restrict__ sigma, int nk, int n2, int nv, int v0, int nvs,
                                   double2* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n2 * nvs) return;
  const int e = t / nvs, v = t - e * nvs;
  double2 acc = make_double2(0.0, 0.0);
  for (int k = 0; k < nk; ++k) acc = cadd(acc, sigma[((size_t)k * n2 + e) * nv + v0 + v]);
  out[t] = make_double2(acc.x / nk, acc.y / nk);
}

}  // namespace dga

using namespace dga;

static int glue_status(const char* who) {
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("%s: launch failed: %s", who, cudaGetErrorString(err));
    return 1;
  }
  return 0;
}

extern "C" {

int dga_g_full_c128(const void* sigma, const void* ek, int n_orb, int nk, int niv, double mu, double beta, void* g,
                    cudaStream_t stream) {
  if (!sigma || !ek || !g || n_orb < 1 || n_orb > 4 || nk <= 0 || niv <= 0 || !(beta > 0.0)) {
    dga_set_error("dga_g_full_c128: invalid arguments (n_orb in 1..4)");
    return DGA_ERR_ARG;
  }
  const int nv = 2 * niv;
  const long long n = (long long)nk * nv;
  const int blocks = (int)((n + 255) / 256 < 65535 ? (n + 255) / 256 : 65535);
  const double2* s = (const double2*)sigma;
  const double2* e = (const double2*)ek;
  double2* o = (double2*)g;
  switch (n_orb) {
    case 1: g_full_kernel<1><<<blocks, 256, 0, stream>>>(s, e, nk, nv, mu, beta, o); break;
    case 2: g_full_kernel<2><<<blocks, 256, 0, stream>>>(s, e, nk, nv, mu, beta, o); break;
    case 3: g_full_kernel<3><<<blocks, 256, 0, stream>>>(s, e, nk, nv, mu, beta, o); break;
    default: g_full_kernel<4><<<blocks, 256, 0, stream>>>(s, e, nk, nv, mu, beta, o); break;
  }
  return glue_status("dga_g_full_c128") ? DGA_ERR_LAUNCH : DGA_OK;
}

int dga_fill_sums_c128(const void* sigma, const void* ek, const double* s0, int n_orb, int nk, int niv, double mu,
                       double beta, double* s_out, double* t_out, cudaStream_t stream) {
  if (!sigma || !ek || !s0 || !s_out || !t_out || n_orb < 1 || n_orb > 4 || nk <= 0 || niv <= 0 || !(beta > 0.0)) {
    dga_set_error("dga_fill_sums_c128: invalid arguments (n_orb in 1..4)");
    return DGA_ERR_ARG;
  }
  const int nv = 2 * niv;
  const int blocks = nk < 4 * device_sm_count() ? nk : 4 * device_sm_count();
  const double2* s = (const double2*)sigma;
  const double2* e = (const double2*)ek;
  switch (n_orb) {
    case 1: fill_sums_kernel<1><<<blocks, 128, 0, stream>>>(s, e, s0, nk, nv, mu, beta, s_out, t_out); break;
    case 2: fill_sums_kernel<2><<<blocks, 128, 0, stream>>>(s, e, s0, nk, nv, mu, beta, s_out, t_out); break;
    case 3: fill_sums_kernel<3><<<blocks, 128, 0, stream>>>(s, e, s0, nk, nv, mu, beta, s_out, t_out); break;
    default: fill_sums_kernel<4><<<blocks, 128, 0, stream>>>(s, e, s0, nk, nv, mu, beta, s_out, t_out); break;
  }
  return glue_status("dga_fill_sums_c128") ? DGA_ERR_LAUNCH : DGA_OK;
}

int dga_sigma_kmean_c128(const void* sigma, int n_orb, int nk, int nv, int v0, int nvs, void* out,
                         cudaStream_t stream) {
  if (!sigma || !out || n_orb < 1 || nk <= 0 || nv <= 0 || v0 < 0 || nvs <= 0 || v0 + nvs > nv) {
    dga_set_error("dga_sigma_kmean_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const int n2 = n_orb * n_orb, n = n2 * nvs;
  sigma_kmean_kernel<<<(n + 127) / 128, 128, 0, stream>>>((const double2*)sigma, nk, n2, nv, v0, nvs, (double2*)out);
  return glue_status("dga_sigma_kmean_c128") ? DGA_ERR_LAUNCH : DGA_OK;
}

}  // extern "C"
