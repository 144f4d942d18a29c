// Small-matrix stages of the ladder pass, all in the compound orbital basis [(o1,o2),(o4,o3)] where the
// upstream einsums are plain n^2 x n^2 matrix products:
//
//   * dga_chi0_prep_c128:    chi0^-1(q,w,nu) per core nu (four_point.py:601-613) and the nu sums
//                            chi0_full_sum, chi0_core_sum (nonlocal_sde.py:824-835);
//   * dga_chi_phys_c128:     chi_r(q,w) = [(sum_nu X/beta + chi0_full - chi0_core)^-1 + U_r + V_r^q]^-1
//                            (nonlocal_sde.py:167-182, 298) from the BSE output X;
//   * dga_lambda_c128:       FP64 Newton root-find of the lambda-correction and its application
//                            (lambda_correction.py:13-73);
//   * dga_kernel_assembly_c128: gamma_r = beta chi0^-1 X (nonlocal_sde.py:159-164) and
//                            K = -K_dc + K_dens + 3 K_magn with K_r = U_r (gamma - gamma U_r chi_r [- 2/3 1])
//                            (nonlocal_sde.py:201-215, 841-853);
//   * dga_dc_kernel_c128:    K_dc = ((U_adcb / beta^2) chi0) . F_dc cut to the core box (nonlocal_sde.py:185-198),
//                            a batched complex GEMM over w.
#include "dga_common.cuh"

namespace dga {

constexpr int MAX_N2 = 16;  // up to 4 orbitals

// In-place Gauss-Jordan inverse of an n x n matrix with partial (row) pivoting on |re|+|im|; element (r, c)
// at m[(r * n + c) * st].  Returns false on an exact zero pivot.
__device__ bool gj_inverse(double2* m, int n, int st) {
  int piv[MAX_N2];
  bool ok = true;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = cabs1(m[(k * n + k) * st]);
    for (int i = k + 1; i < n; ++i) {
      const double v = cabs1(m[(i * n + k) * st]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    piv[k] = p;
    if (p != k) {
      for (int j = 0; j < n; ++j) {
        double2 t = m[(k * n + j) * st];
        m[(k * n + j) * st] = m[(p * n + j) * st];
        m[(p * n + j) * st] = t;
      }
    }
    double2 d = m[(k * n + k) * st];
    if (d.x == 0.0 && d.y == 0.0) {
      ok = false;
      continue;
    }
    const double2 pinv = crecip(d);
    m[(k * n + k) * st] = make_double2(1.0, 0.0);
    for (int j = 0; j < n; ++j) m[(k * n + j) * st] = cmul(m[(k * n + j) * st], pinv);
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      const double2 f = m[(i * n + k) * st];
      m[(i * n + k) * st] = make_double2(0.0, 0.0);
      for (int j = 0; j < n; ++j) cfms(m[(i * n + j) * st], f, m[(k * n + j) * st]);
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k) {
      for (int i = 0; i < n; ++i) {
        double2 t = m[(i * n + k) * st];
        m[(i * n + k) * st] = m[(i * n + p) * st];
        m[(i * n + p) * st] = t;
      }
    }
  }
  return ok;
}

// c = a @ b for n x n matrices (row-major, contiguous)
__device__ __forceinline__ void matmul_n(const double2* a, const double2* b, double2* c, int n) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double2 acc = make_double2(0.0, 0.0);
      for (int k = 0; k < n; ++k) cfma(acc, a[i * n + k], b[k * n + j]);
      c[i * n + j] = acc;
    }
}

// ------------------------------------------------------------------------------------------------
// chi0 preparation: one thread per (q, w, nu_core); sums: one thread per (q, w)
//   chi0: [Q][W][nvf][n2][n2] (device layout written by the bubble), core nu window [shell, shell + nv)
// ------------------------------------------------------------------------------------------------
__global__ void chi0_inverse_kernel(const double2* __restrict__ chi0, int n2, int nvf, int nv, int shell,
                                    long long n_mats, double2* __restrict__ chi0_inv, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s = reinterpret_cast<double2*>(smem_raw);
  const int nn = n2 * n2;
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool active = m < n_mats;
  double2* mine = s + threadIdx.x;  // element e at mine[e * blockDim.x]
  if (active) {
    const long long qw = m / nv;
    const int v = (int)(m - qw * nv);
    const double2* src = chi0 + ((size_t)qw * nvf + shell + v) * nn;
    for (int e = 0; e < nn; ++e) mine[e * blockDim.x] = src[e];
    const bool ok = gj_inverse(mine, n2, blockDim.x);
    double2* dst = chi0_inv + (size_t)m * nn;
    for (int e = 0; e < nn; ++e) dst[e] = mine[e * blockDim.x];
    if (!ok && status) atomicOr(status, DGA_ITEM_SINGULAR);
  }
}

__global__ void chi0_sums_kernel(const double2* __restrict__ chi0, int n2, int nvf, int nv, int shell,
                                 long long n_qw, double inv_beta, double2* __restrict__ full_sum,
                                 double2* __restrict__ core_sum) {
  const int nn = n2 * n2;
  const long long total = n_qw * nn;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long qw = e / nn;
    const int el = (int)(e - qw * nn);
    const double2* base = chi0 + (size_t)qw * nvf * nn + el;
    double fr = 0.0, fi = 0.0, cr = 0.0, ci = 0.0;
    for (int v = 0; v < nvf; ++v) {
      const double2 x = base[(size_t)v * nn];
      fr += x.x;
      fi += x.y;
      if (v >= shell && v < shell + nv) {
        cr += x.x;
        ci += x.y;
      }
    }
    // 1/beta * (1/beta * sum)  (nonlocal_sde.py:824, 835 with local_four_point.py:146-162)
    full_sum[e] = make_double2(inv_beta * (inv_beta * fr), inv_beta * (inv_beta * fi));
    core_sum[e] = make_double2(inv_beta * (inv_beta * cr), inv_beta * (inv_beta * ci));
  }
}

// ------------------------------------------------------------------------------------------------
// physical susceptibility: one warp per (ch, q, w)
//   X: [n_ch][Q][W][N][n2] with row i = p * nv + nu;  uv: [n_ch][Q][n2][n2];  sums: [Q][W][n2][n2]
//   out: [n_ch][Q][W][n2][n2]
// The nu sum reads the item's X block coalesced: lane g * n2 + s (g < G = 32 / n2) sums column s over the rows
// nu = g, g + G, ..., and the G partial sums of a column are added by shuffles.  The two n2 x n2 inverses run on
// one lane from the warp's shared-memory copy.
// ------------------------------------------------------------------------------------------------
constexpr int CP_WARPS = 4;  // items per block
__global__ void __launch_bounds__(32 * CP_WARPS)
chi_phys_kernel(const double2* __restrict__ X, const double2* __restrict__ uv, const double2* __restrict__ full_sum,
                const double2* __restrict__ core_sum, int n2, int nv, int W, int Q, int n_ch, double inv_beta,
                double2* __restrict__ out, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nn = n2 * n2;
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2* mine = reinterpret_cast<double2*>(smem_raw) + (size_t)wib * nn;
  const long long t = blockIdx.x * (long long)CP_WARPS + wib;
  const long long total = (long long)n_ch * Q * W;
  if (t >= total) return;
  const int w = (int)(t % W);
  const int q = (int)((t / W) % Q);
  const int ch = (int)(t / ((long long)W * Q));
  const int N = n2 * nv;
  const double2* x = X + (size_t)t * N * n2;
  const size_t qw = (size_t)q * W + w;
  const int G = 32 / n2, g = lane / n2, sc = lane - g * n2;
  for (int p = 0; p < n2; ++p) {
    double sr = 0.0, si = 0.0;
    if (g < G)
      for (int v = g; v < nv; v += G) {
        const double2 y = x[(size_t)(p * nv + v) * n2 + sc];
        sr += y.x;
        si += y.y;
      }
    for (int h = 1; h < G; ++h) {  // lanes 0 .. n2 - 1 collect the partial sums of lanes sc + h n2
      const int src = min(lane + h * n2, 31);
      const double pr = __shfl_sync(0xffffffffu, sr, src), pi = __shfl_sync(0xffffffffu, si, src);
      if (g == 0) {
        sr += pr;
        si += pi;
      }
    }
    if (g == 0) {
      // (sum / beta + full) - core
      const double2 f = full_sum[qw * nn + p * n2 + sc];
      const double2 c = core_sum[qw * nn + p * n2 + sc];
      const double ar = inv_beta * sr + f.x, ai = inv_beta * si + f.y;
      mine[p * n2 + sc] = make_double2(ar - c.x, ai - c.y);
    }
  }
  __syncwarp();
  if (lane == 0) {
    bool ok = gj_inverse(mine, n2, 1);
    const double2* u = uv + ((size_t)ch * Q + q) * nn;
    for (int e = 0; e < nn; ++e) mine[e] = cadd(mine[e], u[e]);
    ok = gj_inverse(mine, n2, 1) && ok;
    if (!ok && status) atomicOr(status, DGA_ITEM_SINGULAR);
  }
  __syncwarp();
  double2* o = out + (size_t)t * nn;
  for (int e = lane; e < nn; e += 32) o[e] = mine[e];
}

// ------------------------------------------------------------------------------------------------
// lambda correction (single band): one CTA per channel
//   chi: [n_ch][Q][W] (n2 = 1), weights = irrk_count, target[ch] complex
// ------------------------------------------------------------------------------------------------
__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    v = lane < nw ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[0] = v;
  }
  __syncthreads();
  const double r = red[0];
  __syncthreads();
  return r;
}

__device__ double block_min(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    v = lane < nw ? red[lane] : INFINITY;
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
    if (lane == 0) red[0] = v;
  }
  __syncthreads();
  const double r = red[0];
  __syncthreads();
  return r;
}

__global__ void lambda_kernel(const double2* __restrict__ chi, int Q, int W, const long long* __restrict__ weights,
                              const double2* __restrict__ target, double beta, double nk_tot, double delta0,
                              double eps, int maxiter, double* __restrict__ lambda_out, int* __restrict__ iters_out,
                              int* __restrict__ status, double2* __restrict__ chi_out) {
  __shared__ double red[32];
  const int ch = blockIdx.x;
  const double2* c = chi + (size_t)ch * Q * W;
  const int niw = W - 1, nwf = 2 * niw + 1;
  const long long total = (long long)Q * nwf;
  // lambda_start = -min_q 1 / Re chi(q, w = 0)
  double mn = INFINITY;
  for (int q = threadIdx.x; q < Q; q += blockDim.x) mn = fmin(mn, 1.0 / c[(size_t)q * W].x);
  const double lam0 = -block_min(mn, red);
  const double factor = 1.0 / beta / nk_tot;
  const double2 tgt = target[ch];
  double delta = delta0;
  double lam = lam0 + delta;
  double result = lam;
  int it = 0, converged = 0;
  for (; it < maxiter; ++it) {
    double s1r = 0.0, s1i = 0.0, s2r = 0.0, s2i = 0.0;
    for (long long e = threadIdx.x; e < total; e += blockDim.x) {
      const int q = (int)(e / nwf);
      const int wf = (int)(e - (long long)q * nwf);
      const int w = wf - niw;
      double2 x = c[(size_t)q * W + (w < 0 ? -w : w)];
      if (w < 0) x.y = -x.y;
      // chi_lam = 1 / (1 / chi + lam)
      double2 inv = crecip(x);
      inv.x += lam;
      const double2 cl = crecip(inv);
      const double wq = (double)weights[q];
      s1r += wq * cl.x;
      s1i += wq * cl.y;
      const double2 cl2 = cmul(cl, cl);
      s2r += wq * cl2.x;
      s2i += wq * cl2.y;
    }
    s1r = block_sum(s1r, red);
    s1i = block_sum(s1i, red);
    s2r = block_sum(s2r, red);
    s2i = block_sum(s2i, red);
    const double2 f = make_double2(s1r * factor - tgt.x, s1i * factor - tgt.y);
    const double2 fp = make_double2(-s2r * factor, -s2i * factor);
    const double lam_new = lam - cdiv(f, fp).x;
    if (fabs(f.x) < eps) {
      result = lam_new;
      converged = 1;
      break;
    }
    // no root above lambda_start (e.g. a negative target): the Newton steps grow without bound; stop at the
    // last finite iterate and report non-convergence instead of propagating inf/nan
    if (!isfinite(lam_new)) break;
    if (lam_new < lam) {
      delta *= 0.5;
      lam = lam0 + delta;
    } else {
      lam = lam_new;
    }
    result = lam;
  }
  if (threadIdx.x == 0) {
    lambda_out[ch] = result;
    if (iters_out) iters_out[ch] = it;
    if (status && !converged) atomicOr(status, DGA_ITEM_NOCONVERGE);
  }
  // apply to the half range
  for (int e = threadIdx.x; e < Q * W; e += blockDim.x) {
    double2 inv = crecip(c[e]);
    inv.x += result;
    chi_out[(size_t)ch * Q * W + e] = crecip(inv);
  }
}

// ------------------------------------------------------------------------------------------------
// kernel assembly: one warp per (q, w, nu) matrix; lane l computes the elements l, l + 32, ... of every n2 x n2
// product, whose left operands sit in the warp's shared scratch (g3, t1, t2: 3 n2^2 complex)
//   chi0_inv: [Q][W][nv][n2][n2]; X: [2][Q][W][N][n2]; uv: [2][Q][n2][n2]; chi_phys: [2][Q][W][n2][n2]
//   k_dc: [Q][W][nv][n2][n2] or null;  out K: [Q][W][nv][n2][n2];  gamma_out (optional): [2][Q][W][nv][n2][n2]
// ------------------------------------------------------------------------------------------------
constexpr int KA_WARPS = 8;  // matrices per block
// One warp per matrix (q, w, nu); the n2 x n2 products run with the orbital-pair count NN2 fixed at compile time
// (elements per lane EPL), four blocks per SM (two for 4 orbitals, whose accumulators need the registers) to hide
// the latency of the dependent product chain.
template <int NN2>
__global__ void __launch_bounds__(32 * KA_WARPS, NN2 > 9 ? 2 : 4)
kernel_assembly_kernel(const double2* __restrict__ chi0_inv, const double2* __restrict__ X,
                                       const double2* __restrict__ uv, const double2* __restrict__ chi_phys,
                                       const double2* __restrict__ k_dc, int nv, int W, int Q, double beta,
                                       double2* __restrict__ K, double2* __restrict__ gamma_out) {
  constexpr int n2 = NN2, nn = NN2 * NN2, EPL = (nn + 31) / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double2* g3 = reinterpret_cast<double2*>(smem_raw) + (size_t)wib * 3 * nn;
  double2* t1 = g3 + nn;
  double2* t2 = t1 + nn;
  const long long t = blockIdx.x * (long long)KA_WARPS + wib;
  const long long total = (long long)Q * W * nv;
  if (t >= total) return;  // the whole warp; the block has no block-wide barrier
  const int v = (int)(t % nv);
  const long long qw = t / nv;
  const int q = (int)(qw / W);
  const int N = n2 * nv;
  const double2* c0i = chi0_inv + (size_t)t * nn;
  double2 acc[EPL];
#pragma unroll
  for (int j = 0; j < EPL; ++j) {
    const int e = lane + 32 * j;
    acc[j] = make_double2(0.0, 0.0);
    if (e < nn && k_dc) {
      const double2 z = k_dc[(size_t)t * nn + e];
      acc[j] = make_double2(-z.x, -z.y);
    }
  }
#pragma unroll 1
  for (int ch = 0; ch < 2; ++ch) {
    const double2* x = X + ((size_t)ch * Q * W + qw) * N * n2;
    const double2* u = uv + ((size_t)ch * Q + q) * nn;
    const double2* cp = chi_phys + ((size_t)ch * Q * W + qw) * nn;
    double2* go = gamma_out ? gamma_out + ((size_t)ch * Q * W * nv + t) * nn : nullptr;
    // gamma = beta * (chi0_inv @ X_nu)
#pragma unroll
    for (int j = 0; j < EPL; ++j) {
      const int e = lane + 32 * j;
      if (e < nn) {
        const int p = e / n2, sidx = e - p * n2;
        double2 a = make_double2(0.0, 0.0);
#pragma unroll 3
        for (int m = 0; m < n2; ++m) cfma(a, c0i[p * n2 + m], x[(size_t)(m * nv + v) * n2 + sidx]);
        const double2 g = make_double2(beta * a.x, beta * a.y);
        g3[e] = g;
        if (go) go[e] = g;
      }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < EPL; ++j) {  // t1 = gamma @ U_r
      const int e = lane + 32 * j;
      if (e < nn) {
        const int p = e / n2, sidx = e - p * n2;
        double2 a = make_double2(0.0, 0.0);
#pragma unroll 3
        for (int k = 0; k < n2; ++k) cfma(a, g3[p * n2 + k], u[k * n2 + sidx]);
        t1[e] = a;
      }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < EPL; ++j) {  // t2 = gamma - t1 @ chi_r  (- 2/3 on the diagonal in the magnetic channel)
      const int e = lane + 32 * j;
      if (e < nn) {
        const int p = e / n2, sidx = e - p * n2;
        double2 a = make_double2(0.0, 0.0);
#pragma unroll 3
        for (int k = 0; k < n2; ++k) cfma(a, t1[p * n2 + k], cp[k * n2 + sidx]);
        double2 r = csub(g3[e], a);
        if (ch == 1 && p == sidx) r.x += -(2.0 / 3.0);
        t2[e] = r;
      }
    }
    __syncwarp();
    const double f = ch == 0 ? 1.0 : 3.0;
#pragma unroll
    for (int j = 0; j < EPL; ++j) {  // K += f U_r @ t2
      const int e = lane + 32 * j;
      if (e < nn) {
        const int p = e / n2, sidx = e - p * n2;
        double2 a = make_double2(0.0, 0.0);
#pragma unroll 3
        for (int k = 0; k < n2; ++k) cfma(a, u[p * n2 + k], t2[k * n2 + sidx]);
        acc[j].x += f * a.x;
        acc[j].y += f * a.y;
      }
    }
    __syncwarp();  // g3, t1, t2 are rewritten by the next channel
  }
  double2* o = K + (size_t)t * nn;
#pragma unroll
  for (int j = 0; j < EPL; ++j) {
    const int e = lane + 32 * j;
    if (e < nn) o[e] = acc[j];
  }
}

// ------------------------------------------------------------------------------------------------
// K1 = (U_adcb / beta^2) @ chi0 for every (q, w, nu_full): one warp per matrix, written as the row-major GEMM
// operand K1[w][(q, p)][(m, nu)] (row (q, p), column (m, nu), Kd = n2 * nvf columns)
// ------------------------------------------------------------------------------------------------
__global__ void dc_left_kernel(const double2* __restrict__ chi0, const double2* __restrict__ u_perm, int n2, int Q,
                               int W, int nvf, double2* __restrict__ k1) {
  // one warp per matrix t = (q, w, nu), lane l computing the elements l, l + 32, ...
  const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= (long long)Q * W * nvf) return;
  const int nu = (int)(t % nvf), qw = (int)(t / nvf), w = qw % W, q = qw / W;
  const int nn = n2 * n2, Kd = n2 * nvf;
  const double2* c = chi0 + (size_t)t * nn;
  double2* o = k1 + ((size_t)w * Q + q) * n2 * Kd + nu;
  for (int e = lane; e < nn; e += 32) {
    const int i = e / n2, j = e - i * n2;
    double2 a = make_double2(0.0, 0.0);
    for (int k = 0; k < n2; ++k) cfma(a, u_perm[i * n2 + k], c[k * n2 + j]);
    o[(size_t)i * Kd + (size_t)j * nvf] = a;
  }
}

// Batched complex GEMM over w: C(r, c) = sum_k K1[w][r][k] F_dc[w][k][col(c)]
//   r = (q, p) (M = Q n2 rows), k = (m, nu) (Kd = n2 nvf), c = (s, nu') (Nc = n2 nv), col(c) = s nvf + shell + nu'
//   C(r, c) -> K_dc [Q][W][nv][n2][n2] at (q, w, nu', p, s)
// 64 x 64 complex outputs per 256-thread CTA, 4 x 4 per thread; K in steps of 16, the next step's operands loaded
// into registers while the current one multiplies.  A-tile rows are 16 consecutive k (256 contiguous bytes per row).
struct DcGemmArgs {
  const double2* k1;
  const double2* fdc;
  double2* out;
  int Q, W, n2, nvf, nv, shell;
};

constexpr int DG_TM = 64, DG_TN = 64, DG_TK = 16;

__global__ void __launch_bounds__(256, 2) dc_gemm_kernel(DcGemmArgs a) {
  __shared__ double2 As[DG_TK][DG_TM + 1];
  __shared__ double2 Bs[DG_TK][DG_TN];
  const int w = blockIdx.z;
  const int M = a.Q * a.n2, Kd = a.n2 * a.nvf, Nc = a.n2 * a.nv;
  const int r0 = blockIdx.y * DG_TM, c0 = blockIdx.x * DG_TN;
  const int tid = threadIdx.x, ty = tid & 15, tx = tid >> 4;
  const int Nf = a.n2 * a.nvf;
  const double2* A = a.k1 + (size_t)w * M * Kd;
  const double2* B = a.fdc + (size_t)w * Nf * Nf;
  // this thread's loads: A rows ra + 16 i (k = ka), B column cb (k rows kb + 4 i)
  const int ka = tid & 15, ra = tid >> 4;
  const int cb = tid & 63, kb = tid >> 6;
  int bcol = -1;
  if (c0 + cb < Nc) {
    const int col = c0 + cb, sidx = col / a.nv, nup = col - sidx * a.nv;
    bcol = sidx * a.nvf + a.shell + nup;
  }
  double2 ra_v[4], rb_v[4];
  auto load = [&](int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = r0 + ra + 16 * i, k = k0 + ka;
      ra_v[i] = (row < M && k < Kd) ? A[(size_t)row * Kd + k] : make_double2(0.0, 0.0);
      const int kr = k0 + kb + 4 * i;
      rb_v[i] = (bcol >= 0 && kr < Kd) ? B[(size_t)kr * Nf + bcol] : make_double2(0.0, 0.0);
    }
  };
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
  load(0);
  for (int k0 = 0; k0 < Kd; k0 += DG_TK) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      As[ka][ra + 16 * i] = ra_v[i];
      Bs[kb + 4 * i][cb] = rb_v[i];
    }
    __syncthreads();
    if (k0 + DG_TK < Kd) load(k0 + DG_TK);
#pragma unroll
    for (int kk = 0; kk < DG_TK; ++kk) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = r0 + ty + 16 * i;
    if (row >= M) continue;
    const int q = row / a.n2, p = row - q * a.n2;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = c0 + tx + 16 * j;
      if (col >= Nc) continue;
      const int sidx = col / a.nv, nup = col - sidx * a.nv;
      a.out[((((size_t)q * a.W + w) * a.nv + nup) * a.n2 + p) * a.n2 + sidx] = acc[i][j];
    }
  }
}

}  // namespace dga

using namespace dga;

static int vstatus(const char* who) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("%s: launch failed: %s", who, cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

static int small_threads(int n2) {
  // one thread per matrix with its n2 x n2 elements in shared memory (<= 96 KB per block)
  int t = 128;
  while (t > 32 && (size_t)t * n2 * n2 * sizeof(double2) > 96 * 1024) t >>= 1;
  return t;
}

extern "C" {

// chi0_inv: [Q][W][nv][n2][n2]; full_sum/core_sum: [Q][W][n2][n2]; chi0: [Q][W][nvf][n2][n2]
int dga_chi0_prep_c128(const void* chi0, int n_orb, int niv_core, int niv_shell, int niw_half, int n_q, double beta,
                       void* chi0_inv, void* full_sum, void* core_sum, int* status, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv_core, nvf = 2 * (niv_core + niv_shell);
  if (!chi0 || !chi0_inv || !full_sum || !core_sum || n2 > MAX_N2 || n_orb <= 0 || niv_core <= 0 || n_q <= 0 ||
      niw_half <= 0 || niv_shell < 0) {
    dga_set_error("dga_chi0_prep_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const long long n_mats = (long long)n_q * niw_half * nv;
  const int th = small_threads(n2);
  const size_t smem = (size_t)th * n2 * n2 * sizeof(double2);
  cudaFuncSetAttribute(chi0_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  chi0_inverse_kernel<<<(int)((n_mats + th - 1) / th), th, smem, stream>>>(
      (const double2*)chi0, n2, nvf, nv, niv_shell, n_mats, (double2*)chi0_inv, status);
  if (vstatus("dga_chi0_prep_c128")) return DGA_ERR_LAUNCH;
  const long long n_qw = (long long)n_q * niw_half;
  const long long work = n_qw * n2 * n2;
  int blocks = (int)((work + 255) / 256);
  if (blocks > 16 * device_sm_count()) blocks = 16 * device_sm_count();
  chi0_sums_kernel<<<blocks, 256, 0, stream>>>((const double2*)chi0, n2, nvf, nv, niv_shell, n_qw, 1.0 / beta,
                                               (double2*)full_sum, (double2*)core_sum);
  return vstatus("dga_chi0_prep_c128");
}

int dga_chi_phys_c128(const void* X, const void* uv, const void* full_sum, const void* core_sum, int n_orb,
                      int niv_core, int niw_half, int n_q, int n_ch, double beta, void* out, int* status,
                      cudaStream_t stream) {
  const int n2 = n_orb * n_orb;
  if (!X || !uv || !full_sum || !core_sum || !out || n2 > MAX_N2 || n_orb <= 0 || n_ch <= 0) {
    dga_set_error("dga_chi_phys_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const long long total = (long long)n_ch * n_q * niw_half;
  const size_t smem = (size_t)CP_WARPS * n2 * n2 * sizeof(double2);
  chi_phys_kernel<<<(int)((total + CP_WARPS - 1) / CP_WARPS), 32 * CP_WARPS, smem, stream>>>(
      (const double2*)X, (const double2*)uv, (const double2*)full_sum, (const double2*)core_sum, n2, 2 * niv_core,
      niw_half, n_q, n_ch, 1.0 / beta, (double2*)out, status);
  return vstatus("dga_chi_phys_c128");
}

// Single-band lambda correction of n_ch channels (lambda_correction.py:28-73).  chi: [n_ch][Q][W] complex;
// weights: [Q] int64 multiplicities; target: [n_ch] complex; lambda_out: [n_ch]; chi_out: [n_ch][Q][W].
int dga_lambda_c128(const void* chi, int n_q, int niw_half, int n_ch, const long long* weights, const void* target,
                    double beta, double nk_tot, double delta, double eps, int maxiter, double* lambda_out,
                    int* iters_out, int* status, void* chi_out, cudaStream_t stream) {
  if (!chi || !weights || !target || !lambda_out || !chi_out || n_q <= 0 || niw_half <= 0 || n_ch <= 0 ||
      maxiter <= 0) {
    dga_set_error("dga_lambda_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  lambda_kernel<<<n_ch, 1024, 0, stream>>>((const double2*)chi, n_q, niw_half, weights, (const double2*)target, beta,
                                           nk_tot, delta, eps, maxiter, lambda_out, iters_out, status,
                                           (double2*)chi_out);
  return vstatus("dga_lambda_c128");
}

int dga_kernel_assembly_c128(const void* chi0_inv, const void* X, const void* uv, const void* chi_phys,
                             const void* k_dc, int n_orb, int niv_core, int niw_half, int n_q, double beta, void* K,
                             void* gamma_out, cudaStream_t stream) {
  const int n2 = n_orb * n_orb;
  if (!chi0_inv || !X || !uv || !chi_phys || !K || n2 > MAX_N2 || n_orb <= 0) {
    dga_set_error("dga_kernel_assembly_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const long long total = (long long)n_q * niw_half * 2 * niv_core;
  const size_t smem = (size_t)KA_WARPS * 3 * n2 * n2 * sizeof(double2);
  const int blocks = (int)((total + KA_WARPS - 1) / KA_WARPS);
#define DGA_KA_CASE(NN)                                                                                        \
  case NN:                                                                                                     \
    cudaFuncSetAttribute(kernel_assembly_kernel<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    kernel_assembly_kernel<NN><<<blocks, 32 * KA_WARPS, smem, stream>>>(                                       \
        (const double2*)chi0_inv, (const double2*)X, (const double2*)uv, (const double2*)chi_phys,             \
        (const double2*)k_dc, 2 * niv_core, niw_half, n_q, beta, (double2*)K, (double2*)gamma_out);            \
    break;
  switch (n2) {
    DGA_KA_CASE(1)
    DGA_KA_CASE(4)
    DGA_KA_CASE(9)
    DGA_KA_CASE(16)
    default:
      dga_set_error("dga_kernel_assembly_c128: unsupported orbital count (n_orb = %d)", n_orb);
      return DGA_ERR_ARG;
  }
#undef DGA_KA_CASE
  return vstatus("dga_kernel_assembly_c128");
}

// Bytes of the K1 intermediate of dga_dc_kernel_c128.
size_t dga_dc_scratch_bytes(int n_orb, int niv_full, int niw_half, int n_q) {
  return (size_t)n_q * niw_half * 2 * niv_full * n_orb * n_orb * n_orb * n_orb * sizeof(double2);
}

// K_dc [Q][W][nv][n2][n2] from chi0 [Q][W][nvf][n2][n2], u_perm = compound matrix of U_adcb / beta^2
// [n2][n2] and F_dc [W][Nf][Nf] (compound row (d,c,nu), column (f,e,nu'), Nf = n2 * nvf).
int dga_dc_kernel_c128(const void* chi0, const void* u_perm, const void* fdc, int n_orb, int niv_core, int niv_shell,
                       int niw_half, int n_q, void* k_dc, void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv_core, nvf = 2 * (niv_core + niv_shell);
  if (!chi0 || !u_perm || !fdc || !k_dc || !scratch || n2 > MAX_N2 || n_orb <= 0) {
    dga_set_error("dga_dc_kernel_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  if (scratch_bytes < dga_dc_scratch_bytes(n_orb, niv_core + niv_shell, niw_half, n_q)) {
    dga_set_error("dga_dc_kernel_c128: scratch too small");
    return DGA_ERR_SCRATCH;
  }
  const long long n_mats = (long long)n_q * niw_half * nvf;
  dc_left_kernel<<<(int)((n_mats * 32 + 255) / 256), 256, 0, stream>>>((const double2*)chi0, (const double2*)u_perm, n2,
                                                                  n_q, niw_half, nvf, (double2*)scratch);
  if (vstatus("dga_dc_kernel_c128")) return DGA_ERR_LAUNCH;
  DcGemmArgs a;
  a.k1 = (const double2*)scratch;
  a.fdc = (const double2*)fdc;
  a.out = (double2*)k_dc;
  a.Q = n_q;
  a.W = niw_half;
  a.n2 = n2;
  a.nvf = nvf;
  a.nv = nv;
  a.shell = niv_shell;
  dim3 grid((n2 * nv + DG_TN - 1) / DG_TN, (n_q * n2 + DG_TM - 1) / DG_TM, niw_half);
  dc_gemm_kernel<<<grid, 256, 0, stream>>>(a);
  return vstatus("dga_dc_kernel_c128");
}

}  // extern "C"

// Hartree and Fock terms (nonlocal_sde.get_hartree_fock, dgamore/nonlocal_sde.py:31-69), one thread per (k, a, b):
//   fock[k][a][b] = -1/Nq sum_q sum_cd (U + V_q)[a][b][c][d] occ_k[k+q][d][c]  (k + q wrapped per axis)
//   hartree[a][b] = 2 sum_cd (U + V_(q=0))[a][b][c][d] occ[d][c]               (threads of k = 0)
//   u: [n^4]; v_q: [Nq][n^4] over the full grid in row-major (qx, qy, qz) order; occ: [n][n]; occ_k: [Nk][n][n]
//   sigma (optional): [Nk][n][n][nv2]; hartree + fock is added to every frequency (nonlocal_sde.py:884)
__global__ void hartree_fock_kernel(const double2* __restrict__ u, const double2* __restrict__ v_q,
                                    const double2* __restrict__ occ, const double2* __restrict__ occ_k, int n,
                                    int nx, int ny, int nz, double2* __restrict__ hartree,
                                    double2* __restrict__ fock, double2* __restrict__ sigma, int nv2) {
  const int n2 = n * n, nk = nx * ny * nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nk * n2) return;
  const int k = t / n2, ab = t - k * n2;
  const int kx = k / (ny * nz), ky = (k / nz) % ny, kz = k % nz;
  const double2* uab = u + (size_t)ab * n2;
  double2 acc = make_double2(0.0, 0.0);
  for (int qx = 0; qx < nx; ++qx) {
    const int sx = (kx + qx) % nx;
    for (int qy = 0; qy < ny; ++qy) {
      const int sy = (ky + qy) % ny;
      for (int qz = 0; qz < nz; ++qz) {
        const int sz = (kz + qz) % nz;
        const int q = (qx * ny + qy) * nz + qz, kq = (sx * ny + sy) * nz + sz;
        const double2* vab = v_q + ((size_t)q * n2 + ab) * n2;
        const double2* o = occ_k + (size_t)kq * n2;
        for (int c = 0; c < n; ++c)
          for (int d = 0; d < n; ++d) cfma(acc, cadd(uab[c * n + d], vab[c * n + d]), o[d * n + c]);
      }
    }
  }
  const double2 f = cscale(acc, -1.0 / nk);
  fock[(size_t)k * n2 + ab] = f;
  double2 h = make_double2(0.0, 0.0);
  const double2* v0 = v_q + (size_t)ab * n2;
  for (int c = 0; c < n; ++c)
    for (int d = 0; d < n; ++d) cfma(h, cadd(uab[c * n + d], v0[c * n + d]), occ[d * n + c]);
  h = cscale(h, 2.0);
  if (k == 0) hartree[ab] = h;
  if (sigma) {
    double2* sg = sigma + ((size_t)k * n2 + ab) * nv2;
    const double2 hf = cadd(h, f);
    for (int v = 0; v < nv2; ++v) sg[v] = cadd(sg[v], hf);
  }
}

extern "C" int dga_hartree_fock_c128(const void* u, const void* v_q, const void* occ, const void* occ_k, int n_orb,
                                     int nx, int ny, int nz, void* hartree, void* fock, void* sigma, int nv2,
                                     cudaStream_t stream) {
  if (!u || !v_q || !occ || !occ_k || !hartree || !fock || n_orb <= 0 || n_orb > 4 || nx <= 0 || ny <= 0 ||
      nz <= 0 || (long long)nx * ny * nz > (1LL << 24) || (sigma && nv2 <= 0)) {
    dga_set_error("dga_hartree_fock_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const int total = nx * ny * nz * n_orb * n_orb;
  hartree_fock_kernel<<<(total + 127) / 128, 128, 0, stream>>>((const double2*)u, (const double2*)v_q,
                                                                (const double2*)occ, (const double2*)occ_k, n_orb,
                                                                nx, ny, nz, (double2*)hartree, (double2*)fock,
                                                                (double2*)sigma, nv2);
  return vstatus("dga_hartree_fock_c128");
}

