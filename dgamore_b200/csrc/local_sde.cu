// Local Schwinger-Dyson equation on the device (dgamore/local_sde.py:17-217): the local ladder of one atom, the
// producer of the local irreducible vertex Gamma_r, the full vertex F_r, the three-leg vertex and the local
// susceptibility that the nonlocal pass consumes.  Per channel r and w >= 0 (W = niw_core + 1 frequencies), with
// compound index (p = (a,b), nu) x (s = (d,c), nu') (local_four_point.py:206-229) and N = n^2 * 2 niv_core:
//
//   chi_r       = beta G2_r - 2 beta G_ab(nu) G_cd(nu') delta_{w0} [dens]                 (local_sde.py:17-29)
//   Gamma_r     = beta^2 (chi_r^-1 - chi~_core^-1) + U_r                                  (local_sde.py:40-51)
//   F_r         = Gamma_u [1 + chi0 Gamma_u / beta^2]^-1 over the full box (Gamma_u: U_r outside the core) (:75-82)
//   X_r         = sum_nu' [chi0^-1 + (Gamma_r - U_r)/beta^2]^-1 / beta: the ladder BSE at q = 0 (:54-59, 93-99)
//
// chi~ = (chi0^-1 + U_r/beta^2)^-1 over the full box is dense in nu (U_r fills every (nu, nu') entry, as the
// upstream adds it to the block-diagonal chi0^-1), but its core block's inverse has the closed form
//
//   chi~_core^-1 = chi0_core^-1 + 1 1^T (x) U_eff / beta^2,  U_eff = U_r [1 + (S_full - S_core) U_r]^-1,
//
// (the Schur complement of the shell block, with S the (1/beta^2) sum_nu chi0 over the full and core boxes), so
// Gamma_r(i, j) = beta^2 chi_r^-1(i, j) - delta_{nu nu'} beta^2 chi0^-1(nu)[p][s] + (U_r - U_eff)[p][s] needs no
// inversion of a full-box matrix.  The dense inverses chi_r^-1 and the solve for F run in the batched LU of
// bse.cu; X, the three-leg vertex and the shell-corrected susceptibility reuse the nonlocal pass's entries at
// q = 0 with V = 0.
#include "dga_common.cuh"

namespace dga {

constexpr int LOC_MAX_N2 = 16;

// chi0[w][nu][p = (a,b)][s = (d,c)] = -beta G_ad(nu) G_cb(nu - w) for w in [0, W), nu in the box of nvb
// frequencies (bubble_gen.py:20-30); entries whose real and imaginary parts are both below 1e-12 are zeroed as
// filter_small_values (n_point_base.py:205-211) does.
__global__ void local_bubble_kernel(const double2* __restrict__ g, int n, int niv_g, int W, int nvb, double beta,
                                    double2* __restrict__ chi0) {
  const int n2 = n * n;
  const long long total = (long long)W * nvb * n2 * n2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e % n2), p = (int)((e / n2) % n2);
    const int v = (int)((e / ((long long)n2 * n2)) % nvb), w = (int)(e / ((long long)n2 * n2 * nvb));
    const int a = p / n, b = p - a * n, d = s / n, c = s - d * n;
    const int m = v - nvb / 2;
    const double2 gl = g[(size_t)(a * n + d) * 2 * niv_g + niv_g + m];
    const double2 gr = g[(size_t)(c * n + b) * 2 * niv_g + niv_g + m - w];
    double2 x = cmul(gl, gr);
    x.x *= -beta;
    x.y *= -beta;
    if (fabs(x.x) < 1e-12 && fabs(x.y) < 1e-12) x = make_double2(0.0, 0.0);
    chi0[e] = x;
  }
}

// chi[w] (column-major compound, element (i, j) at j N + i) from G2 [a][b][c][d][n_wg][nv][nv] at w0 + w, through
// a 32 x 32 shared-memory tile (G2 is read along nu', chi written along nu).  Grid: (nu' tiles, nu tiles,
// W * n^4).
__global__ void local_chi_kernel(const double2* __restrict__ g2, int n, int nv, int w0, int n_wg,
                                 const double2* __restrict__ g, int niv_g, double beta, int dens,
                                 double2* __restrict__ chi) {
  __shared__ double2 tile[32][33];
  const int n2 = n * n, n4 = n2 * n2, N = n2 * nv;
  const int w = blockIdx.z / n4, o = blockIdx.z - w * n4;
  const int a = o / (n * n2), b = (o / n2) % n, c = (o / n) % n, d = o % n;
  const int v0 = blockIdx.y * 32, vp0 = blockIdx.x * 32;
  const double2* src = g2 + ((size_t)o * n_wg + (w0 + w)) * nv * nv;
  const int gshift = niv_g - nv / 2;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int v = v0 + r, vp = vp0 + threadIdx.x;
    if (v < nv && vp < nv) {
      double2 x = src[(size_t)v * nv + vp];
      x.x *= beta;
      x.y *= beta;
      if (dens && w == 0) {
        const double2 gg = cmul(g[(size_t)(a * n + b) * 2 * niv_g + gshift + v],
                                g[(size_t)(c * n + d) * 2 * niv_g + gshift + vp]);
        x.x -= 2.0 * beta * gg.x;
        x.y -= 2.0 * beta * gg.y;
      }
      tile[r][threadIdx.x] = x;
    }
  }
  __syncthreads();
  const int p = a * n + b, s = d * n + c;
  double2* dst = chi + (size_t)w * N * N;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int vp = vp0 + r, v = v0 + threadIdx.x;
    if (v < nv && vp < nv) dst[(size_t)(s * nv + vp) * N + p * nv + v] = tile[threadIdx.x][r];
  }
}

// ucorr[ch][w] = U_r - U_r [1 + (full - core) U_r]^-1 per (ch, w): one CTA each, the n2 x n2 algebra in shared
// memory (Gauss-Jordan with partial pivoting by one thread; n2 <= 16).  A singular 1 + D U_r sets
// DGA_ITEM_SINGULAR in status[ch * W + w].
__global__ void local_ucorr_kernel(const double2* __restrict__ uv, const double2* __restrict__ full_sum,
                                   const double2* __restrict__ core_sum, int n2, int W, double2* __restrict__ ucorr,
                                   int* __restrict__ status) {
  __shared__ double2 M[LOC_MAX_N2][LOC_MAX_N2], X[LOC_MAX_N2][LOC_MAX_N2], U[LOC_MAX_N2][LOC_MAX_N2];
  const int ch = blockIdx.x / W, w = blockIdx.x - ch * W, tid = threadIdx.x;
  const double2* u = uv + (size_t)ch * n2 * n2;
  const double2* fs = full_sum + (size_t)w * n2 * n2;
  const double2* cs = core_sum + (size_t)w * n2 * n2;
  for (int e = tid; e < n2 * n2; e += blockDim.x) U[e / n2][e % n2] = u[e];
  __syncthreads();
  for (int e = tid; e < n2 * n2; e += blockDim.x) {
    const int i = e / n2, j = e % n2;
    double2 acc = make_double2(i == j ? 1.0 : 0.0, 0.0);
    for (int k = 0; k < n2; ++k) cfma(acc, csub(fs[i * n2 + k], cs[i * n2 + k]), U[k][j]);
    M[i][j] = acc;
    X[i][j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  if (tid == 0) {
    int singular = 0;
    for (int c = 0; c < n2; ++c) {
      int piv = c;
      double best = fabs(M[c][c].x) + fabs(M[c][c].y);
      for (int r = c + 1; r < n2; ++r) {
        const double v = fabs(M[r][c].x) + fabs(M[r][c].y);
        if (v > best) {
          best = v;
          piv = r;
        }
      }
      if (best == 0.0) {
        singular = 1;
        break;
      }
      if (piv != c)
        for (int j = 0; j < n2; ++j) {
          const double2 t = M[c][j];
          M[c][j] = M[piv][j];
          M[piv][j] = t;
          const double2 t2 = X[c][j];
          X[c][j] = X[piv][j];
          X[piv][j] = t2;
        }
      const double2 r = crecip(M[c][c]);
      for (int j = 0; j < n2; ++j) {
        M[c][j] = cmul(M[c][j], r);
        X[c][j] = cmul(X[c][j], r);
      }
      for (int i = 0; i < n2; ++i) {
        if (i == c) continue;
        const double2 f = M[i][c];
        for (int j = 0; j < n2; ++j) {
          cfms(M[i][j], f, M[c][j]);
          cfms(X[i][j], f, X[c][j]);
        }
      }
    }
    status[blockIdx.x] = singular ? DGA_ITEM_SINGULAR : DGA_ITEM_OK;
  }
  __syncthreads();
  double2* out = ucorr + (size_t)blockIdx.x * n2 * n2;
  for (int e = tid; e < n2 * n2; e += blockDim.x) {
    const int i = e / n2, j = e % n2;
    double2 acc = U[i][j];
    for (int k = 0; k < n2; ++k) cfms(acc, U[i][k], X[k][j]);
    out[e] = acc;
  }
}

// gamma[m][(j, i)] = beta^2 chi_inv[m](i, j) - delta_{nu nu'} beta^2 chi0_inv[w][nu][p][s] + ucorr[m][p][s] for
// the 2W matrices m = ch W + w; chi_inv column-major at m * inv_stride.  Grid: (column blocks, 2W).
__global__ void local_gamma_kernel(const double2* __restrict__ chi_inv, long long inv_stride,
                                   const double2* __restrict__ chi0_inv, const double2* __restrict__ ucorr, int n2,
                                   int nv, int W, double beta, double2* __restrict__ gamma) {
  const int m = blockIdx.y, w = m % W, N = n2 * nv;
  const double beta2 = beta * beta;
  const double2* src = chi_inv + (size_t)m * inv_stride;
  const double2* uc = ucorr + (size_t)m * n2 * n2;
  double2* dst = gamma + (size_t)m * N * N;
  for (int j = blockIdx.x; j < N; j += gridDim.x) {
    const int s = j / nv, vp = j - s * nv;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const int p = i / nv, v = i - p * nv;
      const double2 x = src[(size_t)j * N + i];
      double2 y = uc[p * n2 + s];
      y.x += beta2 * x.x;
      y.y += beta2 * x.y;
      if (v == vp) {
        const double2 c = chi0_inv[(((size_t)w * nv + v) * n2 + p) * n2 + s];
        y.x -= beta2 * c.x;
        y.y -= beta2 * c.y;
      }
      dst[(size_t)j * N + i] = y;
    }
  }
}

// Full-box operands of F = Gamma_u [1 + chi0 Gamma_u / beta^2]^-1 for the 2W matrices m = ch W + w:
//   gamma_u[m](i, j) = Gamma_r core element if nu, nu' are both in the core box, else U_r[p][s];
//   mt[m](r, c) = delta_rc + (1/beta^2) sum_t chi0[w][nu_c][p_c][t] gamma_u((t, nu_c), r), i.e. M^T,
// both column-major Nf x Nf.  One 32 x 32 tile of M^T per CTA (threads along c read gamma_u along its rows, the
// tile is transposed in shared memory so the columns of M^T are written contiguously); the CTAs with
// blockIdx.y == 0 also write their column strip of gamma_u.  Grid: (Nf / 32 tiles of c, Nf / 32 tiles of r, 2W).
__global__ void local_fvertex_operands_kernel(const double2* __restrict__ gamma, const double2* __restrict__ uv,
                                              const double2* __restrict__ chi0, int n2, int nvc, int nvf, int W,
                                              double beta, double2* __restrict__ mt, double2* __restrict__ gamma_u) {
  __shared__ double2 tile[32][33];
  const int m = blockIdx.z, ch = m / W, w = m - ch * W;
  const int Nc = n2 * nvc, Nf = n2 * nvf, sh = (nvf - nvc) / 2;
  const double inv_beta2 = 1.0 / (beta * beta);
  const double2* gm = gamma + (size_t)m * Nc * Nc;
  const double2* u = uv + (size_t)ch * n2 * n2;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  auto gu = [&](int i, int j) -> double2 {
    const int p = i / nvf, v = i - p * nvf - sh, s = j / nvf, vp = j - s * nvf - sh;
    if (v >= 0 && v < nvc && vp >= 0 && vp < nvc) return gm[(size_t)(s * nvc + vp) * Nc + p * nvc + v];
    return u[p * n2 + s];
  };
  const int c = c0 + threadIdx.x;
  if (c < Nf) {
    const int pc = c / nvf, vc = c - pc * nvf;
    const double2* c0row = chi0 + (((size_t)w * nvf + vc) * n2 + pc) * n2;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
      const int r = r0 + rr;
      if (r >= Nf) break;
      double2 acc = make_double2(0.0, 0.0);
      for (int t = 0; t < n2; ++t) cfma(acc, c0row[t], gu(t * nvf + vc, r));
      acc.x *= inv_beta2;
      acc.y *= inv_beta2;
      if (r == c) acc.x += 1.0;
      tile[rr][threadIdx.x] = acc;
    }
  }
  __syncthreads();
  double2* dst = mt + (size_t)m * Nf * Nf;
  for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
    const int cw = c0 + cc, r = r0 + threadIdx.x;
    if (cw < Nf && r < Nf) dst[(size_t)cw * Nf + r] = tile[threadIdx.x][cc];
  }
  if (blockIdx.y == 0) {
    double2* gdst = gamma_u + (size_t)m * Nf * Nf;
    for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
      const int j = c0 + cc;
      if (j >= Nf) break;
      for (int i = threadIdx.x; i < Nf; i += blockDim.x) gdst[(size_t)j * Nf + i] = gu(i, j);
    }
  }
}

// inner[w][nu][p][s] = [(V_d - V_d U_d X_d) - (V_m - V_m U_m X_m)] / 2 for w >= 0 (local_sde.py:167-169), with V
// the three-leg vertices [ch][W][nv][n2][n2], X the susceptibilities [ch][W][n2][n2] and U_r the channel
// interactions [ch][n2][n2], all compound orbital matrices.  One CTA per (w, nu).
__global__ void local_inner_kernel(const double2* __restrict__ vrg, const double2* __restrict__ chi,
                                   const double2* __restrict__ uv, int n2, int nv, int W,
                                   double2* __restrict__ inner) {
  __shared__ double2 VU[2][LOC_MAX_N2][LOC_MAX_N2];
  const int w = blockIdx.x / nv, v = blockIdx.x - w * nv;
  const size_t blk = (size_t)n2 * n2;
  for (int e = threadIdx.x; e < 2 * n2 * n2; e += blockDim.x) {
    const int ch = e / (n2 * n2), ps = e - ch * n2 * n2, p = ps / n2, s = ps - p * n2;
    const double2* V = vrg + (((size_t)ch * W + w) * nv + v) * blk;
    const double2* U = uv + (size_t)ch * blk;
    double2 acc = make_double2(0.0, 0.0);
    for (int t = 0; t < n2; ++t) cfma(acc, V[p * n2 + t], U[t * n2 + s]);
    VU[ch][p][s] = acc;
  }
  __syncthreads();
  for (int ps = threadIdx.x; ps < n2 * n2; ps += blockDim.x) {
    const int p = ps / n2, s = ps - p * n2;
    double2 r[2];
    for (int ch = 0; ch < 2; ++ch) {
      const double2* V = vrg + (((size_t)ch * W + w) * nv + v) * blk;
      const double2* X = chi + ((size_t)ch * W + w) * blk;
      double2 acc = V[ps];
      for (int t = 0; t < n2; ++t) cfms(acc, VU[ch][p][t], X[t * n2 + s]);
      r[ch] = acc;
    }
    inner[((size_t)w * nv + v) * blk + ps] = make_double2(0.5 * (r[0].x - r[1].x), 0.5 * (r[0].y - r[1].y));
  }
}

// sigma[i][j][nu] = -1/beta sum_{w = -(W-1)}^{W-1} sum_{k,l,o,p} U_kjop inner_ilpo(w, nu) G_lk(nu - w)
//                   + sum_{c,d} U_dens[i][j][c][d] occ[d][c]                          (local_sde.py:165-172)
// with inner(-w, nu) = conj inner(w, -nu - 1) (local_n_point.py:191-225); u plain [n][n][n][n]; one thread per
// (i, j, nu).
__global__ void local_sigma_kernel(const double2* __restrict__ inner, const double2* __restrict__ u,
                                   const double2* __restrict__ g, const double2* __restrict__ occ, int n, int nv,
                                   int W, int niv_g, double beta, double2* __restrict__ sigma) {
  const int n2 = n * n, e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n2 * nv) return;
  const int v = e % nv, ij = e / nv, i = ij / n, j = ij - i * n;
  const int gshift = niv_g - nv / 2;
  double2 acc = make_double2(0.0, 0.0);
  for (int wf = -(W - 1); wf <= W - 1; ++wf) {
    const int wa = wf < 0 ? -wf : wf, va = wf < 0 ? nv - 1 - v : v;
    const double2* in = inner + ((size_t)wa * nv + va) * n2 * n2;
    for (int l = 0; l < n; ++l) {
      for (int k = 0; k < n; ++k) {
        const double2 glk = g[(size_t)(l * n + k) * 2 * niv_g + gshift + v - wf];
        double2 t = make_double2(0.0, 0.0);
        for (int o = 0; o < n; ++o)
          for (int p = 0; p < n; ++p) {
            double2 x = in[(i * n + l) * n2 + o * n + p];
            if (wf < 0) x.y = -x.y;
            cfma(t, u[((k * n + j) * n + o) * n + p], x);
          }
        cfma(acc, t, glk);
      }
    }
  }
  double2 hf = make_double2(0.0, 0.0);
  for (int c = 0; c < n; ++c)
    for (int d = 0; d < n; ++d) {
      // U_dens[i][j][c][d] = 2 U_ijcd - U_idcj (interaction.py:43-65)
      const double2 uijcd = u[((i * n + j) * n + c) * n + d], uidcj = u[((i * n + d) * n + c) * n + j];
      cfma(hf, make_double2(2.0 * uijcd.x - uidcj.x, 2.0 * uijcd.y - uidcj.y), occ[d * n + c]);
    }
  sigma[e] = make_double2(hf.x - acc.x / beta, hf.y - acc.y / beta);
}

}  // namespace dga

using namespace dga;

static int launch_check(const char* name) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("%s: launch failed: %s", name, cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

static int flat_grid(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  return (int)(g < 4096 ? (g > 0 ? g : 1) : 4096);
}

extern "C" {

int dga_local_bubble_c128(const void* g, int n_orb, int niv_g, int niw_half, int niv_box, double beta, void* chi0,
                          cudaStream_t stream) {
  if (!g || !chi0 || n_orb <= 0 || n_orb * n_orb > LOC_MAX_N2 || niw_half <= 0 || niv_box <= 0 ||
      niv_g < niv_box + niw_half) {
    dga_set_error("dga_local_bubble_c128: invalid arguments (n_orb=%d niv_g=%d niw_half=%d niv=%d)", n_orb, niv_g,
                  niw_half, niv_box);
    return DGA_ERR_ARG;
  }
  const int n2 = n_orb * n_orb;
  const long long total = (long long)niw_half * 2 * niv_box * n2 * n2;
  local_bubble_kernel<<<flat_grid(total, 256), 256, 0, stream>>>((const double2*)g, n_orb, niv_g, niw_half,
                                                                  2 * niv_box, beta, (double2*)chi0);
  return launch_check("dga_local_bubble_c128");
}

int dga_local_chi_c128(const void* g2, int n_orb, int niv, int niw_half, int w0, int n_wg, const void* g, int niv_g,
                       double beta, int dens, void* chi_cm, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, n4 = n2 * n2;
  if (!g2 || !g || !chi_cm || n_orb <= 0 || n2 > LOC_MAX_N2 || niv <= 0 || niw_half <= 0 || w0 < 0 ||
      w0 + niw_half > n_wg || niv_g < niv || (long long)niw_half * n4 > 65535) {
    dga_set_error("dga_local_chi_c128: invalid arguments (n_orb=%d niv=%d niw_half=%d w0=%d n_wg=%d)", n_orb, niv,
                  niw_half, w0, n_wg);
    return DGA_ERR_ARG;
  }
  const int nv = 2 * niv, tiles = (nv + 31) / 32;
  local_chi_kernel<<<dim3(tiles, tiles, niw_half * n4), dim3(32, 8), 0, stream>>>(
      (const double2*)g2, n_orb, nv, w0, n_wg, (const double2*)g, niv_g, beta, dens, (double2*)chi_cm);
  return launch_check("dga_local_chi_c128");
}

int dga_local_ucorr_c128(const void* uv, const void* full_sum, const void* core_sum, int n_orb, int niw_half,
                         void* ucorr, int* status, cudaStream_t stream) {
  const int n2 = n_orb * n_orb;
  if (!uv || !full_sum || !core_sum || !ucorr || !status || n_orb <= 0 || n2 > LOC_MAX_N2 || niw_half <= 0) {
    dga_set_error("dga_local_ucorr_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  local_ucorr_kernel<<<2 * niw_half, 64, 0, stream>>>((const double2*)uv, (const double2*)full_sum,
                                                      (const double2*)core_sum, n2, niw_half, (double2*)ucorr,
                                                      status);
  return launch_check("dga_local_ucorr_c128");
}

int dga_local_gamma_c128(const void* chi_inv, long long inv_stride, const void* chi0_inv, const void* ucorr,
                         int n_orb, int niv, int niw_half, double beta, void* gamma_cm, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, N = n2 * 2 * niv;
  if (!chi_inv || !chi0_inv || !ucorr || !gamma_cm || n_orb <= 0 || n2 > LOC_MAX_N2 || niv <= 0 || niw_half <= 0 ||
      inv_stride < (long long)N * N || 2 * niw_half > 65535) {
    dga_set_error("dga_local_gamma_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const int cols = N < 512 ? N : 512;
  local_gamma_kernel<<<dim3(cols, 2 * niw_half), 256, 0, stream>>>(
      (const double2*)chi_inv, inv_stride, (const double2*)chi0_inv, (const double2*)ucorr, n2, 2 * niv, niw_half,
      beta, (double2*)gamma_cm);
  return launch_check("dga_local_gamma_c128");
}

int dga_local_fvertex_operands_c128(const void* gamma_cm, const void* uv, const void* chi0, int n_orb, int niv_core,
                                    int niv_shell, int niw_half, double beta, void* mt, void* gamma_u,
                                    cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nvf = 2 * (niv_core + niv_shell), Nf = n2 * nvf;
  if (!gamma_cm || !uv || !chi0 || !mt || !gamma_u || n_orb <= 0 || n2 > LOC_MAX_N2 || niv_core <= 0 ||
      niv_shell < 0 || niw_half <= 0 || 2 * niw_half > 65535) {
    dga_set_error("dga_local_fvertex_operands_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const int tiles = (Nf + 31) / 32;
  local_fvertex_operands_kernel<<<dim3(tiles, tiles, 2 * niw_half), dim3(32, 8), 0, stream>>>(
      (const double2*)gamma_cm, (const double2*)uv, (const double2*)chi0, n2, 2 * niv_core, nvf, niw_half, beta,
      (double2*)mt, (double2*)gamma_u);
  return launch_check("dga_local_fvertex_operands_c128");
}

int dga_local_sigma_c128(const void* vrg, const void* chi_phys, const void* uv, const void* u, const void* g,
                         const void* occ, int n_orb, int niv, int niw_half, int niv_g, double beta, void* inner,
                         void* sigma, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv;
  if (!vrg || !chi_phys || !uv || !u || !g || !occ || !inner || !sigma || n_orb <= 0 || n2 > LOC_MAX_N2 ||
      niv <= 0 || niw_half <= 0 || niv_g < niv + niw_half) {
    dga_set_error("dga_local_sigma_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  local_inner_kernel<<<niw_half * nv, 128, 0, stream>>>((const double2*)vrg, (const double2*)chi_phys,
                                                        (const double2*)uv, n2, nv, niw_half, (double2*)inner);
  int rc = launch_check("dga_local_sigma_c128");
  if (rc != DGA_OK) return rc;
  local_sigma_kernel<<<(n2 * nv + 127) / 128, 128, 0, stream>>>((const double2*)inner, (const double2*)u,
                                                               (const double2*)g, (const double2*)occ, n_orb, nv,
                                                               niw_half, niv_g, beta, (double2*)sigma);
  return launch_check("dga_local_sigma_c128");
}

}  // extern "C"
