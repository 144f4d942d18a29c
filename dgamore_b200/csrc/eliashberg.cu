// Eliashberg stage of the ladder hot path:
//
//   * dga_eli_full_vertex_c128: full ladder vertex in the pp frequency box for every (channel, q, w)
//       F_r = beta^2 (D - D chi* D) + (U_r - U_r chi_r U_r) gamma(nu) gamma(nu')
//     (eliashberg_solver.py:175-204 with chi* = A^-1, nonlocal_sde.py:72-82; D = blockdiag_nu chi0^-1).
//     Only the columns of chi* in the pp box are needed, so A is LU-factored once (the BSE core) and solved
//     against the unit vectors of the box, one box frequency (all n^2 orbital pairs) per solve;
//   * dga_eli_pairing_vertex_c128: the PH -> PP (w = 0) frequency transform of eliashberg_solver.py:44-75
//       F_pp[nu,nu'] = -F(w = nu - nu')[nu][-nu'-1], F(-w) = conj(flip F(w)),
//     the singlet/triplet combinations 1/2 F_d -/+ ... (eliashberg_solver.py:620-628) and the matrix layout
//     of the gap equation, Mat[(a,b,nu)][(c,d,nu')] = Gamma[a,c,b,d](nu,nu') (eliashberg_solver.py:418-425);
//   * dga_eli_chi0pp_c128: chi0pp[k][nu][(a,b)][(c,d)] = G_ad(k,nu) conj(G_cb(k,nu)) (bubble_gen.py:268-279);
//   * dga_eli_matvec_c128: one application of the linearised gap equation (eliashberg_solver.py:420-428):
//       g(R) = FFT_k[chi0pp . Delta],  new(R) = Gamma(R) g(R) + s Gamma(-R) g~(-R),  Delta' = IFFT_R(norm new)
//     where g~ is g transposed in its orbitals and reflected in nu (the flipped vertex of eliashberg_solver.py:
//     398-400 rewritten on Gamma(R) itself), so every Gamma(R) is streamed once per application.
#include "dga_common.cuh"

namespace dga {


}  // namespace dga

// The full-vertex kernel shares the LU core and the structured matrix source of the BSE and is implemented in
// bse.cu; this file holds the pp transform and the gap-equation kernels.

namespace dga {

// ------------------------------------------------------------------------------------------------
// pairing vertex: one thread per (st, q, I, J)
//   fph: [2][Q][Wpp][Mb][Mb], rows (p=(a,b), nu_box), cols (s=(d,c), nu'_box)  (p = a*n+b, s = d*n+c)
//   out: [2 (sing, trip)][Q][Mb][Mb], Mat[(a,b,nu)][(c,d,nu')] = Gamma[a,c,b,d](nu,nu')
// ------------------------------------------------------------------------------------------------
__global__ void eli_pairing_vertex_kernel(const double2* __restrict__ fph, int nb, int P, int Q, int Wpp,
                                          double2* __restrict__ out) {
  const int n2 = nb * nb, nvp = 2 * P, Mb = n2 * nvp;
  const long long total = 2LL * Q * Mb * Mb;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int J = (int)(e % Mb);
    const int I = (int)((e / Mb) % Mb);
    const int q = (int)((e / ((long long)Mb * Mb)) % Q);
    const int st = (int)(e / ((long long)Mb * Mb * Q));
    const int pI = I / nvp, nu = I - pI * nvp;
    const int pJ = J / nvp, nup = J - pJ * nvp;
    const int a = pI / nb, b = pI - a * nb;
    const int c = pJ / nb, d = pJ - c * nb;
    // Gamma[o1,o2,o3,o4] = Gamma[a,c,b,d]: F row (o1,o2) = (a,c), column (o4,o3) = (d,b)
    const int prow = a * nb + c, pcol = d * nb + b;
    double2 f[2];
    for (int ch = 0; ch < 2; ++ch) {
      const double2* base = fph + ((size_t)ch * Q + q) * Wpp * (size_t)Mb * Mb;
      double2 v;
      if (nu >= nup) {
        const int w = nu - nup;
        const int r = prow * nvp + nu, cidx = pcol * nvp + (nvp - 1 - nup);
        v = base[((size_t)w * Mb + r) * Mb + cidx];
      } else {
        const int w = nup - nu;
        const int r = prow * nvp + (nvp - 1 - nu), cidx = pcol * nvp + nup;
        v = base[((size_t)w * Mb + r) * Mb + cidx];
        v.y = -v.y;
      }
      f[ch] = make_double2(-v.x, -v.y);  // F_pp = -F(w = nu - nu')[nu][-nu'-1]
    }
    double2 g;
    if (st == 0) {  // singlet: 1/2 F_d - 3/2 F_m
      g = make_double2(0.5 * f[0].x + (-(1.5 * f[1].x)), 0.5 * f[0].y + (-(1.5 * f[1].y)));
    } else {  // triplet: 1/2 F_d + 1/2 F_m
      g = make_double2(0.5 * f[0].x + 0.5 * f[1].x, 0.5 * f[0].y + 0.5 * f[1].y);
    }
    out[(((size_t)st * Q + q) * Mb + I) * Mb + J] = g;
  }
}

// chi0pp[k][nu][(a,b)][(c,d)] = G_ad(k,nu) conj(G_cb(k,nu)) for nu in the pp box, filtered at 1e-12
//   g_k: [Nk][n][n][2 niv_g]
__global__ void eli_chi0pp_kernel(const double2* __restrict__ g_k, int nb, int niv_g, int P, int nk,
                                  double2* __restrict__ out) {
  const int n2 = nb * nb, nvp = 2 * P;
  const long long total = (long long)nk * nvp * n2 * n2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int cd = (int)(e % n2);
    const int ab = (int)((e / n2) % n2);
    const int v = (int)((e / ((long long)n2 * n2)) % nvp);
    const int k = (int)(e / ((long long)n2 * n2 * nvp));
    const int a = ab / nb, b = ab - a * nb, c = cd / nb, d = cd - c * nb;
    const int vi = niv_g - P + v;
    const double2 gad = g_k[(((size_t)k * nb + a) * nb + d) * 2 * niv_g + vi];
    const double2 gcb = g_k[(((size_t)k * nb + c) * nb + b) * 2 * niv_g + vi];
    double2 r = cmul(gad, cconj(gcb));
    if (fabs(r.x) < 1e-12 && fabs(r.y) < 1e-12) r = make_double2(0.0, 0.0);
    out[e] = r;
  }
}

// v[k][(a,b)][nu] = sum_{c,d} chi0pp[k][nu][(a,b)][(c,d)] Delta[k][(c,d)][nu]
__global__ void eli_apply_chi0pp_kernel(const double2* __restrict__ chi0pp, const double2* __restrict__ gap, int n2,
                                        int nvp, int nk, double2* __restrict__ v) {
  const long long total = (long long)nk * n2 * nvp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int nu = (int)(e % nvp);
    const int ab = (int)((e / nvp) % n2);
    const int k = (int)(e / ((long long)nvp * n2));
    const double2* c = chi0pp + (((size_t)k * nvp + nu) * n2 + ab) * n2;
    const double2* g = gap + (size_t)k * n2 * nvp + nu;
    double2 acc = make_double2(0.0, 0.0);
    for (int cd = 0; cd < n2; ++cd) cfma(acc, c[cd], g[(size_t)cd * nvp]);
    v[e] = acc;
  }
}

// Per R: direct[R][I] = sum_J Mat(R)[I][J] g(R)[J];  flip[R][I] = sum_J Mat(R)[I][J] g~(R)[J] with
// g~[(c,d),nu'] = g[(d,c), 2P-1-nu'].  One CTA per R (grid-stride), each warp two rows at a time with lanes
// over J and eight 16-byte loads of Mat(R) per lane in flight, so the Gamma(R) stream keeps enough bytes in
// flight per SM to run at HBM bandwidth.
//   gR: [Nk][n2][nvp] (forward transform of v), mat: [Nk][M][M]
// MT = double2: Gamma(R) in complex128; MT = float2: Gamma(R) stored in complex64 (half the bytes of the stream),
// widened on use, FP64 accumulation.  A warp takes RW rows at a time with U loads per lane and row in flight
// (U = 4 covers a row of up to 128 columns in one pass: M = 120 in the bilayer configuration); the complex64 form
// takes twice the rows so that the bytes in flight stay the same.
constexpr int ELI_APPLY_THREADS = 256;
template <typename MT, int U, int RW>
__global__ void __launch_bounds__(ELI_APPLY_THREADS) eli_vertex_apply_kernel(const MT* __restrict__ mat,
                                                                              const double2* __restrict__ gR, int nb,
                                                                              int nvp, int nk,
                                                                              double2* __restrict__ direct,
                                                                              double2* __restrict__ flip) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n2 = nb * nb, M = n2 * nvp;
  double2* g = reinterpret_cast<double2*>(smem_raw);
  double2* gt = g + M;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const MT zero = {};
  for (int R = blockIdx.x; R < nk; R += gridDim.x) {
    __syncthreads();
    for (int J = threadIdx.x; J < M; J += blockDim.x) {
      const int pJ = J / nvp, nup = J - pJ * nvp;
      const int c = pJ / nb, d = pJ - c * nb;
      g[J] = gR[(size_t)R * M + J];
      gt[J] = gR[(size_t)R * M + (d * nb + c) * nvp + (nvp - 1 - nup)];
    }
    __syncthreads();
    const MT* m = mat + (size_t)R * M * M;
    for (int I0 = RW * warp; I0 < M; I0 += RW * nw) {
      double2 a[RW], b[RW];
#pragma unroll
      for (int r = 0; r < RW; ++r) a[r] = b[r] = make_double2(0.0, 0.0);
      for (int J0 = 0; J0 < M; J0 += 32 * U) {
        MT x[RW][U];
#pragma unroll
        for (int r = 0; r < RW; ++r)
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int J = J0 + 32 * u + lane;
            x[r][u] = (I0 + r < M && J < M) ? m[(size_t)(I0 + r) * M + J] : zero;
          }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int J = J0 + 32 * u + lane;
          if (J < M) {
            const double2 gj = g[J], gtj = gt[J];
#pragma unroll
            for (int r = 0; r < RW; ++r) {
              const double2 xv = to_c64(x[r][u]);
              cfma(a[r], xv, gj);
              cfma(b[r], xv, gtj);
            }
          }
        }
      }
#pragma unroll
      for (int r = 0; r < RW; ++r)
        for (int off = 16; off > 0; off >>= 1) {
          a[r].x += __shfl_down_sync(0xffffffffu, a[r].x, off);
          a[r].y += __shfl_down_sync(0xffffffffu, a[r].y, off);
          b[r].x += __shfl_down_sync(0xffffffffu, b[r].x, off);
          b[r].y += __shfl_down_sync(0xffffffffu, b[r].y, off);
        }
      if (lane == 0) {
#pragma unroll
        for (int r = 0; r < RW; ++r)
          if (I0 + r < M) {
            direct[(size_t)R * M + I0 + r] = a[r];
            flip[(size_t)R * M + I0 + r] = b[r];
          }
      }
    }
  }
}

// tot[R][I] = direct[R][I] + sign * flip[-R][I]
__global__ void eli_combine_kernel(const double2* __restrict__ direct, const double2* __restrict__ flip, int M,
                                   int nx, int ny, int nz, double sign, double2* __restrict__ tot) {
  const int nk = nx * ny * nz;
  const long long total = (long long)nk * M;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(e % M);
    const int R = (int)(e / M);
    const int x = R / (ny * nz), rem = R - x * ny * nz, y = rem / nz, z = rem - y * nz;
    const int xm = x ? nx - x : 0, ym = y ? ny - y : 0, zm = z ? nz - z : 0;
    const int Rm = (xm * ny + ym) * nz + zm;
    const double2 a = direct[e], b = flip[(size_t)Rm * M + I];
    tot[e] = make_double2(a.x + sign * b.x, a.y + sign * b.y);
  }
}

}  // namespace dga

using namespace dga;

static int eli_status(const char* who) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("%s: launch failed: %s", who, cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

static int eli_blocks(long long work) {
  long long b = (work + 255) / 256;
  const long long cap = 16LL * device_sm_count();
  if (b > cap) b = cap;
  return (int)(b > 0 ? b : 1);
}

extern "C" {

// Pairing vertices (singlet, triplet) in the gap-equation layout from the PH full vertices of the pp box.
//   fph: [2 (dens, magn)][Q][Wpp][Mb][Mb]; out: [2 (sing, trip)][Q][Mb][Mb]; Mb = n^2 * 2P; Wpp >= 2P.
int dga_eli_pairing_vertex_c128(const void* fph, int n_orb, int niv_pp, int n_q, int w_pp, void* out,
                                cudaStream_t stream) {
  if (!fph || !out || n_orb <= 0 || niv_pp <= 0 || n_q <= 0 || w_pp < 2 * niv_pp) {
    dga_set_error("dga_eli_pairing_vertex_c128: invalid arguments (w_pp must cover 2 niv_pp)");
    return DGA_ERR_ARG;
  }
  const long long Mb = (long long)n_orb * n_orb * 2 * niv_pp;
  eli_pairing_vertex_kernel<<<eli_blocks(2LL * n_q * Mb * Mb), 256, 0, stream>>>(
      (const double2*)fph, n_orb, niv_pp, n_q, w_pp, (double2*)out);
  return eli_status("dga_eli_pairing_vertex_c128");
}

// chi0pp[Nk][2P][(a,b)][(c,d)] from G(k) [Nk][n][n][2 niv_g] (pp box centred at niv_g).
int dga_eli_chi0pp_c128(const void* g_k, int n_orb, int niv_g, int niv_pp, int nk, void* out, cudaStream_t stream) {
  if (!g_k || !out || n_orb <= 0 || niv_pp <= 0 || niv_g < niv_pp || nk <= 0) {
    dga_set_error("dga_eli_chi0pp_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const long long total = (long long)nk * 2 * niv_pp * n_orb * n_orb * n_orb * n_orb;
  eli_chi0pp_kernel<<<eli_blocks(total), 256, 0, stream>>>((const double2*)g_k, n_orb, niv_g, niv_pp, nk,
                                                           (double2*)out);
  return eli_status("dga_eli_chi0pp_c128");
}

// Bytes of the work buffer of dga_eli_matvec_c128 (four [Nk][M] vectors).
size_t dga_eli_matvec_scratch_bytes(int n_orb, int niv_pp, int nk) {
  return 4 * (size_t)nk * n_orb * n_orb * 2 * niv_pp * sizeof(double2);
}

// gap_out = IFFT_R[norm (Gamma(R) g(R) + sign Gamma(-R) g~(-R))], g = FFT_k(chi0pp . gap)
//   mat: [Nk][M][M] = sign_channel * FFT_q of the pairing vertex in the gap-equation layout (full BZ);
//   chi0pp: [Nk][2P][n2][n2]; gap, gap_out: [Nk][n2][2P]; tw_fwd / tw_inv: FFT twiddles (x, y, z)
int dga_dft_planes_c128(const void* in, long long in_s_hi, long long in_s_lo, long long in_s_r, void* out,
                        long long out_s_hi, long long out_s_lo, long long out_s_r, int n_lo, int n_planes, int nx,
                        int ny, int nz, const void* tw, double scale, cudaStream_t stream);

}  // extern "C"

// The gap-equation application with Gamma(R) stored as MT (complex128 or complex64); everything else FP64.
template <typename MT, int U, int RW>
static int eli_matvec(const char* who, const void* mat, const void* chi0pp, const void* gap, int n_orb, int niv_pp,
                      int nx, int ny, int nz, const void* tw_fwd, const void* tw_inv, double beta, double sign,
                      void* gap_out, void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nvp = 2 * niv_pp, M = n2 * nvp, nk = nx * ny * nz;
  if (!mat || !chi0pp || !gap || !gap_out || !scratch || !tw_fwd || !tw_inv || n_orb <= 0 || niv_pp <= 0 || nk <= 0) {
    dga_set_error("%s: invalid arguments", who);
    return DGA_ERR_ARG;
  }
  if (scratch_bytes < dga_eli_matvec_scratch_bytes(n_orb, niv_pp, nk)) {
    dga_set_error("%s: scratch too small", who);
    return DGA_ERR_SCRATCH;
  }
  double2* s0 = (double2*)scratch;
  double2* s1 = s0 + (size_t)nk * M;
  double2* s2 = s1 + (size_t)nk * M;
  double2* s3 = s2 + (size_t)nk * M;
  eli_apply_chi0pp_kernel<<<eli_blocks((long long)nk * M), 256, 0, stream>>>(
      (const double2*)chi0pp, (const double2*)gap, n2, nvp, nk, s0);
  if (eli_status(who)) return DGA_ERR_LAUNCH;
  int rc = dga_dft_planes_c128(s0, 1, 0, M, s1, 1, 0, M, 1, M, nx, ny, nz, tw_fwd, 1.0, stream);
  if (rc) return rc;
  const size_t smem = 2 * (size_t)M * sizeof(double2);
  cudaFuncSetAttribute(eli_vertex_apply_kernel<MT, U, RW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int apply_cap = 8 * device_sm_count();
  eli_vertex_apply_kernel<MT, U, RW><<<nk < apply_cap ? nk : apply_cap, ELI_APPLY_THREADS, smem, stream>>>(
      (const MT*)mat, s1, n_orb, nvp, nk, s2, s3);
  if (eli_status(who)) return DGA_ERR_LAUNCH;
  eli_combine_kernel<<<eli_blocks((long long)nk * M), 256, 0, stream>>>(s2, s3, M, nx, ny, nz, sign, s0);
  if (eli_status(who)) return DGA_ERR_LAUNCH;
  // ifftn(norm * new) with norm = 0.5 / (Nk beta) (eliashberg_solver.py:418, 428)
  const double norm = 0.5 / (double)nk / beta;
  return dga_dft_planes_c128(s0, 1, 0, M, gap_out, 1, 0, M, 1, M, nx, ny, nz, tw_inv, norm / (double)nk, stream);
}

// complex128 -> complex64 narrowing (round to nearest) of n elements.
__global__ void narrow_c64_kernel(const double2* __restrict__ src, float2* __restrict__ dst, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    dst[e] = make_float2((float)src[e].x, (float)src[e].y);
}

extern "C" {

int dga_eli_matvec_c128(const void* mat, const void* chi0pp, const void* gap, int n_orb, int niv_pp, int nx, int ny,
                        int nz, const void* tw_fwd, const void* tw_inv, double beta, double sign, void* gap_out,
                        void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  return eli_matvec<double2, 4, 2>("dga_eli_matvec_c128", mat, chi0pp, gap, n_orb, niv_pp, nx, ny, nz, tw_fwd, tw_inv,
                                beta, sign, gap_out, scratch, scratch_bytes, stream);
}

int dga_eli_matvec_c64mat_c128(const void* mat_c64, const void* chi0pp, const void* gap, int n_orb, int niv_pp, int nx,
                               int ny, int nz, const void* tw_fwd, const void* tw_inv, double beta, double sign,
                               void* gap_out, void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  return eli_matvec<float2, 4, 4>("dga_eli_matvec_c64mat_c128", mat_c64, chi0pp, gap, n_orb, niv_pp, nx, ny, nz, tw_fwd,
                               tw_inv, beta, sign, gap_out, scratch, scratch_bytes, stream);
}

int dga_narrow_c128_to_c64(const void* src, void* dst, long long n, cudaStream_t stream) {
  if (!src || !dst || n < 0) {
    dga_set_error("dga_narrow_c128_to_c64: invalid arguments");
    return DGA_ERR_ARG;
  }
  if (n == 0) return DGA_OK;
  narrow_c64_kernel<<<eli_blocks(n), 256, 0, stream>>>((const double2*)src, (float2*)dst, n);
  return eli_status("dga_narrow_c128_to_c64") ? DGA_ERR_LAUNCH : DGA_OK;
}

}  // extern "C"
