// Brillouin-zone transforms of the ladder hot path, all built on one shared-memory plane DFT:
//
//   * dga_dft_planes_c128: batched separable DFT of momentum planes (G(k) -> G(R), Sigma(R) -> Sigma(k));
//   * dga_bubble_c128:     chi0[q_irr,a,b,c,d,w,nu] = -beta/Nk * IFFT_R[G_ad(R,nu) G_cb(-R,nu-w)]
//                          (dgamore/bubble_gen.py:33-69), product, inverse transform, irreducible-q pick,
//                          scaling and the 1e-12 filter (n_point_base.py:205-211) fused in one kernel;
//   * dga_sigma_partial_c128 / dga_sigma_reduce_c128: Sigma_ij(R,nu) = sum_w sum_ad G_ad(R,nu-w) K_aijd(-R,w,nu)
//                          (nonlocal_sde.py:544-594), with K(-R) = sum_q K(q) e^{iqR} formed per plane from
//                          the irreducible kernel through the IBZ -> FBZ map (n_point_base.py:489-494) and the
//                          w < 0 half from K(q,-w,nu) = conj K(q,w,-nu-1) (local_n_point.py:191-225).
//
// A plane (Nk = nx*ny*nz points, C order) sits in shared memory; each axis is a direct DFT against a
// host-built FP64 twiddle table (e^{2 pi i m / n}, sign folded in), so the transform needs no FFT plan and
// handles any grid (16, 32, 48, 64, ...).  Work per plane is Nk*(nx+ny+nz) complex FMAs.
#include "dga_common.cuh"

namespace dga {

constexpr int BZ_THREADS = 256;
constexpr int BZ_MAX_NK = 4096;
constexpr int BZ_MAX_AXIS = 128;

struct Grid3 {
  int nx, ny, nz, nk;
};

// twiddle tables in shared memory: tw[0..nx) for x, then y, then z
__device__ __forceinline__ void load_twiddles(double2* s_tw, const double2* tw, const Grid3 g) {
  for (int i = threadIdx.x; i < g.nx + g.ny + g.nz; i += blockDim.x) s_tw[i] = tw[i];
}

// DFT along x of an nx x (ny nz) plane in shared memory (in -> out, both [x][yz]; twx = the nx twiddles),
// followed by a barrier.
constexpr int XR = 4;  // outputs per thread of the blocked axis passes
__device__ __forceinline__ void dft_axis_x(const double2* in, double2* out, const double2* twx, const Grid3 g) {
  const int T = blockDim.x, nyz = g.ny * g.nz;
  // A thread computes the outputs kx = grp + j ngx (j < XR) of one yz column, so each load serves XR
  // products (the twiddle loads are warp broadcasts); every output still sums over x in order.
  const int ngx = (g.nx + XR - 1) / XR;
  for (int t = threadIdx.x; t < ngx * nyz; t += T) {
    const int grp = t / nyz, yz = t - grp * nyz;
    double2 acc[XR];
    int m[XR], kx[XR];
#pragma unroll
    for (int j = 0; j < XR; ++j) {
      acc[j] = make_double2(0.0, 0.0);
      m[j] = 0;
      kx[j] = min(grp + j * ngx, g.nx - 1);  // outputs past nx are computed on a valid index and dropped
    }
    for (int x = 0; x < g.nx; ++x) {
      const double2 v = in[x * nyz + yz];
#pragma unroll
      for (int j = 0; j < XR; ++j) {
        cfma(acc[j], v, twx[m[j]]);
        m[j] += kx[j];
        if (m[j] >= g.nx) m[j] -= g.nx;
      }
    }
#pragma unroll
    for (int j = 0; j < XR; ++j)
      if (grp + j * ngx < g.nx) out[(grp + j * ngx) * nyz + yz] = acc[j];
  }
  __syncthreads();
}

// out[kx][y][z] = sum_x in[x][y][z] * twx[(kx*x) % nx], then along y, then z (skipped when the axis has
// length 1).  Result ends in `a` (the input buffer); `b` is work space.  Both buffers hold g.nk points.
__device__ void plane_dft(double2* a, double2* b, const double2* s_tw, const Grid3 g) {
  const int T = blockDim.x;
  const double2* twx = s_tw;
  const double2* twy = s_tw + g.nx;
  const double2* twz = s_tw + g.nx + g.ny;
  const int nyz = g.ny * g.nz;
  dft_axis_x(a, b, twx, g);  // x axis: a -> b
  const int ngx = (g.nx + XR - 1) / XR;
  // y axis: b -> a.  A thread computes the outputs of one (ky, z) for the rows kx = grp + j ngx (j < XR), so each
  // twiddle load (distinct across the lanes) serves XR products and the row loads are warp broadcasts; every
  // output still sums over y in order.
  for (int t = threadIdx.x; t < ngx * nyz; t += T) {
    const int grp = t / nyz, r = t - grp * nyz;
    const int ky = r / g.nz, z = r - ky * g.nz;
    double2 acc[XR];
    const double2* row[XR];
#pragma unroll
    for (int j = 0; j < XR; ++j) {
      acc[j] = make_double2(0.0, 0.0);
      row[j] = b + min(grp + j * ngx, g.nx - 1) * nyz + z;  // rows past nx are read on a valid row and dropped
    }
    int m = 0;
    for (int y = 0; y < g.ny; ++y) {
      const double2 w = twy[m];
#pragma unroll
      for (int j = 0; j < XR; ++j) cfma(acc[j], row[j][y * g.nz], w);
      m += ky;
      if (m >= g.ny) m -= g.ny;
    }
#pragma unroll
    for (int j = 0; j < XR; ++j)
      if (grp + j * ngx < g.nx) a[(grp + j * ngx) * nyz + r] = acc[j];
  }
  __syncthreads();
  if (g.nz > 1) {
    for (int e = threadIdx.x; e < g.nk; e += T) {
      const int base = (e / g.nz) * g.nz, kz = e - base;
      double2 acc = make_double2(0.0, 0.0);
      int m = 0;
      for (int z = 0; z < g.nz; ++z) {
        cfma(acc, a[base + z], twz[m]);
        m += kz;
        if (m >= g.nz) m -= g.nz;
      }
      b[e] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < g.nk; e += T) a[e] = b[e];
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// batched plane DFT with strided input/output addressing:
//   element (plane p = p_hi * n_lo + p_lo, point R) at p_hi*s_hi + p_lo*s_lo + R*s_r
// ------------------------------------------------------------------------------------------------
struct PlaneAddr {
  long long s_hi, s_lo, s_r;
  int n_lo;
  __device__ __forceinline__ long long at(int p, int r) const {
    const int hi = p / n_lo, lo = p - hi * n_lo;
    return hi * s_hi + lo * s_lo + (long long)r * s_r;
  }
};

__global__ void __launch_bounds__(BZ_THREADS) dft_planes_kernel(const double2* __restrict__ in, PlaneAddr ia,
                                                                 double2* __restrict__ out, PlaneAddr oa,
                                                                 int n_planes, Grid3 g,
                                                                 const double2* __restrict__ tw, double scale,
                                                                 const int* __restrict__ gather) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* a = reinterpret_cast<double2*>(smem_raw);
  double2* b = a + g.nk;
  double2* s_tw = b + g.nk;
  load_twiddles(s_tw, tw, g);
  for (int p = blockIdx.x; p < n_planes; p += gridDim.x) {
    __syncthreads();
    for (int r = threadIdx.x; r < g.nk; r += blockDim.x) a[r] = in[ia.at(p, gather ? gather[r] : r)];
    __syncthreads();
    plane_dft(a, b, s_tw, g);
    for (int r = threadIdx.x; r < g.nk; r += blockDim.x) {
      double2 v = a[r];
      out[oa.at(p, r)] = make_double2(v.x * scale, v.y * scale);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// bubble: one CTA per (w, nu, a, d), looping over (c, b)
//   g_r: [T][n][n][Nk] with slot t = nu_index + niv + niw (nu_index in [-niv-niw, niv))
// Per (c, b) plane P(R) = G_ad(R) G_cb(-R), stored transposed as P[(y, z)][x] so that reads across x are
// conflict-free; the (y, z) sums are taken only at the distinct (qy, qz) pairs of the irreducible q list
// (T[x][j] = sum_yz P[(y,z)][x] e^{i (qy_j y + qz_j z)}), then one x sum per irreducible q.  Work per plane
// Nk * n_pairs + Q * nx complex FMAs (the wedge of a 32 x 32 grid has 17 pairs: 22K instead of a full x transform
// plus the q sums, 38K).
// ------------------------------------------------------------------------------------------------
struct OutStrides7 {
  long long q, w, v, a, b, c, d;
};

constexpr int BUB_GR = 4;  // (qy, qz) pairs per thread in the (y, z) sums

__global__ void __launch_bounds__(BZ_THREADS, 3) bubble_kernel(const double2* __restrict__ g_r, int nb, int niv,
                                                             int niw, Grid3 g, const int* __restrict__ q_irr,
                                                             int n_qirr, const double2* __restrict__ tw,
                                                             double beta, double2* __restrict__ out,
                                                             OutStrides7 os) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ldp = g.nx + 1;  // padded row: the transposed stores of one warp spread over all banks
  double2* P = reinterpret_cast<double2*>(smem_raw);  // [yz][x], row stride ldp
  double2* Tt = P + (size_t)ldp * g.ny * g.nz;          // [x][pair]
  double2* s_tw = Tt + g.nk;
  int* s_q = reinterpret_cast<int*>(s_tw + g.nx + g.ny + g.nz);  // [n_qirr][3]
  int* s_j = s_q + 3 * n_qirr;                                    // pair index of each q
  int* s_pair = s_j + n_qirr;                                     // [n_pairs][2] (qy, qz)
  int* s_np = s_pair + 2 * n_qirr;
  load_twiddles(s_tw, tw, g);
  for (int i = threadIdx.x; i < 3 * n_qirr; i += blockDim.x) s_q[i] = q_irr[i];
  __syncthreads();
  // distinct (qy, qz) pairs in order of first appearance: s_j[i] = the first q with the same pair (i itself for
  // that first q), then, in q order, the first q of a pair numbers it and every later q copies its number (its
  // first q, at a smaller index, is already numbered)
  for (int i = threadIdx.x; i < n_qirr; i += blockDim.x) {
    int lead = i;
    for (int k = 0; k < i; ++k)
      if (s_q[3 * k + 1] == s_q[3 * i + 1] && s_q[3 * k + 2] == s_q[3 * i + 2]) {
        lead = k;
        break;
      }
    s_j[i] = lead;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int np = 0;
    for (int i = 0; i < n_qirr; ++i) {
      if (s_j[i] == i) {
        s_pair[2 * np] = s_q[3 * i + 1];
        s_pair[2 * np + 1] = s_q[3 * i + 2];
        s_j[i] = np++;
      } else {
        s_j[i] = s_j[s_j[i]];
      }
    }
    *s_np = np;
  }
  __syncthreads();
  const int np = *s_np;

  const int nv = 2 * niv, W = niw + 1;
  const int n2 = nb * nb;
  const int total = W * nv * n2;
  const int nyz = g.ny * g.nz;
  const double inv_nk = 1.0 / (double)g.nk;
  const double pref = -beta / (double)g.nk;
  const double2* twx = s_tw;
  const double2* twy = s_tw + g.nx;
  const double2* twz = s_tw + g.nx + g.ny;
  const int ngp = (np + BUB_GR - 1) / BUB_GR;
  for (int blk = blockIdx.x; blk < total; blk += gridDim.x) {
    const int ad = blk % n2;
    const int v = (blk / n2) % nv;
    const int w = blk / (n2 * nv);
    const int a = ad / nb, d = ad - a * nb;
    const int t1 = v + niw;      // G(nu)
    const int t2 = v + niw - w;  // G(nu - w)
    const double2* gad = g_r + (((size_t)t1 * nb + a) * nb + d) * g.nk;
    for (int cb = 0; cb < n2; ++cb) {
      const int c = cb / nb, b = cb - c * nb;
      const double2* gcb = g_r + (((size_t)t2 * nb + c) * nb + b) * g.nk;
      __syncthreads();
      for (int r = threadIdx.x; r < g.nk; r += blockDim.x) {
        const int x = r / nyz, yz = r - x * nyz, y = yz / g.nz, z = yz - y * g.nz;
        const int xm = x ? g.nx - x : 0, ym = y ? g.ny - y : 0, zm = z ? g.nz - z : 0;
        P[yz * ldp + x] = cmul(gad[r], gcb[(xm * g.ny + ym) * g.nz + zm]);
      }
      __syncthreads();
      // T[x][j] for BUB_GR pairs j per thread: consecutive threads take consecutive x (conflict-free P reads)
      for (int t = threadIdx.x; t < g.nx * ngp; t += blockDim.x) {
        const int x = t % g.nx, jg = t / g.nx;
        double2 acc[BUB_GR];
        int jy[BUB_GR], jz[BUB_GR], my[BUB_GR], mz[BUB_GR];
#pragma unroll
        for (int u = 0; u < BUB_GR; ++u) {
          const int j = min(jg * BUB_GR + u, np - 1);  // pairs past np are computed on a valid pair and dropped
          acc[u] = make_double2(0.0, 0.0);
          jy[u] = s_pair[2 * j];
          jz[u] = s_pair[2 * j + 1];
          my[u] = 0;
        }
        for (int y = 0; y < g.ny; ++y) {
#pragma unroll
          for (int u = 0; u < BUB_GR; ++u) mz[u] = 0;
          for (int z = 0; z < g.nz; ++z) {
            const double2 pv = P[(y * g.nz + z) * ldp + x];
#pragma unroll
            for (int u = 0; u < BUB_GR; ++u) {
              const double2 tt = g.nz > 1 ? cmul(twy[my[u]], twz[mz[u]]) : twy[my[u]];
              cfma(acc[u], pv, tt);
              mz[u] += jz[u];
              if (mz[u] >= g.nz) mz[u] -= g.nz;
            }
          }
#pragma unroll
          for (int u = 0; u < BUB_GR; ++u) {
            my[u] += jy[u];
            if (my[u] >= g.ny) my[u] -= g.ny;
          }
        }
#pragma unroll
        for (int u = 0; u < BUB_GR; ++u)
          if (jg * BUB_GR + u < np) Tt[x * np + jg * BUB_GR + u] = acc[u];
      }
      __syncthreads();
      for (int iq = threadIdx.x; iq < n_qirr; iq += blockDim.x) {
        const int qx = s_q[3 * iq], j = s_j[iq];
        double2 acc = make_double2(0.0, 0.0);
        int mx = 0;
        for (int x = 0; x < g.nx; ++x) {
          cfma(acc, Tt[x * np + j], twx[mx]);
          mx += qx;
          if (mx >= g.nx) mx -= g.nx;
        }
        double re = (acc.x * inv_nk) * pref;
        double im = (acc.y * inv_nk) * pref;
        if (fabs(re) < 1e-12 && fabs(im) < 1e-12) {
          re = 0.0;
          im = 0.0;
        }
        out[iq * os.q + w * os.w + v * os.v + a * os.a + b * os.b + c * os.c + d * os.d] = make_double2(re, im);
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Sigma through the irreducible wedge of real space.  Without per-k orbital rotations the full-zone kernel is
// K(q) = K_irr(rep q), invariant under the grid's point group, and so is F(R) = sum_q K(q) e^{iqR}: it is needed
// only at the irreducible R, where it is one complex GEMM over the irreducible q,
//   Kw[plane][r] = sum_{q_irr} K[q_irr][plane] S[q_irr][r],   S[q_irr][r] = sum_{q in star(q_irr)} e^{i q R_r},
// (plane = (w, nu, row, col)), and the contraction reads F(R) = Kw[plane][rep R] (w < 0: the conjugate, since
// R and -R share a representative when the group holds the inversion).  Work: Q^2 per plane instead of a plane
// transform of Nk (nx + ny + nz).
// ------------------------------------------------------------------------------------------------
constexpr int SW_TK = 16;

// C[p][r] = sum_q A[q][p] B[q][r]: A = K [Q][P] (planes contiguous), B = S [Q][Q], C = Kw [P][Q].  A TM x TN output
// tile per 256-thread CTA, 4 x 4 per thread (TM * TN = 4096), K in steps of 16 with the next step's operands loaded
// into registers while the current one multiplies.
template <int TM, int TN>
__global__ void __launch_bounds__(256, 2) sigma_wedge_gemm_kernel(const double2* __restrict__ A,
                                                                  const double2* __restrict__ B, long long P, int Q,
                                                                  double2* __restrict__ C) {
  static_assert(TM * TN == 4096, "4 x 4 outputs per thread of 256");
  constexpr int AL = TM * SW_TK / 256, BL = TN * SW_TK / 256;  // tile elements loaded per thread
  __shared__ double2 As[SW_TK][TM + 1];
  __shared__ double2 Bs[SW_TK][TN];
  const long long p0 = (long long)blockIdx.x * TM;
  const int r0 = blockIdx.y * TN;
  const int tid = threadIdx.x, ty = tid % (TM / 4), tx = tid / (TM / 4);
  double2 ra[AL], rb[BL];
  auto load = [&](int k0) {
#pragma unroll
    for (int i = 0; i < AL; ++i) {  // element e = tid + 256 i of the TK x TM tile: row q = e / TM, column e % TM
      const int e = tid + 256 * i, q = k0 + e / TM;
      const long long p = p0 + e % TM;
      ra[i] = (q < Q && p < P) ? A[(size_t)q * P + p] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int i = 0; i < BL; ++i) {
      const int e = tid + 256 * i, q = k0 + e / TN, r = r0 + e % TN;
      rb[i] = (q < Q && r < Q) ? B[(size_t)q * Q + r] : make_double2(0.0, 0.0);
    }
  };
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
  load(0);
  for (int k0 = 0; k0 < Q; k0 += SW_TK) {
#pragma unroll
    for (int i = 0; i < AL; ++i) {
      const int e = tid + 256 * i;
      As[e / TM][e % TM] = ra[i];
    }
#pragma unroll
    for (int i = 0; i < BL; ++i) {
      const int e = tid + 256 * i;
      Bs[e / TN][e % TN] = rb[i];
    }
    __syncthreads();
    if (k0 + SW_TK < Q) load(k0 + SW_TK);
#pragma unroll
    for (int kk = 0; kk < SW_TK; ++kk) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty + (TM / 4) * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx + (TN / 4) * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long long p = p0 + ty + (TM / 4) * i;
    if (p >= P) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + tx + (TN / 4) * j;
      if (r < Q) C[(size_t)p * Q + r] = acc[i][j];
    }
  }
}

// Partial sums of the wedge form: as sigma_partial_kernel, with the plane K(-R) read from Kw through the
// representative of each R instead of transformed.  kw: [W][nv][n2][n2][Q] (plane-major).
template <int MAXR>
__global__ void __launch_bounds__(BZ_THREADS, MAXR <= 4 ? 3 : 1)
    sigma_wedge_partial_kernel(const double2* __restrict__ kw, const double2* __restrict__ g_r, int nb, int niv,
                               int niw, int Q, int nk, const int* __restrict__ irrk_inv, int n_chunks,
                               double2* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int* s_inv = reinterpret_cast<int*>(smem_raw);
  for (int i = threadIdx.x; i < nk; i += blockDim.x) s_inv[i] = irrk_inv[i];
  __syncthreads();
  const int n2 = nb * nb, nv = 2 * niv, nwf = 2 * niw + 1;
  const int per_chunk = (nwf + n_chunks - 1) / n_chunks;
  const int total = niv * n2 * n_chunks;
  int rep[MAXR];
#pragma unroll
  for (int k = 0; k < MAXR; ++k) {
    const int r = threadIdx.x + k * BZ_THREADS;
    rep[k] = r < nk ? s_inv[r] : 0;
  }
  for (int blk = blockIdx.x; blk < total; blk += gridDim.x) {
    const int chunk = blk % n_chunks;
    const int ij = (blk / n_chunks) % n2;
    const int v = blk / (n_chunks * n2);
    const int i = ij / nb, j = ij - i * nb;
    double2 acc[MAXR];
#pragma unroll
    for (int k = 0; k < MAXR; ++k) acc[k] = make_double2(0.0, 0.0);
    const int wf0 = chunk * per_chunk, wf1 = min(nwf, wf0 + per_chunk);
    for (int wf = wf0; wf < wf1; ++wf) {
      const int w = wf - niw;
      const bool neg = w < 0;
      const int wa = neg ? -w : w;
      const int vi = neg ? (niv - 1 - v) : (niv + v);
      for (int ad = 0; ad < n2; ++ad) {
        const int a = ad / nb, d = ad - a * nb;
        const int row = a * nb + i, col = d * nb + j;
        const double2* plane = kw + ((((size_t)wa * nv + vi) * n2 + row) * n2 + col) * Q;
        const double2* gp = g_r + (((size_t)(v - w + niw) * nb + a) * nb + d) * nk;
#pragma unroll
        for (int k = 0; k < MAXR; ++k) {
          const int r = threadIdx.x + k * BZ_THREADS;
          if (r < nk) {
            double2 kv = plane[rep[k]];
            if (neg) kv.y = -kv.y;
            cfma(acc[k], gp[r], kv);
          }
        }
      }
    }
    double2* o = part + (((size_t)chunk * niv + v) * n2 + ij) * nk;
#pragma unroll
    for (int k = 0; k < MAXR; ++k) {
      const int r = threadIdx.x + k * BZ_THREADS;
      if (r < nk) o[r] = acc[k];
    }
  }
}

// ------------------------------------------------------------------------------------------------
// IBZ -> FBZ with the auto-mode orbital rotation (n_point_base.py:462-507, symmetry_reduction.py:791-902):
//   dst[k](o1,o2,o3,o4; f) = sigma_k^2 sum U_{o1 p} U*_{o2 q} U_{o3 r} U*_{o4 s} [src[irrk_inv[k]](p,q,r,s; f)]^(*conj_k)
// for four-orbital objects whose per-k block holds the orbital indices at strides st[0..3] and frequency pairs
// (f1 < F1, f2 < F2) at f1 t1 + f2 t2.  One CTA per (k, chunk of frequency pairs): the chunk is staged in shared
// memory and transformed one orbital index at a time (n-term sums); a point whose U_k is the identity without
// conjugation is a plain copy.
// ------------------------------------------------------------------------------------------------
struct RotLayout {
  long long st[4];
  long long t1, t2;
  int F1, F2;
  long long block;  // elements per k
};

__global__ void __launch_bounds__(BZ_THREADS) fbz_rotate_kernel(const double2* __restrict__ src,
                                                                 const int* __restrict__ irrk_inv,
                                                                 const double2* __restrict__ us,
                                                                 const double* __restrict__ sigmas,
                                                                 const unsigned char* __restrict__ conjs, int n,
                                                                 RotLayout L, int fc, double2* __restrict__ dst) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n4 = n * n * n * n;
  double2* X = reinterpret_cast<double2*>(smem_raw);  // [fc][n4]
  double2* Y = X + (size_t)fc * n4;
  __shared__ double2 U[16];
  __shared__ int ident;
  const int k = blockIdx.y;
  const long long nf = (long long)L.F1 * L.F2;
  const long long f0 = (long long)blockIdx.x * fc;
  if (f0 >= nf) return;
  const int nfc = (int)min((long long)fc, nf - f0);
  const int tid = threadIdx.x, T = blockDim.x;
  if (tid < n * n) U[tid] = us[(size_t)k * n * n + tid];
  __syncthreads();
  if (tid == 0) {
    int id = conjs[k] ? 0 : 1;
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        const double2 u = U[a * n + b];
        if (u.y != 0.0 || u.x != (a == b ? 1.0 : 0.0)) id = 0;
      }
    ident = id;
  }
  __syncthreads();
  const double2* s = src + (size_t)irrk_inv[k] * L.block;
  double2* d = dst + (size_t)k * L.block;
  auto offset = [&](int fl, int e) -> long long {
    const long long f = f0 + fl;
    const int f1 = (int)(f / L.F2), f2 = (int)(f - (long long)f1 * L.F2);
    const int o4 = e % n, o3 = (e / n) % n, o2 = (e / (n * n)) % n, o1 = e / (n * n * n);
    return f1 * L.t1 + f2 * L.t2 + o1 * L.st[0] + o2 * L.st[1] + o3 * L.st[2] + o4 * L.st[3];
  };
  if (ident) {
    for (int e = tid; e < nfc * n4; e += T) {
      const long long off = offset(e / n4, e % n4);
      d[off] = s[off];
    }
    return;
  }
  const bool cj = conjs[k] != 0;
  for (int e = tid; e < nfc * n4; e += T) {
    double2 v = s[offset(e / n4, e % n4)];
    if (cj) v.y = -v.y;
    X[e] = v;
  }
  __syncthreads();
  // one orbital index at a time: position 0 and 2 with U, 1 and 3 with U*
  int stride = n * n * n;
  for (int pos = 0; pos < 4; ++pos) {
    const bool dag = (pos & 1) != 0;
    for (int e = tid; e < nfc * n4; e += T) {
      const int fl = e / n4, r = e - fl * n4;
      const int a = (r / stride) % n, base = r - a * stride;
      double2 acc = make_double2(0.0, 0.0);
      for (int p = 0; p < n; ++p) {
        double2 u = U[a * n + p];
        if (dag) u.y = -u.y;
        cfma(acc, u, X[(size_t)fl * n4 + base + p * stride]);
      }
      Y[e] = acc;
    }
    __syncthreads();
    double2* t = X;
    X = Y;
    Y = t;
    stride /= n;
  }
  const double sg = sigmas ? sigmas[k] * sigmas[k] : 1.0;
  for (int e = tid; e < nfc * n4; e += T) {
    const double2 v = X[e];
    d[offset(e / n4, e % n4)] = make_double2(sg * v.x, sg * v.y);
  }
}

// ------------------------------------------------------------------------------------------------
// Sigma partial sums: CTA per (nu >= 0, i, j, w-chunk)
//   kern: [Q][W][nv][n2][n2] irreducible kernel, matrix row (a,i), column (d,j); W = niw+1, nv = 2 niv
//   g_r:  [T][n][n][Nk] with slot t = nu_index + niw, nu_index in [-niw, niv+niw)
//   part: [n_chunks][niv][n2][Nk]
//   MAXR: accumulators per thread (Nk <= MAXR * BZ_THREADS), so small grids hold fewer registers and keep more
//   CTAs resident
// ------------------------------------------------------------------------------------------------
template <int MAXR>
__global__ void __launch_bounds__(BZ_THREADS, MAXR <= 4 ? 3 : 1) sigma_partial_kernel(const double2* __restrict__ kern,
                                                                    const double2* __restrict__ g_r, int nb, int niv,
                                                                    int niw, int Q, Grid3 g,
                                                                    const int* __restrict__ irrk_inv,
                                                                    const double2* __restrict__ tw, int n_chunks,
                                                                    double2* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* Pa = reinterpret_cast<double2*>(smem_raw);
  double2* Pb = Pa + g.nk;
  double2* s_tw = Pb + g.nk;
  int* s_inv = reinterpret_cast<int*>(s_tw + g.nx + g.ny + g.nz);
  load_twiddles(s_tw, tw, g);
  for (int i = threadIdx.x; i < g.nk; i += blockDim.x) s_inv[i] = irrk_inv[i];

  const int n2 = nb * nb, nv = 2 * niv, W = niw + 1, nwf = 2 * niw + 1;
  const int per_chunk = (nwf + n_chunks - 1) / n_chunks;
  const int total = niv * n2 * n_chunks;
  for (int blk = blockIdx.x; blk < total; blk += gridDim.x) {
    const int chunk = blk % n_chunks;
    const int ij = (blk / n_chunks) % n2;
    const int v = blk / (n_chunks * n2);
    const int i = ij / nb, j = ij - i * nb;
    double2 acc[MAXR];
#pragma unroll
    for (int k = 0; k < MAXR; ++k) acc[k] = make_double2(0.0, 0.0);
    const int wf0 = chunk * per_chunk, wf1 = min(nwf, wf0 + per_chunk);
    for (int wf = wf0; wf < wf1; ++wf) {
      const int w = wf - niw;
      const bool neg = w < 0;
      const int wa = neg ? -w : w;
      const int vi = neg ? (niv - 1 - v) : (niv + v);
      for (int ad = 0; ad < n2; ++ad) {
        const int a = ad / nb, d = ad - a * nb;
        const int row = a * nb + i, col = d * nb + j;
        __syncthreads();
        for (int r = threadIdx.x; r < g.nk; r += blockDim.x) {
          double2 kv = kern[((((size_t)s_inv[r] * W + wa) * nv + vi) * n2 + row) * n2 + col];
          if (neg) kv.y = -kv.y;
          Pa[r] = kv;
        }
        __syncthreads();
        plane_dft(Pa, Pb, s_tw, g);
        const double2* gp = g_r + (((size_t)(v - w + niw) * nb + a) * nb + d) * g.nk;
#pragma unroll
        for (int k = 0; k < MAXR; ++k) {
          const int r = threadIdx.x + k * BZ_THREADS;
          if (r < g.nk) cfma(acc[k], gp[r], Pa[r]);
        }
      }
    }
    double2* o = part + (((size_t)chunk * niv + v) * n2 + ij) * g.nk;
#pragma unroll
    for (int k = 0; k < MAXR; ++k) {
      const int r = threadIdx.x + k * BZ_THREADS;
      if (r < g.nk) o[r] = acc[k];
    }
  }
}

// Neumaier-compensated sum over the chunk partials, times -1/2 / (beta Nk): sig_r[niv][n2][Nk]
__global__ void sigma_reduce_kernel(const double2* __restrict__ part, int n_chunks, long long n_out, double factor,
                                    double2* __restrict__ sig_r) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_out;
       e += (long long)gridDim.x * blockDim.x) {
    double sr = 0.0, cr = 0.0, si = 0.0, ci = 0.0;
    for (int c = 0; c < n_chunks; ++c) {
      const double2 x = part[(size_t)c * n_out + e];
      double t = sr + x.x;
      cr += (fabs(sr) >= fabs(x.x)) ? (sr - t) + x.x : (x.x - t) + sr;
      sr = t;
      t = si + x.y;
      ci += (fabs(si) >= fabs(x.y)) ? (si - t) + x.y : (x.y - t) + si;
      si = t;
    }
    sig_r[e] = make_double2((sr + cr) * factor, (si + ci) * factor);
  }
}

// Sigma(k) planes [niv][n][n][Nk] -> upstream layout [Nk][n][n][2 niv] with the nu < 0 half as
// conj(Sigma(k, -nu-1)) (self_energy.py:109-120)
__global__ void sigma_full_nu_kernel(const double2* __restrict__ sig_k, int nb, int niv, int nk,
                                     double2* __restrict__ out) {
  const int n2 = nb * nb;
  const long long total = (long long)niv * n2 * nk;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % nk);
    const int ij = (int)((e / nk) % n2);
    const int v = (int)(e / ((long long)nk * n2));
    const double2 s = sig_k[e];
    double2* o = out + ((size_t)r * n2 + ij) * 2 * niv;
    o[niv + v] = s;
    o[niv - 1 - v] = make_double2(s.x, -s.y);
  }
}

}  // namespace dga

using namespace dga;

static int check_grid(int nx, int ny, int nz, const char* who) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || nx > BZ_MAX_AXIS || ny > BZ_MAX_AXIS || nz > BZ_MAX_AXIS ||
      nx * ny * nz > BZ_MAX_NK) {
    dga_set_error("%s: unsupported momentum grid %dx%dx%d (at most %d points, %d per axis)", who, nx, ny, nz,
                  BZ_MAX_NK, BZ_MAX_AXIS);
    return DGA_ERR_ARG;
  }
  return DGA_OK;
}

static int launch_status(const char* who) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("%s: launch failed: %s", who, cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

static int grid_cap(long long work) {
  const long long cap = 8LL * device_sm_count();
  long long g = work < cap ? work : cap;
  return (int)(g > 0 ? g : 1);
}

extern "C" {

// Batched separable DFT of momentum planes.  tw holds nx + ny + nz FP64 twiddles e^{s 2 pi i m / n}
// (the caller folds the sign s in); each plane is multiplied by `scale` on output.
int dga_dft_planes_c128(const void* in, long long in_s_hi, long long in_s_lo, long long in_s_r, void* out,
                        long long out_s_hi, long long out_s_lo, long long out_s_r, int n_lo, int n_planes, int nx,
                        int ny, int nz, const void* tw, double scale, cudaStream_t stream) {
  if (check_grid(nx, ny, nz, "dga_dft_planes_c128")) return DGA_ERR_ARG;
  if (!in || !out || !tw || n_planes <= 0 || n_lo <= 0) {
    dga_set_error("dga_dft_planes_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  Grid3 g{nx, ny, nz, nx * ny * nz};
  PlaneAddr ia{in_s_hi, in_s_lo, in_s_r, n_lo}, oa{out_s_hi, out_s_lo, out_s_r, n_lo};
  const size_t smem = (2 * (size_t)g.nk + nx + ny + nz) * sizeof(double2);
  cudaFuncSetAttribute(dft_planes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dft_planes_kernel<<<grid_cap(n_planes), BZ_THREADS, smem, stream>>>((const double2*)in, ia, (double2*)out, oa,
                                                                      n_planes, g, (const double2*)tw, scale, nullptr);
  return launch_status("dga_dft_planes_c128");
}

// Same as dga_dft_planes_c128 with the input point of output R read from gather[R] (an IBZ -> FBZ expansion
// by the inverse irreducible map, n_point_base.py:489-494, folded into the transform's load).
int dga_dft_planes_gather_c128(const void* in, long long in_s_hi, long long in_s_lo, long long in_s_r, void* out,
                               long long out_s_hi, long long out_s_lo, long long out_s_r, int n_lo, int n_planes,
                               int nx, int ny, int nz, const void* tw, double scale, const int* gather,
                               cudaStream_t stream) {
  if (check_grid(nx, ny, nz, "dga_dft_planes_gather_c128")) return DGA_ERR_ARG;
  if (!in || !out || !tw || !gather || n_planes <= 0 || n_lo <= 0) {
    dga_set_error("dga_dft_planes_gather_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  Grid3 g{nx, ny, nz, nx * ny * nz};
  PlaneAddr ia{in_s_hi, in_s_lo, in_s_r, n_lo}, oa{out_s_hi, out_s_lo, out_s_r, n_lo};
  const size_t smem = (2 * (size_t)g.nk + nx + ny + nz) * sizeof(double2);
  cudaFuncSetAttribute(dft_planes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dft_planes_kernel<<<grid_cap(n_planes), BZ_THREADS, smem, stream>>>((const double2*)in, ia, (double2*)out, oa,
                                                                      n_planes, g, (const double2*)tw, scale, gather);
  return launch_status("dga_dft_planes_gather_c128");
}

// Fused bubble.  g_r: [2 niv + niw][n][n][Nk] forward transforms of G(k) for nu indices [-niv-niw, niv);
// q_irr: [n_qirr][3] index triples; tw: inverse-transform twiddles (e^{+2 pi i m/n}); out addressed by the
// seven element strides (q, w, nu, a, b, c, d).
int dga_bubble_c128(const void* g_r, int n_orb, int niv, int niw, int nx, int ny, int nz, const int* q_irr,
                    int n_qirr, const void* tw, double beta, void* out, const long long* out_strides,
                    cudaStream_t stream) {
  if (check_grid(nx, ny, nz, "dga_bubble_c128")) return DGA_ERR_ARG;
  if (!g_r || !q_irr || !tw || !out || !out_strides || n_orb <= 0 || niv <= 0 || niw < 0 || n_qirr <= 0) {
    dga_set_error("dga_bubble_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  Grid3 g{nx, ny, nz, nx * ny * nz};
  OutStrides7 os{out_strides[0], out_strides[1], out_strides[2], out_strides[3],
                 out_strides[4], out_strides[5], out_strides[6]};
  if ((long long)n_qirr > (long long)g.nk) {
    dga_set_error("dga_bubble_c128: more irreducible q points (%d) than grid points", n_qirr);
    return DGA_ERR_ARG;
  }
  const size_t smem = (2 * (size_t)g.nk + (size_t)ny * nz + nx + ny + nz) * sizeof(double2) +
                      (6 * (size_t)n_qirr + 1) * sizeof(int);
  cudaFuncSetAttribute(bubble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const long long work = (long long)(niw + 1) * 2 * niv * n_orb * n_orb;
  const long long cap = 64LL * device_sm_count();
  bubble_kernel<<<(int)(work < cap ? work : cap), BZ_THREADS, smem, stream>>>(
      (const double2*)g_r, n_orb, niv, niw, g, q_irr, n_qirr, (const double2*)tw, beta, (double2*)out, os);
  return launch_status("dga_bubble_c128");
}

size_t dga_sigma_scratch_bytes(int n_orb, int niv, int nk, int n_chunks);

// Scratch bytes of dga_sigma_wedge_c128: the partial sums of dga_sigma_c128 plus the wedge transform Kw.
size_t dga_sigma_wedge_scratch_bytes(int n_orb, int niv, int niw, int n_q, int nk, int n_chunks) {
  const size_t planes = (size_t)(niw + 1) * 2 * niv * n_orb * n_orb * n_orb * n_orb;
  return dga_sigma_scratch_bytes(n_orb, niv, nk, n_chunks) + planes * (size_t)n_q * sizeof(double2);
}

// dga_sigma_c128 through the irreducible wedge of real space (see sigma_wedge_gemm_kernel); s_star [Q][Q] is
// S[q_irr][r] = sum over the star of q_irr of e^{+i q R_r} for the irreducible R_r = the points irrk_ind names.
int dga_sigma_wedge_c128(const void* kern, const void* g_r, int n_orb, int niv, int niw, int n_q, int nx, int ny,
                         int nz, const int* irrk_inv, const void* s_star, const void* tw_inv, double beta,
                         int n_chunks, int gemm_tile, void* out, void* scratch, size_t scratch_bytes,
                         cudaStream_t stream) {
  if (check_grid(nx, ny, nz, "dga_sigma_wedge_c128")) return DGA_ERR_ARG;
  if (!kern || !g_r || !irrk_inv || !s_star || !tw_inv || !out || !scratch || n_orb <= 0 || niv <= 0 || niw < 0 ||
      n_q <= 0 || n_chunks <= 0 || gemm_tile < 0 || gemm_tile > 1) {
    dga_set_error("dga_sigma_wedge_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  Grid3 g{nx, ny, nz, nx * ny * nz};
  const int n2 = n_orb * n_orb;
  const size_t need = dga_sigma_wedge_scratch_bytes(n_orb, niv, niw, n_q, g.nk, n_chunks);
  if (scratch_bytes < need) {
    dga_set_error("dga_sigma_wedge_c128: scratch too small (%zu < %zu)", scratch_bytes, need);
    return DGA_ERR_SCRATCH;
  }
  double2* part = (double2*)scratch;
  double2* sig = part + (size_t)n_chunks * niv * n2 * g.nk;
  double2* kw = sig + (size_t)niv * n2 * g.nk;
  const long long P = (long long)(niw + 1) * 2 * niv * n2 * n2;
  // GEMM tile (rows of planes x columns of irreducible R): 0 = 64 x 64, 1 = 128 x 32
  auto gemm = [&](auto kernel, int tm, int tn) {
    dim3 ggrid((unsigned)((P + tm - 1) / tm), (unsigned)((n_q + tn - 1) / tn));
    kernel<<<ggrid, 256, 0, stream>>>((const double2*)kern, (const double2*)s_star, P, n_q, kw);
  };
  if (gemm_tile == 0) gemm(sigma_wedge_gemm_kernel<64, 64>, 64, 64);
  else gemm(sigma_wedge_gemm_kernel<128, 32>, 128, 32);
  if (launch_status("dga_sigma_wedge_c128")) return DGA_ERR_LAUNCH;
  const size_t smem = sizeof(int) * (size_t)g.nk;
  const long long work = (long long)niv * n2 * n_chunks;
  auto partial = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kernel<<<grid_cap(work), BZ_THREADS, smem, stream>>>(kw, (const double2*)g_r, n_orb, niv, niw, n_q, g.nk,
                                                         irrk_inv, n_chunks, part);
  };
  if (g.nk <= 4 * BZ_THREADS) partial(sigma_wedge_partial_kernel<4>);
  else if (g.nk <= 8 * BZ_THREADS) partial(sigma_wedge_partial_kernel<8>);
  else partial(sigma_wedge_partial_kernel<16>);
  if (launch_status("dga_sigma_wedge_c128")) return DGA_ERR_LAUNCH;
  const long long n_out = (long long)niv * n2 * g.nk;
  sigma_reduce_kernel<<<grid_cap((n_out + 255) / 256), 256, 0, stream>>>(part, n_chunks, n_out,
                                                                         -0.5 / beta / (double)g.nk, sig);
  if (launch_status("dga_sigma_wedge_c128")) return DGA_ERR_LAUNCH;
  const size_t dsmem = (2 * (size_t)g.nk + nx + ny + nz) * sizeof(double2);
  cudaFuncSetAttribute(dft_planes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem);
  PlaneAddr pa{(long long)g.nk, 0, 1, 1};
  dft_planes_kernel<<<grid_cap(niv * n2), BZ_THREADS, dsmem, stream>>>(sig, pa, part, pa, niv * n2, g,
                                                                       (const double2*)tw_inv, 1.0 / (double)g.nk,
                                                                       nullptr);
  if (launch_status("dga_sigma_wedge_c128")) return DGA_ERR_LAUNCH;
  sigma_full_nu_kernel<<<grid_cap((n_out + 255) / 256), 256, 0, stream>>>(part, n_orb, niv, g.nk, (double2*)out);
  return launch_status("dga_sigma_wedge_c128");
}

// Expansion of a four-orbital object from the irreducible to the full zone with the auto-mode orbital rotation;
// layout and arguments in include/dga_b200.h.
int dga_fbz_rotate_c128(const void* src, const int* irrk_inv, int nk, const void* us, const double* sigmas,
                        const unsigned char* conjs, int n_orb, const long long* orb_strides, long long f1_stride,
                        int f1_count, long long f2_stride, int f2_count, long long block, void* dst,
                        cudaStream_t stream) {
  if (!src || !irrk_inv || !us || !conjs || !orb_strides || !dst || n_orb <= 0 || n_orb > 4 || nk <= 0 ||
      nk > 65535 || f1_count <= 0 || f2_count <= 0 || block <= 0) {
    dga_set_error("dga_fbz_rotate_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  RotLayout L;
  for (int i = 0; i < 4; ++i) L.st[i] = orb_strides[i];
  L.t1 = f1_stride;
  L.t2 = f2_stride;
  L.F1 = f1_count;
  L.F2 = f2_count;
  L.block = block;
  const int n4 = n_orb * n_orb * n_orb * n_orb;
  int fc = (int)((96 * 1024) / ((size_t)n4 * 2 * sizeof(double2)));
  if (fc > 64) fc = 64;
  if (fc < 1) fc = 1;
  const long long nf = (long long)f1_count * f2_count;
  const long long chunks = (nf + fc - 1) / fc;
  if (chunks > 0x7fffffffLL) {
    dga_set_error("dga_fbz_rotate_c128: too many frequency chunks");
    return DGA_ERR_ARG;
  }
  const size_t smem = (size_t)fc * n4 * 2 * sizeof(double2);
  cudaFuncSetAttribute(fbz_rotate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  fbz_rotate_kernel<<<dim3((unsigned)chunks, nk), BZ_THREADS, smem, stream>>>(
      (const double2*)src, irrk_inv, (const double2*)us, sigmas, conjs, n_orb, L, fc, (double2*)dst);
  return launch_status("dga_fbz_rotate_c128");
}

// Bytes of the partial-sum buffer of dga_sigma_c128.
size_t dga_sigma_scratch_bytes(int n_orb, int niv, int nk, int n_chunks) {
  return (size_t)n_chunks * niv * n_orb * n_orb * nk * sizeof(double2) * 2;
}

}  // extern "C"

// The real-space contraction of the Sigma computation: partial sums per bosonic chunk, then their sum times
// -1/(2 beta Nk) into sig[nu >= 0][(i,j)][R] (planes contiguous in R).
static int sigma_contract(const void* kern, const void* g_r, int n_orb, int niv, int niw, int n_q, Grid3 g,
                          const int* irrk_inv, const void* tw_inv, double beta, int n_chunks, double2* part,
                          double2* sig, cudaStream_t stream) {
  const int n2 = n_orb * n_orb;
  const size_t smem = (2 * (size_t)g.nk + g.nx + g.ny + g.nz) * sizeof(double2) + sizeof(int) * (size_t)g.nk;
  const long long work = (long long)niv * n2 * n_chunks;
  auto partial = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kernel<<<grid_cap(work), BZ_THREADS, smem, stream>>>((const double2*)kern, (const double2*)g_r, n_orb, niv, niw,
                                                         n_q, g, irrk_inv, (const double2*)tw_inv, n_chunks, part);
  };
  static_assert(16 * BZ_THREADS >= BZ_MAX_NK, "the largest accumulator set covers the largest grid");
  if (g.nk <= 4 * BZ_THREADS) partial(sigma_partial_kernel<4>);
  else if (g.nk <= 8 * BZ_THREADS) partial(sigma_partial_kernel<8>);
  else partial(sigma_partial_kernel<16>);
  if (launch_status("dga_sigma_c128")) return DGA_ERR_LAUNCH;
  const long long n_out = (long long)niv * n2 * g.nk;
  const double factor = -0.5 / beta / (double)g.nk;
  sigma_reduce_kernel<<<grid_cap((n_out + 255) / 256), 256, 0, stream>>>(part, n_chunks, n_out, factor, sig);
  return launch_status("dga_sigma_c128");
}

extern "C" {

// Real-space Sigma for nu >= 0, the result of calculate_sigma_from_kernel_fft_cpu/_gpu/_auto
// (dgamore/nonlocal_sde.py:544-652) before the caller's ifft and to_full_niv_range: out [niv][n2][Nk] (planes
// contiguous in R, R in row-major grid order).  Arguments and scratch as dga_sigma_c128.
int dga_sigma_rspace_c128(const void* kern, const void* g_r, int n_orb, int niv, int niw, int n_q, int nx, int ny,
                          int nz, const int* irrk_inv, const void* tw_inv, double beta, int n_chunks, void* out,
                          void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (check_grid(nx, ny, nz, "dga_sigma_rspace_c128")) return DGA_ERR_ARG;
  if (!kern || !g_r || !irrk_inv || !tw_inv || !out || !scratch || n_orb <= 0 || niv <= 0 || niw < 0 ||
      n_chunks <= 0) {
    dga_set_error("dga_sigma_rspace_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  Grid3 g{nx, ny, nz, nx * ny * nz};
  const size_t need = dga_sigma_scratch_bytes(n_orb, niv, g.nk, n_chunks);
  if (scratch_bytes < need) {
    dga_set_error("dga_sigma_rspace_c128: scratch too small (%zu < %zu)", scratch_bytes, need);
    return DGA_ERR_SCRATCH;
  }
  return sigma_contract(kern, g_r, n_orb, niv, niw, n_q, g, irrk_inv, tw_inv, beta, n_chunks, (double2*)scratch,
                        (double2*)out, stream)
             ? DGA_ERR_LAUNCH
             : DGA_OK;
}

// Sigma(k, nu) from the irreducible kernel (nonlocal_sde.py:544-594 and 876-879).
//   kern:   [Q][niw+1][2 niv][n2][n2] (row (a,i), column (d,j));  irrk_inv: [Nk]
//   g_r:    [niv + 2 niw][n][n][Nk] forward transforms of G(k) for nu indices [-niw, niv + niw)
//   tw_inv: e^{+2 pi i m / n} twiddles;  out: [Nk][n][n][2 niv] (upstream SelfEnergy layout)
//   scratch: dga_sigma_scratch_bytes(n_orb, niv, Nk, n_chunks) bytes
int dga_sigma_c128(const void* kern, const void* g_r, int n_orb, int niv, int niw, int n_q, int nx, int ny, int nz,
                   const int* irrk_inv, const void* tw_inv, double beta, int n_chunks, void* out, void* scratch,
                   size_t scratch_bytes, cudaStream_t stream) {
  if (check_grid(nx, ny, nz, "dga_sigma_c128")) return DGA_ERR_ARG;
  if (!kern || !g_r || !irrk_inv || !tw_inv || !out || !scratch || n_orb <= 0 || niv <= 0 || niw < 0 ||
      n_chunks <= 0) {
    dga_set_error("dga_sigma_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  Grid3 g{nx, ny, nz, nx * ny * nz};
  const int n2 = n_orb * n_orb;
  const size_t need = dga_sigma_scratch_bytes(n_orb, niv, g.nk, n_chunks);
  if (scratch_bytes < need) {
    dga_set_error("dga_sigma_c128: scratch too small (%zu < %zu)", scratch_bytes, need);
    return DGA_ERR_SCRATCH;
  }
  double2* part = (double2*)scratch;
  double2* sig = part + (size_t)n_chunks * niv * n2 * g.nk;
  if (sigma_contract(kern, g_r, n_orb, niv, niw, n_q, g, irrk_inv, tw_inv, beta, n_chunks, part, sig, stream))
    return DGA_ERR_LAUNCH;
  const long long n_out = (long long)niv * n2 * g.nk;
  // inverse transform over R (normalised 1/Nk), planes contiguous; result back into `part`
  size_t smem = (2 * (size_t)g.nk + nx + ny + nz) * sizeof(double2);
  cudaFuncSetAttribute(dft_planes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  PlaneAddr pa{(long long)g.nk, 0, 1, 1};
  dft_planes_kernel<<<grid_cap(niv * n2), BZ_THREADS, smem, stream>>>(sig, pa, part, pa, niv * n2, g,
                                                                      (const double2*)tw_inv, 1.0 / (double)g.nk,
                                                                      nullptr);
  if (launch_status("dga_sigma_c128")) return DGA_ERR_LAUNCH;
  sigma_full_nu_kernel<<<grid_cap((n_out + 255) / 256), 256, 0, stream>>>(part, n_orb, niv, g.nk, (double2*)out);
  return launch_status("dga_sigma_c128");
}

}  // extern "C"
