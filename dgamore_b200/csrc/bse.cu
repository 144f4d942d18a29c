// Batched ladder Bethe-Salpeter solve for every (channel, q, w) work item.
//
// For one item the compound-index matrix (row (o1,o2,nu), column (o4,o3,nu'), N = n^2 * 2 niv) is
//
//     A = (blockdiag_nu chi0^-1(q,w,nu) + Gamma_r(w) / beta^2) - (U_r + V_r^q) / beta^2
//
// (dgamore/nonlocal_sde.py:85-96 assembled through FourPoint.add, four_point.py:332-430), and the result is
//
//     X[(o1,o2,nu), (o4,o3)] = sum_nu' (A^-1)[(o1,o2,nu), (o4,o3,nu')] / beta
//
// (four_point.py:620-642; equivalently the solve against the n^2 selector right-hand sides of
// four_point.py:644-684).  Each CTA owns one item at a time (persistent loop over a device work list):
//
//   1. form A column-major in the CTA's scratch slot (Gamma_r is pre-permuted to the same column-major
//      compound layout once per request, so this is a coalesced stream plus a block-diagonal add);
//   2. blocked right-looking LU with partial pivoting (panel width NB): the panel is factored column by
//      column with the LAPACK pivot measure |re|+|im| and first-index ties (izamax), the panel's row
//      interchanges are applied to the other columns, the U12 row block is solved against L11 from shared
//      memory, and the trailing matrix is updated by a 64x64-tiled complex GEMM from shared memory;
//   3. the permuted selector right-hand side is solved by blocked forward and back substitution and
//      written out divided by beta.
//
// The same LU core serves the FP64 drop-in (R = double) and the mixed form (R = float for the
// factorisation, FP64 residuals and refinement; see bse_mixed below).
#include "bse_core.cuh"

#include <stdio.h>

namespace dga {

#ifndef DGA_MIXED_MIN_BLOCKS
#define DGA_MIXED_MIN_BLOCKS 3  // resident CTAs per SM the mixed-precision kernels are compiled for
#endif
constexpr int BSE_THREADS = 128;
constexpr int BSE_NB = 32;  // panel width (also the row-block of the triangular solves)
constexpr int BSE_TM = 32;  // trailing-update row tile
constexpr int BSE_TN = 64;  // trailing-update column strip
constexpr int BSE_MAX_N = 2048;
constexpr int MAX_RHS = 16;  // n2 <= 16 (up to 4 orbitals)

// ----------------------------------------------------------------------------------------------
// Block-wide arg-max of the pivot measure: larger value wins, ties go to the smaller row index.
// ----------------------------------------------------------------------------------------------
template <typename R>
__device__ int block_argmax(R v, int idx, R* s_val, int* s_idx) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    R ov = __shfl_down_sync(0xffffffffu, v, off);
    int oi = __shfl_down_sync(0xffffffffu, idx, off);
    argmax_merge(v, idx, ov, oi);
  }
  if (lane == 0) {
    s_val[warp] = v;
    s_idx[warp] = idx;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    v = lane < nw ? s_val[lane] : R(-1);
    idx = lane < nw ? s_idx[lane] : 0x7fffffff;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      R ov = __shfl_down_sync(0xffffffffu, v, off);
      int oi = __shfl_down_sync(0xffffffffu, idx, off);
      argmax_merge(v, idx, ov, oi);
    }
    if (lane == 0) {
      s_val[0] = v;
      s_idx[0] = idx;
    }
  }
  __syncthreads();
  int r = s_idx[0];
  __syncthreads();
  return r;
}

// ----------------------------------------------------------------------------------------------
// Shared-memory layout of one CTA: the GEMM tiles and the panel/triangular-solve buffers are never live at
// the same time, so they share storage.
// ----------------------------------------------------------------------------------------------
template <typename C>
struct BseSmem {
  union {
    struct {
      C Ls[BSE_NB][BSE_TM];      // L21 row tile (k, row)
      C Us[BSE_TN][BSE_NB + 1];  // U12 column strip (col, k), padded
    } g;
    struct {
      C L11[BSE_NB][BSE_NB + 1];
      C L11i[BSE_NB][BSE_NB + 1];  // inverse of the unit lower triangle of L11
      C A12[BSE_NB][BSE_NB + 1];   // A12 chunk of the U12 solve (col, k); solved block of the RHS solves
    } t;
  } u;
  C row[BSE_NB];
  double red_val[32];
  int red_idx[32];
  int flag;
};

// X = L^-1 for the unit lower triangular nb x nb block in L11 (column c of X by thread c):
// X[r][c] = -sum_{k=c}^{r-1} L[r][k] X[k][c] for r > c, X[c][c] = 1.
template <typename C>
__device__ void unit_lower_inverse(BseSmem<C>& sm, int nb) {
  using R = decltype(C::x);
  const int c = threadIdx.x;
  if (c < nb) {
    for (int r = 0; r < c; ++r) sm.u.t.L11i[r][c] = cmake<C>(R(0), R(0));
    sm.u.t.L11i[c][c] = cmake<C>(R(1), R(0));
    for (int r = c + 1; r < nb; ++r) {
      C acc = cmake<C>(R(0), R(0));
      for (int k = c; k < r; ++k) cfms(acc, sm.u.t.L11[r][k], sm.u.t.L11i[k][c]);
      sm.u.t.L11i[r][c] = acc;
    }
  }
}

// ----------------------------------------------------------------------------------------------
// LU with partial pivoting of the N x N column-major matrix A (leading dimension ld) in place.
// piv[j] receives the row exchanged with row j.  Returns true if an exact zero pivot was met.
// ----------------------------------------------------------------------------------------------
template <typename C>
__device__ bool lu_factor(C* __restrict__ A, int N, int ld, int* __restrict__ piv, BseSmem<C>& sm) {
  using R = decltype(C::x);
  const int tid = threadIdx.x, T = blockDim.x;
  bool singular = false;

  for (int k0 = 0; k0 < N; k0 += BSE_NB) {
    const int nb = min(BSE_NB, N - k0);
    // ---- panel factorisation (columns k0 .. k0+nb-1) ----
    // pivot candidates of the first panel column; later columns get theirs from the previous update
    R best = R(-1);
    int bidx = 0x7fffffff;
    for (int i = k0 + tid; i < N; i += T) {
      R v = cabs1(A[(size_t)k0 * ld + i]);
      if (v > best) {
        best = v;
        bidx = i;
      }
    }
    for (int jj = 0; jj < nb; ++jj) {
      const int j = k0 + jj;
      int p;
      {
        double dv = (double)best;  // reduce in double precision storage (R may be float)
        p = block_argmax<double>(dv, bidx, sm.red_val, sm.red_idx);
      }
      if (p >= N) p = j;  // cannot happen for j < N; keeps the index in range regardless
      if (tid == 0) piv[j] = p;
      if (p != j) {
        for (int c = tid; c < nb; c += T) {
          C* col = A + (size_t)(k0 + c) * ld;
          C t = col[j];
          col[j] = col[p];
          col[p] = t;
        }
      }
      __syncthreads();
      const C d = A[(size_t)j * ld + j];
      const bool zero = (d.x == R(0) && d.y == R(0));
      if (zero) singular = true;
      const C rinv = zero ? cmake<C>(R(0), R(0)) : crecip(d);
      const int ncols = nb - jj - 1;
      for (int c = tid; c < ncols; c += T) sm.row[c] = A[(size_t)(j + 1 + c) * ld + j];
      __syncthreads();
      best = R(-1);
      bidx = 0x7fffffff;
      for (int i = j + 1 + tid; i < N; i += T) {
        C l = A[(size_t)j * ld + i];
        if (!zero) l = cmul(l, rinv);
        A[(size_t)j * ld + i] = l;
        // batched loads: 8 independent loads in flight before the updates
        for (int c0 = 0; c0 < ncols; c0 += 8) {
          C v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (c0 + u < ncols) v[u] = A[(size_t)(j + 1 + c0 + u) * ld + i];
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (c0 + u < ncols) {
              cfms(v[u], l, sm.row[c0 + u]);
              A[(size_t)(j + 1 + c0 + u) * ld + i] = v[u];
            }
          if (c0 == 0) {  // column j+1 just updated: its pivot candidate (look-ahead)
            const R a = cabs1(v[0]);
            if (a > best) {
              best = a;
              bidx = i;
            }
          }
        }
      }
      __syncthreads();
    }
    // ---- L11 and its inverse in shared memory ----
    for (int e = tid; e < nb * nb; e += T) {
      const int r = e % nb, c = e / nb;
      sm.u.t.L11[r][c] = A[(size_t)(k0 + c) * ld + k0 + r];
    }
    __syncthreads();
    unit_lower_inverse(sm, nb);
    // ---- row interchanges on the columns outside the panel ----
    // When every pivot row lies below the panel and no two coincide, the interchanges are independent pairs
    // and are applied in parallel over (interchange, column); otherwise they run in order per column.
    const int k1 = k0 + nb;
    if (tid < 32) {
      bool ok = true;
      if (tid < nb) {
        const int p = piv[k0 + tid];
        if (p != k0 + tid) {
          if (p < k1) ok = false;
          for (int o = 0; o < nb; ++o)
            if (o != tid && piv[k0 + o] == p) ok = false;
        }
      }
      const unsigned all_ok = __all_sync(0xffffffffu, ok);
      if (tid == 0) sm.flag = all_ok ? 1 : 0;
    }
    __syncthreads();
    if (sm.flag) {
      const int ncol = N - nb;
      for (int e = tid; e < nb * ncol; e += T) {
        const int jj = e / ncol;
        int c = e - jj * ncol;
        c = c < k0 ? c : c + nb;  // skip the panel columns
        const int p = piv[k0 + jj];
        if (p != k0 + jj) {
          C* col = A + (size_t)c * ld;
          C t = col[k0 + jj];
          col[k0 + jj] = col[p];
          col[p] = t;
        }
      }
    } else {
      for (int c = tid; c < N; c += T) {
        if (c >= k0 && c < k1) continue;
        C* col = A + (size_t)c * ld;
        for (int jj = 0; jj < nb; ++jj) {
          const int p = piv[k0 + jj];
          if (p != k0 + jj) {
            C t = col[k0 + jj];
            col[k0 + jj] = col[p];
            col[p] = t;
          }
        }
      }
    }
    __syncthreads();
    // ---- U12 = L11^-1 A12, in chunks of 32 columns staged through shared memory ----
    for (int c0 = k1; c0 < N; c0 += BSE_NB) {
      const int cw = min(BSE_NB, N - c0);
      for (int e = tid; e < nb * cw; e += T) {
        const int c = e / nb, k = e % nb;
        sm.u.t.A12[c][k] = A[(size_t)(c0 + c) * ld + k0 + k];
      }
      __syncthreads();
      for (int e = tid; e < cw * (BSE_NB / 8); e += T) {
        const int c = e % cw, g = e / cw;  // 8-row groups
        C out[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) out[u] = cmake<C>(R(0), R(0));
        for (int k = 0; k < nb; ++k) {
          const C a = sm.u.t.A12[c][k];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int r = g * 8 + u;
            if (r < nb && k <= r) cfma(out[u], sm.u.t.L11i[r][k], a);
          }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int r = g * 8 + u;
          if (r < nb) A[(size_t)(c0 + c) * ld + k0 + r] = out[u];
        }
      }
      __syncthreads();
    }
    // ---- trailing update A22 -= L21 U12: column strips of BSE_TN, row tiles of BSE_TM ----
    const int nt = N - k1;
    if (nt > 0) {
      const int ty = tid % (BSE_TM / 4), tx = tid / (BSE_TM / 4);  // 8 x 16 thread grid, 4x4 outputs each
      for (int cs = k1; cs < N; cs += BSE_TN) {
        for (int e = tid; e < nb * BSE_TN; e += T) {
          const int c = e / nb, k = e % nb;
          sm.u.g.Us[c][k] = (cs + c < N) ? A[(size_t)(cs + c) * ld + k0 + k] : cmake<C>(R(0), R(0));
        }
        for (int rt = k1; rt < N; rt += BSE_TM) {
          C acc[4][4];
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int c = cs + tx + 16 * b;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
              const int r = rt + ty + 8 * a;
              acc[a][b] = (c < N && r < N) ? A[(size_t)c * ld + r] : cmake<C>(R(0), R(0));
            }
          }
          for (int e = tid; e < nb * BSE_TM; e += T) {
            const int k = e / BSE_TM, r = e % BSE_TM;
            sm.u.g.Ls[k][r] = (rt + r < N) ? A[(size_t)(k0 + k) * ld + rt + r] : cmake<C>(R(0), R(0));
          }
          __syncthreads();
#pragma unroll 4
          for (int k = 0; k < nb; ++k) {
            C lv[4], uv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) lv[a] = sm.u.g.Ls[k][ty + 8 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) uv[b] = sm.u.g.Us[tx + 16 * b][k];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
              for (int b = 0; b < 4; ++b) cfms(acc[a][b], lv[a], uv[b]);
          }
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int c = cs + tx + 16 * b;
            if (c < N) {
              C* col = A + (size_t)c * ld;
#pragma unroll
              for (int a = 0; a < 4; ++a) {
                const int r = rt + ty + 8 * a;
                if (r < N) col[r] = acc[a][b];
              }
            }
          }
          __syncthreads();
        }
      }
    }
  }
  return singular;
}

// ----------------------------------------------------------------------------------------------
// Solve (L U) Y = B in place for the n_rhs columns of Y (column-major, leading dimension N), with the LU
// factors of lu_factor (unit lower L below the diagonal, U on and above).  Blocked by 32 rows: the diagonal
// block is solved by one warp per right-hand side (lane = row, the solved value broadcast by shuffle), the
// rest of the rows are updated from the block copy in shared memory.
// ----------------------------------------------------------------------------------------------
template <typename C, typename CY, int NR>
__device__ void lu_solve_inplace(const C* __restrict__ A, int N, int ld, CY* __restrict__ Y, BseSmem<C>& sm) {
  constexpr int n_rhs = NR;
  // factor elements a thread has in flight in the row updates: eight where each one feeds several right-hand
  // sides; with one to three the registers go to the factorisation around the solve instead
  constexpr int SOLVE_LOADS = NR >= 4 ? 8 : 1;
  using R = decltype(C::x);
  using RY = decltype(CY::x);
  const int tid = threadIdx.x, T = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = T >> 5;
  CY* yb = reinterpret_cast<CY*>(&sm.u.t.A12[0][0]);  // [n_rhs][32] solved block
  // forward: L z = b
  for (int b0 = 0; b0 < N; b0 += BSE_NB) {
    const int bn = min(BSE_NB, N - b0);
    for (int e = tid; e < bn * bn; e += T) {
      const int r = e % bn, c = e / bn;
      sm.u.t.L11[r][c] = A[(size_t)(b0 + c) * ld + b0 + r];
    }
    __syncthreads();
    for (int s = warp; s < n_rhs; s += nwarps) {
      CY y = lane < bn ? Y[(size_t)s * N + b0 + lane] : cmake<CY>(RY(0), RY(0));
      for (int r = 0; r < bn; ++r) {
        CY yr;
        yr.x = __shfl_sync(0xffffffffu, y.x, r);
        yr.y = __shfl_sync(0xffffffffu, y.y, r);
        if (lane > r && lane < bn) {
          const C l = sm.u.t.L11[lane][r];
          cfms(y, cmake<CY>((RY)l.x, (RY)l.y), yr);
        }
      }
      if (lane < bn) {
        Y[(size_t)s * N + b0 + lane] = y;
        yb[s * 32 + lane] = y;
      }
    }
    __syncthreads();
    // rows below the block: one thread per row, every right-hand side at once (each L element read once,
    // SOLVE_LOADS of them in flight; the products are summed in ascending r)
    for (int i = b0 + bn + tid; i < N; i += T) {
      CY acc[NR];
#pragma unroll
      for (int s = 0; s < NR; ++s) acc[s] = Y[(size_t)s * N + i];
      if constexpr (SOLVE_LOADS == 1) {
        for (int r = 0; r < bn; ++r) {
          const C l = A[(size_t)(b0 + r) * ld + i];
          const CY lw = cmake<CY>((RY)l.x, (RY)l.y);
#pragma unroll
          for (int s = 0; s < NR; ++s) cfms(acc[s], lw, yb[s * 32 + r]);
        }
      } else {
        for (int r0 = 0; r0 < bn; r0 += SOLVE_LOADS) {
          C l[SOLVE_LOADS];
#pragma unroll
          for (int u = 0; u < SOLVE_LOADS; ++u)
            l[u] = (r0 + u < bn) ? A[(size_t)(b0 + r0 + u) * ld + i] : cmake<C>(R(0), R(0));
#pragma unroll
          for (int u = 0; u < SOLVE_LOADS; ++u) {
            if (r0 + u >= bn) break;
            const CY lw = cmake<CY>((RY)l[u].x, (RY)l[u].y);
#pragma unroll
            for (int s = 0; s < NR; ++s) cfms(acc[s], lw, yb[s * 32 + r0 + u]);
          }
        }
      }
#pragma unroll
      for (int s = 0; s < NR; ++s) Y[(size_t)s * N + i] = acc[s];
    }
    __syncthreads();
  }
  // backward: U y = z
  const int nblk = (N + BSE_NB - 1) / BSE_NB;
  for (int blk = nblk - 1; blk >= 0; --blk) {
    const int b0 = blk * BSE_NB;
    const int bn = min(BSE_NB, N - b0);
    for (int e = tid; e < bn * bn; e += T) {
      const int r = e % bn, c = e / bn;
      sm.u.t.L11[r][c] = A[(size_t)(b0 + c) * ld + b0 + r];
    }
    __syncthreads();
    for (int s = warp; s < n_rhs; s += nwarps) {
      CY y = lane < bn ? Y[(size_t)s * N + b0 + lane] : cmake<CY>(RY(0), RY(0));
      for (int r = bn - 1; r >= 0; --r) {
        if (lane == r) {
          const C u = sm.u.t.L11[r][r];
          y = cdiv(y, cmake<CY>((RY)u.x, (RY)u.y));
        }
        CY yr;
        yr.x = __shfl_sync(0xffffffffu, y.x, r);
        yr.y = __shfl_sync(0xffffffffu, y.y, r);
        if (lane < r) {
          const C u = sm.u.t.L11[lane][r];
          cfms(y, cmake<CY>((RY)u.x, (RY)u.y), yr);
        }
      }
      if (lane < bn) {
        Y[(size_t)s * N + b0 + lane] = y;
        yb[s * 32 + lane] = y;
      }
    }
    __syncthreads();
    // rows above the block: one thread per row, every right-hand side at once (each U element read once,
    // SOLVE_LOADS of them in flight, summed in ascending r)
    for (int i = tid; i < b0; i += T) {
      CY acc[NR];
#pragma unroll
      for (int s = 0; s < NR; ++s) acc[s] = Y[(size_t)s * N + i];
      if constexpr (SOLVE_LOADS == 1) {
        for (int r = 0; r < bn; ++r) {
          const C u = A[(size_t)(b0 + r) * ld + i];
          const CY uw = cmake<CY>((RY)u.x, (RY)u.y);
#pragma unroll
          for (int s = 0; s < NR; ++s) cfms(acc[s], uw, yb[s * 32 + r]);
        }
      } else {
        for (int r0 = 0; r0 < bn; r0 += SOLVE_LOADS) {
          C uu[SOLVE_LOADS];
#pragma unroll
          for (int u = 0; u < SOLVE_LOADS; ++u)
            uu[u] = (r0 + u < bn) ? A[(size_t)(b0 + r0 + u) * ld + i] : cmake<C>(R(0), R(0));
#pragma unroll
          for (int u = 0; u < SOLVE_LOADS; ++u) {
            if (r0 + u >= bn) break;
            const CY uw = cmake<CY>((RY)uu[u].x, (RY)uu[u].y);
#pragma unroll
            for (int s = 0; s < NR; ++s) cfms(acc[s], uw, yb[s * 32 + r0 + u]);
          }
        }
      }
#pragma unroll
      for (int s = 0; s < NR; ++s) Y[(size_t)s * N + i] = acc[s];
    }
    __syncthreads();
  }
}

// Y = P * S where S is the n2-column selector (S[j, s] = 1 if the orbital pair of row j is s) and P the
// row permutation recorded in piv.  perm is shared scratch of N ints.
template <typename CY>
__device__ void permuted_selector(CY* __restrict__ Y, int N, int nv, int n_rhs, const int* __restrict__ piv,
                                  int* __restrict__ perm) {
  using RY = decltype(CY::x);
  const int tid = threadIdx.x, T = blockDim.x;
  for (int i = tid; i < N; i += T) perm[i] = i;
  __syncthreads();
  if (tid == 0) {
    for (int i = 0; i < N; ++i) {
      const int p = piv[i];
      if (p != i) {
        int t = perm[i];
        perm[i] = perm[p];
        perm[p] = t;
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < N * n_rhs; e += T) {
    const int i = e % N, s = e / N;
    Y[(size_t)s * N + i] = cmake<CY>((perm[i] / nv == s) ? RY(1) : RY(0), RY(0));
  }
  __syncthreads();
}

// ----------------------------------------------------------------------------------------------
// One work item in FP64: form A, LU, selector solve, X = Y / beta into out (rows (p,nu), n2 columns).
// Returns the item's status bits.  All threads of the CTA call it.
// ----------------------------------------------------------------------------------------------
template <typename Source, int NR>
__device__ int solve_item_fp64(const Source& src, const WorkItem& wi, int N, int nv, double beta,
                               double2* __restrict__ o, double2* __restrict__ A, double2* __restrict__ Y,
                               BseSmem<double2>& sm, int* piv, int* perm) {
  const int tid = threadIdx.x, T = blockDim.x;
  // form A column by column; the (pair, nu) split of a thread's rows advances by T = q_T nv + r_T per step
  {
    const int pr0 = tid / nv, vr0 = tid - pr0 * nv;
    const int qT = T / nv, rT = T - qT * nv;
    int pc = 0, vc = 0;
    for (int j = 0; j < N; ++j) {
      double2* col = A + (size_t)j * N;
      int pr = pr0, vr = vr0;
      for (int i = tid; i < N; i += T) {
        col[i] = src.element(wi.ch, wi.q, wi.w, N, i, j, pr, vr, pc, vc);
        pr += qT;
        vr += rT;
        if (vr >= nv) {
          vr -= nv;
          ++pr;
        }
      }
      if (++vc == nv) {
        vc = 0;
        ++pc;
      }
    }
  }
  __syncthreads();
  const bool singular = lu_factor<double2>(A, N, N, piv, sm);
  permuted_selector<double2>(Y, N, nv, NR, piv, perm);
  lu_solve_inplace<double2, double2, NR>(A, N, N, Y, sm);
  // X[i][s] = Y[i][s] / beta, finiteness check
  if (tid == 0) sm.flag = 0;
  __syncthreads();
  bool bad = false;
  for (int e = tid; e < N * NR; e += T) {
    const int i = e / NR, s = e % NR;
    double2 y = Y[(size_t)s * N + i];
    y.x = y.x / beta;
    y.y = y.y / beta;
    if (!cfinite(y)) bad = true;
    o[e] = y;
  }
  if (bad) atomicOr(&sm.flag, DGA_ITEM_NONFINITE);
  __syncthreads();
  const int st = (singular ? DGA_ITEM_SINGULAR : 0) | sm.flag;
  __syncthreads();
  return st;
}

// FP64 kernel: one CTA per work item, persistent over the list.
template <typename Source, int NR>
__global__ void __launch_bounds__(BSE_THREADS, 3)
    bse_solve_sum_fp64_kernel(Source src, const WorkItem* __restrict__ work, int n_items, int N, int n2,
                              int nv, int W, int Q, double beta, double2* __restrict__ out,
                              int* __restrict__ status, double2* __restrict__ scratch, size_t slot_elems,
                              int redo_only) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BseSmem<double2>& sm = *reinterpret_cast<BseSmem<double2>*>(smem_raw);
  int* piv = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<double2>));
  int* perm = piv + N;
  double2* A = scratch + (size_t)blockIdx.x * slot_elems;
  double2* Y = A + (size_t)N * N;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    // re-solve mode: only the items whose status says the mixed solve did not converge or was not finite
    if (redo_only && (status[item] & DGA_ITEM_REDO) == 0) continue;
    const WorkItem wi = work[item];
    double2* o = out + (((size_t)wi.ch * Q + wi.q) * W + wi.w) * (size_t)N * n2;
    const int st = solve_item_fp64<Source, NR>(src, wi, N, nv, beta, o, A, Y, sm, piv, perm);
    if (threadIdx.x == 0 && status) status[item] = st;
  }
}

// ----------------------------------------------------------------------------------------------
// Mixed form: FP32 LU (same core, float2 storage, FP32 trailing updates) and FP64 iterative refinement.
//
//   Y0 = (LU)^-1 P S with the FP32 factors and FP64 accumulation of the triangular solves;
//   repeat: r = S - A Y with A formed on the fly in FP64 from Gamma_r, chi0^-1 and U_r + V_r^q,
//           d = (LU)^-1 P r,  Y += d,  until the correction, or the error left after it as estimated from the
//           observed contraction, is below tol max|Y| (refine_converged), or max_iter corrections.
//
// FP64 is used only for A in the residual, the residual accumulation and Y.  Items that do not reach the
// tolerance are flagged DGA_ITEM_NOCONVERGE (the host re-solves them with the FP64 kernel).
// ----------------------------------------------------------------------------------------------

// byte offset of the [n2][n2] column-sum block after the pivot and permutation arrays, 16-byte aligned
__host__ __device__ inline size_t mixed_colsum_offset(int N) {
  return (sizeof(BseSmem<float2>) + 2 * sizeof(int) * (size_t)N + 15) & ~(size_t)15;
}

// One work item in the mixed form (FP32 LU, FP64 refinement).  Returns the status bits; *iters = corrections.
template <int NR>
__device__ int solve_item_mixed(const StructuredSource& src, const WorkItem& wi, int N, int nv, double beta,
                                int max_iter, double tol, double2* __restrict__ o, float2* __restrict__ A,
                                double2* __restrict__ Y, double2* __restrict__ Rb, BseSmem<float2>& sm, int* piv,
                                int* perm, double2* colsum, int* iters) {
  const int tid = threadIdx.x, T = blockDim.x;
  {
    const int pr0 = tid / nv, vr0 = tid - pr0 * nv;
    const int qT = T / nv, rT = T - qT * nv;
    int pc = 0, vc = 0;
    for (int j = 0; j < N; ++j) {
      float2* col = A + (size_t)j * N;
      int pr = pr0, vr = vr0;
      for (int i = tid; i < N; i += T) {
        const double2 a = src.element(wi.ch, wi.q, wi.w, N, i, j, pr, vr, pc, vc);
        col[i] = make_float2((float)a.x, (float)a.y);
        pr += qT;
        vr += rT;
        if (vr >= nv) {
          vr -= nv;
          ++pr;
        }
      }
      if (++vc == nv) {
        vc = 0;
        ++pc;
      }
    }
  }
  __syncthreads();
  const bool singular = lu_factor<float2>(A, N, N, piv, sm);
  permuted_selector<double2>(Y, N, nv, NR, piv, perm);
  lu_solve_inplace<float2, double2, NR>(A, N, N, Y, sm);
  double prev = 0.0;
  for (int e = tid; e < N * NR; e += T) prev = fmax(prev, fmax(fabs(Y[e].x), fabs(Y[e].y)));
  prev = block_max(prev, sm.red_val);
  int it = 0;
  bool converged = false;
  for (; it < max_iter; ++it) {
    structured_residual_permuted<NR>(src, wi.ch, wi.q, wi.w, N, nv, Y, Rb, perm, colsum,
                                     reinterpret_cast<double2*>(&sm.u));
    lu_solve_inplace<float2, double2, NR>(A, N, N, Rb, sm);
    double dmax = 0.0, ymax = 0.0;
    for (int e = tid; e < N * NR; e += T) {
      const double2 d = Rb[e];
      const double2 y = cadd(Y[e], d);
      Y[e] = y;
      dmax = fmax(dmax, fmax(fabs(d.x), fabs(d.y)));
      ymax = fmax(ymax, fmax(fabs(y.x), fabs(y.y)));
    }
    dmax = block_max(dmax, sm.red_val);
    ymax = block_max(ymax, sm.red_val);
    if (isnan(dmax) || refine_converged(dmax, ymax, prev, tol)) {  // NaN is flagged below
      converged = !isnan(dmax);
      ++it;
      break;
    }
    prev = dmax;
  }
  if (tid == 0) sm.flag = 0;
  __syncthreads();
  bool bad = false;
  for (int e = tid; e < N * NR; e += T) {
    const int i = e / NR, sidx = e % NR;
    double2 y = Y[(size_t)sidx * N + i];
    y.x = y.x / beta;
    y.y = y.y / beta;
    if (!cfinite(y)) bad = true;
    o[e] = y;
  }
  if (bad) atomicOr(&sm.flag, DGA_ITEM_NONFINITE);
  __syncthreads();
  const int st = (singular ? DGA_ITEM_SINGULAR : 0) | sm.flag | (converged ? 0 : DGA_ITEM_NOCONVERGE);
  *iters = it;
  __syncthreads();
  return st;
}

template <int NR>
__global__ void __launch_bounds__(BSE_THREADS, DGA_MIXED_MIN_BLOCKS)
    bse_solve_sum_mixed_kernel(StructuredSource src, const WorkItem* __restrict__ work, int n_items, int N, int n2,
                               int nv, int W, int Q, double beta, int max_iter, double tol,
                               double2* __restrict__ out, int* __restrict__ status, int* __restrict__ iters,
                               unsigned char* __restrict__ scratch, size_t slot_bytes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BseSmem<float2>& sm = *reinterpret_cast<BseSmem<float2>*>(smem_raw);
  int* piv = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<float2>));
  int* perm = piv + N;
  double2* colsum = reinterpret_cast<double2*>(smem_raw + mixed_colsum_offset(N));
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  float2* A = reinterpret_cast<float2*>(slot);
  double2* Y = reinterpret_cast<double2*>(slot + (((size_t)N * N * sizeof(float2) + 255) & ~(size_t)255));
  double2* Rb = Y + (size_t)N * n2;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const WorkItem wi = work[item];
    double2* o = out + (((size_t)wi.ch * Q + wi.q) * W + wi.w) * (size_t)N * n2;
    int it = 0;
    const int st = solve_item_mixed<NR>(src, wi, N, nv, beta, max_iter, tol, o, A, Y, Rb, sm, piv, perm, colsum,
                                        &it);
    if (threadIdx.x == 0) {
      if (status) status[item] = st;
      if (iters) iters[item] = it;
    }
  }
}

// ----------------------------------------------------------------------------------------------
// Heterogeneous batch: one persistent launch over the work items of several problems (requests) whose
// sizes differ (niv, niw, number of q points, beta, inputs) but which share the number of orbitals, so that
// the RHS count NR = n_orb^2 is a compile-time constant of the launch.  Each item names its problem, whose
// descriptor carries the sizes, the resident inputs and the output.  The per-item body is the same as the
// single-problem kernels.
// ----------------------------------------------------------------------------------------------
// One item of a batch: the problem's descriptor gives its sizes, inputs and output; returns the status bits.
template <bool MIXED, int NR>
__device__ __forceinline__ int multi_item(const dga_bse_problem& d, const MultiItem& mi, int n_max, int max_iter,
                                          double tol, unsigned char* slot, unsigned char* smem_raw, int* it_out) {
  {
    struct {
      StructuredSource src;
      int N, n2, nv, W, Q;
      double beta;
      double2* out;
    } pb;
    pb.n2 = d.n_orb * d.n_orb;
    pb.nv = 2 * d.niv;
    pb.N = pb.n2 * pb.nv;
    pb.W = d.niw_half;
    pb.Q = d.n_q;
    pb.beta = d.beta;
    pb.out = (double2*)d.out;
    pb.src.gamma_cm = (const double2*)d.gamma_cm;
    pb.src.chi0_inv = (const double2*)d.chi0_inv;
    pb.src.uv = (const double2*)d.uv;
    pb.src.n2 = pb.n2;
    pb.src.nv = pb.nv;
    pb.src.W = pb.W;
    pb.src.Q = pb.Q;
    pb.src.inv_beta2 = d.inv_beta2;
    const WorkItem wi{mi.ch, mi.q, mi.w};
    double2* o = pb.out + (((size_t)wi.ch * pb.Q + wi.q) * pb.W + wi.w) * (size_t)pb.N * pb.n2;
    int st = 0, it = 0;
    if (MIXED) {
      BseSmem<float2>& sm = *reinterpret_cast<BseSmem<float2>*>(smem_raw);
      int* piv = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<float2>));
      int* perm = piv + n_max;
      double2* colsum = reinterpret_cast<double2*>(smem_raw + mixed_colsum_offset(n_max));
      float2* A = reinterpret_cast<float2*>(slot);
      double2* Y = reinterpret_cast<double2*>(slot + (((size_t)pb.N * pb.N * sizeof(float2) + 255) & ~(size_t)255));
      double2* Rb = Y + (size_t)pb.N * pb.n2;
      st = solve_item_mixed<NR>(pb.src, wi, pb.N, pb.nv, pb.beta, max_iter, tol, o, A, Y, Rb, sm, piv, perm, colsum, &it);
    } else {
      BseSmem<double2>& sm = *reinterpret_cast<BseSmem<double2>*>(smem_raw);
      int* piv = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<double2>));
      int* perm = piv + n_max;
      double2* A = reinterpret_cast<double2*>(slot);
      double2* Y = A + (size_t)pb.N * pb.N;
      st = solve_item_fp64<StructuredSource, NR>(pb.src, wi, pb.N, pb.nv, pb.beta, o, A, Y, sm, piv, perm);
    }
    *it_out = it;
    return st;
  }
}

template <bool MIXED, int NR>
__global__ void __launch_bounds__(BSE_THREADS, MIXED ? DGA_MIXED_MIN_BLOCKS : 3)
    bse_multi_kernel(const dga_bse_problem* __restrict__ probs, const MultiItem* __restrict__ work, int n_items,
                     int n_max, int max_iter, double tol, int* __restrict__ status, int* __restrict__ iters,
                     unsigned char* __restrict__ scratch, size_t slot_bytes, int redo_only) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (redo_only && (status[item] & DGA_ITEM_REDO) == 0) continue;
    const MultiItem mi = work[item];
    const dga_bse_problem d = probs[mi.prob];
    int it = 0;
    const int st = multi_item<MIXED, NR>(d, mi, n_max, max_iter, tol, slot, smem_raw, &it);
    __syncthreads();  // every thread has read status[item] before it is rewritten
    if (threadIdx.x == 0) {
      status[item] = st;
      if (iters && !redo_only) iters[item] = it;
    }
  }
}

// Batch whose problems differ in orbital count (the 2-orbital bilayer next to a 1-orbital lattice, say): the same
// per-item body, with the right-hand-side count chosen per item from its problem's n_orb.  Shared memory and the
// scratch slot are sized for the largest problem of the launch.
template <bool MIXED>
__global__ void __launch_bounds__(BSE_THREADS, MIXED ? DGA_MIXED_MIN_BLOCKS : 3)
    bse_multi_any_kernel(const dga_bse_problem* __restrict__ probs, const MultiItem* __restrict__ work, int n_items,
                         int n_max, int max_iter, double tol, int* __restrict__ status, int* __restrict__ iters,
                         unsigned char* __restrict__ scratch, size_t slot_bytes, int redo_only) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (redo_only && (status[item] & DGA_ITEM_REDO) == 0) continue;
    const MultiItem mi = work[item];
    const dga_bse_problem d = probs[mi.prob];
    int it = 0, st = 0;
    switch (d.n_orb) {
      case 1: st = multi_item<MIXED, 1>(d, mi, n_max, max_iter, tol, slot, smem_raw, &it); break;
      case 2: st = multi_item<MIXED, 4>(d, mi, n_max, max_iter, tol, slot, smem_raw, &it); break;
      case 3: st = multi_item<MIXED, 9>(d, mi, n_max, max_iter, tol, slot, smem_raw, &it); break;
      default: st = multi_item<MIXED, 16>(d, mi, n_max, max_iter, tol, slot, smem_raw, &it); break;
    }
    __syncthreads();  // every thread has read status[item] before it is rewritten
    if (threadIdx.x == 0) {
      status[item] = st;
      if (iters && !redo_only) iters[item] = it;
    }
  }
}

// ----------------------------------------------------------------------------------------------
// Eliashberg full vertex in the pp frequency box (one CTA per (channel, q, w) item):
//   F[(p,nu),(s,nu')] = beta^2 (delta_{nu nu'} c0(nu)[p][s] - sum_{m,m'} c0(nu)[p][m] chi*[(m,nu),(m',nu')] c0(nu')[m'][s])
//                       + (Z G3(nu) G3(nu'))[p][s],   Z = U_r - U_r chi_r U_r,  c0 = chi0^-1,  G3 = gamma_r
// for nu, nu' in the box [niv - P, niv + P) (eliashberg_solver.py:175-204).  chi* = A^-1 is never formed: the
// LU factors of A are solved against the unit vectors of KB box frequencies at a time (NR = KB n2 columns).
//   g3: [2][Q][W][nv][n2][n2]; chi_phys: [2][Q][W][n2][n2]; out: [2][Q][Wpp][Mb][Mb]
//   slot: A (N x N) | Y (N x NR) | H (2P x n2 x n2) | Z (n2 x n2), complex128
// ----------------------------------------------------------------------------------------------
template <int NR>
__global__ void __launch_bounds__(BSE_THREADS, 3)
    eli_full_vertex_kernel(StructuredSource src, const WorkItem* __restrict__ work, int n_items, int N, int n2, int nv,
                           int W, int Q, int P, int Wpp, double beta, const double2* __restrict__ g3,
                           const double2* __restrict__ chi_phys, double2* __restrict__ out, int* __restrict__ status,
                           double2* __restrict__ scratch, size_t slot_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BseSmem<double2>& sm = *reinterpret_cast<BseSmem<double2>*>(smem_raw);
  int* piv = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<double2>));
  int* perm = piv + N;
  double2* A = scratch + (size_t)blockIdx.x * slot_elems;
  double2* Y = A + (size_t)N * N;
  const int nvp = 2 * P, Mb = n2 * nvp, KB = NR / n2, off = nv / 2 - P;
  double2* H = Y + (size_t)N * NR;
  double2* Z = H + (size_t)nvp * n2 * n2;
  const int tid = threadIdx.x, T = blockDim.x;
  const double beta2 = beta * beta;

  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const WorkItem wi = work[item];
    {
      const int pr0 = tid / nv, vr0 = tid - pr0 * nv;
      const int qT = T / nv, rT = T - qT * nv;
      int pc = 0, vc = 0;
      for (int j = 0; j < N; ++j) {
        double2* col = A + (size_t)j * N;
        int pr = pr0, vr = vr0;
        for (int i = tid; i < N; i += T) {
          col[i] = src.element(wi.ch, wi.q, wi.w, N, i, j, pr, vr, pc, vc);
          pr += qT;
          vr += rT;
          if (vr >= nv) {
            vr -= nv;
            ++pr;
          }
        }
        if (++vc == nv) {
          vc = 0;
          ++pc;
        }
      }
    }
    __syncthreads();
    const bool singular = lu_factor<double2>(A, N, N, piv, sm);
    // row permutation of the factorisation
    for (int i = tid; i < N; i += T) perm[i] = i;
    __syncthreads();
    if (tid == 0) {
      for (int i = 0; i < N; ++i) {
        const int p = piv[i];
        if (p != i) {
          const int t = perm[i];
          perm[i] = perm[p];
          perm[p] = t;
        }
      }
    }
    // Z = U_r - U_r chi_r U_r, then H(nu) = Z G3(nu) for the box frequencies
    const double2* uvq = src.uv + ((size_t)wi.ch * Q + wi.q) * n2 * n2;
    const double2* cp = chi_phys + (((size_t)wi.ch * Q + wi.q) * W + wi.w) * n2 * n2;
    for (int e = tid; e < n2 * n2; e += T) {
      const int p = e / n2, s = e - p * n2;
      double2 acc = uvq[e];
      for (int t = 0; t < n2; ++t) {
        double2 cu = make_double2(0.0, 0.0);
        for (int u = 0; u < n2; ++u) cfma(cu, cp[t * n2 + u], uvq[u * n2 + s]);
        cfms(acc, uvq[p * n2 + t], cu);
      }
      Z[e] = acc;
    }
    __syncthreads();
    const double2* g3q = g3 + ((((size_t)wi.ch * Q + wi.q) * W + wi.w) * nv) * n2 * n2;
    for (int e = tid; e < nvp * n2 * n2; e += T) {
      const int vb = e / (n2 * n2), ps = e - vb * n2 * n2, p = ps / n2, s = ps - p * n2;
      const double2* g = g3q + (size_t)(off + vb) * n2 * n2;
      double2 acc = make_double2(0.0, 0.0);
      for (int t = 0; t < n2; ++t) cfma(acc, Z[p * n2 + t], g[t * n2 + s]);
      H[e] = acc;
    }
    __syncthreads();
    double2* o = out + (((size_t)wi.ch * Q + wi.q) * Wpp + wi.w) * (size_t)Mb * Mb;
    for (int v0 = 0; v0 < nvp; v0 += KB) {
      // unit vectors of the box columns (m', nu') for nu' in [v0, v0 + KB), permuted by the pivots
      for (int e = tid; e < N * NR; e += T) {
        const int i = e % N, sidx = e / N;
        const int kk = sidx / n2, mp = sidx - kk * n2;
        const int vb = v0 + kk;
        const int j = mp * nv + off + vb;
        Y[(size_t)sidx * N + i] = make_double2((vb < nvp && perm[i] == j) ? 1.0 : 0.0, 0.0);
      }
      __syncthreads();
      lu_solve_inplace<double2, double2, NR>(A, N, N, Y, sm);
      // F columns (s, nu') for the KB box frequencies of this chunk, rows (p, nu) of the box
      for (int e = tid; e < Mb * KB * n2; e += T) {
        const int sidx = e % n2;
        const int kk = (e / n2) % KB;
        const int row = e / (n2 * KB);
        const int vbp = v0 + kk;
        if (vbp >= nvp) continue;
        const int p = row / nvp, vb = row - p * nvp;
        const int vr = off + vb, vc = off + vbp;
        const double2* c0r = src.chi0_inv + (((size_t)wi.q * W + wi.w) * nv + vr) * n2 * n2;
        const double2* c0c = src.chi0_inv + (((size_t)wi.q * W + wi.w) * nv + vc) * n2 * n2;
        // t = sum_{m,m'} c0r[p][m] chi*[(m,vr),(m',vc)] c0c[m'][s]
        double2 t = make_double2(0.0, 0.0);
        for (int m = 0; m < n2; ++m) {
          double2 inner = make_double2(0.0, 0.0);
          for (int mp = 0; mp < n2; ++mp) cfma(inner, Y[(size_t)(kk * n2 + mp) * N + m * nv + vr], c0c[mp * n2 + sidx]);
          cfma(t, c0r[p * n2 + m], inner);
        }
        double2 f1 = make_double2(-t.x, -t.y);
        if (vb == vbp) f1 = cadd(f1, c0r[p * n2 + sidx]);
        f1 = cscale(f1, beta2);
        // (Z G3(nu)) G3(nu')
        const double2* hrow = H + (size_t)vb * n2 * n2 + p * n2;
        const double2* gcol = g3q + (size_t)vc * n2 * n2;
        double2 f2 = make_double2(0.0, 0.0);
        for (int u = 0; u < n2; ++u) cfma(f2, hrow[u], gcol[u * n2 + sidx]);
        o[(size_t)row * Mb + sidx * nvp + vbp] = cadd(f1, f2);
      }
      __syncthreads();
    }
    if (tid == 0 && status) status[item] = singular ? DGA_ITEM_SINGULAR : 0;
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------------------------
// Dense batched LU and solves with many right-hand sides (the local Schwinger-Dyson equation's full inverses,
// numpy.linalg.inv behind LocalFourPoint.invert, local_four_point.py:298-310).  The factorisation is lu_factor
// (LAPACK's pivot order) with one CTA per matrix; the solves spread over (matrix, block of DENSE_RHS right-hand
// sides) CTAs, each streaming the factors once for its block.
// ----------------------------------------------------------------------------------------------
constexpr int DENSE_RHS = 16;

__global__ void __launch_bounds__(BSE_THREADS, 3)
    dense_lu_kernel(double2* __restrict__ a, int N, int n_mat, long long mat_stride, int* __restrict__ piv_out,
                    int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BseSmem<double2>& sm = *reinterpret_cast<BseSmem<double2>*>(smem_raw);
  int* piv = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<double2>));
  for (int m = blockIdx.x; m < n_mat; m += gridDim.x) {
    const bool singular = lu_factor<double2>(a + (size_t)m * mat_stride, N, N, piv, sm);
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) piv_out[(size_t)m * N + i] = piv[i];
    if (threadIdx.x == 0) status[m] = singular ? DGA_ITEM_SINGULAR : DGA_ITEM_OK;
    __syncthreads();
  }
}

// out_m[:, k] = A_m^-1 B_m[:, k] for k < n_rhs, column-major with leading dimension N, in blocks of DENSE_RHS
// columns (columns n_rhs .. of the last block are solved for zero right-hand sides).  B_m(r, k) =
// b[m b_sm + r b_sr + k b_sk], or the identity when b is null.  A non-finite solution element sets
// DGA_ITEM_NONFINITE in status[m].
__global__ void __launch_bounds__(BSE_THREADS, 3)
    dense_solve_kernel(const double2* __restrict__ lu, const int* __restrict__ piv, int N, int n_mat,
                       long long lu_stride, const double2* __restrict__ b, long long b_sm, long long b_sr,
                       long long b_sk, int n_rhs, double2* __restrict__ out, long long out_stride,
                       int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BseSmem<double2>& sm = *reinterpret_cast<BseSmem<double2>*>(smem_raw);
  int* perm = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<double2>));
  const int tid = threadIdx.x, T = blockDim.x;
  const int n_blk = (n_rhs + DENSE_RHS - 1) / DENSE_RHS;
  for (int t = blockIdx.x; t < n_mat * n_blk; t += gridDim.x) {
    const int m = t / n_blk, k0 = (t - m * n_blk) * DENSE_RHS;
    const int* pv = piv + (size_t)m * N;
    for (int i = tid; i < N; i += T) perm[i] = i;
    __syncthreads();
    if (tid == 0) {
      for (int i = 0; i < N; ++i) {
        const int p = pv[i];
        if (p != i) {
          const int s = perm[i];
          perm[i] = perm[p];
          perm[p] = s;
        }
      }
    }
    __syncthreads();
    double2* Y = out + (size_t)m * out_stride + (size_t)k0 * N;
    for (int e = tid; e < N * DENSE_RHS; e += T) {
      const int i = e % N, k = e / N, col = k0 + k;
      double2 v = make_double2(0.0, 0.0);
      if (col < n_rhs) {
        const int r = perm[i];
        if (b)
          v = b[m * b_sm + r * b_sr + col * b_sk];
        else if (r == col)
          v.x = 1.0;
      }
      Y[(size_t)k * N + i] = v;
    }
    __syncthreads();
    lu_solve_inplace<double2, double2, DENSE_RHS>(lu + (size_t)m * lu_stride, N, N, Y, sm);
    int bad = 0;
    for (int e = tid; e < N * DENSE_RHS; e += T) {
      const double2 v = Y[e];
      bad |= !(isfinite(v.x) && isfinite(v.y));
    }
    if (__syncthreads_or(bad) && tid == 0) atomicOr(status + m, DGA_ITEM_NONFINITE);
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------------------------
// Eliashberg full vertex fused into the FP64 BSE (eliashberg_solver.py:175-204): an item with w < Wpp keeps its LU
// factors after the selector solve and solves the unit vectors of the pp box with them, writing
//   f1[(p,nu),(s,nu')] = beta^2 (delta_{nu nu'} c0(nu)[p][s] - sum_{m,m'} c0(nu)[p][m] chi*[(m,nu),(m',nu')] c0(nu')[m'][s])
// for nu, nu' in [niv - P, niv + P).  The ladder term (Z G3(nu) G3(nu'), which needs the lambda-corrected chi_r and
// the three-leg vertex of the whole pass) is added afterwards by eli_ladder_term_kernel; f1 + term is the sum
// eli_full_vertex_kernel forms, in the same order, from the same factors.
// ----------------------------------------------------------------------------------------------
template <int NRB>
__device__ void eli_box_epilogue(const StructuredSource& src, const WorkItem& wi, int N, int n2, int nv, int W, int P,
                                 double beta2, const double2* __restrict__ A, double2* __restrict__ Y,
                                 const int* __restrict__ perm, double2* __restrict__ o, BseSmem<double2>& sm) {
  const int tid = threadIdx.x, T = blockDim.x;
  const int nvp = 2 * P, Mb = n2 * nvp, KB = NRB / n2, off = nv / 2 - P;
  for (int v0 = 0; v0 < nvp; v0 += KB) {
    for (int e = tid; e < N * NRB; e += T) {
      const int i = e % N, sidx = e / N;
      const int kk = sidx / n2, mp = sidx - kk * n2;
      const int vb = v0 + kk;
      const int j = mp * nv + off + vb;
      Y[(size_t)sidx * N + i] = make_double2((kk < KB && vb < nvp && perm[i] == j) ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    lu_solve_inplace<double2, double2, NRB>(A, N, N, Y, sm);
    for (int e = tid; e < Mb * KB * n2; e += T) {
      const int sidx = e % n2;
      const int kk = (e / n2) % KB;
      const int row = e / (n2 * KB);
      const int vbp = v0 + kk;
      if (vbp >= nvp) continue;
      const int p = row / nvp, vb = row - p * nvp;
      const int vr = off + vb, vc = off + vbp;
      const double2* c0r = src.chi0_inv + (((size_t)wi.q * W + wi.w) * nv + vr) * n2 * n2;
      const double2* c0c = src.chi0_inv + (((size_t)wi.q * W + wi.w) * nv + vc) * n2 * n2;
      double2 t = make_double2(0.0, 0.0);
      for (int m = 0; m < n2; ++m) {
        double2 inner = make_double2(0.0, 0.0);
        for (int mp = 0; mp < n2; ++mp) cfma(inner, Y[(size_t)(kk * n2 + mp) * N + m * nv + vr], c0c[mp * n2 + sidx]);
        cfma(t, c0r[p * n2 + m], inner);
      }
      double2 f1 = make_double2(-t.x, -t.y);
      if (vb == vbp) f1 = cadd(f1, c0r[p * n2 + sidx]);
      o[(size_t)row * Mb + sidx * nvp + vbp] = cscale(f1, beta2);
    }
    __syncthreads();
  }
}

// FP64 BSE (as bse_solve_sum_fp64_kernel) with the pp-box epilogue for items w < Wpp; NRB = box columns per solve
// (KB = NRB / n2 box frequencies).  out_pp: [2][Q][Wpp][Mb][Mb].
template <int NR, int NRB>
__global__ void __launch_bounds__(BSE_THREADS, 3)
    bse_fp64_eli_kernel(StructuredSource src, const WorkItem* __restrict__ work, int n_items, int N, int n2, int nv,
                        int W, int Q, double beta, double2* __restrict__ out, int P, int Wpp,
                        double2* __restrict__ out_pp, int* __restrict__ status, double2* __restrict__ scratch,
                        size_t slot_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BseSmem<double2>& sm = *reinterpret_cast<BseSmem<double2>*>(smem_raw);
  int* piv = reinterpret_cast<int*>(smem_raw + sizeof(BseSmem<double2>));
  int* perm = piv + N;
  double2* A = scratch + (size_t)blockIdx.x * slot_elems;
  double2* Y = A + (size_t)N * N;
  const int Mb = n2 * 2 * P;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const WorkItem wi = work[item];
    double2* o = out + (((size_t)wi.ch * Q + wi.q) * W + wi.w) * (size_t)N * n2;
    const int st = solve_item_fp64<StructuredSource, NR>(src, wi, N, nv, beta, o, A, Y, sm, piv, perm);
    if (wi.w < Wpp) {
      double2* opp = out_pp + (((size_t)wi.ch * Q + wi.q) * Wpp + wi.w) * (size_t)Mb * Mb;
      eli_box_epilogue<NRB>(src, wi, N, n2, nv, W, P, beta * beta, A, Y, perm, opp, sm);
    }
    if (threadIdx.x == 0 && status) status[item] = st;
  }
}

// f[ch][q][w] += (Z G3(nu)) G3(nu') over the pp box, Z = U_r - U_r chi_r U_r (the second term of the full vertex,
// eliashberg_solver.py:175-204); one CTA per (ch, q, w < Wpp), Z and H(nu) = Z G3(nu) in shared memory.
//   g3: [2][Q][W][nv][n2][n2]; chi_phys: [2][Q][W][n2][n2]; uv: [2][Q][n2][n2]; f: [2][Q][Wpp][Mb][Mb]
__global__ void eli_ladder_term_kernel(const double2* __restrict__ uv, const double2* __restrict__ g3,
                                       const double2* __restrict__ chi_phys, int n2, int nv, int W, int Q, int P,
                                       int Wpp, double2* __restrict__ f) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* Z = reinterpret_cast<double2*>(smem_raw);
  double2* H = Z + n2 * n2;
  const int wq = blockIdx.x, w = wq % Wpp, q = (wq / Wpp) % Q, ch = wq / (Wpp * Q);
  const int tid = threadIdx.x, T = blockDim.x;
  const int nvp = 2 * P, Mb = n2 * nvp, off = nv / 2 - P;
  const double2* uvq = uv + ((size_t)ch * Q + q) * n2 * n2;
  const double2* cp = chi_phys + (((size_t)ch * Q + q) * W + w) * n2 * n2;
  for (int e = tid; e < n2 * n2; e += T) {
    const int p = e / n2, s = e - p * n2;
    double2 acc = uvq[e];
    for (int t = 0; t < n2; ++t) {
      double2 cu = make_double2(0.0, 0.0);
      for (int u = 0; u < n2; ++u) cfma(cu, cp[t * n2 + u], uvq[u * n2 + s]);
      cfms(acc, uvq[p * n2 + t], cu);
    }
    Z[e] = acc;
  }
  __syncthreads();
  const double2* g3q = g3 + ((((size_t)ch * Q + q) * W + w) * nv) * n2 * n2;
  for (int e = tid; e < nvp * n2 * n2; e += T) {
    const int vb = e / (n2 * n2), ps = e - vb * n2 * n2, p = ps / n2, s = ps - p * n2;
    const double2* g = g3q + (size_t)(off + vb) * n2 * n2;
    double2 acc = make_double2(0.0, 0.0);
    for (int t = 0; t < n2; ++t) cfma(acc, Z[p * n2 + t], g[t * n2 + s]);
    H[e] = acc;
  }
  __syncthreads();
  double2* o = f + (size_t)wq * Mb * Mb;
  for (int e = tid; e < Mb * Mb; e += T) {
    const int row = e / Mb, colx = e - row * Mb;  // column index sidx * nvp + vbp
    const int sidx = colx / nvp, vbp = colx - sidx * nvp;
    const int p = row / nvp, vb = row - p * nvp;
    const double2* hrow = H + (size_t)vb * n2 * n2 + p * n2;
    const double2* gcol = g3q + (size_t)(off + vbp) * n2 * n2;
    double2 f2 = make_double2(0.0, 0.0);
    for (int u = 0; u < n2; ++u) cfma(f2, hrow[u], gcol[u * n2 + sidx]);
    o[e] = cadd(o[e], f2);
  }
}

}  // namespace dga

using namespace dga;

static size_t bse_smem_bytes(int N) { return sizeof(BseSmem<double2>) + 2 * sizeof(int) * (size_t)N; }

template <typename K>
static int grid_for(K kernel, int n_items, size_t smem) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, BSE_THREADS, smem);
  if (per_sm < 1) per_sm = 1;
  int g = sms * per_sm;
  return n_items < g ? n_items : g;
}

static int bse_grid(int n_items, size_t smem) {
  return grid_for(bse_solve_sum_fp64_kernel<StructuredSource, 9>, n_items, smem);
}

static bool supported_rhs(int n2) { return n2 == 1 || n2 == 4 || n2 == 9 || n2 == 16; }

// Launches the FP64 kernel instantiated for n2 right-hand sides (1, 4, 9 or 16 orbital pairs).
template <typename Source>
static void launch_fp64(int n2, int grid, size_t smem, cudaStream_t stream, const Source& src, const WorkItem* work,
                        int n_items, int N, int nv, int W, int Q, double beta, double2* out, int* status,
                        double2* scratch, size_t slot, int redo) {
#define DGA_FP64_CASE(NRV)                                                                                        \
  case NRV:                                                                                                       \
    cudaFuncSetAttribute(bse_solve_sum_fp64_kernel<Source, NRV>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                         (int)smem);                                                                              \
    bse_solve_sum_fp64_kernel<Source, NRV><<<grid, BSE_THREADS, smem, stream>>>(                                  \
        src, work, n_items, N, NRV, nv, W, Q, beta, out, status, scratch, slot, redo);                            \
    break;
  switch (n2) {
    DGA_FP64_CASE(1)
    DGA_FP64_CASE(4)
    DGA_FP64_CASE(9)
    DGA_FP64_CASE(16)
    default:
      break;
  }
#undef DGA_FP64_CASE
}

extern "C" {

// Scratch bytes the FP64 BSE entry points need for a launch over n_items items of compound size N with
// n2 right-hand sides: one N x N matrix plus N x n2 solution per resident CTA.
size_t dga_bse_scratch_bytes(int N, int n2, int n_items) {
  if (N <= 0 || n2 <= 0 || n_items <= 0) return 0;
  const size_t smem = bse_smem_bytes(N);
  const int grid = bse_grid(n_items, smem);
  return (size_t)grid * ((size_t)N * N + (size_t)N * n2) * sizeof(double2);
}

int dga_bse_solve_sum_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                           const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work,
                           int n_items, void* out, int* status, void* scratch, size_t scratch_bytes,
                           cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || n_ch <= 0 || n_items <= 0 || N > BSE_MAX_N) {
    dga_set_error("dga_bse_solve_sum_c128: invalid sizes (n_orb=%d niv=%d niw_half=%d n_q=%d n_ch=%d items=%d)",
                  n_orb, niv, niw_half, n_q, n_ch, n_items);
    return DGA_ERR_ARG;
  }
  if (!gamma_cm || !chi0_inv || !uv || !work || !out || !scratch) {
    dga_set_error("dga_bse_solve_sum_c128: null pointer argument");
    return DGA_ERR_ARG;
  }
  const size_t smem = bse_smem_bytes(N);
  const int grid = bse_grid(n_items, smem);
  const size_t slot = (size_t)N * N + (size_t)N * n2;
  if (scratch_bytes < (size_t)grid * slot * sizeof(double2)) {
    dga_set_error("dga_bse_solve_sum_c128: scratch too small (%zu < %zu)", scratch_bytes,
                  (size_t)grid * slot * sizeof(double2));
    return DGA_ERR_SCRATCH;
  }
  StructuredSource src;
  src.gamma_cm = (const double2*)gamma_cm;
  src.chi0_inv = (const double2*)chi0_inv;
  src.uv = (const double2*)uv;
  src.n2 = n2;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  src.inv_beta2 = inv_beta2;
  launch_fp64(n2, grid, smem, stream, src, (const WorkItem*)work, n_items, N, nv, niw_half, n_q, beta,
              (double2*)out, status, (double2*)scratch, slot, 0);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_bse_solve_sum_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

// FP64 re-solve of the items a mixed launch flagged (status & (NOCONVERGE | NONFINITE)); other items are left
// untouched.  Same arguments as dga_bse_solve_sum_c128 with `status` read and rewritten for the re-solved items;
// the scratch may be sized for a smaller grid (grid_limit CTAs).
int dga_bse_resolve_fp64_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                              const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work, int n_items,
                              void* out, int* status, int grid_limit, void* scratch, size_t scratch_bytes,
                              cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || n_ch <= 0 || n_items <= 0 || N > BSE_MAX_N ||
      grid_limit <= 0 || !gamma_cm || !chi0_inv || !uv || !work || !out || !status || !scratch) {
    dga_set_error("dga_bse_resolve_fp64_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const size_t smem = bse_smem_bytes(N);
  int grid = bse_grid(n_items, smem);
  if (grid > grid_limit) grid = grid_limit;
  const size_t slot = (size_t)N * N + (size_t)N * n2;
  if (scratch_bytes < (size_t)grid * slot * sizeof(double2)) {
    dga_set_error("dga_bse_resolve_fp64_c128: scratch too small");
    return DGA_ERR_SCRATCH;
  }
  StructuredSource src;
  src.gamma_cm = (const double2*)gamma_cm;
  src.chi0_inv = (const double2*)chi0_inv;
  src.uv = (const double2*)uv;
  src.n2 = n2;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  src.inv_beta2 = inv_beta2;
  launch_fp64(n2, grid, smem, stream, src, (const WorkItem*)work, n_items, N, nv, niw_half, n_q, beta,
              (double2*)out, status, (double2*)scratch, slot, 1);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_bse_resolve_fp64_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

// Generic FourPoint.invert_and_sum_over_last_vn (four_point.py:620-642): the matrix is given explicitly in
// the FourPoint layout [q][o1][o2][o3][o4][w][nu][nu'] (half w range); out is [q][w][N][n2].
int dga_invert_sum_dense_c128(int n_orb, int niv, int niw_half, int n_q, double beta, const void* mat,
                              const int* work, int n_items, void* out, int* status, void* scratch,
                              size_t scratch_bytes, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || n_items <= 0 || N > BSE_MAX_N || !mat || !work ||
      !out || !scratch) {
    dga_set_error("dga_invert_sum_dense_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const size_t smem = bse_smem_bytes(N);
  const int grid = bse_grid(n_items, smem);
  const size_t slot = (size_t)N * N + (size_t)N * n2;
  if (scratch_bytes < (size_t)grid * slot * sizeof(double2)) {
    dga_set_error("dga_invert_sum_dense_c128: scratch too small");
    return DGA_ERR_SCRATCH;
  }
  DenseSource src;
  src.mat = (const double2*)mat;
  src.nb = n_orb;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  launch_fp64(n2, grid, smem, stream, src, (const WorkItem*)work, n_items, N, nv, niw_half, n_q, beta,
              (double2*)out, status, (double2*)scratch, slot, 0);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_invert_sum_dense_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"


static size_t mixed_smem_bytes(int N, int n2) { return mixed_colsum_offset(N) + (size_t)n2 * n2 * sizeof(double2); }

static size_t mixed_slot_bytes(int N, int n2) {
  return (((size_t)N * N * sizeof(float2) + 255) & ~(size_t)255) + 2 * (size_t)N * n2 * sizeof(double2);
}
// Default launch of the mixed form: the block-form kernel (4) wherever its solve phase fits shared memory (it is
// the fastest at every size measured, N = 40 to 720); else, from N = 320, the shared-memory-panel kernel with
// tensor-core trailing tiles (3) or FP32 tiles (1), else the 128-thread kernel (2).
static int default_mixed_kernel(int N, int n2) {
  if (dga_block_supported(N, n2)) return 4;
  if (N < 320) return 2;
  if (dga_panel_supported(N, n2, true)) return 3;
  if (dga_panel_supported(N, n2)) return 1;
  return 2;
}

// Grid and scratch slot of the mixed kernels that own their launch geometry (1, 3: panel; 4: block form).
static int owned_grid(int kernel, int n2, int N, int n_items) {
  return kernel == 4 ? dga_block_grid(n2, n_items) : dga_panel_grid(n2, N, n_items, kernel == 3);
}
static size_t owned_slot(int kernel, int N, int n2) {
  return kernel == 4 ? dga_block_slot_bytes(N, n2) : dga_panel_slot_bytes(N, n2);
}

static int mixed_grid(int n_items, size_t smem) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  (void)sms;
  return grid_for(bse_solve_sum_mixed_kernel<9>, n_items, smem);
}

extern "C" {

// Scratch bytes of dga_bse_solve_sum_mixed_c128: one N x N complex64 matrix and two N x n2 complex128
// blocks per resident CTA.
size_t dga_bse_mixed_scratch_bytes(int N, int n2, int n_items) {
  if (N <= 0 || n2 <= 0 || n_items <= 0) return 0;
  const int kernel = default_mixed_kernel(N, n2);
  if (kernel != 2) return (size_t)owned_grid(kernel, n2, N, n_items) * owned_slot(kernel, N, n2);
  const size_t smem = mixed_smem_bytes(N, n2);
  return (size_t)mixed_grid(n_items, smem) * mixed_slot_bytes(N, n2);
}

// Mixed-precision ladder BSE: same inputs and output as dga_bse_solve_sum_c128; FP32 LU, FP64 residuals and
// refinement to tol (refine_converged) within max_iter corrections.  iters: per-item corrections (optional).
int dga_bse_solve_sum_mixed_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                                 const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work,
                                 int n_items, int max_iter, double tol, void* out, int* status, int* iters,
                                 void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || n_ch <= 0 || n_items <= 0 || N > BSE_MAX_N ||
      n2 > MAX_RHS || max_iter < 0) {
    dga_set_error("dga_bse_solve_sum_mixed_c128: invalid sizes (n_orb=%d niv=%d niw_half=%d n_q=%d n_ch=%d items=%d)",
                  n_orb, niv, niw_half, n_q, n_ch, n_items);
    return DGA_ERR_ARG;
  }
  if (!gamma_cm || !chi0_inv || !uv || !work || !out || !scratch) {
    dga_set_error("dga_bse_solve_sum_mixed_c128: null pointer argument");
    return DGA_ERR_ARG;
  }
  const int kernel = default_mixed_kernel(N, n2);
  const bool panel = kernel != 2;
  const size_t smem = mixed_smem_bytes(N, n2);
  const int grid = panel ? owned_grid(kernel, n2, N, n_items) : mixed_grid(n_items, smem);
  const size_t slot = panel ? owned_slot(kernel, N, n2) : mixed_slot_bytes(N, n2);
  if (scratch_bytes < (size_t)grid * slot) {
    dga_set_error("dga_bse_solve_sum_mixed_c128: scratch too small (%zu < %zu)", scratch_bytes, (size_t)grid * slot);
    return DGA_ERR_SCRATCH;
  }
  StructuredSource src;
  src.gamma_cm = (const double2*)gamma_cm;
  src.chi0_inv = (const double2*)chi0_inv;
  src.uv = (const double2*)uv;
  src.n2 = n2;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  src.inv_beta2 = inv_beta2;
  if (panel) {
    // from N = 320: the block-form kernel (bse_block.cu, two 256-thread CTAs per SM), or where it does not fit the
    // shared-memory panel (bse_panel.cu, one 512-thread CTA per SM)
    cudaError_t err =
        kernel == 4 ? dga_block_launch(grid, src, (const WorkItem*)work, n_items, N, n2, nv, niw_half, n_q, beta,
                                       max_iter, tol, (double2*)out, status, iters, (unsigned char*)scratch, slot,
                                       stream)
                    : dga_panel_launch(grid, src, (const WorkItem*)work, n_items, N, n2, nv, niw_half, n_q, beta,
                                       max_iter, tol, (double2*)out, status, iters, (unsigned char*)scratch, slot,
                                       stream, kernel == 3);
    if (err != cudaSuccess) {
      dga_set_error("dga_bse_solve_sum_mixed_c128: launch failed: %s", cudaGetErrorString(err));
      return DGA_ERR_LAUNCH;
    }
    return DGA_OK;
  }
#define DGA_MIXED_CASE(NRV)                                                                                       \
  case NRV:                                                                                                       \
    cudaFuncSetAttribute(bse_solve_sum_mixed_kernel<NRV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    bse_solve_sum_mixed_kernel<NRV><<<grid, BSE_THREADS, smem, stream>>>(                                          \
        src, (const WorkItem*)work, n_items, N, NRV, nv, niw_half, n_q, beta, max_iter, tol, (double2*)out, status, \
        iters, (unsigned char*)scratch, slot);                                                                    \
    break;
  switch (n2) {
    DGA_MIXED_CASE(1)
    DGA_MIXED_CASE(4)
    DGA_MIXED_CASE(9)
    DGA_MIXED_CASE(16)
    default:
      break;
  }
#undef DGA_MIXED_CASE
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_bse_solve_sum_mixed_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"


// ------------------------------------------------------------------------------------------------
// Eliashberg full vertex (host side)
// ------------------------------------------------------------------------------------------------
static int eli_rhs(int n2) { return n2 == 9 ? 9 : 16; }

static size_t eli_slot_elems(int N, int n2, int P) {
  return (size_t)N * N + (size_t)N * eli_rhs(n2) + (size_t)2 * P * n2 * n2 + (size_t)n2 * n2;
}

extern "C" {

// Scratch bytes of dga_eli_full_vertex_c128 for n_items items.
size_t dga_eli_vertex_scratch_bytes(int n_orb, int niv, int niv_pp, int n_items) {
  const int n2 = n_orb * n_orb, N = n2 * 2 * niv;
  if (!supported_rhs(n2) || n_items <= 0) return 0;
  const size_t smem = bse_smem_bytes(N);
  const int grid = grid_for(eli_full_vertex_kernel<16>, n_items, smem);
  return (size_t)grid * eli_slot_elems(N, n2, niv_pp) * sizeof(double2);
}

// Full ladder vertex of both channels in the pp box (eliashberg_solver.py:175-204) for the work items
// (ch, q, w) with w < w_pp; inputs as dga_bse_solve_sum_c128 plus gamma_r (g3 [2][Q][W][nv][n2][n2]) and the
// physical susceptibility (chi_phys [2][Q][W][n2][n2]); out: [2][Q][w_pp][Mb][Mb], Mb = n2 * 2 niv_pp.
int dga_eli_full_vertex_c128(int n_orb, int niv, int niw_half, int n_q, int niv_pp, int w_pp, double beta,
                             double inv_beta2, const void* gamma_cm, const void* chi0_inv, const void* uv,
                             const void* g3, const void* chi_phys, const int* work, int n_items, void* out,
                             int* status, void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || niv_pp <= 0 || niv_pp > niv ||
      w_pp <= 0 || w_pp > niw_half || n_items <= 0 || N > BSE_MAX_N || !gamma_cm || !chi0_inv || !uv || !g3 ||
      !chi_phys || !work || !out || !scratch) {
    dga_set_error("dga_eli_full_vertex_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const size_t smem = bse_smem_bytes(N);
  const int NR = eli_rhs(n2);
  int grid = NR == 9 ? grid_for(eli_full_vertex_kernel<9>, n_items, smem)
                     : grid_for(eli_full_vertex_kernel<16>, n_items, smem);
  const size_t slot = eli_slot_elems(N, n2, niv_pp);
  if (scratch_bytes < (size_t)grid * slot * sizeof(double2)) {
    dga_set_error("dga_eli_full_vertex_c128: scratch too small");
    return DGA_ERR_SCRATCH;
  }
  StructuredSource src;
  src.gamma_cm = (const double2*)gamma_cm;
  src.chi0_inv = (const double2*)chi0_inv;
  src.uv = (const double2*)uv;
  src.n2 = n2;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  src.inv_beta2 = inv_beta2;
  if (NR == 9) {
    eli_full_vertex_kernel<9><<<grid, BSE_THREADS, smem, stream>>>(
        src, (const WorkItem*)work, n_items, N, n2, nv, niw_half, n_q, niv_pp, w_pp, beta, (const double2*)g3,
        (const double2*)chi_phys, (double2*)out, status, (double2*)scratch, slot);
  } else {
    eli_full_vertex_kernel<16><<<grid, BSE_THREADS, smem, stream>>>(
        src, (const WorkItem*)work, n_items, N, n2, nv, niw_half, n_q, niv_pp, w_pp, beta, (const double2*)g3,
        (const double2*)chi_phys, (double2*)out, status, (double2*)scratch, slot);
  }
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_eli_full_vertex_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"


// ------------------------------------------------------------------------------------------------
// Heterogeneous batch (host side)
// ------------------------------------------------------------------------------------------------
// Launch geometry of a batch.  In the mixed form every request must have the same default kernel as when it runs
// alone (default_mixed_kernel), so that a request's results are the same in a batch and alone; *kernel receives
// it (1, 3: shared-memory panel, 4: block form, 2: 128-thread kernel; always 2 in FP64).  Returns false for an
// invalid batch.  Problems may differ in orbital count (*n2_max receives the largest n_orb^2, *hetero whether they
// differ); such a batch runs kernels that choose the right-hand-side count per item: the 128-thread kernels, or
// the block-form kernel for orbital counts 1 to 3 (the 4-orbital block kernel is compiled alone).  The
// shared-memory-panel kernels take one orbital count per launch.
static bool batch_dims(const dga_bse_problem* probs, int n_prob, int mixed, int* n_max, size_t* slot, int* kernel,
                       int* n2_max = nullptr, bool* hetero = nullptr) {
  *n_max = 0;
  *slot = 0;
  *kernel = 2;
  if (n_prob <= 0) return false;
  int n2m = 0;
  bool het = false;
  for (int p = 0; p < n_prob; ++p) {
    const int n2 = probs[p].n_orb * probs[p].n_orb;
    const int N = n2 * 2 * probs[p].niv;
    if (probs[p].n_orb <= 0 || !supported_rhs(n2) || probs[p].niv <= 0 || N > BSE_MAX_N) return false;
    het |= probs[p].n_orb != probs[0].n_orb;
    if (mixed) {
      const int k = default_mixed_kernel(N, n2);
      if (p == 0) *kernel = k;
      if (k != *kernel) return false;
    }
    if (N > *n_max) *n_max = N;
    if (n2 > n2m) n2m = n2;
  }
  const bool panel = *kernel != 2;
  if (het && panel && (*kernel != 4 || n2m > 9)) return false;
  for (int p = 0; p < n_prob; ++p) {
    const int n2 = probs[p].n_orb * probs[p].n_orb;
    const int N = n2 * 2 * probs[p].niv;
    const size_t sl = panel ? owned_slot(*kernel, N, n2)
                      : mixed ? mixed_slot_bytes(N, n2)
                              : ((size_t)N * N + (size_t)N * n2) * sizeof(double2);
    if (sl > *slot) *slot = sl;
  }
  *slot = (*slot + 255) & ~(size_t)255;
  if (n2_max) *n2_max = n2m;
  if (hetero) *hetero = het;
  return true;
}

static size_t batch_smem(int n_max, int n2, int mixed) {
  return mixed ? mixed_smem_bytes(n_max, n2) : bse_smem_bytes(n_max);
}

static int batch_grid_hetero(int mixed, int n_items, size_t smem) {
  return mixed ? grid_for(bse_multi_any_kernel<true>, n_items, smem)
               : grid_for(bse_multi_any_kernel<false>, n_items, smem);
}

template <bool MIXED, int NR>
static int batch_grid(int n_items, size_t smem) {
  return grid_for(bse_multi_kernel<MIXED, NR>, n_items, smem);
}

static int batch_grid_any(int mixed, int n2, int n_items, size_t smem) {
#define DGA_BATCH_GRID(R) \
  if (n2 == R) return mixed ? batch_grid<true, R>(n_items, smem) : batch_grid<false, R>(n_items, smem);
  DGA_BATCH_GRID(1)
  DGA_BATCH_GRID(4)
  DGA_BATCH_GRID(9)
  DGA_BATCH_GRID(16)
#undef DGA_BATCH_GRID
  return 0;
}

extern "C" {

// Scratch bytes of dga_bse_solve_sum_batch_c128 (probs is a HOST array here); 0 for an invalid batch.
size_t dga_bse_batch_scratch_bytes(const dga_bse_problem* probs, int n_prob, int n_items, int mode) {
  int n_max = 0, kernel = 2, n2_max = 0;
  size_t slot = 0;
  bool hetero = false;
  const int mixed = mode == 1;
  if (!probs || n_items <= 0 || mode < 0 || mode > 2 ||
      !batch_dims(probs, n_prob, mixed, &n_max, &slot, &kernel, &n2_max, &hetero))
    return 0;
  const int n2 = probs[0].n_orb * probs[0].n_orb;
  const bool panel = kernel != 2;
  if (panel)
    return (size_t)(kernel == 4 ? dga_block_grid(hetero ? 0 : n2, n_items)
                                : dga_panel_batch_grid(n2, n_max, n_items, kernel == 3)) *
           slot;
  if (hetero) return (size_t)batch_grid_hetero(mixed, n_items, batch_smem(n_max, n2_max, mixed)) * slot;
  return (size_t)batch_grid_any(mixed, n2, n_items, batch_smem(n_max, n2, mixed)) * slot;
}

// One persistent launch over the (problem, ch, q, w) items of several problems of the same orbital count whose
// frequency boxes, q sets, beta and inputs differ.
//   probs_host: the descriptors (read on the host for the launch geometry); probs_dev: the same array in device
//   memory (read by the kernel); work: [n_items][4] ints (problem, channel, q, w) in device memory; mode: 0 =
//   FP64 LU, 1 = FP32 LU + FP64 refinement (max_iter, tol), 2 = FP64 re-solve of the items whose status holds
//   NOCONVERGE or NONFINITE; status / iters: [n_items] (iters may be null).  The grid is the smaller of the
//   resident CTAs, n_items and scratch_bytes / slot: a smaller scratch buffer caps the launch's HBM footprint.
int dga_bse_solve_sum_batch_c128(const dga_bse_problem* probs_host, const void* probs_dev, int n_prob, const int* work,
                                 int n_items, int mode, int max_iter, double tol, int* status, int* iters,
                                 void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  int n_max = 0, kernel = 2, n2_max = 0;
  size_t slot = 0;
  bool hetero = false;
  const int mixed = mode == 1;
  if (!probs_host || !probs_dev || !work || !scratch || !status || n_items <= 0 || max_iter < 0 || mode < 0 ||
      mode > 2 || !batch_dims(probs_host, n_prob, mixed, &n_max, &slot, &kernel, &n2_max, &hetero)) {
    dga_set_error("dga_bse_solve_sum_batch_c128: invalid arguments (n_orb in {1,2,3,4}; in the mixed form all "
                  "problems take the same default kernel, and problems of different n_orb take the block-form or "
                  "the 128-thread kernel with n_orb at most 3)");
    return DGA_ERR_ARG;
  }
  for (int p = 0; p < n_prob; ++p) {
    const dga_bse_problem& d = probs_host[p];
    if (!d.gamma_cm || !d.chi0_inv || !d.uv || !d.out || d.niw_half <= 0 || d.n_q <= 0) {
      dga_set_error("dga_bse_solve_sum_batch_c128: problem %d has a null pointer or empty size", p);
      return DGA_ERR_ARG;
    }
  }
  const int n2 = probs_host[0].n_orb * probs_host[0].n_orb;
  const size_t smem = batch_smem(n_max, hetero ? n2_max : n2, mixed);
  const bool panel = kernel != 2;
  int grid = panel    ? (kernel == 4 ? dga_block_grid(hetero ? 0 : n2, n_items)
                                     : dga_panel_batch_grid(n2, n_max, n_items, kernel == 3))
             : hetero ? batch_grid_hetero(mixed, n_items, smem)
                      : batch_grid_any(mixed, n2, n_items, smem);
  if (scratch_bytes < slot) {
    dga_set_error("dga_bse_solve_sum_batch_c128: scratch too small (%zu < one slot of %zu)", scratch_bytes, slot);
    return DGA_ERR_SCRATCH;
  }
  if ((size_t)grid > scratch_bytes / slot) grid = (int)(scratch_bytes / slot);
  const int redo = mode == 2;
  const dga_bse_problem* pd = (const dga_bse_problem*)probs_dev;
  const MultiItem* wk = (const MultiItem*)work;
  unsigned char* sc = (unsigned char*)scratch;
  if (panel) {
    cudaError_t err =
        kernel == 4 ? dga_block_batch_launch(grid, hetero ? 0 : n2, pd, wk, n_items, n_max, max_iter, tol, status,
                                             iters, sc, slot, stream)
                    : dga_panel_batch_launch(grid, n2, pd, wk, n_items, n_max, max_iter, tol, status, iters, sc, slot,
                                             stream, kernel == 3);
    if (err != cudaSuccess) {
      dga_set_error("dga_bse_solve_sum_batch_c128: launch failed: %s", cudaGetErrorString(err));
      return DGA_ERR_LAUNCH;
    }
    return DGA_OK;
  }
  if (hetero) {
    if (mixed)
      bse_multi_any_kernel<true><<<grid, BSE_THREADS, smem, stream>>>(pd, wk, n_items, n_max, max_iter, tol, status,
                                                                      iters, sc, slot, 0);
    else
      bse_multi_any_kernel<false><<<grid, BSE_THREADS, smem, stream>>>(pd, wk, n_items, n_max, max_iter, tol, status,
                                                                       iters, sc, slot, redo);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
      dga_set_error("dga_bse_solve_sum_batch_c128: launch failed: %s", cudaGetErrorString(err));
      return DGA_ERR_LAUNCH;
    }
    return DGA_OK;
  }
#define DGA_BATCH_CASE(R)                                                                                          \
  case R:                                                                                                          \
    if (mixed)                                                                                                     \
      bse_multi_kernel<true, R><<<grid, BSE_THREADS, smem, stream>>>(pd, wk, n_items, n_max, max_iter, tol, status, \
                                                                     iters, sc, slot, 0);                         \
    else                                                                                                           \
      bse_multi_kernel<false, R><<<grid, BSE_THREADS, smem, stream>>>(pd, wk, n_items, n_max, max_iter, tol,       \
                                                                      status, iters, sc, slot, redo);             \
    break;
  switch (n2) {
    DGA_BATCH_CASE(1)
    DGA_BATCH_CASE(4)
    DGA_BATCH_CASE(9)
    DGA_BATCH_CASE(16)
  }
#undef DGA_BATCH_CASE
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_bse_solve_sum_batch_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"

// Loads the code of the block-form BSE kernels ahead of their first launch (see include/dga_b200.h).
extern "C" int dga_bse_preload(void) {
  if (dga_block_preload()) {
    dga_set_error("dga_bse_preload: a kernel could not be loaded: %s", cudaGetErrorString(cudaGetLastError()));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

extern "C" int dga_bse_default_kernel(int n_orb, int niv, int mixed) {
  const int n2 = n_orb * n_orb, N = n2 * 2 * niv;
  if (n_orb <= 0 || niv <= 0 || !supported_rhs(n2) || N > BSE_MAX_N) return -1;
  return mixed ? default_mixed_kernel(N, n2) : 2;
}

// ------------------------------------------------------------------------------------------------
// Tuned entry: the same solves with an explicit kernel choice and CTAs per SM (the autotuner's knobs)
// ------------------------------------------------------------------------------------------------
static int sm_count() { return device_sm_count(); }

// 1 = panel kernel, 2 = 128-thread kernel, 3 = panel kernel with tensor-core trailing tiles,
// -1 = the requested kernel cannot run this size
static int tuned_kernel(int mixed, int N, int n2, const dga_bse_tuning* t) {
  const int k = t ? t->kernel : 0;
  if (k < 0 || k > 4) return -1;
  if (!mixed) return (k == 1 || k == 3 || k == 4) ? -1 : 2;
  if (k == 0) return default_mixed_kernel(N, n2);
  if (k == 1 && !dga_panel_supported(N, n2)) return -1;
  if (k == 3 && !dga_panel_supported(N, n2, true)) return -1;
  if (k == 4 && !dga_block_supported(N, n2)) return -1;
  return k;
}

static int tuned_grid(int kernel, int mixed, int N, int n2, int n_items, const dga_bse_tuning* t, size_t* slot,
                      size_t* smem) {
  if (kernel == 1 || kernel == 3) {
    *slot = dga_panel_slot_bytes(N, n2);
    *smem = 0;
    return dga_panel_grid(n2, N, n_items, kernel == 3);
  }
  if (kernel == 4) {
    *slot = dga_block_slot_bytes(N, n2);
    *smem = 0;
    return dga_block_grid(n2, n_items);
  }
  int grid;
  if (mixed) {
    *smem = mixed_smem_bytes(N, n2);
    *slot = mixed_slot_bytes(N, n2);
    grid = mixed_grid(n_items, *smem);
  } else {
    *smem = bse_smem_bytes(N);
    *slot = ((size_t)N * N + (size_t)N * n2) * sizeof(double2);
    grid = bse_grid(n_items, *smem);
  }
  const int cps = t ? t->ctas_per_sm : 0;
  if (cps > 0) {
    const int cap = sm_count() * cps;
    if (grid > cap) grid = cap;
  }
  return grid;
}

extern "C" {

size_t dga_bse_tuned_scratch_bytes(int N, int n2, int n_items, int mixed, const dga_bse_tuning* t) {
  if (N <= 0 || !supported_rhs(n2) || n_items <= 0 || N > BSE_MAX_N) return 0;
  const int kernel = tuned_kernel(mixed, N, n2, t);
  if (kernel < 0) return 0;
  size_t slot = 0, smem = 0;
  return (size_t)tuned_grid(kernel, mixed, N, n2, n_items, t, &slot, &smem) * slot;
}

int dga_bse_solve_sum_tuned_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                                 const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work,
                                 int n_items, int mixed, int max_iter, double tol, void* out, int* status, int* iters,
                                 const dga_bse_tuning* t, void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || n_ch <= 0 || n_items <= 0 ||
      N > BSE_MAX_N || max_iter < 0 || (mixed != 0 && mixed != 1)) {
    dga_set_error("dga_bse_solve_sum_tuned_c128: invalid sizes (n_orb=%d niv=%d niw_half=%d n_q=%d items=%d)", n_orb,
                  niv, niw_half, n_q, n_items);
    return DGA_ERR_ARG;
  }
  if (!gamma_cm || !chi0_inv || !uv || !work || !out || !scratch || (mixed && !status)) {
    dga_set_error("dga_bse_solve_sum_tuned_c128: null pointer argument");
    return DGA_ERR_ARG;
  }
  const int kernel = tuned_kernel(mixed, N, n2, t);
  if (kernel < 0) {
    dga_set_error("dga_bse_solve_sum_tuned_c128: kernel %d cannot run N=%d in this precision", t ? t->kernel : 0, N);
    return DGA_ERR_ARG;
  }
  size_t slot = 0, smem = 0;
  const int grid = tuned_grid(kernel, mixed, N, n2, n_items, t, &slot, &smem);
  if (scratch_bytes < (size_t)grid * slot) {
    dga_set_error("dga_bse_solve_sum_tuned_c128: scratch too small (%zu < %zu)", scratch_bytes, (size_t)grid * slot);
    return DGA_ERR_SCRATCH;
  }
  StructuredSource src;
  src.gamma_cm = (const double2*)gamma_cm;
  src.chi0_inv = (const double2*)chi0_inv;
  src.uv = (const double2*)uv;
  src.n2 = n2;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  src.inv_beta2 = inv_beta2;
  cudaError_t err;
  if (kernel == 1 || kernel == 3) {
    err = dga_panel_launch(grid, src, (const WorkItem*)work, n_items, N, n2, nv, niw_half, n_q, beta, max_iter, tol,
                           (double2*)out, status, iters, (unsigned char*)scratch, slot, stream, kernel == 3,
                           t ? t->wait_limit : 0);
  } else if (kernel == 4) {
    err = dga_block_launch(grid, src, (const WorkItem*)work, n_items, N, n2, nv, niw_half, n_q, beta, max_iter, tol,
                           (double2*)out, status, iters, (unsigned char*)scratch, slot, stream, t ? t->wait_limit : 0);
  } else if (mixed) {
#define DGA_TUNED_MIXED_CASE(NRV)                                                                                    \
  case NRV:                                                                                                          \
    cudaFuncSetAttribute(bse_solve_sum_mixed_kernel<NRV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
    bse_solve_sum_mixed_kernel<NRV><<<grid, BSE_THREADS, smem, stream>>>(                                            \
        src, (const WorkItem*)work, n_items, N, NRV, nv, niw_half, n_q, beta, max_iter, tol, (double2*)out, status,  \
        iters, (unsigned char*)scratch, slot);                                                                       \
    break;
    switch (n2) {
      DGA_TUNED_MIXED_CASE(1)
      DGA_TUNED_MIXED_CASE(4)
      DGA_TUNED_MIXED_CASE(9)
      DGA_TUNED_MIXED_CASE(16)
    }
#undef DGA_TUNED_MIXED_CASE
    err = cudaGetLastError();
  } else {
    launch_fp64(n2, grid, smem, stream, src, (const WorkItem*)work, n_items, N, nv, niw_half, n_q, beta,
                (double2*)out, status, (double2*)scratch, slot / sizeof(double2), 0);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) {
    dga_set_error("dga_bse_solve_sum_tuned_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Allocation-free variant of dga_bse_solve_sum_c128.
//
// Some callers of this library cannot call cudaMalloc: a host program that binds only this C ABI and has no
// device allocator of its own, or a steady-state serving loop that must never trigger cudaMalloc's implicit
// device-wide synchronisation.  For them the per-CTA working matrices live in the fixed array below, which is
// part of this library's device image: every GPU that loads the library holds these 64 MiB until the process
// exits.  In host code `g_bse_noalloc_scratch` is only a host-side stand-in for the array, not a device
// address, so the device address is looked up once per device with cudaGetSymbolAddress and cached.
// ------------------------------------------------------------------------------------------------

#include <mutex>

#define DGA_BSE_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define DGA_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double2 g_bse_noalloc_scratch[DGA_BSE_NOALLOC_SCRATCH_BYTES / sizeof(double2)];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_ptr[DGA_NOALLOC_MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device (looked up on the first call per device).
static int noalloc_scratch_ptr(void** out) {
  int dev = -1;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess || dev < 0 || dev >= DGA_NOALLOC_MAX_DEVICES) {
    dga_set_error("dga_bse_solve_sum_noalloc_c128: no usable current device (%s)", cudaGetErrorString(err));
    return DGA_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    err = cudaGetSymbolAddress(&p, g_bse_noalloc_scratch);
    if (err != cudaSuccess || !p) {
      dga_set_error("dga_bse_solve_sum_noalloc_c128: cudaGetSymbolAddress failed: %s", cudaGetErrorString(err));
      return DGA_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return DGA_OK;
}

extern "C" {

// Same result as dga_bse_solve_sum_c128 without a caller scratch buffer.  At most
// DGA_BSE_NOALLOC_SCRATCH_BYTES (64 MiB) of working matrices are used: as many CTAs run as there are
// (N*N + N*n2)*16-byte slots in it (at least one), so a compound size N above about 2040 is rejected.
// The first call on a device looks up the array's device address (this can load the module); make that first
// call before any stream capture.  Calls share the array, so calls that overlap on the GPU (different streams
// or threads without ordering between them) race; calls on one stream are ordered and safe.  Each item
// rewrites its slot completely before reading it, so nothing has to be cleared between calls.
int dga_bse_solve_sum_noalloc_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta,
                                   double inv_beta2, const void* gamma_cm, const void* chi0_inv, const void* uv,
                                   const int* work, int n_items, void* out, int* status, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || n_ch <= 0 || n_items <= 0) {
    dga_set_error("dga_bse_solve_sum_noalloc_c128: invalid sizes (n_orb=%d niv=%d niw_half=%d n_q=%d n_ch=%d "
                  "items=%d)", n_orb, niv, niw_half, n_q, n_ch, n_items);
    return DGA_ERR_ARG;
  }
  const size_t slot = (size_t)N * N + (size_t)N * n2;
  const size_t capacity_slots = DGA_BSE_NOALLOC_SCRATCH_BYTES / (slot * sizeof(double2));
  if (N > BSE_MAX_N || capacity_slots < 1) {
    dga_set_error("dga_bse_solve_sum_noalloc_c128: compound size N=%d needs %zu bytes per matrix, more than the "
                  "fixed %llu-byte scratch; use dga_bse_solve_sum_c128 with a caller buffer", N,
                  slot * sizeof(double2), (unsigned long long)DGA_BSE_NOALLOC_SCRATCH_BYTES);
    return DGA_ERR_SCRATCH;
  }
  if (!gamma_cm || !chi0_inv || !uv || !work || !out) {
    dga_set_error("dga_bse_solve_sum_noalloc_c128: null pointer argument");
    return DGA_ERR_ARG;
  }
  void* scratch = nullptr;
  int rc = noalloc_scratch_ptr(&scratch);
  if (rc != DGA_OK) return rc;
  const size_t smem = bse_smem_bytes(N);
  int grid = bse_grid(n_items, smem);
  if ((size_t)grid > capacity_slots) grid = (int)capacity_slots;
  StructuredSource src;
  src.gamma_cm = (const double2*)gamma_cm;
  src.chi0_inv = (const double2*)chi0_inv;
  src.uv = (const double2*)uv;
  src.n2 = n2;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  src.inv_beta2 = inv_beta2;
  launch_fp64(n2, grid, smem, stream, src, (const WorkItem*)work, n_items, N, nv, niw_half, n_q, beta,
              (double2*)out, status, (double2*)scratch, slot, 0);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_bse_solve_sum_noalloc_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"

extern "C" {

// Batched dense LU with partial pivoting of n_mat N x N column-major matrices a + m*mat_stride (in place).
int dga_lu_batched_c128(void* a, int N, int n_mat, long long mat_stride, int* piv, int* status, cudaStream_t stream) {
  if (!a || !piv || !status || N <= 0 || N > DGA_DENSE_MAX_N || n_mat <= 0 || mat_stride < (long long)N * N) {
    dga_set_error("dga_lu_batched_c128: invalid arguments (N=%d n_mat=%d)", N, n_mat);
    return DGA_ERR_ARG;
  }
  const size_t smem = bse_smem_bytes(N);
  const int grid = grid_for(dense_lu_kernel, n_mat, smem);
  dense_lu_kernel<<<grid, BSE_THREADS, smem, stream>>>((double2*)a, N, n_mat, mat_stride, piv, status);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_lu_batched_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

// Solves with the factors of dga_lu_batched_c128 for n_rhs right-hand sides (b null: the identity).
int dga_lu_solve_batched_c128(const void* lu, const int* piv, int N, int n_mat, long long lu_stride, const void* b,
                              long long b_stride_m, long long b_stride_r, long long b_stride_k, int n_rhs, void* out,
                              long long out_stride, int* status, cudaStream_t stream) {
  const long long cols = ((long long)n_rhs + DENSE_RHS - 1) / DENSE_RHS * DENSE_RHS;
  if (!lu || !piv || !out || !status || N <= 0 || N > DGA_DENSE_MAX_N || n_mat <= 0 || n_rhs <= 0 ||
      lu_stride < (long long)N * N || out_stride < cols * N || (!b && n_rhs > N)) {
    dga_set_error("dga_lu_solve_batched_c128: invalid arguments (N=%d n_mat=%d n_rhs=%d)", N, n_mat, n_rhs);
    return DGA_ERR_ARG;
  }
  const size_t smem = bse_smem_bytes(N);
  const long long n_tasks = (long long)n_mat * (cols / DENSE_RHS);
  if (n_tasks > 0x7fffffffLL) {
    dga_set_error("dga_lu_solve_batched_c128: too many right-hand-side blocks");
    return DGA_ERR_ARG;
  }
  const int grid = grid_for(dense_solve_kernel, (int)n_tasks, smem);
  dense_solve_kernel<<<grid, BSE_THREADS, smem, stream>>>((const double2*)lu, piv, N, n_mat, lu_stride,
                                                          (const double2*)b, b_stride_m, b_stride_r, b_stride_k,
                                                          n_rhs, (double2*)out, out_stride, status);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_lu_solve_batched_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"

extern "C" {

// Scratch bytes of dga_bse_solve_sum_eli_c128 for n_items items of size N.
size_t dga_bse_eli_scratch_bytes(int N, int n2, int n_items) {
  if (N <= 0 || !supported_rhs(n2) || n_items <= 0) return 0;
  const size_t smem = bse_smem_bytes(N);
  const int grid = grid_for(bse_fp64_eli_kernel<9, 9>, n_items, smem);
  return (size_t)grid * ((size_t)N * N + (size_t)N * eli_rhs(n2)) * sizeof(double2);
}

// dga_bse_solve_sum_c128 whose items with w < w_pp also write the chi* part of the Eliashberg full vertex in the pp
// box (niv_pp) from the same LU factors: out_pp [2][Q][w_pp][Mb][Mb], Mb = n2 * 2 niv_pp; dga_eli_ladder_term_c128
// completes it to the vertex dga_eli_full_vertex_c128 computes.
int dga_bse_solve_sum_eli_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                               const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work,
                               int n_items, int niv_pp, int w_pp, void* out, void* out_pp, int* status, void* scratch,
                               size_t scratch_bytes, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv, N = n2 * nv;
  if (!supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 || n_ch != 2 || n_items <= 0 ||
      N > BSE_MAX_N || niv_pp <= 0 || niv_pp > niv || w_pp <= 0 || w_pp > niw_half || !gamma_cm || !chi0_inv ||
      !uv || !work || !out || !out_pp || !scratch) {
    dga_set_error("dga_bse_solve_sum_eli_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const size_t smem = bse_smem_bytes(N);
  const size_t slot = (size_t)N * N + (size_t)N * eli_rhs(n2);
  int grid = 0;
  switch (n2) {
    case 1: grid = grid_for(bse_fp64_eli_kernel<1, 16>, n_items, smem); break;
    case 4: grid = grid_for(bse_fp64_eli_kernel<4, 16>, n_items, smem); break;
    case 9: grid = grid_for(bse_fp64_eli_kernel<9, 9>, n_items, smem); break;
    default: grid = grid_for(bse_fp64_eli_kernel<16, 16>, n_items, smem); break;
  }
  if (scratch_bytes < (size_t)grid * slot * sizeof(double2)) {
    dga_set_error("dga_bse_solve_sum_eli_c128: scratch too small");
    return DGA_ERR_SCRATCH;
  }
  StructuredSource src;
  src.gamma_cm = (const double2*)gamma_cm;
  src.chi0_inv = (const double2*)chi0_inv;
  src.uv = (const double2*)uv;
  src.n2 = n2;
  src.nv = nv;
  src.W = niw_half;
  src.Q = n_q;
  src.inv_beta2 = inv_beta2;
#define DGA_ELI_CASE(NRV, NRB)                                                                                 \
  case NRV:                                                                                                    \
    bse_fp64_eli_kernel<NRV, NRB><<<grid, BSE_THREADS, smem, stream>>>(                                        \
        src, (const WorkItem*)work, n_items, N, n2, nv, niw_half, n_q, beta, (double2*)out, niv_pp, w_pp,      \
        (double2*)out_pp, status, (double2*)scratch, slot);                                                    \
    break;
  switch (n2) {
    DGA_ELI_CASE(1, 16)
    DGA_ELI_CASE(4, 16)
    DGA_ELI_CASE(9, 9)
    DGA_ELI_CASE(16, 16)
  }
#undef DGA_ELI_CASE
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_bse_solve_sum_eli_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

// f += (Z G3(nu)) G3(nu') over the pp box for every (ch, q, w < w_pp), Z = U_r - U_r chi_r U_r: completes the
// out_pp of dga_bse_solve_sum_eli_c128 to the full vertex (g3 [2][Q][W][nv][n2][n2], chi_phys [2][Q][W][n2][n2]
// lambda-corrected, uv [2][Q][n2][n2]).
int dga_eli_ladder_term_c128(const void* uv, const void* g3, const void* chi_phys, int n_orb, int niv, int niw_half,
                             int n_q, int niv_pp, int w_pp, void* f, cudaStream_t stream) {
  const int n2 = n_orb * n_orb, nv = 2 * niv;
  if (!uv || !g3 || !chi_phys || !f || !supported_rhs(n2) || n_orb <= 0 || niv <= 0 || niw_half <= 0 || n_q <= 0 ||
      niv_pp <= 0 || niv_pp > niv || w_pp <= 0 || w_pp > niw_half) {
    dga_set_error("dga_eli_ladder_term_c128: invalid arguments");
    return DGA_ERR_ARG;
  }
  const size_t smem = ((size_t)n2 * n2 + (size_t)2 * niv_pp * n2 * n2) * sizeof(double2);
  cudaFuncSetAttribute(eli_ladder_term_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  eli_ladder_term_kernel<<<2 * n_q * w_pp, 256, smem, stream>>>((const double2*)uv, (const double2*)g3,
                                                              (const double2*)chi_phys, n2, nv, niw_half, n_q,
                                                              niv_pp, w_pp, (double2*)f);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    dga_set_error("dga_eli_ladder_term_c128: launch failed: %s", cudaGetErrorString(err));
    return DGA_ERR_LAUNCH;
  }
  return DGA_OK;
}

}  // extern "C"
