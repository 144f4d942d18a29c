// Mixed-precision ladder BSE with the LU panel in shared memory.
//
// Same result as the mixed form of bse.cu (complex64 LU, FP64 iterative refinement of
// X = sum_nu' A^-1 / beta, dgamore/four_point.py:620-684), organised so that no phase of the factorisation
// waits on global memory column by column.  One 512-thread CTA per SM owns one (channel, q, w) item at a time:
//
//   1. A is formed in FP64 from Gamma_r, chi0^-1 and U_r + V_r^q (StructuredSource::element) and stored as
//      complex64, column-major, in the CTA's scratch slot;
//   2. right-looking LU with partial pivoting (LAPACK pivot measure |re|+|im|, first-index ties), 32-column
//      panels.  The m x 32 panel is loaded into shared memory and factored there: each warp owns a contiguous
//      block of rows, two barriers per column, and every warp computes the next column's pivot candidate
//      while it applies the current column's rank-1 update.  The factored panel is written back and stays in
//      shared memory as the L21 operand of the trailing update.  The panel's row interchanges are applied to
//      the columns on its right while U12 = L11^-1 A12 is formed, one 64-column strip at a time (the rows the
//      interchanges touch are read once, then written once), and each strip's 128 x 64 tiles of the trailing
//      matrix are updated in FP32 with L21 and U12 from shared memory.  The interchanges are never applied to
//      the columns left of the panel: the forward substitution applies each panel's interchanges to the
//      right-hand sides before that panel's elimination, which is the same product P_k, L_k^-1 as LAPACK's.
//   3. The n2 selector right-hand sides are solved in FP32 with the right-hand sides held in shared memory;
//      the FP64 refinement loop r = S - A Y (A formed on the fly in FP64), d = (LU)^-1 r, Y += d stops when
//      the correction, or the error left after it as estimated from the observed contraction, is below
//      tol max|Y| (refine_converged).  Items that do not converge, or whose result is not finite, are flagged.
//
// Shared memory holds the m x 32 complex64 panel (256 B per row), so N is limited to about 790 (the 227 KB
// opt-in limit); larger items use the 128-thread kernel of bse.cu.
#include "bse_core.cuh"
#include "tc_tile.cuh"

namespace dga {

constexpr int PT = 512;       // threads per CTA
constexpr int PW = PT / 32;   // warps
static_assert(PW <= 32 && 32 % PW == 0, "a warp merges the PW warp candidates of the pivot search");
constexpr int PNB = 32;       // panel width
constexpr int PSB = 8;        // sub-panel width inside the panel factorisation
constexpr int PTM = 128;      // trailing tile rows
constexpr int PTN = 64;       // trailing strip columns
static_assert(4 * PW == PTN, "prefetch_c_tile gives each warp four columns of a strip");
constexpr int P_MAX_SMEM = 232448;  // 227 KB opt-in shared memory per block on sm_100
#ifndef DGA_PANEL_TILE_UNROLL
#define DGA_PANEL_TILE_UNROLL 8
#endif
constexpr int P_TILE_UNROLL = DGA_PANEL_TILE_UNROLL;  // unroll of the trailing tiles' k loop

// ----------------------------------------------------------------------------------------------
// Shared-memory layout (ldp = leading dimension of the panel = the largest N the launch serves)
// ----------------------------------------------------------------------------------------------
// The panel region also holds the solve's right-hand sides (up to 16 x ldp complex64) followed by the residual's
// staging ([32][16] and [16][16] complex128), so small ldp need more than the panel itself.
// With the tensor-core trailing update (tc) the region also holds the six 32 KB TF32 operand buffers (A_hi, A_lo
// for two tiles in flight, B_hi, B_lo of the strip).
__host__ __device__ inline size_t panel_region_bytes(int ldp, bool tc = false) {
  const size_t panel = (size_t)ldp * PNB * sizeof(float2);
  const size_t solve = (size_t)16 * ldp * sizeof(float2) + 32 + (32 * 16 + 16 * 16) * sizeof(double2);
  size_t r = panel > solve ? panel : solve;
  if (tc && r < 6 * (size_t)TC_OPERAND_FLOATS * sizeof(float)) r = 6 * (size_t)TC_OPERAND_FLOATS * sizeof(float);
  return (r + 127) & ~(size_t)127;
}
constexpr size_t P_FIXED = 16 * sizeof(double)                 // redd
                           + PNB * (PNB + 1) * sizeof(float2)  // L11i
                           + PNB * PTN * sizeof(float2)        // Us
                           + 16 * sizeof(float) + 16 * sizeof(int)  // red_val, red_idx
                           + 64 * sizeof(int) * 2              // s_row, s_cont
                           + 4 * sizeof(int)                   // misc
                           + 48;                               // tile barriers [2], panel-load barrier, TMEM address
__host__ __device__ inline size_t panel_smem_bytes(int ldp, bool tc = false) {
  return panel_region_bytes(ldp, tc) + P_FIXED + sizeof(int) * (size_t)ldp;
}

struct PanelSmem {
  float2* P;     // [PNB][ldp] panel, column-major (also the solve and residual staging area)
  double* redd;  // [16]
  float2* L11i;  // [PNB][PNB+1] inverse of the unit lower triangle of L11
  float2* Us;    // [PNB][PTN] U12 strip
  float* red_val;
  int* red_idx;
  int* s_row;   // [64] rows touched by the panel's interchanges: slots 0..31 the panel rows, 32.. the others
  int* s_cont;  // [64] old row whose content ends up in s_row[slot]
  int* misc;    // [0] rows below the panel that receive another row, [1] status bits, [2] tensor-core wait failure
  uint64_t* bar;    // [2] completion barriers of the two tensor-core tiles in flight
  uint64_t* pbar;   // completion barrier of the panel's bulk load
  uint32_t* tslot;  // TMEM address of the two tile accumulators
  int* piv;     // [ldp] row interchanged with row j
  int ldp;
  long long wait_limit;  // polls of the bounded waits inside an item (the drains at exit use TC_WAIT_LIMIT)
  long long inject;      // > 0: the CTA's first wait is on a phase nothing completes (test hook), this many polls

  __device__ PanelSmem(unsigned char* base, int ldp_, bool tc, long long wait_limit_)
      : ldp(ldp_), wait_limit(wait_limit_ > 0 ? wait_limit_ : TC_WAIT_LIMIT), inject(wait_limit_ < 0 ? -wait_limit_ : 0) {
    unsigned char* p = base;
    P = reinterpret_cast<float2*>(p);
    p += panel_region_bytes(ldp, tc);
    redd = reinterpret_cast<double*>(p);
    p += 16 * sizeof(double);
    bar = reinterpret_cast<uint64_t*>(p);
    p += 16;
    pbar = reinterpret_cast<uint64_t*>(p);
    p += 16;
    tslot = reinterpret_cast<uint32_t*>(p);
    p += 16;
    L11i = reinterpret_cast<float2*>(p);
    p += PNB * (PNB + 1) * sizeof(float2);
    Us = reinterpret_cast<float2*>(p);
    p += PNB * PTN * sizeof(float2);
    red_val = reinterpret_cast<float*>(p);
    p += 16 * sizeof(float);
    red_idx = reinterpret_cast<int*>(p);
    p += 16 * sizeof(int);
    s_row = reinterpret_cast<int*>(p);
    p += 64 * sizeof(int);
    s_cont = reinterpret_cast<int*>(p);
    p += 64 * sizeof(int);
    misc = reinterpret_cast<int*>(p);
    p += 4 * sizeof(int);
    piv = reinterpret_cast<int*>(p);
  }
};

// Warp-wide argmax of the pivot candidates (v, idx), in every lane: the largest v, ties to the smallest idx (the
// rule of argmax_merge).  Non-negative floats order as their bit patterns, so two integer reductions do it; a
// negative or NaN v is no candidate.
__device__ __forceinline__ void warp_argmax(float& v, int& idx) {
  const bool ok = v >= 0.f;
  const unsigned key = ok ? __float_as_uint(v) : 0u;
  const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
  const unsigned imin = __reduce_min_sync(0xffffffffu, (ok && key == kmax) ? (unsigned)idx : 0x7fffffffu);
  v = __uint_as_float(kmax);
  idx = (int)imin;
}

// ----------------------------------------------------------------------------------------------
// Factor the m x nb panel in shared memory (column-major, leading dimension ldp) with partial pivoting.
// Rows are local to the panel (row r = global row k0 + r); piv[k0 + j] receives the global pivot row.
// Returns true if an exact zero pivot was met (the column is then left unscaled, as LAPACK's zgetf2 does).
// ----------------------------------------------------------------------------------------------
__device__ bool panel_factor(PanelSmem& s, int m, int nb, int k0) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float2* P = s.P;
  const int ldp = s.ldp;
  const int rpw = (m + PW - 1) / PW;
  const int r0 = warp * rpw, r1 = min(m, r0 + rpw);
  bool singular = false;
  {
    float best = -1.f;
    int bidx = 0x7fffffff;
    for (int r = r0 + lane; r < r1; r += 32) {
      const float v = cabs1(P[r]);
      if (v > best) {
        best = v;
        bidx = r;
      }
    }
    warp_argmax(best, bidx);
    if (lane == 0) {
      s.red_val[warp] = best;
      s.red_idx[warp] = bidx;
    }
  }
  for (int jj = 0; jj < nb; ++jj) {
    __syncthreads();  // this column's candidates are in place; the previous update is complete
    // every warp merges the 16 warp candidates (lanes l and l + 16 holding the same one), so all lanes of all
    // warps agree on the pivot
    float bv = s.red_val[lane & (PW - 1)];
    int p = s.red_idx[lane & (PW - 1)];
    warp_argmax(bv, p);
    if (p < jj || p >= m) p = jj;  // cannot happen (row jj itself is a candidate); keeps p in range
    if (tid == 0) s.piv[k0 + jj] = k0 + p;
    if (p != jj && tid < nb) {
      float2* col = P + (size_t)tid * ldp;
      const float2 t = col[jj];
      col[jj] = col[p];
      col[p] = t;
    }
    __syncthreads();  // pivot row in place
    const float2 d = P[(size_t)jj * ldp + jj];
    const bool zero = (d.x == 0.f && d.y == 0.f);
    singular |= zero;
    const float2 rinv = zero ? make_float2(0.f, 0.f) : crecip(d);
    // rank-1 update restricted to the current 8-column sub-panel; the columns to its right are brought up to
    // date by one triangular solve and one rank-8 update when the sub-panel is complete
    const int c1 = jj + 1;
    const int cend = min(nb, (jj / PSB + 1) * PSB);
    float best = -1.f;
    int bidx = 0x7fffffff;
    for (int r = max(r0, c1) + lane; r < r1; r += 32) {
      float2 l = P[(size_t)jj * ldp + r];
      if (!zero) l = cmul(l, rinv);
      P[(size_t)jj * ldp + r] = l;
      if (c1 < cend) {
        float2 v = P[(size_t)c1 * ldp + r];
        cfms(v, l, P[(size_t)c1 * ldp + jj]);
        P[(size_t)c1 * ldp + r] = v;
        const float a = cabs1(v);
        if (a > best) {
          best = a;
          bidx = r;
        }
        for (int c = c1 + 1; c < cend; ++c) {
          float2 x = P[(size_t)c * ldp + r];
          cfms(x, l, P[(size_t)c * ldp + jj]);
          P[(size_t)c * ldp + r] = x;
        }
      }
    }
    if (c1 == cend && cend < nb) {
      const int cb = cend - PSB;
      __syncthreads();  // the sub-panel's multipliers are final
      // U block rows cb .. cend-1 of the columns to the right: unit lower solve with the sub-panel's L11
      for (int c = cend + tid; c < nb; c += PT) {
        float2* col = P + (size_t)c * ldp + cb;
        float2 x[PSB];
#pragma unroll
        for (int k = 0; k < PSB; ++k) x[k] = col[k];
#pragma unroll
        for (int k = 1; k < PSB; ++k)
#pragma unroll
          for (int q = 0; q < k; ++q) cfms(x[k], P[(size_t)(cb + q) * ldp + cb + k], x[q]);
#pragma unroll
        for (int k = 0; k < PSB; ++k) col[k] = x[k];
      }
      __syncthreads();
      // rank-8 update of the rows below, with the next column's pivot candidate
      for (int r = max(r0, cend) + lane; r < r1; r += 32) {
        float2 l[PSB];
#pragma unroll
        for (int k = 0; k < PSB; ++k) l[k] = P[(size_t)(cb + k) * ldp + r];
        for (int c = cend; c < nb; ++c) {
          const float4* u4 = reinterpret_cast<const float4*>(P + (size_t)c * ldp + cb);
          float2 v = P[(size_t)c * ldp + r];
#pragma unroll
          for (int k2 = 0; k2 < PSB / 2; ++k2) {
            const float4 uu = u4[k2];
            cfms(v, l[2 * k2], make_float2(uu.x, uu.y));
            cfms(v, l[2 * k2 + 1], make_float2(uu.z, uu.w));
          }
          P[(size_t)c * ldp + r] = v;
          if (c == cend) {
            const float a = cabs1(v);
            if (a > best) {
              best = a;
              bidx = r;
            }
          }
        }
      }
    }
    warp_argmax(best, bidx);
    if (lane == 0) {
      s.red_val[warp] = best;
      s.red_idx[warp] = bidx;
    }
  }
  __syncthreads();
  return singular;
}

// Inverses of the panel's diagonal blocks, lane = row, warp w doing columns w and 31 - w (equal chain lengths):
// X = L11^-1 (unit lower) into s.L11i for U12 and into linv, and Z = U11^-1 (upper) into uinv (both stored
// transposed, [column][row], zero outside the triangle and beyond nb) for the triangular solves, whose diagonal
// steps are then products.
__device__ void panel_diag_inverses(PanelSmem& s, int nb, float2* __restrict__ linv, float2* __restrict__ uinv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float2 dinv = lane < nb ? crecip(s.P[(size_t)lane * s.ldp + lane]) : make_float2(0.f, 0.f);
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    const int c = h == 0 ? warp : PNB - 1 - warp;
    float2 x = make_float2(lane == c ? 1.f : 0.f, 0.f);
    for (int k = c; k < nb - 1; ++k) {
      const float xk_re = __shfl_sync(0xffffffffu, x.x, k);
      const float xk_im = __shfl_sync(0xffffffffu, x.y, k);
      if (lane > k && lane < nb) cfms(x, s.P[(size_t)k * s.ldp + lane], make_float2(xk_re, xk_im));
    }
    if (lane >= nb || lane < c) x = make_float2(0.f, 0.f);
    s.L11i[lane * (PNB + 1) + c] = x;
    linv[c * PNB + lane] = x;
    // U11 z = e_c by back substitution, U[r][k] = P[k * ldp + r] for r <= k
    float2 rhs = make_float2(lane == c ? 1.f : 0.f, 0.f), z = make_float2(0.f, 0.f);
    for (int k = min(c, nb - 1); k >= 0; --k) {
      if (lane == k) z = cmul(rhs, dinv);
      const float zr = __shfl_sync(0xffffffffu, z.x, k), zi = __shfl_sync(0xffffffffu, z.y, k);
      if (lane < k) cfms(rhs, s.P[(size_t)k * s.ldp + lane], make_float2(zr, zi));
    }
    if (lane > c || lane >= nb) z = make_float2(0.f, 0.f);
    uinv[c * PNB + lane] = z;
  }
}

// Net effect of the panel's interchanges on the rows they touch (one warp): after the sequential swaps
// (k0+t <-> piv[k0+t]) row s_row[slot] holds the old content of row s_cont[slot].
__device__ void panel_interchange_map(PanelSmem& s, int k0, int nb) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return;
  s.s_row[lane] = k0 + lane;
  s.s_cont[lane] = k0 + lane;
  int n_tgt = 0;
  __syncwarp();
  for (int t = 0; t < nb; ++t) {
    const int p = s.piv[k0 + t];
    if (p == k0 + t) continue;
    int slot;
    if (p < k0 + nb) {
      slot = p - k0;
    } else {
      const unsigned hit = __ballot_sync(0xffffffffu, lane < n_tgt && s.s_row[32 + lane] == p);
      if (hit) {
        slot = 32 + __ffs(hit) - 1;
      } else {
        slot = 32 + n_tgt;
        if (lane == 0) {
          s.s_row[slot] = p;
          s.s_cont[slot] = p;
        }
        ++n_tgt;
      }
    }
    __syncwarp();
    if (lane == 0) {
      const int tmp = s.s_cont[t];
      s.s_cont[t] = s.s_cont[slot];
      s.s_cont[slot] = tmp;
    }
    __syncwarp();
  }
  if (lane == 0) s.misc[0] = n_tgt;
}

// ----------------------------------------------------------------------------------------------
// LU of the N x N complex64 column-major matrix A (leading dimension N) in place.
// ----------------------------------------------------------------------------------------------
// TC = true: the trailing tiles run on the tensor cores (tc_tile.cuh); L21 is then read back from global memory
// (the panel region holds the tile operands), and parity tracks the phase of the tile completion barrier.
// A has NC >= N columns: columns N .. NC-1 are extra right-hand sides, which receive every interchange and
// trailing update, so that they end as L^-1 P times their start (the forward substitution done in passing).
// L2 prefetch of rows [r0, r1) of columns [c0, c0 + nc) of the item's matrix (column-major, leading dimension
// N), one bulk prefetch per column by the calling warp's lanes.  The range is widened to 16-byte boundaries, which stays
// inside the item's slot (A starts 256-byte aligned and its selector columns follow column N - 1).
__device__ __forceinline__ void prefetch_factor_cols(const float2* A, int N, int c0, int nc, int r0, int r1) {
  const int lane = threadIdx.x & 31;
  if (r1 <= r0) return;
  for (int c = lane; c < nc; c += 32) {
    const float2* col = A + (size_t)(c0 + c) * N;
    const uintptr_t a = reinterpret_cast<uintptr_t>(col + r0) & ~(uintptr_t)15;
    const uintptr_t e = (reinterpret_cast<uintptr_t>(col + r1) + 15) & ~(uintptr_t)15;
    bulk_prefetch_l2(reinterpret_cast<const void*>(a), (uint32_t)(e - a));
  }
}

// L2 prefetch of rows [r0, min(r0 + nr, N)) of the strip's columns [cs, cs + cw), spread over the CTA's warps
// (warp w takes columns 4w .. 4w + 3; PW * 4 = PTN covers the strip).
__device__ __forceinline__ void prefetch_c_tile(const float2* A, int N, int cs, int cw, int r0, int nr) {
  const int c0 = 4 * (threadIdx.x >> 5);
  if (c0 < cw) prefetch_factor_cols(A, N, cs + c0, min(4, cw - c0), r0, min(r0 + nr, N));
}

// inv: per panel b, L11^-1 at inv + 2048 b and U11^-1 at inv + 2048 b + 1024 (panel_diag_inverses).
template <bool TC>
__device__ bool panel_lu(float2* __restrict__ A, int N, int NC, PanelSmem& s, uint32_t& parity,
                         float2* __restrict__ inv) {
  const int tid = threadIdx.x;
  bool singular = false;
  for (int k0 = 0; k0 < N; k0 += PNB) {
    const int nb = min(PNB, N - k0), m = N - k0, k1 = k0 + nb;
    // ---- load the panel: one bulk copy (TMA engine) per column, global -> shared, completing on the panel
    // barrier; the fence orders every thread's earlier accesses (its writes of these columns, its reads of the
    // panel region) before the copies.  Once any bounded wait of this CTA has run out (misc[2]) the CTA issues
    // no more bulk copies or tiles: the panel is then read with plain loads, so the barrier's only phase that
    // can still be pending is the one whose wait ran out (drained at exit) ----
    fence_proxy_async_all();
    __syncthreads();
    if (s.misc[2] == 0) {
      if (tid < 32) {
        if (tid == 0) mbar_expect_tx(s.pbar, (uint32_t)((size_t)m * nb * sizeof(float2)));
        __syncwarp();
        for (int c = tid; c < nb; c += 32)
          bulk_g2s(s.P + (size_t)c * s.ldp, A + (size_t)(k0 + c) * N + k0, (uint32_t)(m * sizeof(float2)), s.pbar);
      }
      if (!mbar_wait(s.pbar, (parity >> 2) & 1u, s.wait_limit)) s.misc[2] = 1;  // flags the item
      parity ^= 4u;
    } else {
      for (int e = tid; e < m * nb; e += PT) {
        const int c = e / m, r = e - c * m;
        s.P[(size_t)c * s.ldp + r] = __ldcg(A + (size_t)(k0 + c) * N + k0 + r);
      }
    }
    __syncthreads();
    singular |= panel_factor(s, m, nb, k0);
    for (int e = tid; e < m * nb; e += PT) {
      const int c = e / m, r = e - c * m;
      A[(size_t)(k0 + c) * N + k0 + r] = s.P[(size_t)c * s.ldp + r];
    }
    if (k1 >= NC) break;
    panel_diag_inverses(s, nb, inv + (size_t)(k0 / PNB) * 2 * PNB * PNB, inv + (size_t)(k0 / PNB) * 2 * PNB * PNB + PNB * PNB);
    panel_interchange_map(s, k0, nb);
    __syncthreads();
    const int n_tgt = s.misc[0];
    // ---- per 64-column strip: interchanges + U12, then the strip's trailing tiles ----
    for (int cs = k1; cs < NC; cs += PTN) {
      const int cw = min(PTN, NC - cs);
      // L2 prefetch of the strip's first two C tiles (warp w: columns 4w .. 4w + 3); the tile loop keeps two
      // tiles ahead, so the C stream reads from L2 instead of waiting on DRAM
      if (TC) prefetch_c_tile(A, N, cs, cw, k1, 2 * TC_M);
      {
        // warp w handles columns w, w + 16, w + 32, w + 48 of the strip; lane = row of the U block (reads of the
        // touched rows are coalesced along the column).  Every old value is read, and U12 computed, before the
        // barrier; the writes follow it.
        const int lane = tid & 31, warp = tid >> 5;
        float2 u[PTN / PW], tv[PTN / PW];
        const int src_row = s.s_cont[lane];
        const int tgt_src = lane < n_tgt ? s.s_cont[32 + lane] : 0;
        float2 av[PTN / PW];
#pragma unroll
        for (int q = 0; q < PTN / PW; ++q) {
          const int c = warp + PW * q;
          const float2* colp = A + (size_t)(cs + c) * N;
          av[q] = (c < cw && lane < nb) ? __ldcg(colp + src_row) : make_float2(0.f, 0.f);
          tv[q] = (c < cw && lane < n_tgt) ? __ldcg(colp + tgt_src) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int q = 0; q < PTN / PW; ++q) {
          float2 acc = make_float2(0.f, 0.f);
#pragma unroll
          for (int k = 0; k < PNB; ++k) {
            const float re = __shfl_sync(0xffffffffu, av[q].x, k), im = __shfl_sync(0xffffffffu, av[q].y, k);
            cfma(acc, s.L11i[lane * (PNB + 1) + k], make_float2(re, im));
          }
          u[q] = acc;
        }
        __syncthreads();  // every old value of the touched rows is read before any is overwritten
        const int tgt_row = lane < n_tgt ? s.s_row[32 + lane] : 0;
#pragma unroll
        for (int q = 0; q < PTN / PW; ++q) {
          const int c = warp + PW * q;
          float2* colw = A + (size_t)(cs + c) * N;
          const bool act = c < cw && lane < nb;
          if (act) colw[k0 + lane] = u[q];
          s.Us[lane * PTN + c] = act ? u[q] : make_float2(0.f, 0.f);
          if (c < cw && lane < n_tgt) colw[tgt_row] = tv[q];
        }
      }
      __syncthreads();
      if (TC) {
        // U12 strip -> the B operand of the real product (tc_tile.cuh), split into TF32 pairs: row 2c + s of B
        // (K-major) holds, for k = 2j, 2j + 1, the four reals (Re U, -Im U) (s = 0) or (Im U, Re U) (s = 1);
        // a thread writes one 16-byte chunk, consecutive threads consecutive rows of a core matrix.
        float* b_hi = reinterpret_cast<float*>(s.P) + 4 * TC_OPERAND_FLOATS;  // after the two tiles' A buffers
        float* b_lo = b_hi + TC_OPERAND_FLOATS;
#pragma unroll
        for (int e = tid; e < TC_NR * (TC_KR / 4); e += PT) {
          const int row = e & (TC_NR - 1), j = e >> 7;  // B row (2c + s) and 16-byte K chunk (k = 2j, 2j + 1)
          const int c = row >> 1, sgn = row & 1;
          const float2 u0 = s.Us[(2 * j) * PTN + c], u1 = s.Us[(2 * j + 1) * PTN + c];
          const float4 x = sgn ? make_float4(u0.y, u0.x, u1.y, u1.x) : make_float4(u0.x, -u0.y, u1.x, -u1.y);
          const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
          *reinterpret_cast<float4*>(b_hi + tc_off(row, 4 * j)) = h;
          *reinterpret_cast<float4*>(b_lo + tc_off(row, 4 * j)) = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
        }
      }
      if (TC) {
        // trailing tiles of the strip on the tensor cores, 128 rows x 64 complex columns per tile, two tiles in
        // flight: while the MMAs of tile i run, the threads stage tile i + 1 (L21 rows into the other A buffers,
        // C into the other TMEM accumulator), then wait for tile i and write it back.
        float* const a_base = reinterpret_cast<float*>(s.P);
        const float* b_hi = a_base + 4 * TC_OPERAND_FLOATS;
        const float* b_lo = b_hi + TC_OPERAND_FLOATS;
        const int lane = tid & 31, warp = tid >> 5;
        const uint32_t tbase = *s.tslot;
        const uint32_t taddr = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + 32 * (warp >> 2);
        const int ntiles = (N - k1 + TC_M - 1) / TC_M;
        float v[32];
        auto stage = [&](int i) {
          const int rt = k1 + i * TC_M;
          float* ah = a_base + (i & 1) * 2 * TC_OPERAND_FLOATS;
          float* al = ah + TC_OPERAND_FLOATS;
          {  // L21 rows rt .. rt + 127 (written back with the panel): a thread takes a row and 4 chunks of 2 k
            const int row = tid & (TC_M - 1), cg = tid >> 7;
            const int r = rt + row;
            const bool rok = r < N;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int ch = cg + 4 * j;
              const float2 x0 = rok ? __ldcg(A + (size_t)(k0 + 2 * ch) * N + r) : make_float2(0.f, 0.f);
              const float2 x1 = rok ? __ldcg(A + (size_t)(k0 + 2 * ch + 1) * N + r) : make_float2(0.f, 0.f);
              const float4 h = make_float4(tf32_hi(x0.x), tf32_hi(x0.y), tf32_hi(x1.x), tf32_hi(x1.y));
              const float4 l = make_float4(x0.x - h.x, x0.y - h.y, x1.x - h.z, x1.y - h.w);
              *reinterpret_cast<float4*>(ah + tc_off(row, 4 * ch)) = h;
              *reinterpret_cast<float4*>(al + tc_off(row, 4 * ch)) = l;
            }
          }
          const int r = rt + 32 * (warp & 3) + lane, cb = cs + 16 * (warp >> 2);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = cb + j;
            const float2 x = (r < N && c < NC) ? __ldcg(A + (size_t)c * N + r) : make_float2(0.f, 0.f);
            v[2 * j] = x.x;
            v[2 * j + 1] = x.y;
          }
          tmem_st32(taddr + (i & 1) * TC_NR, v);
          tmem_wait_st();
          tc_fence_async_smem();
        };
        bool live = true;
        auto issue = [&](int i) {  // after a barrier: every operand and accumulator of tile i is in place
          live = s.misc[2] == 0;   // a CTA whose tensor-core wait ever ran out issues no more tiles
          if (live && tid == 0) {
            tc_fence_after();
            const float* ah = a_base + (i & 1) * 2 * TC_OPERAND_FLOATS;
            tc_issue_tile(tbase + (i & 1) * TC_NR, ah, ah + TC_OPERAND_FLOATS, b_hi, b_lo, s.bar + (i & 1));
          }
        };
        auto finish = [&](int i) {
          const int bsel = i & 1;
          const bool ok = live && mbar_wait(s.bar + bsel, (parity >> bsel) & 1u, s.wait_limit);
          if (live) parity ^= 1u << bsel;
          tc_fence_after();
          if (ok) {
            tmem_ld32(taddr + bsel * TC_NR, v);
            tmem_wait_ld();
            const int r = k1 + i * TC_M + 32 * (warp & 3) + lane, cb = cs + 16 * (warp >> 2);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int c = cb + j;
              if (r < N && c < NC) A[(size_t)c * N + r] = make_float2(v[2 * j], v[2 * j + 1]);
            }
          } else {
            s.misc[2] = 1;
          }
        };
        if (ntiles > 0) {  // the last panel can have columns to its right (the extra ones) but no rows below
          stage(0);
          tc_fence_before();
          __syncthreads();
          issue(0);
        }
        for (int i = 0; i < ntiles; ++i) {
          if (i + 2 < ntiles) prefetch_c_tile(A, N, cs, cw, k1 + (i + 2) * TC_M, TC_M);
          if (i + 1 < ntiles) stage(i + 1);
          finish(i);
          if (i + 1 < ntiles) {
            tc_fence_before();
            __syncthreads();
            issue(i + 1);
          }
        }
        tc_fence_before();
      } else {
      // trailing tiles of the strip, 128 x 64: thread (ty, tx) owns rows rt + 2ty + {0,1} + {0,64} and columns
        // cs + 2tx + {0,1} + {0,32} (row pairs and column pairs move as one 16-byte access; N is even), with the
        // real and imaginary parts in separate scalar accumulators.
        const int ty = tid & 31, tx = tid >> 5;
        const float2* up = s.Us + 2 * tx;
        for (int rt = k1; rt < N; rt += PTM) {
          float cr[16], ci[16];  // index (column j of 4) * 4 + (row i of 4)
          const int rbase = rt + 2 * ty;
          const bool full = rt + PTM <= N && cs + PTN <= NC;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int c = cs + 2 * tx + (j & 1) + 32 * (j >> 1);
#pragma unroll
            for (int ap = 0; ap < 2; ++ap) {
              const int r = rbase + 64 * ap;
              float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
              if (full || (c < NC && r < N)) v = *reinterpret_cast<const float4*>(A + (size_t)c * N + r);
              cr[j * 4 + 2 * ap] = v.x;
              ci[j * 4 + 2 * ap] = v.y;
              cr[j * 4 + 2 * ap + 1] = v.z;
              ci[j * 4 + 2 * ap + 1] = v.w;
            }
          }
          const bool r0ok = full || rbase < N, r1ok = full || rbase + 64 < N;
          const float2* lp0 = s.P + (r0ok ? rbase - k0 : 0);
          const float2* lp1 = s.P + (r1ok ? rbase + 64 - k0 : 0);
#pragma unroll P_TILE_UNROLL
          for (int k = 0; k < nb; ++k) {
            float4 l0 = *reinterpret_cast<const float4*>(lp0 + (size_t)k * s.ldp);
            float4 l1 = *reinterpret_cast<const float4*>(lp1 + (size_t)k * s.ldp);
            if (!r0ok) l0 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (!r1ok) l1 = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 u0 = *reinterpret_cast<const float4*>(up + k * PTN);
            const float4 u1 = *reinterpret_cast<const float4*>(up + k * PTN + 32);
            const float lr[4] = {l0.x, l0.z, l1.x, l1.z}, li[4] = {l0.y, l0.w, l1.y, l1.w};
            const float ur[4] = {u0.x, u0.z, u1.x, u1.z}, ui[4] = {u0.y, u0.w, u1.y, u1.w};
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                cr[j * 4 + i] = fmaf(-lr[i], ur[j], cr[j * 4 + i]);
                cr[j * 4 + i] = fmaf(li[i], ui[j], cr[j * 4 + i]);
                ci[j * 4 + i] = fmaf(-lr[i], ui[j], ci[j * 4 + i]);
                ci[j * 4 + i] = fmaf(-li[i], ur[j], ci[j * 4 + i]);
              }
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int c = cs + 2 * tx + (j & 1) + 32 * (j >> 1);
#pragma unroll
            for (int ap = 0; ap < 2; ++ap) {
              const int r = rbase + 64 * ap;
              if (full || (c < NC && r < N))
                *reinterpret_cast<float4*>(A + (size_t)c * N + r) =
                    make_float4(cr[j * 4 + 2 * ap], ci[j * 4 + 2 * ap], cr[j * 4 + 2 * ap + 1], ci[j * 4 + 2 * ap + 1]);
            }
          }
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();
  return singular;
}

// ----------------------------------------------------------------------------------------------
// In-place solve (L U) y = b for the NR right-hand sides y[s][i] (complex64, shared memory, stride ldy),
// with the factors of panel_lu and its interchanges piv (applied panel by panel in the forward pass).
// ----------------------------------------------------------------------------------------------

// Prefetch of step b of a triangular solve: the factor block the step's update reads and its diagonal inverse.
__device__ __forceinline__ void prefetch_solve_step(const float2* A, int N, const float2* inv, int b, bool forward) {
  const int nblk = (N + PNB - 1) / PNB;
  if (b < 0 || b >= nblk) return;
  const int k0 = b * PNB, nb = min(PNB, N - k0);
  if (forward) prefetch_factor_cols(A, N, k0, nb, k0 + nb, N);
  else prefetch_factor_cols(A, N, k0, nb, 0, k0);
  if ((threadIdx.x & 31) == 0)
    bulk_prefetch_l2(inv + (size_t)b * 2 * PNB * PNB + (forward ? 0 : PNB * PNB), PNB * PNB * sizeof(float2));
}

// Triangular solves with the factors in A (column-major, leading dimension N) and the inverses of their diagonal
// blocks in inv, for NR right-hand sides y[r * ldy + i] in shared memory.  A step of either solve is a product
// with the block's inverse (warp r for right-hand side r, lane = row) followed by the update of the rows beyond
// the block (thread per row).  The next step's inverse is staged into sinv (shared, 2 x 32 x 32, double
// buffered) during the update, and the factor blocks two steps ahead are prefetched into L2.
template <int NR>
__device__ void panel_solve(const float2* __restrict__ A, int N, const int* piv, float2* y, int ldy,
                            const float2* __restrict__ inv, float2* sinv, bool forward = true) {
  static_assert(PNB * PNB == 2 * PT, "the staging of a block inverse gives every thread two elements");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (N + PNB - 1) / PNB;
  const int nf = forward ? nblk : 0, nsteps = nf + nblk;
  // step st: forward block st (st < nf), else backward block nblk - 1 - (st - nf)
  auto step_block = [&](int st) { return st < nf ? st : nblk - 1 - (st - nf); };
  auto step_inv = [&](int st) { return inv + (size_t)step_block(st) * 2 * PNB * PNB + (st < nf ? 0 : PNB * PNB); };
  if (warp == PW - 1) {
    for (int st = 0; st < 2 && st < nsteps; ++st) prefetch_solve_step(A, N, inv, step_block(st), st < nf);
  }
  {
    const float2* src = step_inv(0);
    sinv[tid] = src[tid];
    sinv[tid + PT] = src[tid + PT];
  }
  __syncthreads();
  for (int st = 0; st < nsteps; ++st) {
    const bool fwd = st < nf;
    const int b = step_block(st), k0 = b * PNB, nb = min(PNB, N - k0);
    const float2* sv = sinv + (st & 1) * PNB * PNB;
    if (warp == PW - 1 && st + 2 < nsteps) prefetch_solve_step(A, N, inv, step_block(st + 2), st + 2 < nf);
    if (fwd) {  // the panel's row interchanges
      if (warp == 0 && lane < NR) {
        float2* ys = y + (size_t)lane * ldy;
        for (int t = 0; t < nb; ++t) {
          const int p = piv[k0 + t];
          if (p != k0 + t) {
            const float2 tmp = ys[k0 + t];
            ys[k0 + t] = ys[p];
            ys[p] = tmp;
          }
        }
      }
      __syncthreads();
    }
    // diagonal block: y_b <- inv_b y_b
    if (warp < NR) {
      float2* ys = y + (size_t)warp * ldy + k0;
      float2 acc = make_float2(0.f, 0.f);
#pragma unroll 8
      for (int k = 0; k < nb; ++k) cfma(acc, sv[k * PNB + lane], ys[k]);
      __syncwarp();
      if (lane < nb) ys[lane] = acc;
    }
    float2 nx0 = make_float2(0.f, 0.f), nx1 = nx0;  // the next step's inverse, stored after the update
    if (st + 1 < nsteps) {
      const float2* src = step_inv(st + 1);
      nx0 = src[tid];
      nx1 = src[tid + PT];
    }
    __syncthreads();
    // update of the rows beyond the block: forward rows [k0 + nb, N), backward rows [0, k0)
    const int i0 = fwd ? k0 + nb : 0, i1 = fwd ? N : k0;
    for (int i = i0 + tid; i < i1; i += PT) {
      float2 acc[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) acc[r] = y[(size_t)r * ldy + i];
      for (int k = 0; k < nb; k += 16) {  // 16 factor loads in flight
        float2 l[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) l[u] = (k + u < nb) ? __ldcg(A + (size_t)(k0 + k + u) * N + i) : make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 16; ++u)
          if (k + u < nb) {
#pragma unroll
            for (int r = 0; r < NR; ++r) cfms(acc[r], l[u], y[(size_t)r * ldy + k0 + k + u]);
          }
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) y[(size_t)r * ldy + i] = acc[r];
    }
    if (st + 1 < nsteps) {
      float2* dst = sinv + ((st + 1) & 1) * PNB * PNB;
      dst[tid] = nx0;
      dst[tid + PT] = nx1;
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------------------------
// One work item: form, factor, solve, refine.  Returns the status bits; *iters = number of corrections.
//   slot: A (N x N complex64) | Y (NR x N complex128) | Rb (NR x N complex128)
// ----------------------------------------------------------------------------------------------
// slot: A with its n2 selector columns (N x (N + n2) complex64) | Y (n2 x N complex128) | Rb (n2 x N complex128)
//       | inverses of the diagonal blocks (2 x 32 x 32 complex64 per 32-column panel)
__host__ __device__ inline size_t panel_a_bytes(int N, int n2) {
  return ((size_t)N * (N + n2) * sizeof(float2) + 255) & ~(size_t)255;
}
__host__ __device__ inline size_t panel_slot_bytes(int N, int n2) {
  return panel_a_bytes(N, n2) + 2 * (size_t)N * n2 * sizeof(double2) +
         (size_t)((N + PNB - 1) / PNB) * 2 * PNB * PNB * sizeof(float2);
}

template <int NR, bool TC>
__device__ int solve_item_panel(const StructuredSource& src, const WorkItem& wi, int N, int nv, double beta,
                                int max_iter, double tol, double2* __restrict__ o, unsigned char* slot, PanelSmem& s,
                                int* iters, uint32_t& parity) {
  const int tid = threadIdx.x;
  float2* A = reinterpret_cast<float2*>(slot);
  double2* Y = reinterpret_cast<double2*>(slot + panel_a_bytes(N, NR));
  double2* Rb = Y + (size_t)N * NR;
  float2* inv = reinterpret_cast<float2*>(Rb + (size_t)N * NR);
  // ---- form A in complex64: thread t owns rows t and t + PT (N <= 2 PT here), 8 columns of loads in flight ----
  // element (i, j) as StructuredSource::element: (chi0^-1 [block diagonal] + Gamma / beta^2) + (-(U + V) / beta^2)
  {
    const double2* gam = src.gamma_cm + ((size_t)(wi.ch * src.W + wi.w) * N) * N;
    const double2* c0 = src.chi0_inv + ((size_t)wi.q * src.W + wi.w) * nv * NR * NR;
    const double2* uvq = src.uv + ((size_t)wi.ch * src.Q + wi.q) * NR * NR;
    const double ib2 = src.inv_beta2;
    int ri[2], pr[2], vr[2];
    bool rok[2];
#pragma unroll
    for (int a2 = 0; a2 < 2; ++a2) {
      ri[a2] = tid + a2 * PT;
      rok[a2] = ri[a2] < N;
      pr[a2] = rok[a2] ? ri[a2] / nv : 0;
      vr[a2] = rok[a2] ? ri[a2] - pr[a2] * nv : 0;
    }
    for (int j0 = 0; j0 < N; j0 += 8) {
      double2 g[2][8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2)
          g[a2][u] = (rok[a2] && j0 + u < N) ? __ldcg(gam + (size_t)(j0 + u) * N + ri[a2]) : make_double2(0.0, 0.0);
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = j0 + u;
        if (j >= N) break;
        const int pc = j / nv, vc = j - pc * nv;
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2) {
          if (!rok[a2]) continue;
          const double2 uu = uvq[pr[a2] * NR + pc];
          double re = __dmul_rn(g[a2][u].x, ib2);
          double im = __dmul_rn(g[a2][u].y, ib2);
          if (vr[a2] == vc) {
            const double2 c = c0[(size_t)vr[a2] * NR * NR + pr[a2] * NR + pc];
            re = __dadd_rn(c.x, re);
            im = __dadd_rn(c.y, im);
          }
          re = __dadd_rn(re, -__dmul_rn(uu.x, ib2));
          im = __dadd_rn(im, -__dmul_rn(uu.y, ib2));
          A[(size_t)j * N + ri[a2]] = make_float2((float)re, (float)im);
        }
      }
    }
    // the n2 selector columns S[(p, nu)][s] = delta_ps, factored along with A (panel_lu's extra columns)
#pragma unroll
    for (int a2 = 0; a2 < 2; ++a2)
      if (rok[a2])
        for (int r = 0; r < NR; ++r) A[(size_t)(N + r) * N + ri[a2]] = make_float2(pr[a2] == r ? 1.f : 0.f, 0.f);
  }
  __syncthreads();
  const bool singular = panel_lu<TC>(A, N, N + NR, s, parity, inv);
  // ---- initial solve against the selector: S[(p,nu)][s] = delta_{p s} ----
  const int ldy = N;
  float2* y = s.P;
  double2* ys = reinterpret_cast<double2*>(s.P) + (((size_t)NR * N + 1) / 2 + 1);  // after y, 16-byte aligned
  double2* colsum = ys + 32 * NR;
  // the selector columns hold L^-1 P S after the factorisation: only the back substitution is left
  for (int e = tid; e < NR * N; e += PT) y[e] = A[(size_t)N * N + e];
  __syncthreads();
  panel_solve<NR>(A, N, s.piv, y, ldy, inv, s.Us, false);
  double prev = 0.0;
  for (int e = tid; e < NR * N; e += PT) {
    Y[e] = make_double2(y[e].x, y[e].y);
    prev = fmax(prev, (double)fmaxf(fabsf(y[e].x), fabsf(y[e].y)));
  }
  prev = block_max(prev, s.redd);
  int it = 0;
  bool converged = false;
  for (; it < max_iter; ++it) {
    structured_residual_permuted<NR>(src, wi.ch, wi.q, wi.w, N, nv, Y, Rb, nullptr, colsum, ys);
    for (int e = tid; e < NR * N; e += PT) y[e] = make_float2((float)Rb[e].x, (float)Rb[e].y);
    __syncthreads();
    panel_solve<NR>(A, N, s.piv, y, ldy, inv, s.Us);
    double dmax = 0.0, ymax = 0.0;
    for (int e = tid; e < NR * N; e += PT) {
      const double2 d = make_double2(y[e].x, y[e].y);
      const double2 v = cadd(Y[e], d);
      Y[e] = v;
      dmax = fmax(dmax, fmax(fabs(d.x), fabs(d.y)));
      ymax = fmax(ymax, fmax(fabs(v.x), fabs(v.y)));
    }
    dmax = block_max(dmax, s.redd);
    ymax = block_max(ymax, s.redd);
    if (isnan(dmax) || refine_converged(dmax, ymax, prev, tol)) {  // NaN is flagged below
      converged = !isnan(dmax);
      ++it;
      break;
    }
    prev = dmax;
  }
  if (tid == 0) s.misc[1] = 0;
  __syncthreads();
  bool bad = false;
  for (int e = tid; e < N * NR; e += PT) {
    const int i = e / NR, r = e - i * NR;
    double2 v = Y[(size_t)r * N + i];
    v.x = v.x / beta;
    v.y = v.y / beta;
    if (!cfinite(v)) bad = true;
    o[e] = v;
  }
  if (bad) atomicOr(&s.misc[1], DGA_ITEM_NONFINITE);
  __syncthreads();
  // a bounded wait that ran out leaves the factors incomplete: flag the item for the FP64 re-solve
  const int st = (singular ? DGA_ITEM_SINGULAR : 0) | s.misc[1] | (converged ? 0 : DGA_ITEM_NOCONVERGE) |
                 (s.misc[2] ? DGA_ITEM_WAIT_TIMEOUT : 0);
  *iters = it;
  __syncthreads();
  return st;
}

// TMEM for the tensor-core tiles: one warp allocates 256 columns (two 128 x 128 fp32 accumulators, one per tile in
// flight) for the CTA's lifetime; the two completion barriers are initialised once.  At exit, a CTA whose wait
// ever ran out waits once more, with the full limit, for the panel load and each tile still in flight before the
// columns are freed; panel_kernel_end returns false if one of those waits also ran out (the launch is then
// suspect: every item of the CTA is flagged DGA_ITEM_WAIT_TIMEOUT).
template <bool TC>
__device__ void panel_kernel_begin(PanelSmem& s) {
  if (threadIdx.x == 0) {
    s.misc[2] = 0;
    mbar_init(s.pbar);
    if (s.inject) mbar_init(s.pbar + 1);  // the test hook's barrier: nothing ever arrives on it
  }
  if (TC) {
    if ((threadIdx.x >> 5) == 0) tc_alloc(s.tslot, 2 * TC_NR);
    if (threadIdx.x == 0) {
      mbar_init(s.bar);
      mbar_init(s.bar + 1);
    }
    tc_fence_before();
  }
  __syncthreads();
  if (TC) tc_fence_after();
  if (s.inject) {
    // test hook (dga_bse_tuning.wait_limit < 0): a bounded wait on a phase that nothing completes runs out, and
    // the CTA takes the path of a real timeout -- no more bulk copies or tiles, every item flagged
    if (!mbar_wait(s.pbar + 1, 0u, s.inject)) s.misc[2] = 1;
    __syncthreads();
  }
}

template <bool TC>
__device__ bool panel_kernel_end(PanelSmem& s, uint32_t parity) {
  __syncthreads();
  bool drained = true;
  // a panel load whose wait ran out may still be landing
  if (s.misc[2]) drained &= mbar_wait(s.pbar, ((parity >> 2) & 1u) ^ 1u);
  if (TC) {
    tc_fence_before();
    __syncthreads();
    if (s.misc[2]) {  // a wait ran out: give each tile still in flight one more full wait before freeing TMEM
      drained &= mbar_wait(s.bar, (parity & 1u) ^ 1u);
      drained &= mbar_wait(s.bar + 1, ((parity >> 1) & 1u) ^ 1u);
    }
    if ((threadIdx.x >> 5) == 0) tc_dealloc(*s.tslot, 2 * TC_NR);
  }
  return __syncthreads_and(drained ? 1 : 0) != 0;
}

// Flags every item the CTA processed when a drain wait at exit ran out.
__device__ __forceinline__ void flag_cta_items(int* status, int n_items) {
  if (!status) return;
  for (int item = blockIdx.x + threadIdx.x * gridDim.x; item < n_items; item += blockDim.x * gridDim.x)
    atomicOr(status + item, DGA_ITEM_WAIT_TIMEOUT);
}

template <int NR, bool TC>
__global__ void __launch_bounds__(PT, 1)
    bse_panel_mixed_kernel(StructuredSource src, const WorkItem* __restrict__ work, int n_items, int N, int nv, int W,
                           int Q, double beta, int max_iter, double tol, double2* __restrict__ out,
                           int* __restrict__ status, int* __restrict__ iters, unsigned char* __restrict__ scratch,
                           size_t slot_bytes, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PanelSmem s(smem_raw, N, TC, wait_limit);
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  uint32_t parity = 0;
  panel_kernel_begin<TC>(s);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const WorkItem wi = work[item];
    double2* o = out + (((size_t)wi.ch * Q + wi.q) * W + wi.w) * (size_t)N * NR;
    int it = 0;
    const int st = solve_item_panel<NR, TC>(src, wi, N, nv, beta, max_iter, tol, o, slot, s, &it, parity);
    if (threadIdx.x == 0) {
      if (status) status[item] = st;
      if (iters) iters[item] = it;
    }
  }
  if (!panel_kernel_end<TC>(s, parity)) flag_cta_items(status, n_items);
}

// Heterogeneous batch (requests of one orbital count): see bse_multi_kernel in bse.cu.
template <int NR, bool TC>
__global__ void __launch_bounds__(PT, 1)
    bse_panel_multi_kernel(const dga_bse_problem* __restrict__ probs, const MultiItem* __restrict__ work,
                           int n_items, int n_max, int max_iter, double tol, int* __restrict__ status,
                           int* __restrict__ iters, unsigned char* __restrict__ scratch, size_t slot_bytes,
                           long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PanelSmem s(smem_raw, n_max, TC, wait_limit);
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  uint32_t parity = 0;
  panel_kernel_begin<TC>(s);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const MultiItem mi = work[item];
    const dga_bse_problem d = probs[mi.prob];
    StructuredSource src;
    src.gamma_cm = (const double2*)d.gamma_cm;
    src.chi0_inv = (const double2*)d.chi0_inv;
    src.uv = (const double2*)d.uv;
    src.n2 = NR;
    src.nv = 2 * d.niv;
    src.W = d.niw_half;
    src.Q = d.n_q;
    src.inv_beta2 = d.inv_beta2;
    const int N = NR * src.nv;
    const WorkItem wi{mi.ch, mi.q, mi.w};
    double2* o = (double2*)d.out + (((size_t)wi.ch * src.Q + wi.q) * src.W + wi.w) * (size_t)N * NR;
    int it = 0;
    const int st = solve_item_panel<NR, TC>(src, wi, N, src.nv, d.beta, max_iter, tol, o, slot, s, &it, parity);
    if (threadIdx.x == 0) {
      status[item] = st;
      if (iters) iters[item] = it;
    }
  }
  if (!panel_kernel_end<TC>(s, parity)) flag_cta_items(status, n_items);
}

}  // namespace dga

using namespace dga;

// ----------------------------------------------------------------------------------------------
// Host side (called from bse.cu)
// ----------------------------------------------------------------------------------------------
bool dga_panel_supported(int N, int n2, bool tc) {
#ifdef DGA_DISABLE_PANEL
  return false;
#else
  return (n2 == 1 || n2 == 4 || n2 == 9 || n2 == 16) && N > 0 && panel_smem_bytes(N, tc) <= (size_t)P_MAX_SMEM;
#endif
}

size_t dga_panel_slot_bytes(int N, int n2) { return (panel_slot_bytes(N, n2) + 255) & ~(size_t)255; }

template <typename K>
static int panel_grid_for(K kernel, int n_items, size_t smem) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, PT, smem);
  if (per_sm < 1) per_sm = 1;
  const int g = sms * per_sm;
  return n_items < g ? n_items : g;
}

template <bool TC>
static int panel_grid_tc(int n2, int N, int n_items) {
  const size_t smem = panel_smem_bytes(N, TC);
  switch (n2) {
    case 1: return panel_grid_for(bse_panel_mixed_kernel<1, TC>, n_items, smem);
    case 4: return panel_grid_for(bse_panel_mixed_kernel<4, TC>, n_items, smem);
    case 9: return panel_grid_for(bse_panel_mixed_kernel<9, TC>, n_items, smem);
    default: return panel_grid_for(bse_panel_mixed_kernel<16, TC>, n_items, smem);
  }
}

int dga_panel_grid(int n2, int N, int n_items, bool tc) {
  return tc ? panel_grid_tc<true>(n2, N, n_items) : panel_grid_tc<false>(n2, N, n_items);
}

template <bool TC>
static int panel_batch_grid_tc(int n2, int n_max, int n_items) {
  const size_t smem = panel_smem_bytes(n_max, TC);
  switch (n2) {
    case 1: return panel_grid_for(bse_panel_multi_kernel<1, TC>, n_items, smem);
    case 4: return panel_grid_for(bse_panel_multi_kernel<4, TC>, n_items, smem);
    case 9: return panel_grid_for(bse_panel_multi_kernel<9, TC>, n_items, smem);
    default: return panel_grid_for(bse_panel_multi_kernel<16, TC>, n_items, smem);
  }
}

int dga_panel_batch_grid(int n2, int n_max, int n_items, bool tc) {
  return tc ? panel_batch_grid_tc<true>(n2, n_max, n_items) : panel_batch_grid_tc<false>(n2, n_max, n_items);
}

template <bool TC>
static void panel_launch_tc(int grid, const StructuredSource& src, const WorkItem* work, int n_items, int N, int n2,
                            int nv, int W, int Q, double beta, int max_iter, double tol, double2* out, int* status,
                            int* iters, unsigned char* scratch, size_t slot_bytes, cudaStream_t stream,
                            long long wait_limit) {
  const size_t smem = panel_smem_bytes(N, TC);
#define DGA_PANEL_CASE(R)                                                                                          \
  case R:                                                                                                          \
    bse_panel_mixed_kernel<R, TC><<<grid, PT, smem, stream>>>(src, work, n_items, N, nv, W, Q, beta, max_iter, tol, \
                                                              out, status, iters, scratch, slot_bytes, wait_limit); \
    break;
  switch (n2) {
    DGA_PANEL_CASE(1)
    DGA_PANEL_CASE(4)
    DGA_PANEL_CASE(9)
    DGA_PANEL_CASE(16)
  }
#undef DGA_PANEL_CASE
}

cudaError_t dga_panel_launch(int grid, const StructuredSource& src, const WorkItem* work, int n_items, int N, int n2,
                             int nv, int W, int Q, double beta, int max_iter, double tol, double2* out, int* status,
                             int* iters, unsigned char* scratch, size_t slot_bytes, cudaStream_t stream, bool tc,
                             long long wait_limit) {
  if (tc)
    panel_launch_tc<true>(grid, src, work, n_items, N, n2, nv, W, Q, beta, max_iter, tol, out, status, iters, scratch,
                          slot_bytes, stream, wait_limit);
  else
    panel_launch_tc<false>(grid, src, work, n_items, N, n2, nv, W, Q, beta, max_iter, tol, out, status, iters,
                           scratch, slot_bytes, stream, wait_limit);
  return cudaGetLastError();
}

template <bool TC>
static void panel_batch_launch_tc(int grid, int n2, const dga_bse_problem* probs, const MultiItem* work, int n_items,
                                  int n_max, int max_iter, double tol, int* status, int* iters, unsigned char* scratch,
                                  size_t slot_bytes, cudaStream_t stream, long long wait_limit) {
  const size_t smem = panel_smem_bytes(n_max, TC);
#define DGA_PANEL_CASE(R)                                                                                           \
  case R:                                                                                                           \
    bse_panel_multi_kernel<R, TC><<<grid, PT, smem, stream>>>(probs, work, n_items, n_max, max_iter, tol, status, \
                                                              iters, scratch, slot_bytes, wait_limit);             \
    break;
  switch (n2) {
    DGA_PANEL_CASE(1)
    DGA_PANEL_CASE(4)
    DGA_PANEL_CASE(9)
    DGA_PANEL_CASE(16)
  }
#undef DGA_PANEL_CASE
}

cudaError_t dga_panel_batch_launch(int grid, int n2, const dga_bse_problem* probs, const MultiItem* work, int n_items,
                                   int n_max, int max_iter, double tol, int* status, int* iters,
                                   unsigned char* scratch, size_t slot_bytes, cudaStream_t stream, bool tc,
                                   long long wait_limit) {
  if (tc)
    panel_batch_launch_tc<true>(grid, n2, probs, work, n_items, n_max, max_iter, tol, status, iters, scratch,
                                slot_bytes, stream, wait_limit);
  else
    panel_batch_launch_tc<false>(grid, n2, probs, work, n_items, n_max, max_iter, tol, status, iters, scratch,
                                 slot_bytes, stream, wait_limit);
  return cudaGetLastError();
}
