// Pieces shared by the BSE solvers (bse.cu, bse_panel.cu): how a work item's matrix is formed, the work-item
// records, the arg-max merge of the pivot search and the FP64 residual of the mixed-precision forms.
#pragma once

#include "dga_common.cuh"
#include "tc_tile.cuh"

namespace dga {

// ----------------------------------------------------------------------------------------------
// Matrix sources: how A(i, j) of a work item is formed
// ----------------------------------------------------------------------------------------------

// A formed from the resident ladder inputs (structured form of nonlocal_sde.py:85-96).
struct StructuredSource {
  const double2* gamma_cm;  // [n_ch][W][N][N]: column-major compound Gamma_r(w): element (i,j) at j*N + i
  const double2* chi0_inv;  // [Q][W][nv][n2][n2]: chi0^-1 orbital matrices, row (o1,o2), column (o4,o3)
  const double2* uv;        // [n_ch][Q][n2][n2]: U_r + V_r^q, row (o1,o2), column (o4,o3)
  int n2, nv, W, Q;
  double inv_beta2;  // 1 / beta**2 computed on the host exactly as the upstream does

  // Element (i, j) in FP64, with the upstream's order of operations: (chi0inv_diag + Gamma*ib2) + (-(uv*ib2)).
  __device__ __forceinline__ double2 element(int ch, int q, int w, int N, int i, int j, int pr, int vr, int pc,
                                             int vc) const {
    const double2 g = gamma_cm[((size_t)(ch * W + w) * N + j) * N + i];
    const double2 u = uv[((size_t)ch * Q + q) * n2 * n2 + pr * n2 + pc];
    double re = __dmul_rn(g.x, inv_beta2);
    double im = __dmul_rn(g.y, inv_beta2);
    if (vr == vc) {
      const double2 c = chi0_inv[(((size_t)q * W + w) * nv + vr) * n2 * n2 + pr * n2 + pc];
      re = __dadd_rn(c.x, re);
      im = __dadd_rn(c.y, im);
    }
    re = __dadd_rn(re, -__dmul_rn(u.x, inv_beta2));
    im = __dadd_rn(im, -__dmul_rn(u.y, inv_beta2));
    return make_double2(re, im);
  }
};

// A given explicitly in the upstream FourPoint layout [q][o1][o2][o3][o4][w][nu][nu'] (the generic
// FourPoint.invert_and_sum_over_last_vn, four_point.py:620-642).
struct DenseSource {
  const double2* mat;  // [Q][n][n][n][n][W][nv][nv]
  int nb, nv, W, Q;

  __device__ __forceinline__ double2 element(int ch, int q, int w, int N, int i, int j, int pr, int vr, int pc,
                                             int vc) const {
    const int o1 = pr / nb, o2 = pr - o1 * nb;
    const int o4 = pc / nb, o3 = pc - o4 * nb;
    size_t idx = ((((size_t)q * nb + o1) * nb + o2) * nb + o3) * nb + o4;
    idx = ((idx * W + w) * nv + vr) * nv + vc;
    return mat[idx];
  }
};

struct WorkItem {
  int ch, q, w;
};

struct MultiItem {
  int prob, ch, q, w;
};

// ----------------------------------------------------------------------------------------------
// Pivot arg-max merge: larger value wins, ties go to the smaller row index (LAPACK izamax order).
// ----------------------------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void argmax_merge(R& v, int& idx, R ov, int oidx) {
  if (ov > v || (ov == v && oidx < idx)) {
    v = ov;
    idx = oidx;
  }
}

__device__ inline double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    v = lane < nw ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    if (lane == 0) red[0] = v;
  }
  __syncthreads();
  const double r = red[0];
  __syncthreads();
  return r;
}


// Stopping test of the iterative refinement after a correction d_k (max-norms): the correction itself is below
// tol max|Y|, or the error left after it, estimated from the observed contraction rho = |d_k| / |d_(k-1)| as the
// geometric tail |d_k| rho / (1 - rho), is.  For the first correction d_(k-1) is the initial solution Y_0 (its
// error is the first correction, so rho is again the contraction of one step).
__device__ inline bool refine_converged(double dmax, double ymax, double prev, double tol) {
  if (dmax <= tol * ymax) return true;
  const double rho = prev > 0.0 ? dmax / prev : 1.0;
  return rho < 0.5 && dmax * rho / (1.0 - rho) <= tol * ymax;
}

// ----------------------------------------------------------------------------------------------
// FP64 residual of the mixed forms
// ----------------------------------------------------------------------------------------------
// r[s][i] = S[perm[i]][s] - (A Y)[perm[i]][s]: the residual of original row perm[i], stored at position i
// (so the correction solve needs no separate permutation; perm == nullptr keeps the original order).  colsum: shared [n2][n2]; ys: shared [32][n2]
// staging of Y rows, so the Gamma stream is the only global traffic of the inner loop.
template <int NR>
__device__ void structured_residual_permuted(const StructuredSource& src, int ch, int q, int w, int N, int nv,
                                             const double2* __restrict__ Y, double2* __restrict__ Rp,
                                             const int* __restrict__ perm, double2* colsum, double2* ys) {
  constexpr int n2 = NR;
  const int tid = threadIdx.x, T = blockDim.x;
  // column sums over nu' of Y for the rank-n2 (U_r + V_r^q) part
  for (int e = tid; e < n2 * n2; e += T) {
    const int pc = e / n2, sidx = e - pc * n2;
    double2 acc = make_double2(0.0, 0.0);
    const double2* y = Y + (size_t)sidx * N + pc * nv;
    for (int v = 0; v < nv; ++v) acc = cadd(acc, y[v]);
    colsum[pc * n2 + sidx] = acc;
  }
  __syncthreads();
  const double2* gam = src.gamma_cm + (size_t)(ch * src.W + w) * N * N;
  const double2* uvq = src.uv + ((size_t)ch * src.Q + q) * n2 * n2;
  const uint64_t keep = l2_policy_evict_last();  // Gamma_r(w) is shared by every q of the (channel, w)
  for (int pos0 = 0; pos0 < N; pos0 += T) {
    const int pos = pos0 + tid;
    const bool active = pos < N;
    const int i = active ? (perm ? perm[pos] : pos) : 0;
    double2 acc[NR];
#pragma unroll
    for (int sidx = 0; sidx < NR; ++sidx) acc[sidx] = make_double2(0.0, 0.0);
    // Gamma part: sum_j Gamma[i][j] Y[j][s], Y staged 32 rows at a time; the next 32 Gamma columns are
    // prefetched into L2 (one bulk prefetch per column by the last warp) while this chunk is summed
    for (int j0 = 0; j0 < N; j0 += 32) {
      const int jw = min(32, N - j0);
      if ((tid >> 5) == (T >> 5) - 1 && j0 + 32 + (tid & 31) < N)
        bulk_prefetch_l2(gam + (size_t)(j0 + 32 + (tid & 31)) * N, (uint32_t)(N * sizeof(double2)));
      for (int e = tid; e < jw * NR; e += T) {
        const int jj = e % jw, sidx = e / jw;
        ys[jj * NR + sidx] = Y[(size_t)sidx * N + j0 + jj];
      }
      __syncthreads();
      if (active) {
        for (int jj0 = 0; jj0 < jw; jj0 += 8) {  // 8 Gamma loads in flight
          double2 g[8];
#pragma unroll
          for (int u = 0; u < 8; ++u)
            g[u] = (jj0 + u < jw) ? ld_d2_hint(gam + (size_t)(j0 + jj0 + u) * N + i, keep) : make_double2(0.0, 0.0);
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (jj0 + u < jw) {
#pragma unroll
              for (int sidx = 0; sidx < NR; ++sidx) cfma(acc[sidx], g[u], ys[(jj0 + u) * NR + sidx]);
            }
        }
      }
      __syncthreads();
    }
    if (active) {
      const int pr = i / nv, vr = i - pr * nv;
      const double2* c0 = src.chi0_inv + (((size_t)q * src.W + w) * nv + vr) * n2 * n2 + pr * n2;
#pragma unroll
      for (int sidx = 0; sidx < NR; ++sidx) {
        double2 a = cscale(acc[sidx], src.inv_beta2);
        double2 d = make_double2(0.0, 0.0), u = make_double2(0.0, 0.0);
        for (int pc = 0; pc < n2; ++pc) {
          cfma(d, c0[pc], Y[(size_t)sidx * N + pc * nv + vr]);
          cfma(u, uvq[pr * n2 + pc], colsum[pc * n2 + sidx]);
        }
        a = cadd(a, d);
        a = csub(a, cscale(u, src.inv_beta2));
        const double sel = (pr == sidx) ? 1.0 : 0.0;
        Rp[(size_t)sidx * N + pos] = make_double2(sel - a.x, -a.y);
      }
    }
  }
  __syncthreads();
}

}  // namespace dga

// Host side of the shared-memory-panel mixed kernel (bse_panel.cu), used by the entry points in bse.cu.
bool dga_panel_supported(int N, int n2, bool tc = false);
size_t dga_panel_slot_bytes(int N, int n2);
int dga_panel_grid(int n2, int N, int n_items, bool tc = false);
int dga_panel_batch_grid(int n2, int n_max, int n_items, bool tc = false);
cudaError_t dga_panel_launch(int grid, const dga::StructuredSource& src, const dga::WorkItem* work, int n_items, int N,
                             int n2, int nv, int W, int Q, double beta, int max_iter, double tol, double2* out,
                             int* status, int* iters, unsigned char* scratch, size_t slot_bytes, cudaStream_t stream,
                             bool tc = false, long long wait_limit = 0);
// Host side of the block-form mixed kernel (bse_block.cu): pivoting restricted to 32 x 32 diagonal blocks, every
// update on the tensor cores, two 256-thread CTAs per SM.
bool dga_block_supported(int N, int n2);
int dga_block_preload();  // nonzero if a kernel could not be loaded
size_t dga_block_slot_bytes(int N, int n2);
int dga_block_grid(int n2, int n_items);
cudaError_t dga_block_launch(int grid, const dga::StructuredSource& src, const dga::WorkItem* work, int n_items, int N,
                             int n2, int nv, int W, int Q, double beta, int max_iter, double tol, double2* out,
                             int* status, int* iters, unsigned char* scratch, size_t slot_bytes, cudaStream_t stream,
                             long long wait_limit = 0);
cudaError_t dga_block_batch_launch(int grid, int n2, const dga_bse_problem* probs, const dga::MultiItem* work,
                                   int n_items, int n_max, int max_iter, double tol, int* status, int* iters,
                                   unsigned char* scratch, size_t slot_bytes, cudaStream_t stream,
                                   long long wait_limit = 0);
cudaError_t dga_panel_batch_launch(int grid, int n2, const dga_bse_problem* probs, const dga::MultiItem* work,
                                   int n_items, int n_max, int max_iter, double tol, int* status, int* iters,
                                   unsigned char* scratch, size_t slot_bytes, cudaStream_t stream, bool tc = false,
                                   long long wait_limit = 0);
