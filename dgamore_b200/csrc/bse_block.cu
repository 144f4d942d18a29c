// Mixed-precision ladder BSE, block form: the LU's pivot search restricted to 32 x 32 diagonal blocks, every
// update on the tensor cores (kernel choice 4 of dga_bse_tuning).
//
// Same result as the other mixed kernels: X = sum_nu' A^-1 / beta for each (channel, q, w) work item
// (dgamore/four_point.py:620-684, reached from nonlocal_sde.py:85-156), with A = chi0^-1 + (Gamma_r - U_r - V_r^q)
// / beta^2 formed in FP64 (the upstream's order of operations) and stored as complex64, factored with FP32-level
// products, and refined in FP64 until the correction is below tol max|Y|.
//
// Factorisation: block Gaussian elimination on 32 x 32 blocks in Schur-complement form.  Step k:
//   D_k^-1   inverse of the current diagonal block, by Gauss-Jordan elimination with partial pivoting inside the
//            block (the whole CTA; the row interchanges end up inside D_k^-1);
//   A[>k, >k] -= (A[>k, k] D_k^-1) A[k, >k]   the trailing update on the tensor cores: per 128-row block the
//            product L' = A[rows, k] D_k^-1 is one tensor-core product whose result becomes the A operand of the
//            block's 128 x 32 tiles, whose B operands are the block row's split planes (built once per step).
// The block row and the block column stay as they are, so A = L U with L = [I; A_ik D_k^-1] and U = [D_k, A_kj]:
//   forward   z_k = D_k^-1 y_k, then y_i -= A_ik z_k for i > k;
//   backward  y_k <- D_k^-1 y_k, then y_i -= A_ik y_k for i < k.
// The n2 selector columns ride along as extra columns, so after the factorisation they hold the forward result.
// Restricting the pivot search to the diagonal block removes the CTA-wide, column-by-column pivot chain; the
// FP64 refinement restores full accuracy (one correction at the 3-orbital size, as with partial pivoting).  An
// exactly singular diagonal block, or a refinement that does not converge (small pivots inside a block), flags
// the item DGA_ITEM_NOCONVERGE for the FP64 re-solve with partial pivoting.
//
// Tensor-core products (tcgen05.mma kind::tf32): complex operands as planar (Re, Im) TF32 matrices with the
// three-term split x = x_hi + x_lo (A B ~ A_lo B_hi + A_hi B_lo + A_hi B_hi, the dropped A_lo B_lo is 2^-22
// relative), four real products per complex product with the signs from the instruction descriptor's negate
// bit; the (Re, Im) accumulators, 128 x 32 fp32 each, live in tensor memory.  Operands are K-major without
// swizzle in shared memory: element (row, k) of a plane at float offset kb_off(row, k).
//
// One 256-thread CTA per item, two CTAs per SM (about 105 KB of shared memory and 128 TMEM columns each), so the
// latency-bound steps of one item (diagonal inverses, triangular solves, the FP64 residual) overlap the other
// item's tiles.  Every wait on a tile's completion barrier is bounded; a CTA whose wait runs out issues no more
// tiles, flags its items DGA_ITEM_WAIT_TIMEOUT and drains what it issued before exiting.
#include "bse_core.cuh"
#include "tc_tile.cuh"

namespace dga {

constexpr int KT = 256;        // threads per CTA
constexpr int KW = KT / 32;    // warps
constexpr int KB = 32;         // diagonal block size (the pivot search stays inside it) = K of every product
constexpr int KTM = 128;       // tile rows (TMEM lanes)
constexpr int KTN = 32;        // tile complex columns
constexpr int KAP = KTM * KB;  // floats of one A plane (128 x 32)
constexpr int KBP = KTN * KB;  // floats of one B plane (32 x 32)
constexpr int K_REGION = 4 * KAP * 4 + 2 * 4 * KBP * 4;  // A planes (64 KB) + two B plane sets (2 x 16 KB)
constexpr int K_DLD = 33;                                 // leading dimension of the diagonal inverse in smem
constexpr uint32_t K_SBO = 1024;                          // 8 rows x 32 floats: stride byte offset of a plane
constexpr uint32_t K_WAIT_HINT_NS = 1000;  // longest suspension of one poll of a tile wait
constexpr uint32_t K_A_COL = 128;      // TMEM A operand planes (4 x 32 columns) after the accumulators
constexpr uint32_t K_TMEM_COLS = 256;  // two tiles in flight x (Re, Im) x 32 columns, then the A operand planes

// kind::tf32, D fp32, A and B tf32 K-major, M = 128, N = 32; bit 13 negates A.
constexpr uint32_t K_IDESC_POS = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(KTN >> 3) << 17) |
                                 ((uint32_t)(KTM >> 4) << 24);
constexpr uint32_t K_IDESC_NEG = K_IDESC_POS | (1u << 13);

__host__ __device__ __forceinline__ int kb_off(int row, int k) {
  return (row >> 3) * 256 + (k >> 2) * 32 + (row & 7) * 4 + (k & 3);
}

__host__ __device__ inline size_t block_smem_bytes() {
  return (size_t)K_REGION + KB * K_DLD * sizeof(float2) + 32 /*bars*/ + 16 /*probe*/ + 16 /*tslot*/ +
         16 /*misc*/ + 8 * sizeof(double) /*redd*/;
}

// Solve-phase use of the region: y [NR][N] complex64 | ys [32][NR] + colsum [NR][NR] complex128 | two staged
// diagonal inverses [2][32][33] complex64 (rows padded against bank conflicts) | the forward solve's D^-1 y_b
// [NR][32] complex64.
__host__ __device__ inline size_t block_solve_bytes(int N, int NR) {
  const size_t y = (((size_t)NR * N * sizeof(float2)) + 15) & ~(size_t)15;
  return y + (size_t)(32 * NR + NR * NR) * sizeof(double2) + 2 * KB * K_DLD * sizeof(float2) +
         (size_t)NR * KB * sizeof(float2);
}

struct BlockSmem {
  float* a_pl;    // [4][KAP] A planes (Re hi, Re lo, Im hi, Im lo) of L'; also the Gauss-Jordan workspace
  float2* cbuf;   // [2][32][128] the C tiles of a strip pair, column-major (aliases a_pl)
  float* b_pl;    // [2][4][KBP] B planes of a strip pair
  float2* y;      // solve phase: right-hand sides [NR][N]
  double2* ys;    // solve phase: [32][NR] staging of the residual
  double2* colsum;  // solve phase: [NR][NR]
  float2* sinv;   // solve phase: [2][32][K_DLD] staged diagonal inverses
  float2* zb;     // solve phase: [NR][32] D^-1 y_b of the forward solve
  float2* dinv;   // [32][K_DLD] current diagonal inverse, row-major
  uint64_t* bar;  // [4] completion barriers: [0] the products of a strip pair (four issuing threads), [1] the L'
                  // product (two), [2] bulk copies of a pair's C tiles, [3] those of its B planes
  uint64_t* probe;  // test hook: a barrier nothing arrives on
  uint32_t* tslot;  // TMEM base address
  int* misc;      // [0] a wait ran out, [1] status bits of the item, [2] the item met a singular diagonal block
  double* redd;   // [8] block reductions
  long long wait_limit, inject;

  __device__ BlockSmem(unsigned char* base, int N, int NR, long long wl)
      : wait_limit(wl > 0 ? wl : TC_WAIT_LIMIT), inject(wl < 0 ? -wl : 0) {
    unsigned char* p = base;
    a_pl = reinterpret_cast<float*>(p);
    cbuf = reinterpret_cast<float2*>(p);
    b_pl = a_pl + 4 * KAP;
    y = reinterpret_cast<float2*>(p);
    const size_t yb = (((size_t)NR * N * sizeof(float2)) + 15) & ~(size_t)15;
    ys = reinterpret_cast<double2*>(p + yb);
    colsum = ys + 32 * NR;
    sinv = reinterpret_cast<float2*>(colsum + NR * NR);
    zb = sinv + 2 * KB * K_DLD;
    p += K_REGION;
    dinv = reinterpret_cast<float2*>(p);
    p += KB * K_DLD * sizeof(float2);
    bar = reinterpret_cast<uint64_t*>(p);
    p += 32;
    probe = reinterpret_cast<uint64_t*>(p);
    p += 16;
    tslot = reinterpret_cast<uint32_t*>(p);
    p += 16;
    misc = reinterpret_cast<int*>(p);
    p += 16;
    redd = reinterpret_cast<double*>(p);
  }
};

// Tile bookkeeping of one thread, in two registers (bit i for barrier i): pend, a phase has been issued that this
// thread has not yet seen complete; par, the parity of the next phase to wait for.  By construction a barrier has
// at most one phase in flight.
constexpr int K_NBAR = 4;
struct TileCount {
  uint32_t pend = 0u, par = 0u;
  __device__ __forceinline__ void issued(int i) { pend |= 1u << i; }
  __device__ __forceinline__ void observed(int i) {
    pend &= ~(1u << i);
    par ^= 1u << i;
  }
};

// slot: A with its NR selector columns (N x (N + NR) complex64, column-major) | D_k^-1 per block (32 x 32
// complex64, row-major) | B operands of the block row, split and laid out per 32-column strip (4 planes x 32 x 32
// floats per strip) | Y, Rb (NR x N complex128 each)
__host__ __device__ inline size_t block_a_bytes(int N, int NR) {
  return ((size_t)N * (N + NR) * sizeof(float2) + 255) & ~(size_t)255;
}
__host__ __device__ inline int block_nblk(int N) { return (N + KB - 1) / KB; }
__host__ __device__ inline int block_nstrips(int N, int NR) {
  const int NC = N + NR;
  return NC > KB ? (NC - KB + KTN - 1) / KTN : 1;
}
__host__ __device__ inline size_t block_slot_bytes(int N, int NR) {
  return block_a_bytes(N, NR) + (size_t)block_nblk(N) * KB * KB * sizeof(float2) +
         (size_t)block_nstrips(N, NR) * 4 * KBP * sizeof(float) + 2 * (size_t)NR * N * sizeof(double2);
}

__device__ __forceinline__ void split4(float4 x, float4& h, float4& l) {
  h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
  l = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
}

// Stores four consecutive-k complex values (K positions k .. k+3 of `row`) as the four planes of an operand.
__device__ __forceinline__ void store_planes(float* planes, int plane_floats, int row, int k, float2 v0, float2 v1,
                                             float2 v2, float2 v3) {
  float4 h, l;
  const int o = kb_off(row, k);
  split4(make_float4(v0.x, v1.x, v2.x, v3.x), h, l);
  *reinterpret_cast<float4*>(planes + o) = h;
  *reinterpret_cast<float4*>(planes + plane_floats + o) = l;
  split4(make_float4(v0.y, v1.y, v2.y, v3.y), h, l);
  *reinterpret_cast<float4*>(planes + 2 * plane_floats + o) = h;
  *reinterpret_cast<float4*>(planes + 3 * plane_floats + o) = l;
}

// One half of the complex product of a 32-deep chunk, issued by one thread: part 0 the real accumulator d (Ar Br
// - Ai Bi), part 1 the imaginary one (Ar Bi + Ai Br).  The two parts go to different accumulators, so two threads
// issue them side by side (a single thread issues a tcgen05.mma only every ~50 cycles, while the tensor pipe takes
// an M = 128, N = 32 product every ~16).  Each of the four real products is the three-term split (lo hi + hi lo +
// hi hi), six MMAs per K step of 8.
//   issue_planar_part: A planes in shared memory, D = A B (the first product initialises d);
//   issue_planar_tmem_part: A planes in tensor memory (Re hi, Re lo, Im hi, Im lo at a_tm + 0, 32, 64, 96),
//   D -= A B.
__device__ __forceinline__ void issue_planar_part(uint32_t d, const float* a_pl, const float* b_pl, int part) {
  const uint32_t a0 = smem_u32(a_pl), b0 = smem_u32(b_pl);
  const uint32_t ar_h = a0, ar_l = a0 + KAP * 4, ai_h = a0 + 2 * KAP * 4, ai_l = a0 + 3 * KAP * 4;
  const uint32_t br_h = b0, br_l = b0 + KBP * 4, bi_h = b0 + 2 * KBP * 4, bi_l = b0 + 3 * KBP * 4;
  // part 0: (Ar, Br) +, (Ai, Bi) -;  part 1: (Ar, Bi) +, (Ai, Br) +
  const uint32_t b1h = part ? bi_h : br_h, b1l = part ? bi_l : br_l;
  const uint32_t b2h = part ? br_h : bi_h, b2l = part ? br_l : bi_l;
  const uint32_t s2 = part ? K_IDESC_POS : K_IDESC_NEG;
#pragma unroll
  for (int j = 0; j < KB / 8; ++j) {
    const uint32_t o = 256u * j;  // K step of 8 reals = two core matrices along K
    tc_mma_desc(d, ar_l + o, b1h + o, K_SBO, K_IDESC_POS, j > 0 ? 1u : 0u);
    tc_mma_desc(d, ar_h + o, b1l + o, K_SBO, K_IDESC_POS, 1u);
    tc_mma_desc(d, ar_h + o, b1h + o, K_SBO, K_IDESC_POS, 1u);
    tc_mma_desc(d, ai_l + o, b2h + o, K_SBO, s2, 1u);
    tc_mma_desc(d, ai_h + o, b2l + o, K_SBO, s2, 1u);
    tc_mma_desc(d, ai_h + o, b2h + o, K_SBO, s2, 1u);
  }
}

__device__ __forceinline__ void issue_planar_tmem_part(uint32_t d, uint32_t a_tm, const float* b_pl, int part) {
  const uint32_t b0 = smem_u32(b_pl);
  const uint32_t ar_h = a_tm, ar_l = a_tm + 32, ai_h = a_tm + 64, ai_l = a_tm + 96;
  const uint32_t br_h = b0, br_l = b0 + KBP * 4, bi_h = b0 + 2 * KBP * 4, bi_l = b0 + 3 * KBP * 4;
  // part 0: (Ar, Br) -, (Ai, Bi) +;  part 1: (Ar, Bi) -, (Ai, Br) -
  const uint32_t b1h = part ? bi_h : br_h, b1l = part ? bi_l : br_l;
  const uint32_t b2h = part ? br_h : bi_h, b2l = part ? br_l : bi_l;
  const uint32_t s2 = part ? K_IDESC_NEG : K_IDESC_POS;
#pragma unroll
  for (int j = 0; j < KB / 8; ++j) {
    const uint32_t o = 256u * j, t = 8u * j;  // K step of 8: 256 bytes of a shared plane, 8 TMEM columns
    tc_mma_tmem_a(d, ar_l + t, b1h + o, K_SBO, K_IDESC_NEG, 1u);
    tc_mma_tmem_a(d, ar_h + t, b1l + o, K_SBO, K_IDESC_NEG, 1u);
    tc_mma_tmem_a(d, ar_h + t, b1h + o, K_SBO, K_IDESC_NEG, 1u);
    tc_mma_tmem_a(d, ai_l + t, b2h + o, K_SBO, s2, 1u);
    tc_mma_tmem_a(d, ai_h + t, b2l + o, K_SBO, s2, 1u);
    tc_mma_tmem_a(d, ai_h + t, b2h + o, K_SBO, s2, 1u);
  }
}

// ----------------------------------------------------------------------------------------------
// Forming A (complex64, column-major) and the NR selector columns S[(p, nu)][s] = delta_ps
// ----------------------------------------------------------------------------------------------
// Element (i, j) as StructuredSource::element: (chi0^-1 [block diagonal] + Gamma / beta^2) + (-(U + V) / beta^2);
// a thread owns rows tid, tid + KT, tid + 2 KT of a pass (a warp reads 512 contiguous bytes of a Gamma column per
// load) with eight columns of Gamma loads in flight.
template <int NR>
__device__ __forceinline__ void block_form_a(const StructuredSource& src, const WorkItem& wi, int N, int nv, float2* __restrict__ A) {
  constexpr int RPT = 3, CPI = 4;  // rows per thread and pass, columns per iteration
  const int tid = threadIdx.x;
  const double2* gam = src.gamma_cm + ((size_t)(wi.ch * src.W + wi.w) * N) * N;
  const double2* c0 = src.chi0_inv + ((size_t)wi.q * src.W + wi.w) * nv * NR * NR;
  const double2* uvq = src.uv + ((size_t)wi.ch * src.Q + wi.q) * NR * NR;
  const double ib2 = src.inv_beta2;
  const uint64_t keep = l2_policy_evict_last();  // Gamma_r(w) is shared by every q of the (channel, w)
  for (int pass = 0; pass * RPT * KT < N; ++pass) {
    int ri[RPT], pr[RPT], vr[RPT];
    bool rok[RPT];
#pragma unroll
    for (int a = 0; a < RPT; ++a) {
      ri[a] = pass * RPT * KT + tid + a * KT;
      rok[a] = ri[a] < N;
      pr[a] = rok[a] ? ri[a] / nv : 0;
      vr[a] = rok[a] ? ri[a] - pr[a] * nv : 0;
    }
    if (!rok[0]) break;
    for (int j0 = 0; j0 < N; j0 += CPI) {
      // L2 prefetch of Gamma columns 8 iterations ahead (one bulk prefetch per column)
      if (tid < CPI && j0 + 8 * CPI + tid < N)
        bulk_prefetch_l2(gam + (size_t)(j0 + 8 * CPI + tid) * N, (uint32_t)(N * sizeof(double2)));
      double2 g[CPI][RPT];
#pragma unroll
      for (int u = 0; u < CPI; ++u)
#pragma unroll
        for (int a = 0; a < RPT; ++a)
          g[u][a] = (rok[a] && j0 + u < N) ? ld_d2_hint(gam + (size_t)(j0 + u) * N + ri[a], keep) : make_double2(0.0, 0.0);
#pragma unroll
      for (int u = 0; u < CPI; ++u) {
        const int j = j0 + u;
        if (j >= N) break;
        const int pc = j / nv, vc = j - pc * nv;
#pragma unroll
        for (int a = 0; a < RPT; ++a) {
          if (!rok[a]) continue;
          const double2 uu = uvq[pr[a] * NR + pc];
          double re = __dmul_rn(g[u][a].x, ib2);
          double im = __dmul_rn(g[u][a].y, ib2);
          if (vr[a] == vc) {
            const double2 c = c0[(size_t)vr[a] * NR * NR + pr[a] * NR + pc];
            re = __dadd_rn(c.x, re);
            im = __dadd_rn(c.y, im);
          }
          re = __dadd_rn(re, -__dmul_rn(uu.x, ib2));
          im = __dadd_rn(im, -__dmul_rn(uu.y, ib2));
          A[(size_t)j * N + ri[a]] = make_float2((float)re, (float)im);
        }
      }
    }
#pragma unroll
    for (int a = 0; a < RPT; ++a)
      if (rok[a])
        for (int r = 0; r < NR; ++r) A[(size_t)(N + r) * N + ri[a]] = make_float2(pr[a] == r ? 1.f : 0.f, 0.f);
  }
}

// ----------------------------------------------------------------------------------------------
// D_k^-1 by Gauss-Jordan elimination of [D | I] with the pivot search inside the block, by the whole CTA: lane =
// row, warp w owns the 16 columns w + 8t of the 64 (8 of D, 8 of I).  Per pivot step: the owner warp of column jj
// finds the pivot (largest |re| + |im|, ties to the smaller row, NaN no candidate); every thread reads the old
// values it needs; then writes row jj <- (old row p) / pivot and row i <- (old row i, or old row jj for i = p) -
// f_i (new row jj).  aug: [64][K_DLD] column-major workspace; sp: {p, ok} and the pivot value, shared.
// Writes D^-1 row-major to s.dinv (ld K_DLD) and inv (ld 32), zero outside the nb x nb block.  Returns false
// (in every thread) if a pivot column was exactly zero or not finite.
// ----------------------------------------------------------------------------------------------
__device__ __forceinline__ bool block_diag_inverse(const float2* __restrict__ A, int N, int k0, int nb, float2* aug, float2* dinv,
                                   float2* __restrict__ inv, int* sp, float2* sd) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < 2 * KB / KW; ++t) {
    const int c = warp + KW * t;  // t < 4: columns of D, t >= 4: columns of I
    float2 x;
    if (c < KB)
      x = (c < nb && lane < nb) ? __ldcg(A + (size_t)(k0 + c) * N + k0 + lane) : make_float2(c == lane ? 1.f : 0.f, 0.f);
    else
      x = make_float2(c - KB == lane ? 1.f : 0.f, 0.f);
    aug[c * K_DLD + lane] = x;
  }
  if (threadIdx.x == 0) sp[1] = 1;
  __syncthreads();
  for (int jj = 0; jj < nb; ++jj) {
    if (warp == (jj & (KW - 1))) {
      float v = (lane >= jj && lane < nb) ? cabs1(aug[jj * K_DLD + lane]) : -1.f;
      const bool cand = v >= 0.f;
      const unsigned key = cand ? __float_as_uint(v) : 0u;
      const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
      const unsigned imin = __reduce_min_sync(0xffffffffu, (cand && key == kmax) ? (unsigned)lane : 0x7fffffffu);
      v = __uint_as_float(kmax);
      int p = (int)imin;
      const bool good = (v > 0.f) && isfinite(v) && p >= jj && p < nb;
      if (!good) p = jj;
      if (lane == 0) {
        sp[0] = p;
        if (!good) sp[1] = 0;
        *sd = good ? aug[jj * K_DLD + p] : make_float2(0.f, 0.f);
      }
    }
    __syncthreads();
    const int p = sp[0];
    const float2 d = *sd;
    const float2 rinv = (d.x != 0.f || d.y != 0.f) ? crecip(d) : make_float2(0.f, 0.f);
    // old values: this row (row jj's for i = p), the factor in column jj, the new pivot row
    const int i = lane;
    const int src = (i == p) ? jj : i;
    const float2 f = (i == jj) ? make_float2(0.f, 0.f) : aug[jj * K_DLD + src];
    float2 old[2 * KB / KW], prow[2 * KB / KW];
#pragma unroll
    for (int t = 0; t < 2 * KB / KW; ++t) {
      const int c = warp + KW * t;
      old[t] = aug[c * K_DLD + src];
      prow[t] = cmul(aug[c * K_DLD + p], rinv);
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < 2 * KB / KW; ++t) {
      const int c = warp + KW * t;
      float2 x = prow[t];
      if (i != jj) {
        x = old[t];
        cfms(x, f, prow[t]);
      }
      aug[c * K_DLD + i] = x;
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < KB * KB; e += KT) {
    const int r = e >> 5, k = e & 31;
    const float2 x = (r < nb && k < nb) ? aug[(KB + k) * K_DLD + r] : make_float2(0.f, 0.f);
    dinv[r * K_DLD + k] = x;
    inv[r * KB + k] = x;
  }
  const bool ok = sp[1] != 0;
  __syncthreads();
  return ok;
}

// ----------------------------------------------------------------------------------------------
// Tile waits (bounded) and the drain at exit
// ----------------------------------------------------------------------------------------------
// A completion is counted only when this thread saw it; a wait that runs out (or is skipped because another
// thread's ran out) leaves the phase outstanding for the drain at exit.  The result is made warp-uniform, since
// the TMEM loads that follow are warp-collective.
__device__ __forceinline__ bool tile_wait(BlockSmem& s, TileCount& tc, int b) {
  bool ok = false;
  if (s.misc[0] == 0) ok = mbar_wait_sleep(s.bar + b, (tc.par >> b) & 1u, s.wait_limit, K_WAIT_HINT_NS);
  if (ok) tc.observed(b);
  ok = __all_sync(0xffffffffu, ok);
  if (!ok) s.misc[0] = 1;
  return ok;
}

// ----------------------------------------------------------------------------------------------
// Split planes of the block row A[k0:k1, k1:NC] per 32-column strip, in bop (the B operands of the trailing tiles):
// plane element (c, k) = A[k0 + k][k1 + 32 st + c]; zero beyond the row's columns.  Two threads per column, each a
// 128-byte run of it.
// ----------------------------------------------------------------------------------------------
__device__ __forceinline__ void block_row_planes(const float2* __restrict__ A, int N, int NC, int k0, int k1, float* __restrict__ bop) {
  const int ncols = NC - k1;
  if (ncols <= 0 || k1 >= N) return;
  const int nst = (ncols + KTN - 1) / KTN;
  for (int e = threadIdx.x; e < nst * KTN * 2; e += KT) {
    const int jl = e >> 1, h = e & 1, j = k1 + jl;
    const int st = jl >> 5, c = jl & 31;
    float* sp = bop + (size_t)st * 4 * KBP;
    const float4* col = reinterpret_cast<const float4*>(A + (size_t)j * N + k0 + 16 * h);
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      float4 x0 = make_float4(0.f, 0.f, 0.f, 0.f), x1 = x0;
      if (j < NC) {
        x0 = __ldcg(col + 2 * g);
        x1 = __ldcg(col + 2 * g + 1);
      }
      store_planes(sp, KBP, c, 16 * h + 4 * g, make_float2(x0.x, x0.y), make_float2(x0.z, x0.w),
                   make_float2(x1.x, x1.y), make_float2(x1.z, x1.w));
    }
  }
}

// ----------------------------------------------------------------------------------------------
// Trailing update (below): L' in tensor memory, strips of C and B by bulk copy, two strips in flight.
// ----------------------------------------------------------------------------------------------
// Hint to bring the C tile A[r0 : r0 + 128, c0 : c0 + 32] into L2 (one prefetch per column, by one warp).
__device__ __forceinline__ void prefetch_tile_l2(const float2* A, int N, int NC, int r0, int c0) {
  const int lane = threadIdx.x & 31;
  const int c = c0 + lane;
  if (c >= NC || r0 >= N) return;
  const int r1 = min(N, r0 + KTM);
  const uintptr_t a = reinterpret_cast<uintptr_t>(A + (size_t)c * N + r0) & ~(uintptr_t)15;
  const uintptr_t e = (reinterpret_cast<uintptr_t>(A + (size_t)c * N + r1) + 15) & ~(uintptr_t)15;
  bulk_prefetch_l2(reinterpret_cast<const void*>(a), (uint32_t)(e - a));
}

// L' = A[r0 : r0 + 128, kc : kc + 32] D^-1 on the tensor cores (D^-1 row-major in global memory, dinv), into TMEM
// buffer 0, then split into the tensor-memory A operand planes (Re hi, Re lo, Im hi, Im lo at columns K_A_COL + 0,
// 32, 64, 96 of the CTA's allocation).  Stages A21 in the shared A planes and D^-1 in B buffer 1; every thread takes
// part; ends with a barrier.
__device__ __forceinline__ void block_l21(const float2* __restrict__ A, int N, int r0, int kc, const float2* __restrict__ dinv,
                          BlockSmem& s, TileCount& tc) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t tbase = *s.tslot;
  const uint32_t tl = tbase + ((uint32_t)(32 * (warp & 3)) << 16);
  const int hh = warp >> 2;
  {  // A planes: rows r0 .. r0 + 127 of the block column (16 k per thread, loads coalesced along the rows)
    const int rl = tid & (KTM - 1), h = tid >> 7, r = r0 + rl;
    const bool rok = r < N;
    float2 v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) v[u] = rok ? __ldcg(A + (size_t)(kc + 16 * h + u) * N + r) : make_float2(0.f, 0.f);
#pragma unroll
    for (int g = 0; g < 4; ++g) store_planes(s.a_pl, KAP, rl, 16 * h + 4 * g, v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3]);
  }
  // B planes of D^-1: element (i, k) = D^-1[k][i], so that the product below is A21 D^-1
  for (int e = tid; e < KB * (KB / 4); e += KT) {
    const int i = e >> 3, k = (e & 7) * 4;
    store_planes(s.b_pl + 4 * KBP, KBP, i, k, __ldcg(dinv + k * KB + i), __ldcg(dinv + (k + 1) * KB + i),
                 __ldcg(dinv + (k + 2) * KB + i), __ldcg(dinv + (k + 3) * KB + i));
  }
  tc_fence_async_smem();
  tc_fence_before();
  __syncthreads();
  const bool live = s.misc[0] == 0;
  if (live && (tid == 0 || tid == 32)) {  // real part by thread 0, imaginary part by thread 32
    const int part = tid >> 5;
    tc_fence_after();
    issue_planar_part(tbase + 32 * part, s.a_pl, s.b_pl + 4 * KBP, part);
    tc_commit(s.bar + 1);
  }
  if (live) tc.issued(1);
  const bool ok = live && tile_wait(s, tc, 1);
  tc_fence_after();
  if (ok) {
    float re[16], im[16];
    tmem_ld16(tl + 16 * hh, re);
    tmem_ld16(tl + 32 + 16 * hh, im);
    tmem_wait_ld();
    float rh[16], rlo[16], ih[16], il[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      rh[j] = tf32_hi(re[j]);
      rlo[j] = re[j] - rh[j];
      ih[j] = tf32_hi(im[j]);
      il[j] = im[j] - ih[j];
    }
    const uint32_t a2 = tl + K_A_COL + 16 * hh;
    tmem_st16(a2, rh);
    tmem_st16(a2 + 32, rlo);
    tmem_st16(a2 + 64, ih);
    tmem_st16(a2 + 96, il);
    tmem_wait_st();
  }
  tc_fence_before();
  __syncthreads();
}

// Bulk copies (issued by one warp) of a strip pair's operands, strips st and st + 1 (if it exists) into buffers 0
// and 1: the C tiles A[r0 : r0 + rows, c0 : c0 + 32] (one copy of rows x 8 bytes per column inside the matrix,
// column-major in cbuf) on barrier 2, and the block row's B planes (16 KB per strip, one copy) on barrier 3.  rows
// and r0 are even and N is even, so every copy starts on a 16-byte boundary and moves a multiple of 16 bytes.
__device__ __forceinline__ void copy_c_pair(const float2* __restrict__ A, int N, int NC, int r0, int rows, int c0,
                                            BlockSmem& s) {
  const int lane = threadIdx.x & 31;
  const int ncols = min(2 * KTN, NC - c0);
  if (lane == 0) mbar_expect_tx(s.bar + 2, (uint32_t)(ncols * rows) * (uint32_t)sizeof(float2));
  __syncwarp();
  const uint64_t pol = l2_policy_evict_first();  // the slot's matrix streams through L2
  for (int c = lane; c < ncols; c += 32)
    bulk_g2s_hint(s.cbuf + (size_t)c * KTM, A + (size_t)(c0 + c) * N + r0, (uint32_t)(rows * sizeof(float2)), s.bar + 2,
                  pol);
}
__device__ __forceinline__ void copy_b_pair(const float* __restrict__ bsrc, int nstrips, BlockSmem& s) {
  if ((threadIdx.x & 31) == 0) {
    mbar_expect_tx(s.bar + 3, (uint32_t)(nstrips * 4 * KBP * sizeof(float)));
    bulk_g2s(s.b_pl, bsrc, (uint32_t)(nstrips * 4 * KBP * sizeof(float)), s.bar + 3);
  }
}

// Trailing update A[k1:N, k1:NC] -= (A[k1:N, k0:k1] D^-1) A[k0:k1, k1:NC]: per 128-row block, L' goes to the
// tensor-memory A operand; then its 32-column strips go two at a time.  A strip pair's C tiles and B planes arrive
// by bulk copy; all eight warps move the C tiles into tensor memory (warp w: TMEM lanes 32 (w % 4) .., tile w / 4);
// threads 0, 32, 64, 96 issue the real and imaginary halves of the two tiles' products (a single thread issues a
// tcgen05.mma only every ~50 cycles or more, so the products of a pair go out four at a time); once they have
// completed, the next pair's B planes are copied in (its C tiles went out as soon as this pair's had moved on) and
// all warps move the results back to A.  The second CTA on the SM fills the tensor pipe while this one moves tiles.
__device__ __forceinline__ void block_trailing(float2* __restrict__ A, int N, int NC, int k0, int k1, BlockSmem& s,
                                               const float* __restrict__ bop, const float2* __restrict__ dinv,
                                               TileCount& tc) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (k1 >= N) return;
  const int nrb = (N - k1 + KTM - 1) / KTM, nst = (NC - k1 + KTN - 1) / KTN, npair = (nst + 1) / 2;
  const uint32_t tbase = *s.tslot;
  const uint32_t tl = tbase + ((uint32_t)(32 * (warp & 3)) << 16);
  const int row_t = 32 * (warp & 3) + lane;  // this thread's tile row (its TMEM lane)
  const int tile = warp >> 2;                // the tile of the pair this warp moves
  constexpr int COPIER = KW - 1;
  for (int rb = 0; rb < nrb; ++rb) {
    const int r0 = k1 + rb * KTM, rows = min(KTM, N - r0);
    block_l21(A, N, r0, k0, dinv, s, tc);  // every product of the previous row block has completed
    if (s.misc[0] == 0) {
      if (warp == COPIER) {
        copy_c_pair(A, N, NC, r0, rows, k1, s);
        copy_b_pair(bop, min(2, nst), s);
      }
      tc.issued(2);
      tc.issued(3);
    }
    for (int p = 0; p < npair; ++p) {
      const int st = 2 * p + tile, c0 = k1 + st * KTN;
      const bool has = st < nst;  // this warp's tile exists (the last pair may hold one strip)
      if (warp == KW - 2 && 2 * p + 4 < nst) {
        prefetch_tile_l2(A, N, NC, r0, k1 + (2 * p + 4) * KTN);
        if (2 * p + 5 < nst) prefetch_tile_l2(A, N, NC, r0, k1 + (2 * p + 5) * KTN);
      }
      if (tile_wait(s, tc, 2) && has) {  // C tile -> TMEM: row row_t, 32 complex columns
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const float2* cb = s.cbuf + (size_t)(tile * KTN + 16 * hh) * KTM + row_t;
          float re[16], im[16];
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) {
            const float2 x = cb[jj * KTM];
            re[jj] = x.x;
            im[jj] = x.y;
          }
          tmem_st16(tl + 64 * tile + 16 * hh, re);
          tmem_st16(tl + 64 * tile + 32 + 16 * hh, im);
        }
        tmem_wait_st();
      }
      tile_wait(s, tc, 3);
      tc_fence_before();
      __syncthreads();
      const bool live = s.misc[0] == 0;
      if (live) {
        if (tid < 128 && lane == 0) {  // threads 0, 32, 64, 96: tile tid / 64, part (tid / 32) % 2
          const int t = tid >> 6, part = (tid >> 5) & 1;
          if (2 * p + t < nst) {
            tc_fence_after();
            issue_planar_tmem_part(tbase + 64 * t + 32 * part, tbase + K_A_COL, s.b_pl + t * 4 * KBP, part);
            tc_commit(s.bar);
          } else {
            mbar_arrive(s.bar);
          }
        }
        tc.issued(0);
        // the pair's C buffers have moved on: the next pair's C tiles go out now
        if (p + 1 < npair) {
          if (warp == COPIER) copy_c_pair(A, N, NC, r0, rows, k1 + (2 * p + 2) * KTN, s);
          tc.issued(2);
        }
        const bool done = tile_wait(s, tc, 0);
        tc_fence_after();
        // the products have completed: the next pair's B planes go out, then the results go back to A
        if (p + 1 < npair) {
          if (warp == COPIER && done) copy_b_pair(bop + (size_t)(2 * p + 2) * 4 * KBP, min(2, nst - 2 * p - 2), s);
          tc.issued(3);
        }
        if (done && has) {
          const int r = r0 + row_t;
          const uint64_t pol = l2_policy_evict_first();
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            float re[16], im[16];
            tmem_ld16(tl + 64 * tile + 16 * hh, re);
            tmem_ld16(tl + 64 * tile + 32 + 16 * hh, im);
            tmem_wait_ld();
            const int cb = c0 + 16 * hh;
            if (r < N) {
#pragma unroll
              for (int jj = 0; jj < 16; ++jj)
                if (cb + jj < NC) st_f2_hint(A + (size_t)(cb + jj) * N + r, make_float2(re[jj], im[jj]), pol);
            }
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------------------------
// Triangular solves with the block factors for NR right-hand sides y[r * ldy + i] in shared memory: with
// `forward` the full solve (L then U), else the back substitution alone (the selector columns already hold L^-1 S).
//   forward sweep (L y = r):  for each block b: z_b = D_b^-1 y_b (warp per right-hand side, lane = row, into zb),
//                             then the rows below y_i -= A[i, b] z_b (thread per row);
//   back substitution (U x = y): for each block b from the last: y_b <- D_b^-1 y_b, then the rows above
//                             y_i -= A[i, b] y_b.
// The inverse of the next block is staged into sinv (double buffered) during each update.
// ----------------------------------------------------------------------------------------------
template <int NR>
__device__ __forceinline__ void block_solve(const float2* __restrict__ A, int N, float2* y, int ldy, const float2* __restrict__ inv,
                            float2* sinv, float2* zb, bool forward) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = block_nblk(N);
  // rows [i0, i1): y_i -= sum_k A[i][k0 + k] v[r][k], v = y + k0 (backward) or zb (forward)
  auto update = [&](int k0, int nb, int i0, int i1, const float2* v, int ldv) {
    for (int i = i0 + tid; i < i1; i += KT) {
      float2 acc[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) acc[r] = y[(size_t)r * ldy + i];
      for (int k = 0; k < nb; k += 16) {
        float2 l[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) l[u] = (k + u < nb) ? __ldcg(A + (size_t)(k0 + k + u) * N + i) : make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 16; ++u)
          if (k + u < nb) {
#pragma unroll
            for (int r = 0; r < NR; ++r) cfms(acc[r], l[u], v[(size_t)r * ldv + k + u]);
          }
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) y[(size_t)r * ldy + i] = acc[r];
    }
  };
  // one sweep over the blocks: fwd = forward elimination (L), else back substitution (U)
  // L2 prefetch of the column panel of block bb that a sweep's update reads: rows below it (forward) or above it
  auto prefetch_panel = [&](int bb, bool fwd) {
    if (warp != KW - 1) return;
    const int p0 = bb * KB, pn = min(KB, N - p0);
    const int rlo = fwd ? p0 + pn : 0, rhi = fwd ? N : p0;
    if (lane < pn && rhi > rlo)
      bulk_prefetch_l2(A + (size_t)(p0 + lane) * N + rlo, (uint32_t)((rhi - rlo) * sizeof(float2)));
  };
  auto sweep = [&](bool fwd) {
    auto blk = [&](int st) { return fwd ? st : nblk - 1 - st; };
    prefetch_panel(blk(0), fwd);
    for (int e = tid; e < KB * KB; e += KT) sinv[(e >> 5) * K_DLD + (e & 31)] = inv[(size_t)blk(0) * KB * KB + e];
    __syncthreads();
    for (int st = 0; st < nblk; ++st) {
      const int b = blk(st);
      const int k0 = b * KB, nb = min(KB, N - k0), k1 = k0 + nb;
      const float2* sv = sinv + (st & 1) * KB * K_DLD;
      if (st + 1 < nblk) prefetch_panel(blk(st + 1), fwd);
      for (int r = warp; r < NR; r += KW) {  // D_b^-1 y_b
        float2* yr = y + (size_t)r * ldy + k0;
        float2 acc = make_float2(0.f, 0.f);
        for (int k = 0; k < nb; ++k) cfma(acc, sv[lane * K_DLD + k], yr[k]);
        if (fwd) {
          zb[r * KB + lane] = acc;
        } else {
          __syncwarp();
          if (lane < nb) yr[lane] = acc;
        }
      }
      float2 nx[KB * KB / KT];
      if (st + 1 < nblk) {
#pragma unroll
        for (int u = 0; u < KB * KB / KT; ++u) nx[u] = inv[(size_t)blk(st + 1) * KB * KB + tid + u * KT];
      }
      __syncthreads();
      if (fwd) update(k0, nb, k1, N, zb, KB);
      else update(k0, nb, 0, k0, y + k0, ldy);
      if (st + 1 < nblk) {
        float2* dst = sinv + ((st + 1) & 1) * KB * K_DLD;
#pragma unroll
        for (int u = 0; u < KB * KB / KT; ++u) {
          const int e = tid + u * KT;
          dst[(e >> 5) * K_DLD + (e & 31)] = nx[u];
        }
      }
      __syncthreads();
    }
  };
  if (forward) sweep(true);
  sweep(false);
}

// ----------------------------------------------------------------------------------------------
// One work item: form, factor, solve, refine.  Returns the status bits; *iters = number of corrections.
// ----------------------------------------------------------------------------------------------
template <int NR>
__device__ __forceinline__ int solve_item_block(const StructuredSource& src, const WorkItem& wi, int N, int nv, double beta,
                                int max_iter, double tol, double2* __restrict__ o, unsigned char* slot, BlockSmem& s,
                                TileCount& tc, int* iters) {
  const int tid = threadIdx.x;
  const int NC = N + NR;
  float2* A = reinterpret_cast<float2*>(slot);
  float2* inv = reinterpret_cast<float2*>(slot + block_a_bytes(N, NR));
  float* bop = reinterpret_cast<float*>(inv + (size_t)block_nblk(N) * KB * KB);
  double2* Y = reinterpret_cast<double2*>(bop + (size_t)block_nstrips(N, NR) * 4 * KBP);
  double2* Rb = Y + (size_t)N * NR;
  if (tid == 0) {
    s.misc[1] = 0;
    s.misc[2] = 0;
  }
  block_form_a<NR>(src, wi, N, nv, A);
  __syncthreads();
  // ---- factorisation ----
  for (int k0 = 0; k0 < N; k0 += KB) {
    const int nb = min(KB, N - k0), k1 = k0 + nb;
    {  // the block reductions' scratch holds the pivot step's broadcast here
      const bool ok = block_diag_inverse(A, N, k0, nb, reinterpret_cast<float2*>(s.a_pl), s.dinv,
                                         inv + (size_t)(k0 / KB) * KB * KB, reinterpret_cast<int*>(s.redd),
                                         reinterpret_cast<float2*>(s.redd + 2));
      if (!ok && threadIdx.x == 0) s.misc[2] = 1;
    }
    __syncthreads();
    block_row_planes(A, N, NC, k0, k1, bop);
    __syncthreads();
    block_trailing(A, N, NC, k0, k1, s, bop, inv + (size_t)(k0 / KB) * KB * KB, tc);
  }
  __syncthreads();
  // ---- initial solve: the selector columns hold the forward result L^-1 S; back substitution only ----
  const int ldy = N;
  for (int e = tid; e < NR * N; e += KT) s.y[e] = A[(size_t)N * N + e];
  __syncthreads();
  block_solve<NR>(A, N, s.y, ldy, inv, s.sinv, s.zb, false);
  double prev = 0.0;
  for (int e = tid; e < NR * N; e += KT) {
    Y[e] = make_double2(s.y[e].x, s.y[e].y);
    prev = fmax(prev, (double)fmaxf(fabsf(s.y[e].x), fabsf(s.y[e].y)));
  }
  prev = block_max(prev, s.redd);
  int it = 0;
  bool converged = false;
  for (; it < max_iter; ++it) {
    structured_residual_permuted<NR>(src, wi.ch, wi.q, wi.w, N, nv, Y, Rb, nullptr, s.colsum, s.ys);
    for (int e = tid; e < NR * N; e += KT) s.y[e] = make_float2((float)Rb[e].x, (float)Rb[e].y);
    __syncthreads();
    block_solve<NR>(A, N, s.y, ldy, inv, s.sinv, s.zb, true);
    double dmax = 0.0, ymax = 0.0;
    for (int e = tid; e < NR * N; e += KT) {
      const double2 d = make_double2(s.y[e].x, s.y[e].y);
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
  __syncthreads();
  bool bad = false;
  for (int e = tid; e < N * NR; e += KT) {
    const int i = e / NR, r = e - i * NR;
    double2 v = Y[(size_t)r * N + i];
    v.x = v.x / beta;
    v.y = v.y / beta;
    if (!cfinite(v)) bad = true;
    o[e] = v;
  }
  if (bad) atomicOr(&s.misc[1], DGA_ITEM_NONFINITE);
  __syncthreads();
  // a singular diagonal block is no proof of a singular matrix: such items go to the FP64 re-solve (with partial
  // pivoting), which reports DGA_ITEM_SINGULAR if the matrix itself is
  const int st = s.misc[1] | ((converged && !s.misc[2]) ? 0 : DGA_ITEM_NOCONVERGE) |
                 (s.misc[0] ? DGA_ITEM_WAIT_TIMEOUT : 0);
  *iters = it;
  __syncthreads();
  return st;
}

__device__ __forceinline__ void block_kernel_begin(BlockSmem& s) {
  if (threadIdx.x == 0) {
    s.misc[0] = 0;
#pragma unroll
    for (int b = 0; b < K_NBAR; ++b) mbar_init(s.bar + b, b == 0 ? 4u : b == 1 ? 2u : 1u);  // issuing threads
    if (s.inject) mbar_init(s.probe);
  }
  if ((threadIdx.x >> 5) == 0) tc_alloc(s.tslot, K_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (s.inject) {
    // test hook (dga_bse_tuning.wait_limit < 0): a bounded wait on a phase that nothing completes runs out, and
    // the CTA takes the path of a real timeout
    if (!mbar_wait(s.probe, 0u, s.inject)) s.misc[0] = 1;
    __syncthreads();
  }
}

// Drains every tile still in flight (full limit) and frees TMEM; false if a drain wait ran out.
__device__ __forceinline__ bool block_kernel_end(BlockSmem& s, const TileCount& tc) {
  tc_fence_before();
  __syncthreads();
  bool drained = true;
#pragma unroll
  for (int b = 0; b < K_NBAR; ++b)
    if ((tc.pend >> b) & 1u) drained &= mbar_wait(s.bar + b, (tc.par >> b) & 1u);
  tc_fence_after();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc_dealloc(*s.tslot, K_TMEM_COLS);
  return __syncthreads_and(drained ? 1 : 0) != 0;
}

template <int NR>
__global__ void __launch_bounds__(KT, 2)
    bse_block_mixed_kernel(StructuredSource src, const WorkItem* __restrict__ work, int n_items, int N, int nv, int W,
                           int Q, double beta, int max_iter, double tol, double2* __restrict__ out,
                           int* __restrict__ status, int* __restrict__ iters, unsigned char* __restrict__ scratch,
                           size_t slot_bytes, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  BlockSmem s(smem_raw, N, NR, wait_limit);
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  TileCount tc;
  block_kernel_begin(s);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (s.misc[0]) {  // a wait ran out: the CTA issues nothing more, its remaining items go to the FP64 re-solve
      if (threadIdx.x == 0) {
        if (status) status[item] = DGA_ITEM_WAIT_TIMEOUT;
        if (iters) iters[item] = 0;
      }
      continue;
    }
    const WorkItem wi = work[item];
    double2* o = out + (((size_t)wi.ch * Q + wi.q) * W + wi.w) * (size_t)N * NR;
    int it = 0;
    const int st = solve_item_block<NR>(src, wi, N, nv, beta, max_iter, tol, o, slot, s, tc, &it);
    if (threadIdx.x == 0) {
      if (status) status[item] = st;
      if (iters) iters[item] = it;
    }
  }
  if (!block_kernel_end(s, tc) && status) {
    for (int item = blockIdx.x + threadIdx.x * gridDim.x; item < n_items; item += blockDim.x * gridDim.x)
      atomicOr(status + item, DGA_ITEM_WAIT_TIMEOUT);
  }
}

// Batches (see bse_multi_kernel in bse.cu): each item reads its request's descriptor; shared memory and the
// scratch slot are sized for the largest request of the launch.  bse_block_multi_kernel<NR> takes one orbital
// count; bse_block_multi_any_kernel chooses the right-hand-side count per item (orbital counts 1 to 3).
template <int NR>
__device__ __forceinline__ void block_batch_item(const dga_bse_problem& d, const MultiItem& mi, int max_iter,
                                                 double tol, unsigned char* slot, unsigned char* smem_raw,
                                                 long long wait_limit, TileCount& tc, int* st, int* it) {
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
  BlockSmem s(smem_raw, N, NR, wait_limit);  // the same shared memory, solve-phase offsets for this N
  const WorkItem wi{mi.ch, mi.q, mi.w};
  double2* o = (double2*)d.out + (((size_t)wi.ch * src.Q + wi.q) * src.W + wi.w) * (size_t)N * NR;
  *st = solve_item_block<NR>(src, wi, N, src.nv, d.beta, max_iter, tol, o, slot, s, tc, it);
}

template <int NR>
__global__ void __launch_bounds__(KT, 2)
    bse_block_multi_kernel(const dga_bse_problem* __restrict__ probs, const MultiItem* __restrict__ work,
                           int n_items, int n_max, int max_iter, double tol, int* __restrict__ status,
                           int* __restrict__ iters, unsigned char* __restrict__ scratch, size_t slot_bytes,
                           long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  BlockSmem s0(smem_raw, n_max, NR, wait_limit);
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  TileCount tc;
  block_kernel_begin(s0);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (s0.misc[0]) {
      if (threadIdx.x == 0) {
        status[item] = DGA_ITEM_WAIT_TIMEOUT;
        if (iters) iters[item] = 0;
      }
      continue;
    }
    const MultiItem mi = work[item];
    int st = 0, it = 0;
    block_batch_item<NR>(probs[mi.prob], mi, max_iter, tol, slot, smem_raw, wait_limit, tc, &st, &it);
    if (threadIdx.x == 0) {
      status[item] = st;
      if (iters) iters[item] = it;
    }
  }
  if (!block_kernel_end(s0, tc)) {
    for (int item = blockIdx.x + threadIdx.x * gridDim.x; item < n_items; item += blockDim.x * gridDim.x)
      atomicOr(status + item, DGA_ITEM_WAIT_TIMEOUT);
  }
}

__global__ void __launch_bounds__(KT, 2)
    bse_block_multi_any_kernel(const dga_bse_problem* __restrict__ probs, const MultiItem* __restrict__ work,
                               int n_items, int n_max, int max_iter, double tol, int* __restrict__ status,
                               int* __restrict__ iters, unsigned char* __restrict__ scratch, size_t slot_bytes,
                               long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  BlockSmem s0(smem_raw, n_max, 1, wait_limit);
  unsigned char* slot = scratch + (size_t)blockIdx.x * slot_bytes;
  TileCount tc;
  block_kernel_begin(s0);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (s0.misc[0]) {
      if (threadIdx.x == 0) {
        status[item] = DGA_ITEM_WAIT_TIMEOUT;
        if (iters) iters[item] = 0;
      }
      continue;
    }
    const MultiItem mi = work[item];
    const dga_bse_problem d = probs[mi.prob];
    int st = 0, it = 0;
    switch (d.n_orb) {
      case 1: block_batch_item<1>(d, mi, max_iter, tol, slot, smem_raw, wait_limit, tc, &st, &it); break;
      case 2: block_batch_item<4>(d, mi, max_iter, tol, slot, smem_raw, wait_limit, tc, &st, &it); break;
      default: block_batch_item<9>(d, mi, max_iter, tol, slot, smem_raw, wait_limit, tc, &st, &it); break;
    }
    if (threadIdx.x == 0) {
      status[item] = st;
      if (iters) iters[item] = it;
    }
  }
  if (!block_kernel_end(s0, tc)) {
    for (int item = blockIdx.x + threadIdx.x * gridDim.x; item < n_items; item += blockDim.x * gridDim.x)
      atomicOr(status + item, DGA_ITEM_WAIT_TIMEOUT);
  }
}

}  // namespace dga

using namespace dga;

// ----------------------------------------------------------------------------------------------
// Host side (called from bse.cu)
// ----------------------------------------------------------------------------------------------
bool dga_block_supported(int N, int n2) {
  if (!(n2 == 1 || n2 == 4 || n2 == 9 || n2 == 16) || N <= 0 || N > 2048) return false;
  return block_solve_bytes(N, n2) <= (size_t)K_REGION;
}

size_t dga_block_slot_bytes(int N, int n2) { return (block_slot_bytes(N, n2) + 255) & ~(size_t)255; }

// Two CTAs per SM need the whole shared-memory carve-out of the SM's unified L1/shared storage.
template <int NR>
static void block_set_attributes() {
  cudaFuncSetAttribute(bse_block_mixed_kernel<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)block_smem_bytes());
  cudaFuncSetAttribute(bse_block_mixed_kernel<NR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(bse_block_multi_kernel<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)block_smem_bytes());
  cudaFuncSetAttribute(bse_block_multi_kernel<NR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
}

template <int NR>
static int block_ctas_per_sm_nr();

template <int NR>
static int block_grid_nr(int n_items) {
  int per_sm = block_ctas_per_sm_nr<NR>();
  if (per_sm < 1) per_sm = 1;
  const int g = device_sm_count() * per_sm;
  return n_items < g ? n_items : g;
}

// Resident CTAs per SM from the kernel's registers and shared memory (two at most: two CTAs hold 256 of the SM's
// 512 TMEM columns).  Computed here rather than by cudaOccupancyMaxActiveBlocksPerMultiprocessor, which answers 1
// for this kernel although its register and shared-memory limits both allow 2 (as the profiler's occupancy
// section reports).
template <int NR>
static int block_ctas_per_sm_nr() {
  block_set_attributes<NR>();
  cudaFuncAttributes fa;
  int dev = 0, regs_sm = 0, smem_sm = 0, reserved = 0;
  if (cudaFuncGetAttributes(&fa, bse_block_mixed_kernel<NR>) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess)
    return -1;
  const long long regs_cta = (long long)((fa.numRegs + 7) / 8 * 8) * KT;
  const long long smem_cta = (long long)block_smem_bytes() + fa.sharedSizeBytes + reserved;
  long long per_sm = 2;
  if (regs_cta * per_sm > regs_sm) per_sm = regs_sm / regs_cta;
  if (smem_cta * per_sm > smem_sm) per_sm = smem_sm / smem_cta;
  return per_sm < 1 ? 1 : (int)per_sm;
}

// Resident CTAs per SM of the block-form kernel for n2 right-hand sides (the occupancy the launch gets).
extern "C" int dga_bse_block_ctas_per_sm(int n2) {
  switch (n2) {
    case 1: return block_ctas_per_sm_nr<1>();
    case 4: return block_ctas_per_sm_nr<4>();
    case 9: return block_ctas_per_sm_nr<9>();
    case 16: return block_ctas_per_sm_nr<16>();
    default: return -1;
  }
}

// Loads every block-form kernel now (CUDA loads a kernel's code at its first launch otherwise, which can take tens
// of milliseconds for these): cudaFuncGetAttributes brings each function in.
int dga_block_preload() {
  cudaFuncAttributes fa;
  int bad = 0;
  bad |= cudaFuncGetAttributes(&fa, bse_block_multi_any_kernel) != cudaSuccess;
#define DGA_BLOCK_LOAD(R)                                                               \
  bad |= cudaFuncGetAttributes(&fa, bse_block_mixed_kernel<R>) != cudaSuccess;          \
  bad |= cudaFuncGetAttributes(&fa, bse_block_multi_kernel<R>) != cudaSuccess;
  DGA_BLOCK_LOAD(1)
  DGA_BLOCK_LOAD(4)
  DGA_BLOCK_LOAD(9)
  DGA_BLOCK_LOAD(16)
#undef DGA_BLOCK_LOAD
  return bad;
}

// n2 = 0: the batch kernel that chooses the right-hand-side count per item (same launch bounds and shared memory).
int dga_block_grid(int n2, int n_items) {
  switch (n2) {
    case 0: return block_grid_nr<9>(n_items);
    case 1: return block_grid_nr<1>(n_items);
    case 4: return block_grid_nr<4>(n_items);
    case 9: return block_grid_nr<9>(n_items);
    default: return block_grid_nr<16>(n_items);
  }
}

cudaError_t dga_block_launch(int grid, const StructuredSource& src, const WorkItem* work, int n_items, int N, int n2,
                             int nv, int W, int Q, double beta, int max_iter, double tol, double2* out, int* status,
                             int* iters, unsigned char* scratch, size_t slot_bytes, cudaStream_t stream,
                             long long wait_limit) {
  const size_t smem = block_smem_bytes();
#define DGA_BLOCK_CASE(R)                                                                                         \
  case R:                                                                                                         \
    block_set_attributes<R>();                                                                                    \
    bse_block_mixed_kernel<R><<<grid, KT, smem, stream>>>(src, work, n_items, N, nv, W, Q, beta, max_iter, tol,    \
                                                          out, status, iters, scratch, slot_bytes, wait_limit);   \
    break;
  switch (n2) {
    DGA_BLOCK_CASE(1)
    DGA_BLOCK_CASE(4)
    DGA_BLOCK_CASE(9)
    DGA_BLOCK_CASE(16)
  }
#undef DGA_BLOCK_CASE
  return cudaGetLastError();
}

cudaError_t dga_block_batch_launch(int grid, int n2, const dga_bse_problem* probs, const MultiItem* work, int n_items,
                                   int n_max, int max_iter, double tol, int* status, int* iters,
                                   unsigned char* scratch, size_t slot_bytes, cudaStream_t stream,
                                   long long wait_limit) {
  const size_t smem = block_smem_bytes();
#define DGA_BLOCK_CASE(R)                                                                                          \
  case R:                                                                                                          \
    block_set_attributes<R>();                                                                                     \
    bse_block_multi_kernel<R><<<grid, KT, smem, stream>>>(probs, work, n_items, n_max, max_iter, tol, status,     \
                                                          iters, scratch, slot_bytes, wait_limit);                 \
    break;
  switch (n2) {
    case 0:  // orbital counts 1 to 3 in one launch
      cudaFuncSetAttribute(bse_block_multi_any_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(bse_block_multi_any_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared);
      bse_block_multi_any_kernel<<<grid, KT, smem, stream>>>(probs, work, n_items, n_max, max_iter, tol, status,
                                                             iters, scratch, slot_bytes, wait_limit);
      break;
    DGA_BLOCK_CASE(1)
    DGA_BLOCK_CASE(4)
    DGA_BLOCK_CASE(9)
    DGA_BLOCK_CASE(16)
  }
#undef DGA_BLOCK_CASE
  return cudaGetLastError();
}
