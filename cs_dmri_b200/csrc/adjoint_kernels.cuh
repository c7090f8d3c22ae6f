// Derivatives of the SHORE fit and of the maps taken on its coefficients.
//
// The reference has no derivatives; these kernels differentiate the solution
// maps its solvers compute:
//
//   L1 (src/solver/fista.rs:70-143) minimises (1/(2n)) ||M c - s||^2 + alpha ||c||_1
//   (with c >= 0 when non_negative).  On the support S = {k : c_k != 0} the
//   optimality condition is  G_SS c_S = M_S^T s - n alpha sign(c_S),  G = M^T M,
//   so dc_S/ds = G_SS^{-1} M_S^T, dc_S/dalpha = -n G_SS^{-1} sign(c_S) and the
//   off-support derivatives vanish (implicit differentiation on the converged
//   support).  For an upstream gradient gc the adjoint is
//       w_S = G_SS^{-1} gc_S  (w = 0 off S),   grad_s = M w,
//       grad_alpha = -n sign(c_S) . w_S.
//
//   L2 (src/solver/tikhonov.rs:26-76) solves H c = M^T s with
//   H = M^T M + lambda_N N + lambda_L L, one matrix for all voxels:
//       w = H^{-1} gc,  grad_s = M w,
//       grad_lambda_N = -w . (N c),  grad_lambda_L = -w . (L c).
//
// The L1 factorisations and solves run every sum in index order with
// separate multiply and add (no fused multiply-add), as a sequential FP64
// evaluation does; the L2 adjoint's w = H^{-1} gc and grad_s = M w are
// fixed-matrix applies (k_apply_dmma).
#pragma once

namespace csd {

struct AdjointParams {
  const double* G;     // L1: Kp x Kp Gram M^T M; L2: the lower Cholesky factor of H (row-major, Kp stride)
  const double* X;     // fitted coefficients, V rows of stride ldx
  int64_t ldx;
  const double* GC;    // upstream gradient on the coefficients, V rows of stride ldg
  int64_t ldg;
  int64_t V;
  int K, Kp, radial_order;
  double n_samples;    // n of the 1/(2n) data term
  double* W;           // V x Kp adjoint solution w (zero off the support)
  double* ghyper;      // V x 2 (nullable): L1 (d/dalpha, 0); L2 (d/dlambda_N, d/dlambda_L)
  unsigned long long* n_singular;  // voxels whose G_SS was not positive definite (nullable)
  // L1 two-pass schedule: voxels whose support exceeds `cap` are appended to
  // `overflow` in the first pass and solved by a second pass with cap = K
  // over that list (`list`, length *list_len).
  int cap;
  const int64_t* list;
  const unsigned long long* list_len;
  int64_t* overflow;
  unsigned long long* n_overflow;
};

// Start of column j of a packed lower triangle of order s stored by columns.
__device__ __forceinline__ int packed_col(int j, int s) { return j * s - (j * (j - 1)) / 2; }

// Per-warp shared memory of k_l1_adjoint, in doubles: the packed factor of a
// support of up to `cap` (cap (cap + 1) / 2) and the support list (K ints).
__host__ __device__ __forceinline__ int l1_adjoint_warp_doubles(int cap, int K) {
  return ((cap * (cap + 1) / 2 + (K + 1) / 2) + 1) & ~1;
}

// L1 adjoint, one warp per voxel.  The support is compacted with ballots
// (index order), G_SS gathered into the warp's packed lower triangle and
// factored right-looking (every entry receives its updates in index order,
// as a sequential L L^T does), then L y = gc_S by columns and L^T w = y by
// columns from the last row up; w is scattered into the voxel's row of W.
// A support matrix that is not positive definite leaves the voxel's w and
// alpha gradient NaN and is counted.
template <int RPL>  // ceil(K / 32)
__global__ void __launch_bounds__(256) k_l1_adjoint(AdjointParams p) {
  extern __shared__ __align__(16) double adj_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const int K = p.K, Kp = p.Kp, cap = p.cap;
  double* T = adj_smem + static_cast<size_t>(warp) * l1_adjoint_warp_doubles(cap, K);
  int* sidx = reinterpret_cast<int*>(T + cap * (cap + 1) / 2);
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  const int64_t n_items = p.list ? static_cast<int64_t>(*p.list_len) : p.V;
  for (int64_t it = static_cast<int64_t>(blockIdx.x) * nw + warp; it < n_items;
       it += static_cast<int64_t>(gridDim.x) * nw) {
    const int64_t v = p.list ? p.list[it] : it;
    const double* x = p.X + v * p.ldx;
    int s = 0;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int k = lane + 32 * r;
      const bool nz = k < K && x[k] != 0.0;
      const unsigned b = __ballot_sync(kFull, nz);
      if (nz) sidx[s + __popc(b & ((1u << lane) - 1u))] = k;
      s += __popc(b);
    }
    __syncwarp();
    if (s > cap) {  // solved by the second pass
      if (lane == 0) p.overflow[atomicAdd(p.n_overflow, 1ull)] = v;
      __syncwarp();
      continue;
    }
    double rv[RPL], sg[RPL];
#pragma unroll
    for (int c = 0; c < RPL; ++c) {
      const int q = lane + 32 * c;
      rv[c] = 0.0;
      sg[c] = 0.0;
      if (q < s) {
        const int k = sidx[q];
        rv[c] = p.GC[v * p.ldg + k];
        sg[c] = x[k] > 0.0 ? 1.0 : -1.0;
      }
    }
    for (int j = 0; j < s; ++j) {
      const int cj = packed_col(j, s);
      const double* gj = p.G + static_cast<size_t>(sidx[j]) * Kp;
      for (int i = j + lane; i < s; i += 32) T[cj + i - j] = gj[sidx[i]];
    }
    __syncwarp();
    bool ok = true;
    for (int j = 0; j < s; ++j) {
      const int cj = packed_col(j, s);
      const double d = T[cj];
      if (!(d > 0.0)) {  // every lane read the same pivot
        ok = false;
        break;
      }
      const double ljj = sqrt(d);
      __syncwarp();
      if (lane == 0) T[cj] = ljj;
      for (int i = j + 1 + lane; i < s; i += 32) T[cj + i - j] = __ddiv_rn(T[cj + i - j], ljj);
      __syncwarp();
      for (int k = j + 1; k < s; ++k) {
        const int ck = packed_col(k, s);
        const double lkj = T[cj + k - j];
        for (int i = k + lane; i < s; i += 32) T[ck + i - k] = __dsub_rn(T[ck + i - k], __dmul_rn(T[cj + i - j], lkj));
      }
      __syncwarp();
    }
    double* wrow = p.W + v * Kp;
    if (!ok) {
      for (int k = lane; k < Kp; k += 32) wrow[k] = nan;
      if (lane == 0) {
        if (p.ghyper) {
          p.ghyper[2 * v] = nan;
          p.ghyper[2 * v + 1] = nan;
        }
        if (p.n_singular) atomicAdd(p.n_singular, 1ull);
      }
      __syncwarp();
      continue;
    }
    // L y = gc_S
    for (int i = 0; i < s; ++i) {
      const int ci = packed_col(i, s);
      const int owner = i & 31, oc = i >> 5;
      double yi = 0.0;
#pragma unroll
      for (int c = 0; c < RPL; ++c)
        if (c == oc && lane == owner) yi = __ddiv_rn(rv[c], T[ci]);
      yi = __shfl_sync(kFull, yi, owner);
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int q = lane + 32 * c;
        if (q > i && q < s) rv[c] = __dsub_rn(rv[c], __dmul_rn(T[ci + q - i], yi));
        if (q == i) rv[c] = yi;
      }
    }
    // L^T w = y
    for (int i = s - 1; i >= 0; --i) {
      const int owner = i & 31, oc = i >> 5;
      double wi = 0.0;
#pragma unroll
      for (int c = 0; c < RPL; ++c)
        if (c == oc && lane == owner) wi = __ddiv_rn(rv[c], T[packed_col(i, s)]);
      wi = __shfl_sync(kFull, wi, owner);
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int q = lane + 32 * c;
        if (q < i) rv[c] = __dsub_rn(rv[c], __dmul_rn(T[packed_col(q, s) + i - q], wi));
        if (q == i) rv[c] = wi;
      }
    }
    double dot = 0.0;
#pragma unroll
    for (int c = 0; c < RPL; ++c) dot = __dadd_rn(dot, __dmul_rn(sg[c], rv[c]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(kFull, dot, o);
    for (int k = lane; k < Kp; k += 32) wrow[k] = 0.0;
    __syncwarp();
#pragma unroll
    for (int c = 0; c < RPL; ++c) {
      const int q = lane + 32 * c;
      if (q < s) wrow[sidx[q]] = rv[c];
    }
    if (lane == 0 && p.ghyper) {
      p.ghyper[2 * v] = -p.n_samples * dot;
      p.ghyper[2 * v + 1] = 0.0;
    }
    __syncwarp();
  }
}

// L2 adjoint: w = H^{-1} gc is one fixed-matrix product per voxel (the
// explicit inverse, built once per table and regularisation from the factor
// by its own solves, applied on the FP64 tensor cores by k_apply_dmma), and
// this kernel takes the hyper-parameter gradients from it, one warp per voxel:
// grad_lambda_N = -sum_k w_k c_k (n(n+1))^2, grad_lambda_L = -sum_k w_k c_k
// (l(l+1))^2 (the diagonal regularisation matrices of src/basis/shore.rs).
template <int RPL>
__global__ void __launch_bounds__(256) k_l2_hyper(const double* __restrict__ W, int64_t ldw,
                                                  const double* __restrict__ X, int64_t ldx, int64_t V, int K,
                                                  int radial_order, double* __restrict__ ghyper) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  double wn[RPL], wl[RPL];  // this lane's regularisation weights
#pragma unroll
  for (int c = 0; c < RPL; ++c) {
    const int row = lane + 32 * c;
    wn[c] = wl[c] = 0.0;
    if (row < K) {
      int n = 0, l = 0, kk = 0;
      col_to_nlk(radial_order, row, &n, &l, &kk);
      const double nn = static_cast<double>(n * (n + 1)), ll = static_cast<double>(l * (l + 1));
      wn[c] = nn * nn;
      wl[c] = ll * ll;
    }
  }
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * nw + warp; v < V; v += static_cast<int64_t>(gridDim.x) * nw) {
    double dn = 0.0, dl = 0.0;
#pragma unroll
    for (int c = 0; c < RPL; ++c) {
      const int row = lane + 32 * c;
      if (row < K) {
        const double wc = __dmul_rn(W[v * ldw + row], X[v * ldx + row]);
        dn = __dadd_rn(dn, __dmul_rn(wc, wn[c]));
        dl = __dadd_rn(dl, __dmul_rn(wc, wl[c]));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      dn += __shfl_xor_sync(kFull, dn, o);
      dl += __shfl_xor_sync(kFull, dl, o);
    }
    if (lane == 0) {
      ghyper[2 * v] = -dn;
      ghyper[2 * v + 1] = -dl;
    }
  }
}

// Identity rows (K x Kp, zero padded): the right-hand sides whose solves give
// the rows of H^{-1}.
__global__ void k_identity_rows(double* __restrict__ I, int K, int Kp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < K * Kp) I[i] = ((i % Kp) == (i / Kp)) ? 1.0 : 0.0;
}

// out[v][r] = sum over k < cols of At[k * rows + r] in[v][k]: a fixed matrix
// A (rows x cols, stored transposed so that a warp's lanes read consecutive
// rows) applied to every voxel's vector, FP64 with fused multiply-adds in
// index order.  Eight voxels per warp: their inputs are staged in the warp's
// shared slice as [k][voxel], so each coalesced load of a column of A feeds
// eight FMAs with operands from four 16-byte broadcast reads.  Outputs in
// FP64 and / or rounded to FP32 (each nullable).
__global__ void __launch_bounds__(256) k_apply64(const double* __restrict__ At, int rows, int cols,
                                                 const double* __restrict__ in, int64_t ldin, int64_t V,
                                                 double* __restrict__ out, float* __restrict__ out32,
                                                 int64_t ldout) {
  extern __shared__ __align__(16) double apply_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sI = apply_smem + static_cast<size_t>(warp) * 8 * cols;
  const int64_t groups = (V + 7) / 8;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp; g < groups; g += nwarps) {
    const int64_t v0 = 8 * g;
    const int nv = V - v0 < 8 ? static_cast<int>(V - v0) : 8;
    __syncwarp();
    for (int j = 0; j < 8; ++j)
      for (int k = lane; k < cols; k += 32) sI[k * 8 + j] = j < nv ? in[(v0 + j) * ldin + k] : 0.0;
    __syncwarp();
    const double2* sI2 = reinterpret_cast<const double2*>(sI);
    for (int r = lane; r < rows; r += 32) {
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int k = 0; k < cols; ++k) {
        const double a = At[static_cast<size_t>(k) * rows + r];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double2 xv = sI2[k * 4 + j];
          acc[2 * j] = fma(a, xv.x, acc[2 * j]);
          acc[2 * j + 1] = fma(a, xv.y, acc[2 * j + 1]);
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (j < nv) {
          if (out) out[(v0 + j) * ldout + r] = acc[j];
          if (out32) out32[(v0 + j) * ldout + r] = static_cast<float>(acc[j]);
        }
    }
  }
}

// The same product on the FP64 tensor cores, for a matrix that fits in
// shared memory: A is staged once per persistent CTA in m8n8k4 A-fragment
// order, frag[(mt * KT + kt) * 32 + lane] = A[8 mt + lane / 4][4 kt + lane % 4]
// (zero padded; read from At), so each fragment is one conflict-free 256-byte
// read.  A warp takes 8 voxels at a time: out^T (rows x 8) = A in^T, the
// voxels' inputs as B fragments, reused across a chunk of kApplyMtc row tiles
// held as accumulators.  The fragments come from global memory, so they are
// fetched well ahead of their DMMAs: with KT <= kApplyKtr (inputs of up to 96
// entries) a group's KT fragments sit in registers and serve every row
// chunk, and the next group's are loaded while this one computes; longer
// inputs stream through a ring of kApplyPf fragments.  Every tile accumulates
// its k-steps in increasing order either way.
constexpr int kApplyMtc = 12;
constexpr int kApplyKtr = 24;
constexpr int kApplyPf = 8;

template <bool kRegs>
__global__ void __launch_bounds__(256, 1) k_apply_dmma(const double* __restrict__ At, int rows, int cols,
                                                       const double* __restrict__ in, int64_t ldin, int64_t V,
                                                       double* __restrict__ out, float* __restrict__ out32,
                                                       int64_t ldout) {
  extern __shared__ __align__(16) double sA[];
  const int MT = (rows + 7) / 8, KT = (cols + 3) / 4;
  const int n_frag = MT * KT * 32;
  for (int i0 = threadIdx.x; i0 < n_frag; i0 += 8 * blockDim.x) {  // eight loads in flight per thread
    double vals[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * blockDim.x;
      const int lane = i & 31, t = i >> 5, mt = t / KT, kt = t % KT;
      const int r = 8 * mt + (lane >> 2), k = 4 * kt + (lane & 3);
      vals[u] = (i < n_frag && r < rows && k < cols) ? At[static_cast<size_t>(k) * rows + r] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (i0 + u * static_cast<int>(blockDim.x) < n_frag) sA[i0 + u * blockDim.x] = vals[u];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3;
  const int64_t groups = (V + 7) / 8;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  auto frag = [&](int64_t grp, int kt) -> double {  // this lane's B entry of k-step kt of a group
    const int64_t vb = 8 * grp + g;
    const int k = 4 * kt + q;
    return (grp < groups && vb < V && k < cols) ? in[vb * ldin + k] : 0.0;
  };
  auto store = [&](int64_t v0, int mt0, const double (&d)[kApplyMtc][2]) {
#pragma unroll
    for (int j = 0; j < kApplyMtc; ++j) {
      const int r = 8 * (mt0 + j) + g;
      if (mt0 + j >= MT || r >= rows) continue;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t vv = v0 + 2 * q + e;
        if (vv < V) {
          if (out) out[vv * ldout + r] = d[j][e];
          if (out32) out32[vv * ldout + r] = static_cast<float>(d[j][e]);
        }
      }
    }
  };
  int64_t grp = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
  if constexpr (kRegs) {
    double bn[kApplyKtr];
#pragma unroll
    for (int kt = 0; kt < kApplyKtr; ++kt) bn[kt] = kt < KT ? frag(grp, kt) : 0.0;
    for (; grp < groups; grp += nwarps) {
      double bc[kApplyKtr];
#pragma unroll
      for (int kt = 0; kt < kApplyKtr; ++kt) {
        bc[kt] = bn[kt];
        bn[kt] = kt < KT ? frag(grp + nwarps, kt) : 0.0;  // the next group's, in flight meanwhile
      }
      for (int mt0 = 0; mt0 < MT; mt0 += kApplyMtc) {
        double d[kApplyMtc][2];
#pragma unroll
        for (int j = 0; j < kApplyMtc; ++j) d[j][0] = d[j][1] = 0.0;
#pragma unroll
        for (int kt = 0; kt < kApplyKtr; ++kt) {
          if (kt >= KT) break;
#pragma unroll
          for (int j = 0; j < kApplyMtc; ++j)
            if (mt0 + j < MT) dmma_m8n8k4(d[j][0], d[j][1], sA[((mt0 + j) * KT + kt) * 32 + lane], bc[kt]);
        }
        store(8 * grp, mt0, d);
      }
    }
  } else {
    for (; grp < groups; grp += nwarps) {
      for (int mt0 = 0; mt0 < MT; mt0 += kApplyMtc) {
        double d[kApplyMtc][2];
#pragma unroll
        for (int j = 0; j < kApplyMtc; ++j) d[j][0] = d[j][1] = 0.0;
        // slot u holds k-step kt0 + u; once its DMMAs have read it, it is
        // refilled with k-step kt0 + u + kApplyPf (no register moves, which
        // would wait for loads still in flight)
        double bq[kApplyPf];
#pragma unroll
        for (int u = 0; u < kApplyPf; ++u) bq[u] = frag(grp, u);
        for (int kt0 = 0; kt0 < KT; kt0 += kApplyPf) {
#pragma unroll
          for (int u = 0; u < kApplyPf; ++u) {
            const int kt = kt0 + u;
            if (kt < KT) {
#pragma unroll
              for (int j = 0; j < kApplyMtc; ++j)
                if (mt0 + j < MT) dmma_m8n8k4(d[j][0], d[j][1], sA[((mt0 + j) * KT + kt) * 32 + lane], bq[u]);
              bq[u] = frag(grp, kt + kApplyPf);
            }
          }
        }
        store(8 * grp, mt0, d);
      }
    }
  }
}

__global__ void k_fill_u32(uint32_t* __restrict__ a, int64_t n, uint32_t v) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// RTOP of FP64 coefficients (src/scalars/microstructure.rs:98-118):
// max(sum_n (c_n00 / E0) (-1)^n w_n, 0), NaN when E0 is zero or not finite.
__device__ __forceinline__ double rtop64(const MicroConsts& mc, const double* c, double* e0_out) {
  double e0 = 0.0;
  const double inv = 1.0 / sqrt(4.0 * CUDART_PI);
  for (int n = 0; n <= mc.radial_order; ++n) e0 += c[mc.n00[n]] * mc.r0[n] * inv;
  *e0_out = e0;
  if (!isfinite(e0) || e0 == 0.0) return __longlong_as_double(0x7ff8000000000000ll);
  double a = 0.0;
  for (int n = 0; n <= mc.radial_order; ++n) {
    const double sign = (n % 2 == 0) ? 1.0 : -1.0;
    a += (c[mc.n00[n]] / e0) * sign * mc.rtop_w[n];
  }
  return fmax(a, 0.0);
}

__global__ void k_rtop64(const MicroConsts* __restrict__ mcp, const double* __restrict__ C, int64_t ldc, int64_t V,
                         double* __restrict__ out) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  double e0;
  out[v] = rtop64(*mcp, C + v * ldc, &e0);
}

// d RTOP / d c_(n,0,0) = ((-1)^n w_n - RTOP r0_n / sqrt(4 pi)) / E0 where
// RTOP > 0; zero where the clamp at 0 is active; NaN where RTOP is NaN and
// the upstream gradient is not zero.  Other coefficients get zero.
__global__ void k_rtop64_adjoint(const MicroConsts* __restrict__ mcp, const double* __restrict__ C, int64_t ldc,
                                 int64_t V, const double* __restrict__ g, double* __restrict__ GC, int64_t ldgc) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const MicroConsts& mc = *mcp;
  double e0;
  const double rt = rtop64(mc, C + v * ldc, &e0);
  double* o = GC + v * ldgc;
  for (int k = 0; k < mc.K; ++k) o[k] = 0.0;
  const double gv = g[v];
  if (isnan(rt)) {
    if (gv != 0.0)
      for (int k = 0; k < mc.K; ++k) o[k] = rt;
    return;
  }
  if (!(rt > 0.0)) return;
  const double inv = 1.0 / sqrt(4.0 * CUDART_PI);
  for (int n = 0; n <= mc.radial_order; ++n) {
    const double sign = (n % 2 == 0) ? 1.0 : -1.0;
    o[mc.n00[n]] = gv * ((sign * mc.rtop_w[n] - rt * mc.r0[n] * inv) / e0);
  }
}

}  // namespace csd
