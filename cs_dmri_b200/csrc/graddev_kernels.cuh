// Per-voxel SHORE fit with a per-voxel design matrix: gradient-deviation
// tensors and per-voxel dropped samples.
//
// The reference has the per-voxel effective table (src/graddev.rs:160-185:
// q = T^T g, b_eff = b |q|^2, dir = q / |q|) but fits SHORE with one shared
// design; here every voxel's design is built from its own table on the fly,
// from the rows it keeps, and fitted by the reference's FISTA
// (src/solver/fista.rs:38-143) with its own Lipschitz constant
// L_v = sigma_max(M_v)^2 / n_v.
//
// One persistent CTA per SM takes voxels from a queue.  Per voxel:
//   1. kept rows, effective b and direction per row;
//   2. G_v = M_v^T M_v on the FP64 tensor cores (DMMA m8n8k4): the geometry
//      of every kept row first, then 64 rows at a time in factored form in
//      shared memory (radial factors per (n, l) and SH values per (l, k); a
//      design entry is the product of one of each, formed as the DMMA
//      operand fragment is loaded), each warp accumulating one rectangle or
//      two triangles of 8 x 8 tiles of the upper triangle in registers
//      (GramPlan); b_v = M_v^T s_v alongside;
//   3. lambda_max(G_v) by Lanczos (a fixed number of steps, the largest Ritz
//      value by multisection of the tridiagonal's Sturm count, one point per
//      thread);
//   4. FISTA in the Gram form with G_v in shared memory (one thread per row of
//      the product, 16-byte loads), the reference's update and stopping rule.
#pragma once

namespace csd {

constexpr int kGdChunk = 64;       // design rows per Gram chunk (one thread per row and value group)
constexpr int kGdLanczos = 40;     // Lanczos steps (capped at K)
constexpr int kGdRcp = 17;         // reciprocals 1 / i, i < 17 (radial orders <= 16)
// Lanczos steps in the converged-optimum modes, with the support iterations'
// step 1 / (1.12 L) from that estimate: over sampled brain-phantom designs
// the 10-step Ritz value stays within 1.048 of lambda_max (16 steps: 1.010)
constexpr int kGdLanczosKkt = 10;
constexpr double kGdKktLipMargin = 1.12;

struct GraddevParams {
  const float* S;           // V x N signals
  const double* T;          // V x 9 deviation tensors (row-major), or nullptr (identity)
  const uint8_t* keep;      // V x N sample mask (non-zero = use), or nullptr (every sample)
  const double* bvals;      // N
  const double* bvecs;      // N x 3
  int N, K, radial_order;
  double zeta, qdenom, b0_thr;
  double alpha;             // when alpha_v is null
  const double* alpha_v;    // V, or nullptr
  double tol;
  int max_iter, non_negative;
  const double* mom;        // (t_k - 1) / t_{k+1}, k < max_iter
  int64_t V;
  unsigned long long* queue;
  double* X;                // V x K coefficients
  uint32_t* iters;          // V
  uint8_t* conv;            // V
  double* lipschitz;        // V (nullable)
  int* n_rows;              // V (nullable): samples kept
  unsigned long long* iter_total;  // executed FISTA iterations, summed (nullable)
  // converged-optimum mode (kkt != 0): kkt_iters FISTA iterations find the
  // support, one warp polishes on G_v and certifies (polish_warp); a voxel it
  // cannot certify gets the reference FISTA from zero, uncertified
  int kkt;
  // mixed != 0 (with kkt): G_v kept as FP32 planes hi + lo; the Lanczos
  // estimate and the support iterations run in FP32 on hi, the polish and any
  // fallback in FP64 on hi + lo
  int mixed;
  int kkt_iters, kkt_rounds;
  double kappa;
  double* kkt_out;                   // V (nullable): largest KKT residual, NaN when uncertified
  unsigned long long* n_uncertified; // (nullable)
  unsigned long long* round_total;   // polish solves, summed (nullable)
};

// Shared-memory plan (doubles unless noted), shared by host and device.
// While G is built its region holds a chunk of kGdChunk design rows in
// factored form: each entry of the design is the product of a radial factor
// (one per (n, l)) and a real SH value (one per (l, k)), so a chunk keeps the
// rows' NL radial factors (row stride RS, one more slot that holds 0 for the
// padding columns) and NSH SH values (row stride YS); both strides are odd,
// so the fragment loads of four consecutive rows fall in distinct banks.
struct GdLayout {
  int K, Kp, LDG, LDF, NL, NSH, RS, YS, LC;
  size_t g, vec, red, tri, tab, rows, colmap, nzv, nzi, total_bytes;
  __host__ __device__ GdLayout(int K_, int radial_order, int N) {
    K = K_;
    Kp = 8 * ((K + 7) / 8);
    LDG = K + (K & 1);   // even row stride of G: 16-byte rows, conflict-free 16-byte loads
    // row stride of the FP32 planes: 16-byte rows, an odd number of them, so
    // that 8 rows' 16-byte loads at one column fall in distinct banks
    LDF = 4 * ((K + 3) / 4);
    if ((LDF / 4) % 2 == 0) LDF += 4;
    NL = 0;
    for (int n = 0; n <= radial_order; ++n) NL += n / 2 + 1;
    NSH = (radial_order / 2 + 1) * (radial_order + 1);
    RS = (NL + 1) | 1;
    YS = NSH | 1;
    const size_t chunk = static_cast<size_t>(kGdChunk) * (RS + YS) + 8 * static_cast<size_t>(N);
    const size_t gk64 = static_cast<size_t>(K) * LDG, gk32 = static_cast<size_t>(K) * LDF;  // gk32: two FP32 planes
    const size_t gk = gk64 > gk32 ? gk64 : gk32;
    const size_t gsize = gk > chunk ? gk : chunk;
    g = 0;
    vec = (gsize + 1) & ~static_cast<size_t>(1);           // b, x, y, gy, v_prev, v, w: 7 * Kp
    red = vec + 7 * static_cast<size_t>(Kp);                 // 32 reduction slots
    tri = red + 32;                                          // Lanczos alpha / beta: 2 * 64
    tab = tri + 128;                                         // kappa per (n, l), SH norm per (l, k)
    rows = tab + ((static_cast<size_t>(NL + NSH) + 1) & ~static_cast<size_t>(1));  // N ints
    colmap = rows + (static_cast<size_t>(N) + 1) / 2;        // column map (ints)
    // FISTA's nonzero entries of y, one list per partial sum of the product
    // (gd_gemv_nz): values (doubles) and indices (ints), LC slots each
    LC = (K + 3) / 4 + 4;
    nzv = colmap + (static_cast<size_t>(K) + 1) / 2;
    nzi = nzv + 4 * static_cast<size_t>(LC);
    total_bytes = 8 * (nzi + 2 * static_cast<size_t>(LC) + 2);
  }
};

// Block-wide sum of one value per thread; every thread gets the same result
// (fixed order: warp trees, then the warp sums in order).  `red` has 32 slots.
__device__ __forceinline__ double gd_block_sum(double a, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
  __syncthreads();
  if (lane == 0) red[warp] = a;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

// The same sum into slots no thread reads any more, so without the barrier
// before the write: the caller separates the reads of an earlier sum into
// `slots` from this write by a barrier of its own.
__device__ __forceinline__ double gd_block_sum_fresh(double a, double* slots) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
  if (lane == 0) slots[warp] = a;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += slots[w];
  return s;
}

// out[i] = sum_j G[i][j] v[j] for i < K, one thread per row: 16-byte loads of
// G's row and of v (both in shared memory), four per step, into four
// independent partial sums added at the end.
__device__ __forceinline__ void gd_gemv(const double* G, int LDG, int K, const double* v, double* out) {
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    const double2* gr = reinterpret_cast<const double2*>(G + static_cast<size_t>(i) * LDG);
    const double2* v2 = reinterpret_cast<const double2*>(v);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const int h = K >> 1;
    int j = 0;
    for (; j + 3 < h; j += 4) {  // eight loads in flight per step
      const double2 g0 = gr[j], g1 = gr[j + 1], g2 = gr[j + 2], g3 = gr[j + 3];
      const double2 w0 = v2[j], w1 = v2[j + 1], w2 = v2[j + 2], w3 = v2[j + 3];
      a0 = fma(g0.x, w0.x, a0);
      a1 = fma(g0.y, w0.y, a1);
      a2 = fma(g1.x, w1.x, a2);
      a3 = fma(g1.y, w1.y, a3);
      a0 = fma(g2.x, w2.x, a0);
      a1 = fma(g2.y, w2.y, a1);
      a2 = fma(g3.x, w3.x, a2);
      a3 = fma(g3.y, w3.y, a3);
    }
    for (; j < h; ++j) {
      const double2 g0 = gr[j], w0 = v2[j];
      a0 = fma(g0.x, w0.x, a0);
      a1 = fma(g0.y, w0.y, a1);
    }
    if (K & 1) a2 = fma(G[static_cast<size_t>(i) * LDG + K - 1], v[K - 1], a2);
    out[i] = (a0 + a1) + (a2 + a3);
  }
}

// Which of gd_gemv's four partial sums takes entry e: e mod 4 in its main
// loop, e mod 2 in the remainder loop, the third for the last of an odd K.
__device__ __forceinline__ int gd_gemv_sum_of(int e, int K) {
  const int h = K >> 1, main = 8 * (h / 4);
  return e < main ? (e & 3) : (e < 2 * h ? (e & 1) : 2);
}

// gd_gemv for a vector with few nonzeros: `cnt[r]` entries of sum r are
// listed, in increasing index, as (nzi[r LC + k], nzv[r LC + k]).  Each sum
// adds the same products in the same order as gd_gemv's, without the zero
// ones (an exact product of zero leaves a sum unchanged: a sum that starts
// at +0 never becomes -0), so the result is bit for bit gd_gemv's.
__device__ __forceinline__ void gd_gemv_nz(const double* G, int LDG, int K, const int* cnt, const double* nzv,
                                           const int* nzi, int LC, double* out) {
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    const double* gr = G + static_cast<size_t>(i) * LDG;
    const int n0 = cnt[0], n1 = cnt[1], n2 = cnt[2], n3 = cnt[3];
    const int nmax = max(max(n0, n1), max(n2, n3));
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    for (int k = 0; k < nmax; ++k) {
      if (k < n0) a0 = fma(gr[nzi[k]], nzv[k], a0);
      if (k < n1) a1 = fma(gr[nzi[LC + k]], nzv[LC + k], a1);
      if (k < n2) a2 = fma(gr[nzi[2 * LC + k]], nzv[2 * LC + k], a2);
      if (k < n3) a3 = fma(gr[nzi[3 * LC + k]], nzv[3 * LC + k], a3);
    }
    out[i] = (a0 + a1) + (a2 + a3);
  }
}

// The same product with FP32 entries, vector and sums: G_v's hi plane (row
// stride LDF), four entries per 16-byte load.
__device__ __forceinline__ void gd_gemv32(const float* G, int LDF, int K, const float* v, float* out) {
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    const float4* gr = reinterpret_cast<const float4*>(G + static_cast<size_t>(i) * LDF);
    const float4* v4 = reinterpret_cast<const float4*>(v);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    const int h = K >> 2;
#pragma unroll 4
    for (int j = 0; j < h; ++j) {
      const float4 g = gr[j], w = v4[j];
      a0 = fmaf(g.x, w.x, a0);
      a1 = fmaf(g.y, w.y, a1);
      a2 = fmaf(g.z, w.z, a2);
      a3 = fmaf(g.w, w.w, a3);
    }
    for (int j = 4 * h; j < K; ++j) a0 = fmaf(G[static_cast<size_t>(i) * LDF + j], v[j], a0);
    out[i] = (a0 + a1) + (a2 + a3);
  }
}

// The FP64 product with G_v rebuilt from its planes (hi + lo per entry).
__device__ __forceinline__ void gd_gemv_hl(const float* Gh, const float* Gl, int LDF, int K, const double* v,
                                           double* out) {
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    const float4* hr = reinterpret_cast<const float4*>(Gh + static_cast<size_t>(i) * LDF);
    const float4* lr = reinterpret_cast<const float4*>(Gl + static_cast<size_t>(i) * LDF);
    const double2* v2 = reinterpret_cast<const double2*>(v);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const int h = K >> 2;
    for (int j = 0; j < h; ++j) {
      const float4 gh = hr[j], gl = lr[j];
      const double2 w0 = v2[2 * j], w1 = v2[2 * j + 1];
      a0 = fma(static_cast<double>(gh.x) + static_cast<double>(gl.x), w0.x, a0);
      a1 = fma(static_cast<double>(gh.y) + static_cast<double>(gl.y), w0.y, a1);
      a2 = fma(static_cast<double>(gh.z) + static_cast<double>(gl.z), w1.x, a2);
      a3 = fma(static_cast<double>(gh.w) + static_cast<double>(gl.w), w1.y, a3);
    }
    for (int j = 4 * h; j < K; ++j) {
      const size_t e = static_cast<size_t>(i) * LDF + j;
      a0 = fma(static_cast<double>(Gh[e]) + static_cast<double>(Gl[e]), v[j], a0);
    }
    out[i] = (a0 + a1) + (a2 + a3);
  }
}

// Work split of G's upper triangle of MT x MT tiles (8 x 8 each) between the
// CTA's 8 warps.  The tile indices fall into NG groups of GS; a pair of
// groups I < J is a GS x GS rectangle of tiles, a group I alone the triangle
// of tiles (i, j), i <= j, inside it.  Warps 0 .. NR-1 take one rectangle
// each, the others TPT triangles each.  Per k-step a warp then loads 2 GS
// operand fragments (one per tile row or column it touches) for up to GS^2
// products, where a list of independent tiles needs two loads per product.
template <int MT>
struct GramPlan {
  static constexpr int GS = (MT > 9) ? 5 : 3;
  static constexpr int NG = (MT + GS - 1) / GS;
  static constexpr int NR = NG * (NG - 1) / 2;              // rectangles
  static constexpr int TW = 8 - NR;                          // warps on triangles
  static constexpr int TPT = (NG + TW - 1) / TW;             // triangles per such warp
  static constexpr int TRI = GS * (GS + 1) / 2;              // tiles of one triangle
  static constexpr int ACC = (GS * GS > TPT * TRI) ? GS * GS : TPT * TRI;
  static_assert(NR <= 8 && TW >= 1 && TPT <= 2, "gram plan");
};

// Count of eigenvalues of the symmetric tridiagonal (a, b) below x (Sturm).
__device__ __forceinline__ int sturm_below(const double* a, const double* b, int m, double x) {
  int c = 0;
  double d = a[0] - x;
  if (d < 0.0) ++c;
  for (int i = 1; i < m; ++i) {
    const double dd = (d == 0.0) ? 1e-300 : d;
    d = (a[i] - x) - b[i - 1] * b[i - 1] / dd;
    if (d < 0.0) ++c;
  }
  return c;
}

template <int MT>
__global__ void __launch_bounds__(256, (MT <= 9) ? 2 : 1) k_graddev_fit(GraddevParams p) {
  using GP = GramPlan<MT>;
  constexpr int GS = GP::GS;
  extern __shared__ __align__(16) double gd_smem[];
  const GdLayout L(p.K, p.radial_order, p.N);
  const int K = p.K, Kp = L.Kp, NL = L.NL, NSH = L.NSH, RS = L.RS, YS = L.YS, N = p.N;
  double* G = gd_smem + L.g;
  double* Rv = G;                                  // chunk: kGdChunk x RS radial factors (aliases G while it is built)
  double* Yv = Rv + kGdChunk * RS;                 // kGdChunk x YS real SH values
  double* gall = Yv + kGdChunk * YS;               // N x 8 per kept row: r, theta, phi, signal, cos phi, u, exp(-u/2)
  double* vb = gd_smem + L.vec;
  double* vx = vb + Kp;
  double* vy = vx + Kp;
  double* vgy = vy + Kp;
  double* lv_prev = vgy + Kp;
  double* lv = lv_prev + Kp;
  double* lw = lv + Kp;
  double* red = gd_smem + L.red;
  double* ta = gd_smem + L.tri;
  double* tb = ta + 64;
  double* kap = gd_smem + L.tab;                   // NL: kappa(zeta, n, l)
  double* shn = kap + NL;                          // NSH: SH normalisation of (l, k)
  int* rows = reinterpret_cast<int*>(gd_smem + L.rows);
  int* col_map = reinterpret_cast<int*>(gd_smem + L.colmap);  // K: radial factor | SH entry << 16
  double* nzv = gd_smem + L.nzv;                                // FISTA's nonzero y entries, by partial sum
  int* nzi = reinterpret_cast<int*>(gd_smem + L.nzi);
  __shared__ int gd_wcnt[8][4];  // per warp and partial sum: nonzero y entries
  __shared__ int gd_ncnt[4];     // per partial sum
  __shared__ int64_t s_v;
  __shared__ int s_n;
  __shared__ double s_lmax;
  __shared__ int s_first;
  __shared__ uint16_t gd_tri[kTriTable];  // (row, col) of a packed triangle, for the polish
  __shared__ double gd_rcp[kGdRcp];       // 1 / i: the recurrences' divisors as products
  for (int i = threadIdx.x; i < kGdRcp; i += blockDim.x) gd_rcp[i] = i > 0 ? 1.0 / i : 0.0;
  for (int e = threadIdx.x; e < kTriTable; e += blockDim.x) {
    const int r = tri_row(e);
    gd_tri[e] = static_cast<uint16_t>((r << 8) | (e - pk_row(r)));
  }
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, q = lane & 3;

  // column -> (radial factor, SH entry) and the per-(n, l) / per-(l, k)
  // constants, once per CTA (the same expressions as dev_shore_radial and
  // dev_brainsuite_sh evaluate per entry)
  for (int col = tid; col < K; col += blockDim.x) {
    int n, l, k;
    col_to_nlk(p.radial_order, col, &n, &l, &k);
    int nl = 0;
    for (int nn = 0; nn < n; ++nn) nl += nn / 2 + 1;
    int lk = 0;
    for (int ll = 0; ll < l; ll += 2) lk += 2 * ll + 1;
    col_map[col] = (nl + l / 2) | ((lk + k) << 16);
  }
  for (int j = tid; j < NL + NSH; j += blockDim.x) {
    if (j < NL) {
      int nn = 0, rem = j;
      while (rem >= nn / 2 + 1) {
        rem -= nn / 2 + 1;
        ++nn;
      }
      kap[j] = dev_kappa(p.zeta, nn, 2 * rem);
    } else {
      int l = 0, rem = j - NL;
      while (rem >= 2 * l + 1) {
        rem -= 2 * l + 1;
        l += 2;
      }
      const int m = (rem < l) ? l - rem : (rem == l ? 0 : rem - l);
      shn[j - NL] = sqrt((2.0 * l + 1.0) / (4.0 * CUDART_PI) * dev_factorial(l - m) / dev_factorial(l + m));
    }
  }
  __syncthreads();
  // this warp's share of G's upper triangle (GramPlan): tile-index groups ga
  // (and gb), and this lane's design column in each tile row / column it
  // touches, as (radial factor | SH entry << 16); padding columns point at
  // the chunk rows' zero slot
  const bool is_rect = warp < GP::NR;
  int ga = GP::NG, gb = GP::NG;  // NG: none
  if (is_rect) {
    int rem = warp;
    ga = 0;
    while (rem >= GP::NG - 1 - ga) {
      rem -= GP::NG - 1 - ga;
      ++ga;
    }
    gb = ga + 1 + rem;
  } else {
    ga = (warp - GP::NR) * GP::TPT;
    if (GP::TPT == 2) gb = ga + 1;
    if (ga > GP::NG) ga = GP::NG;
    if (gb > GP::NG) gb = GP::NG;
  }
  int ca[GS], cb[GS];
#pragma unroll
  for (int i = 0; i < GS; ++i) {
    const int c1 = 8 * (ga * GS + i) + g, c2 = 8 * (gb * GS + i) + g;
    ca[i] = (ga < GP::NG && c1 < K) ? col_map[c1] : NL;
    cb[i] = (gb < GP::NG && c2 < K) ? col_map[c2] : NL;
  }

  unsigned long long executed = 0;
  while (true) {
    if (tid == 0) s_v = static_cast<int64_t>(atomicAdd(p.queue, 1ull));
    __syncthreads();
    const int64_t v = s_v;
    if (v >= p.V) break;
    // ---- 1. kept rows, in order
    if (warp == 0) {
      int cnt = 0;
      for (int base = 0; base < N; base += 32) {
        const int i = base + lane;
        const bool k = i < N && (p.keep ? p.keep[v * N + i] != 0 : true);
        const unsigned bal = __ballot_sync(kFull, k);
        if (k) rows[cnt + __popc(bal & ((1u << lane) - 1u))] = i;
        cnt += __popc(bal);
      }
      if (lane == 0) s_n = cnt;
    }
    for (int i = tid; i < Kp; i += blockDim.x) vb[i] = 0.0;
    __syncthreads();
    const int n = s_n;

    // ---- 2. Gram matrix and right-hand side
    // effective geometry of every kept row (one thread per row)
    for (int r = tid; r < n; r += blockDim.x) {
      const int i = rows[r];
      const double b = p.bvals[i];
      const double gx = p.bvecs[3 * i], gy = p.bvecs[3 * i + 1], gz = p.bvecs[3 * i + 2];
      const double gn = sqrt(gx * gx + gy * gy + gz * gz);
      double be = b, dx = gx, dy = gy, dz = gz;
      if (b > p.b0_thr && gn > 1e-12) {  // graddev.rs:171-177 (identity frame rotation)
        double Tm[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) Tm[e] = p.T ? p.T[v * 9 + e] : ((e % 4 == 0) ? 1.0 : 0.0);
        const double ux = gx / gn, uy = gy / gn, uz = gz / gn;
        const double qx = Tm[0] * ux + Tm[3] * uy + Tm[6] * uz;  // q = T^T g
        const double qy = Tm[1] * ux + Tm[4] * uy + Tm[7] * uz;
        const double qz = Tm[2] * ux + Tm[5] * uy + Tm[8] * uz;
        const double q2 = qx * qx + qy * qy + qz * qz;
        const double qn = sqrt(q2);
        be = b * q2;
        dx = qx / qn;
        dy = qy / qn;
        dz = qz / qn;
      }
      // q-value and spherical angles as in k_design (src/basis/shore.rs:122-178)
      const double qv = (be <= p.b0_thr) ? 0.0 : sqrt(be / p.qdenom);
      const double x = dx * qv, y = dy * qv, z = dz * qv;
      const double rr = sqrt(x * x + y * y + z * z);
      double th = atan2(y, x);
      const double ph = (rr > 0.0) ? acos(fmin(fmax(z / rr, -1.0), 1.0)) : 0.0;
      if (isnan(th)) th = 0.0;
      const double u = rr * rr / p.zeta;
      gall[8 * r] = rr;
      gall[8 * r + 1] = th;
      gall[8 * r + 2] = ph;
      gall[8 * r + 3] = static_cast<double>(p.S[v * N + i]);
      gall[8 * r + 4] = cos(ph);
      gall[8 * r + 5] = u;
      gall[8 * r + 6] = exp(-u * 0.5);
    }
    __syncthreads();
    double acc[GP::ACC][2];  // this warp's tiles of G (declared after the geometry: fewer live registers there)
#pragma unroll
    for (int s = 0; s < GP::ACC; ++s) acc[s][0] = acc[s][1] = 0.0;
    for (int c0 = 0; c0 < n; c0 += kGdChunk) {
      const double* geo = gall + 8 * static_cast<size_t>(c0);

      // the chunk's rows in factored form, one thread per row in each of four
      // groups: radial factors for l = 0 and l >= 6 (group 0) and for
      // l = 2, 4 (group 3); real SH values for even m (group 1) and odd m
      // (group 2).  The formulas are those of dev_shore_radial and
      // dev_brainsuite_sh, with the costly steps replaced: integer powers by
      // products, the recurrences' divisions by reciprocal products, and
      // cos / sin of m theta by rotation.  So the entries agree with the
      // shared-design kernel's to a few units in the last place, not bit for
      // bit.  Rows past the last kept one are zero.
      {
        const int t = tid % kGdChunk, grp = tid / kGdChunk;
        const double* gt = geo + 8 * t;
        const int R = p.radial_order;
        double* Rt = Rv + t * RS;
        double* Yt = Yv + t * YS;
        if (c0 + t >= n) {
          if (grp == 0)
            for (int j = 0; j < RS; ++j) Rt[j] = 0.0;
          else if (grp == 1)
            for (int j = 0; j < YS; ++j) Yt[j] = 0.0;
        } else if (grp == 0 || grp == 3) {
          // exp(-u/2) u^(l/2) L_{n-l}^{(l+1/2)}(u): the generalised Laguerre
          // polynomials of every degree n - l from one three-term recurrence
          // per l, with the divisor k + 1 taken as a product with 1 / (k + 1)
          const double u = gt[5];
          if (grp == 0) Rt[NL] = 0.0;  // the padding columns' factor
          double upow = 1.0;
          for (int l = 0; l <= R; l += 2) {
            if (l > 0) upow *= u;  // u^(l/2) by products
            if ((grp == 0) != (l == 0 || l >= 6)) continue;
            const double al = static_cast<double>(l) + 0.5;
            double lkm1 = 1.0, lk = 1.0 + al - u;
            for (int deg = 0; l + deg <= R; ++deg) {
              double lag;
              if (deg == 0) {
                lag = 1.0;
              } else if (deg == 1) {
                lag = lk;
              } else {
                const double kf = deg - 1;
                const double lkp1 = ((2.0 * kf + 1.0 + al - u) * lk - (kf + al) * lkm1) * gd_rcp[deg];
                lkm1 = lk;
                lk = lkp1;
                lag = lk;
              }
              const int nn = l + deg;
              const int j = ((nn & 1) ? ((nn + 1) / 2) * ((nn + 1) / 2) : (nn / 2) * (nn / 2 + 1)) + l / 2;
              Rt[j] = kap[j] * lag * gt[6] * upow;
            }
          }
        } else {
          // P_l^m for l = m, m + 1, ..., R (dev_assoc_legendre's steps), times
          // the SH normalisation and cos / sin of m theta (by rotation from
          // those of theta)
          const double x = gt[4];
          double s1, c1;
          sincos(gt[1], &s1, &c1);
          double cm = 1.0, sm = 0.0;
          const double s2 = sqrt(2.0);
          for (int mm = 0; mm <= R; ++mm) {
            if (mm > 0) {
              if (mm == 1) {
                cm = c1;
                sm = s1;
              } else {
                const double cn = fma(cm, c1, -sm * s1), sn = fma(sm, c1, cm * s1);
                cm = cn;
                sm = sn;
              }
            }
            if ((mm & 1) != (grp == 2 ? 1 : 0)) continue;
            double pmm = 1.0;
            if (mm > 0) {
              const double somx2 = sqrt(fmax((1.0 - x) * (1.0 + x), 0.0));
              double fact = 1.0;
              for (int i = 0; i < mm; ++i) {
                pmm *= -fact * somx2;
                fact += 2.0;
              }
            }
            // the SH values of P_l^mm, l even: (l, l) for m = 0 (1 / sqrt(4 pi)
            // at l = 0), (l, l - m) with cos and (l, l + m) with sin otherwise
            auto emit = [&](int l, double P) {
              const int lk = (l / 2) * (l - 1);
              if (mm == 0) {
                Yt[lk + l] = (l == 0) ? 1.0 / sqrt(4.0 * CUDART_PI) : shn[lk + l] * P;
              } else {
                const double plc = shn[lk + l - mm] * P;
                Yt[lk + l - mm] = s2 * plc * cm;
                const double pls = shn[lk + l + mm] * P;
                Yt[lk + l + mm] = s2 * (((mm + 1) % 2 == 0) ? 1.0 : -1.0) * pls * sm;
              }
            };
            if (mm % 2 == 0) emit(mm, pmm);
            if (mm + 1 > R) continue;
            double pmmp1 = x * (2.0 * mm + 1.0) * pmm;
            if ((mm + 1) % 2 == 0) emit(mm + 1, pmmp1);
            for (int ll = mm + 2; ll <= R; ++ll) {
              const double llf = ll, mf = mm;
              const double pll = ((2.0 * llf - 1.0) * x * pmmp1 - (llf + mf - 1.0) * pmm) * gd_rcp[ll - mm];
              pmm = pmmp1;
              pmmp1 = pll;
              if (ll % 2 == 0) emit(ll, pll);
            }
          }
        }
      }
      __syncthreads();
      const int rows_here = min(kGdChunk, n - c0);
      for (int col = tid; col < K; col += blockDim.x) {
        const int cm = col_map[col], rj = cm & 0xffff, yj = cm >> 16;
        double a = vb[col];
        for (int t = 0; t < rows_here; ++t)
          a = __dadd_rn(a, __dmul_rn(Rv[t * RS + rj] * Yv[t * YS + yj], geo[8 * t + 3]));
        vb[col] = a;
      }
      // this warp's tiles: the operand fragments of a k-step are design
      // entries (rows 4 kk + q, this lane's columns), formed as radial factor
      // x SH value; rows past n are zero
#pragma unroll 2
      for (int kk = 0; kk < (rows_here + 3) / 4; ++kk) {
        const double* Rr = Rv + (4 * kk + q) * RS;
        const double* Yr = Yv + (4 * kk + q) * YS;
        double fa[GS], fb[GS];
#pragma unroll
        for (int i = 0; i < GS; ++i) {
          fa[i] = Rr[ca[i] & 0xffff] * Yr[ca[i] >> 16];
          fb[i] = Rr[cb[i] & 0xffff] * Yr[cb[i] >> 16];
        }
        if (is_rect) {
#pragma unroll
          for (int i = 0; i < GS; ++i)
#pragma unroll
            for (int j = 0; j < GS; ++j)
              if (gb * GS + j < MT) dmma_m8n8k4(acc[i * GS + j][0], acc[i * GS + j][1], fa[i], fb[j]);
        } else {
#pragma unroll
          for (int i = 0; i < GS; ++i)
#pragma unroll
            for (int j = i; j < GS; ++j) {
              const int e = i * GS - i * (i - 1) / 2 + (j - i);  // (i, j) in the packed triangle
              if (ga * GS + j < MT) dmma_m8n8k4(acc[e][0], acc[e][1], fa[i], fa[j]);
              if (GP::TPT == 2 && gb * GS + j < MT)
                dmma_m8n8k4(acc[GP::TRI + e][0], acc[GP::TRI + e][1], fb[i], fb[j]);
            }
        }
      }
      __syncthreads();
    }
    // G from the tiles (and the mirror of each off-diagonal tile): FP64, or
    // in the mixed mode the planes hi = fl32(G), lo = fl32(G - hi)
    const bool mixed = p.mixed != 0;
    const int LDF = L.LDF;
    float* Ghi = reinterpret_cast<float*>(G);
    float* Glo = Ghi + static_cast<size_t>(K) * LDF;
    auto put = [&](int mt, int nt, const double (&d)[2]) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = 8 * mt + g, j = 8 * nt + 2 * q + e;
        if (i < K && j < K) {
          if (mixed) {
            const float hi = __double2float_rn(d[e]);
            const float lo = __double2float_rn(d[e] - static_cast<double>(hi));
            Ghi[i * LDF + j] = hi;
            Glo[i * LDF + j] = lo;
            if (mt != nt) {
              Ghi[j * LDF + i] = hi;
              Glo[j * LDF + i] = lo;
            }
          } else {
            G[i * L.LDG + j] = d[e];
            if (mt != nt) G[j * L.LDG + i] = d[e];  // a diagonal tile holds both halves itself
          }
        }
      }
    };
    if (is_rect) {
#pragma unroll
      for (int i = 0; i < GS; ++i)
#pragma unroll
        for (int j = 0; j < GS; ++j)
          if (ga * GS + i < MT && gb * GS + j < MT) put(ga * GS + i, gb * GS + j, acc[i * GS + j]);
    } else {
#pragma unroll
      for (int i = 0; i < GS; ++i)
#pragma unroll
        for (int j = i; j < GS; ++j) {
          const int e = i * GS - i * (i - 1) / 2 + (j - i);
          if (ga * GS + j < MT) put(ga * GS + i, ga * GS + j, acc[e]);
          if (GP::TPT == 2 && gb * GS + j < MT) put(gb * GS + i, gb * GS + j, acc[GP::TRI + e]);
        }
    }
    __syncthreads();

    // ---- 3. lambda_max(G) by Lanczos: `steps` steps, the largest Ritz value
    // left in s_lmax (a lower bound of lambda_max, exact to ~1e-12 at 40)
    const int LDG = L.LDG;
    // the FP64 product with G_v (from its planes in the mixed mode)
    auto gemv64 = [&](const double* vin, double* vout) {
      if (mixed)
        gd_gemv_hl(Ghi, Glo, LDF, K, vin, vout);
      else
        gd_gemv(G, LDG, K, vin, vout);
    };
    // `lowp`: the vectors are FP32 (in the same slots) and the product uses
    // G_v's hi plane; the sums and the tridiagonal stay FP64
    auto run_lanczos = [&](int steps, bool lowp) {
      const int m = min(K, steps);
      float* lv32 = reinterpret_cast<float*>(lv);
      float* lvp32 = reinterpret_cast<float*>(lv_prev);
      float* lw32 = reinterpret_cast<float*>(lw);
      auto get = [&](const double* d, const float* f, int i) -> double {
        return lowp ? static_cast<double>(f[i]) : d[i];
      };
      auto set = [&](double* d, float* f, int i, double x) {
        if (lowp)
          f[i] = static_cast<float>(x);
        else
          d[i] = x;
      };
      for (int i = tid; i < Kp; i += blockDim.x) {
        set(lv, lv32, i, (i < K) ? 1.0 + 0.5 * sin(1.7 * i + 0.3) : 0.0);  // fixed start vector
        set(lv_prev, lvp32, i, 0.0);
      }
      {
        const double e = (tid < K) ? get(lv, lv32, tid) : 0.0;  // K <= blockDim.x
        const double inv = 1.0 / sqrt(gd_block_sum(e * e, red));
        if (tid < K) set(lv, lv32, tid, get(lv, lv32, tid) * inv);
      }
      __syncthreads();
      int msteps = m;
      double beta_prev = 0.0;
      // three barriers a step: w_i, v_i and v_prev_i are this thread's own
      // entries (one row of the product per thread), the two sums use slots
      // 0-7 and 8-15 of `red` (each read before the step's last barrier), and
      // the last barrier orders the new v before the next step's product
      for (int j = 0; j < m; ++j) {
        if (lowp)
          gd_gemv32(Ghi, LDF, K, lv32, lw32);
        else
          gemv64(lv, lw);
        const double wi = (tid < K) ? get(lw, lw32, tid) : 0.0, vi = (tid < K) ? get(lv, lv32, tid) : 0.0;
        const double al = gd_block_sum_fresh(wi * vi, red);
        const double wn = (tid < K) ? wi - al * vi - beta_prev * get(lv_prev, lvp32, tid) : 0.0;
        const double bt = sqrt(gd_block_sum_fresh(wn * wn, red + 8));
        if (tid == 0) {
          ta[j] = al;
          tb[j] = bt;
        }
        if (!(bt > 1e-300 * fabs(al)) || j == m - 1) {  // every thread holds the same bt
          msteps = j + 1;
          break;
        }
        if (tid < K) {
          set(lv_prev, lvp32, tid, vi);
          set(lv, lv32, tid, wn / bt);
        }
        beta_prev = bt;
        __syncthreads();
      }
      __syncthreads();
      {  // largest eigenvalue of the tridiagonal: multisection at one point per thread
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < msteps; ++i) {
          const double r = (i > 0 ? fabs(tb[i - 1]) : 0.0) + (i < msteps - 1 ? fabs(tb[i]) : 0.0);
          lo = fmin(lo, ta[i] - r);
          hi = fmax(hi, ta[i] + r);
        }
        const int P = blockDim.x;  // points lo + (hi - lo) (t + 1) / (P + 1)
        for (int round = 0; round < 12 && hi - lo > 1e-16 * fmax(fabs(hi), fabs(lo)); ++round) {
          if (tid == 0) s_first = P;
          __syncthreads();
          const double x = lo + (hi - lo) * (tid + 1) / (P + 1.0);
          if (sturm_below(ta, tb, msteps, x) == msteps) atomicMin(&s_first, tid);  // x above every eigenvalue
          __syncthreads();
          const int first = s_first;  // the top eigenvalue lies in (x_{first-1}, x_first]
          const double nlo = lo + (hi - lo) * first / (P + 1.0);
          hi = lo + (hi - lo) * (first + 1) / (P + 1.0);
          lo = nlo;
          __syncthreads();
        }
        if (tid == 0) s_lmax = 0.5 * (lo + hi);
      }
      __syncthreads();
    };
    // the converged-optimum mode only needs a safe step for its support
    // iterations (the polish certifies the minimiser whatever the path): fewer
    // steps and a margin; a voxel it does not certify reruns the full count
    run_lanczos(p.kkt ? kGdLanczosKkt : kGdLanczos, mixed);
    const double nv = static_cast<double>(n);
    double lip = (n > 0) ? fmax(s_lmax / nv, 2.220446049250313e-16) : 0.0;

    // ---- 4. FISTA (src/solver/fista.rs:70-143), Gram form
    const double n_inv = (n > 0) ? 1.0 / nv : 0.0;
    double step = (n > 0) ? 1.0 / (p.kkt ? lip * kGdKktLipMargin : lip) : 0.0;
    const double alpha_v = p.alpha_v ? p.alpha_v[v] : p.alpha;
    double thr = __dmul_rn(step, alpha_v);
    // `max_it` iterations from zero, stopping early below `tol` (never with tol 0)
    auto run_fista = [&](int max_it, double tol, bool& converged) -> int {
      for (int i = tid; i < Kp; i += blockDim.x) {
        vx[i] = 0.0;
        vy[i] = 0.0;
      }
      __syncthreads();
      int it = 0;
      converged = false;
      // tol 0 (a fixed iteration count) needs no stopping test: no reductions
      const bool check = tol > 0.0;
      // with the FP64 matrix the reference rule's product reads only y's
      // nonzero entries, listed after each update (gd_gemv_nz; one more
      // barrier a step).  Measured at 300k voxels: order 8 0.909 -> 0.828 s;
      // the converged-optimum modes' 16-32 iterations from zero gained
      // nothing at order 8 and lost 5 % at order 6, so they keep the dense one.
      const bool sparse = !mixed && check && K > 96;
      const int my_sum = (tid < K) ? gd_gemv_sum_of(tid, K) : 0;
      unsigned bal[4] = {0u, 0u, 0u, 0u};
      double yn = 0.0;
      auto list_nonzeros = [&]() {  // after a barrier that follows the counts' writes
        if (tid < K && yn != 0.0) {
          const unsigned mine = my_sum == 0 ? bal[0] : (my_sum == 1 ? bal[1] : (my_sum == 2 ? bal[2] : bal[3]));
          int off = __popc(mine & ((1u << lane) - 1u));
          for (int w = 0; w < warp; ++w) off += gd_wcnt[w][my_sum];
          nzi[my_sum * L.LC + off] = tid;
          nzv[my_sum * L.LC + off] = yn;
        }
        if (tid < 4) {
          int t = 0;
          for (int w = 0; w < 8; ++w) t += gd_wcnt[w][tid];
          gd_ncnt[tid] = t;
        }
      };
      if (tid < 4) gd_ncnt[tid] = 0;  // y = 0
      __syncthreads();
      double mom_next = (max_it > 0) ? p.mom[0] : 0.0;
      while (n > 0 && it < max_it) {
        const double mom = mom_next;
        if (it + 1 < max_it) mom_next = p.mom[it + 1];  // in flight during the product
        if (sparse)
          gd_gemv_nz(G, LDG, K, gd_ncnt, nzv, nzi, L.LC, vgy);
        else
          gemv64(vy, vgy);
        __syncthreads();
        double dx2 = 0.0, xn2 = 0.0;
        yn = 0.0;
        if (tid < K) {
          const int i = tid;
          const double grad = __dmul_rn(__dsub_rn(vgy[i], vb[i]), n_inv);
          const double cand = __dsub_rn(vy[i], __dmul_rn(step, grad));
          double sv;
          if (cand > thr)
            sv = __dsub_rn(cand, thr);
          else if (cand < -thr)
            sv = __dadd_rn(cand, thr);
          else
            sv = 0.0;
          const double xn = p.non_negative ? fmax(sv, 0.0) : sv;
          const double d = __dsub_rn(xn, vx[i]);
          yn = __dadd_rn(xn, __dmul_rn(mom, d));
          vy[i] = yn;
          vx[i] = xn;
          dx2 = __dmul_rn(d, d);
          xn2 = __dmul_rn(xn, xn);
        }
        if (sparse) {
          const bool nz = tid < K && yn != 0.0;
#pragma unroll
          for (int r = 0; r < 4; ++r) bal[r] = __ballot_sync(kFull, nz && my_sum == r);
          if (lane < 4) gd_wcnt[warp][lane] = __popc(lane == 0 ? bal[0] : (lane == 1 ? bal[1] : (lane == 2 ? bal[2] : bal[3])));
        }
        if (!check) {
          ++it;
          __syncthreads();  // the new y before the next product
          if (sparse) {
            list_nonzeros();
            __syncthreads();
          }
          continue;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          dx2 += __shfl_xor_sync(kFull, dx2, o);
          xn2 += __shfl_xor_sync(kFull, xn2, o);
        }
        if (lane == 0) {
          red[2 * warp] = dx2;
          red[2 * warp + 1] = xn2;
        }
        __syncthreads();
        if (sparse) list_nonzeros();
        double sdx = 0.0, sxn = 0.0;
        for (int w = 0; w < 8; ++w) {
          sdx += red[2 * w];
          sxn += red[2 * w + 1];
        }
        ++it;
        const double rel = sqrt(sdx) / fmax(sqrt(sxn), 1e-12);
        // red is next written after the next iteration's first barrier, which
        // every thread reaches only once it has read it; the lists need one
        if (sparse) __syncthreads();
        if (rel < tol) {
          converged = true;
          break;
        }
      }
      __syncthreads();  // the polish reuses red and the vectors as scratch
      return it;
    };
    // the mixed mode's support iterations: the same update in FP32 on G_v's
    // hi plane, a fixed count, x_i and b_i in the registers of thread i and y
    // in FP32 in y's slot; x is left in FP64 in vx for the polish
    auto run_fista32 = [&](int iters) -> int {
      float* y32 = reinterpret_cast<float*>(vy);
      float* gy32 = reinterpret_cast<float*>(vgy);
      const float step32 = static_cast<float>(step), thr32 = static_cast<float>(thr);
      const float ninv32 = static_cast<float>(n_inv);
      const float bi = (tid < K) ? static_cast<float>(vb[tid]) : 0.f;
      float xi = 0.f;
      for (int i = tid; i < Kp; i += blockDim.x) y32[i] = 0.f;
      __syncthreads();
      double mom_next = (iters > 0) ? p.mom[0] : 0.0;
      for (int it = 0; n > 0 && it < iters; ++it) {
        const float mom = static_cast<float>(mom_next);
        if (it + 1 < iters) mom_next = p.mom[it + 1];
        gd_gemv32(Ghi, LDF, K, y32, gy32);
        __syncthreads();
        if (tid < K) {
          const float grad = (gy32[tid] - bi) * ninv32;
          const float cand = y32[tid] - step32 * grad;
          float sv = 0.f;
          if (cand > thr32)
            sv = cand - thr32;
          else if (cand < -thr32)
            sv = cand + thr32;
          const float xn = p.non_negative ? fmaxf(sv, 0.f) : sv;
          y32[tid] = xn + mom * (xn - xi);
          xi = xn;
        }
        __syncthreads();  // the new y before the next product
      }
      for (int i = tid; i < Kp; i += blockDim.x) vx[i] = (i == tid && i < K) ? static_cast<double>(xi) : 0.0;
      __syncthreads();
      return n > 0 ? iters : 0;
    };
    bool converged = false;
    int it = (p.kkt && mixed) ? run_fista32(p.kkt_iters)
                              : run_fista(p.kkt ? p.kkt_iters : p.max_iter, p.kkt ? 0.0 : p.tol, converged);
    double kkt_val = 0.0;
    int rounds = 0;
    if (p.kkt) {
      // polish on G_v by warp 0, its scratch in the vectors FISTA no longer
      // needs (y, G y, the Lanczos vectors and the reduction / tridiagonal
      // slots: 5 Kp + 160 doubles; b and x stay)
      constexpr int RPL = (8 * MT + 31) / 32;
      const int cap = (K > 72) ? 32 : 24;
      if (warp == 0 && n > 0) {
        double* T = vy;
        double* zw = T + cap * (cap + 1) / 2;
        double* zj = zw + cap;
        int* sidx = reinterpret_cast<int*>(zj + Kp);
        int* fl = sidx + Kp;
        double c[RPL];
#pragma unroll
        for (int qq = 0; qq < RPL; ++qq) {
          const int j = lane + 32 * qq;
          const double x0 = j < K ? vx[j] : 0.0;
          int f = x0 > 0.0 ? 1 : (x0 < 0.0 ? -1 : 0);
          if (p.non_negative && f < 0) f = 0;
          c[qq] = f != 0 ? x0 : 0.0;
          if (j < Kp) fl[j] = f;
        }
        __syncwarp();
        bool ovf = false;
        const bool cert =
            mixed ? polish_warp<RPL, 1>(GramHiLo{Ghi, Glo, LDF}, K, Kp, cap, vb, fl, c, T, zw, zj, sidx, gd_tri, nv,
                                        n_inv, alpha_v, p.non_negative, p.kappa, p.kkt_rounds, rounds, kkt_val, ovf)
                  : polish_warp<RPL, 1>(GramDense{G, LDG}, K, Kp, cap, vb, fl, c, T, zw, zj, sidx, gd_tri, nv,
                                        n_inv, alpha_v, p.non_negative, p.kappa, p.kkt_rounds, rounds, kkt_val, ovf);
        if (cert) {
#pragma unroll
          for (int qq = 0; qq < RPL; ++qq)
            if (lane + 32 * qq < K) vx[lane + 32 * qq] = c[qq];
        }
        if (lane == 0) {
          s_first = cert ? 1 : 0;
          s_lmax = cert ? kkt_val : 0.0;
          ta[0] = static_cast<double>(rounds);
        }
      }
      __syncthreads();
      const bool cert = n > 0 && s_first == 1;
      rounds = (n > 0) ? static_cast<int>(ta[0]) : 0;
      kkt_val = s_lmax;
      __syncthreads();
      if (!cert && n > 0) {  // the reference FISTA from zero, reported uncertified
        run_lanczos(kGdLanczos, false);  // the reference's step, from the full Lanczos count
        lip = fmax(s_lmax / nv, 2.220446049250313e-16);
        step = 1.0 / lip;
        thr = __dmul_rn(step, alpha_v);
        bool conv_ref = false;
        it += run_fista(p.max_iter, p.tol, conv_ref);
      }
      converged = cert || n == 0;
      if (tid == 0) {
        if (p.kkt_out) p.kkt_out[v] = cert || n == 0 ? kkt_val : __longlong_as_double(0x7ff8000000000000ll);
        if (!cert && n > 0 && p.n_uncertified) atomicAdd(p.n_uncertified, 1ull);
        if (p.round_total) atomicAdd(p.round_total, static_cast<unsigned long long>(rounds));
      }
    }
    for (int i = tid; i < K; i += blockDim.x) p.X[v * K + i] = vx[i];
    if (tid == 0) {
      p.iters[v] = static_cast<uint32_t>(it + rounds);
      p.conv[v] = converged ? 1 : 0;
      if (p.lipschitz) p.lipschitz[v] = lip;
      if (p.n_rows) p.n_rows[v] = n;
    }
    executed += static_cast<unsigned long long>(it);
    __syncthreads();
  }
  if (tid == 0 && p.iter_total) atomicAdd(p.iter_total, executed);
}

}  // namespace csd
