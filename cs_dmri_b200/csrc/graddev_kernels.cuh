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
//   2. G_v = M_v^T M_v on the FP64 tensor cores (DMMA m8n8k4): the design is
//      generated 32 rows at a time into shared memory (radial factors per
//      (n, l) and SH values per (l, m), multiplied per column), each warp
//      accumulating a fixed set of 8 x 8 tiles of the upper triangle in
//      registers; b_v = M_v^T s_v alongside;
//   3. lambda_max(G_v) by Lanczos (a fixed number of steps, the largest Ritz
//      value by multisection of the tridiagonal's Sturm count across a warp);
//   4. FISTA in the Gram form with G_v in shared memory (one warp per row of
//      the product, lanes over the columns), the reference's update and
//      stopping rule.
#pragma once

namespace csd {

constexpr int kGdChunk = 32;       // design rows per Gram chunk
constexpr int kGdLanczos = 48;     // Lanczos steps (capped at K)

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
};

// Shared-memory plan (doubles unless noted), shared by host and device.
struct GdLayout {
  int K, Kp, LDM, NL, NSH;
  size_t g, vec, red, tri, rows, colmap, total_bytes;
  __host__ __device__ GdLayout(int K_, int radial_order, int N) {
    K = K_;
    Kp = 8 * ((K + 7) / 8);
    LDM = Kp + 4;  // chunk row stride: conflict-free fragment loads
    NL = 0;
    for (int n = 0; n <= radial_order; ++n) NL += n / 2 + 1;
    NSH = (radial_order / 2 + 1) * (radial_order + 1);
    const size_t chunk = static_cast<size_t>(kGdChunk) * (LDM + NL + NSH + 4);
    const size_t gsize = static_cast<size_t>(K) * K > chunk ? static_cast<size_t>(K) * K : chunk;
    g = 0;
    vec = (gsize + 1) & ~static_cast<size_t>(1);           // b, x, y, gy, v_prev, v, w: 7 * Kp
    red = vec + 7 * static_cast<size_t>(Kp);                 // 16 reduction slots
    tri = red + 16;                                          // Lanczos alpha / beta: 2 * 64
    rows = tri + 128;                                        // N ints, then the column map (2 K ints)
    colmap = rows + (static_cast<size_t>(N) + 1) / 2;
    total_bytes = 8 * (colmap + static_cast<size_t>(K) + 1);
  }
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
__global__ void __launch_bounds__(256, 1) k_graddev_fit(GraddevParams p) {
  constexpr int NT = MT * (MT + 1) / 2;  // upper-triangle tiles of G
  constexpr int TPW = (NT + 7) / 8;      // tiles per warp
  constexpr int RPL = (8 * MT + 31) / 32;
  extern __shared__ __align__(16) double gd_smem[];
  const GdLayout L(p.K, p.radial_order, p.N);
  const int K = p.K, Kp = L.Kp, LDM = L.LDM, NL = L.NL, NSH = L.NSH, N = p.N;
  double* G = gd_smem + L.g;
  double* Mc = G;                                  // chunk: kGdChunk x LDM (aliases G while it is built)
  double* rad = Mc + kGdChunk * LDM;               // kGdChunk x NL
  double* shv = rad + kGdChunk * NL;               // kGdChunk x NSH
  double* geo = shv + kGdChunk * NSH;              // kGdChunk x 4: r, theta, phi, signal
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
  int* rows = reinterpret_cast<int*>(gd_smem + L.rows);
  int* col_nl = reinterpret_cast<int*>(gd_smem + L.colmap);
  int* col_lk = col_nl + K;
  __shared__ int64_t s_v;
  __shared__ int s_n;
  __shared__ double s_lmax;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, q = lane & 3;

  // column -> (radial block, SH entry) maps, once per CTA
  for (int col = tid; col < K; col += blockDim.x) {
    int n, l, k;
    col_to_nlk(p.radial_order, col, &n, &l, &k);
    int nl = 0;
    for (int nn = 0; nn < n; ++nn) nl += nn / 2 + 1;
    col_nl[col] = nl + l / 2;
    int lk = 0;
    for (int ll = 0; ll < l; ll += 2) lk += 2 * ll + 1;
    col_lk[col] = lk + k;
  }
  // this warp's tiles of the upper triangle, packed (mt << 8) | nt; nt >= MT
  // marks an unused slot
  int tile[TPW];
#pragma unroll
  for (int s = 0; s < TPW; ++s) {
    const int tau = warp + 8 * s;
    int mt = 0, rem = tau;
    while (mt < MT && rem >= MT - mt) {
      rem -= MT - mt;
      ++mt;
    }
    tile[s] = (mt << 8) | (mt + rem);
  }
  __syncthreads();

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
    double acc[TPW][2];
#pragma unroll
    for (int s = 0; s < TPW; ++s) acc[s][0] = acc[s][1] = 0.0;
    for (int c0 = 0; c0 < n; c0 += kGdChunk) {
      if (tid < kGdChunk) {
        const int r = c0 + tid;
        double rr = 0.0, th = 0.0, ph = 0.0, sig = 0.0;
        if (r < n) {
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
          rr = sqrt(x * x + y * y + z * z);
          th = atan2(y, x);
          ph = (rr > 0.0) ? acos(fmin(fmax(z / rr, -1.0), 1.0)) : 0.0;
          if (isnan(th)) th = 0.0;
          sig = static_cast<double>(p.S[v * N + i]);
        }
        geo[4 * tid] = rr;
        geo[4 * tid + 1] = th;
        geo[4 * tid + 2] = ph;
        geo[4 * tid + 3] = (r < n) ? sig : 0.0;
      }
      __syncthreads();
      for (int task = tid; task < kGdChunk * (NL + NSH); task += blockDim.x) {
        const int t = task / (NL + NSH), j = task % (NL + NSH);
        const bool ok = c0 + t < n;
        if (j < NL) {
          int nn = 0, rem = j;
          while (rem >= nn / 2 + 1) {
            rem -= nn / 2 + 1;
            ++nn;
          }
          rad[t * NL + j] = ok ? dev_shore_radial(nn, 2 * rem, geo[4 * t], p.zeta) : 0.0;
        } else {
          int l = 0, rem = j - NL;
          while (rem >= 2 * l + 1) {
            rem -= 2 * l + 1;
            l += 2;
          }
          shv[t * NSH + (j - NL)] = ok ? dev_brainsuite_sh(l, rem, geo[4 * t + 1], geo[4 * t + 2]) : 0.0;
        }
      }
      __syncthreads();
      for (int task = tid; task < kGdChunk * Kp; task += blockDim.x) {
        const int t = task / Kp, col = task % Kp;
        Mc[t * LDM + col] = (col < K) ? rad[t * NL + col_nl[col]] * shv[t * NSH + col_lk[col]] : 0.0;
      }
      __syncthreads();
      for (int col = tid; col < K; col += blockDim.x) {
        double a = vb[col];
        for (int t = 0; t < kGdChunk; ++t) a = __dadd_rn(a, __dmul_rn(Mc[t * LDM + col], geo[4 * t + 3]));
        vb[col] = a;
      }
#pragma unroll 1
      for (int kk = 0; kk < kGdChunk / 4; ++kk) {
        const double* rowp = Mc + (4 * kk + q) * LDM + g;
#pragma unroll
        for (int s = 0; s < TPW; ++s)
          if ((tile[s] & 0xff) < MT) dmma_m8n8k4(acc[s][0], acc[s][1], rowp[8 * (tile[s] >> 8)], rowp[8 * (tile[s] & 0xff)]);
      }
      __syncthreads();
    }
    // G from the tiles (and the mirror of each off-diagonal tile)
#pragma unroll
    for (int s = 0; s < TPW; ++s) {
      const int mt = tile[s] >> 8, nt = tile[s] & 0xff;
      if (nt >= MT) continue;
      const int i = 8 * mt + g;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = 8 * nt + 2 * q + e;
        if (i < K && j < K) {
          G[i * K + j] = acc[s][e];
          if (mt != nt) G[j * K + i] = acc[s][e];  // a diagonal tile holds both halves itself
        }
      }
    }
    __syncthreads();

    // ---- 3. lambda_max(G) by Lanczos
    const int m = min(K, kGdLanczos);
    {
      double nrm = 0.0;
      for (int i = tid; i < Kp; i += blockDim.x) {
        const double e = (i < K) ? 1.0 + 0.5 * sin(1.7 * i + 0.3) : 0.0;  // fixed start vector
        lv[i] = e;
        lv_prev[i] = 0.0;
      }
      __syncthreads();
      for (int i = 0; i < K; ++i) nrm += lv[i] * lv[i];  // every thread, same order
      const double inv = 1.0 / sqrt(nrm);
      __syncthreads();
      for (int i = tid; i < K; i += blockDim.x) lv[i] *= inv;
      __syncthreads();
    }
    int msteps = m;
    double beta_prev = 0.0;
    for (int j = 0; j < m; ++j) {
      // w = G v
      double vl[RPL];
#pragma unroll
      for (int c = 0; c < RPL; ++c) vl[c] = (lane + 32 * c < K) ? lv[lane + 32 * c] : 0.0;
      for (int i = warp; i < K; i += 8) {
        double a = 0.0;
#pragma unroll
        for (int c = 0; c < RPL; ++c)
          if (lane + 32 * c < K) a = fma(G[i * K + lane + 32 * c], vl[c], a);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
        if (lane == 0) lw[i] = a;
      }
      __syncthreads();
      double al = 0.0;
      for (int i = 0; i < K; ++i) al += lw[i] * lv[i];
      __syncthreads();
      for (int i = tid; i < K; i += blockDim.x) lw[i] = lw[i] - al * lv[i] - beta_prev * lv_prev[i];
      __syncthreads();
      double bt = 0.0;
      for (int i = 0; i < K; ++i) bt += lw[i] * lw[i];
      bt = sqrt(bt);
      if (tid == 0) {
        ta[j] = al;
        tb[j] = bt;
      }
      if (!(bt > 1e-300 * fabs(al)) || j == m - 1) {
        msteps = j + 1;
        __syncthreads();
        break;
      }
      for (int i = tid; i < K; i += blockDim.x) {
        lv_prev[i] = lv[i];
        lv[i] = lw[i] / bt;
      }
      beta_prev = bt;
      __syncthreads();
    }
    if (warp == 0) {  // largest eigenvalue of the tridiagonal: 32-point multisection
      double lo = 1e300, hi = -1e300;
      for (int i = 0; i < msteps; ++i) {
        const double r = (i > 0 ? fabs(tb[i - 1]) : 0.0) + (i < msteps - 1 ? fabs(tb[i]) : 0.0);
        lo = fmin(lo, ta[i] - r);
        hi = fmax(hi, ta[i] + r);
      }
      for (int round = 0; round < 24 && hi - lo > 1e-16 * fmax(fabs(hi), fabs(lo)); ++round) {
        const double x = lo + (hi - lo) * (lane + 1) / 33.0;
        const bool all_below = sturm_below(ta, tb, msteps, x) == msteps;  // x above every eigenvalue
        const unsigned bal = __ballot_sync(kFull, all_below);
        const int first = bal ? __ffs(bal) - 1 : 32;  // lowest point above the top eigenvalue
        const double nlo = lo + (hi - lo) * first / 33.0;
        const double nhi = lo + (hi - lo) * (first + 1) / 33.0;
        lo = __shfl_sync(kFull, nlo, 0);
        hi = __shfl_sync(kFull, nhi, 0);
      }
      if (lane == 0) s_lmax = 0.5 * (lo + hi);
    }
    __syncthreads();
    const double nv = static_cast<double>(n);
    const double lip = (n > 0) ? fmax(s_lmax / nv, 2.220446049250313e-16) : 0.0;

    // ---- 4. FISTA (src/solver/fista.rs:70-143), Gram form
    const double n_inv = (n > 0) ? 1.0 / nv : 0.0;
    const double step = (n > 0) ? 1.0 / lip : 0.0;
    const double thr = __dmul_rn(step, p.alpha_v ? p.alpha_v[v] : p.alpha);
    for (int i = tid; i < Kp; i += blockDim.x) {
      vx[i] = 0.0;
      vy[i] = 0.0;
    }
    __syncthreads();
    int it = 0;
    bool converged = false;
    while (n > 0 && it < p.max_iter) {
      double yl[RPL];
#pragma unroll
      for (int c = 0; c < RPL; ++c) yl[c] = (lane + 32 * c < K) ? vy[lane + 32 * c] : 0.0;
      for (int i = warp; i < K; i += 8) {
        double a = 0.0;
#pragma unroll
        for (int c = 0; c < RPL; ++c)
          if (lane + 32 * c < K) a = fma(G[i * K + lane + 32 * c], yl[c], a);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
        if (lane == 0) vgy[i] = a;
      }
      __syncthreads();
      const double mom = p.mom[it];
      double dx2 = 0.0, xn2 = 0.0;
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
        vy[i] = __dadd_rn(xn, __dmul_rn(mom, d));
        vx[i] = xn;
        dx2 = __dmul_rn(d, d);
        xn2 = __dmul_rn(xn, xn);
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
      double sdx = 0.0, sxn = 0.0;
      for (int w = 0; w < 8; ++w) {
        sdx += red[2 * w];
        sxn += red[2 * w + 1];
      }
      ++it;
      const double rel = sqrt(sdx) / fmax(sqrt(sxn), 1e-12);
      __syncthreads();  // red and vy are rewritten next iteration
      if (rel < p.tol) {
        converged = true;
        break;
      }
    }
    for (int i = tid; i < K; i += blockDim.x) p.X[v * K + i] = vx[i];
    if (tid == 0) {
      p.iters[v] = static_cast<uint32_t>(it);
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
