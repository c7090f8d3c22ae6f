// setup_kernels.cuh - once-per-gradient-table kernels.
//
// Everything the reference builds once per fit before its voxel loop
// (src/fit.rs:718-795): the SHORE design matrix M, the Gram matrix G = M^T M,
// the FISTA Lipschitz constant L = sigma_max(M)^2 / n (src/solver/fista.rs:
// 38-63), the Cholesky factor of the Tikhonov normal matrix
// (src/solver/tikhonov.rs:26-52) and the packed operand tiles the solve
// kernels read.  All FP64.  These run on K x K or N x K data (K <= 145,
// N ~ 10^2..10^3), so they are latency kernels: one thread per entry or one
// CTA for a factorisation.
#pragma once

#include "device_math.cuh"

namespace csd {

// Column index -> (n, l, k-in-block) of the BrainSuite SHORE order
// (src/basis/shore.rs:29-44, 158-175).
__device__ __forceinline__ void col_to_nlk(int radial_order, int col, int* n_out, int* l_out,
                                           int* k_out) {
  int c = 0;
  for (int n = 0; n <= radial_order; ++n) {
    for (int l = 0; l <= n; l += 2) {
      const int bs = 2 * l + 1;
      if (col < c + bs) {
        *n_out = n;
        *l_out = l;
        *k_out = col - c;
        return;
      }
      c += bs;
    }
  }
  *n_out = *l_out = *k_out = 0;
}

// M[i, col] = R_nl(q_i) * Y^BS_{l,k}(theta_i, phi_i), row-major N x K
// (src/basis/shore.rs:122-178).  `qdenom` = 4 pi^2 tau computed on the host
// in the reference's order (src/qspace.rs:136-149).
__global__ void k_design(const double* __restrict__ bvals, const double* __restrict__ bvecs,
                         int N, int K, int radial_order, double zeta, double qdenom,
                         double b0_threshold, double* __restrict__ M) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<long long>(N) * K) return;
  const int i = static_cast<int>(idx / K);
  const int col = static_cast<int>(idx % K);
  const double b = bvals[i];
  const double q = (b <= b0_threshold) ? 0.0 : sqrt(b / qdenom);
  const double x = bvecs[3 * i] * q, y = bvecs[3 * i + 1] * q, z = bvecs[3 * i + 2] * q;
  // cart2sphere (src/math.rs:157-166); a NaN azimuth becomes 0 (shore.rs:134).
  const double r = sqrt(x * x + y * y + z * z);
  double theta = atan2(y, x);
  const double phi = (r > 0.0) ? acos(fmin(fmax(z / r, -1.0), 1.0)) : 0.0;
  if (isnan(theta)) theta = 0.0;
  int n, l, k;
  col_to_nlk(radial_order, col, &n, &l, &k);
  M[idx] = dev_shore_radial(n, l, r, zeta) * dev_brainsuite_sh(l, k, theta, phi);
}

// Padded Gram matrix G = M^T M (Kp x Kp, zeros outside K x K) and the
// regularised Tikhonov normal matrix A = G + lambda_N N + lambda_L L
// (src/solver/tikhonov.rs:34-46, src/basis/shore.rs:180-195).
__global__ void k_gram(const double* __restrict__ M, int N, int K, int Kp, int radial_order,
                       double lambda_n, double lambda_l, double* __restrict__ G,
                       double* __restrict__ A) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= Kp * Kp) return;
  const int i = idx / Kp, j = idx % Kp;
  double acc = 0.0;
  if (i < K && j < K) {
    for (int r = 0; r < N; ++r) acc += M[static_cast<size_t>(r) * K + i] * M[static_cast<size_t>(r) * K + j];
  }
  G[idx] = acc;
  if (A) {
    double a = acc;
    if (i == j && i < K) {
      int n, l, kk;
      col_to_nlk(radial_order, i, &n, &l, &kk);
      const double nn = static_cast<double>(n * (n + 1));
      const double ll = static_cast<double>(l * (l + 1));
      a += lambda_n * (nn * nn);
      a += lambda_l * (ll * ll);
    }
    A[idx] = a;
  }
}

// lambda_max(G) by power iteration with a Rayleigh-quotient estimate, one
// CTA.  The SHORE Gram matrix has its top two eigenvalues within ~5 %, so the
// loop runs until the quotient has not moved for 64 consecutive steps
// to within 4 ulp (quadratic convergence of the quotient makes that machine
// precision), with a hard cap.  Output: lipschitz = max(lambda_max / n, DBL_EPSILON)
// (src/solver/fista.rs:96-109).
__global__ void k_lipschitz(const double* __restrict__ G, int Kp, int N, int max_steps,
                            double* __restrict__ out_lipschitz, double* __restrict__ out_lambda) {
  extern __shared__ double sm[];
  double* sG = sm;                // Kp * Kp
  double* v = sG + Kp * Kp;       // Kp
  double* w = v + Kp;             // Kp
  __shared__ double red[32];
  __shared__ double s_lambda;
  __shared__ int s_stable;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < Kp * Kp; i += nt) sG[i] = G[i];
  // Deterministic start vector with no special structure.
  for (int i = tid; i < Kp; i += nt) v[i] = 1.0 + 0.37 * static_cast<double>((i * 7919) % 101) / 101.0;
  if (tid == 0) {
    s_lambda = 0.0;
    s_stable = 0;
  }
  __syncthreads();
  auto block_sum = [&](double x) -> double {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((tid & 31) == 0) red[tid >> 5] = x;
    __syncthreads();
    double s = 0.0;
    if (tid < 32) {
      s = (tid < (nt + 31) / 32) ? red[tid] : 0.0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    __syncthreads();
    if (tid == 0) red[0] = s;
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
  };
  // normalise start
  {
    double p = 0.0;
    for (int i = tid; i < Kp; i += nt) p += v[i] * v[i];
    const double nrm = sqrt(block_sum(p));
    for (int i = tid; i < Kp; i += nt) v[i] /= nrm;
    __syncthreads();
  }
  for (int step = 0; step < max_steps; ++step) {
    double p = 0.0;
    for (int i = tid; i < Kp; i += nt) {
      double acc = 0.0;
      for (int k = 0; k < Kp; ++k) acc += sG[i * Kp + k] * v[k];
      w[i] = acc;
      p += acc * v[i];
    }
    const double lam = block_sum(p);
    double q = 0.0;
    for (int i = tid; i < Kp; i += nt) q += w[i] * w[i];
    const double wn = sqrt(block_sum(q));
    for (int i = tid; i < Kp; i += nt) v[i] = w[i] / wn;
    if (tid == 0) {
      s_stable = (fabs(lam - s_lambda) <= 4.0e-16 * fabs(lam)) ? s_stable + 1 : 0;
      s_lambda = lam;
    }
    __syncthreads();
    if (s_stable >= 64) break;
  }
  if (tid == 0) {
    const double lam = s_lambda;
    const double sigma = sqrt(fmax(lam, 0.0));
    const double lip = sigma * sigma * (1.0 / static_cast<double>(N));
    *out_lipschitz = fmax(lip, 2.220446049250313e-16);
    if (out_lambda) *out_lambda = lam;
  }
}

// In-place right-looking Cholesky A = L L^T of the leading K x K block of a
// Kp x Kp matrix, one CTA.  Writes 0 to *ok_out if A is not positive definite
// (the reference panics there, src/solver/tikhonov.rs:44).  The accumulation
// order of every entry is the left-looking order k = 0, 1, ..., so results
// match a sequential LL^T factorisation.
__global__ void k_cholesky(double* __restrict__ A, int K, int Kp, int* __restrict__ ok_out) {
  extern __shared__ double sA[];
  __shared__ int s_ok;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < K * K; i += nt) sA[i] = A[(i / K) * Kp + (i % K)];
  if (tid == 0) s_ok = 1;
  __syncthreads();
  for (int j = 0; j < K; ++j) {
    if (tid == 0) {
      const double d = sA[j * K + j];
      if (!(d > 0.0)) s_ok = 0;
      sA[j * K + j] = sqrt(fmax(d, 0.0));
    }
    __syncthreads();
    if (!s_ok) break;
    const double ljj = sA[j * K + j];
    for (int i = j + 1 + tid; i < K; i += nt) sA[i * K + j] = __ddiv_rn(sA[i * K + j], ljj);
    __syncthreads();
    const int rem = K - j - 1;
    for (int t = tid; t < rem * rem; t += nt) {
      const int i = j + 1 + t / rem, k = j + 1 + t % rem;
      if (k <= i) sA[i * K + k] = __dsub_rn(sA[i * K + k], __dmul_rn(sA[i * K + j], sA[k * K + j]));
    }
    __syncthreads();
  }
  for (int i = tid; i < Kp * Kp; i += nt) {
    const int r = i / Kp, c = i % Kp;
    A[i] = (r < K && c < K && c <= r) ? sA[r * K + c] : 0.0;
  }
  if (tid == 0) *ok_out = s_ok;
}

// Pack the symmetric Gram matrix into m8n8k4 DMMA A-operand tiles:
// frag[(mt * KT + kt) * 32 + lane] = G[8 mt + lane / 4][4 kt + lane % 4].
// One 256-byte line per (mt, kt) tile, read conflict-free by a warp.
__global__ void k_pack_gfrag(const double* __restrict__ G, int Kp, double* __restrict__ frag) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int MT = Kp / 8, KT = Kp / 4;
  if (idx >= MT * KT * 32) return;
  const int lane = idx & 31, tile = idx >> 5;
  const int mt = tile / KT, kt = tile % KT;
  frag[idx] = G[(8 * mt + lane / 4) * Kp + 4 * kt + (lane & 3)];
}

// Rows of an N x K matrix copied into N x Kp rows with zero padding.
__global__ void k_pad_rows(const double* __restrict__ src, int N, int K, int Kp, double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * Kp) return;
  const int r = i / Kp, c = i % Kp;
  dst[i] = c < K ? src[r * K + c] : 0.0;
}

}  // namespace csd
