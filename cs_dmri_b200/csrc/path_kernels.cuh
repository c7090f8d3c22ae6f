// path_kernels.cuh - per-voxel alpha strategies on the device.
//
// AlphaStrategy (src/solver/alpha.rs:195-318) picks alpha per voxel:
//   AlphaMaxRatio   alpha = alpha_max * ratio
//   PathBic         a warm-started descending log path of alphas, keep the
//                   point of minimum BIC (ties to the larger alpha)
//   PathL2Anchored  same path, keep the first (largest-alpha) point whose
//                   RSS <= (1 + slack) RSS_L2, else the point of minimum RSS
// with alpha_max = ||M^T s||_inf / n and the zero result for alpha_max == 0.
// The path is walked one point at a time over the whole volume: each point is
// one FISTA launch over the voxels still in play, warm-started in place from
// the previous point (fista.rs:164-178), then one residual pass and the
// selection update below.  Under PathL2Anchored a voxel leaves the work list
// as soon as it is selected: the later points of its path cannot change the
// result, so they are not computed.
#pragma once

#include <cstdint>

namespace csd {

// alpha_max_v = max_k |b_v[k]| / n (src/solver/alpha.rs:47-53); zero flag.
__global__ void k_alpha_max(const double* __restrict__ B, int64_t V, int K, int Kp, int N,
                            double* __restrict__ amax, uint8_t* __restrict__ zero) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  double m = 0.0;
  for (int k = 0; k < K; ++k) m = fmax(m, fabs(B[v * Kp + k]));
  const double a = m / static_cast<double>(N);
  amax[v] = a;
  zero[v] = (a == 0.0) ? 1 : 0;
}

// alpha_v = alpha_max_v * ratio (src/solver/alpha.rs:229-236).
__global__ void k_alpha_ratio(const double* __restrict__ amax, int64_t V, double ratio,
                              double* __restrict__ alpha) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  alpha[v] = amax[v] * ratio;
}

// Point i of log_path(alpha_max_v, n, eps) (src/solver/alpha.rs:57-69) for
// the voxels of `list`.
__global__ void k_path_alpha(const double* __restrict__ amax, const int64_t* __restrict__ list,
                             int64_t n_work, int i, int n, double eps,
                             double* __restrict__ alpha) {
  const int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w >= n_work) return;
  const int64_t v = list[w];
  const double lmax = log(amax[v]);
  const double lmin = log(amax[v] * eps);
  const double t = static_cast<double>(i) / static_cast<double>(n - 1);
  alpha[v] = exp(lmax + t * (lmin - lmax));
}

struct PathState {
  double* best;        // V: best BIC (PathBic) or best RSS (L2 fallback)
  uint8_t* selected;   // V: PathL2Anchored point chosen
  uint8_t* active;     // V: still on the path (work-list flag)
  double* alpha_sel;   // V
  uint32_t* it_sel;    // V
  uint8_t* conv_sel;   // V
  double* alpha_fb;    // V
  uint32_t* it_fb;     // V
  uint8_t* conv_fb;    // V
  int8_t* copy_code;   // V: 0 none, 1 -> Xsel, 2 -> Xfb (this point)
};

// Selection update after path point `i` for the voxels of `list`.
// mode 2 = PathBic (bic_argmin, alpha.rs:107-128),
// mode 3 = PathL2Anchored (l2_anchored_argmax, alpha.rs:140-165).
__global__ void k_path_update(int mode, const int64_t* __restrict__ list, int64_t n_work, int N,
                              const double* __restrict__ resid, const int* __restrict__ nnz,
                              const double* __restrict__ alpha, const uint32_t* __restrict__ iters,
                              const uint8_t* __restrict__ conv, const double* __restrict__ rss_l2,
                              double slack, PathState s) {
  const int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w >= n_work) return;
  const int64_t v = list[w];
  const double rss = resid[v] * resid[v];
  int8_t code = 0;
  if (mode == 2) {
    const double n = static_cast<double>(N);
    const double rc = fmax(rss, 2.2250738585072014e-308);
    const double b = n * log(rc / n) + log(n) * static_cast<double>(nnz[v]);
    if (b < s.best[v]) {
      s.best[v] = b;
      s.alpha_sel[v] = alpha[v];
      s.it_sel[v] = iters[v];
      s.conv_sel[v] = conv[v];
      code = 1;
    }
  } else {
    const double thr = (1.0 + slack) * rss_l2[v];
    if (rss <= thr) {
      s.selected[v] = 1;
      s.active[v] = 0;
      s.alpha_sel[v] = alpha[v];
      s.it_sel[v] = iters[v];
      s.conv_sel[v] = conv[v];
      code = 1;
    } else if (rss < s.best[v]) {
      s.best[v] = rss;
      s.alpha_fb[v] = alpha[v];
      s.it_fb[v] = iters[v];
      s.conv_fb[v] = conv[v];
      code = 2;
    }
  }
  s.copy_code[v] = code;
}

// Copy the coefficients of this path point to the selected / fallback store.
__global__ void k_path_copy(const int64_t* __restrict__ list, int64_t n_work, int Kp,
                            const int8_t* __restrict__ code, const double* __restrict__ X,
                            double* __restrict__ Xsel, double* __restrict__ Xfb) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= n_work * Kp) return;
  const int64_t v = list[e / Kp];
  const int k = static_cast<int>(e % Kp);
  const int8_t c = code[v];
  if (c == 1)
    Xsel[v * Kp + k] = X[v * Kp + k];
  else if (c == 2)
    Xfb[v * Kp + k] = X[v * Kp + k];
}

// PathL2Anchored voxels that never met the slack bound take their
// minimum-RSS point.
__global__ void k_path_finalize(int64_t V, int Kp, const uint8_t* __restrict__ zero, PathState s,
                                const double* __restrict__ Xfb, double* __restrict__ Xsel) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= V * Kp) return;
  const int64_t v = e / Kp;
  const int k = static_cast<int>(e % Kp);
  if (zero[v] || s.selected[v]) return;
  Xsel[v * Kp + k] = Xfb[v * Kp + k];
  if (k == 0) {
    s.alpha_sel[v] = s.alpha_fb[v];
    s.it_sel[v] = s.it_fb[v];
    s.conv_sel[v] = s.conv_fb[v];
  }
}

// Zero-voxel results (alpha 0, 0 iterations, converged) for the maps.
__global__ void k_zero_voxels(int64_t V, const uint8_t* __restrict__ zero,
                              double* __restrict__ alpha, uint32_t* __restrict__ iters,
                              uint8_t* __restrict__ conv) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V || !zero[v]) return;
  alpha[v] = 0.0;
  iters[v] = 0;
  conv[v] = 1;
}

// Flag array -> list of positions (u8 flags over V), via the mask compaction
// kernels; this builds the u8 "still active" array for them.
__global__ void k_init_active(int64_t V, const uint8_t* __restrict__ zero,
                              uint8_t* __restrict__ active) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  active[v] = zero[v] ? 0 : 1;
}

}  // namespace csd
