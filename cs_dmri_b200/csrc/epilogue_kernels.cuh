// Post-fit maps over a SHORE coefficient volume: the signal on a new gradient
// table (src/synth.rs:15-84), the Tournier-ordered ODF SH coefficients
// (src/odf.rs:79-102, python/src/models.rs:201-250) and the propagator
// scalars RTOP, RTAP, RTPP, MSD, QIV, NG (src/scalars/microstructure.rs).
//
// All three read a (X, Y, Z, K) f32 volume once and are bound by HBM; the
// per-voxel arithmetic is FP64 in the reference's order, rounded to f32 at
// the end as the reference does.
#pragma once

#include <cstdint>

namespace csd {

constexpr int kApplyTile = 16;  // voxels per tile of k_apply_rows

// out[v, i] = f32( sum_k AT[k, i] * c[v, k] ) for every voxel v of the
// volume, the products summed in k order in FP64 (the reference's gemv
// column order, synth.rs:60 / models.rs:238-243).  A voxel outside `mask`
// (if given), or with every coefficient exactly zero when `skip_zero` is set
// (synth.rs:55-58), is written as zeros.  AT is K x R, R contiguous.
__global__ void __launch_bounds__(256) k_apply_rows(const float* __restrict__ coeffs, int64_t nvox, int K,
                                                    const double* __restrict__ AT, int R,
                                                    const uint8_t* __restrict__ mask, int skip_zero,
                                                    float* __restrict__ out) {
  extern __shared__ double sc[];  // [kApplyTile][K]
  __shared__ int act[kApplyTile];
  const int64_t ntiles = (nvox + kApplyTile - 1) / kApplyTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t v0 = tile * kApplyTile;
    const int nv = static_cast<int>(nvox - v0 < kApplyTile ? nvox - v0 : kApplyTile);
    for (int idx = threadIdx.x; idx < nv * K; idx += blockDim.x)
      sc[idx] = static_cast<double>(coeffs[v0 * K + idx]);
    __syncthreads();
    if (threadIdx.x < nv) {
      const int v = threadIdx.x;
      int a = mask ? (mask[v0 + v] != 0) : 1;
      if (a && skip_zero) {
        int any = 0;
        for (int k = 0; k < K; ++k) any |= (sc[v * K + k] != 0.0);
        a = any;
      }
      act[v] = a;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nv * R; idx += blockDim.x) {
      const int v = idx / R, i = idx - v * R;
      float o = 0.0f;
      if (act[v]) {
        double acc = 0.0;
        const double* cv = sc + v * K;
        for (int k = 0; k < K; ++k) acc = __dadd_rn(acc, __dmul_rn(__ldg(AT + static_cast<size_t>(k) * R + i), cv[k]));
        o = static_cast<float>(acc);
      }
      out[v0 * R + idx] = o;
    }
    __syncthreads();
  }
}

// BrainSuite SHORE column -> (n, l, k within the 2l+1 block), index order of
// src/basis/shore.rs:29-51.
__device__ __forceinline__ void shore_col(int col, int radial_order, int& n, int& l, int& k) {
  int c = 0;
  for (int nn = 0; nn <= radial_order; ++nn)
    for (int ll = 0; ll <= nn; ll += 2) {
      if (col < c + 2 * ll + 1) {
        n = nn;
        l = ll;
        k = col - c;
        return;
      }
      c += 2 * ll + 1;
    }
  n = l = k = 0;
}

// Transposed SHORE -> Tournier projection, PT (K x R), R = (lmax+1)(lmax+2)/2:
// one non-zero per column, radial_factor(n, l) times the BrainSuite ->
// Tournier sign, at row l(l+1)/2 + m (odf.rs:56-102).  PT must be zeroed.
__global__ void k_tournier_projT(int K, int radial_order, double zeta, int lmax, int R, double* __restrict__ PT) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= K) return;
  int n, l, k;
  shore_col(col, radial_order, n, l, k);
  if (l > lmax) return;
  const int base = l * (l + 1) / 2;
  int row;
  double sign = 1.0;
  if (k < l) {
    row = base + (l - k);  // cosine block, m = +(l - k)
  } else if (k == l) {
    row = base;
  } else {
    const int j = k - l;  // sine block, m = -j, sign (-1)^(j+1)
    row = base - j;
    sign = (j % 2 == 1) ? 1.0 : -1.0;
  }
  PT[static_cast<size_t>(col) * R + row] = dev_radial_factor(n, l, zeta) * sign;
}

// ---------------------------------------------------------------- scalars

constexpr int kMicroMaxN = 16;       // radial orders up to 15
constexpr int kMicroMaxBlocks = 90;  // (n, l) blocks up to radial order 15

// Per-basis constants of src/scalars/microstructure.rs, kept factor by factor
// so that every per-voxel sum runs the reference's operations in its order.
struct MicroConsts {
  int radial_order, K, n_blocks;
  double zeta;
  int n00[kMicroMaxN];           // flat index of (n, 0, 0)
  double r0[kMicroMaxN];         // kappa(n, 0) L_n^(1/2)(0)
  double rtop_w[kMicroMaxN];     // sqrt(16 pi zeta^1.5 Gamma(n + 1.5) / n!)
  double msd_w[kMicroMaxN];      // sqrt(9 Gamma(n + 1.5) / (8 pi^6 zeta^3.5 n!))
  double hyp[kMicroMaxN];        // 2F1(-n, 5/2; 3/2; 2)
  double kap0[kMicroMaxN];       // kappa(zeta, n, 0)
  double gam[kMicroMaxN];        // Gamma(n + 1.5)
  double fact[kMicroMaxN];       // n!
  double qiv_pre;                // 6 sqrt(2 pi) zeta^2.5
  int blk_start[kMicroMaxBlocks], blk_len[kMicroMaxBlocks], blk_l[kMicroMaxBlocks];
  double rtap_k[kMicroMaxBlocks], rtpp_k[kMicroMaxBlocks], alpha[kMicroMaxBlocks];
  double rtap_pre, rtpp_pre;     // 1 / mu^2, 1 / mu with mu = 1 / (2 pi sqrt(zeta))
};

__device__ __forceinline__ double dev_binomial_float(double n, unsigned k) {  // math.rs:150-152
  return lanczos_gamma(n + 1.0) / (dev_factorial(k) * lanczos_gamma(n - static_cast<double>(k) + 1.0));
}

// microstructure.rs:284-298 (the trailing factor 2 of dipy's rtap_vec *= 2)
__device__ double dev_rtap_kappa(unsigned j, unsigned l) {
  const double jf = j, lf = l;
  const double kap = pow(-1.0, static_cast<double>(static_cast<int>(j) - 1)) * pow(2.0, -(lf + 3.0) / 2.0) / CUDART_PI;
  double sum = 0.0;
  for (unsigned k = 0; k < j; ++k) {
    const double kf = k;
    const double sign = (k % 2 == 0) ? 1.0 : -1.0;
    const double bin = dev_binomial_float(jf + lf - 0.5, j - k - 1);
    const double g = lanczos_gamma((lf + 1.0) / 2.0 + kf);
    const double hp = pow(0.5, (lf + 1.0) / 2.0 + kf);
    sum += sign * bin * g / (dev_factorial(k) * hp);
  }
  return 2.0 * kap * sum;
}

// microstructure.rs:301-315
__device__ double dev_rtpp_kappa(unsigned j, unsigned l) {
  const double jf = j, lf = l;
  const double pre = pow(-0.5, lf / 2.0) / sqrt(CUDART_PI);
  double sum = 0.0;
  for (unsigned k = 0; k < j; ++k) {
    const double kf = k;
    const double sign = (k % 2 == 0) ? 1.0 : -1.0;
    const double bin = dev_binomial_float(jf + lf - 0.5, j - k - 1);
    const double g = lanczos_gamma(lf / 2.0 + kf + 0.5);
    const double hp = pow(0.5, lf / 2.0 + 0.5 + kf);
    sum += sign * bin * g / (dev_factorial(k) * hp);
  }
  return pre * sum;
}

// One thread fills the constants (a few hundred scalars, once per call).
__global__ void k_micro_consts(int radial_order, double zeta, MicroConsts* __restrict__ mc) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  mc->radial_order = radial_order;
  mc->zeta = zeta;
  int start = 0, nb = 0;
  for (int n = 0; n <= radial_order; ++n)
    for (int l = 0; l <= n; l += 2) {
      if (l == 0) mc->n00[n] = start;
      mc->blk_start[nb] = start;
      mc->blk_len[nb] = 2 * l + 1;
      mc->blk_l[nb] = l;
      const unsigned j = static_cast<unsigned>(n - l + 1);
      mc->rtap_k[nb] = dev_rtap_kappa(j, l);
      mc->rtpp_k[nb] = dev_rtpp_kappa(j, l);
      // alpha(n, l) (microstructure.rs:272-278)
      const double sign = ((l / 2) % 2 == 0) ? 1.0 : -1.0;
      const double num = 2.0 * CUDART_PI * pow(zeta, 1.5) * lanczos_gamma(static_cast<double>(n) + 1.5);
      const double den = pow(2.0, static_cast<double>(l)) * dev_factorial(n - l);
      mc->alpha[nb] = sign * sqrt(num / den);
      start += 2 * l + 1;
      ++nb;
    }
  mc->K = start;
  mc->n_blocks = nb;
  for (int n = 0; n <= radial_order; ++n) {
    const double g = lanczos_gamma(n + 1.5), f = dev_factorial(n);
    mc->r0[n] = dev_kappa(zeta, n, 0) * dev_gen_laguerre(n, 0.5, 0.0);
    mc->rtop_w[n] = sqrt(16.0 * CUDART_PI * pow(zeta, 1.5) * g / f);
    mc->msd_w[n] = sqrt(9.0 * g / (8.0 * pow(CUDART_PI, 6.0) * pow(zeta, 3.5) * f));
    mc->hyp[n] = dev_hyp2f1(-static_cast<double>(n), 2.5, 1.5, 2.0);
    mc->kap0[n] = dev_kappa(zeta, n, 0);
    mc->gam[n] = g;
    mc->fact[n] = f;
  }
  mc->qiv_pre = 6.0 * sqrt(2.0 * CUDART_PI) * pow(zeta, 2.5);
  const double mu = 1.0 / (2.0 * CUDART_PI * sqrt(zeta));
  mc->rtap_pre = 1.0 / (mu * mu);
  mc->rtpp_pre = 1.0 / mu;
}

// RTAP (rtap = true) or RTPP of one voxel along the unit direction given as
// spherical angles (microstructure.rs:224-270).
__device__ double dev_direction_scalar(const float* __restrict__ c, double e0, const MicroConsts& mc,
                                       double theta, double phi, bool rtap) {
  double acc = 0.0;
  for (int b = 0; b < mc.n_blocks; ++b) {
    const double kern = rtap ? mc.rtap_k[b] : mc.rtpp_k[b];
    if (kern == 0.0) continue;
    const double scale = kern / mc.alpha[b];
    const int l = mc.blk_l[b], s = mc.blk_start[b];
    double inner = 0.0;
    for (int k = 0; k < mc.blk_len[b]; ++k)
      inner += (static_cast<double>(c[s + k]) / e0) * dev_brainsuite_sh(l, k, theta, phi);
    acc += scale * inner;
  }
  return fmax((rtap ? mc.rtap_pre : mc.rtpp_pre) * acc, 0.0);
}

// The six scalars of every masked voxel, unit-scaled in f32
// (io/microstructure.rs:175-218): out[s * V + v] for s = rtop, rtap, rtpp,
// msd, qiv, ng.  dirs (X, Y, Z, 3) may be null; a zero or non-finite
// direction leaves RTAP / RTPP NaN (python/src/models.rs:311-319).
__global__ void k_microstructure(const float* __restrict__ coeffs, const int64_t* __restrict__ vox, int64_t V,
                                 const float* __restrict__ dirs, const MicroConsts* __restrict__ mcp, float s_rtop,
                                 float s_rtap, float s_rtpp, float s_msd, float s_qiv, float s_ng,
                                 float* __restrict__ out) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const MicroConsts& mc = *mcp;
  const int64_t p = vox[v];
  const float* c = coeffs + p * mc.K;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  // E(0) (microstructure.rs:76-88)
  double e0 = 0.0;
  const double inv = 1.0 / sqrt(4.0 * CUDART_PI);
  for (int n = 0; n <= mc.radial_order; ++n) e0 += static_cast<double>(c[mc.n00[n]]) * mc.r0[n] * inv;
  const bool bad = !isfinite(e0) || e0 == 0.0;
  double rtop = nan, msd = nan, qiv = nan, ng = nan, rtap = nan, rtpp = nan;
  if (!bad) {
    double a = 0.0, m = 0.0, q = 0.0;
    for (int n = 0; n <= mc.radial_order; ++n) {
      const double cn = static_cast<double>(c[mc.n00[n]]) / e0;
      const double sign = (n % 2 == 0) ? 1.0 : -1.0;
      a += cn * sign * mc.rtop_w[n];
      m += cn * sign * mc.msd_w[n] * mc.hyp[n];
      q += cn * mc.kap0[n] * mc.gam[n] / mc.fact[n] * mc.hyp[n];
    }
    rtop = fmax(a, 0.0);
    msd = fmax(m, 0.0);
    const double q2 = mc.qiv_pre * q;
    if (isfinite(q2) && q2 > 0.0) qiv = 1.0 / q2;
    double total = 0.0;
    for (int k = 0; k < mc.K; ++k) {
      const double cn = static_cast<double>(c[k]) / e0;
      total += cn * cn;
    }
    if (total == 0.0) {
      ng = 0.0;
    } else {
      const double c0 = static_cast<double>(c[0]) / e0;
      ng = sqrt(fmax(1.0 - (c0 * c0) / total, 0.0));
    }
    if (dirs) {
      const float* d = dirs + p * 3;
      const bool any = d[0] != 0.0f || d[1] != 0.0f || d[2] != 0.0f;
      const bool fin = isfinite(d[0]) && isfinite(d[1]) && isfinite(d[2]);
      if (any && fin) {
        const double x = d[0], y = d[1], z = d[2];
        const double norm = sqrt(x * x + y * y + z * z);
        if (isfinite(norm) && norm != 0.0) {
          const double in = 1.0 / norm;
          const double dx = x * in, dy = y * in, dz = z * in;
          const double r = sqrt(dx * dx + dy * dy + dz * dz);
          const double theta = atan2(dy, dx);
          const double phi = r > 0.0 ? acos(fmin(fmax(dz / r, -1.0), 1.0)) : 0.0;
          rtap = dev_direction_scalar(c, e0, mc, theta, phi, true);
          rtpp = dev_direction_scalar(c, e0, mc, theta, phi, false);
        }
      }
    }
  }
  out[0 * V + v] = static_cast<float>(rtop) * s_rtop;
  out[1 * V + v] = static_cast<float>(rtap) * s_rtap;
  out[2 * V + v] = static_cast<float>(rtpp) * s_rtpp;
  out[3 * V + v] = static_cast<float>(msd) * s_msd;
  out[4 * V + v] = static_cast<float>(qiv) * s_qiv;
  out[5 * V + v] = static_cast<float>(ng) * s_ng;
}

}  // namespace csd
