// ODF sampling, GFA and peak extraction per voxel (src/io/odx_out.rs:1008-1090
// computes the same quantities on the ODF sampled on a hemisphere).
#pragma once

namespace csd {

constexpr int kPeakMaxRows = 11;   // hemisphere vertices per lane: up to 352 (frequency 8 has 321)
constexpr int kPeakMax = 8;        // peaks kept per voxel

struct PeakParams {
  const float* coeffs;    // nvox x K coefficient volume
  const int64_t* vox;     // V masked voxel indices
  int64_t V;
  int K, R;               // coefficients, hemisphere vertices
  const double* At;       // K x R ODF amplitude of each coefficient on each vertex
  const double* dirs;     // R x 3 unit vertices
  const int* nb_off;      // R + 1 neighbour offsets on the hemisphere mesh
  const int* nb;          // neighbours (hemisphere indices; antipodes folded)
  int npeaks;
  double rel_thr, cos_sep;
  float* gfa;             // V
  float* pdir;            // V x npeaks x 3 (zeros past the peaks found)
  float* pval;            // V x npeaks ODF amplitude at the peak
  float* pqa;             // V x npeaks amplitude minus the voxel's minimum amplitude (>= 0)
  int at_in_smem;         // stage At in shared memory once per CTA (when it fits)
};

// One warp per voxel.  Amplitudes a_r = sum_k A[r][k] c_k in FP64 (lane
// owns vertices lane + 32 j), clipped at 0 (negative lobes are not sampled);
// GFA = sqrt(max(0, n / (n - 1) (m2 - m1^2 / n) / m2)) over the n sampled
// vertices (0 when m2 = 0), as odx_out.rs:1036-1050 writes it; peaks: vertices
// whose amplitude is positive and not below any mesh neighbour's, taken in
// decreasing amplitude (ties: lower index first), stopping below rel_thr x
// the largest, skipping any within the separation angle of a kept one
// (|cos| >= cos_sep, antipodes included), up to npeaks.
__global__ void __launch_bounds__(512) k_odf_peaks(PeakParams p) {
  extern __shared__ __align__(16) double pk_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const int K = p.K, R = p.R;
  const size_t at_sz = p.at_in_smem ? static_cast<size_t>(K) * R : 0;
  double* sat = pk_smem;                                                 // K x R (staged At), or empty
  double* sc = pk_smem + at_sz + static_cast<size_t>(warp) * (K + R);  // coefficients, then amplitudes
  double* sa = sc + K;
  const double* At = p.at_in_smem ? sat : p.At;
  if (p.at_in_smem) {
    for (size_t i = threadIdx.x; i < at_sz; i += blockDim.x) sat[i] = p.At[i];
    __syncthreads();
  }
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * nw + warp; v < p.V; v += static_cast<int64_t>(gridDim.x) * nw) {
    const float* c = p.coeffs + p.vox[v] * K;
    __syncwarp();
    for (int k = lane; k < K; k += 32) sc[k] = static_cast<double>(c[k]);
    __syncwarp();
    double a[kPeakMaxRows];
#pragma unroll
    for (int j = 0; j < kPeakMaxRows; ++j) a[j] = 0.0;
    for (int k = 0; k < K; ++k) {
      const double ck = sc[k];
      const double* row = At + static_cast<size_t>(k) * R;
#pragma unroll
      for (int j = 0; j < kPeakMaxRows; ++j) {
        const int r = lane + 32 * j;
        if (r < R) a[j] = fma(row[r], ck, a[j]);
      }
    }
    double m1 = 0.0, m2 = 0.0, mn = __longlong_as_double(0x7ff0000000000000ll);
#pragma unroll
    for (int j = 0; j < kPeakMaxRows; ++j) {
      const int r = lane + 32 * j;
      if (r < R) {
        a[j] = fmax(a[j], 0.0);
        sa[r] = a[j];
        m1 += a[j];
        m2 += a[j] * a[j];
        mn = fmin(mn, a[j]);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      m1 += __shfl_xor_sync(kFull, m1, o);
      m2 += __shfl_xor_sync(kFull, m2, o);
      mn = fmin(mn, __shfl_xor_sync(kFull, mn, o));
    }
    __syncwarp();
    const double n = static_cast<double>(R);
    if (lane == 0)
      p.gfa[v] = (m2 > 0.0 && R > 1) ? static_cast<float>(sqrt(fmax((n / (n - 1.0)) * (m2 - m1 * m1 / n) / m2, 0.0)))
                                     : 0.0f;
    // local maxima on the mesh
    unsigned cand = 0;
#pragma unroll
    for (int j = 0; j < kPeakMaxRows; ++j) {
      const int r = lane + 32 * j;
      if (r < R && a[j] > 0.0) {
        bool is_max = true;
        for (int q = p.nb_off[r]; q < p.nb_off[r + 1]; ++q) is_max = is_max && a[j] >= sa[p.nb[q]];
        if (is_max) cand |= 1u << j;
      }
    }
    double kd[kPeakMax][3];
    int kept = 0;
    double top = 0.0;
    for (int round = 0; round < R && kept < p.npeaks; ++round) {
      // the largest remaining candidate (ties: lower vertex index)
      double bv = -1.0;
      int br = 0x7fffffff;
#pragma unroll
      for (int j = 0; j < kPeakMaxRows; ++j)
        if (cand & (1u << j)) {
          const int r = lane + 32 * j;
          if (a[j] > bv || (a[j] == bv && r < br)) {
            bv = a[j];
            br = r;
          }
        }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(kFull, bv, o);
        const int orr = __shfl_xor_sync(kFull, br, o);
        if (ov > bv || (ov == bv && orr < br)) {
          bv = ov;
          br = orr;
        }
      }
      if (bv < 0.0) break;  // no candidate left
      if (round == 0) top = bv;
      if (bv < p.rel_thr * top) break;
      if ((br & 31) == lane) cand &= ~(1u << (br >> 5));
      const double dx = p.dirs[3 * br], dy = p.dirs[3 * br + 1], dz = p.dirs[3 * br + 2];
      bool far = true;
      for (int q = 0; q < kept; ++q) far = far && fabs(dx * kd[q][0] + dy * kd[q][1] + dz * kd[q][2]) < p.cos_sep;
      if (!far) continue;
      kd[kept][0] = dx;
      kd[kept][1] = dy;
      kd[kept][2] = dz;
      if (lane == 0) {
        float* d = p.pdir + (v * p.npeaks + kept) * 3;
        d[0] = static_cast<float>(dx);
        d[1] = static_cast<float>(dy);
        d[2] = static_cast<float>(dz);
        p.pval[v * p.npeaks + kept] = static_cast<float>(bv);
        p.pqa[v * p.npeaks + kept] = static_cast<float>(fmax(bv - mn, 0.0));
      }
      ++kept;
    }
    if (lane == 0)
      for (int q = kept; q < p.npeaks; ++q) {
        float* d = p.pdir + (v * p.npeaks + q) * 3;
        d[0] = d[1] = d[2] = 0.0f;
        p.pval[v * p.npeaks + q] = 0.0f;
        p.pqa[v * p.npeaks + q] = 0.0f;
      }
  }
}

}  // namespace csd
