// icls_kernels.cuh - amplitude-positivity SHORE fit (Goldfarb-Idnani ICLS).
//
// The reference fits min 1/2 ||M x - s||^2 subject to C x >= 0, where row p
// of C maps SHORE coefficients to the ODF amplitude on direction p of a
// 321-direction hemisphere (src/solver/shore_icls.rs:41-71), with the
// Goldfarb-Idnani dual active-set method (src/solver/icls.rs:261-410):
//
//   G = M^T M + eps I = L L^T,  x0 = G^{-1} M^T s,
//   repeat: p = most violated inactive constraint (C_p x < -tol), or stop;
//           step directions from the factorisation of the active normals,
//           t1 = min u_i / r_i over r_i > tol (drop step),
//           t2 = -s_p / (z . n_p) (full step), t = min(t1, t2);
//           full step adds p, partial step drops the blocking constraint.
//
// The reference keeps J = L^{-T} Q (K x K) per solve and updates it with
// Givens rotations.  Here the same method is carried out in the coordinates
// x~ = L^T x, where the constraint normals become the columns of
// W = L^{-1} C^T (computed once): with Q1 an orthonormal basis of the active
// transformed normals and R (q x q, upper triangular) such that
// W_A = Q1 R - the first q columns of the reference's Q and its R -
//   d1 = Q1^T w_p (the reference's d[0..q)),  v = w_p - Q1 d1,
//   z . n_p = v . v,  r = R^{-1} d1,  x~ += t v  (x += t z, z = L^{-T} v).
// Adding appends v / |v| to Q1 and [d1; |v|] to R; dropping shifts R and
// restores it with the reference's row Givens rotations, applied to the
// columns of Q1 as the reference applies them to J.  Per voxel this keeps
// K x q (q <= rank C <= n_sh) instead of K x K.  At the end x = L^{-T} x~.
#pragma once

#include "device_math.cuh"

namespace csd {

// 2F1 power series, terminating (src/math.rs:130-145).
__device__ __forceinline__ double dev_hyp2f1(double a, double b, double c, double z) {
  double sum = 1.0, term = 1.0;
  for (int k = 0; k < 200; ++k) {
    const double kf = k;
    term *= (a + kf) * (b + kf) / ((c + kf) * (kf + 1.0)) * z;
    sum += term;
    if (term == 0.0) break;
    if (fabs(term) < 1e-15 * fmax(fabs(sum), 1.0)) break;
  }
  return sum;
}

// Radial factor C*G*F of the analytic SHORE ODF (src/odf.rs:35-49).
__device__ __forceinline__ double dev_radial_factor(unsigned n, unsigned l, double zeta) {
  const double nf = n, lf = l;
  const double sign = (((static_cast<int>(n) - static_cast<int>(l) / 2) % 2) == 0) ? 1.0 : -1.0;
  const double c_nl = sign * sqrt(2.0 * dev_factorial(n - l) / (pow(zeta, 1.5) * lanczos_gamma(nf + 1.5)));
  const double g_nl = (lanczos_gamma(lf / 2.0 + 1.5) * lanczos_gamma(nf + 1.5)) /
                      (lanczos_gamma(lf + 1.5) * dev_factorial(n - l)) * pow(0.5, -lf / 2.0 - 1.5);
  const double f_nl = dev_hyp2f1(-nf + lf, lf / 2.0 + 1.5, lf + 1.5, 2.0);
  return c_nl * g_nl * f_nl;
}

// Degree l, Tournier order m_T and sign of SHORE column col (BrainSuite
// block position k of degree l): cosine m = l - k, m = 0, sine m = -(k - l)
// with sign (-1)^(j+1) on the sine block (src/odf.rs:57-102).
__device__ __forceinline__ void shore_column_sh(int col, int radial_order, int& n, int& l, int& mT,
                                                double& sign) {
  int k = 0;
  n = l = 0;
  {
    int c = 0;
    bool found = false;
    for (int nn = 0; nn <= radial_order && !found; ++nn)
      for (int ll = 0; ll <= nn; ll += 2) {
        if (col < c + 2 * ll + 1) {
          n = nn;
          l = ll;
          k = col - c;
          found = true;
          break;
        }
        c += 2 * ll + 1;
      }
  }
  sign = 1.0;
  if (k < l) {
    mT = l - k;
  } else if (k == l) {
    mT = 0;
  } else {
    const int j = k - l;
    mT = -j;
    sign = (j % 2 == 1) ? 1.0 : -1.0;
  }
}

// The MRtrix real SH of degree l, order m_T at direction p, rounded through
// float32 as the reference receives it (src/solver/shore_icls.rs:52-64).
__device__ __forceinline__ double sh_amplitude32(const double* __restrict__ dirs, int p, int l, int mT) {
  const double x = dirs[3 * p], y = dirs[3 * p + 1], z = dirs[3 * p + 2];
  const double r = sqrt(x * x + y * y + z * z);
  const double theta = atan2(y, x);
  const double phi = (r > 0.0) ? acos(fmin(fmax(z / r, -1.0), 1.0)) : 0.0;
  const unsigned am = static_cast<unsigned>(mT < 0 ? -mT : mT);
  const double norm = sqrt((2.0 * l + 1.0) / (4.0 * CUDART_PI) * dev_factorial(l - am) / dev_factorial(l + am));
  const double pl = norm * dev_assoc_legendre(l, am, cos(phi));
  double yv;
  if (mT < 0)
    yv = sqrt(2.0) * pl * sin(am * theta);
  else if (mT == 0)
    yv = pl;
  else
    yv = sqrt(2.0) * pl * cos(am * theta);
  return static_cast<double>(static_cast<float>(yv));
}

// C[p, col] = Y_T(dir_p)[j] * (radial_factor(n, l) * sign) where column col
// projects onto Tournier SH index j with `sign` (src/odf.rs:57-102).  Only
// one Tournier row of the projection is non-zero per SHORE column, so this
// is the matrix product Y P.
__global__ void k_constraint(const double* __restrict__ dirs, int m, int K, int radial_order, double zeta,
                             double* __restrict__ C) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= m * K) return;
  const int p = idx / K, col = idx % K;
  int n, l, mT;
  double sign;
  shore_column_sh(col, radial_order, n, l, mT, sign);
  C[idx] = sh_amplitude32(dirs, p, l, mT) * (dev_radial_factor(n, l, zeta) * sign);
}

// The factors of C = Y P: Y[j][p] (nsh x m_pad, zero past m) the amplitude
// of Tournier SH j = l (l + 1) / 2 + m_T at direction p, and column col of
// P as its one non-zero pf[col] in row jcol[col]; C[p, col] = Y[jcol[col]][p]
// * pf[col] holds bit for bit.
__global__ void k_constraint_factors(const double* __restrict__ dirs, int m, int m_pad, int K, int radial_order,
                                     int lmax, double zeta, double* __restrict__ Y, double* __restrict__ pf,
                                     int* __restrict__ jcol) {
  const int nsh = (lmax + 1) * (lmax + 2) / 2;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < nsh * m_pad) {
    const int j = idx / m_pad, p = idx % m_pad;
    int l = 0;
    while ((l + 2) * (l + 3) / 2 - (l + 2) <= j) l += 2;  // j in [l(l+1)/2 - l, l(l+1)/2 + l]
    const int mT = j - l * (l + 1) / 2;
    Y[idx] = p < m ? sh_amplitude32(dirs, p, l, mT) : 0.0;
  }
  if (idx < K) {
    int n, l, mT;
    double sign;
    shore_column_sh(idx, radial_order, n, l, mT, sign);
    pf[idx] = dev_radial_factor(n, l, zeta) * sign;
    jcol[idx] = l * (l + 1) / 2 + mT;
  }
}

// A[i, i] += eps for i < K (G + eps I of src/solver/icls.rs:204-207).
__global__ void k_add_diag(double* __restrict__ A, int K, int Kp, double eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < K) A[i * Kp + i] += eps;
}

// W = L^{-1} C^T, stored K x m_pad (k-major, so that a scan over constraints
// reads consecutive addresses): one thread per constraint, forward
// substitution in index order.
__global__ void k_icls_w(const double* __restrict__ L, int K, int Kp, const double* __restrict__ C, int m,
                         int m_pad, double* __restrict__ W) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m_pad) return;
  if (p >= m) {
    for (int i = 0; i < K; ++i) W[static_cast<size_t>(i) * m_pad + p] = 0.0;
    return;
  }
  for (int i = 0; i < K; ++i) {
    double s = C[static_cast<size_t>(p) * K + i];
    for (int k = 0; k < i; ++k) s -= L[i * Kp + k] * W[static_cast<size_t>(k) * m_pad + p];
    W[static_cast<size_t>(i) * m_pad + p] = s / L[i * Kp + i];
  }
}

struct IclsParams {
  const double* B;          // V x Kp: M^T s
  const double* L;          // Kp x Kp: Cholesky factor of M^T M + eps I
  const double* W;          // K x m_pad: L^{-1} C^T
  double* Q1;               // scratch: per warp K x qmax, row-major
  double* X;                // V x Kp out
  uint32_t* iters;          // V
  uint8_t* conv;            // V
  int64_t V;
  int K, Kp, m, m_pad, qmax, max_iter;
  double tol;
  unsigned long long* queue;
  int* overflow;            // set when an active set would exceed qmax
  unsigned long long* iter_total;
};

constexpr int kIclsWarps = 8;

// Per-warp shared state (doubles): x~, v, w (K each), R (qmax^2), d1, r, u
// (qmax each), then qmax ints of active indices and m_pad / 32 mask words.
__host__ __device__ inline int icls_warp_words(int K, int qmax, int m_pad) {
  const int doubles = 3 * K + qmax * qmax + 3 * qmax;
  const int ints = qmax + m_pad / 32;
  return doubles + (ints + 1) / 2;
}

// One warp per voxel (voxels from an atomic queue).  Vectors of length K are
// spread over the lanes (row k on lane k mod 32); the constraint scan spreads
// constraints over the lanes; active-set quantities of length q live on lanes
// 0..q-1 (and 32..63 when qmax > 32).
template <int RPL>
__global__ void __launch_bounds__(32 * kIclsWarps) k_icls(IclsParams p) {
  extern __shared__ __align__(16) double ism[];
  const int K = p.K, qmax = p.qmax, m = p.m, m_pad = p.m_pad;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* xt = ism + static_cast<size_t>(warp) * icls_warp_words(K, qmax, m_pad);
  double* vv = xt + K;
  double* ww = vv + K;
  double* R = ww + K;
  double* d1 = R + qmax * qmax;
  double* rr = d1 + qmax;
  double* uu = rr + qmax;
  int* act = reinterpret_cast<int*>(uu + qmax);
  unsigned* bits = reinterpret_cast<unsigned*>(act + qmax);
  double* Q = p.Q1 + (static_cast<size_t>(blockIdx.x) * kIclsWarps + warp) * K * qmax;
  const int nwords = m_pad / 32;
  unsigned long long executed = 0;

  while (true) {
    unsigned long long vq = 0;
    if (lane == 0) vq = atomicAdd(p.queue, 1ull);
    vq = __shfl_sync(kFull, vq, 0);
    if (vq >= static_cast<unsigned long long>(p.V)) break;
    const int64_t v = static_cast<int64_t>(vq);

    // x~ = L^{-1} M^T s (forward substitution; x0 = G^{-1} M^T s, icls.rs:271-273)
    {
      double rv[RPL];
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int row = lane + 32 * c;
        rv[c] = (row < K) ? p.B[v * p.Kp + row] : 0.0;
      }
      for (int i = 0; i < K; ++i) {
        const int owner = i & 31, oc = i >> 5;
        double xi = 0.0;
#pragma unroll
        for (int c = 0; c < RPL; ++c)
          if (c == oc && lane == owner) xi = rv[c] / __ldg(p.L + i * p.Kp + i);
        xi = __shfl_sync(kFull, xi, owner);
#pragma unroll
        for (int c = 0; c < RPL; ++c) {
          const int row = lane + 32 * c;
          if (row > i && row < K) rv[c] -= __ldg(p.L + row * p.Kp + i) * xi;
          if (row == i) rv[c] = xi;
        }
      }
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int row = lane + 32 * c;
        if (row < K) xt[row] = rv[c];
      }
    }
    for (int wI = lane; wI < nwords; wI += 32) bits[wI] = 0u;
    __syncwarp();

    int q = 0, iters = 0;
    bool converged = false, overflow = false;
    while (true) {
      iters += 1;
      if (iters > p.max_iter) break;
      // ---- most violated inactive constraint (icls.rs:298-317): smallest
      // value below -tol, first index on ties
      double best = -p.tol;
      int bestp = -1;
      for (int c = lane; c < m; c += 32) {
        if ((bits[c >> 5] >> (c & 31)) & 1u) continue;
        double s = 0.0;
        for (int k = 0; k < K; ++k) s += __ldg(p.W + static_cast<size_t>(k) * m_pad + c) * xt[k];
        if (s < best) {
          best = s;
          bestp = c;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, o);
        const int op = __shfl_xor_sync(kFull, bestp, o);
        if (op >= 0 && (bestp < 0 || ob < best || (ob == best && op < bestp))) {
          best = ob;
          bestp = op;
        }
      }
      if (bestp < 0) {
        converged = true;
        break;
      }
      double sp = best;
      for (int k = lane; k < K; k += 32) ww[k] = __ldg(p.W + static_cast<size_t>(k) * m_pad + bestp);
      __syncwarp();

      bool stop = false;
      while (true) {  // inner loop: drop blocking constraints until p is added
        // d1 = Q1^T w, v = w - Q1 d1, one re-orthogonalisation pass
        for (int c = lane; c < q; c += 32) {
          double a = 0.0;
          for (int k = 0; k < K; ++k) a += Q[k * qmax + c] * ww[k];
          d1[c] = a;
        }
        __syncwarp();
        for (int k = lane; k < K; k += 32) {
          double a = ww[k];
          for (int c = 0; c < q; ++c) a -= Q[k * qmax + c] * d1[c];
          vv[k] = a;
        }
        __syncwarp();
        if (q > 0) {
          for (int c = lane; c < q; c += 32) {
            double a = 0.0;
            for (int k = 0; k < K; ++k) a += Q[k * qmax + c] * vv[k];
            rr[c] = a;  // correction, reused as scratch
          }
          __syncwarp();
          for (int k = lane; k < K; k += 32) {
            double a = vv[k];
            for (int c = 0; c < q; ++c) a -= Q[k * qmax + c] * rr[c];
            vv[k] = a;
          }
          for (int c = lane; c < q; c += 32) d1[c] += rr[c];
          __syncwarp();
        }
        double zn = 0.0;
        for (int k = lane; k < K; k += 32) zn += vv[k] * vv[k];
        for (int o = 16; o > 0; o >>= 1) zn += __shfl_xor_sync(kFull, zn, o);

        // r = R^{-1} d1 (upper triangular, icls.rs:331-341), column order
        for (int c = lane; c < q; c += 32) rr[c] = d1[c];
        __syncwarp();
        for (int i = q - 1; i >= 0; --i) {
          const double ri = rr[i] / R[i * qmax + i];
          __syncwarp();
          for (int c = lane; c < i; c += 32) rr[c] -= R[c * qmax + i] * ri;
          if (lane == (i & 31)) rr[i] = ri;
          __syncwarp();
        }

        // step lengths (icls.rs:343-368)
        double t1 = INFINITY;
        int drop = -1;
        for (int c = lane; c < q; c += 32) {
          if (rr[c] > p.tol) {
            const double ratio = uu[c] / rr[c];
            if (ratio < t1) {
              t1 = ratio;
              drop = c;
            }
          }
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ot = __shfl_xor_sync(kFull, t1, o);
          const int od = __shfl_xor_sync(kFull, drop, o);
          if (od >= 0 && (drop < 0 || ot < t1 || (ot == t1 && od < drop))) {
            t1 = ot;
            drop = od;
          }
        }
        const double t2 = (zn > p.tol) ? -sp / zn : INFINITY;
        const double t = fmin(t1, t2);
        if (!isfinite(t)) {
          stop = true;  // infeasible
          break;
        }
        for (int c = lane; c < q; c += 32) uu[c] -= t * rr[c];
        for (int k = lane; k < K; k += 32) xt[k] += t * vv[k];
        __syncwarp();
        if (isfinite(t2) && t == t2) {
          // full step: constraint p joins the active set
          if (q >= qmax) {
            overflow = true;
            stop = true;
            break;
          }
          const double nv = sqrt(zn);
          for (int k = lane; k < K; k += 32) Q[k * qmax + q] = vv[k] / nv;
          for (int c = lane; c < q; c += 32) R[c * qmax + q] = d1[c];
          if (lane == 0) {
            R[q * qmax + q] = nv;
            act[q] = bestp;
            uu[q] = t;
            bits[bestp >> 5] |= 1u << (bestp & 31);
          }
          __syncwarp();
          q += 1;
          break;
        }
        // partial step: the blocking constraint leaves (icls.rs:385-398, 465-501)
        sp += t * zn;
        const int kd = drop;
        const int dropped = act[kd];
        __syncwarp();
        for (int col = kd; col < q - 1; ++col) {
          for (int row = lane; row < q; row += 32) R[row * qmax + col] = R[row * qmax + col + 1];
          __syncwarp();
        }
        for (int row = lane; row < q; row += 32) R[row * qmax + q - 1] = 0.0;
        __syncwarp();
        for (int i = kd; i < q - 1; ++i) {
          const double a = R[i * qmax + i], b = R[(i + 1) * qmax + i];
          if (b == 0.0) continue;
          const double rn = sqrt(a * a + b * b);
          const double cg = a / rn, sg = b / rn;
          __syncwarp();
          for (int col = i + lane; col < q - 1; col += 32) {
            const double ri = R[i * qmax + col], rip1 = R[(i + 1) * qmax + col];
            R[i * qmax + col] = cg * ri + sg * rip1;
            R[(i + 1) * qmax + col] = -sg * ri + cg * rip1;
          }
          for (int k = lane; k < K; k += 32) {
            const double qa = Q[k * qmax + i], qb = Q[k * qmax + i + 1];
            Q[k * qmax + i] = cg * qa + sg * qb;
            Q[k * qmax + i + 1] = -sg * qa + cg * qb;
          }
          __syncwarp();
        }
        // remove entry kd from the active list and multipliers
        if (lane == 0) {
          for (int c = kd; c < q - 1; ++c) {
            act[c] = act[c + 1];
            uu[c] = uu[c + 1];
          }
          bits[dropped >> 5] &= ~(1u << (dropped & 31));
        }
        __syncwarp();
        q -= 1;
      }
      if (stop) break;
    }
    executed += static_cast<unsigned long long>(iters - 1);

    // x = L^{-T} x~ (back substitution)
    {
      double rv[RPL];
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int row = lane + 32 * c;
        rv[c] = (row < K) ? xt[row] : 0.0;
      }
      for (int i = K - 1; i >= 0; --i) {
        const int owner = i & 31, oc = i >> 5;
        double xi = 0.0;
#pragma unroll
        for (int c = 0; c < RPL; ++c)
          if (c == oc && lane == owner) xi = rv[c] / __ldg(p.L + i * p.Kp + i);
        xi = __shfl_sync(kFull, xi, owner);
#pragma unroll
        for (int c = 0; c < RPL; ++c) {
          const int row = lane + 32 * c;
          if (row < i) rv[c] -= __ldg(p.L + i * p.Kp + row) * xi;
          if (row == i) rv[c] = xi;
        }
      }
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int row = lane + 32 * c;
        if (row < p.Kp) p.X[v * p.Kp + row] = (row < K) ? rv[c] : 0.0;
      }
    }
    if (lane == 0) {
      p.iters[v] = static_cast<uint32_t>(iters - 1);
      p.conv[v] = converged ? 1 : 0;
      if (overflow) atomicAdd(p.overflow, 1);
    }
    __syncwarp();
  }
  if (p.iter_total && lane == 0) atomicAdd(p.iter_total, executed);
}

// ------------------------------------------------------------ Gram form
//
// The same method with the constraint values carried instead of recomputed.
// With Gamma = W^T W (Gamma[c][p] = w_c . w_p, once per table) every
// quantity of a step is a product with Gamma:
//   d1 = Q1^T w_p = R^-T Gamma[A, p]      (Q1 = W_A R^-1 is never formed),
//   z . n_p = |v|^2 = Gamma[p, p] - |d1|^2,   r = R^-1 d1,
//   v = w_p - W_A r,  so the constraint values s = W^T x~ move by
//   t (Gamma[:, p] - Gamma[:, A] r) and x = L^-T x~ by t (u_p - U_A r),
//   U = L^-T W = G^-1 C^T (once per table).
// A step therefore costs (q + 1) columns of Gamma and of U^T instead of the
// K-wide products with Q1, and the scan for the most violated constraint
// reads s from registers instead of recomputing W^T x~ (m x K) every
// iteration.  The unconstrained minimiser x0 = G^-1 b is one product with
// the inverse (no per-voxel substitution), and the first s = C x0 comes from
// C = Y P: z0 = P x0 (one term per column) and s = Y z0, with Y (nsh x m) in
// shared memory.  The reference's multiplier rule is kept as is (a full step
// pushes t for the new constraint), so drops follow its iteration path; the
// carried s and x differ from recomputed ones by rounding only.  Active sets
// of up to 32 are held one entry per lane (rank C = nsh <= 28 for lmax <= 6).

__global__ void k_icls_gram_setup(const double* __restrict__ W, int K, int m_pad, double* __restrict__ Gam) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(m_pad) * m_pad) return;
  const int c = static_cast<int>(idx / m_pad), q = static_cast<int>(idx % m_pad);
  double a = 0.0;
  for (int k = 0; k < K; ++k)
    a = fma(W[static_cast<size_t>(k) * m_pad + c], W[static_cast<size_t>(k) * m_pad + q], a);
  Gam[idx] = a;
}

// The Gram form's x-space operators, one thread per row: UT row c = L^-T w_c
// = G^-1 c_c (c < m_pad; zero for the padding constraints), and row i of Ginv
// = G^-1 e_i (i < K), by the factor's substitutions.  Columns K .. Kp-1 are 0.
__global__ void k_icls_gram_solves(const double* __restrict__ L, int K, int Kp, const double* __restrict__ W,
                                   int m_pad, double* __restrict__ UT, double* __restrict__ Ginv) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  double* z;
  if (idx < m_pad) {
    z = UT + static_cast<size_t>(idx) * Kp;
    for (int r = 0; r < K; ++r) z[r] = W[static_cast<size_t>(r) * m_pad + idx];
  } else if (idx < m_pad + K) {
    const int i = idx - m_pad;
    z = Ginv + static_cast<size_t>(i) * Kp;
    for (int r = 0; r < K; ++r) {  // L y = e_i
      double a = (r == i) ? 1.0 : 0.0;
      for (int k = 0; k < r; ++k) a -= L[r * Kp + k] * z[k];
      z[r] = a / L[r * Kp + r];
    }
  } else {
    return;
  }
  for (int r = K - 1; r >= 0; --r) {  // L^T z = y, in place
    double a = z[r];
    for (int k = r + 1; k < K; ++k) a -= L[k * Kp + r] * z[k];
    z[r] = a / L[r * Kp + r];
  }
  for (int r = K; r < Kp; ++r) z[r] = 0.0;
}

struct IclsGramParams {
  const double* B;      // V x Kp: M^T s
  const double* Ginv;   // Kp x Kp: (M^T M + eps I)^-1, symmetric
  const double* Gam;    // m_pad x m_pad: W^T W
  const double* UT;     // m_pad x Kp: row c = u_c = L^-T w_c = G^-1 c_c
  const double* Y;      // nsh x m_pad: C = Y P
  const double* pf;     // K: the non-zero of column col of P ...
  const int* jcol;      // K: ... and its row
  double* X;            // V x Kp out
  uint32_t* iters;      // V
  uint8_t* conv;        // V
  int64_t V;
  int K, Kp, m, m_pad, nsh, max_iter;
  double tol;
  unsigned long long* queue;
  int* overflow;
  unsigned long long* iter_total;
};

constexpr int kIclsGramWarps = 16;
constexpr int kIclsGramRs = 33;                     // row stride of R (conflict-free rows and columns)
// Per warp: R (32 x 33); at the start of a voxel, before R is in use, its
// first K entries hold x0 and entries 1024.. hold z0.
constexpr int kIclsGramWarpDoubles = 32 * kIclsGramRs;

__host__ __device__ inline size_t icls_gram_smem(int nsh, int m_pad) {
  return sizeof(double) * (static_cast<size_t>(nsh) * m_pad + static_cast<size_t>(kIclsGramWarps) * kIclsGramWarpDoubles);
}

// One warp per voxel, voxels from an atomic queue.  Constraint c lives on
// lane c % 32 (slot c / 32): its value s and active flag in registers; entry
// i < q of the active set (its constraint, multiplier, d1, r) on lane i.
template <int RPL, int CPL>  // ceil(K / 32); m_pad / 32
__global__ void __launch_bounds__(32 * kIclsGramWarps, 1) k_icls_gram(IclsGramParams p) {
  extern __shared__ __align__(16) double gsm[];
  const int K = p.K, Kp = p.Kp, m = p.m, mp = p.m_pad, nsh = p.nsh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Ysh = gsm;  // [nsh][m_pad]
  for (int e = threadIdx.x; e < nsh * mp; e += blockDim.x) Ysh[e] = p.Y[e];
  __syncthreads();
  double* R = gsm + static_cast<size_t>(nsh) * mp + static_cast<size_t>(warp) * kIclsGramWarpDoubles;
  double* x0s = R;          // [K], K <= 1024
  double* z0 = R + 1024;    // [32]
  const int qcap = nsh < 32 ? nsh : 32;
  unsigned long long executed = 0;

  while (true) {
    unsigned long long vq = 0;
    if (lane == 0) vq = atomicAdd(p.queue, 1ull);
    vq = __shfl_sync(kFull, vq, 0);
    if (vq >= static_cast<unsigned long long>(p.V)) break;
    const int64_t v = static_cast<int64_t>(vq);

    // x0 = G^-1 M^T s (icls.rs:271-273) as one product with the inverse
    // (b staged in the warp's slice, G^-1 read by rows: coalesced over lanes)
    for (int k = lane; k < K; k += 32) x0s[k] = p.B[v * Kp + k];
    __syncwarp();
    double xt[RPL];  // the iterate x, row lane + 32 c
#pragma unroll
    for (int c = 0; c < RPL; ++c) xt[c] = 0.0;
    for (int k = 0; k < K; ++k) {
      const double bk = x0s[k];
      const double* gk = p.Ginv + static_cast<size_t>(k) * Kp + lane;
#pragma unroll
      for (int c = 0; c < RPL; ++c)
        if (lane + 32 * c < K) xt[c] = fma(__ldg(gk + 32 * c), bk, xt[c]);
    }
    __syncwarp();
    // s = C x0 = Y (P x0): z0[j] sums its columns in index order
#pragma unroll
    for (int c = 0; c < RPL; ++c) {
      const int row = lane + 32 * c;
      if (row < K) x0s[row] = xt[c];
    }
    __syncwarp();
    if (lane < nsh) {
      double zj = 0.0;
      for (int col = 0; col < K; ++col)
        if (__ldg(p.jcol + col) == lane) zj = fma(__ldg(p.pf + col), x0s[col], zj);
      z0[lane] = zj;
    }
    __syncwarp();
    double s[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) s[c] = 0.0;
    for (int j = 0; j < nsh; ++j) {
      const double zj = z0[j];
#pragma unroll
      for (int c = 0; c < CPL; ++c) s[c] = fma(Ysh[j * mp + lane + 32 * c], zj, s[c]);
    }
    __syncwarp();

    unsigned actbits = 0u;  // bit c: constraint lane + 32 c is active
    int q = 0, a_i = -1;    // active set size; this lane's active constraint (lane < q)
    double u_i = 0.0;       // its multiplier
    int iters = 0;
    bool converged = false, overflow = false;
    while (true) {
      iters += 1;
      if (iters > p.max_iter) break;
      // most violated inactive constraint (icls.rs:298-317): smallest value
      // below -tol, first index on ties
      double best = -p.tol;
      int bestp = -1;
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int ci = lane + 32 * c;
        if (ci < m && !((actbits >> c) & 1u) && s[c] < best) {
          best = s[c];
          bestp = ci;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, o);
        const int op = __shfl_xor_sync(kFull, bestp, o);
        if (op >= 0 && (bestp < 0 || ob < best || (ob == best && op < bestp))) {
          best = ob;
          bestp = op;
        }
      }
      if (bestp < 0) {
        converged = true;
        break;
      }
      double sp = best;
      const double gpp = __ldg(p.Gam + static_cast<size_t>(bestp) * mp + bestp);
      bool stop = false;
      while (true) {  // inner loop: drop blocking constraints until p is added
        // d1 = R^-T Gamma[A, p] (forward substitution by columns of R^T)
        double d1 = (lane < q) ? __ldg(p.Gam + static_cast<size_t>(a_i) * mp + bestp) : 0.0;
        for (int k = 0; k < q; ++k) {
          const double dk = __shfl_sync(kFull, d1, k) / R[k * kIclsGramRs + k];
          if (lane == k) d1 = dk;
          else if (lane > k && lane < q) d1 = fma(-R[k * kIclsGramRs + lane], dk, d1);
        }
        double dd = d1 * d1;
        for (int o = 16; o > 0; o >>= 1) dd += __shfl_xor_sync(kFull, dd, o);
        const double zn = gpp - dd;  // z . n_p = |v|^2
        // r = R^-1 d1 (back substitution by columns, icls.rs:331-341)
        double rr = d1;
        for (int i = q - 1; i >= 0; --i) {
          const double ri = __shfl_sync(kFull, rr, i) / R[i * kIclsGramRs + i];
          if (lane == i) rr = ri;
          else if (lane < i) rr = fma(-R[lane * kIclsGramRs + i], ri, rr);
        }
        // step lengths (icls.rs:343-368)
        double t1 = INFINITY;
        int drop = -1;
        if (lane < q && rr > p.tol) {
          t1 = u_i / rr;
          drop = lane;
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ot = __shfl_xor_sync(kFull, t1, o);
          const int od = __shfl_xor_sync(kFull, drop, o);
          if (od >= 0 && (drop < 0 || ot < t1 || (ot == t1 && od < drop))) {
            t1 = ot;
            drop = od;
          }
        }
        const double t2 = (zn > p.tol) ? -sp / zn : INFINITY;
        const double t = fmin(t1, t2);
        if (!isfinite(t)) {
          stop = true;  // infeasible
          break;
        }
        if (lane < q) u_i -= t * rr;
        // s += t (Gamma[:, p] - Gamma[:, A] r), x += t (u_p - U_A r) (= L^-T of x~'s step)
        {
          double ds[CPL], dx[RPL];
          const double* gp = p.Gam + static_cast<size_t>(bestp) * mp + lane;
          const double* wp = p.UT + static_cast<size_t>(bestp) * Kp + lane;
#pragma unroll
          for (int c = 0; c < CPL; ++c) ds[c] = __ldg(gp + 32 * c);
#pragma unroll
          for (int c = 0; c < RPL; ++c) dx[c] = (lane + 32 * c < Kp) ? __ldg(wp + 32 * c) : 0.0;
          for (int i = 0; i < q; ++i) {
            const double ri = __shfl_sync(kFull, rr, i);
            const int ai = __shfl_sync(kFull, a_i, i);
            const double* ga = p.Gam + static_cast<size_t>(ai) * mp + lane;
            const double* wa = p.UT + static_cast<size_t>(ai) * Kp + lane;
#pragma unroll
            for (int c = 0; c < CPL; ++c) ds[c] = fma(-ri, __ldg(ga + 32 * c), ds[c]);
#pragma unroll
            for (int c = 0; c < RPL; ++c)
              if (lane + 32 * c < Kp) dx[c] = fma(-ri, __ldg(wa + 32 * c), dx[c]);
          }
#pragma unroll
          for (int c = 0; c < CPL; ++c) s[c] = fma(t, ds[c], s[c]);
#pragma unroll
          for (int c = 0; c < RPL; ++c) xt[c] = fma(t, dx[c], xt[c]);
        }
        if (isfinite(t2) && t == t2) {
          // full step: constraint p joins the active set
          if (q >= qcap) {
            overflow = true;
            stop = true;
            break;
          }
          if (lane < q) R[lane * kIclsGramRs + q] = d1;
          if (lane == q) {
            R[q * kIclsGramRs + q] = sqrt(zn);
            a_i = bestp;
            u_i = t;
          }
          if (lane == (bestp & 31)) actbits |= 1u << (bestp >> 5);
          __syncwarp();
          q += 1;
          break;
        }
        // partial step: the blocking constraint leaves (icls.rs:385-398, 465-501)
        sp += t * zn;
        const int kd = drop;
        const int dropped = __shfl_sync(kFull, a_i, kd);
        if (lane < q) {  // each lane shifts its own row of R left past column kd
          for (int col = kd; col < q - 1; ++col) R[lane * kIclsGramRs + col] = R[lane * kIclsGramRs + col + 1];
          R[lane * kIclsGramRs + q - 1] = 0.0;
        }
        __syncwarp();
        for (int i = kd; i < q - 1; ++i) {
          const double aa = R[i * kIclsGramRs + i], bb = R[(i + 1) * kIclsGramRs + i];
          if (bb == 0.0) continue;
          const double rn = sqrt(aa * aa + bb * bb);
          const double cg = aa / rn, sg = bb / rn;
          __syncwarp();
          for (int col = i + lane; col < q - 1; col += 32) {
            const double ri = R[i * kIclsGramRs + col], rj = R[(i + 1) * kIclsGramRs + col];
            R[i * kIclsGramRs + col] = cg * ri + sg * rj;
            R[(i + 1) * kIclsGramRs + col] = -sg * ri + cg * rj;
          }
          __syncwarp();
        }
        {  // entry kd leaves the active list and the multipliers
          const double un = __shfl_down_sync(kFull, u_i, 1);
          const int an = __shfl_down_sync(kFull, a_i, 1);
          if (lane >= kd && lane < q - 1) {
            u_i = un;
            a_i = an;
          } else if (lane == q - 1) {
            u_i = 0.0;
            a_i = -1;
          }
        }
        if (lane == (dropped & 31)) actbits &= ~(1u << (dropped >> 5));
        __syncwarp();
        q -= 1;
      }
      if (stop) break;
    }
    executed += static_cast<unsigned long long>(iters - 1);

#pragma unroll
    for (int c = 0; c < RPL; ++c) {
      const int row = lane + 32 * c;
      if (row < Kp) p.X[v * Kp + row] = (row < K) ? xt[c] : 0.0;
    }
    if (lane == 0) {
      p.iters[v] = static_cast<uint32_t>(iters - 1);
      p.conv[v] = converged ? 1 : 0;
      if (overflow) atomicAdd(p.overflow, 1);
    }
    __syncwarp();
  }
  if (p.iter_total && lane == 0) atomicAdd(p.iter_total, executed);
}

}  // namespace csd
