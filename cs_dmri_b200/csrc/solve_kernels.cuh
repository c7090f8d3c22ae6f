// solve_kernels.cuh - the per-voxel kernels of the SHORE volume fit.
//
//   k_mask_count / k_scan_blocks / k_mask_compact
//       masked voxel list in canonical x-y-z order (src/voxel_loop.rs:28-42)
//   k_rhs         b_v = M^T s_v for every masked voxel (the A^T s of every
//                 solver: fista.rs:90-93 in Gram form, tikhonov.rs:62,
//                 alpha.rs:51)
//   k_fista_fp64  warm-startable FISTA iterations (src/solver/fista.rs:70-143)
//                 in Gram form on FP64 DMMA tensor cores, 8 voxels per warp,
//                 slots refilled from a device work queue as voxels converge
//   k_tikhonov    L L^T c = b by forward/back substitution
//                 (src/solver/tikhonov.rs:60-76)
//   k_epilogue    residual ||s - M c||, R^2, BIC, diagnostic maps and the
//                 scatter into the (X, Y, Z, K) coefficient volume
//                 (src/fit.rs:115-155, 264-318)
#pragma once

#include <cstdint>

namespace csd {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------ compaction

constexpr int kCompactBlock = 1024;

__global__ void k_mask_count(const uint8_t* __restrict__ mask, int64_t n,
                             int* __restrict__ block_counts) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kCompactBlock;
  int c = 0;
  for (int i = threadIdx.x; i < kCompactBlock; i += blockDim.x) {
    const int64_t g = base + i;
    c += (g < n && mask[g] != 0) ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
  __shared__ int red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < (blockDim.x + 31) / 32; ++w) s += red[w];
    block_counts[blockIdx.x] = s;
  }
}

// Exclusive scan of the per-block counts, one CTA; total written to *total.
__global__ void k_scan_blocks(int* __restrict__ counts, int nblocks, long long* __restrict__ total) {
  __shared__ long long carry;
  __shared__ long long warp_sums[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nblocks; base += blockDim.x) {
    const int i = base + threadIdx.x;
    long long v = (i < nblocks) ? counts[i] : 0;
    // inclusive warp scan
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(kFull, x, o);
      if ((threadIdx.x & 31) >= o) x += y;
    }
    if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      long long w = (threadIdx.x < blockDim.x / 32) ? warp_sums[threadIdx.x] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(kFull, w, o);
        if (threadIdx.x >= o) w += y;
      }
      warp_sums[threadIdx.x] = w;
    }
    __syncthreads();
    const long long warp_prefix = (threadIdx.x >= 32) ? warp_sums[(threadIdx.x >> 5) - 1] : 0;
    const long long excl = carry + warp_prefix + x - v;
    if (i < nblocks) counts[i] = static_cast<int>(excl);
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_mask_compact(const uint8_t* __restrict__ mask, int64_t n,
                               const int* __restrict__ block_offsets, int64_t* __restrict__ vox) {
  // blockDim.x == kCompactBlock / 4; each thread scans 4 consecutive voxels.
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kCompactBlock;
  const int t = threadIdx.x;
  int flags[4];
  int c = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t g = base + 4 * t + j;
    flags[j] = (g < n && mask[g] != 0) ? 1 : 0;
    c += flags[j];
  }
  int x = c;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, x, o);
    if ((t & 31) >= o) x += y;
  }
  __shared__ int ws[32];
  if ((t & 31) == 31) ws[t >> 5] = x;
  __syncthreads();
  if (t < 32) {
    int w = (t < blockDim.x / 32) ? ws[t] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, w, o);
      if (t >= o) w += y;
    }
    ws[t] = w;
  }
  __syncthreads();
  int pos = block_offsets[blockIdx.x] + ((t >= 32) ? ws[(t >> 5) - 1] : 0) + x - c;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (flags[j]) vox[pos++] = base + 4 * t + j;
  }
}

// ---------------------------------------------------------------- A^T s

// b_v[k] = sum_i M[i, k] * s_v[i] for a tile of 64 voxels x Kp columns,
// sweeping N in chunks of 32 rows staged in shared memory.  Thread (tv, tk)
// owns voxel tv and the contiguous columns [tk*NC, tk*NC + NC); its M reads
// are warp-uniform 16-byte broadcasts and the signal tile is padded against
// bank conflicts.  Rows are accumulated in index order, as M^T s is.
template <int KP>
__global__ void __launch_bounds__(256) k_rhs(const float* __restrict__ data,
                                             const int64_t* __restrict__ vox, int64_t V, int N,
                                             const double* __restrict__ M, int K,
                                             double* __restrict__ B) {
  constexpr int TV = 64, TR = 32, NC = KP / 4, SLD = TR + 1;
  extern __shared__ __align__(16) double rsm[];
  double* sM = rsm;              // TR x KP
  double* sS = rsm + TR * KP;    // TV x SLD
  const int tid = threadIdx.x;
  const int tv = tid & 63, tk = tid >> 6;
  const int64_t v0 = static_cast<int64_t>(blockIdx.x) * TV;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  for (int r0 = 0; r0 < N; r0 += TR) {
    for (int e = tid; e < TV * TR; e += 256) {
      const int lv = e / TR, lr = e % TR;
      const int64_t v = v0 + lv;
      const int r = r0 + lr;
      double sv = 0.0;
      if (v < V && r < N) sv = static_cast<double>(data[vox[v] * N + r]);
      sS[lv * SLD + lr] = sv;
    }
    for (int e = tid; e < TR * KP; e += 256) {
      const int lr = e / KP, k = e % KP;
      const int r = r0 + lr;
      sM[lr * KP + k] = (r < N && k < K) ? M[static_cast<size_t>(r) * K + k] : 0.0;
    }
    __syncthreads();
#pragma unroll 2
    for (int lr = 0; lr < TR; ++lr) {
      const double sv = sS[tv * SLD + lr];
      const double2* mrow = reinterpret_cast<const double2*>(sM + lr * KP + tk * NC);
#pragma unroll
      for (int c = 0; c < NC / 2; ++c) {
        const double2 m2 = mrow[c];
        acc[2 * c] = fma(m2.x, sv, acc[2 * c]);
        acc[2 * c + 1] = fma(m2.y, sv, acc[2 * c + 1]);
      }
    }
    __syncthreads();
  }
  const int64_t v = v0 + tv;
  if (v < V) {
#pragma unroll
    for (int c = 0; c < NC; ++c) B[v * KP + tk * NC + c] = acc[c];
  }
}

// ------------------------------------------------------------------ FISTA

// D(8x8) += A(8x4, row) * B(4x8, col) in FP64 on the tensor cores.
// Not volatile: the instruction has no side effects, so the compiler may
// interleave independent DMMAs with the fragment loads.
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

struct FistaParams {
  const double* gfrag;         // packed Gram tiles, MT*KT*32
  const double* B;             // V x Kp
  double* X;                   // V x Kp out
  const double* warm;          // V x Kp warm start, or nullptr
  uint32_t* iters;             // V
  uint8_t* conv;               // V
  int64_t V;
  double n_inv;                // 1 / n_samples
  double step;                 // 1 / L
  double thr;                  // step * alpha (when alpha_v is null)
  const double* alpha_v;       // per-voxel alpha (V), or nullptr
  double tol;
  int max_iter;
  int non_negative;
  unsigned long long* queue;   // next unassigned position in the work list
  const int64_t* list;         // work list of voxel positions, or nullptr (= 0..V-1)
  int64_t n_work;              // length of the work list
  unsigned long long* iter_total;  // executed iterations, summed (nullable); the fit's counters
                                   // [iterations, k-steps, voxels parked by the two-pass schedule]
  const double* mom;           // Nesterov momentum (t_k - 1) / t_{k+1}, k < max_iter
  unsigned long long* kstep_total;  // executed DMMA k-steps (each MT DMMAs), summed (nullable)
  // Two-pass schedule (k_fista_v3 only).  Pass 1 (cap > 0, resume = 0): a
  // voxel that has neither converged nor reached max_iter after `cap`
  // iterations stores its exact state - x in X, the next momentum point y
  // in Y - appends its position to `pend` with a prediction of the
  // iterations it still needs in `pend_key`, and frees its slot.  Pass 2
  // (resume = 1) takes such voxels (in the order of `list`, `*n_work_dev` of
  // them) from that state at iteration `cap`.  The per-voxel arithmetic is
  // unchanged, so the iterates are those of a single pass.
  int cap;
  int resume;
  double* Y;                            // V x Kp
  int64_t* pend;                        // positions left unfinished by pass 1
  float* pend_key;                      // predicted remaining iterations / 2^16, in [2^-16, 1]
  unsigned long long* n_pend;           // entries in pend
  const unsigned long long* n_work_dev; // work-list length on the device (nullptr: n_work)
};

// One warp fits 8 voxels at a time (the 8 columns of an m8n8k4 tile).  Lane
// l holds rows 8*mt + l/4 of voxel columns 2*(l%4) + {0,1} for every row tile
// mt: the DMMA accumulator layout, so the elementwise FISTA update, the
// per-voxel norms (a 3-step xor shuffle over the 8 lanes of a column) and the
// per-voxel state all stay in registers.  y goes through a per-warp shared
// buffer once per iteration to become the next B operand.  G's tiles are
// staged once per CTA in shared memory.  A voxel leaves its slot when its
// relative change drops below tol or it reaches max_iter, exactly the
// reference's per-voxel stopping rule, and the slot is refilled from the
// queue, so no lane waits for the slowest voxel of a fixed batch.
template <int MT>
__global__ void __launch_bounds__(256) k_fista_fp64(FistaParams p) {
  constexpr int KP = 8 * MT, KT = 2 * MT;
  extern __shared__ __align__(16) double smem[];
  double* sG = smem;                                   // MT*KT*32
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* ybuf = sG + MT * KT * 32 + warp * (KP * 8);  // KP x 8, row-major [k][voxel]
  for (int i = threadIdx.x; i < MT * KT * 32; i += blockDim.x) sG[i] = p.gfrag[i];
  __syncthreads();

  const int g = lane >> 2;     // row within a tile / B-fragment column
  const int q = lane & 3;      // column pair / B-fragment row

  double x[MT][2], y[MT][2], b[MT][2];
  int64_t vid[2] = {-1, -1};
  int it[2] = {0, 0};
  double t[2] = {1.0, 1.0};
  double thr[2] = {p.thr, p.thr};
  bool need[2] = {true, true};
  bool exhausted = false;
  unsigned long long executed = 0;  // voxel-iterations run by this warp

  while (true) {
    // ---- refill finished or empty slots from the queue (warp-aggregated)
    {
      const unsigned n0 = __ballot_sync(kFull, lane < 4 && need[0]);
      const unsigned n1 = __ballot_sync(kFull, lane < 4 && need[1]);
      unsigned colmask = 0;
#pragma unroll
      for (int l = 0; l < 4; ++l)
        colmask |= (((n0 >> l) & 1u) << (2 * l)) | (((n1 >> l) & 1u) << (2 * l + 1));
      const int nneed = __popc(colmask);
      if (nneed > 0) {
        // `base` is warp-uniform; V_END marks "nothing left to hand out".
        const unsigned long long V_END = static_cast<unsigned long long>(p.n_work);
        unsigned long long base = V_END;
        if (!exhausted) {
          if (lane == 0) base = atomicAdd(p.queue, static_cast<unsigned long long>(nneed));
          base = __shfl_sync(kFull, base, 0);
          if (base + nneed >= V_END) exhausted = true;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          if (!need[j]) continue;
          const int col = 2 * q + j;
          const unsigned long long cand = base + __popc(colmask & ((1u << col) - 1u));
          const int64_t nv = (cand < V_END)
                                 ? (p.list ? p.list[cand] : static_cast<int64_t>(cand))
                                 : -1;
          vid[j] = nv;
          it[j] = 0;
          t[j] = 1.0;
          thr[j] = (p.alpha_v && nv >= 0) ? __dmul_rn(p.step, p.alpha_v[nv]) : p.thr;
          need[j] = false;
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) {
            const int row = 8 * mt + g;
            if (nv >= 0) {
              b[mt][j] = p.B[nv * KP + row];
              x[mt][j] = p.warm ? p.warm[nv * KP + row] : 0.0;
            } else {
              b[mt][j] = 0.0;
              x[mt][j] = 0.0;
            }
            y[mt][j] = x[mt][j];
          }
        }
      }
    }
    const bool any_active = __any_sync(kFull, vid[0] >= 0 || vid[1] >= 0);
    if (!any_active) break;
    executed += (g == 0) ? ((vid[0] >= 0) + (vid[1] >= 0)) : 0;

    // ---- y -> shared, as the B operand [k][voxel]
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      const int row = 8 * mt + g;
      *reinterpret_cast<double2*>(&ybuf[row * 8 + 2 * q]) = make_double2(y[mt][0], y[mt][1]);
    }
    __syncwarp();

    // ---- acc = G y on the FP64 tensor cores
    double acc[MT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const double bf = ybuf[(4 * kt + q) * 8 + g];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const double af = sG[(mt * KT + kt) * 32 + lane];
        dmma_m8n8k4(acc[mt][0], acc[mt][1], af, bf);
      }
    }
    __syncwarp();

    // ---- proximal gradient step and momentum (fista.rs:95-113)
    double tn[2], mom[2], dx2[2] = {0.0, 0.0}, xn2[2] = {0.0, 0.0};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      tn[j] = 0.5 * (1.0 + sqrt(1.0 + 4.0 * t[j] * t[j]));
      mom[j] = (t[j] - 1.0) / tn[j];
    }
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const double grad = __dmul_rn(__dsub_rn(acc[mt][j], b[mt][j]), p.n_inv);
        const double cand = __dsub_rn(y[mt][j], __dmul_rn(p.step, grad));
        double sv;
        if (cand > thr[j])
          sv = __dsub_rn(cand, thr[j]);
        else if (cand < -thr[j])
          sv = __dadd_rn(cand, thr[j]);
        else
          sv = 0.0;
        const double xn = p.non_negative ? fmax(sv, 0.0) : sv;
        const double d = __dsub_rn(xn, x[mt][j]);
        y[mt][j] = __dadd_rn(xn, __dmul_rn(mom[j], d));
        dx2[j] = __dadd_rn(dx2[j], __dmul_rn(d, d));
        xn2[j] = __dadd_rn(xn2[j], __dmul_rn(xn, xn));
        x[mt][j] = xn;
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        dx2[j] += __shfl_xor_sync(kFull, dx2[j], o);
        xn2[j] += __shfl_xor_sync(kFull, xn2[j], o);
      }
    }

    // ---- per-voxel stopping rule (fista.rs:115-127) and write-out
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (vid[j] < 0) continue;
      const double rel = sqrt(dx2[j]) / fmax(sqrt(xn2[j]), 1e-12);
      t[j] = tn[j];
      it[j] += 1;
      const bool converged = rel < p.tol;
      if (converged || it[j] >= p.max_iter) {
        const int64_t v = vid[j];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) p.X[v * KP + 8 * mt + g] = x[mt][j];
        if (g == 0) {
          p.iters[v] = static_cast<uint32_t>(it[j]);
          p.conv[v] = converged ? 1 : 0;
        }
        need[j] = true;
      }
    }
  }
  if (p.iter_total) {
    for (int o = 16; o > 0; o >>= 1) executed += __shfl_xor_sync(kFull, executed, o);
    if (lane == 0) atomicAdd(p.iter_total, executed);
  }
}

// FISTA, one warp per 8 voxel slots (as k_fista_fp64) with a lighter
// per-iteration path:
//  * y lives only in the warp's shared B-operand buffer and b in a
//    thread-private shared buffer, so registers hold just x and the
//    accumulators and 12 warps fit per SM;
//  * the k-step loop is outermost, so consecutive DMMAs update different
//    accumulators (no dependent DMMA back to back), and a k-step whose y
//    entries are exactly zero for all eight voxels is skipped (it would add
//    only zeros): the iterates are sparse, so about half the DMMAs go;
//  * the momentum (t_k - 1) / t_{k+1} comes from a table: t_k depends only on
//    the iteration index, and the host evaluates the same IEEE expressions;
//  * the stopping test sqrt(dx2) / max(sqrt(xn2), 1e-12) < tol is evaluated
//    exactly only when dx2 <= 4 tol^2 max(xn2, 1e-24); above that bound the
//    ratio exceeds 2 tol, far outside rounding, so the decision is unchanged.
// The per-element update and the accumulation order of G y are those of
// k_fista_fp64, so both kernels return identical iterates.
//
// G_IN_SMEM = false (large K, where the tiles would crowd out the warp
// buffers): the tiles are read through the L1/L2 caches instead.
template <int MT, int WARPS, bool G_IN_SMEM>
__global__ void __launch_bounds__(32 * WARPS) k_fista_v3(FistaParams p) {
  constexpr int KP = 8 * MT, KT = 2 * MT;
  constexpr int G_WORDS = G_IN_SMEM ? MT * KT * 32 : 0;
  extern __shared__ __align__(16) double smem3[];
  const double* sG = G_IN_SMEM ? smem3 : p.gfrag;                 // MT * KT * 32 (k_pack_gfrag)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* ybuf = smem3 + G_WORDS + warp * (2 * KP * 8);           // KP x 8 [k][voxel]
  double* bbuf = ybuf + KP * 8;                                    // thread-private [mt][lane][2]
  if (G_IN_SMEM) {
    for (int i = threadIdx.x; i < MT * KT * 32; i += blockDim.x) smem3[i] = p.gfrag[i];
    __syncthreads();
  }

  const int g = lane >> 2, q = lane & 3;
  double x[MT][2];
  int64_t vid[2] = {-1, -1};
  int it[2] = {0, 0};
  double thr[2] = {p.thr, p.thr};
  bool need[2] = {true, true};
  bool exhausted = false;
  unsigned long long executed = 0, ksteps = 0;
  const double tol2x4 = 4.0 * p.tol * p.tol;
  float sl[2] = {0.f, 0.f}, skl[2] = {0.f, 0.f};  // pass 1: sums of log2(rel^2) and k log2(rel^2)
  const int w0 = p.cap - p.cap / 2;                 // window of the slope fit: iterations w0+1 .. cap

  while (true) {
    // ---- refill (warp-aggregated queue)
    {
      const unsigned n0 = __ballot_sync(kFull, lane < 4 && need[0]);
      const unsigned n1 = __ballot_sync(kFull, lane < 4 && need[1]);
      unsigned colmask = 0;
#pragma unroll
      for (int l = 0; l < 4; ++l)
        colmask |= (((n0 >> l) & 1u) << (2 * l)) | (((n1 >> l) & 1u) << (2 * l + 1));
      const int nneed = __popc(colmask);
      if (nneed > 0) {
        const unsigned long long V_END = p.n_work_dev ? *p.n_work_dev : static_cast<unsigned long long>(p.n_work);
        unsigned long long base = V_END;
        if (!exhausted) {
          if (lane == 0) base = atomicAdd(p.queue, static_cast<unsigned long long>(nneed));
          base = __shfl_sync(kFull, base, 0);
          if (base + nneed >= V_END) exhausted = true;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          if (!need[j]) continue;
          const int col = 2 * q + j;
          const unsigned long long cand = base + __popc(colmask & ((1u << col) - 1u));
          const int64_t nv = (cand < V_END) ? (p.list ? p.list[cand] : static_cast<int64_t>(cand)) : -1;
          vid[j] = nv;
          it[j] = p.resume ? p.cap : 0;
          sl[j] = skl[j] = 0.f;
          thr[j] = (p.alpha_v && nv >= 0) ? __dmul_rn(p.step, p.alpha_v[nv]) : p.thr;
          need[j] = false;
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) {
            const int row = 8 * mt + g;
            double bv = 0.0, xv = 0.0, yv = 0.0;
            if (nv >= 0) {
              bv = p.B[nv * KP + row];
              if (p.resume) {
                xv = p.X[nv * KP + row];
                yv = p.Y[nv * KP + row];
              } else {
                xv = p.warm ? p.warm[nv * KP + row] : 0.0;
                yv = xv;
              }
            }
            x[mt][j] = xv;
            bbuf[(mt * 32 + lane) * 2 + j] = bv;
            ybuf[row * 8 + col] = yv;
          }
        }
      }
    }
    if (!__any_sync(kFull, vid[0] >= 0 || vid[1] >= 0)) break;
    executed += (g == 0) ? ((vid[0] >= 0) + (vid[1] >= 0)) : 0;
    __syncwarp();

    // ---- acc = G y on the FP64 tensor cores
    double acc[MT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const double bf = ybuf[(4 * kt + q) * 8 + g];
      // A k-step whose four y entries are exactly zero for all eight voxels
      // adds only zeros: skip it (soft thresholding keeps most of y at 0).
      if (__any_sync(kFull, bf != 0.0)) {
        ++ksteps;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          const double af = G_IN_SMEM ? sG[(mt * KT + kt) * 32 + lane] : __ldg(sG + (mt * KT + kt) * 32 + lane);
          dmma_m8n8k4(acc[mt][0], acc[mt][1], af, bf);
        }
      }
    }
    __syncwarp();

    // ---- proximal gradient step and momentum (fista.rs:95-113)
    double mom[2], dx2[2] = {0.0, 0.0}, xn2[2] = {0.0, 0.0};
#pragma unroll
    for (int j = 0; j < 2; ++j) mom[j] = (vid[j] >= 0) ? p.mom[it[j]] : 0.0;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      const int row = 8 * mt + g;
      const double2 yv = *reinterpret_cast<const double2*>(&ybuf[row * 8 + 2 * q]);
      const double2 bv = *reinterpret_cast<const double2*>(&bbuf[(mt * 32 + lane) * 2]);
      const double yy[2] = {yv.x, yv.y}, bb[2] = {bv.x, bv.y};
      double yo[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const double grad = __dmul_rn(__dsub_rn(acc[mt][j], bb[j]), p.n_inv);
        const double cand = __dsub_rn(yy[j], __dmul_rn(p.step, grad));
        double sv;
        if (cand > thr[j])
          sv = __dsub_rn(cand, thr[j]);
        else if (cand < -thr[j])
          sv = __dadd_rn(cand, thr[j]);
        else
          sv = 0.0;
        const double xn = p.non_negative ? fmax(sv, 0.0) : sv;
        const double d = __dsub_rn(xn, x[mt][j]);
        yo[j] = __dadd_rn(xn, __dmul_rn(mom[j], d));
        dx2[j] = fma(d, d, dx2[j]);
        xn2[j] = fma(xn, xn, xn2[j]);
        x[mt][j] = xn;
      }
      *reinterpret_cast<double2*>(&ybuf[row * 8 + 2 * q]) = make_double2(yo[0], yo[1]);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        dx2[j] += __shfl_xor_sync(kFull, dx2[j], o);
        xn2[j] += __shfl_xor_sync(kFull, xn2[j], o);
      }
    }

    // ---- per-voxel stopping rule (fista.rs:115-127) and write-out
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (vid[j] < 0) continue;
      it[j] += 1;
      if (p.cap > 0 && !p.resume && it[j] > w0) {
        const float l2 = log2f(fmaxf(static_cast<float>(dx2[j] / fmax(xn2[j], 1e-24)), 1e-37f));
        sl[j] += l2;
        skl[j] = fmaf(static_cast<float>(it[j] - w0), l2, skl[j]);
      }
      bool converged = false;
      if (!(dx2[j] > tol2x4 * fmax(xn2[j], 1e-24))) {
        const double rel = sqrt(dx2[j]) / fmax(sqrt(xn2[j]), 1e-12);
        converged = rel < p.tol;
      }
      if (converged || it[j] >= p.max_iter) {
        const int64_t v = vid[j];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) p.X[v * KP + 8 * mt + g] = x[mt][j];
        if (g == 0) {
          p.iters[v] = static_cast<uint32_t>(it[j]);
          p.conv[v] = converged ? 1 : 0;
        }
        need[j] = true;
        vid[j] = -1;
      } else if (it[j] == p.cap && !p.resume) {
        // pass 1 of the two-pass schedule: park the voxel (y is this lane's
        // own entries of the next B operand, written above)
        const int64_t v = vid[j];
        const int col = 2 * q + j;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          const int row = 8 * mt + g;
          p.X[v * KP + row] = x[mt][j];
          p.Y[v * KP + row] = ybuf[row * 8 + col];
        }
        if (g == 0) {
          const unsigned long long slot = atomicAdd(p.n_pend, 1ull);
          p.pend[slot] = v;
          // remaining iterations: the least-squares line through log2(rel^2)
          // over the window, extended to log2(tol^2) (no decrease: the most)
          const float n = static_cast<float>(p.cap - w0), km = 0.5f * (n + 1.f);
          const float lm = sl[j] / n;
          const float sxx = n * (n * n - 1.f) / 12.f;
          const float slope = (skl[j] - km * sl[j]) / sxx;
          const float lc = lm + slope * (n - km);
          const float target = 2.f * log2f(static_cast<float>(p.tol));
          const float rem = slope < 0.f ? (target - lc) / slope : 65536.f;
          p.pend_key[slot] = fminf(fmaxf(rem, 1.f), 65536.f) * (1.f / 65536.f);
        }
        need[j] = true;
        vid[j] = -1;
      }
    }
    __syncwarp();
  }
  if (p.iter_total) {
    for (int o = 16; o > 0; o >>= 1) executed += __shfl_xor_sync(kFull, executed, o);
    if (lane == 0) atomicAdd(p.iter_total, executed);
  }
  if (p.kstep_total && lane == 0) atomicAdd(p.kstep_total, ksteps);
}

// Order of the second pass of the two-pass FISTA schedule: the voxels that
// pass 1 parked, largest predicted remaining iteration count first (the ones
// likely to need the most iterations start first instead of finishing
// alone).  A bucket sort on the float bits of the key: 8 buckets per octave
// from 2^-24 (smaller keys share the lowest bucket, larger ones and NaN the
// highest); within a bucket the order is arbitrary, which changes no result.
constexpr int kSchedBins = 256;
constexpr unsigned kSchedBinBase = (127u - 24u) << 3;

__device__ __forceinline__ int sched_bin(float key) {
  const unsigned u = __float_as_uint(key) >> 20;  // sign 0: exponent and 3 mantissa bits
  const int b = static_cast<int>(u) - static_cast<int>(kSchedBinBase);
  return b < 0 ? 0 : (b >= kSchedBins ? kSchedBins - 1 : b);
}

// hist[b] += keys in bucket b (hist zeroed by the caller); the key count is
// added to *parked_total (nullable).
__global__ void __launch_bounds__(256) k_sched_hist(const float* __restrict__ key,
                                                    const unsigned long long* __restrict__ n_key,
                                                    unsigned* __restrict__ hist,
                                                    unsigned long long* __restrict__ parked_total) {
  __shared__ unsigned sh[kSchedBins];
  if (parked_total && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(parked_total, *n_key);
  for (int b = threadIdx.x; b < kSchedBins; b += blockDim.x) sh[b] = 0;
  __syncthreads();
  const int64_t n = static_cast<int64_t>(*n_key);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    atomicAdd(&sh[sched_bin(key[i])], 1u);
  __syncthreads();
  for (int b = threadIdx.x; b < kSchedBins; b += blockDim.x)
    if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

// order[] = pend[] by bucket, highest bucket first.  Block `blk` handles one
// contiguous segment: it reserves a run in each bucket with one atomic per
// bucket (cursor zeroed by the caller), then places its entries.  256 threads.
__global__ void __launch_bounds__(256) k_sched_order(const int64_t* __restrict__ pend, const float* __restrict__ key,
                                                     const unsigned long long* __restrict__ n_key,
                                                     const unsigned* __restrict__ hist, unsigned* __restrict__ cursor,
                                                     int64_t* __restrict__ order) {
  __shared__ unsigned scan[kSchedBins], base[kSchedBins], cnt[kSchedBins];
  const int t = threadIdx.x;
  // base[b] = entries in buckets above b (inclusive scan over reversed buckets)
  scan[t] = hist[kSchedBins - 1 - t];
  cnt[t] = 0;
  __syncthreads();
  for (int o = 1; o < kSchedBins; o <<= 1) {
    const unsigned v = t >= o ? scan[t - o] : 0u;
    __syncthreads();
    scan[t] += v;
    __syncthreads();
  }
  base[kSchedBins - 1 - t] = scan[t] - hist[kSchedBins - 1 - t];
  const int64_t n = static_cast<int64_t>(*n_key);
  const int64_t seg = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = static_cast<int64_t>(blockIdx.x) * seg, hi = lo + seg < n ? lo + seg : n;
  for (int64_t i = lo + t; i < hi; i += blockDim.x) atomicAdd(&cnt[sched_bin(key[i])], 1u);
  __syncthreads();
  base[t] += cnt[t] ? atomicAdd(&cursor[t], cnt[t]) : 0u;
  cnt[t] = 0;
  __syncthreads();
  for (int64_t i = lo + t; i < hi; i += blockDim.x) {
    const int b = sched_bin(key[i]);
    order[base[b] + atomicAdd(&cnt[b], 1u)] = pend[i];
  }
}

// max_iter == 0: every voxel of the work list keeps its starting point.
__global__ void k_fista_noop(FistaParams p, int Kp) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= p.n_work * (Kp + 1)) return;
  const int64_t w = e / (Kp + 1);
  const int k = static_cast<int>(e % (Kp + 1));
  const int64_t v = p.list ? p.list[w] : w;
  if (k < Kp) {
    p.X[v * Kp + k] = p.warm ? p.warm[v * Kp + k] : 0.0;
  } else {
    p.iters[v] = 0;
    p.conv[v] = 0;
  }
}

// --------------------------------------------------------------- Tikhonov

// c = (L L^T)^{-1} b, one warp per voxel.  Lane l owns rows l, l + 32, ...;
// forward then backward substitution in the column (axpy) order, so every
// entry accumulates its terms in index order as a sequential solve does.
// L is staged in shared memory with a padded row stride.
template <int RPL>  // rows per lane = ceil(K / 32)
__global__ void __launch_bounds__(256) k_tikhonov(const double* __restrict__ Lg, int K, int Kp,
                                                  const double* __restrict__ B,
                                                  double* __restrict__ X, int64_t V) {
  extern __shared__ double sL[];  // K x (K + 1)
  const int ld = K + 1;
  for (int i = threadIdx.x; i < K * K; i += blockDim.x) sL[(i / K) * ld + (i % K)] = Lg[(i / K) * Kp + (i % K)];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); v < V;
       v += warps_total) {
    double r[RPL];
#pragma unroll
    for (int c = 0; c < RPL; ++c) {
      const int row = lane + 32 * c;
      r[c] = (row < K) ? B[v * Kp + row] : 0.0;
    }
    // forward: L y = b
    for (int i = 0; i < K; ++i) {
      const int owner = i & 31, oc = i >> 5;
      double yi = 0.0;
#pragma unroll
      for (int c = 0; c < RPL; ++c)
        if (c == oc && lane == owner) yi = __ddiv_rn(r[c], sL[i * ld + i]);
      yi = __shfl_sync(kFull, yi, owner);
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int row = lane + 32 * c;
        if (row > i && row < K) r[c] = __dsub_rn(r[c], __dmul_rn(sL[row * ld + i], yi));
        if (row == i) r[c] = yi;
      }
    }
    // backward: L^T x = y
    for (int i = K - 1; i >= 0; --i) {
      const int owner = i & 31, oc = i >> 5;
      double xi = 0.0;
#pragma unroll
      for (int c = 0; c < RPL; ++c)
        if (c == oc && lane == owner) xi = __ddiv_rn(r[c], sL[i * ld + i]);
      xi = __shfl_sync(kFull, xi, owner);
#pragma unroll
      for (int c = 0; c < RPL; ++c) {
        const int row = lane + 32 * c;
        if (row < i) r[c] = __dsub_rn(r[c], __dmul_rn(sL[i * ld + row], xi));
        if (row == i) r[c] = xi;
      }
    }
#pragma unroll
    for (int c = 0; c < RPL; ++c) {
      const int row = lane + 32 * c;
      if (row < Kp) X[v * Kp + row] = (row < K) ? r[c] : 0.0;
    }
  }
}

// --------------------------------------------------------------- epilogue

struct EpilogueParams {
  const float* data;
  const int64_t* vox;
  int64_t V;
  int N, K, Kp;
  const double* Mt;         // Kp x N row-major (transposed design, zero rows past K)
  const double* X;          // V x Kp
  const uint32_t* iters;    // V, or nullptr (then iteration count 1)
  float* coeffs;            // X*Y*Z*K volume (pre-zeroed)
  double* coef64;           // V x K, or nullptr
  float* r2;                // maps (nullable)
  float* resid;
  uint32_t* iter_map;
  uint8_t* kind_map;
  float* alpha_map;
  float* bic_map;
  uint8_t kind;
  double alpha;             // alpha written to the alpha map (Fixed)
  const double* alpha_v;    // per-voxel alpha (V), overrides `alpha` if set
  const uint8_t* zero_v;    // per-voxel "alpha_max == 0" flag (V), or nullptr:
                            // such voxels report residual 0 and BIC 0
                            // (VoxelAlphaResult::zero, src/solver/alpha.rs:179-188)
  double* resid_out;        // V, or nullptr: residual_l2 per voxel (FP64)
  int* nnz_out;             // V, or nullptr: exactly non-zero coefficients
  const int64_t* list;      // subset of positions to process, or nullptr (= all V)
  int64_t n_work;           // length of `list` (or V)
  bool scatter;             // write coefficients and maps (false: residuals only)
};

// Eight voxels per warp: lane l computes rows i = l, l+32, ... of
// r_v = s_v - M c_v for all eight voxels at once, so each coalesced load of a
// column of M^T feeds eight FMAs.  Then residual_l2 = ||r||, R^2 = 1 - RSS /
// sum (s - mean)^2 with the mean taken first (src/fit.rs:115-128), BIC with
// the count of exactly non-zero coefficients (src/solver/alpha.rs:99-103,
// 217-219), and the scatter of coefficients and map entries.
__global__ void __launch_bounds__(256) k_epilogue(EpilogueParams p) {
  extern __shared__ __align__(16) double sx[];  // per warp: Kp x 8, [k][voxel]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* xs = sx + warp * (p.Kp * 8);
  const int64_t groups = (p.n_work + 7) / 8;
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t gi = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp; gi < groups;
       gi += warps_total) {
    const int64_t w0 = gi * 8;
    const int nv = static_cast<int>((p.n_work - w0) < 8 ? (p.n_work - w0) : 8);
    int64_t vv[8], li[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      vv[j] = (j < nv) ? (p.list ? p.list[w0 + j] : w0 + j) : 0;
      li[j] = (j < nv) ? p.vox[vv[j]] : 0;
    }
    for (int e = lane; e < p.Kp * 8; e += 32) {
      const int k = e >> 3, j = e & 7;
      xs[e] = (j < nv) ? p.X[vv[j] * p.Kp + k] : 0.0;
    }
    __syncwarp();
    double rss[8], ssum[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) rss[j] = ssum[j] = 0.0;
    for (int i = lane; i < p.N; i += 32) {
      double acc[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = 0.0;
      for (int k = 0; k < p.K; ++k) {
        const double m = __ldg(p.Mt + static_cast<size_t>(k) * p.N + i);
        const double2* xk = reinterpret_cast<const double2*>(xs + k * 8);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const double2 xv = xk[h];
          acc[2 * h] = fma(m, xv.x, acc[2 * h]);
          acc[2 * h + 1] = fma(m, xv.y, acc[2 * h + 1]);
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (j < nv) {
          const double si = static_cast<double>(p.data[li[j] * p.N + i]);
          const double r = si - acc[j];
          rss[j] = fma(r, r, rss[j]);
          ssum[j] += si;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      for (int o = 16; o > 0; o >>= 1) {
        rss[j] += __shfl_xor_sync(kFull, rss[j], o);
        ssum[j] += __shfl_xor_sync(kFull, ssum[j], o);
      }
    double sst[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) sst[j] = 0.0;
    for (int i = lane; i < p.N; i += 32) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (j < nv) {
          const double d = static_cast<double>(p.data[li[j] * p.N + i]) - ssum[j] / static_cast<double>(p.N);
          sst[j] = fma(d, d, sst[j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      for (int o = 16; o > 0; o >>= 1) sst[j] += __shfl_xor_sync(kFull, sst[j], o);
    for (int j = 0; j < nv; ++j) {
      const int64_t v = vv[j];
      int nnz = 0;
      for (int k = lane; k < p.K; k += 32) {
        const double c = xs[k * 8 + j];
        nnz += (c != 0.0) ? 1 : 0;
        if (p.scatter) {
          p.coeffs[li[j] * p.K + k] = static_cast<float>(c);
          if (p.coef64) p.coef64[v * p.K + k] = c;
        }
      }
      for (int o = 16; o > 0; o >>= 1) nnz += __shfl_xor_sync(kFull, nnz, o);
      if (lane == 0) {
        const bool zero = p.zero_v && p.zero_v[v];
        const double resid = zero ? 0.0 : sqrt(rss[j]);
        const double ss_res = resid * resid;
        const double r2 = sst[j] > 0.0 ? 1.0 - ss_res / sst[j] : 0.0;
        const double a = p.alpha_v ? p.alpha_v[v] : p.alpha;
        if (p.resid_out) p.resid_out[v] = resid;
        if (p.nnz_out) p.nnz_out[v] = nnz;
        if (p.scatter) {
          if (p.r2) p.r2[li[j]] = static_cast<float>(r2);
          if (p.resid) p.resid[li[j]] = static_cast<float>(resid);
          if (p.iter_map) p.iter_map[li[j]] = p.iters ? p.iters[v] : 1u;
          if (p.kind_map) p.kind_map[li[j]] = p.kind;
          if (p.alpha_map) p.alpha_map[li[j]] = static_cast<float>(a);
          if (p.bic_map) {
            const double n = static_cast<double>(p.N);
            const double rc = fmax(ss_res, 2.2250738585072014e-308);
            p.bic_map[li[j]] =
                zero ? 0.0f
                     : static_cast<float>(n * log(rc / n) + log(n) * static_cast<double>(nnz));
          }
        }
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------- DMMA residual / rhs

// Pack a row-major rows x cols matrix (leading dimension ld) into m8n8k4
// A-operand tiles of an Rp x Cp zero-padded copy:
// frag[(mt * (Cp / 4) + kt) * 32 + lane] = A[8 mt + lane / 4][4 kt + lane % 4],
// where A = src (transpose = 0) or src^T (transpose = 1).
__global__ void k_pack_afrag(const double* __restrict__ src, int rows, int cols, int ld, int transpose,
                             int Rp, int Cp, double* __restrict__ frag) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= Rp * Cp) return;
  const int lane = idx & 31, tile = idx >> 5;
  const int CT = Cp / 4;
  const int mt = tile / CT, kt = tile % CT;
  const int r = 8 * mt + lane / 4, c = 4 * kt + (lane & 3);
  double v = 0.0;
  if (!transpose) {
    if (r < rows && c < cols) v = src[static_cast<size_t>(r) * ld + c];
  } else {
    if (r < cols && c < rows) v = src[static_cast<size_t>(c) * ld + r];
  }
  frag[idx] = v;
}

// b_v = M^T s_v on the FP64 tensor cores, eight voxels per warp: the packed
// M^T tiles (K_pad x N_pad) are staged once per persistent CTA; each warp
// stages its voxels' signals (float32, padded rows) and accumulates
// D(K_pad x 8) over the N_pad / 4 k-steps in row order.
//
// `data` may be device memory or pinned host memory mapped into the device
// address space; each masked voxel's row is read exactly once, and when
// `sig_out` is set the rows are also written there, compacted (V x N), for the
// residual pass.
template <int KP>
__global__ void __launch_bounds__(256) k_rhs_dmma(const float* __restrict__ data,
                                                  const int64_t* __restrict__ vox, int64_t V, int N,
                                                  int Np, const double* __restrict__ mtfrag,
                                                  double* __restrict__ B, float* __restrict__ sig_out) {
  constexpr int MT = KP / 8;
  constexpr int LPV = 9;   // signal values per lane per voxel: the host selects this kernel for N_pad <= 288
  extern __shared__ __align__(16) double rd_sm[];
  const int KTN = Np / 4;
  const int SLD = Np + 4;  // padded row stride (floats) of a staged signal
  double* sA = rd_sm;      // KP * Np
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* sbuf = reinterpret_cast<float*>(rd_sm + static_cast<size_t>(KP) * Np) + warp * 8 * SLD;
  for (int i = threadIdx.x; i < KP * Np; i += blockDim.x) sA[i] = mtfrag[i];
  __syncthreads();
  const int g = lane >> 2, q = lane & 3;
  const int64_t groups = (V + 7) / 8;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  // The next group's signals are loaded into registers while the current
  // group's DMMAs run (72 loads in flight per lane), so the signal fetch
  // latency hides behind the tensor work.
  float pre[8][LPV];
  auto fetch = [&](int64_t gi) {
    const int64_t v0 = gi * 8;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const bool ok = gi < groups && v0 + j < V;
      const float* src = ok ? data + vox[v0 + j] * N : nullptr;
#pragma unroll
      for (int t = 0; t < LPV; ++t) {
        const int i = lane + 32 * t;
        pre[j][t] = (src && i < N) ? __ldg(src + i) : 0.0f;
      }
    }
  };
  int64_t gi = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
  fetch(gi);
  for (; gi < groups; gi += stride) {
    const int64_t v0 = gi * 8;
    const int nv = static_cast<int>((V - v0) < 8 ? (V - v0) : 8);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float* dst = (sig_out && j < nv) ? sig_out + (v0 + j) * N : nullptr;
#pragma unroll
      for (int t = 0; t < LPV; ++t) {
        const int i = lane + 32 * t;
        if (i < Np) sbuf[j * SLD + i] = pre[j][t];
        if (dst && i < N) dst[i] = pre[j][t];
      }
    }
    __syncwarp();
    fetch(gi + stride);
    double acc[MT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
    for (int kt = 0; kt < KTN; ++kt) {
      const double bf = static_cast<double>(sbuf[g * SLD + 4 * kt + q]);
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) dmma_m8n8k4(acc[mt][0], acc[mt][1], sA[(mt * KTN + kt) * 32 + lane], bf);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int col = 2 * q + j;
      if (col < nv) {
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) B[(v0 + col) * KP + 8 * mt + g] = acc[mt][j];
      }
    }
    __syncwarp();
  }
}

struct ResidParams {
  const float* data;
  const int64_t* vox;
  const float* sig;      // compact signals (V x N) indexed by position, or nullptr (= data via vox)
  const int64_t* list;   // positions to process, or nullptr (= 0..n_work-1)
  int64_t n_work;
  int N, Np;
  const double* mfrag;   // packed M tiles (N_pad x K_pad)
  const double* X;       // V x K_pad
  double* resid_out;     // V: ||s - M c||
  double* sst_out;       // V: sum (s - mean)^2, or nullptr
};

// ||s_v - M c_v|| and sum (s_v - mean_v)^2 on the FP64 tensor cores, eight
// voxels per warp; packed M tiles staged once per persistent CTA.  Three row
// tiles are accumulated at a time (three independent DMMA chains), the signal
// is read at the accumulator's (row, voxel) positions, and the per-voxel sums
// are reduced over the eight lanes of each voxel column.  The mean is taken
// before the sum of squared deviations (src/fit.rs:120-128).
template <int KP>
__global__ void __launch_bounds__(256) k_resid_dmma(ResidParams p) {
  constexpr int KT = KP / 4;
  extern __shared__ __align__(16) double re_sm[];
  double* sA = re_sm;  // Np * KP
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* xbuf = re_sm + static_cast<size_t>(p.Np) * KP + warp * (KP * 8);
  for (int i = threadIdx.x; i < p.Np * KP; i += blockDim.x) sA[i] = p.mfrag[i];
  __syncthreads();
  const int g = lane >> 2, q = lane & 3;
  const int MTN = p.Np / 8;
  const int64_t groups = (p.n_work + 7) / 8;
  for (int64_t gi = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp; gi < groups;
       gi += static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5)) {
    const int64_t w0 = gi * 8;
    const int nv = static_cast<int>((p.n_work - w0) < 8 ? (p.n_work - w0) : 8);
    // lanes 0..7 resolve voxel position / volume index of column `lane`
    int64_t my_v = 0, my_li = 0;
    if (lane < nv) {
      my_v = p.list ? p.list[w0 + lane] : w0 + lane;
      my_li = p.sig ? my_v : p.vox[my_v];
    }
    for (int e = lane; e < KP * 8; e += 32) {
      const int k = e >> 3, j = e & 7;
      const int64_t vj = __shfl_sync(kFull, my_v, j);
      xbuf[e] = (j < nv) ? p.X[vj * KP + k] : 0.0;
    }
    // the loop above has every lane take part in every shuffle (KP * 8 is a
    // multiple of 32)
    __syncwarp();
    const int64_t li0 = __shfl_sync(kFull, my_li, 2 * q);
    const int64_t li1 = __shfl_sync(kFull, my_li, 2 * q + 1);
    const bool ok0 = 2 * q < nv, ok1 = 2 * q + 1 < nv;
    const float* sbase = p.sig ? p.sig : p.data;
    const float* s0 = sbase + li0 * p.N;
    const float* s1 = sbase + li1 * p.N;
    double rss[2] = {0.0, 0.0}, ssum[2] = {0.0, 0.0};
    for (int mt0 = 0; mt0 < MTN; mt0 += 3) {
      // this chunk's samples are requested before its DMMAs, so their
      // latency overlaps the tensor work
      float sa[3][2];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int row = 8 * (mt0 + c) + g;
        const bool in = mt0 + c < MTN && row < p.N;
        sa[c][0] = (in && ok0) ? __ldg(s0 + row) : 0.0f;
        sa[c][1] = (in && ok1) ? __ldg(s1 + row) : 0.0f;
      }
      double acc[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int kt = 0; kt < KT; ++kt) {
        const double bf = xbuf[(4 * kt + q) * 8 + g];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (mt0 + c < MTN) dmma_m8n8k4(acc[c][0], acc[c][1], sA[((mt0 + c) * KT + kt) * 32 + lane], bf);
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int row = 8 * (mt0 + c) + g;
        if (mt0 + c < MTN && row < p.N) {
          if (ok0) {
            const double sv = static_cast<double>(sa[c][0]);
            const double r = sv - acc[c][0];
            rss[0] = fma(r, r, rss[0]);
            ssum[0] += sv;
          }
          if (ok1) {
            const double sv = static_cast<double>(sa[c][1]);
            const double r = sv - acc[c][1];
            rss[1] = fma(r, r, rss[1]);
            ssum[1] += sv;
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        rss[j] += __shfl_xor_sync(kFull, rss[j], o);
        ssum[j] += __shfl_xor_sync(kFull, ssum[j], o);
      }
    double sst[2] = {0.0, 0.0};
    if (p.sst_out) {
      const double mean0 = ssum[0] / static_cast<double>(p.N), mean1 = ssum[1] / static_cast<double>(p.N);
      for (int row = g; row < p.N; row += 8) {
        if (ok0) {
          const double d = static_cast<double>(s0[row]) - mean0;
          sst[0] = fma(d, d, sst[0]);
        }
        if (ok1) {
          const double d = static_cast<double>(s1[row]) - mean1;
          sst[1] = fma(d, d, sst[1]);
        }
      }
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) sst[j] += __shfl_xor_sync(kFull, sst[j], o);
    }
    const int64_t v0 = __shfl_sync(kFull, my_v, 2 * q);
    const int64_t v1 = __shfl_sync(kFull, my_v, 2 * q + 1);
    if (g == 0) {
      if (ok0) {
        p.resid_out[v0] = sqrt(rss[0]);
        if (p.sst_out) p.sst_out[v0] = sst[0];
      }
      if (ok1) {
        p.resid_out[v1] = sqrt(rss[1]);
        if (p.sst_out) p.sst_out[v1] = sst[1];
      }
    }
    __syncwarp();
  }
}

struct FinalizeParams {
  const int64_t* vox;
  const int64_t* list;
  int64_t n_work;
  int N, K, Kp;
  const double* X;          // V x Kp
  const double* resid;      // V (from k_resid_dmma), or nullptr when no map needs it
  const double* sst;        // V, or nullptr (only needed with maps)
  const uint32_t* iters;    // V or nullptr (iteration count 1)
  const uint8_t* zero_v;    // V or nullptr
  const double* alpha_v;    // V or nullptr
  double alpha;
  uint8_t kind;
  bool scatter;
  float* coeffs;
  float *r2, *resid_map, *alpha_map, *bic_map;
  uint32_t* iter_map;
  uint8_t* kind_map;
  int* nnz_out;
};

// Scatter of one voxel per warp: coefficients to the (X, Y, Z, K) volume,
// exactly-non-zero count, R^2 = 1 - RSS / SST, BIC and the map entries.
__global__ void __launch_bounds__(256) k_finalize(FinalizeParams p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp; w < p.n_work; w += warps_total) {
    const int64_t v = p.list ? p.list[w] : w;
    const int64_t li = p.vox[v];
    int nnz = 0;
    for (int k = lane; k < p.K; k += 32) {
      const double c = p.X[v * p.Kp + k];
      nnz += (c != 0.0) ? 1 : 0;
      if (p.scatter) p.coeffs[li * p.K + k] = static_cast<float>(c);
    }
    for (int o = 16; o > 0; o >>= 1) nnz += __shfl_xor_sync(kFull, nnz, o);
    if (lane == 0) {
      if (p.nnz_out) p.nnz_out[v] = nnz;
      if (p.scatter) {
        const bool zero = p.zero_v && p.zero_v[v];
        const double resid = (zero || !p.resid) ? 0.0 : p.resid[v];
        const double ss_res = resid * resid;
        const double sst = p.sst ? p.sst[v] : 0.0;
        if (p.r2) p.r2[li] = static_cast<float>(sst > 0.0 ? 1.0 - ss_res / sst : 0.0);
        if (p.resid_map) p.resid_map[li] = static_cast<float>(resid);
        if (p.iter_map) p.iter_map[li] = p.iters ? p.iters[v] : 1u;
        if (p.kind_map) p.kind_map[li] = p.kind;
        if (p.alpha_map) p.alpha_map[li] = static_cast<float>(p.alpha_v ? p.alpha_v[v] : p.alpha);
        if (p.bic_map) {
          const double n = static_cast<double>(p.N);
          const double rc = fmax(ss_res, 2.2250738585072014e-308);
          p.bic_map[li] = zero ? 0.0f
                               : static_cast<float>(n * log(rc / n) + log(n) * static_cast<double>(nnz));
        }
      }
    }
  }
}

// ---------------------------------------------------------------- utility

// M^T, padded to Kp rows (rows past K are zero), row-major Kp x N.
__global__ void k_transpose_design(const double* __restrict__ M, int N, int K, int Kp,
                                   double* __restrict__ Mt) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= Kp * N) return;
  const int k = idx / N, i = idx % N;
  Mt[idx] = (k < K) ? M[static_cast<size_t>(i) * K + k] : 0.0;
}

__global__ void k_iota(int64_t* __restrict__ a, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

// Signals of the FISTA autotuning batch: one tensor per voxel on the table,
// S0 1000 exp(-b (l_perp + (l_par - l_perp) (g . u)^2)) with l_par 1.7e-3,
// l_perp 0.3e-3 and a direction u hashed from the voxel index - data whose
// fits have the sparsity, and so the k-step skipping, of real ones.
__global__ void k_tune_signal(const double* __restrict__ bvals, const double* __restrict__ bvecs, int N,
                              int64_t V, float* __restrict__ S) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= V * N) return;
  const int64_t v = idx / N;
  const int i = static_cast<int>(idx % N);
  unsigned long long z = static_cast<unsigned long long>(v) * 0x9E3779B97F4A7C15ull + 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 31)) * 0x94D049BB133111EBull;
  z ^= z >> 29;
  const double cz = 2.0 * static_cast<double>(z & 0xffffff) / 16777216.0 - 1.0;
  const double ph = 6.283185307179586 * static_cast<double>((z >> 24) & 0xffffff) / 16777216.0;
  const double sz = sqrt(fmax(1.0 - cz * cz, 0.0));
  const double gu = bvecs[3 * i] * sz * cos(ph) + bvecs[3 * i + 1] * sz * sin(ph) + bvecs[3 * i + 2] * cz;
  S[idx] = static_cast<float>(1000.0 * exp(-bvals[i] * (0.3e-3 + 1.4e-3 * gu * gu)));
}

// b = M^T s of the autotuning batch, one thread per (voxel, coefficient).
__global__ void k_tune_rhs(const double* __restrict__ M, int N, int K, int Kp, const float* __restrict__ S,
                           int64_t V, double* __restrict__ B) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= V * Kp) return;
  const int64_t v = idx / Kp;
  const int k = static_cast<int>(idx % Kp);
  double acc = 0.0;
  if (k < K)
    for (int i = 0; i < N; ++i) acc += M[static_cast<size_t>(i) * K + k] * static_cast<double>(S[v * N + i]);
  B[idx] = acc;
}

__global__ void k_fill_f64(double* __restrict__ a, int64_t n, double v) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

__global__ void k_square(const double* __restrict__ a, double* __restrict__ b, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i] * a[i];
}

// map[vox[v]] = (float) a[v]
__global__ void k_scatter_f64_to_f32(const double* __restrict__ a, const int64_t* __restrict__ vox,
                                     int64_t V, float* __restrict__ map) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v < V) map[vox[v]] = static_cast<float>(a[v]);
}

}  // namespace csd
