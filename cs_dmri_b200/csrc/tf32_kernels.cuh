// Converged-optimum L1 fit (precision MIXED_KKT / FP64_KKT): the LASSO
// minimiser of (1/(2n)) ||M c - s||^2 + alpha ||c||_1 (src/solver/fista.rs:4-7)
// to FP64 accuracy, certified per voxel by its KKT conditions, in three steps:
//
//  1. support identification: a fixed number of FISTA iterations
//     (fista.rs:89-128 in Gram form, step 1/L, the reference's momentum) on
//     the 5th-generation tensor cores in TF32 with FP32 accumulation
//     (k_fista_tf32) - or, for FP64_KKT, on the FP64 kernel;
//  2. k_l1_polish: the optimality condition on the support S and signs
//     sigma of that iterate, G_SS c_S = b_S - n alpha sigma_S (b = M^T s),
//     solved in FP64 (Cholesky of G_SS); coefficients whose sign disagrees
//     leave S, and the coordinate that violates |g_j| <= alpha most
//     (g = (G c - b) / n) joins it, until no sign disagrees and every
//     off-support |g_j| is within alpha (1 + kappa): the KKT certificate of
//     the reference's tests/common/mod.rs:127-153;
//  3. voxels not certified after the round limit are fitted by the FP64
//     FISTA kernel with the reference's stopping rule and polished again.
//
// Low-precision products cannot follow the reference's FP64 iterate path
// (the Gram product cancels about four orders of magnitude), but they find
// the support: the exact solve on it then gives the optimum itself, which the
// reference's tol = 1e-6 iterate only approaches (about 4e-5 away at the
// median).
#pragma once

#include <cstdint>

namespace csd {
namespace tf {

constexpr int TILE = 128;                      // voxels per tile (MMA M)
constexpr int THREADS = 256;                   // two threads per voxel
constexpr int TMEM_COLS = 128;                 // fp32 accumulator columns (N <= 80 used)
constexpr uint64_t kWaitNs = 2000000000ull;    // give up on one MMA batch after 2 s

// Operand geometry for K coefficients.  A = the tile's momentum points y
// (TILE x KA, fp32 read as TF32), B = the scaled Gram matrix (NB x KA),
// both canonical K-major without swizzle: 8 rows x 16 bytes (4 elements)
// per core matrix, K-adjacent core matrices 128 bytes apart, 8-row groups
// SBO bytes apart.  One MMA k-step covers 8 elements (32 bytes).
template <int K>
struct Shape {
  static constexpr int KS = (K + 7) / 8;           // MMA k-steps
  static constexpr int KA = 8 * KS;                // K extent of A and B
  static constexpr int NB = 16 * ((K + 15) / 16);  // MMA N (multiple of 16)
  static constexpr int SBO = (KA / 4) * 128;
  static constexpr int A_BYTES = (TILE / 8) * SBO;
  static constexpr int B_BYTES = (NB / 8) * SBO;
  static constexpr int CPT = 4 * ((K + 7) / 8);    // columns per thread (a multiple of 4)
  // Dynamic shared memory of a launch: at least 72 KB, so that at most three
  // CTAs share an SM and their tensor-memory allocations (128 columns each)
  // always fit in its 512 columns.
  static constexpr size_t SMEM = (A_BYTES + B_BYTES) > 73728 ? (A_BYTES + B_BYTES) : 73728;
  // kind::tf32 instruction descriptor: F32 accumulate, A and B TF32,
  // both K-major, N = NB, M = 128.
  static constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(NB >> 3) << 17) |
                                    (static_cast<uint32_t>(TILE >> 4) << 24);
  static_assert(NB <= TMEM_COLS, "accumulator columns");
};

__host__ __device__ inline int op_off(int row, int j, int sbo) {
  return (row >> 3) * sbo + (j >> 2) * 128 + (row & 7) * 16 + (j & 3) * 4;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t sbo) {
  // start address, leading byte offset 128, stride byte offset, version 1, no swizzle
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFF) | (static_cast<uint64_t>(128 >> 4) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (static_cast<uint64_t>(1) << 46);
}
__device__ __forceinline__ void mma_tf32(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dt),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void ld4(uint32_t taddr, float (&v)[4]) {
  uint32_t a, b, c, d;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
               : "r"(taddr));
  v[0] = __uint_as_float(a);
  v[1] = __uint_as_float(b);
  v[2] = __uint_as_float(c);
  v[3] = __uint_as_float(d);
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t try_wait(const uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done;
}
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

}  // namespace tf

// B operand of k_fista_tf32: G / (n L) rounded to TF32, zero padded, in the
// operand layout (NB x KA).  One thread per element.
template <int K>
__global__ void k_gtf32(const double* __restrict__ G, int Kp, double scale, float* __restrict__ out) {
  using S = tf::Shape<K>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S::NB * S::KA) return;
  const int n = i / S::KA, k = i % S::KA;
  const float v = (n < K && k < K) ? tf::to_tf32(static_cast<float>(G[n * Kp + k] * scale)) : 0.f;
  out[tf::op_off(n, k, S::SBO) / 4] = v;
}

struct Tf32Params {
  const float* gop;            // B operand (Shape<K>::B_BYTES), from k_gtf32
  const double* B;             // right-hand sides M^T s, rows of stride Kp
  int Kp;
  float* X32;                  // out: the iterate after `iters` iterations, rows of stride Kp
  double c_step;               // 1 / (n L): scale of b
  double step;                 // 1 / L
  double thr;                  // step * alpha (when alpha_v is null)
  const double* alpha_v;       // per-voxel alpha, or nullptr
  int iters;                   // iterations per tile
  const double* mom;           // Nesterov momentum (t_k - 1) / t_{k+1}, k < iters
  int non_negative;
  const int64_t* list;         // work list of voxel positions, or nullptr (= 0 .. n_work-1)
  int64_t n_work;
  unsigned long long* queue;   // next unassigned tile
  unsigned long long* batches; // MMA batches issued (one per tile iteration), summed
  int* error;                  // set to 1 when a tensor-core wait gives up
  unsigned long long wait_ns;  // limit of one wait for the tensor cores
};

// TF32 FISTA on tiles of 128 voxels.  Two CTAs per SM: while one waits for
// its products the other updates.  Per iteration one thread issues KS MMAs
// D = Y G~ (D in tensor memory, lane r = voxel r), the 256 threads read D
// back (two threads per voxel, CPT columns each) and apply the FISTA update
//     z = y - (D - b~),  x+ = soft(z, alpha / L),  y+ = x+ + mom (x+ - x)
// with G~ = G / (n L), b~ = b / (n L), writing y+ over y in the A operand.
// x and b~ stay in registers.  Every voxel of a tile runs exactly `iters`
// iterations, so a tile has no tail.  A NaN sample gives a NaN b~ and keeps
// that voxel's row NaN (rows do not mix in the product); the polish reports
// such a voxel as zero and uncertified.
template <int K, bool NONNEG>
__global__ void __launch_bounds__(tf::THREADS, 2) k_fista_tf32(Tf32Params p) {
  using namespace tf;
  using S = Shape<K>;
  constexpr int CPT = S::CPT;
  extern __shared__ __align__(1024) unsigned char smem_tf[];
  unsigned char* sA = smem_tf;
  unsigned char* sB = sA + S::A_BYTES;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ __align__(8) uint64_t mbar_b;  // the B operand's bulk copy
  __shared__ uint32_t tmem_slot;
  __shared__ int s_abort;
  __shared__ unsigned long long s_tile;
  constexpr int MOM_SMEM = 512;
  __shared__ float s_mom[MOM_SMEM];

  const int tid = threadIdx.x, warp = tid >> 5;
  const int part = tid >> 7, r = tid & (TILE - 1);
  const uint32_t lane_base = static_cast<uint32_t>((warp & 3) * 32) << 16;
  const int j_lo = part * CPT;

  for (int i = tid; i < S::A_BYTES / 16; i += THREADS) reinterpret_cast<uint4*>(sA)[i] = make_uint4(0, 0, 0, 0);
  for (int i = tid; i < min(p.iters, MOM_SMEM); i += THREADS) s_mom[i] = static_cast<float>(p.mom[i]);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar_b)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  fence_before();
  __syncthreads();
  fence_after();
  // B (the TF32 Gram operand, already in its shared-memory image in global
  // memory) by one bulk copy on the copy engine; 16-byte aligned addresses
  // and a size that is a multiple of 16 bytes, no multicast
  static_assert(S::B_BYTES % 16 == 0 && S::A_BYTES % 16 == 0, "bulk copy granularity");
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&mbar_b)),
                 "r"(static_cast<uint32_t>(S::B_BYTES))
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(sB)),
        "l"(p.gop), "r"(static_cast<uint32_t>(S::B_BYTES)), "r"(smem_u32(&mbar_b))
        : "memory");
    uint32_t done = 0;
    const uint64_t t0 = globaltimer_ns();
    while (!done && globaltimer_ns() - t0 < kWaitNs) done = try_wait(&mbar_b, 0);
    if (!done) {  // give the copy a second bound to land before the CTA can leave
      s_abort = 1;
      const uint64_t t1 = globaltimer_ns();
      while (!done && globaltimer_ns() - t1 < kWaitNs) done = try_wait(&mbar_b, 0);
    }
  }
  __syncthreads();
  const uint32_t tbase = tmem_slot;
  const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
  const int64_t n_tiles = (p.n_work + TILE - 1) / TILE;
  uint32_t phase = 0;
  unsigned long long n_batches = 0;

  while (!s_abort) {  // (set before the first tile only if the operand copy failed)
    __syncthreads();  // every thread has read the previous tile index
    if (tid == 0) s_tile = atomicAdd(p.queue, 1ull);
    __syncthreads();
    const unsigned long long tile = s_tile;
    if (tile >= static_cast<unsigned long long>(n_tiles)) break;
    const int64_t pos = static_cast<int64_t>(tile) * TILE + r;
    const int64_t v = pos < p.n_work ? (p.list ? p.list[pos] : pos) : -1;
    const float thr = static_cast<float>(v >= 0 && p.alpha_v ? p.step * p.alpha_v[v] : p.thr);
    float x[CPT], bb[CPT];
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
      const int j = j_lo + i;
      x[i] = 0.f;
      bb[i] = (v >= 0 && j < K) ? static_cast<float>(p.B[v * p.Kp + j] * p.c_step) : 0.f;
    }
    // y = 0: this thread's columns of its row
#pragma unroll
    for (int c = 0; c < CPT / 4; ++c)
      if (j_lo + 4 * c < S::KA)
        *reinterpret_cast<float4*>(sA + op_off(r, j_lo + 4 * c, S::SBO)) = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int it = 0; it < p.iters; ++it) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      fence_before();
      __syncthreads();  // y visible to the tensor core; the previous D reads are done
      if (tid == 0) {
        fence_after();
#pragma unroll
        for (int ks = 0; ks < S::KS; ++ks)
          mma_tf32(tbase, desc(a_base + ks * 256, S::SBO), desc(b_base + ks * 256, S::SBO), S::IDESC, ks ? 1u : 0u);
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
        ++n_batches;
      }
      const float mom = it < MOM_SMEM ? s_mom[it] : static_cast<float>(p.mom[it]);
      if (tid == 0) {  // one thread waits; the others sleep in the barrier
        uint32_t done = 0;
        const uint64_t t0 = globaltimer_ns();
        while (!done && globaltimer_ns() - t0 < p.wait_ns) done = try_wait(&mbar, phase);
        if (!done) s_abort = 1;
      }
      phase ^= 1u;
      __syncthreads();
      fence_after();
      if (s_abort) break;
      // D in groups of three 4-column chunks: three loads, one wait
      constexpr int NCH = CPT / 4;
#pragma unroll
      for (int g = 0; g < (NCH + 2) / 3; ++g) {
        float d[3][4];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          const int c = 3 * g + u;
          if (c < NCH && j_lo + 4 * c < K)  // warp-uniform
            ld4(tbase + lane_base + static_cast<uint32_t>(j_lo + 4 * c), d[u]);
        }
        wait_ld();
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          const int c = 3 * g + u, j0 = j_lo + 4 * c;
          if (c < NCH && j0 < K) {
            float4* yp = reinterpret_cast<float4*>(sA + op_off(r, j0, S::SBO));
            const float4 y4 = *yp;
            const float yv[4] = {y4.x, y4.y, y4.z, y4.w};
            float yn[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const int i = 4 * c + k;
              const float z = yv[k] - (d[u][k] - bb[i]);
              // soft threshold: z - clamp(z, -thr, thr) (zero inside the band),
              // or its non-negative form max(z - thr, 0)
              const float xn = NONNEG ? fmaxf(z - thr, 0.f) : z - fminf(fmaxf(z, -thr), thr);
              yn[k] = fmaf(mom, xn - x[i], xn);
              x[i] = xn;
            }
            *yp = make_float4(yn[0], yn[1], yn[2], yn[3]);
          }
        }
      }
    }
    if (s_abort) break;
    if (v >= 0) {
#pragma unroll
      for (int i = 0; i < CPT; ++i)
        if (j_lo + i < K) p.X32[v * p.Kp + j_lo + i] = x[i];
    }
  }
  if (s_abort && tid == 0) {
    atomicExch(p.error, 1);
    // let any products still in flight land before the columns are freed
    uint32_t done = 0;
    const uint64_t t0 = globaltimer_ns();
    while (!done && globaltimer_ns() - t0 < tf::kWaitNs) done = tf::try_wait(&mbar, phase ^ 1u);
  }
  if (tid == 0 && p.batches) atomicAdd(p.batches, n_batches);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(tf::TMEM_COLS));
}

// ---------------------------------------------------------------- polish

struct PolishParams {
  const double* G;             // Kp x Kp Gram M^T M
  const double* B;             // right-hand sides, rows of stride Kp
  const float* S32;            // starting iterate (support and signs), rows of stride Kp; or
  const double* S64;           //   the same in FP64 (one of the two is set)
  double* X;                   // out: FP64 coefficients, rows of stride Kp
  uint32_t* iters;             // out: it_base + rounds (or iters[v] + rounds with it_add)
  uint8_t* conv;               // out: 1 = KKT certified
  double* kkt;                 // out (nullable): max of the active and inactive KKT residuals
  int K, Kp;
  double n_samples;
  double alpha;                // when alpha_v is null
  const double* alpha_v;
  int non_negative;
  double kappa;                // certificate: every off-support |g_j| <= alpha (1 + kappa)
  int rounds;                  // round limit
  int it_base;
  int it_add;                  // add the rounds to iters[v] instead of it_base
  int keep_on_fail;            // leave X untouched for voxels not certified (a fallback fit's result)
  int cap;                     // largest support held in the warp's shared slice
  const int64_t* list;         // work list (nullable: 0 .. n_work-1)
  const unsigned long long* list_len;  // its device-side length (nullable: n_work)
  int64_t n_work;
  int64_t* overflow;           // voxels whose support outgrew `cap`
  unsigned long long* n_overflow;
  int64_t* failed;             // voxels not certified within the round limit (nullable)
  unsigned long long* n_failed;
  unsigned long long* n_uncertified;  // voxels not certified, counted (nullable)
  unsigned long long* round_total;    // rounds, summed (nullable)
  unsigned long long* kkt_max_bits;   // largest KKT residual of a certified voxel, as bits (nullable)
};

// Per-warp shared memory of k_l1_polish in doubles: the packed factor, the
// solve's right-hand side / solution by support position, the solution and
// b by coefficient, then the support list and the signs (ints).
__host__ __device__ __forceinline__ int polish_warp_doubles(int cap, int Kp) {
  return cap * (cap + 1) / 2 + cap + 2 * Kp + Kp;  // the last Kp doubles hold 2 Kp ints
}

// Start of row i of a packed lower triangle stored by rows, and the row of
// its entry e.
__device__ __forceinline__ int pk_row(int i) { return (i * (i + 1)) >> 1; }
__device__ __forceinline__ int tri_row(int e) {
  int r = static_cast<int>((sqrtf(8.f * static_cast<float>(e) + 1.f) - 1.f) * 0.5f);
  r += pk_row(r + 1) <= e;
  r -= pk_row(r) > e;
  return r;
}
constexpr int kTriTable = 32 * 33 / 2;  // entries of a packed triangle of order 32

// Row and column of entry e of a packed lower triangle, from the table when
// the triangle has order <= 32.
__device__ __forceinline__ void tri_entry(const uint16_t* tab, int e, int& r, int& k) {
  if (e < kTriTable) {
    const int rc = tab[e];
    r = rc >> 8;
    k = rc & 0xFF;
  } else {
    r = tri_row(e);
    k = e - pk_row(r);
  }
}

// Symmetric Gram matrix read by the polish: FP64 entries G[i * ld + j] in
// global or shared memory ...
struct GramDense {
  const double* p;
  int ld;
  __device__ __forceinline__ double operator()(int i, int j) const { return p[i * ld + j]; }
};
// ... or two FP32 planes hi + lo with G = hi + lo to 48 bits (hi = fl32(G),
// lo = fl32(G - hi)), each entry rebuilt in FP64.
struct GramHiLo {
  const float* hi;
  const float* lo;
  int ld;
  __device__ __forceinline__ double operator()(int i, int j) const {
    return static_cast<double>(hi[i * ld + j]) + static_cast<double>(lo[i * ld + j]);
  }
};

// The active-set polish of one voxel by one warp (the method described at
// k_l1_polish below).  G is a GramDense or GramHiLo; bw (Kp doubles) holds b; fl (Kp ints) the signs of
// the starting support and c (coefficient j = lane + 32 q) the starting
// point, both set by the caller; T, zw, zj, sidx are the warp's scratch (a
// support of up to `cap`).  On return c holds the certified minimiser when
// the voxel is certified; `round` counts the solves, `kkt_val` is the largest
// KKT residual of a certified voxel, `overflowed` reports a support above
// `cap` (the caller retries with more room).
template <int RPL, int RPS, class GM>
__device__ bool polish_warp(const GM& G, int K, int Kp, int cap, const double* bw, int* fl,
                            double (&c)[RPL], double* T, double* zw, double* zj, int* sidx,
                            const uint16_t* tri_rc, double n, double n_inv, double alpha, int non_negative,
                            double kappa, int max_rounds, int& round, double& kkt_val, bool& overflowed) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  bool certified = false;
  overflowed = false;
  kkt_val = 0.0;
  round = 0;
  int s = 0;
    while (round < max_rounds) {
      ++round;
      // support in index order
      s = 0;
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int j = lane + 32 * q;
        const bool in = j < K && fl[j] != 0;
        const unsigned bal = __ballot_sync(full, in);
        if (in) sidx[s + __popc(bal & ((1u << lane) - 1u))] = j;
        s += __popc(bal);
      }
      __syncwarp();
      if (s > cap) {
        overflowed = true;
        break;
      }
      // G_SS into the packed lower triangle (by rows), one entry per lane
      for (int e = lane; e < pk_row(s); e += 32) {
        int i, k;
        tri_entry(tri_rc, e, i, k);
        T[e] = G(sidx[i], sidx[k]);
      }
      // right-hand side b_S - n alpha sigma_S in registers: entry q = lane + 32 c
      double rv[RPS];
#pragma unroll
      for (int cc = 0; cc < RPS; ++cc) {
        const int q = lane + 32 * cc;
        rv[cc] = q < s ? bw[sidx[q]] - n * alpha * static_cast<double>(fl[sidx[q]]) : 0.0;
      }
      __syncwarp();
      // Cholesky by columns: column jc scaled by 1 / L_jj, then the trailing
      // triangle updated one entry per lane.  The diagonal keeps 1 / L_jj
      // for the solves.
      bool pd = true;
      for (int jc = 0; jc < s; ++jc) {
        const double d = T[pk_row(jc) + jc];
        if (!(d > 0.0)) {  // every lane read the same pivot
          pd = false;
          break;
        }
        const double rinv = rsqrt(d);
        for (int i = jc + 1 + lane; i < s; i += 32) T[pk_row(i) + jc] *= rinv;
        __syncwarp();
        if (lane == 0) T[pk_row(jc) + jc] = rinv;
        const int m = s - jc - 1;
        for (int e = lane; e < pk_row(m); e += 32) {
          int r, kk;
          tri_entry(tri_rc, e, r, kk);
          const int i = jc + 1 + r, k = jc + 1 + kk;
          T[pk_row(i) + k] = fma(-T[pk_row(i) + jc], T[pk_row(k) + jc], T[pk_row(i) + k]);
        }
        __syncwarp();
      }
      if (!pd) break;
      // L y = rhs, then L^T z = y, in registers (entry i lives in lane i % 32)
      for (int i = 0; i < s; ++i) {
        double sel = rv[0];
#pragma unroll
        for (int cc = 1; cc < RPS; ++cc)
          if (cc == (i >> 5)) sel = rv[cc];
        const double yi = __shfl_sync(full, sel, i & 31) * T[pk_row(i) + i];
#pragma unroll
        for (int cc = 0; cc < RPS; ++cc) {
          const int q = lane + 32 * cc;
          if (q > i && q < s) rv[cc] = fma(-T[pk_row(q) + i], yi, rv[cc]);
          if (q == i) rv[cc] = yi;
        }
      }
      for (int i = s - 1; i >= 0; --i) {
        double sel = rv[0];
#pragma unroll
        for (int cc = 1; cc < RPS; ++cc)
          if (cc == (i >> 5)) sel = rv[cc];
        const double zi = __shfl_sync(full, sel, i & 31) * T[pk_row(i) + i];
        const int ri = pk_row(i);
#pragma unroll
        for (int cc = 0; cc < RPS; ++cc) {
          const int q = lane + 32 * cc;
          if (q < i) rv[cc] = fma(-T[ri + q], zi, rv[cc]);
          if (q == i) rv[cc] = zi;
        }
      }
      for (int j = lane; j < Kp; j += 32) zj[j] = 0.0;
      __syncwarp();
#pragma unroll
      for (int cc = 0; cc < RPS; ++cc) {
        const int q = lane + 32 * cc;
        if (q < s) {
          zw[q] = rv[cc];
          zj[sidx[q]] = rv[cc];
        }
      }
      __syncwarp();
      // a coefficient that would change sign: move towards z up to the first
      // zero crossing, and drop the coefficients that reach zero there
      double tq[RPL];
      double tmin = 2.0;
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int j = lane + 32 * q;
        tq[q] = 2.0;
        if (j < K && fl[j] != 0) {
          const double z = zj[j];
          if (z * static_cast<double>(fl[j]) <= 0.0) tq[q] = c[q] / (c[q] - z);  // in [0, 1)
        }
        tmin = fmin(tmin, tq[q]);
      }
      for (int o = 16; o > 0; o >>= 1) tmin = fmin(tmin, __shfl_xor_sync(full, tmin, o));
      if (tmin < 1.0) {
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
          const int j = lane + 32 * q;
          if (j < K && fl[j] != 0) {
            const double cn = fma(tmin, zj[j] - c[q], c[q]);
            if (tq[q] <= tmin * (1.0 + 1e-12) || cn * static_cast<double>(fl[j]) <= 0.0) {
              fl[j] = 0;
              c[q] = 0.0;
            } else {
              c[q] = cn;
            }
          }
        }
        __syncwarp();
        continue;
      }
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int j = lane + 32 * q;
        c[q] = j < K ? zj[j] : 0.0;
      }
      // g = (G c - b) / n; the worst off-support violation joins S with the
      // sign opposite to g_j (+1 for a non-negative fit)
      double best = -INFINITY, act = 0.0;
      int bj = 0x7fffffff, bsg = 0;
      double gq[RPL];
#pragma unroll
      for (int q = 0; q < RPL; ++q) gq[q] = 0.0;
      for (int i = 0; i < s; ++i) {  // G symmetric: row S_i, columns j = lane + 32 q
        const int si = sidx[i];
        const double zi = zw[i];
#pragma unroll
        for (int q = 0; q < RPL; ++q)
          if (lane + 32 * q < K) gq[q] = fma(G(si, lane + 32 * q), zi, gq[q]);
      }
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int j = lane + 32 * q;
        if (j < K) {
          const double g = (gq[q] - bw[j]) * n_inv;
          if (fl[j] != 0) {
            act = fmax(act, fabs(g + alpha * static_cast<double>(fl[j])));
          } else {
            const double exc = non_negative ? -g - alpha : fabs(g) - alpha;
            if (exc > best) {
              best = exc;
              bj = j;
              bsg = (non_negative || g < 0.0) ? 1 : -1;
            }
          }
        }
      }
      for (int o = 16; o > 0; o >>= 1) {  // arg-max over the warp, ties to the lowest index
        const double ob = __shfl_xor_sync(full, best, o);
        const int oj = __shfl_xor_sync(full, bj, o);
        const int os = __shfl_xor_sync(full, bsg, o);
        if (ob > best || (ob == best && oj < bj)) {
          best = ob;
          bj = oj;
          bsg = os;
        }
        act = fmax(act, __shfl_xor_sync(full, act, o));
      }
      __syncwarp();
      if (best > kappa * alpha && bj < K) {
        if (lane == 0) fl[bj] = bsg;  // joins at zero; the next solve gives it its sign
        __syncwarp();
        continue;
      }
      certified = true;
      kkt_val = fmax(act, fmax(best, 0.0));
      break;
    }
  return certified;
}

// One warp per voxel, an active-set method in the manner of Lawson and
// Hanson's NNLS with signs in place of the non-negativity: the current point
// c keeps the signs sigma of its support S (c_j sigma_j > 0 on S, c_j = 0
// off it).  A round solves the sign-fixed problem on S, G_SS z = b_S -
// n alpha sigma_S (the LASSO objective on the orthant of sigma).  If every
// z_j keeps its sign, c = z; then the coordinate with the largest
// off-support violation |g_j| - alpha > kappa alpha (g = (G c - b) / n)
// joins S with sigma_j = -sign(g_j), or, with none left, c is certified.  If
// some z_j changes sign, c moves towards z up to the first coordinate that
// reaches zero, which leaves S, and the round repeats on the smaller S.  The
// objective decreases at every move, so no support is visited twice; a
// coordinate that joins S after a consistent solve takes its sign in the
// next solve (the NNLS argument), so the method ends at the minimiser.  It
// starts from the support-identification iterate, whose support and signs
// are nearly right (most voxels certify in the first round).  G is read
// through L1.
template <int RPL, int RPS>  // ceil(K / 32); ceil(cap / 32)
__global__ void __launch_bounds__(256, 4) k_l1_polish(PolishParams p) {
  extern __shared__ __align__(16) double pol_smem[];
  // (row, column) of the entries of a packed lower triangle of order <= 32
  __shared__ uint16_t tri_rc[kTriTable];
  for (int e = threadIdx.x; e < kTriTable; e += blockDim.x) {
    const int r = tri_row(e);
    tri_rc[e] = static_cast<uint16_t>((r << 8) | (e - pk_row(r)));
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int K = p.K, Kp = p.Kp, cap = p.cap;
  double* T = pol_smem + static_cast<size_t>(warp) * polish_warp_doubles(cap, Kp);
  double* zw = T + cap * (cap + 1) / 2;   // [cap] rhs, then the solution, by support position
  double* zj = zw + cap;                  // [Kp] the solution by coefficient
  double* bw = zj + Kp;                   // [Kp] b
  int* sidx = reinterpret_cast<int*>(bw + Kp);
  int* fl = sidx + Kp;                    // sign of each coefficient on S, 0 off it
  const unsigned full = 0xffffffffu;
  const double n = p.n_samples, n_inv = 1.0 / p.n_samples;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  const int64_t n_items = p.list_len ? static_cast<int64_t>(*p.list_len) : p.n_work;
  unsigned long long rounds_sum = 0;

  for (int64_t item = static_cast<int64_t>(blockIdx.x) * nw + warp; item < n_items;
       item += static_cast<int64_t>(gridDim.x) * nw) {
    const int64_t v = p.list ? p.list[item] : item;
    const double alpha = p.alpha_v ? p.alpha_v[v] : p.alpha;
    double c[RPL];  // current point, coefficient j = lane + 32 q
    bool finite = true;
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
      const int j = lane + 32 * q;
      double s0 = 0.0, b = 0.0;
      if (j < K) {
        b = p.B[v * Kp + j];
        s0 = p.S32 ? static_cast<double>(p.S32[v * Kp + j]) : p.S64[v * Kp + j];
      }
      if (j < Kp) bw[j] = b;
      finite = finite && isfinite(b) && isfinite(s0);
      int f = s0 > 0.0 ? 1 : (s0 < 0.0 ? -1 : 0);
      if (p.non_negative && f < 0) f = 0;
      c[q] = f != 0 ? s0 : 0.0;
      if (j < Kp) fl[j] = f;
    }
    finite = __all_sync(full, finite);
    __syncwarp();
    if (!finite) {  // a NaN or infinite sample: zero coefficients, not certified
      for (int j = lane; j < Kp; j += 32) p.X[v * Kp + j] = 0.0;
      if (lane == 0) {
        p.conv[v] = 0;
        p.iters[v] = p.it_add ? p.iters[v] : static_cast<uint32_t>(p.it_base);
        if (p.kkt) p.kkt[v] = nan;
        if (p.n_uncertified) atomicAdd(p.n_uncertified, 1ull);
      }
      __syncwarp();
      continue;
    }
    bool overflowed = false;
    double kkt_val = 0.0;
    int round = 0;
    const bool certified = polish_warp<RPL, RPS>(GramDense{p.G, Kp}, K, Kp, cap, bw, fl, c, T, zw, zj, sidx, tri_rc, n, n_inv,
                                                 alpha, p.non_negative, p.kappa, p.rounds, round, kkt_val,
                                                 overflowed);
    rounds_sum += round;
    if (overflowed) {
      if (lane == 0) p.overflow[atomicAdd(p.n_overflow, 1ull)] = v;
      __syncwarp();
      continue;
    }
    if (certified || !p.keep_on_fail) {
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int j = lane + 32 * q;
        if (j < Kp) p.X[v * Kp + j] = (certified && j < K) ? c[q] : 0.0;
      }
    }
    if (lane == 0) {
      p.conv[v] = certified ? 1 : 0;
      p.iters[v] = (p.it_add ? p.iters[v] : static_cast<uint32_t>(p.it_base)) + static_cast<uint32_t>(round);
      if (p.kkt) p.kkt[v] = certified ? kkt_val : nan;
      if (!certified && p.failed) p.failed[atomicAdd(p.n_failed, 1ull)] = v;
      // a pass with a failure list hands its failures on; the last pass counts them
      if (!certified && !p.failed && p.n_uncertified) atomicAdd(p.n_uncertified, 1ull);
      if (certified && p.kkt_max_bits)  // a non-negative double orders as its bit pattern
        atomicMax(p.kkt_max_bits, static_cast<unsigned long long>(__double_as_longlong(kkt_val)));
    }
    __syncwarp();
  }
  if (p.round_total && lane == 0) atomicAdd(p.round_total, rounds_sum);  // every lane holds the warp's count
}

}  // namespace csd
