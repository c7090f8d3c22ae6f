// Mixed-precision FISTA (radial order 6, K = 72) on the 5th-generation tensor
// cores: the Gram products run as exact int8 digit-slice GEMMs
// (tcgen05.mma kind::i8, int32 accumulators in tensor memory) and every other
// piece of state stays FP64.
//
// The FISTA update needs G y - b (fista.rs:90-107 in Gram form).  Written
// incrementally, with d_k = x_k - x_{k-1}, u_k = G x_k - b and P_k = G d_k,
//
//     G y_k - b = u_k + mom_{k-1} P_k,     u_k = u_{k-1} + P_k,
//
// so the only product per iteration is P = G d.  d is scaled per voxel to a
// 30-bit integer q (|q| <= 2^30) and split into four balanced base-256 digits
// (each in [-128, 127]); every column of G is scaled to a 38-bit integer and
// split into five.  The 14 digit pairs with s + t <= 4 are summed per level
// l = s + t on the tensor cores, exactly, in int32; the five level sums are
// recombined in FP64.  The product is then accurate to about 2^-32 of
// max|d| * max|G column| - where a plain TF32/BF16 product (2^-11 / 2^-8)
// would leave the FP64 iterate path - and u carries the FP64 accumulation.
//
// A voxel whose stopping decision could flip under that rounding (relative
// change within 1 % of tol at the stop, or a near miss followed by more
// iterations) is written to a list; the host re-runs those voxels on the FP64
// kernel, so every output either follows the FP64 iterate path closely or is
// the FP64 result itself.
//
// One CTA per SM holds a tile of 128 voxels: TMEM lane r = voxel r, two
// threads per voxel (coefficients split 36/36), x and d in registers, u in
// shared memory.  Per iteration: FP64 update -> per-voxel exponent -> digits
// to shared memory -> one thread issues 36 MMAs (the planes of a level are
// concatenated along K) -> tcgen05.commit to an mbarrier -> tcgen05.ld.
#pragma once

#include <cstdint>

namespace csd {
namespace i8 {

constexpr int KC = 72;                         // coefficients (radial order 6)
constexpr int NB = 80;                         // MMA N: coefficients padded to a multiple of 16
constexpr int ND = 4, NG = 5, NLEV = 5;        // digits of d, digits of G, kept levels
constexpr int A_CH = ND * 5 + 1;               // 16-byte K chunks per 8-row group (+1 zero chunk)
constexpr int B_CH = NG * 5 + 1;
constexpr int A_SBO = A_CH * 128;              // byte stride between 8-row core-matrix groups
constexpr int B_SBO = B_CH * 128;
constexpr int TILE = 128;                      // voxels per CTA (MMA M)
constexpr int A_BYTES = (TILE / 8) * A_SBO;    // 43008
constexpr int B_BYTES = (NB / 8) * B_SBO;      // 33280
constexpr int THREADS = 256;                   // two threads per voxel
constexpr int TMEM_COLS = 512;                 // NLEV * NB = 400 used
constexpr int D_BITS = 30, G_BITS = 38;
constexpr int MMAS_PER_ITER = 3 + 5 + 8 + 10 + 10;
constexpr uint64_t kWaitNs = 2000000000ull;    // give up on one MMA batch after 2 s
constexpr int RING = 16;                       // prefetched voxels per CTA
constexpr int MOM_SMEM = 1024;                 // momentum factors held in shared memory
constexpr int PRODUCER_WARP = 7;               // tops the prefetch ring up while the MMAs run
// dynamic shared memory: A, B, u [KC][TILE], prefetch ring (b and warm rows;
// u, x and d rows of resumed voxels),
// momentum table, column exponents, per-voxel state
constexpr size_t kSmem = A_BYTES + B_BYTES + sizeof(double) * KC * TILE + sizeof(double) * 3 * RING * KC +
                         sizeof(double) * MOM_SMEM + sizeof(double) * RING + sizeof(int64_t) * RING +
                         sizeof(int) * NB + sizeof(double) * 5 * TILE + sizeof(int64_t) * 2 * TILE +
                         sizeof(unsigned) * 2 * TILE + sizeof(int) * 5 * TILE + sizeof(int) * RING;

// Byte offset of digit plane s, coefficient j of voxel row r in the A operand
// (canonical K-major, no swizzle: 8 rows x 16 bytes per core matrix).
__host__ __device__ inline int a_off(int r, int s, int j) {
  return (r >> 3) * A_SBO + (5 * s + (j >> 4)) * 128 + (r & 7) * 16 + (j & 15);
}
// Byte offset of digit t of G[j][n] in the B operand; planes are stored in
// descending t so that every level's pairs are one contiguous K range.
__host__ __device__ inline int b_off(int n, int t, int j) {
  return (n >> 3) * B_SBO + (5 * (4 - t) + (j >> 4)) * 128 + (n & 7) * 16 + (j & 15);
}

}  // namespace i8

// G's digit planes (B operand layout) and per-column exponents: one block of
// 128 threads per output column n < NB; f[n] is the smallest f with
// max_j |G[j][n]| < 2^f.
__global__ void k_gdigits(const double* __restrict__ G, int Kp, uint8_t* __restrict__ gdig, int* __restrict__ fexp) {
  const int n = blockIdx.x;
  __shared__ double red[128];
  double m = 0.0;
  if (n < i8::KC)
    for (int j = threadIdx.x; j < i8::KC; j += blockDim.x) m = fmax(m, fabs(G[j * Kp + n]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const double mx = red[0];
  int f = 0;
  if (mx > 0.0) f = ilogb(mx) + 1;  // mx < 2^f
  if (threadIdx.x == 0) fexp[n] = f;
  if (n >= i8::KC) return;
  const double sc = ldexp(1.0, i8::G_BITS - f);
  for (int j = threadIdx.x; j < i8::KC; j += blockDim.x) {
    const long long q = llrint(G[j * Kp + n] * sc);  // |q| <= 2^38
    const unsigned long long w = static_cast<unsigned long long>(q) + 0x80808080ull;
#pragma unroll
    for (int t = 1; t < i8::NG; ++t)  // balanced digits: byte (4 - t) of w minus 128
      gdig[i8::b_off(n, t, j)] = static_cast<uint8_t>(((w >> (8 * (4 - t))) & 0xFF) ^ 0x80);
    gdig[i8::b_off(n, 0, j)] = static_cast<uint8_t>(static_cast<int8_t>(static_cast<long long>(w) >> 32));
  }
}

struct MixedParams {
  const uint8_t* gdig;         // B operand bytes (i8::B_BYTES)
  const int* fexp;             // i8::NB column exponents
  const double* B;             // V x 72 right-hand sides M^T s
  double* X;                   // V x 72 out
  const double* warm;          // V x 72 warm start, or nullptr
  uint32_t* iters;
  uint8_t* conv;
  double c_step;               // step * n_inv
  double thr;                  // step * alpha (when alpha_v is null)
  double step;
  const double* alpha_v;       // per-voxel alpha, or nullptr
  double tol;
  double band;                 // relative half-width of the stop-decision guard band
  int max_iter;
  int non_negative;
  unsigned long long* queue;
  const int64_t* list;
  int64_t n_work;
  const double* mom;
  unsigned long long* iter_total;
  int64_t* flagged;            // voxel ids to re-run in FP64
  unsigned long long* n_flagged;
  unsigned long long* batches; // MMA batches issued (36 MMAs each), summed
  int* error;                  // set to 1 when a tensor-core wait gives up
  unsigned long long wait_ns;  // limit of one wait for the tensor cores (the drain after a
                               // give-up keeps its own kWaitNs bound)
  // Two-pass schedule (as FistaParams).  Pass 1 (cap > 0, resume = 0): a
  // voxel neither finished nor flagged after `cap` iterations stores its
  // exact state - x, d and u rows in Xp, Dp, Up and its guard-band flag in
  // Np - appends its position to `pend` with a prediction of the iterations
  // it still needs in `pend_key`, and frees its slot; its X row stays
  // untouched (a flagged voxel's FP64 re-run starts from the original
  // point).  Pass 2 (resume = 1) takes those voxels (the order of `list`,
  // `*n_work_dev` of them) from that state at iteration `cap`.
  int cap;
  int resume;
  double* Xp;
  double* Dp;
  double* Up;
  uint8_t* Np;
  int64_t* pend;
  float* pend_key;
  unsigned long long* n_pend;
  const unsigned long long* n_work_dev;
};

namespace i8 {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo) {
  // start address, leading byte offset 128 (the two 16-byte K halves of a
  // 32-byte k-step), stride byte offset (8-row groups), version 1, no swizzle
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFF) | (static_cast<uint64_t>(128 >> 4) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (static_cast<uint64_t>(1) << 46);
}
// kind::i8 instruction descriptor: s32 accumulate, A and B signed, K-major,
// N = 80, M = 128.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(NB >> 3) << 17) |
                            (static_cast<uint32_t>(TILE >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dt),
      "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
}
__device__ __forceinline__ void ld4(uint32_t taddr, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
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

// Exact int32 -> double without a conversion instruction: the bit pattern
// (0x43380000, v + 2^31) is the double 1.5 * 2^52 + 2^31 + v.
__device__ __forceinline__ double i2d(int v) {
  return __hiloint2double(0x43380000, static_cast<int>(static_cast<unsigned>(v) ^ 0x80000000u)) -
         (0x1.8p52 + 0x1p31);
}
// Recombined level sums 256 * (L0 + 2^-8 L1 + 2^-16 L2 + 2^-24 L3 + 2^-32 L4)
// = A + 2^-16 B + 2^-24 C with A = 256 L0 + L1, B = 256 L2 + L3, C = L4, all
// exact in int32 (|L0| <= 72 * 65^2, |L2| <= 3 * 72 * 128^2).
__device__ __forceinline__ double combine(uint32_t l0, uint32_t l1, uint32_t l2, uint32_t l3, uint32_t l4) {
  const int a = static_cast<int>(l0) * 256 + static_cast<int>(l1);
  const int b = static_cast<int>(l2) * 256 + static_cast<int>(l3);
  const int c = static_cast<int>(l4);
  return fma(fma(i2d(c), 0x1p-8, i2d(b)), 0x1p-16, i2d(a));
}
// 2^e as a double for -1000 < e < 1000.
__device__ __forceinline__ double pow2(int e) { return __hiloint2double((e + 1023) << 20, 0); }

// q = rint(d * scale) for |d * scale| <= 2^30, then the four balanced digits
// as the bytes of a word: byte b = digit (3 - b).
__device__ __forceinline__ uint32_t digits(double d, double scale) {
  const double t = fma(d, scale, 0x1.8p52);  // + 1.5 * 2^52: rounds to an integer in the low word
  const uint32_t q = static_cast<uint32_t>(__double2loint(t));
  return (q + 0x00808080u) ^ 0x00808080u;
}
// Transpose four digit words (coefficients j..j+3) into four plane words.
__device__ __forceinline__ void planes4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t (&pl)[4]) {
  const uint32_t t0 = __byte_perm(w0, w1, 0x5140), t1 = __byte_perm(w2, w3, 0x5140);
  const uint32_t t2 = __byte_perm(w0, w1, 0x7362), t3 = __byte_perm(w2, w3, 0x7362);
  pl[3] = __byte_perm(t0, t1, 0x5410);  // byte 0 of each word = digit 3
  pl[2] = __byte_perm(t0, t1, 0x7632);  // byte 1 = digit 2
  pl[1] = __byte_perm(t2, t3, 0x5410);  // byte 2 = digit 1
  pl[0] = __byte_perm(t2, t3, 0x7632);  // byte 3 = digit 0 (top, signed)
}

// The coefficients of part p (0 or 1): two 16-coefficient groups and one
// 4-coefficient quarter of the last group.  Local index i -> coefficient.
__device__ __forceinline__ int coef_of(int part, int i) {
  return i < 32 ? ((i >> 4) * 32 + part * 16 + (i & 15)) : (64 + part * 4 + (i - 32));
}

}  // namespace i8

__global__ void __launch_bounds__(i8::THREADS, 1) k_fista_i8(MixedParams p) {
  using namespace i8;
  constexpr int CPT = 36;  // coefficients per thread
  extern __shared__ __align__(1024) unsigned char smem_i8[];
  unsigned char* sA = smem_i8;                                   // A_BYTES
  unsigned char* sB = sA + A_BYTES;                              // B_BYTES
  double* sU = reinterpret_cast<double*>(sB + B_BYTES);          // [KC][TILE]
  double* rB = sU + KC * TILE;                                   // [RING][KC] prefetched b rows
  double* rW = rB + RING * KC;                                   // [RING][KC] prefetched warm rows
  double* rD = rW + RING * KC;                                   // [RING][KC] d rows of resumed voxels
  double* sMom = rD + RING * KC;                                 // [MOM_SMEM]
  double* rThr = sMom + MOM_SMEM;                                // [RING]
  int64_t* rVid = reinterpret_cast<int64_t*>(rThr + RING);       // [RING]
  int* sF = reinterpret_cast<int*>(rVid + RING);                 // [NB]
  double* sDx = reinterpret_cast<double*>(sF + NB);              // [2][TILE]
  double* sXn = sDx + 2 * TILE;                                  // [2][TILE]
  double* sThr = sXn + 2 * TILE;                                 // [TILE]
  int64_t* sVid = reinterpret_cast<int64_t*>(sThr + TILE);       // [TILE] current voxel
  int64_t* sOld = sVid + TILE;                                   // [TILE] voxel to write out
  unsigned* sMax = reinterpret_cast<unsigned*>(sOld + TILE);     // [2][TILE] max |d| high words
  int* sIt = reinterpret_cast<int*>(sMax + 2 * TILE);            // [TILE]
  int* sNear = sIt + TILE;                                       // [TILE]
  int* sFin = sNear + TILE;                                      // [TILE] 1: slot emptied this pass
  int* sSrc = sFin + TILE;                                       // [TILE] ring entry of a new voxel, -1: direct
  int* sPark = sSrc + TILE;                                      // [TILE] 1: the emptied slot's voxel is parked
  int* rNear = sPark + TILE;                                     // [RING] guard flag of a resumed voxel
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_abort, s_head, s_tail, s_exhausted;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int part = tid >> 7, r = tid & (TILE - 1);
  // warp w reads TMEM lanes 32 (w % 4) .. + 31: the rows of its voxels
  const uint32_t lane_base = static_cast<uint32_t>((warp & 3) * 32) << 16;
  const int n_mom = min(p.max_iter, MOM_SMEM);

  // ---- one-time setup: zero the A operand (pads stay zero), stage G's digits
  for (int i = tid; i < A_BYTES / 16; i += THREADS) reinterpret_cast<uint4*>(sA)[i] = make_uint4(0, 0, 0, 0);
  for (int i = tid; i < B_BYTES / 16; i += THREADS)
    reinterpret_cast<uint4*>(sB)[i] = reinterpret_cast<const uint4*>(p.gdig)[i];
  for (int i = tid; i < NB; i += THREADS) sF[i] = p.fexp[i];
  for (int i = tid; i < n_mom; i += THREADS) sMom[i] = p.mom[i];
  if (tid < TILE) {
    sVid[tid] = -1;
    sOld[tid] = -1;
    sIt[tid] = 0;
    sNear[tid] = 0;
    sFin[tid] = 0;
    sSrc[tid] = -1;
    sPark[tid] = 0;
    sThr[tid] = p.thr;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
    s_head = 0;
    s_tail = 0;
    s_exhausted = 0;
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tbase = tmem_slot;

  double x[CPT], d[CPT];
#pragma unroll
  for (int i = 0; i < CPT; ++i) x[i] = d[i] = 0.0;
  int e_vox = 0;          // exponent of this voxel's current digits
  uint32_t phase = 0;
  bool have_p = false;    // TMEM holds P for the current voxels
  unsigned long long executed = 0, n_batches = 0;
  const double tol = p.tol;
  const double lo_band = tol * (1.0 - p.band), hi_band = tol * (1.0 + p.band);
  // The stopping rule ||dx|| < tol max(||x||, 1e-12) (fista.rs:115-127) and
  // the guard band, compared in squares: a rounding-level difference from the
  // square-root form can only matter inside the band, where the FP64 kernel
  // decides anyway.
  const double tol2 = tol * tol, lo2 = lo_band * lo_band, hi2 = hi_band * hi_band;
  const unsigned long long nwork =
      p.n_work_dev ? *p.n_work_dev : static_cast<unsigned long long>(p.n_work);  // work-list length
  // pass 1 of the two-pass schedule: sums of log2(rel^2) and k log2(rel^2)
  // over iterations w0+1 .. cap of this thread's slot (part-0 threads)
  const int w0 = p.cap - p.cap / 2;
  float ksl = 0.f, kskl = 0.f;

  while (true) {
    const int64_t vid = sVid[r];
    // ---- phase 1: FP64 update from P = G d (skipped before the first MMA).
    // tcgen05.ld / wait::ld are .sync.aligned: every lane of the warp runs
    // them, empty slots included; an empty slot's results are discarded (its
    // x and d are cleared below and the stopping rule skips it).
    if (have_p) {
      const int it = sIt[r];
      const double mom_prev = it == 0 ? 0.0 : (it <= n_mom ? sMom[it - 1] : p.mom[it - 1]);
      const double thr = sThr[r];
      const double c = p.c_step;
      double dx2 = 0.0, xn2 = 0.0;
      unsigned mx = 0;
#pragma unroll
      for (int g4 = 0; g4 < CPT / 4; ++g4) {  // 4-coefficient batches
        const int j0 = coef_of(part, 4 * g4);
        uint32_t lv[NLEV][4];
#pragma unroll
        for (int l = 0; l < NLEV; ++l) ld4(tbase + lane_base + l * NB + j0, lv[l]);
        wait_ld();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int i = 4 * g4 + k, j = j0 + k;
          const double P = combine(lv[0][k], lv[1][k], lv[2][k], lv[3][k], lv[4][k]) * pow2(e_vox + sF[j] - 20);
          const double u = sU[j * TILE + r] + P;
          sU[j * TILE + r] = u;
          const double gy = fma(mom_prev, P, u);        // G y - b
          const double y = fma(mom_prev, d[i], x[i]);
          const double cand = fma(-c, gy, y);
          const double a = fabs(cand) - thr;             // soft threshold; NaN -> 0 as the reference
          double xn = a > 0.0 ? copysign(a, cand) : 0.0;
          if (p.non_negative) xn = fmax(xn, 0.0);
          const double dn = xn - x[i];
          dx2 = fma(dn, dn, dx2);
          xn2 = fma(xn, xn, xn2);
          mx = max(mx, static_cast<unsigned>(__double2hiint(dn)) & 0x7FFFFFFFu);
          x[i] = xn;
          d[i] = dn;
        }
      }
      sDx[part * TILE + r] = dx2;
      sXn[part * TILE + r] = xn2;
      sMax[part * TILE + r] = mx;
    }
    if (warp == PRODUCER_WARP) cp_async_wait_all();  // prefetched rows have landed
    fence_before();
    __syncthreads();  // B1: partial norms and prefetched rows visible; TMEM reads done

    // ---- stopping rule, guard and refill decision (one thread per voxel)
    if (part == 0) {
      const int64_t v = sVid[r];
      bool finish = false, write_out = true, park = false;
      if (have_p && v >= 0) {
        ++executed;
        const int it = sIt[r] + 1;
        sIt[r] = it;
        const double dx2 = sDx[r] + sDx[TILE + r];
        const double ref2 = fmax(sXn[r] + sXn[TILE + r], 1e-24);
        const bool converged = dx2 < tol2 * ref2;
        bool flag;
        if (converged) {
          flag = dx2 >= lo2 * ref2;
        } else {
          flag = sNear[r] != 0;
          sNear[r] = dx2 < hi2 * ref2 ? 1 : 0;
        }
        if (converged || it >= p.max_iter) {
          finish = true;
          p.iters[v] = static_cast<uint32_t>(it);
          p.conv[v] = converged ? 1 : 0;
        }
        if (flag) {
          // a stopping decision within the guard band: the FP64 kernel re-runs
          // this voxel and overwrites its outputs, so it leaves the tile now.
          // Its X row is left untouched: a path fit warm-starts from X in
          // place, and the re-run must start from the same point.
          const unsigned long long k = atomicAdd(p.n_flagged, 1ull);
          p.flagged[k] = v;
          finish = true;
          write_out = false;
        }
        if (p.cap > 0 && !p.resume && !finish) {
          if (it > w0) {
            const float l2 = log2f(fmaxf(static_cast<float>(dx2 / ref2), 1e-37f));
            ksl += l2;
            kskl = fmaf(static_cast<float>(it - w0), l2, kskl);
          }
          if (it == p.cap) {
            // park: remaining iterations predicted by the least-squares line
            // through log2(rel^2) over the window, extended to log2(tol^2)
            const float n = static_cast<float>(p.cap - w0), km = 0.5f * (n + 1.f);
            const float slope = (kskl - km * ksl) / (n * (n * n - 1.f) / 12.f);
            const float lc = ksl / n + slope * (n - km);
            const float rem = slope < 0.f ? (2.f * log2f(static_cast<float>(tol)) - lc) / slope : 65536.f;
            const unsigned long long k = atomicAdd(p.n_pend, 1ull);
            p.pend[k] = v;
            p.pend_key[k] = fminf(fmaxf(rem, 1.f), 65536.f) * (1.f / 65536.f);
            p.Np[v] = static_cast<uint8_t>(sNear[r]);
            finish = true;
            park = true;
          }
        }
      }
      sFin[r] = finish ? 1 : 0;
      sPark[r] = park ? 1 : 0;
      sOld[r] = (finish && (write_out || park)) ? v : -1;
      // refill: the next prefetched voxel, else straight from the work queue
      const bool need = finish || v < 0;
      const unsigned m = __ballot_sync(0xffffffffu, need);
      if (m) {
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&s_head, __popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (need) {
          const int pos = base + __popc(m & ((1u << lane) - 1u));
          int64_t nv = -1;
          int src = -1;
          double thr = p.thr;
          if (pos < s_tail) {
            src = pos % RING;
            nv = rVid[src];
            thr = rThr[src];
          } else if (!*reinterpret_cast<volatile int*>(&s_exhausted)) {
            const unsigned long long k = atomicAdd(p.queue, 1ull);
            if (k < nwork) {
              nv = p.list ? p.list[k] : static_cast<int64_t>(k);
              if (p.alpha_v) thr = p.step * p.alpha_v[nv];
            } else {
              atomicExch(&s_exhausted, 1);
            }
          }
          sVid[r] = nv;
          sSrc[r] = src;
          sIt[r] = p.resume ? p.cap : 0;
          sNear[r] = (p.resume && nv >= 0) ? (src >= 0 ? rNear[src] : static_cast<int>(p.Np[nv])) : 0;
          sThr[r] = thr;
          ksl = kskl = 0.f;
        }
      }
    }
    __syncthreads();  // B2
    if (tid == 0 && s_head > s_tail) s_head = s_tail;  // positions past the tail went to the queue

    // ---- write out finished voxels, load new ones, partial max |d|
    {
      if (sFin[r] && sOld[r] >= 0) {
        const int64_t ov = sOld[r];
        if (sPark[r]) {
#pragma unroll
          for (int i = 0; i < CPT; ++i) {
            const int j = coef_of(part, i);
            p.Xp[ov * KC + j] = x[i];
            p.Dp[ov * KC + j] = d[i];
            p.Up[ov * KC + j] = sU[j * TILE + r];
          }
        } else {
#pragma unroll
          for (int i = 0; i < CPT; ++i) p.X[ov * KC + coef_of(part, i)] = x[i];
        }
      }
      const int64_t nv = sVid[r];
      const bool fresh = nv >= 0 && (sFin[r] || vid < 0);
      const bool reset = fresh || nv < 0;  // slots that keep their voxel keep x and d
      if (reset) {
        // new and emptied slots start from zero (bitwise, so a non-finite
        // finished voxel cannot leak into the next one)
#pragma unroll
        for (int i = 0; i < CPT; ++i) {
          x[i] = __longlong_as_double(0ll);
          d[i] = __longlong_as_double(0ll);
        }
      }
      if (fresh && p.resume) {
        // a parked voxel: its x, d and u rows as pass 1 left them
        const int src = sSrc[r];
        if (src >= 0) {
#pragma unroll
          for (int i = 0; i < CPT; ++i) {
            const int j = coef_of(part, i);
            sU[j * TILE + r] = rB[src * KC + j];
            x[i] = rW[src * KC + j];
            d[i] = rD[src * KC + j];
          }
        } else {
#pragma unroll
          for (int i = 0; i < CPT; ++i) {
            const int j = coef_of(part, i);
            sU[j * TILE + r] = p.Up[nv * KC + j];
            x[i] = p.Xp[nv * KC + j];
            d[i] = p.Dp[nv * KC + j];
          }
        }
      } else if (fresh) {
        // u = -b for the new voxel.  A warm start x_0 enters as d = x_0, so the
        // first product gives u_0 = G x_0 - b and the first update sees y_0 = x_0.
        const int src = sSrc[r];
        if (src >= 0) {
#pragma unroll
          for (int i = 0; i < CPT; ++i) {
            const int j = coef_of(part, i);
            sU[j * TILE + r] = -rB[src * KC + j];
            if (p.warm) x[i] = d[i] = rW[src * KC + j];
          }
        } else {
          // direct loads (the first fill, or an empty ring): all in flight at once
#pragma unroll
          for (int i = 0; i < CPT; ++i) d[i] = p.B[nv * KC + coef_of(part, i)];
#pragma unroll
          for (int i = 0; i < CPT; ++i) sU[coef_of(part, i) * TILE + r] = -d[i];
#pragma unroll
          for (int i = 0; i < CPT; ++i) x[i] = d[i] = p.warm ? p.warm[nv * KC + coef_of(part, i)] : 0.0;
        }
      }
      if (reset) {  // continuing voxels wrote max |d| in phase 1
        unsigned mx = 0;
#pragma unroll
        for (int i = 0; i < CPT; ++i) mx = max(mx, static_cast<unsigned>(__double2hiint(d[i])) & 0x7FFFFFFFu);
        sMax[part * TILE + r] = mx;
      }
    }
    const int any = __syncthreads_or(part == 0 && sVid[r] >= 0);  // B3
    if (!any) break;

    // ---- digits of d (per-voxel exponent) into the A operand
    {
      const unsigned mx = max(sMax[r], sMax[TILE + r]);
      int e = static_cast<int>(mx >> 20) - 1022;  // max |d| < 2^e
      e = min(max(e, -990), 990);                  // zero / tiny: digits round to 0
      e_vox = e;
      const double sc = pow2(D_BITS - e);
#pragma unroll
      for (int g16 = 0; g16 < 2; ++g16) {
        uint32_t pl[4][4];
#pragma unroll
        for (int w4 = 0; w4 < 4; ++w4) {
          const int i = 16 * g16 + 4 * w4;
          uint32_t t[4];
          planes4(digits(d[i], sc), digits(d[i + 1], sc), digits(d[i + 2], sc), digits(d[i + 3], sc), t);
#pragma unroll
          for (int q = 0; q < 4; ++q) pl[q][w4] = t[q];
        }
        const int j0 = coef_of(part, 16 * g16);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4*>(sA + a_off(r, q, j0)) = make_uint4(pl[q][0], pl[q][1], pl[q][2], pl[q][3]);
      }
      {
        uint32_t t[4];
        planes4(digits(d[32], sc), digits(d[33], sc), digits(d[34], sc), digits(d[35], sc), t);
        const int j0 = coef_of(part, 32);
#pragma unroll
        for (int q = 0; q < 4; ++q) *reinterpret_cast<uint32_t*>(sA + a_off(r, q, j0)) = t[q];
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();  // B4: digits visible to the tensor core
    fence_after();

    // ---- 36 MMAs: level l accumulates its digit pairs along one K range
    if (tid == 0) {
      const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
#pragma unroll
      for (int l = 0; l < NLEV; ++l) {
        const int s_lo = l > 4 ? l - 4 : 0, s_hi = l < 3 ? l : 3;
        const int nks = (5 * (s_hi - s_lo + 1) + 1) / 2;
        const uint32_t a0 = a_base + 5 * s_lo * 128, b0 = b_base + 5 * (4 - l + s_lo) * 128;
#pragma unroll
        for (int ks = 0; ks < nks; ++ks)
          mma(tbase + l * NB, umma_desc(a0 + ks * 256, A_SBO), umma_desc(b0 + ks * 256, B_SBO), ks ? 1u : 0u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar))
                   : "memory");
      ++n_batches;
    }
    // ---- while the products run: top the prefetch ring up (ids, thresholds,
    // b rows and warm rows by cp.async; they are waited for before B1)
    if (warp == PRODUCER_WARP && !*reinterpret_cast<volatile int*>(&s_exhausted)) {
      const int head = s_head, tail = s_tail;
      const int space = RING - (tail - head);
      if (space > 0) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(p.queue, static_cast<unsigned long long>(space));
        base = __shfl_sync(0xffffffffu, base, 0);
        const unsigned long long nw = nwork;
        const int ok = base >= nw ? 0 : static_cast<int>(min(static_cast<unsigned long long>(space), nw - base));
        if (lane < ok) {
          const int e = (tail + lane) % RING;
          const int64_t nv = p.list ? p.list[base + lane] : static_cast<int64_t>(base + lane);
          rVid[e] = nv;
          rThr[e] = p.alpha_v ? p.step * p.alpha_v[nv] : p.thr;
          if (p.resume) {
            rNear[e] = static_cast<int>(p.Np[nv]);
            for (int c = 0; c < KC / 2; ++c) {
              cp_async16(rB + e * KC + 2 * c, p.Up + nv * KC + 2 * c);
              cp_async16(rW + e * KC + 2 * c, p.Xp + nv * KC + 2 * c);
              cp_async16(rD + e * KC + 2 * c, p.Dp + nv * KC + 2 * c);
            }
          } else {
            for (int c = 0; c < KC / 2; ++c) {
              cp_async16(rB + e * KC + 2 * c, p.B + nv * KC + 2 * c);
              if (p.warm) cp_async16(rW + e * KC + 2 * c, p.warm + nv * KC + 2 * c);
            }
          }
        }
        cp_async_commit();
        __syncwarp();
        if (lane == 0) {
          s_tail = tail + ok;
          if (ok < space) s_exhausted = 1;
        }
      }
    }
    // ---- wait for the products (bounded)
    uint32_t done = 0;
    const uint64_t t_start = globaltimer_ns();
    while (!done && globaltimer_ns() - t_start < p.wait_ns) done = try_wait(&mbar, phase);
    if (!done) {
      s_abort = 1;
      atomicExch(p.error, 1);
    }
    phase ^= 1;
    fence_after();
    have_p = true;
    __syncthreads();
    if (s_abort) break;
  }
  if (warp == PRODUCER_WARP) cp_async_wait_all();
  if (s_abort && tid == 0) {
    // let any products still in flight land before the columns are freed
    uint32_t done = 0;
    const uint64_t t_start = globaltimer_ns();
    while (!done && globaltimer_ns() - t_start < kWaitNs) done = try_wait(&mbar, phase ^ 1u);
  }

  if (tid == 0 && p.batches) atomicAdd(p.batches, n_batches);
  if (p.iter_total && part == 0) {
    for (int o = 16; o > 0; o >>= 1) executed += __shfl_xor_sync(0xffffffffu, executed, o);
    if (lane == 0) atomicAdd(p.iter_total, executed);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TMEM_COLS));
}

constexpr size_t kMixedSmem = i8::kSmem;

}  // namespace csd
