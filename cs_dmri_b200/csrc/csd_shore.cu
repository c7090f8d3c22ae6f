// csd_shore.cu - host runtime and C ABI of the B200 SHORE volume fit.
//
// Replaces cs_dmri's fit_shore (src/fit.rs:687-805) and the three
// fit_volume_* drivers (src/fit.rs:74-527) at volume granularity.  The host
// side validates the specification exactly as the reference does (shell
// guard, alpha-strategy checks, radial order), then queues the device
// pipeline on one stream:
//
//   setup (cached per gradient table): design M, Gram G, Lipschitz L,
//         Tikhonov factor, packed DMMA tiles, M^T
//   compaction of the mask -> masked voxel list (x-y-z order)
//   b = M^T s for every masked voxel
//   solve: FISTA (fixed / ratio / path strategies) or Tikhonov
//   epilogue: residual, R^2, BIC, maps, scatter to (X, Y, Z, K)
//
// Every per-voxel computation runs on the GPU; the host only handles the
// gradient table (shells, TORTOISE deltas) and the one-number read-backs
// (masked voxel count, factorisation status, executed iteration total).

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <map>
#include <set>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/csd_shore.h"
#include "device_math.cuh"
#include "path_kernels.cuh"
#include "setup_kernels.cuh"
#include "solve_kernels.cuh"
#include "icls_kernels.cuh"
#include "mixed_kernels.cuh"
#include "tf32_kernels.cuh"
#include "epilogue_kernels.cuh"
#include "adjoint_kernels.cuh"
#include "odf_kernels.cuh"
#include "graddev_kernels.cuh"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTortoiseGmax = 80e-3;  // src/qspace.rs:262
constexpr double kGyro = 267.51532e6;    // src/qspace.rs:265
constexpr double kShellTolerance = 50.0; // src/fit.rs:618

struct Error {
  int code;
  std::string msg;
};

#define CSD_CUDA(call)                                                                         \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) throw Error{CSD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

#define CSD_LAUNCH()                                                                          \
  do {                                                                                         \
    cudaError_t e_ = cudaGetLastError();                                                       \
    if (e_ != cudaSuccess) throw Error{CSD_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)}; \
    ++h->launches;                                                                             \
  } while (0)

// Device buffer that grows on demand; freed when the handle that owns it is
// destroyed (csd_destroy makes the handle's device current first).
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void ensure(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (bytes <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    CSD_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

uint64_t fnv1a(uint64_t h, const void* data, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

// Gradient table on the host (src/qspace.rs:90-227, python/src/lib.rs:89-105).
struct HostGtab {
  std::vector<double> bvals, bvecs;
  double big = 0, small = 0, b0 = 50.0, tau = 0;
  int delta_source = 0;
  std::vector<double> shells;  // mean b of the non-zero shells, ascending
};

void tortoise_deltas(const std::vector<double>& bvals, double gmax, double* big, double* small) {
  double max_b = 0.0;
  for (double b : bvals) max_b = std::max(max_b, b);
  if (max_b <= 0.0) {
    const double small_ms = std::pow(1.0, 1.0 / 3.0);
    *big = 3.0 * small_ms * 1e-3;
    *small = small_ms * 1e-3;
    return;
  }
  const double temp = max_b / kGyro / kGyro / gmax / gmax / 2.0 * 1e6;
  const double small_ms = std::pow(temp, 1.0 / 3.0) * 1000.0;
  *big = small_ms * 3.0 * 1e-3;
  *small = small_ms * 1e-3;
}

// Non-zero shells: a gradient joins the first shell within the tolerance,
// whose b is the running mean; shells sorted by b (src/qspace.rs:171-197).
std::vector<double> dwi_shells(const std::vector<double>& bvals, double b0_threshold) {
  std::vector<double> b;
  std::vector<size_t> cnt;
  for (double v : bvals) {
    if (v <= b0_threshold) continue;
    size_t s = 0;
    for (; s < b.size(); ++s)
      if (std::fabs(b[s] - v) <= kShellTolerance) break;
    if (s < b.size()) {
      const double n = static_cast<double>(cnt[s]);
      b[s] = (b[s] * n + v) / (n + 1.0);
      cnt[s] += 1;
    } else {
      b.push_back(v);
      cnt.push_back(1);
    }
  }
  std::stable_sort(b.begin(), b.end());
  return b;
}

HostGtab make_gtab(const csd_gtab* g) {
  HostGtab t;
  t.bvals.assign(g->bvals, g->bvals + g->n);
  t.bvecs.assign(g->bvecs, g->bvecs + 3 * static_cast<size_t>(g->n));
  if (!std::isnan(g->big_delta) && !std::isnan(g->small_delta)) {
    t.big = g->big_delta;
    t.small = g->small_delta;
    t.delta_source = 0;
  } else {
    tortoise_deltas(t.bvals, kTortoiseGmax, &t.big, &t.small);
    t.delta_source = 1;
  }
  t.b0 = g->b0_threshold;
  t.tau = t.big - t.small / 3.0;
  t.shells = dwi_shells(t.bvals, t.b0);
  return t;
}

int n_coeffs(int radial_order) {
  int k = 0;
  for (int n = 0; n <= radial_order; ++n)
    for (int l = 0; l <= n; l += 2) k += 2 * l + 1;
  return k;
}

// Solve-kernel tile count for K coefficients (rows padded to 8).
int mt_for(int K) { return (K + 7) / 8; }

// Amplitude-constraint directions: a 642-vertex geodesic icosphere (regular
// icosahedron, three midpoint subdivisions projected to the unit sphere) and
// one direction of each antipodal pair, 321 unit vectors.  The reference uses
// DSI Studio's ODF8 hemisphere, a sphere of the same construction and size
// (src/solver/shore_icls.rs:52).
std::vector<double> hemisphere_directions() {
  const double ph = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<std::array<double, 3>> v = {{-1, ph, 0}, {1, ph, 0},   {-1, -ph, 0}, {1, -ph, 0},
                                          {0, -1, ph}, {0, 1, ph},   {0, -1, -ph}, {0, 1, -ph},
                                          {ph, 0, -1}, {ph, 0, 1},   {-ph, 0, -1}, {-ph, 0, 1}};
  for (auto& a : v) {
    const double n = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (auto& c : a) c /= n;
  }
  std::vector<std::array<int, 3>> f = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                                       {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                       {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                                       {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
  for (int level = 0; level < 3; ++level) {
    std::map<std::pair<int, int>, int> mid;
    auto midpoint = [&](int a, int b) {
      const auto key = std::make_pair(std::min(a, b), std::max(a, b));
      const auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      std::array<double, 3> c = {v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]};
      const double n = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      for (auto& e : c) e /= n;
      v.push_back(c);
      mid[key] = static_cast<int>(v.size()) - 1;
      return static_cast<int>(v.size()) - 1;
    };
    std::vector<std::array<int, 3>> nf;
    nf.reserve(f.size() * 4);
    for (const auto& t : f) {
      const int a = midpoint(t[0], t[1]), b = midpoint(t[1], t[2]), c = midpoint(t[2], t[0]);
      nf.push_back({t[0], a, c});
      nf.push_back({t[1], b, a});
      nf.push_back({t[2], c, b});
      nf.push_back({a, b, c});
    }
    f.swap(nf);
  }
  std::vector<double> out;
  const double e = 1e-12;
  for (const auto& a : v) {
    const bool keep = (a[2] > e) || (std::fabs(a[2]) <= e && a[1] > e) ||
                      (std::fabs(a[2]) <= e && std::fabs(a[1]) <= e && a[0] > 0.0);
    if (keep) out.insert(out.end(), a.begin(), a.end());
  }
  return out;
}

}  // namespace

struct csd_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  int launches = 0;
  cudaEvent_t ev[10] = {};  // 8, 9: the mixed-precision FISTA kernel
  csd_fit_timing timing{};

  // setup cache
  uint64_t setup_key = 0;
  bool setup_valid = false;
  bool chol_valid = false;
  uint64_t chol_key = 0;
  int N = 0, K = 0, Kp = 0;
  double lipschitz = 0.0, lambda_max = 0.0;
  DevBuf bvals, bvecs, M, Mt, G, A, gfrag, mfrag, mtfrag, scal, ok;
  int Np = 0;               // N padded to a multiple of 8
  bool dmma_rhs = false;    // M^T tiles fit in shared memory
  bool dmma_resid = false;  // M tiles fit in shared memory
  int smem_optin = 0;
  bool dmma_rhs_possible(int n, int k) const {
    const int kp = 8 * ((k + 7) / 8);
    const int np = 8 * ((n + 7) / 8);
    const size_t bytes = sizeof(double) * static_cast<size_t>(np) * kp + sizeof(float) * 8 * 8 * (np + 4);
    // k_rhs_dmma holds up to 9 samples per lane (N_pad <= 288)
    return (kp == 8 || kp == 32 || kp == 72) && np <= 288 && bytes <= static_cast<size_t>(smem_optin);
  }
  // Tikhonov solution operator P = H^-1 M^T in DMMA fragment order (as
  // mtfrag), so an L2 fit is the single product c = P s; built with the factor
  DevBuf pfrag, ptmp;
  bool pfrag_valid = false;
  DevBuf hinv;                // H^{-1} of the current factor (L2 adjoint)
  bool hinv_valid = false;
  uint64_t hinv_key = 0;
  DevBuf mom;      // Nesterov momentum table (t_k - 1) / t_{k+1}
  int mom_len = 0;
  // amplitude-ICLS setup: constraint C (m x K), factor of M^T M + eps I, W = L^{-1} C^T
  bool icls_valid = false;
  uint64_t icls_key = 0;
  int icls_m = 0, icls_m_pad = 0, icls_lmax = 0, icls_qmax = 0;
  DevBuf dirs, Cmat, Le, Wi, Q1, ovf;
  // Gram form of the amplitude ICLS (active sets <= 32): W^T W, G^-1 C^T,
  // G^-1, C = Y P
  DevBuf icls_gam, icls_ut, icls_ginv, icls_y, icls_pf, icls_jcol;
  bool icls_gram = false;  // the Gram-form kernel serves this table
  int icls_nsh = 0;
  int opt_icls = 0;        // 0 = Gram form where it applies, 1 = the Q1 form
  // int8 digit planes of G for the mixed-precision FISTA (radial order 6)
  DevBuf gdig, gfexp;
  int precision = CSD_PRECISION_FP64;  // precision of the current fit

  // per-fit buffers
  DevBuf data, mask, coeffs, r2, resid, iters_map, kind_map, alpha_map, bic_map, rss_map;
  DevBuf blk, total, vox, B, X, iters, conv, queue, itotal, resid_v, sst_v, nnz_v, sig;
  const float* sig_compact = nullptr;  // compact masked signals of the current fit, if any
  DevBuf amax, zero, alpha_v, Xsel, Xfb, Xl2, rss_l2, list, active, pbest, psel, pact, palpha_sel,
      pit_sel, pconv_sel, palpha_fb, pit_fb, pconv_fb, pcode;
  DevBuf flagged, mixstat;  // guard re-run list; [n_flagged, batches, error]
  DevBuf pcoef, pmat, pout, pgt, pgv, pdir, pconst;  // post-fit maps
  // pipelined host-buffer fit: rhs stream + two compute streams, chunk events
  cudaStream_t pipe[4] = {nullptr, nullptr, nullptr, nullptr};  // rhs, two solve streams, output zero-fill
  cudaEvent_t pev[20] = {};
  cudaEvent_t oev[15] = {};  // pipelined fit: chunk k's slab of the output is on the host
  DevBuf iota;
  // differentiable fit: adjoint solution w, overflow list and its count, RTOP constants
  DevBuf adjW, adjovf, adjstat, adjconst;
  DevBuf gdtab, gdq;  // per-voxel-design fit: gradient table, queue and iteration count
  int adjconst_order = -1;
  double adjconst_zeta = 0.0;
  int sm_cap = 0;  // > 0: FISTA grids use at most this many SMs
  // device-side call order (HandleOrder): recorded at the end of each call
  cudaEvent_t order_ev = nullptr;
  bool order_recorded = false;
  // two-pass FISTA schedule: parked state (Y), parked positions, their keys,
  // the second pass's order, and per call slot [count, bucket counts,
  // bucket cursors]; a call uses slot sched_slot and entries from sched_base
  // on (the pipelined fit runs chunks concurrently, one slot each)
  DevBuf schedY, schedPend, schedKey, schedOrder, schedCnt;
  DevBuf schedD, schedU, schedN;  // the mixed kernel's parked d and u rows and guard flags
  int sched_slot = 0;
  int64_t sched_base = 0;
  int sched_off = 0;  // > 0: single pass (an explicit order was given, or timing runs)
  // FISTA autotuning (per gradient table): warps per CTA of k_fista_v3 and
  // the batch times of the two candidates
  int fista_warps = 0;
  float tune_ms[2] = {0.f, 0.f};
  std::map<uint64_t, std::array<float, 3>> tune_cache;  // table key -> (warps, ms12, ms16)
  // converged-optimum modes: the support-identification iteration count the
  // autotuner chose per (table, mode), and its candidates' batch times
  std::map<uint64_t, std::array<float, 5>> kkt_tune_cache;  // -> (iterations, ms at 16, 24, 32, 48)
  // the same choice for the per-voxel-design fit, per (table, order, mode)
  std::map<uint64_t, std::array<float, 5>> gd_tune_cache;
  int kkt_iters_used = 0;
  float kkt_tune_ms[4] = {0.f, 0.f, 0.f, 0.f};
  bool kkt_tuning = false;
  DevBuf tuneB, tuneX, tuneIt, tuneConv, tuneQ;
  double mixed_ms = 0.0, mixed_ops = 0.0;
  unsigned long long mixed_rerun = 0;
  // converged-optimum modes: the TF32 B operand (per table), the iterate,
  // per-voxel KKT residuals, overflow / failure lists, counters
  // [batches, error, n_overflow, n_failed, rounds, kkt max bits, n_failed2]
  DevBuf gtf32, x32, kktv, kktovf, kktfail, kktstat;
  uint64_t gtf32_key = 0;
  bool gtf32_valid = false;
  cudaEvent_t kev[5] = {};
  // tuning options (csd_set_option); -1 / 0 = default
  int opt_shape = 0;
  int opt_schedule = -1;
  int opt_kkt_iters = 0;  // 0: the autotuner's choice per table
  int opt_kkt_rounds = 48;
  // page-locked, mapped staging volume for pageable host inputs: the masked
  // rows are gathered into it on host threads and read in place by the device
  float* stage = nullptr;
  size_t stage_bytes = 0;
  float* ostage = nullptr;  // page-locked output volume for pageable outputs of the pipelined fit
  size_t ostage_bytes = 0;
  unsigned long long opt_wait_ns = 2000000000ull;  // tensor-core completion waits
  unsigned long long kkt_batches = 0, kkt_fallback = 0, kkt_rounds = 0, kkt_uncertified = 0, kkt_iter_add = 0;
  unsigned long long kkt_overflow = 0;  // supports that outgrew the first polish pass
  double kkt_max = 0.0;
  float kkt_ms[3] = {0.f, 0.f, 0.f};  // iterate, first polish, fallback (FISTA + last polish)
  float kkt_ms_last_polish = 0.f;
};

namespace {

// Device-side call order on a handle.  Every call shares the handle's buffers
// (table set-up, scratch); the device entry points return with their work
// still queued on the caller's stream, and the other calls run on the
// handle's own stream.  So each call makes its stream wait for the event the
// previous call recorded when it ended, and records it in turn: calls on one
// handle run on the device in the order they were made, whatever streams
// they use.  Inside a stream capture the graph's order applies and the event
// is neither waited on nor recorded.  Declare it once the call's stream is
// in h->stream; it records on that stream when the call returns.
struct HandleOrder {
  csd_handle* h;
  bool active = false;
  explicit HandleOrder(csd_handle* hh) : h(hh) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cs) != cudaSuccess) {
      cudaGetLastError();
      return;  // status unknown (another stream captures in global mode): leave the order alone
    }
    active = cs == cudaStreamCaptureStatusNone;
    if (active && h->order_recorded) CSD_CUDA(cudaStreamWaitEvent(h->stream, h->order_ev, 0));
  }
  ~HandleOrder() {
    if (active && cudaEventRecord(h->order_ev, h->stream) == cudaSuccess) h->order_recorded = true;
  }
  HandleOrder(const HandleOrder&) = delete;
  HandleOrder& operator=(const HandleOrder&) = delete;
};

// A page-locked, mapped host buffer of at least `bytes`, kept across calls.
static float* ensure_pinned(float*& buf, size_t& cap, size_t bytes) {
  if (cap < bytes) {
    if (buf) CSD_CUDA(cudaFreeHost(buf));
    buf = nullptr;
    cap = 0;
    void* p = nullptr;
    CSD_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocMapped | cudaHostAllocPortable));
    buf = static_cast<float*>(p);
    cap = bytes;
  }
  return buf;
}

// fn(lo, hi) over [0, n) split into contiguous ranges on up to 32 host threads.
template <class F>
static void host_parallel(int64_t n, int64_t grain, F fn) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int64_t T = std::min<int64_t>(std::min<unsigned>(hw, 32u), std::max<int64_t>(1, n / grain));
  std::vector<std::thread> pool;
  for (int64_t t = 1; t < T; ++t) pool.emplace_back(fn, n * t / T, n * (t + 1) / T);
  fn(0, n / T);
  for (auto& th : pool) th.join();
}

void set_err(char* err, size_t len, const std::string& msg) {
  if (err && len > 0) std::snprintf(err, len, "%s", msg.c_str());
}

void autotune_fista(csd_handle* h);
void launch_tikhonov(csd_handle* h, const double* B, double* X, int64_t V);

// Build (or reuse) the per-gradient-table device setup.
void ensure_setup(csd_handle* h, const HostGtab& g, int radial_order, double zeta, bool need_chol,
                  double lambda_n, double lambda_l) {
  const int N = static_cast<int>(g.bvals.size());
  const int K = n_coeffs(radial_order);
  const int Kp = 8 * mt_for(K);
  uint64_t key = 1469598103934665603ull;
  key = fnv1a(key, g.bvals.data(), g.bvals.size() * sizeof(double));
  key = fnv1a(key, g.bvecs.data(), g.bvecs.size() * sizeof(double));
  const double sc[4] = {g.tau, g.b0, zeta, static_cast<double>(radial_order)};
  key = fnv1a(key, sc, sizeof sc);
  cudaStream_t st = h->stream;
  if (!(h->setup_valid && h->setup_key == key)) {
    h->setup_valid = false;
    h->chol_valid = false;
    h->pfrag_valid = false;
    h->icls_valid = false;
    h->N = N;
    h->K = K;
    h->Kp = Kp;
    h->bvals.ensure(sizeof(double) * N);
    h->bvecs.ensure(sizeof(double) * 3 * N);
    CSD_CUDA(cudaMemcpyAsync(h->bvals.p, g.bvals.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
    CSD_CUDA(cudaMemcpyAsync(h->bvecs.p, g.bvecs.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    h->M.ensure(sizeof(double) * N * K);
    h->Mt.ensure(sizeof(double) * static_cast<size_t>(Kp) * N);
    h->G.ensure(sizeof(double) * Kp * Kp);
    h->A.ensure(sizeof(double) * Kp * Kp);
    const int MT = Kp / 8, KT = Kp / 4;
    h->gfrag.ensure(sizeof(double) * MT * KT * 32);
    h->scal.ensure(sizeof(double) * 4);
    h->ok.ensure(sizeof(int) * 4);
    // 4 pi^2 tau in the reference's evaluation order (src/qspace.rs:384-385).
    const double qdenom = 4.0 * kPi * kPi * g.tau;
    const long long nk = static_cast<long long>(N) * K;
    csd::k_design<<<static_cast<unsigned>((nk + 255) / 256), 256, 0, st>>>(
        h->bvals.as<double>(), h->bvecs.as<double>(), N, K, radial_order, zeta, qdenom, g.b0,
        h->M.as<double>());
    CSD_LAUNCH();
    csd::k_gram<<<(Kp * Kp + 255) / 256, 256, 0, st>>>(h->M.as<double>(), N, K, Kp, radial_order,
                                                      0.0, 0.0, h->G.as<double>(), nullptr);
    CSD_LAUNCH();
    const size_t lsm = sizeof(double) * (static_cast<size_t>(Kp) * Kp + 2 * Kp);
    CSD_CUDA(cudaFuncSetAttribute(csd::k_lipschitz, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(lsm)));
    csd::k_lipschitz<<<1, 256, lsm, st>>>(h->G.as<double>(), Kp, N, 200000, h->scal.as<double>(),
                                          h->scal.as<double>() + 1);
    CSD_LAUNCH();
    csd::k_pack_gfrag<<<(MT * KT * 32 + 255) / 256, 256, 0, st>>>(h->G.as<double>(), Kp,
                                                                   h->gfrag.as<double>());
    CSD_LAUNCH();

    csd::k_transpose_design<<<(Kp * N + 255) / 256, 256, 0, st>>>(h->M.as<double>(), N, K, Kp,
                                                                  h->Mt.as<double>());
    CSD_LAUNCH();
    if (K == csd::i8::KC) {
      h->gdig.ensure(csd::i8::B_BYTES);
      h->gfexp.ensure(sizeof(int) * csd::i8::NB);
      CSD_CUDA(cudaMemsetAsync(h->gdig.p, 0, csd::i8::B_BYTES, st));
      csd::k_gdigits<<<csd::i8::NB, 128, 0, st>>>(h->G.as<double>(), Kp, h->gdig.as<uint8_t>(), h->gfexp.as<int>());
      CSD_LAUNCH();
    }
    // DMMA operand tiles of M (residual pass) and M^T (right-hand sides),
    // used when they fit in one CTA's shared memory next to the warp buffers.
    const int Np = 8 * ((N + 7) / 8);
    h->Np = Np;
    const size_t resid_smem = sizeof(double) * (static_cast<size_t>(Np) * Kp + 8 * static_cast<size_t>(Kp) * 8);
    const size_t rhs_smem = sizeof(double) * static_cast<size_t>(Np) * Kp + sizeof(float) * 8 * 8 * (Np + 4);
    const bool small_k = (Kp == 8 || Kp == 32 || Kp == 72);
    h->dmma_resid = small_k && resid_smem <= static_cast<size_t>(h->smem_optin);
    h->dmma_rhs = small_k && Np <= 288 && rhs_smem <= static_cast<size_t>(h->smem_optin);
    if (h->dmma_resid || h->dmma_rhs) {
      h->mfrag.ensure(sizeof(double) * static_cast<size_t>(Np) * Kp);
      h->mtfrag.ensure(sizeof(double) * static_cast<size_t>(Np) * Kp);
      csd::k_pack_afrag<<<(Np * Kp + 255) / 256, 256, 0, st>>>(h->M.as<double>(), N, K, K, 0, Np, Kp,
                                                              h->mfrag.as<double>());
      CSD_LAUNCH();
      csd::k_pack_afrag<<<(Np * Kp + 255) / 256, 256, 0, st>>>(h->M.as<double>(), N, K, K, 1, Kp, Np,
                                                              h->mtfrag.as<double>());
      CSD_LAUNCH();
    }
    double sc2[2];
    CSD_CUDA(cudaMemcpyAsync(sc2, h->scal.p, sizeof sc2, cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
    h->lipschitz = sc2[0];
    h->lambda_max = sc2[1];
    h->setup_key = key;
    h->setup_valid = true;
    autotune_fista(h);
  }
  if (need_chol) {
    uint64_t ck = fnv1a(key, &lambda_n, sizeof lambda_n);
    ck = fnv1a(ck, &lambda_l, sizeof lambda_l);
    if (!(h->chol_valid && h->chol_key == ck)) {
      csd::k_gram<<<(Kp * Kp + 255) / 256, 256, 0, st>>>(h->M.as<double>(), N, K, Kp, radial_order,
                                                        lambda_n, lambda_l, h->G.as<double>(),
                                                        h->A.as<double>());
      CSD_LAUNCH();
      const size_t csm = sizeof(double) * static_cast<size_t>(K) * K;
      CSD_CUDA(cudaFuncSetAttribute(csd::k_cholesky, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(csm)));
      csd::k_cholesky<<<1, 256, csm, st>>>(h->A.as<double>(), K, Kp, h->ok.as<int>());
      CSD_LAUNCH();
      int okv = 0;
      CSD_CUDA(cudaMemcpyAsync(&okv, h->ok.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      CSD_CUDA(cudaStreamSynchronize(st));
      if (!okv) throw Error{CSD_ERR_NUMERICAL, "normal-equations matrix should be PD"};
      h->chol_key = ck;
      h->chol_valid = true;
      // P^T = rows H^-1 m_n of the design rows m_n, by the factor's solves,
      // then packed like M^T for the right-hand-side kernel
      h->pfrag_valid = false;
      if (h->dmma_rhs) {
        h->ptmp.ensure(2 * sizeof(double) * static_cast<size_t>(N) * Kp);
        double* mpad = h->ptmp.as<double>();
        double* pt = mpad + static_cast<size_t>(N) * Kp;
        csd::k_pad_rows<<<(N * Kp + 255) / 256, 256, 0, st>>>(h->M.as<double>(), N, K, Kp, mpad);
        CSD_LAUNCH();
        launch_tikhonov(h, mpad, pt, N);
        h->pfrag.ensure(sizeof(double) * static_cast<size_t>(h->Np) * Kp);
        csd::k_pack_afrag<<<(h->Np * Kp + 255) / 256, 256, 0, st>>>(pt, N, K, Kp, 1, Kp, h->Np,
                                                                    h->pfrag.as<double>());
        CSD_LAUNCH();
        h->pfrag_valid = true;
      }
    }
  }
}

constexpr int kIclsGramCpl = 11;  // constraint slots per lane of k_icls_gram (321 directions, m_pad 352)

// Setup of the amplitude-positivity fit (src/solver/shore_icls.rs:41-71,
// src/solver/icls.rs:183-222): constraint matrix on the hemisphere, Cholesky
// factor of M^T M + eps I and W = L^{-1} C^T.  Cached per table and epsilon.
void ensure_icls_setup(csd_handle* h, int radial_order, double zeta, double eps) {
  cudaStream_t st = h->stream;
  uint64_t key = fnv1a(h->setup_key, &eps, sizeof eps);
  if (h->icls_valid && h->icls_key == key) return;
  const int K = h->K, Kp = h->Kp;
  const std::vector<double> dirs = hemisphere_directions();
  const int m = static_cast<int>(dirs.size() / 3);
  const int m_pad = 32 * ((m + 31) / 32);
  const int lmax = radial_order - (radial_order % 2);
  h->icls_m = m;
  h->icls_m_pad = m_pad;
  h->icls_lmax = lmax;
  h->icls_qmax = (lmax + 1) * (lmax + 2) / 2;  // rank of C <= number of SH coefficients
  h->dirs.ensure(sizeof(double) * dirs.size());
  CSD_CUDA(cudaMemcpyAsync(h->dirs.p, dirs.data(), sizeof(double) * dirs.size(), cudaMemcpyHostToDevice, st));
  h->Cmat.ensure(sizeof(double) * static_cast<size_t>(m) * K);
  csd::k_constraint<<<(m * K + 255) / 256, 256, 0, st>>>(h->dirs.as<double>(), m, K, radial_order, zeta,
                                                        h->Cmat.as<double>());
  CSD_LAUNCH();
  h->Le.ensure(sizeof(double) * Kp * Kp);
  CSD_CUDA(cudaMemcpyAsync(h->Le.p, h->G.p, sizeof(double) * Kp * Kp, cudaMemcpyDeviceToDevice, st));
  csd::k_add_diag<<<(K + 255) / 256, 256, 0, st>>>(h->Le.as<double>(), K, Kp, eps);
  CSD_LAUNCH();
  const size_t csm = sizeof(double) * static_cast<size_t>(K) * K;
  CSD_CUDA(cudaFuncSetAttribute(csd::k_cholesky, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(csm)));
  csd::k_cholesky<<<1, 256, csm, st>>>(h->Le.as<double>(), K, Kp, h->ok.as<int>());
  CSD_LAUNCH();
  int okv = 0;
  CSD_CUDA(cudaMemcpyAsync(&okv, h->ok.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CSD_CUDA(cudaStreamSynchronize(st));
  if (!okv) throw Error{CSD_ERR_NUMERICAL, "H^T H + eps I must be positive definite"};
  h->Wi.ensure(sizeof(double) * static_cast<size_t>(K) * m_pad);
  csd::k_icls_w<<<(m_pad + 127) / 128, 128, 0, st>>>(h->Le.as<double>(), K, Kp, h->Cmat.as<double>(), m, m_pad,
                                                      h->Wi.as<double>());
  CSD_LAUNCH();
  // the Gram form: active sets one entry per lane (nsh <= 32), 11 constraint
  // slots per lane (m_pad = 352), x~ in <= 3 registers per lane
  h->icls_nsh = h->icls_qmax;
  h->icls_gram = h->icls_nsh <= 32 && m_pad == 32 * kIclsGramCpl && Kp <= 96 &&
                 csd::icls_gram_smem(h->icls_nsh, m_pad) <= static_cast<size_t>(h->smem_optin);
  if (h->icls_gram) {
    const int64_t n_gam = static_cast<int64_t>(m_pad) * m_pad;
    h->icls_gam.ensure(sizeof(double) * static_cast<size_t>(n_gam));
    csd::k_icls_gram_setup<<<static_cast<unsigned>((n_gam + 255) / 256), 256, 0, st>>>(
        h->Wi.as<double>(), K, m_pad, h->icls_gam.as<double>());
    CSD_LAUNCH();
    h->icls_ut.ensure(sizeof(double) * static_cast<size_t>(m_pad) * Kp);
    h->icls_ginv.ensure(sizeof(double) * static_cast<size_t>(Kp) * Kp);
    CSD_CUDA(cudaMemsetAsync(h->icls_ginv.p, 0, sizeof(double) * static_cast<size_t>(Kp) * Kp, st));
    csd::k_icls_gram_solves<<<(m_pad + K + 127) / 128, 128, 0, st>>>(h->Le.as<double>(), K, Kp, h->Wi.as<double>(),
                                                                   m_pad, h->icls_ut.as<double>(),
                                                                   h->icls_ginv.as<double>());
    CSD_LAUNCH();
    const int ny = h->icls_nsh * m_pad;
    h->icls_y.ensure(sizeof(double) * static_cast<size_t>(ny));
    h->icls_pf.ensure(sizeof(double) * K);
    h->icls_jcol.ensure(sizeof(int) * K);
    csd::k_constraint_factors<<<(std::max(ny, K) + 255) / 256, 256, 0, st>>>(
        h->dirs.as<double>(), m, m_pad, K, radial_order, lmax, zeta, h->icls_y.as<double>(),
        h->icls_pf.as<double>(), h->icls_jcol.as<int>());
    CSD_LAUNCH();
  }
  h->icls_key = key;
  h->icls_valid = true;
}

// Masked voxel list; returns V.
int64_t compact(csd_handle* h, const uint8_t* d_flags, int64_t n, DevBuf& out) {
  cudaStream_t st = h->stream;
  const int nblk = static_cast<int>((n + csd::kCompactBlock - 1) / csd::kCompactBlock);
  h->blk.ensure(sizeof(int) * std::max(nblk, 1));
  h->total.ensure(sizeof(long long));
  out.ensure(sizeof(int64_t) * std::max<int64_t>(n, 1));
  if (nblk == 0) return 0;
  csd::k_mask_count<<<nblk, 256, 0, st>>>(d_flags, n, h->blk.as<int>());
  CSD_LAUNCH();
  csd::k_scan_blocks<<<1, 1024, 0, st>>>(h->blk.as<int>(), nblk, h->total.as<long long>());
  CSD_LAUNCH();
  csd::k_mask_compact<<<nblk, csd::kCompactBlock / 4, 0, st>>>(d_flags, n, h->blk.as<int>(),
                                                              out.as<int64_t>());
  CSD_LAUNCH();
  long long total = 0;
  CSD_CUDA(cudaMemcpyAsync(&total, h->total.p, sizeof total, cudaMemcpyDeviceToHost, st));
  CSD_CUDA(cudaStreamSynchronize(st));
  return static_cast<int64_t>(total);
}

inline unsigned grid1(int64_t n, int bs = 256) { return static_cast<unsigned>((n + bs - 1) / bs); }

// Momentum of FISTA iteration k, (t_k - 1) / t_{k+1} with t_0 = 1 and
// t_{k+1} = (1 + sqrt(1 + 4 t_k^2)) / 2 (src/solver/fista.rs:110-112).  It
// depends on k only; the table is built once per max_iter with the same IEEE
// operations the reference performs inside its loop.
void ensure_mom(csd_handle* h, int max_iter) {
  if (max_iter <= 0 || (h->mom_len >= max_iter && h->mom.p)) return;
  std::vector<double> m(static_cast<size_t>(max_iter));
  volatile double t = 1.0;
  for (int k = 0; k < max_iter; ++k) {
    const double tk = t;
    const double four_tt = 4.0 * tk * tk;
    const double root = std::sqrt(1.0 + four_tt);
    const double tn = 0.5 * (1.0 + root);
    m[k] = (tk - 1.0) / tn;
    t = tn;
  }
  h->mom.ensure(sizeof(double) * m.size());
  CSD_CUDA(cudaMemcpyAsync(h->mom.p, m.data(), sizeof(double) * m.size(), cudaMemcpyHostToDevice, h->stream));
  CSD_CUDA(cudaStreamSynchronize(h->stream));
  h->mom_len = max_iter;
}

template <int MT>
void launch_fista_t(csd_handle* h, const csd::FistaParams& p) {
  constexpr int KP = 8 * MT, KT = 2 * MT;
  const size_t smem = sizeof(double) * (static_cast<size_t>(MT) * KT * 32 + 8 * KP * 8);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_fista_fp64<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  int per_sm = 0;
  CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_fista_fp64<MT>, 256, smem));
  per_sm = std::max(per_sm, 1);
  const int64_t warps_needed = (p.n_work + 7) / 8;
  int64_t blocks = std::min<int64_t>(static_cast<int64_t>(h->num_sms) * per_sm, (warps_needed + 7) / 8);
  blocks = std::max<int64_t>(blocks, 1);
  csd::k_fista_fp64<MT><<<static_cast<unsigned>(blocks), 256, smem, h->stream>>>(p);
  CSD_LAUNCH();
}

// Two-pass schedule: a fit is split at iteration sched_cap() when it has at
// least kSchedMinWaves voxels per FISTA slot (fewer: the slowest voxels start
// in the first wave anyway) and max_iter is above twice the cap.  The slot
// count of the call's grid sets the scale.  The handle option
// CSD_OPT_FISTA_SCHEDULE turns it off (0) or sets the cap (>= 2).
constexpr int kSchedCap = 80;

int sched_cap(const csd_handle* h) {
  const int o = h->opt_schedule;
  if (o < 0 || o == 1) return kSchedCap;
  return o == 0 ? 0 : o;
}
constexpr int64_t kSchedMinWaves = 4;
constexpr size_t kSchedSlotBytes = 4096;  // count (8 B), bucket counts, bucket cursors
constexpr int kSchedSlots = 16;

// Single-pass FISTA for the lifetime of the guard.
struct SchedOff {
  csd_handle* h;
  explicit SchedOff(csd_handle* hh) : h(hh) { ++h->sched_off; }
  ~SchedOff() { --h->sched_off; }
  SchedOff(const SchedOff&) = delete;
  SchedOff& operator=(const SchedOff&) = delete;
};

bool sched_enabled(const csd_handle* h, const csd::FistaParams& p, int64_t slots) {
  const int cap = sched_cap(h);
  if (cap == 0 || h->sched_off > 0 || p.cap != 0 || p.n_work_dev || p.max_iter <= 2 * cap) return false;
  return p.n_work >= kSchedMinWaves * slots;
}

// Scratch of the two-pass schedule for fits over up to V positions.
void ensure_sched(csd_handle* h, int64_t V) {
  h->schedY.ensure(sizeof(double) * static_cast<size_t>(V) * h->Kp);
  h->schedPend.ensure(sizeof(int64_t) * static_cast<size_t>(V));
  h->schedKey.ensure(sizeof(float) * static_cast<size_t>(V));
  h->schedOrder.ensure(sizeof(int64_t) * static_cast<size_t>(V));
  h->schedCnt.ensure(kSchedSlotBytes * kSchedSlots);
}

template <int MT, int WARPS, bool G_IN_SMEM = true>
void launch_fista_v3_t(csd_handle* h, const csd::FistaParams& p) {
  constexpr int KP = 8 * MT;
  // Gram tiles (when staged) + per-warp y and b buffers
  const size_t smem = sizeof(double) * ((G_IN_SMEM ? 2 * static_cast<size_t>(MT) * MT * 32 : 0) + WARPS * 2 * KP * 8);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_fista_v3<MT, WARPS, G_IN_SMEM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  int per_sm = 0;
  CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_fista_v3<MT, WARPS, G_IN_SMEM>, 32 * WARPS, smem));
  per_sm = std::max(per_sm, 1);
  const int64_t warps_needed = (p.n_work + 7) / 8;
  const int sms = h->sm_cap > 0 ? std::min(h->sm_cap, h->num_sms) : h->num_sms;
  int64_t blocks = std::min<int64_t>(static_cast<int64_t>(sms) * per_sm, (warps_needed + WARPS - 1) / WARPS);
  blocks = std::max<int64_t>(blocks, 1);
  csd::FistaParams q = p;
  q.gfrag = h->gfrag.as<double>();
  q.mom = h->mom.as<double>();
  cudaStream_t st = h->stream;
  if (!sched_enabled(h, p, blocks * WARPS * 8)) {
    csd::k_fista_v3<MT, WARPS, G_IN_SMEM><<<static_cast<unsigned>(blocks), 32 * WARPS, smem, st>>>(q);
    CSD_LAUNCH();
    return;
  }
  // pass 1 to the cap; order the parked voxels; pass 2 resumes them
  if (h->sched_slot < 0 || h->sched_slot >= kSchedSlots || h->sched_base < 0 || h->sched_base + p.n_work > p.V)
    throw Error{CSD_ERR_INVALID, "two-pass FISTA schedule: slot or base out of range"};
  ensure_sched(h, p.V);
  char* cnt = static_cast<char*>(h->schedCnt.p) + kSchedSlotBytes * h->sched_slot;
  auto* n_pend = reinterpret_cast<unsigned long long*>(cnt);
  auto* hist = reinterpret_cast<unsigned*>(cnt + 8);
  unsigned* cursor = hist + csd::kSchedBins;
  int64_t* pend = h->schedPend.as<int64_t>() + h->sched_base;
  float* key = h->schedKey.as<float>() + h->sched_base;
  int64_t* order = h->schedOrder.as<int64_t>() + h->sched_base;
  CSD_CUDA(cudaMemsetAsync(cnt, 0, kSchedSlotBytes, st));
  csd::FistaParams q1 = q;
  q1.cap = sched_cap(h);
  q1.resume = 0;
  q1.Y = h->schedY.as<double>();
  q1.pend = pend;
  q1.pend_key = key;
  q1.n_pend = n_pend;
  csd::k_fista_v3<MT, WARPS, G_IN_SMEM><<<static_cast<unsigned>(blocks), 32 * WARPS, smem, st>>>(q1);
  CSD_LAUNCH();
  csd::k_sched_hist<<<h->num_sms, 256, 0, st>>>(key, n_pend, hist, p.iter_total ? p.iter_total + 2 : nullptr);
  CSD_LAUNCH();
  csd::k_sched_order<<<h->num_sms, csd::kSchedBins, 0, st>>>(pend, key, n_pend, hist, cursor, order);
  CSD_LAUNCH();
  CSD_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), st));
  csd::FistaParams q2 = q1;
  q2.resume = 1;
  q2.warm = nullptr;
  q2.list = order;
  q2.n_work_dev = n_pend;
  q2.pend = nullptr;
  q2.pend_key = nullptr;
  csd::k_fista_v3<MT, WARPS, G_IN_SMEM><<<static_cast<unsigned>(blocks), 32 * WARPS, smem, st>>>(q2);
  CSD_LAUNCH();
}

// FISTA kernel variant: 0 = k_fista_fp64 (registers hold x, y, b); 3 / 4 =
// k_fista_v3 with 12 / 16 warps per CTA, chosen per gradient table by
// autotune_fista.  The handle option CSD_OPT_FISTA_SHAPE overrides the choice.
int fista_variant(const csd_handle* h) {
  if (h) {
    if (h->opt_shape == 1) return 0;
    if (h->opt_shape == 12) return 3;
    if (h->opt_shape == 16) return 4;
  }
  return (h && h->fista_warps == 12) ? 3 : 4;
}

void launch_fista(csd_handle* h, int MT, const csd::FistaParams& p);

// Mixed-precision FISTA: int8 digit-slice Gram products on the tensor cores,
// FP64 state; the voxels the stop-decision guard flags are then re-fitted by
// the FP64 kernel from the same starting point.
void launch_fista_mixed(csd_handle* h, const csd::FistaParams& p) {
  using namespace csd::i8;
  cudaStream_t st = h->stream;
  h->flagged.ensure(sizeof(int64_t) * std::max<int64_t>(p.n_work, 1));
  h->mixstat.ensure(4 * sizeof(unsigned long long));
  CSD_CUDA(cudaMemsetAsync(h->mixstat.p, 0, 4 * sizeof(unsigned long long), st));
  csd::MixedParams q{};
  q.gdig = h->gdig.as<uint8_t>();
  q.fexp = h->gfexp.as<int>();
  q.B = p.B;
  q.X = p.X;
  q.warm = p.warm;
  q.iters = p.iters;
  q.conv = p.conv;
  q.c_step = p.step * p.n_inv;
  q.thr = p.thr;
  q.step = p.step;
  q.alpha_v = p.alpha_v;
  q.tol = p.tol;
  q.band = 0.01;
  q.max_iter = p.max_iter;
  q.non_negative = p.non_negative;
  q.queue = p.queue;
  q.list = p.list;
  q.n_work = p.n_work;
  q.mom = h->mom.as<double>();
  q.iter_total = p.iter_total;
  q.flagged = h->flagged.as<int64_t>();
  unsigned long long* stat = h->mixstat.as<unsigned long long>();
  q.n_flagged = stat;
  q.batches = stat + 1;
  q.error = reinterpret_cast<int*>(stat + 2);
  q.wait_ns = h->opt_wait_ns;
  const size_t smem = csd::kMixedSmem;
  CSD_CUDA(cudaFuncSetAttribute(csd::k_fista_i8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  const int64_t tiles = (p.n_work + TILE - 1) / TILE;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(h->num_sms, tiles)));
  CSD_CUDA(cudaEventRecord(h->ev[8], st));
  if (!sched_enabled(h, p, static_cast<int64_t>(grid) * TILE)) {
    csd::k_fista_i8<<<grid, THREADS, smem, st>>>(q);
    CSD_LAUNCH();
  } else {
    // two passes, as launch_fista_v3_t: every voxel to the cap, the parked
    // ones (x, d, u and the guard flag kept) resumed slowest-first
    if (h->sched_slot < 0 || h->sched_slot >= kSchedSlots || h->sched_base < 0 || h->sched_base + p.n_work > p.V)
      throw Error{CSD_ERR_INVALID, "two-pass FISTA schedule: slot or base out of range"};
    ensure_sched(h, p.V);
    h->schedD.ensure(sizeof(double) * static_cast<size_t>(p.V) * KC);
    h->schedU.ensure(sizeof(double) * static_cast<size_t>(p.V) * KC);
    h->schedN.ensure(static_cast<size_t>(p.V));
    char* cnt = static_cast<char*>(h->schedCnt.p) + kSchedSlotBytes * h->sched_slot;
    auto* n_pend = reinterpret_cast<unsigned long long*>(cnt);
    auto* hist = reinterpret_cast<unsigned*>(cnt + 8);
    unsigned* cursor = hist + csd::kSchedBins;
    int64_t* pend = h->schedPend.as<int64_t>() + h->sched_base;
    float* key = h->schedKey.as<float>() + h->sched_base;
    int64_t* order = h->schedOrder.as<int64_t>() + h->sched_base;
    CSD_CUDA(cudaMemsetAsync(cnt, 0, kSchedSlotBytes, st));
    csd::MixedParams q1 = q;
    q1.cap = sched_cap(h);
    q1.Xp = h->schedY.as<double>();
    q1.Dp = h->schedD.as<double>();
    q1.Up = h->schedU.as<double>();
    q1.Np = h->schedN.as<uint8_t>();
    q1.pend = pend;
    q1.pend_key = key;
    q1.n_pend = n_pend;
    csd::k_fista_i8<<<grid, THREADS, smem, st>>>(q1);
    CSD_LAUNCH();
    csd::k_sched_hist<<<h->num_sms, 256, 0, st>>>(key, n_pend, hist, p.iter_total ? p.iter_total + 2 : nullptr);
    CSD_LAUNCH();
    csd::k_sched_order<<<h->num_sms, csd::kSchedBins, 0, st>>>(pend, key, n_pend, hist, cursor, order);
    CSD_LAUNCH();
    CSD_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), st));
    csd::MixedParams q2 = q1;
    q2.resume = 1;
    q2.warm = nullptr;
    q2.list = order;
    q2.n_work_dev = n_pend;
    q2.pend = nullptr;
    q2.pend_key = nullptr;
    csd::k_fista_i8<<<grid, THREADS, smem, st>>>(q2);
    CSD_LAUNCH();
  }
  CSD_CUDA(cudaEventRecord(h->ev[9], st));
  unsigned long long hs[3] = {0, 0, 0};
  CSD_CUDA(cudaMemcpyAsync(hs, stat, sizeof hs, cudaMemcpyDeviceToHost, st));
  CSD_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[8], h->ev[9]) == cudaSuccess) h->mixed_ms += ms;
  h->mixed_ops += static_cast<double>(hs[1]) * MMAS_PER_ITER * 2.0 * TILE * NB * 32;
  if (static_cast<int>(hs[2]) != 0)
    throw Error{CSD_ERR_TIMEOUT, "mixed-precision FISTA: a tensor-core completion wait gave up"};
  if (hs[0] > 0) {
    h->mixed_rerun += hs[0];
    csd::FistaParams r = p;
    r.list = h->flagged.as<int64_t>();
    r.n_work = static_cast<int64_t>(hs[0]);
    r.iter_total = nullptr;  // executed iterations count the mixed pass once
    CSD_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), st));
    const int saved = h->precision;
    h->precision = CSD_PRECISION_FP64;
    launch_fista(h, KC / 8, r);
    h->precision = saved;
  }
}

// Converged-optimum L1 fit (precision MIXED_KKT / FP64_KKT, radial order
// <= 6): support identification by a fixed number of FISTA iterations (TF32
// tensor cores, or the FP64 kernel), the FP64 active-set polish with its KKT
// certificate, a second polish for supports larger than the warp slice, and
// the FP64 FISTA path with the reference stopping rule followed by a last
// polish for the voxels the first polish could not certify.
constexpr double kKktKappa = 1e-9;   // certificate: off-support |g_j| <= alpha (1 + kappa)
constexpr int kKktRoundsFallback = 64;
constexpr int kPolishCap = 32;       // support held by the first polish's warp slice

template <int K, bool NONNEG>
void launch_fista_tf32_nt(csd_handle* h, const csd::Tf32Params& q) {
  using S = csd::tf::Shape<K>;
  CSD_CUDA(cudaFuncSetAttribute(csd::k_fista_tf32<K, NONNEG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(S::SMEM)));
  const int64_t tiles = (q.n_work + csd::tf::TILE - 1) / csd::tf::TILE;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(2LL * h->num_sms, tiles)));
  csd::k_fista_tf32<K, NONNEG><<<grid, csd::tf::THREADS, S::SMEM, h->stream>>>(q);
  CSD_LAUNCH();
}

template <int K>
void launch_fista_tf32_t(csd_handle* h, const csd::Tf32Params& q) {
  if (q.non_negative)
    launch_fista_tf32_nt<K, true>(h, q);
  else
    launch_fista_tf32_nt<K, false>(h, q);
}

template <int K>
void build_gtf32_t(csd_handle* h, double scale) {
  using S = csd::tf::Shape<K>;
  h->gtf32.ensure(S::B_BYTES);
  const int n = S::NB * S::KA;
  csd::k_gtf32<K><<<(n + 255) / 256, 256, 0, h->stream>>>(h->G.as<double>(), h->Kp, scale, h->gtf32.as<float>());
  CSD_LAUNCH();
}

// `items` bounds the grid (a device-side list length may be shorter).
template <int RPL, int RPS>
void launch_polish_t(csd_handle* h, const csd::PolishParams& q, int warps, int64_t items) {
  const size_t smem = sizeof(double) * static_cast<size_t>(warps) * csd::polish_warp_doubles(q.cap, q.Kp);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_l1_polish<RPL, RPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  int per_sm = 0;
  CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_l1_polish<RPL, RPS>, 32 * warps, smem));
  const int64_t need = (std::max<int64_t>(items, 1) + warps - 1) / warps;
  const int blocks = static_cast<int>(std::max<int64_t>(
      1, std::min<int64_t>(static_cast<int64_t>(h->num_sms) * std::max(per_sm, 1), need)));
  csd::k_l1_polish<RPL, RPS><<<blocks, 32 * warps, smem, h->stream>>>(q);
  CSD_LAUNCH();
}

// Supports of up to 32 coefficients keep their vectors in one register per
// lane; the passes with room for all K coefficients take ceil(K / 32).
void launch_polish(csd_handle* h, const csd::PolishParams& q, int warps, int64_t items) {
  const int rpl = (q.K + 31) / 32;
  const bool small = q.cap <= 32;
  if (rpl == 1) {
    launch_polish_t<1, 1>(h, q, warps, items);
  } else if (rpl == 3) {
    if (small)
      launch_polish_t<3, 1>(h, q, warps, items);
    else
      launch_polish_t<3, 3>(h, q, warps, items);
  } else {
    throw Error{CSD_ERR_INVALID, "the converged-optimum polish is built for radial orders <= 6"};
  }
}

void launch_fista_kkt(csd_handle* h, int MT, const csd::FistaParams& p);

// Autotuning of the converged-optimum modes' support-identification
// iteration count, once per gradient table and mode: the whole path (its
// iterations, the polish and any fallback) fits the FISTA autotuner's
// synthetic batch (73,728 single-tensor voxels on the table's own b-values,
// alpha 0.01) with 16, 24, 32 and 48 iterations, once untimed and once timed,
// and the fastest count serves the table's fits.  Every count ends at the
// certified optimum, so the choice changes the time, not the result.
void autotune_kkt(csd_handle* h, int MT, bool non_negative) {
  static constexpr int kCand[4] = {16, 24, 32, 48};
  const uint64_t key = h->setup_key ^ (0x9E3779B97F4A7C15ull * (1 + h->precision + 4 * (non_negative ? 1 : 0)));
  const auto hit = h->kkt_tune_cache.find(key);
  if (hit != h->kkt_tune_cache.end()) {
    h->kkt_iters_used = static_cast<int>(hit->second[0]);
    for (int i = 0; i < 4; ++i) h->kkt_tune_ms[i] = hit->second[1 + i];
    return;
  }
  h->kkt_tuning = true;
  cudaStream_t st = h->stream;
  const int64_t Vt = 73728;
  const int Kp = h->Kp, N = h->N, K = h->K;
  ensure_mom(h, kCand[3]);
  h->tuneB.ensure(sizeof(double) * Vt * Kp);
  h->tuneX.ensure(std::max(sizeof(double) * Vt * Kp, sizeof(float) * Vt * N));
  h->tuneIt.ensure(sizeof(uint32_t) * Vt);
  h->tuneConv.ensure(Vt);
  h->tuneQ.ensure(sizeof(unsigned long long));
  float* S = h->tuneX.as<float>();
  csd::k_tune_signal<<<grid1(Vt * N), 256, 0, st>>>(h->bvals.as<double>(), h->bvecs.as<double>(), N, Vt, S);
  CSD_LAUNCH();
  csd::k_tune_rhs<<<grid1(Vt * Kp), 256, 0, st>>>(h->M.as<double>(), N, K, Kp, S, Vt, h->tuneB.as<double>());
  CSD_LAUNCH();
  csd::FistaParams q{};
  q.gfrag = h->gfrag.as<double>();
  q.B = h->tuneB.as<double>();
  q.X = h->tuneX.as<double>();
  q.iters = h->tuneIt.as<uint32_t>();
  q.conv = h->tuneConv.as<uint8_t>();
  q.V = Vt;
  q.n_inv = 1.0 / static_cast<double>(N);
  q.step = 1.0 / h->lipschitz;
  q.thr = q.step * 0.01;
  q.tol = 1e-6;
  q.max_iter = 1000;
  q.non_negative = non_negative ? 1 : 0;
  q.queue = h->tuneQ.as<unsigned long long>();
  q.n_work = Vt;
  ensure_mom(h, q.max_iter);
  const int saved = h->opt_kkt_iters;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CSD_CUDA(cudaEventCreate(&e0));
  CSD_CUDA(cudaEventCreate(&e1));
  float best = 0.f;
  int best_k = 32;
  for (int c = 0; c < 4; ++c) {
    h->opt_kkt_iters = kCand[c];
    float ms = 0.f;
    for (int pass = 0; pass < 2; ++pass) {
      CSD_CUDA(cudaEventRecord(e0, st));
      launch_fista_kkt(h, MT, q);
      CSD_CUDA(cudaEventRecord(e1, st));
      CSD_CUDA(cudaEventSynchronize(e1));
      if (pass == 1 && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = 0.f;
    }
    h->kkt_tune_ms[c] = ms;
    if (ms > 0.f && (best == 0.f || ms < best)) {
      best = ms;
      best_k = kCand[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->opt_kkt_iters = saved;
  h->kkt_iters_used = best_k;
  h->kkt_tuning = false;
  h->kkt_tune_cache[key] = {static_cast<float>(best_k), h->kkt_tune_ms[0], h->kkt_tune_ms[1], h->kkt_tune_ms[2],
                            h->kkt_tune_ms[3]};
}

void launch_fista_kkt(csd_handle* h, int MT, const csd::FistaParams& p) {
  cudaStream_t st = h->stream;
  const int K = h->K, Kp = h->Kp;
  const int64_t V = p.V;
  if (h->opt_kkt_iters <= 0 && !h->kkt_tuning) {
    autotune_kkt(h, MT, p.non_negative != 0);
    h->kkt_ms[0] = h->kkt_ms[1] = h->kkt_ms[2] = 0.f;  // the tuning batch's time is not this fit's
    h->kkt_iter_add = 0;
  }
  const int k1 = h->opt_kkt_iters > 0 ? h->opt_kkt_iters : h->kkt_iters_used;
  // stat: [0] tensor batches, [1] tensor error, [2] first-pass overflows,
  // [3] failures (the fallback's list), [4] rounds, [5] largest KKT residual
  // (bits), [6] uncertified, [7] unused overflow count
  h->kktstat.ensure(8 * sizeof(unsigned long long));
  auto* stat = h->kktstat.as<unsigned long long>();
  CSD_CUDA(cudaMemsetAsync(stat, 0, 8 * sizeof(unsigned long long), st));
  h->kktv.ensure(sizeof(double) * std::max<int64_t>(V, 1));
  h->kktovf.ensure(sizeof(int64_t) * std::max<int64_t>(p.n_work, 1));
  h->kktfail.ensure(sizeof(int64_t) * std::max<int64_t>(p.n_work, 1));
  for (auto& e : h->kev)
    if (!e) CSD_CUDA(cudaEventCreate(&e));
  CSD_CUDA(cudaEventRecord(h->kev[0], st));

  const bool tf32 = h->precision == CSD_PRECISION_MIXED_KKT;
  if (tf32) {
    if (!(h->gtf32_valid && h->gtf32_key == h->setup_key)) {
      const double scale = p.step * p.n_inv;  // G / (n L)
      switch (K) {
        case 8: build_gtf32_t<8>(h, scale); break;
        case 29: build_gtf32_t<29>(h, scale); break;
        case 72: build_gtf32_t<72>(h, scale); break;
        default: throw Error{CSD_ERR_INVALID, "precision 'mixed-kkt' is built for radial orders 2, 4 and 6"};
      }
      h->gtf32_key = h->setup_key;
      h->gtf32_valid = true;
    }
    h->x32.ensure(sizeof(float) * static_cast<size_t>(V) * Kp);
    csd::Tf32Params q{};
    q.gop = h->gtf32.as<float>();
    q.B = p.B;
    q.Kp = Kp;
    q.X32 = h->x32.as<float>();
    q.c_step = p.step * p.n_inv;
    q.step = p.step;
    q.thr = p.thr;
    q.alpha_v = p.alpha_v;
    q.iters = k1;
    q.mom = h->mom.as<double>();
    q.non_negative = p.non_negative;
    q.list = p.list;
    q.n_work = p.n_work;
    q.queue = p.queue;
    q.batches = stat;
    q.error = reinterpret_cast<int*>(stat + 1);
    q.wait_ns = h->opt_wait_ns;
    CSD_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), st));
    switch (K) {
      case 8: launch_fista_tf32_t<8>(h, q); break;
      case 29: launch_fista_tf32_t<29>(h, q); break;
      case 72: launch_fista_tf32_t<72>(h, q); break;
      default: break;
    }
  } else {
    // FP64 iterations of the same count: tol 0 never stops a voxel early
    csd::FistaParams f = p;
    f.max_iter = k1;
    f.tol = 0.0;
    f.warm = nullptr;
    f.iter_total = nullptr;
    CSD_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), st));
    const int saved = h->precision;
    h->precision = CSD_PRECISION_FP64;
    launch_fista(h, MT, f);
    h->precision = saved;
  }
  CSD_CUDA(cudaEventRecord(h->kev[1], st));

  csd::PolishParams pp{};
  pp.G = h->G.as<double>();
  pp.B = p.B;
  pp.S32 = tf32 ? h->x32.as<float>() : nullptr;
  pp.S64 = tf32 ? nullptr : p.X;
  pp.X = p.X;
  pp.iters = p.iters;
  pp.conv = p.conv;
  pp.kkt = h->kktv.as<double>();
  pp.K = K;
  pp.Kp = Kp;
  pp.n_samples = 1.0 / p.n_inv;
  pp.alpha = p.thr / p.step;
  pp.alpha_v = p.alpha_v;
  pp.non_negative = p.non_negative;
  pp.kappa = kKktKappa;
  pp.rounds = h->opt_kkt_rounds;
  pp.it_base = k1;
  pp.cap = std::min(kPolishCap, K);
  pp.list = p.list;
  pp.n_work = p.n_work;
  pp.overflow = h->kktovf.as<int64_t>();
  pp.n_overflow = stat + 2;
  pp.failed = h->kktfail.as<int64_t>();
  pp.n_failed = stat + 3;
  pp.round_total = stat + 4;
  pp.kkt_max_bits = stat + 5;
  pp.n_uncertified = stat + 6;  // non-finite inputs (failures go to the fallback list)
  launch_polish(h, pp, 8, p.n_work);
  csd::PolishParams po = pp;
  po.list = h->kktovf.as<int64_t>();
  po.list_len = stat + 2;
  // supports that outgrew the warp slice: again with room for all K
  po.cap = K;
  po.overflow = h->kktovf.as<int64_t>();  // unused: cap = K cannot overflow
  po.n_overflow = stat + 7;
  launch_polish(h, po, 4, p.n_work);
  CSD_CUDA(cudaEventRecord(h->kev[2], st));
  unsigned long long hs[6] = {0, 0, 0, 0, 0, 0};
  CSD_CUDA(cudaMemcpyAsync(hs, stat, sizeof hs, cudaMemcpyDeviceToHost, st));
  CSD_CUDA(cudaStreamSynchronize(st));
  if (static_cast<int>(hs[1]) != 0)
    throw Error{CSD_ERR_TIMEOUT, "TF32 FISTA: a tensor-core completion wait gave up"};
  h->kkt_batches = hs[0];
  h->kkt_fallback = hs[3];
  h->kkt_overflow = hs[2];
  if (hs[3] > 0) {
    // the FP64 FISTA path with the reference stopping rule, then a last polish
    csd::FistaParams r = p;
    r.list = h->kktfail.as<int64_t>();
    r.n_work = static_cast<int64_t>(hs[3]);
    r.warm = nullptr;
    CSD_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), st));
    const int saved = h->precision;
    h->precision = CSD_PRECISION_FP64;
    launch_fista(h, MT, r);
    h->precision = saved;
    CSD_CUDA(cudaEventRecord(h->kev[3], st));
    csd::PolishParams pf = pp;
    pf.S32 = nullptr;
    pf.S64 = p.X;
    pf.cap = K;
    pf.rounds = kKktRoundsFallback;
    pf.it_add = 1;
    pf.keep_on_fail = 1;
    pf.list = h->kktfail.as<int64_t>();
    pf.list_len = nullptr;
    pf.n_work = static_cast<int64_t>(hs[3]);
    pf.failed = nullptr;
    pf.n_failed = nullptr;
    pf.overflow = h->kktovf.as<int64_t>();
    pf.n_overflow = stat + 7;
    pf.n_uncertified = stat + 6;
    launch_polish(h, pf, 4, r.n_work);
  }
  CSD_CUDA(cudaEventRecord(h->kev[4], st));
  unsigned long long hs2[3] = {0, 0, 0};
  CSD_CUDA(cudaMemcpyAsync(hs2, stat + 4, sizeof hs2, cudaMemcpyDeviceToHost, st));
  CSD_CUDA(cudaStreamSynchronize(st));
  h->kkt_rounds = hs2[0];
  double mx = 0.0;
  std::memcpy(&mx, &hs2[1], sizeof mx);
  h->kkt_max = mx;
  h->kkt_uncertified = hs2[2];
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->kev[0], h->kev[1]) == cudaSuccess) h->kkt_ms[0] += ms;
  if (cudaEventElapsedTime(&ms, h->kev[1], h->kev[2]) == cudaSuccess) h->kkt_ms[1] += ms;
  if (hs[3] > 0 && cudaEventElapsedTime(&ms, h->kev[2], h->kev[4]) == cudaSuccess) h->kkt_ms[2] += ms;
  if (hs[3] > 0 && cudaEventElapsedTime(&ms, h->kev[3], h->kev[4]) == cudaSuccess) h->kkt_ms_last_polish = ms;
  // executed FISTA iterations: k1 per voxel in the first phase (the fallback
  // fit counted its own)
  h->kkt_iter_add += static_cast<unsigned long long>(p.n_work) * static_cast<unsigned long long>(k1);
}

void launch_fista(csd_handle* h, int MT, const csd::FistaParams& p) {
  if ((h->precision == CSD_PRECISION_MIXED_KKT || h->precision == CSD_PRECISION_FP64_KKT) && p.max_iter > 0) {
    launch_fista_kkt(h, MT, p);
    return;
  }
  if (h->precision == CSD_PRECISION_MIXED && MT * 8 == csd::i8::KC && p.max_iter > 0) {
    launch_fista_mixed(h, p);
    return;
  }
  if (p.max_iter <= 0) {
    // An empty iteration loop: the warm start (or zero) is the result, with
    // 0 iterations and not converged (fista.rs:89-143 with max_iter = 0).
    csd::k_fista_noop<<<grid1(p.n_work * (h->Kp + 1)), 256, 0, h->stream>>>(p, h->Kp);
    CSD_LAUNCH();
    return;
  }
  const int variant = fista_variant(h);
  if (variant == 3 || variant == 4) {
    switch (MT * 8 + variant) {
      case 1 * 8 + 3: launch_fista_v3_t<1, 12>(h, p); return;
      case 1 * 8 + 4: launch_fista_v3_t<1, 16>(h, p); return;
      case 4 * 8 + 3: launch_fista_v3_t<4, 12>(h, p); return;
      case 4 * 8 + 4: launch_fista_v3_t<4, 16>(h, p); return;
      case 9 * 8 + 3: launch_fista_v3_t<9, 12>(h, p); return;
      case 9 * 8 + 4: launch_fista_v3_t<9, 16>(h, p); return;
      default: break;
    }
  }
  if (MT == 19) {  // radial order 8 (K = 145): Gram tiles through the caches
    launch_fista_v3_t<19, 8, false>(h, p);
    return;
  }
  switch (MT) {
    case 1: launch_fista_t<1>(h, p); break;
    case 4: launch_fista_t<4>(h, p); break;
    case 9: launch_fista_t<9>(h, p); break;
    default:
      throw Error{CSD_ERR_INVALID, "FISTA kernels are built for radial orders 2, 4, 6 and 8 (K <= 145); got K = " +
                                       std::to_string(h->K)};
  }
}

template <int KP>
void launch_rhs_t(csd_handle* h, const float* d_data, int64_t V) {
  const size_t smem = sizeof(double) * (32 * KP + 64 * 33);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_rhs<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  csd::k_rhs<KP><<<static_cast<unsigned>((V + 63) / 64), 256, smem, h->stream>>>(
      d_data, h->vox.as<int64_t>(), V, h->N, h->M.as<double>(), h->K, h->B.as<double>());
  CSD_LAUNCH();
}

template <int KP>
void launch_rhs_dmma_t(csd_handle* h, const float* d_data, int64_t V, float* sig_out, const double* frag,
                       double* out) {
  const size_t smem = sizeof(double) * static_cast<size_t>(h->Np) * KP + sizeof(float) * 8 * 8 * (h->Np + 4);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_rhs_dmma<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  const int64_t groups = (V + 7) / 8;
  const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(h->num_sms, (groups + 7) / 8)));
  csd::k_rhs_dmma<KP><<<blocks, 256, smem, h->stream>>>(d_data, h->vox.as<int64_t>(), V, h->N, h->Np, frag, out,
                                                        sig_out);
  CSD_LAUNCH();
}

// b = M^T s for every masked voxel into h->B; or, with `frag` / `out` set (the
// packed Tikhonov operator, DMMA path only), c = P s into `out`.
void launch_rhs(csd_handle* h, const float* d_data, int64_t V, float* sig_out = nullptr,
                const double* frag = nullptr, double* out = nullptr) {
  if (h->dmma_rhs) {
    const double* f = frag ? frag : h->mtfrag.as<double>();
    double* o = out ? out : h->B.as<double>();
    switch (h->Kp) {
      case 8: launch_rhs_dmma_t<8>(h, d_data, V, sig_out, f, o); return;
      case 32: launch_rhs_dmma_t<32>(h, d_data, V, sig_out, f, o); return;
      case 72: launch_rhs_dmma_t<72>(h, d_data, V, sig_out, f, o); return;
      default: break;
    }
  }
  if (frag) throw Error{CSD_ERR_INVALID, "the Tikhonov operator product needs the DMMA right-hand-side kernel"};
  switch (h->Kp) {
    case 8: launch_rhs_t<8>(h, d_data, V); break;
    case 32: launch_rhs_t<32>(h, d_data, V); break;
    case 72: launch_rhs_t<72>(h, d_data, V); break;
    case 152: launch_rhs_t<152>(h, d_data, V); break;
    default: throw Error{CSD_ERR_INVALID, "unsupported coefficient count " + std::to_string(h->K)};
  }
}

void launch_tikhonov(csd_handle* h, const double* B, double* X, int64_t V) {
  const int K = h->K;
  const size_t smem = sizeof(double) * static_cast<size_t>(K) * (K + 1);
  const int rpl = (K + 31) / 32;
  const int blocks = std::max(1, static_cast<int>(std::min<int64_t>((V + 7) / 8, h->num_sms * 8)));
  auto go = [&](auto kern) {
    CSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kern<<<blocks, 256, smem, h->stream>>>(h->A.as<double>(), K, h->Kp, B, X, V);
    CSD_LAUNCH();
  };
  switch (rpl) {
    case 1: go(csd::k_tikhonov<1>); break;
    case 2: go(csd::k_tikhonov<2>); break;
    case 3: go(csd::k_tikhonov<3>); break;
    case 4: go(csd::k_tikhonov<4>); break;
    case 5: go(csd::k_tikhonov<5>); break;
    default: throw Error{CSD_ERR_INVALID, "Tikhonov kernel supports K <= 160"};
  }
}

void launch_epilogue_ffma(csd_handle* h, const csd::EpilogueParams& p) {
  const size_t smem = sizeof(double) * 8 * static_cast<size_t>(h->Kp) * 8;
  const int64_t groups = (p.n_work + 7) / 8;
  const int blocks = std::max(1, static_cast<int>(std::min<int64_t>((groups + 7) / 8, h->num_sms * 16)));
  CSD_CUDA(cudaFuncSetAttribute(csd::k_epilogue, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  csd::k_epilogue<<<blocks, 256, smem, h->stream>>>(p);
  CSD_LAUNCH();
}

template <int KP>
void launch_resid_dmma_t(csd_handle* h, const csd::ResidParams& r) {
  const size_t smem = sizeof(double) * (static_cast<size_t>(h->Np) * KP + 8 * static_cast<size_t>(KP) * 8);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_resid_dmma<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  const int64_t groups = (r.n_work + 7) / 8;
  const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(h->num_sms, (groups + 7) / 8)));
  csd::k_resid_dmma<KP><<<blocks, 256, smem, h->stream>>>(r);
  CSD_LAUNCH();
}

// Residual / R^2 / BIC / scatter pass.  With the M tiles in shared memory the
// residuals run on the FP64 tensor cores (k_resid_dmma) and a light per-voxel
// pass scatters the results (k_finalize); otherwise k_epilogue does both.
// The residuals ||s - M c|| feed only the R^2, residual and BIC maps and the
// explicit per-voxel output (resid_out); a scatter of coefficients alone
// (diagnostics off) skips them.
void launch_epilogue(csd_handle* h, const csd::EpilogueParams& p) {
  if (!h->dmma_resid || p.n_work == 0) {
    if (p.n_work > 0) launch_epilogue_ffma(h, p);
    return;
  }
  const bool need_resid = !p.scatter || p.resid_out || p.r2 || p.resid || p.bic_map;
  const int64_t V = p.V;
  h->resid_v.ensure(sizeof(double) * V);
  h->sst_v.ensure(sizeof(double) * V);
  csd::ResidParams r{};
  r.data = p.data;
  r.vox = p.vox;
  r.sig = h->sig_compact;
  r.list = p.list;
  r.n_work = p.n_work;
  r.N = h->N;
  r.Np = h->Np;
  r.mfrag = h->mfrag.as<double>();
  r.X = p.X;
  r.resid_out = p.resid_out ? p.resid_out : h->resid_v.as<double>();
  r.sst_out = (p.scatter && p.r2) ? h->sst_v.as<double>() : nullptr;
  if (need_resid) {
    switch (h->Kp) {
      case 8: launch_resid_dmma_t<8>(h, r); break;
      case 32: launch_resid_dmma_t<32>(h, r); break;
      case 72: launch_resid_dmma_t<72>(h, r); break;
      default: throw Error{CSD_ERR_INVALID, "unsupported coefficient count"};
    }
  }
  if (!p.scatter && !p.nnz_out) return;
  csd::FinalizeParams f{};
  f.vox = p.vox;
  f.list = p.list;
  f.n_work = p.n_work;
  f.N = p.N;
  f.K = p.K;
  f.Kp = p.Kp;
  f.X = p.X;
  f.resid = need_resid ? r.resid_out : nullptr;
  f.sst = need_resid ? r.sst_out : nullptr;
  f.iters = p.iters;
  f.zero_v = p.zero_v;
  f.alpha_v = p.alpha_v;
  f.alpha = p.alpha;
  f.kind = p.kind;
  f.scatter = p.scatter;
  f.coeffs = p.coeffs;
  f.r2 = p.r2;
  f.resid_map = p.resid;
  f.alpha_map = p.alpha_map;
  f.bic_map = p.bic_map;
  f.iter_map = p.iter_map;
  f.kind_map = p.kind_map;
  f.nnz_out = p.nnz_out;
  const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((p.n_work + 7) / 8, h->num_sms * 16)));
  csd::k_finalize<<<blocks, 256, 0, h->stream>>>(f);
  CSD_LAUNCH();
}

template <int RPL>
void launch_icls_t(csd_handle* h, csd::IclsParams p) {
  const size_t smem = sizeof(double) * csd::kIclsWarps *
                      static_cast<size_t>(csd::icls_warp_words(h->K, h->icls_qmax, h->icls_m_pad));
  CSD_CUDA(cudaFuncSetAttribute(csd::k_icls<RPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  int per_sm = 0;
  CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_icls<RPL>, 32 * csd::kIclsWarps, smem));
  per_sm = std::max(per_sm, 1);
  const int64_t warps_needed = p.V;
  int64_t blocks = std::min<int64_t>(static_cast<int64_t>(h->num_sms) * per_sm,
                                     (warps_needed + csd::kIclsWarps - 1) / csd::kIclsWarps);
  blocks = std::max<int64_t>(blocks, 1);
  h->Q1.ensure(sizeof(double) * static_cast<size_t>(blocks) * csd::kIclsWarps * h->K * h->icls_qmax);
  p.Q1 = h->Q1.as<double>();
  csd::k_icls<RPL><<<static_cast<unsigned>(blocks), 32 * csd::kIclsWarps, smem, h->stream>>>(p);
  CSD_LAUNCH();
}

template <int RPL>
void launch_icls_gram_t(csd_handle* h, const csd::IclsParams& p) {
  csd::IclsGramParams g{};
  g.B = p.B;
  g.Ginv = h->icls_ginv.as<double>();
  g.Gam = h->icls_gam.as<double>();
  g.UT = h->icls_ut.as<double>();
  g.Y = h->icls_y.as<double>();
  g.pf = h->icls_pf.as<double>();
  g.jcol = h->icls_jcol.as<int>();
  g.X = p.X;
  g.iters = p.iters;
  g.conv = p.conv;
  g.V = p.V;
  g.K = p.K;
  g.Kp = p.Kp;
  g.m = p.m;
  g.m_pad = p.m_pad;
  g.nsh = h->icls_nsh;
  g.max_iter = p.max_iter;
  g.tol = p.tol;
  g.queue = p.queue;
  g.overflow = p.overflow;
  g.iter_total = p.iter_total;
  const size_t smem = csd::icls_gram_smem(g.nsh, g.m_pad);
  auto* kern = csd::k_icls_gram<RPL, kIclsGramCpl>;
  CSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * csd::kIclsGramWarps, smem));
  if (per_sm < 1) throw Error{CSD_ERR_CUDA, "Gram-form ICLS: no CTA fits an SM"};
  const int64_t blocks = std::max<int64_t>(
      1, std::min<int64_t>(static_cast<int64_t>(h->num_sms) * per_sm,
                           (p.V + csd::kIclsGramWarps - 1) / csd::kIclsGramWarps));
  kern<<<static_cast<unsigned>(blocks), 32 * csd::kIclsGramWarps, smem, h->stream>>>(g);
  CSD_LAUNCH();
}

void launch_icls(csd_handle* h, const csd::IclsParams& p) {
  if (h->icls_gram && h->opt_icls == 0) {
    switch ((h->K + 31) / 32) {
      case 1: launch_icls_gram_t<1>(h, p); return;
      case 2: launch_icls_gram_t<2>(h, p); return;
      case 3: launch_icls_gram_t<3>(h, p); return;
      default: break;
    }
  }
  switch ((h->K + 31) / 32) {
    case 1: launch_icls_t<1>(h, p); break;
    case 2: launch_icls_t<2>(h, p); break;
    case 3: launch_icls_t<3>(h, p); break;
    case 4: launch_icls_t<4>(h, p); break;
    case 5: launch_icls_t<5>(h, p); break;
    default: throw Error{CSD_ERR_INVALID, "amplitude-ICLS kernel supports K <= 160"};
  }
}

// Device outputs of one fit (all device pointers; maps nullable).
struct DevOut {
  float* coeffs;
  float *r2, *resid, *alpha, *bic, *rss_l2;
  uint32_t* iters;
  uint8_t* kind;
};

struct FitInfo {
  int64_t V = 0;
  uint64_t total_iterations = 0;
  bool has_dist = false;
  double dist[3] = {0, 0, 0};
  double representative_alpha = 0.0;
  const double* Xfinal = nullptr;  // device V x Kp
  const uint8_t* conv_final = nullptr;
  std::string warnings;
  int lmax = 0, n_constraint_dirs = 0;
};

// Validation shared by both entry points (src/fit.rs:555-591, 691-730;
// python/src/models.rs:112-144).
double validate(const csd_shore_spec* s, const HostGtab& g, std::string& warnings) {
  if (s->radial_order <= 0 || s->radial_order % 2 != 0)
    throw Error{CSD_ERR_INVALID,
                "radial_order must be a positive even number, got " + std::to_string(s->radial_order)};
  if (s->precision < CSD_PRECISION_FP64 || s->precision > CSD_PRECISION_FP64_KKT)
    throw Error{CSD_ERR_INVALID, "unknown precision"};
  if ((s->precision == CSD_PRECISION_MIXED_KKT || s->precision == CSD_PRECISION_FP64_KKT) &&
      s->regularization == CSD_REG_L1) {
    if (s->radial_order > 6)
      throw Error{CSD_ERR_INVALID, "the converged-optimum precisions are built for radial orders 2, 4 and 6, got " +
                                       std::to_string(s->radial_order)};
    if (s->alpha_mode != CSD_ALPHA_FIXED && s->alpha_mode != CSD_ALPHA_RATIO)
      throw Error{CSD_ERR_INVALID, "the converged-optimum precisions take alpha_mode fixed or alpha-ratio"};
  }
  if (s->precision == CSD_PRECISION_MIXED && s->regularization == CSD_REG_L1 && s->radial_order != 6)
    throw Error{CSD_ERR_INVALID, "precision 'mixed' is built for radial order 6, got " +
                                     std::to_string(s->radial_order)};
  if (s->max_iter < 0) throw Error{CSD_ERR_INVALID, "max_iter must be >= 0"};
  double path_eps = s->path_eps;
  if (s->regularization == CSD_REG_L1) {
    const int mode = s->alpha_mode;
    if (mode < CSD_ALPHA_FIXED || mode > CSD_ALPHA_L2_ANCHORED)
      throw Error{CSD_ERR_INVALID, "alpha_mode must be fixed, alpha-ratio, path-bic or l2-anchored"};
    if (mode == CSD_ALPHA_RATIO && !(s->alpha_ratio > 0.0 && s->alpha_ratio < 1.0)) {
      char b[128];
      std::snprintf(b, sizeof b, "--alpha-ratio must lie in (0, 1), got %g", s->alpha_ratio);
      throw Error{CSD_ERR_INVALID, b};
    }
    if (mode == CSD_ALPHA_PATH_BIC || mode == CSD_ALPHA_L2_ANCHORED) {
      if (s->path_n_alphas < 2)
        throw Error{CSD_ERR_INVALID, "--path-n-alphas must be \xe2\x89\xa5 2, got " + std::to_string(s->path_n_alphas)};
      if (!(path_eps > 0.0)) path_eps = (mode == CSD_ALPHA_PATH_BIC) ? 1e-3 : 1e-4;
      if (!(path_eps > 0.0 && path_eps < 1.0)) {
        char b[128];
        std::snprintf(b, sizeof b, "--path-eps must lie in (0, 1), got %g", path_eps);
        throw Error{CSD_ERR_INVALID, b};
      }
      if (mode == CSD_ALPHA_L2_ANCHORED && s->slack < 0.0) {
        char b[128];
        std::snprintf(b, sizeof b, "--slack must be \xe2\x89\xa5 0, got %g", s->slack);
        throw Error{CSD_ERR_INVALID, b};
      }
    }
  } else if (s->regularization != CSD_REG_L2 && s->regularization != CSD_REG_NONNEG) {
    throw Error{CSD_ERR_INVALID, "regularization must be l1, l2 or nonneg"};
  }
  if (g.shells.empty())
    throw Error{CSD_ERR_FIT_REFUSED,
                "3D-SHORE needs diffusion-weighted data; every volume is at or below the b=0 threshold"};
  if (g.shells.size() < 2) {
    char what[96];
    std::snprintf(what, sizeof what, "a single shell (b = %.0f s/mm\xc2\xb2)", g.shells[0]);
    if (!s->allow_single_shell)
      throw Error{CSD_ERR_FIT_REFUSED,
                  std::string("3D-SHORE needs diffusion-weighted data on at least 2 b-value shells; this "
                              "series has ") +
                      what +
                      ". With a single shell the radial decay of the signal is not determined by the "
                      "data: a fit would match the measurements, but its propagator-derived scalars "
                      "(RTOP, RTAP, RTPP, MSD, QIV) and the signals it predicts at other b-values would "
                      "reflect the regularization rather than the data. To fit anyway for orientation "
                      "information only, allow single-shell data (--allow-single-shell, or "
                      "allow_single_shell=True in Python)."};
    warnings += std::string("the data have ") + what +
                ": only the orientation information of this fit is meaningful, and "
                "propagator-derived scalars are not computed\n";
  }
  const int K = n_coeffs(s->radial_order);
  const int N = static_cast<int>(g.bvals.size());
  if (N < K && s->regularization != CSD_REG_L1) {
    warnings += std::to_string(N) + " measurements for " + std::to_string(K) +
                " coefficients (radial order " + std::to_string(s->radial_order) +
                "): without L1 regularization the fit is underdetermined and its fit statistics are "
                "not meaningful; use a lower radial order or L1\n";
  }
  return path_eps;
}

void record(csd_handle* h, int i) { CSD_CUDA(cudaEventRecord(h->ev[i], h->stream)); }

// The whole-volume fit on device buffers.
// Autotuning of the FISTA kernel's warps per CTA (12 or 16), once per
// gradient table: both k_fista_v3 variants fit a fixed synthetic batch of
// 73,728 voxels (four waves of slots) - single-tensor signals on the table
// (k_tune_signal), alpha 0.01, exactly 48 iterations each (tol 0) - and the
// faster is used for the table's fits.  Both variants compute identical
// iterates, so the choice never changes a result.  Each candidate runs once
// untimed, then once timed.
void autotune_fista(csd_handle* h) {
  h->fista_warps = 16;
  h->tune_ms[0] = h->tune_ms[1] = 0.f;
  const int MT = h->Kp / 8;
  if (MT != 4 && MT != 9) return;
  const auto hit = h->tune_cache.find(h->setup_key);  // a table seen before on this handle
  if (hit != h->tune_cache.end()) {
    h->fista_warps = static_cast<int>(hit->second[0]);
    h->tune_ms[0] = hit->second[1];
    h->tune_ms[1] = hit->second[2];
    return;
  }
  SchedOff single_pass(h);  // the timed batch runs a fixed 48 iterations per voxel
  cudaStream_t st = h->stream;
  const int64_t Vt = 73728;
  const int its = 48;
  const int Kp = h->Kp, N = h->N, K = h->K;
  ensure_mom(h, its);
  h->tuneB.ensure(sizeof(double) * Vt * Kp);
  h->tuneX.ensure(std::max(sizeof(double) * Vt * Kp, sizeof(float) * Vt * N));
  h->tuneIt.ensure(sizeof(uint32_t) * Vt);
  h->tuneConv.ensure(Vt);
  h->tuneQ.ensure(sizeof(unsigned long long));
  float* S = h->tuneX.as<float>();  // the signals live in X until the right-hand sides are formed
  csd::k_tune_signal<<<grid1(Vt * N), 256, 0, st>>>(h->bvals.as<double>(), h->bvecs.as<double>(), N, Vt, S);
  CSD_LAUNCH();
  csd::k_tune_rhs<<<grid1(Vt * Kp), 256, 0, st>>>(h->M.as<double>(), N, K, Kp, S, Vt, h->tuneB.as<double>());
  CSD_LAUNCH();
  csd::FistaParams p{};
  p.B = h->tuneB.as<double>();
  p.X = h->tuneX.as<double>();
  p.iters = h->tuneIt.as<uint32_t>();
  p.conv = h->tuneConv.as<uint8_t>();
  p.V = Vt;
  p.n_inv = 1.0 / static_cast<double>(N);
  p.step = 1.0 / h->lipschitz;
  p.thr = p.step * 0.01;
  p.tol = 0.0;  // never converges: every voxel runs exactly `its` iterations
  p.max_iter = its;
  p.queue = h->tuneQ.as<unsigned long long>();
  p.n_work = Vt;
  const int saved_cap = h->sm_cap;
  h->sm_cap = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (int c = 0; c < 2; ++c) {
      CSD_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), st));
      CSD_CUDA(cudaEventRecord(h->ev[8], st));
      if (MT == 4)
        c == 0 ? launch_fista_v3_t<4, 12>(h, p) : launch_fista_v3_t<4, 16>(h, p);
      else
        c == 0 ? launch_fista_v3_t<9, 12>(h, p) : launch_fista_v3_t<9, 16>(h, p);
      CSD_CUDA(cudaEventRecord(h->ev[9], st));
      CSD_CUDA(cudaEventSynchronize(h->ev[9]));
      float ms = 0.f;
      if (pass == 1 && cudaEventElapsedTime(&ms, h->ev[8], h->ev[9]) == cudaSuccess) h->tune_ms[c] = ms;
    }
  h->sm_cap = saved_cap;
  h->fista_warps = (h->tune_ms[0] > 0.f && h->tune_ms[0] < h->tune_ms[1]) ? 12 : 16;
  h->tune_cache[h->setup_key] = {static_cast<float>(h->fista_warps), h->tune_ms[0], h->tune_ms[1]};
}

FitInfo run_fit(csd_handle* h, const float* d_data, const uint8_t* d_mask, int64_t nvol,
                const HostGtab& g, const csd_shore_spec* spec, double path_eps, const DevOut& out,
                bool data_on_host = false) {
  FitInfo info;
  h->sig_compact = nullptr;
  cudaStream_t st = h->stream;
  h->launches = 0;
  h->precision = spec->precision;
  h->mixed_ms = 0.0;
  h->mixed_ops = 0.0;
  h->mixed_rerun = 0;
  h->kkt_batches = h->kkt_fallback = h->kkt_rounds = h->kkt_uncertified = h->kkt_iter_add = 0;
  h->kkt_overflow = 0;
  h->kkt_max = 0.0;
  h->kkt_ms[0] = h->kkt_ms[1] = h->kkt_ms[2] = 0.f;
  const bool is_l1 = spec->regularization == CSD_REG_L1;
  const int mode = spec->alpha_mode;
  const bool need_chol = spec->regularization == CSD_REG_L2 || (is_l1 && mode == CSD_ALPHA_L2_ANCHORED);

  record(h, 0);
  ensure_setup(h, g, spec->radial_order, spec->zeta, need_chol, spec->lambda_n, spec->lambda_l);
  const int N = h->N, K = h->K, Kp = h->Kp;
  record(h, 1);

  // Zero the output volumes (coefficients and maps are 0 outside the mask).
  CSD_CUDA(cudaMemsetAsync(out.coeffs, 0, sizeof(float) * static_cast<size_t>(nvol) * K, st));
  if (spec->diagnostics) {
    if (out.r2) CSD_CUDA(cudaMemsetAsync(out.r2, 0, sizeof(float) * nvol, st));
    if (out.resid) CSD_CUDA(cudaMemsetAsync(out.resid, 0, sizeof(float) * nvol, st));
    if (out.iters) CSD_CUDA(cudaMemsetAsync(out.iters, 0, sizeof(uint32_t) * nvol, st));
    if (out.kind) CSD_CUDA(cudaMemsetAsync(out.kind, 0, nvol, st));
    if (out.alpha && is_l1) CSD_CUDA(cudaMemsetAsync(out.alpha, 0, sizeof(float) * nvol, st));
    if (out.bic && is_l1) CSD_CUDA(cudaMemsetAsync(out.bic, 0, sizeof(float) * nvol, st));
    if (out.rss_l2 && is_l1 && mode == CSD_ALPHA_L2_ANCHORED)
      CSD_CUDA(cudaMemsetAsync(out.rss_l2, 0, sizeof(float) * nvol, st));
  }

  const int64_t V = compact(h, d_mask, nvol, h->vox);
  info.V = V;
  if (V == 0) {
    record(h, 2);
    record(h, 3);
    record(h, 4);
    record(h, 5);
    return info;
  }
  h->B.ensure(sizeof(double) * V * Kp);
  h->X.ensure(sizeof(double) * V * Kp);
  h->iters.ensure(sizeof(uint32_t) * V);
  h->conv.ensure(V);
  h->queue.ensure(sizeof(unsigned long long));
  h->itotal.ensure(3 * sizeof(unsigned long long));
  h->resid_v.ensure(sizeof(double) * V);
  h->nnz_v.ensure(sizeof(int) * V);
  CSD_CUDA(cudaMemsetAsync(h->itotal.p, 0, 3 * sizeof(unsigned long long), st));

  // Tikhonov with the DMMA product: c = P s directly into X (no b)
  const bool l2_operator = spec->regularization == CSD_REG_L2 && h->dmma_rhs && h->pfrag_valid;
  const double* rhs_frag = l2_operator ? h->pfrag.as<double>() : nullptr;
  double* rhs_out = l2_operator ? h->X.as<double>() : nullptr;
  if (data_on_host) {
    // `d_data` aliases pinned host memory: read each masked row once over the
    // bus and keep a compact device copy for every later pass.
    h->sig.ensure(sizeof(float) * static_cast<size_t>(V) * N);
    launch_rhs(h, d_data, V, h->sig.as<float>(), rhs_frag, rhs_out);
    h->sig_compact = h->sig.as<float>();
  } else {
    launch_rhs(h, d_data, V, nullptr, rhs_frag, rhs_out);
  }
  record(h, 2);

  csd::EpilogueParams ep{};
  ep.data = d_data;
  ep.vox = h->vox.as<int64_t>();
  ep.V = V;
  ep.N = N;
  ep.K = K;
  ep.Kp = Kp;
  ep.Mt = h->Mt.as<double>();
  ep.n_work = V;

  const int MT = Kp / 8;
  csd::FistaParams fp{};
  fp.gfrag = h->gfrag.as<double>();
  fp.B = h->B.as<double>();
  fp.X = h->X.as<double>();
  fp.iters = h->iters.as<uint32_t>();
  fp.conv = h->conv.as<uint8_t>();
  fp.V = V;
  fp.n_inv = 1.0 / static_cast<double>(N);
  fp.step = 1.0 / h->lipschitz;
  fp.tol = spec->tol;
  fp.max_iter = spec->max_iter;
  fp.non_negative = spec->non_negative;
  fp.queue = h->queue.as<unsigned long long>();
  fp.iter_total = h->itotal.as<unsigned long long>();
  fp.kstep_total = h->itotal.as<unsigned long long>() + 1;
  fp.n_work = V;
  if (is_l1) ensure_mom(h, std::max(spec->max_iter, h->opt_kkt_iters));

  const double* Xfinal = h->X.as<double>();
  const uint32_t* it_final = h->iters.as<uint32_t>();
  const uint8_t* conv_final = h->conv.as<uint8_t>();
  const double* alpha_final = nullptr;
  const uint8_t* zero_final = nullptr;
  uint8_t kind = 1;
  double alpha_const = 0.0;

  if (spec->regularization == CSD_REG_NONNEG) {
    // Goldfarb-Idnani ICLS on the ODF amplitudes (src/fit.rs:783-795)
    kind = 3;
    ensure_icls_setup(h, spec->radial_order, spec->zeta, spec->nonneg_epsilon);
    h->ovf.ensure(sizeof(int));
    CSD_CUDA(cudaMemsetAsync(h->ovf.p, 0, sizeof(int), st));
    CSD_CUDA(cudaMemsetAsync(h->queue.p, 0, sizeof(unsigned long long), st));
    csd::IclsParams ip{};
    ip.B = h->B.as<double>();
    ip.L = h->Le.as<double>();
    ip.W = h->Wi.as<double>();
    ip.X = h->X.as<double>();
    ip.iters = h->iters.as<uint32_t>();
    ip.conv = h->conv.as<uint8_t>();
    ip.V = V;
    ip.K = K;
    ip.Kp = Kp;
    ip.m = h->icls_m;
    ip.m_pad = h->icls_m_pad;
    ip.qmax = h->icls_qmax;
    ip.max_iter = spec->nonneg_max_iter;
    ip.tol = spec->nonneg_tol;
    ip.queue = h->queue.as<unsigned long long>();
    ip.overflow = h->ovf.as<int>();
    ip.iter_total = h->itotal.as<unsigned long long>();
    record(h, 6);
    launch_icls(h, ip);
    record(h, 7);
    int ovf = 0;
    CSD_CUDA(cudaMemcpyAsync(&ovf, h->ovf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
    if (ovf > 0)
      info.warnings += std::to_string(ovf) +
                       " voxel(s) reached an active set larger than the constraint rank; their fits are "
                       "marked not converged\n";
    info.lmax = h->icls_lmax;
    info.n_constraint_dirs = h->icls_m;
  } else if (spec->regularization == CSD_REG_L2) {
    kind = 2;
    record(h, 6);
    if (!l2_operator) launch_tikhonov(h, h->B.as<double>(), h->X.as<double>(), V);
    record(h, 7);
    it_final = nullptr;
    CSD_CUDA(cudaMemsetAsync(h->conv.p, 1, V, st));
    info.total_iterations = static_cast<uint64_t>(V);
  } else {
    // L1 (src/fit.rs:741-774)
    kind = 1;
    if (mode == CSD_ALPHA_FIXED) {
      alpha_const = spec->alpha;
      fp.thr = fp.step * spec->alpha;
      fp.alpha_v = nullptr;
      fp.warm = nullptr;
      CSD_CUDA(cudaMemsetAsync(h->queue.p, 0, sizeof(unsigned long long), st));
      record(h, 6);
      launch_fista(h, MT, fp);
      record(h, 7);
      info.representative_alpha = spec->alpha;
    } else {
      h->amax.ensure(sizeof(double) * V);
      h->zero.ensure(V);
      h->alpha_v.ensure(sizeof(double) * V);
      csd::k_alpha_max<<<grid1(V), 256, 0, st>>>(h->B.as<double>(), V, K, Kp, N, h->amax.as<double>(),
                                                 h->zero.as<uint8_t>());
      CSD_LAUNCH();
      zero_final = h->zero.as<uint8_t>();
      if (mode == CSD_ALPHA_RATIO) {
        csd::k_alpha_ratio<<<grid1(V), 256, 0, st>>>(h->amax.as<double>(), V, spec->alpha_ratio,
                                                     h->alpha_v.as<double>());
        CSD_LAUNCH();
        fp.alpha_v = h->alpha_v.as<double>();
        fp.warm = nullptr;
        // zero voxels are fitted with alpha 0 on a zero right-hand side and
        // then overwritten with the zero result below
        CSD_CUDA(cudaMemsetAsync(h->queue.p, 0, sizeof(unsigned long long), st));
        record(h, 6);
        launch_fista(h, MT, fp);
        record(h, 7);
        csd::k_zero_voxels<<<grid1(V), 256, 0, st>>>(V, h->zero.as<uint8_t>(), h->alpha_v.as<double>(),
                                                     h->iters.as<uint32_t>(), h->conv.as<uint8_t>());
        CSD_LAUNCH();
        alpha_final = h->alpha_v.as<double>();
      } else {
        // Path strategies (src/solver/alpha.rs:249-318).
        const int P = spec->path_n_alphas;
        h->Xsel.ensure(sizeof(double) * V * Kp);
        h->Xfb.ensure(sizeof(double) * V * Kp);
        h->list.ensure(sizeof(int64_t) * V);
        h->active.ensure(V);
        h->pbest.ensure(sizeof(double) * V);
        h->psel.ensure(V);
        h->palpha_sel.ensure(sizeof(double) * V);
        h->pit_sel.ensure(sizeof(uint32_t) * V);
        h->pconv_sel.ensure(V);
        h->palpha_fb.ensure(sizeof(double) * V);
        h->pit_fb.ensure(sizeof(uint32_t) * V);
        h->pconv_fb.ensure(V);
        h->pcode.ensure(V);
        CSD_CUDA(cudaMemsetAsync(h->Xsel.p, 0, sizeof(double) * V * Kp, st));
        CSD_CUDA(cudaMemsetAsync(h->psel.p, 0, V, st));
        CSD_CUDA(cudaMemsetAsync(h->palpha_sel.p, 0, sizeof(double) * V, st));
        CSD_CUDA(cudaMemsetAsync(h->pit_sel.p, 0, sizeof(uint32_t) * V, st));
        CSD_CUDA(cudaMemsetAsync(h->pconv_sel.p, 1, V, st));
        {
          // best metric starts at +inf
          csd::k_fill_f64<<<grid1(V), 256, 0, st>>>(h->pbest.as<double>(), V, INFINITY);
          CSD_LAUNCH();
        }
        csd::PathState ps{};
        ps.best = h->pbest.as<double>();
        ps.selected = h->psel.as<uint8_t>();
        ps.active = h->active.as<uint8_t>();
        ps.alpha_sel = h->palpha_sel.as<double>();
        ps.it_sel = h->pit_sel.as<uint32_t>();
        ps.conv_sel = h->pconv_sel.as<uint8_t>();
        ps.alpha_fb = h->palpha_fb.as<double>();
        ps.it_fb = h->pit_fb.as<uint32_t>();
        ps.conv_fb = h->pconv_fb.as<uint8_t>();
        ps.copy_code = h->pcode.as<int8_t>();
        csd::k_init_active<<<grid1(V), 256, 0, st>>>(V, h->zero.as<uint8_t>(), h->active.as<uint8_t>());
        CSD_LAUNCH();
        const double* rss_l2 = nullptr;
        if (mode == CSD_ALPHA_L2_ANCHORED) {
          // Tikhonov reference RSS per voxel (src/fit.rs:436-438).
          h->Xl2.ensure(sizeof(double) * V * Kp);
          h->rss_l2.ensure(sizeof(double) * V);
          launch_tikhonov(h, h->B.as<double>(), h->Xl2.as<double>(), V);
          csd::EpilogueParams rp = ep;
          rp.X = h->Xl2.as<double>();
          rp.scatter = false;
          rp.resid_out = h->resid_v.as<double>();
          launch_epilogue(h, rp);
          csd::k_square<<<grid1(V), 256, 0, st>>>(h->resid_v.as<double>(), h->rss_l2.as<double>(), V);
          CSD_LAUNCH();
          rss_l2 = h->rss_l2.as<double>();
        }
        record(h, 6);
        int64_t n_work = 0;
        for (int i = 0; i < P; ++i) {
          n_work = compact(h, h->active.as<uint8_t>(), V, h->list);
          if (n_work == 0) break;
          csd::k_path_alpha<<<grid1(n_work), 256, 0, st>>>(h->amax.as<double>(), h->list.as<int64_t>(),
                                                           n_work, i, P, path_eps, h->alpha_v.as<double>());
          CSD_LAUNCH();
          fp.alpha_v = h->alpha_v.as<double>();
          fp.warm = (i == 0) ? nullptr : h->X.as<double>();
          fp.list = h->list.as<int64_t>();
          fp.n_work = n_work;
          CSD_CUDA(cudaMemsetAsync(h->queue.p, 0, sizeof(unsigned long long), st));
          launch_fista(h, MT, fp);
          csd::EpilogueParams rp = ep;
          rp.X = h->X.as<double>();
          rp.scatter = false;
          rp.resid_out = h->resid_v.as<double>();
          rp.nnz_out = h->nnz_v.as<int>();
          rp.list = h->list.as<int64_t>();
          rp.n_work = n_work;
          launch_epilogue(h, rp);
          csd::k_path_update<<<grid1(n_work), 256, 0, st>>>(
              mode, h->list.as<int64_t>(), n_work, N, h->resid_v.as<double>(), h->nnz_v.as<int>(),
              h->alpha_v.as<double>(), h->iters.as<uint32_t>(), h->conv.as<uint8_t>(), rss_l2,
              spec->slack, ps);
          CSD_LAUNCH();
          csd::k_path_copy<<<grid1(n_work * Kp), 256, 0, st>>>(h->list.as<int64_t>(), n_work, Kp,
                                                               h->pcode.as<int8_t>(), h->X.as<double>(),
                                                               h->Xsel.as<double>(), h->Xfb.as<double>());
          CSD_LAUNCH();
        }
        if (mode == CSD_ALPHA_L2_ANCHORED) {
          csd::k_path_finalize<<<grid1(V * Kp), 256, 0, st>>>(V, Kp, h->zero.as<uint8_t>(), ps,
                                                               h->Xfb.as<double>(), h->Xsel.as<double>());
          CSD_LAUNCH();
        }
        record(h, 7);
        Xfinal = h->Xsel.as<double>();
        it_final = h->pit_sel.as<uint32_t>();
        conv_final = h->pconv_sel.as<uint8_t>();
        alpha_final = h->palpha_sel.as<double>();
        csd::k_zero_voxels<<<grid1(V), 256, 0, st>>>(V, h->zero.as<uint8_t>(), h->palpha_sel.as<double>(),
                                                     h->pit_sel.as<uint32_t>(), h->pconv_sel.as<uint8_t>());
        CSD_LAUNCH();
      }
    }
  }

  // Epilogue: residuals, maps, scatter.
  csd::EpilogueParams fpo = ep;
  fpo.X = Xfinal;
  fpo.iters = it_final;
  fpo.coeffs = out.coeffs;
  fpo.scatter = true;
  fpo.kind = kind;
  fpo.alpha = alpha_const;
  fpo.alpha_v = alpha_final;
  fpo.zero_v = zero_final;
  if (spec->diagnostics) {
    fpo.r2 = out.r2;
    fpo.resid = out.resid;
    fpo.iter_map = out.iters;
    fpo.kind_map = out.kind;
    if (is_l1) {
      fpo.alpha_map = out.alpha;
      fpo.bic_map = out.bic;
    }
  }
  if (is_l1 && mode == CSD_ALPHA_L2_ANCHORED && spec->diagnostics && out.rss_l2) {
    csd::k_scatter_f64_to_f32<<<grid1(V), 256, 0, st>>>(h->rss_l2.as<double>(), h->vox.as<int64_t>(), V,
                                                        out.rss_l2);
    CSD_LAUNCH();
  }
  launch_epilogue(h, fpo);
  record(h, 3);

  // executed iteration total and the alpha distribution
  unsigned long long itot[3] = {0, 0, 0};
  if (spec->regularization != CSD_REG_L2) {
    CSD_CUDA(cudaMemcpyAsync(itot, h->itotal.p, sizeof itot, cudaMemcpyDeviceToHost, st));
  }
  CSD_CUDA(cudaStreamSynchronize(st));
  if (spec->regularization != CSD_REG_L2) info.total_iterations = itot[0] + h->kkt_iter_add;
  // executed FP64 tensor work of the FISTA launches: k-steps x row tiles x
  // one m8n8k4 DMMA (8 x 8 x 4 FMA)
  h->timing.tensor_flops = static_cast<double>(itot[1]) * (Kp / 8) * 512.0;
  h->timing.fista_parked = static_cast<int64_t>(itot[2]);
  h->timing.ms_mixed_kernel = static_cast<float>(h->mixed_ms);
  h->timing.int8_tensor_ops = h->mixed_ops;
  h->timing.fp64_rerun_voxels = h->mixed_rerun;
  h->timing.ms_kkt_iterate = h->kkt_ms[0];
  h->timing.ms_kkt_polish = h->kkt_ms[1];
  h->timing.ms_kkt_fallback = h->kkt_ms[2];
  h->timing.kkt_fallback_voxels = static_cast<int64_t>(h->kkt_fallback);
  h->timing.kkt_uncertified = static_cast<int64_t>(h->kkt_uncertified);
  h->timing.kkt_rounds = h->kkt_rounds;
  h->timing.kkt_max = h->kkt_max;
  h->timing.kkt_iterations = (h->precision == CSD_PRECISION_MIXED_KKT || h->precision == CSD_PRECISION_FP64_KKT)
                                 ? (h->opt_kkt_iters > 0 ? h->opt_kkt_iters : h->kkt_iters_used)
                                 : 0;
  for (int i = 0; i < 4; ++i) h->timing.kkt_tune_ms[i] = h->kkt_tune_ms[i];
  h->timing.kkt_overflow = static_cast<int64_t>(h->kkt_overflow);
  if (h->precision == CSD_PRECISION_MIXED_KKT && K <= 80) {
    const int ks = (K + 7) / 8, nb = 16 * ((K + 15) / 16);
    h->timing.tf32_tensor_flops = static_cast<double>(h->kkt_batches) * ks * 2.0 * 128 * nb * 8;
  } else {
    h->timing.tf32_tensor_flops = 0.0;
  }
  if (is_l1 && mode != CSD_ALPHA_FIXED) {
    // median / p10 / p90 by nearest rank (src/fit.rs:334-352)
    std::vector<double> a(V);
    CSD_CUDA(cudaMemcpy(a.data(), alpha_final, sizeof(double) * V, cudaMemcpyDeviceToHost));
    std::sort(a.begin(), a.end());
    auto pct = [&](double q) {
      size_t i = static_cast<size_t>(std::round(static_cast<double>(a.size() - 1) * q));
      return a[std::min(i, a.size() - 1)];
    };
    info.has_dist = true;
    info.dist[0] = pct(0.5);
    info.dist[1] = pct(0.10);
    info.dist[2] = pct(0.90);
    info.representative_alpha = info.dist[0];
  }
  info.Xfinal = Xfinal;
  info.conv_final = conv_final;
  float ms = 0;
  h->timing.ms_setup = (cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]) == cudaSuccess) ? ms : 0.f;
  h->timing.ms_rhs = (cudaEventElapsedTime(&ms, h->ev[1], h->ev[2]) == cudaSuccess) ? ms : 0.f;
  h->timing.ms_solve = (cudaEventElapsedTime(&ms, h->ev[2], h->ev[7]) == cudaSuccess) ? ms : 0.f;
  h->timing.ms_solve_kernel = (cudaEventElapsedTime(&ms, h->ev[6], h->ev[7]) == cudaSuccess) ? ms : 0.f;
  h->timing.ms_epilogue = (cudaEventElapsedTime(&ms, h->ev[7], h->ev[3]) == cudaSuccess) ? ms : 0.f;
  h->timing.ms_total = (cudaEventElapsedTime(&ms, h->ev[0], h->ev[3]) == cudaSuccess) ? ms : 0.f;
  h->timing.launches = h->launches;
  return info;
}

// Fixed-alpha L1 fit of a page-locked host volume with the transfers
// overlapped.  The masked voxels are cut into chunks (kPipePlan: fractions of
// the voxels).  Streams ordered by events only (no kernel waits on
// another):
//   rhs:     right-hand side of chunk 0 on every SM (it reads its rows over
//            the bus, in place), then of the later chunks, one after another,
//            on kPipeRhsCtas SMs while the earlier chunks iterate on the rest;
//   solve:   chunks alternate between two streams, each running its FISTA
//            and scatter, then the copy of the slab of the coefficient
//            volume it covers back to the host.  Chunk k starts once its
//            right-hand side is done, so its CTAs take the SMs that chunk
//            k-1's tail frees; it leaves kPipeRhsCtas SMs free while a later
//            right-hand side may still be running.
//   output:  with a page-locked, mapped output volume the last chunk's
//            slab is written in place instead of copied back after it: a
//            fourth stream zero-fills that slab from the zeroed device volume
//            once the last right-hand side has read its rows (so the fill
//            does not compete with those reads on the bus), and the last
//            chunk's scatter, ordered after the fill, writes its voxels' rows
//            over the bus.  The drain is then the scatter alone.
// A small first chunk shortens the fill (the first right-hand side runs
// alone).
// Results are those of run_fit (same kernels, same per-voxel arithmetic).
constexpr int kPipeRhsCtas = 8;
constexpr double kPipePlan[] = {0.15, 0.425, 0.425};
constexpr int kPipeChunks = sizeof(kPipePlan) / sizeof(kPipePlan[0]);
constexpr int kPipeMaxChunks = 15;  // events pev[0..14]; two-pass schedule slots 1..15
static_assert(kPipeChunks <= kPipeMaxChunks, "pipeline events");

// The chunk plan (fractions of the masked voxels) and the right-hand-side SM
// count.
struct PipePlan {
  std::vector<double> frac;
  int rhs_ctas;
};

PipePlan pipe_plan(int num_sms) {
  return PipePlan{std::vector<double>(kPipePlan, kPipePlan + kPipeChunks), std::min(kPipeRhsCtas, num_sms - 1)};
}

// A pageable host volume whose masked rows the pipelined fit gathers into
// the page-locked staging volume chunk by chunk, each chunk just before its
// right-hand side is queued, so that the gather of chunk k + 1 on the host
// overlaps the device's work on chunk k.
struct HostGather {
  const float* data = nullptr;   // pageable (X, Y, Z, N) volume
  const uint8_t* mask = nullptr; // host mask
  float* stage = nullptr;        // page-locked staging: the volume's shape, or its masked rows in order
  int N = 0;
  bool compact = false;          // stage holds the masked rows only (row j = j-th masked voxel)
};

// The masked voxels of the volume range [lo, hi) in order, the j-th paired
// with compact row c_lo + j, on host threads: each thread counts its range's
// masked voxels first, so that it knows its first row.  on_row(v, row) for
// every masked voxel, on_gap(v0, v1) for every run of unmasked ones.
template <class Row, class Gap>
static void masked_rows(const uint8_t* mask, int64_t lo, int64_t hi, int64_t c_lo, Row on_row, Gap on_gap) {
  const int64_t n = hi - lo;
  if (n <= 0) return;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int64_t T = std::min<int64_t>(std::min<unsigned>(hw, 32u), std::max<int64_t>(1, n / 4096));
  std::vector<int64_t> first(static_cast<size_t>(T) + 1, 0);
  auto each = [&](auto fn) {
    std::vector<std::thread> pool;
    for (int64_t t = 1; t < T; ++t) pool.emplace_back(fn, t, lo + n * t / T, lo + n * (t + 1) / T);
    fn(int64_t{0}, lo, lo + n / T);
    for (auto& th : pool) th.join();
  };
  each([&](int64_t t, int64_t a, int64_t b) {
    int64_t c = 0;
    for (int64_t v = a; v < b; ++v) c += mask[v] != 0;
    first[static_cast<size_t>(t) + 1] = c;
  });
  for (int64_t t = 0; t < T; ++t) first[static_cast<size_t>(t) + 1] += first[static_cast<size_t>(t)];
  each([&](int64_t t, int64_t a, int64_t b) {
    int64_t row = c_lo + first[static_cast<size_t>(t)];
    int64_t v = a;
    while (v < b) {
      if (mask[v]) {
        on_row(v, row++);
        ++v;
      } else {
        int64_t e = v + 1;
        while (e < b && !mask[e]) ++e;
        on_gap(v, e);
        v = e;
      }
    }
  });
}

// The masked rows of volume range [lo, hi) into the staging buffer; in the
// compact layout the first of them goes to row c_lo.
void gather_rows(const HostGather& hg, int64_t lo, int64_t hi, int64_t c_lo = 0) {
  const int N = hg.N;
  const size_t row = sizeof(float) * static_cast<size_t>(N);
  if (hg.compact) {
    masked_rows(hg.mask, lo, hi, c_lo,
                [&](int64_t v, int64_t r) { std::memcpy(hg.stage + r * N, hg.data + v * N, row); },
                [](int64_t, int64_t) {});
    return;
  }
  host_parallel(hi - lo, 4096, [&](int64_t a, int64_t b) {
    for (int64_t v = lo + a; v < lo + b; ++v)
      if (hg.mask[v]) std::memcpy(hg.stage + v * N, hg.data + v * N, row);
  });
}

FitInfo run_fit_pipelined(csd_handle* h, const float* d_data, const uint8_t* d_mask, int64_t nvol,
                          const HostGtab& g, const csd_shore_spec* spec, float* d_coeffs, float* host_coeffs,
                          const HostGather* hg = nullptr, float* user_out = nullptr,
                          const uint8_t* host_mask = nullptr) {
  FitInfo info;
  h->sig_compact = nullptr;
  cudaStream_t st = h->stream;
  h->launches = 0;
  h->precision = spec->precision;
  h->mixed_ms = 0.0;
  h->mixed_ops = 0.0;
  h->mixed_rerun = 0;
  h->kkt_batches = h->kkt_fallback = h->kkt_rounds = h->kkt_uncertified = h->kkt_iter_add = 0;
  h->kkt_overflow = 0;
  h->kkt_max = 0.0;
  h->kkt_ms[0] = h->kkt_ms[1] = h->kkt_ms[2] = 0.f;
  record(h, 0);
  ensure_setup(h, g, spec->radial_order, spec->zeta, false, 0.0, 0.0);
  const int N = h->N, K = h->K, Kp = h->Kp;
  record(h, 1);
  CSD_CUDA(cudaMemsetAsync(d_coeffs, 0, sizeof(float) * static_cast<size_t>(nvol) * K, st));
  const int64_t V = compact(h, d_mask, nvol, h->vox);
  info.V = V;
  if (V == 0) {
    for (int i : {2, 6, 7, 3}) record(h, i);
    if (!user_out)
      CSD_CUDA(cudaMemcpyAsync(host_coeffs, d_coeffs, sizeof(float) * static_cast<size_t>(nvol) * K,
                               cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
    if (user_out) std::memset(user_out, 0, sizeof(float) * static_cast<size_t>(nvol) * K);
    return info;
  }
  const PipePlan plan = pipe_plan(h->num_sms);
  const int C = V >= 65536 ? static_cast<int>(plan.frac.size()) : 1;
  h->B.ensure(sizeof(double) * V * Kp);
  h->X.ensure(sizeof(double) * V * Kp);
  h->iters.ensure(sizeof(uint32_t) * V);
  h->conv.ensure(V);
  h->queue.ensure(sizeof(unsigned long long) * C);
  h->itotal.ensure(3 * sizeof(unsigned long long));
  h->resid_v.ensure(sizeof(double) * V);
  h->sst_v.ensure(sizeof(double) * V);
  h->nnz_v.ensure(sizeof(int) * V);
  h->sig.ensure(sizeof(float) * static_cast<size_t>(V) * N);
  h->iota.ensure(sizeof(int64_t) * V);
  h->sig_compact = h->sig.as<float>();
  CSD_CUDA(cudaMemsetAsync(h->itotal.p, 0, 3 * sizeof(unsigned long long), st));
  CSD_CUDA(cudaMemsetAsync(h->queue.p, 0, sizeof(unsigned long long) * C, st));
  csd::k_iota<<<grid1(V), 256, 0, st>>>(h->iota.as<int64_t>(), V);
  CSD_LAUNCH();
  ensure_mom(h, spec->max_iter);
  // chunk boundaries in voxel positions and their volume indices (for the
  // slab copies back)
  std::vector<int64_t> c0(C + 1), vb(C + 1, nvol);
  c0[0] = 0;
  c0[C] = V;
  double acc = 0.0;
  for (int k = 1; k < C; ++k) {
    acc += plan.frac[static_cast<size_t>(k - 1)];
    c0[k] = std::min<int64_t>(V, static_cast<int64_t>(acc * static_cast<double>(V)) & ~int64_t(7));
  }
  for (int k = 1; k < C; ++k)
    CSD_CUDA(cudaMemcpyAsync(&vb[k], h->vox.as<int64_t>() + c0[k], sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  vb[0] = 0;
  for (auto& p : h->pipe)
    if (!p) CSD_CUDA(cudaStreamCreateWithFlags(&p, cudaStreamNonBlocking));
  for (auto& e : h->pev)
    if (!e) CSD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto& e : h->oev)
    if (!e) CSD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CSD_CUDA(cudaStreamSynchronize(st));  // boundaries on the host; set-up done
  record(h, 2);
  record(h, 6);
  float* d_out_host = nullptr;  // device view of a page-locked, mapped output volume
  {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, host_coeffs) == cudaSuccess && attr.type == cudaMemoryTypeHost &&
        attr.devicePointer)
      d_out_host = static_cast<float*>(attr.devicePointer);
    cudaGetLastError();  // a pageable pointer may leave an error code behind
  }
  if (C < 2) d_out_host = nullptr;  // one chunk: a single copy back
  // Compact host buffers (a staged pageable volume or output): the staging
  // holds the masked rows in order, so the right-hand side reads row i of
  // it for voxel position i, and the coefficients come back as rows in
  // position order (V x K), which the host copies into the caller's volume.
  const bool cin = hg && hg->compact, cout = user_out != nullptr;
  const int64_t* rows_in = cin ? h->iota.as<int64_t>() : h->vox.as<int64_t>();

  const size_t rhs_smem = sizeof(double) * static_cast<size_t>(h->Np) * Kp + sizeof(float) * 8 * 8 * (h->Np + 4);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_rhs_dmma<72>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(rhs_smem)));
  csd::FistaParams fp{};
  fp.B = h->B.as<double>();
  fp.X = h->X.as<double>();
  fp.iters = h->iters.as<uint32_t>();
  fp.conv = h->conv.as<uint8_t>();
  fp.V = V;
  fp.n_inv = 1.0 / static_cast<double>(N);
  fp.step = 1.0 / h->lipschitz;
  fp.thr = fp.step * spec->alpha;
  fp.tol = spec->tol;
  fp.max_iter = spec->max_iter;
  fp.non_negative = spec->non_negative;
  fp.iter_total = h->itotal.as<unsigned long long>();
  fp.kstep_total = h->itotal.as<unsigned long long>() + 1;
  csd::EpilogueParams ep{};
  ep.data = d_data;
  ep.vox = h->vox.as<int64_t>();
  ep.V = V;
  ep.N = N;
  ep.K = K;
  ep.Kp = Kp;
  ep.Mt = h->Mt.as<double>();
  ep.X = h->X.as<double>();
  ep.iters = h->iters.as<uint32_t>();
  ep.coeffs = d_coeffs;
  ep.scatter = true;
  ep.kind = 1;
  ep.alpha = spec->alpha;

  struct Restore {
    csd_handle* h;
    cudaStream_t st;
    ~Restore() {
      h->stream = st;
      h->sm_cap = 0;
      h->sched_slot = 0;
      h->sched_base = 0;
    }
  } restore{h, st};
  ensure_sched(h, V);  // before any chunk runs: chunks share the buffers
  cudaStream_t rs = h->pipe[0];
  auto queue_rhs = [&](int k) {
    const int64_t a = c0[k], n = c0[k + 1] - c0[k];
    const int64_t groups = (n + 7) / 8;
    const int rhs_grid = static_cast<int>(std::min<int64_t>(k == 0 ? h->num_sms : plan.rhs_ctas, (groups + 7) / 8));
    csd::k_rhs_dmma<72><<<std::max(rhs_grid, 1), 256, rhs_smem, rs>>>(
        d_data, rows_in + a, n, N, h->Np, h->mtfrag.as<double>(), h->B.as<double>() + a * Kp,
        h->sig.as<float>() + a * N);
    CSD_LAUNCH();
    CSD_CUDA(cudaEventRecord(h->pev[k], rs));
    if (k == C - 1 && d_out_host && !cout) {
      // zero-fill the last chunk's slab in the host volume once every row has been read
      const int64_t lo = vb[C - 1];
      CSD_CUDA(cudaStreamWaitEvent(h->pipe[3], h->pev[C - 1], 0));
      CSD_CUDA(cudaMemcpyAsync(host_coeffs + lo * K, d_coeffs + lo * K,
                               sizeof(float) * static_cast<size_t>(nvol - lo) * K, cudaMemcpyDeviceToHost,
                               h->pipe[3]));
      CSD_CUDA(cudaEventRecord(h->pev[18], h->pipe[3]));
    }
  };
  // Without a host gather every right-hand side is queued first; with one,
  // chunk k's rows are gathered and its right-hand side queued just before
  // its iterations, so the next chunk's gather overlaps them.
  if (!hg)
    for (int k = 0; k < C; ++k) queue_rhs(k);
  for (int k = 0; k < C; ++k) {
    if (hg) {
      const auto t0 = std::chrono::steady_clock::now();
      gather_rows(*hg, vb[k], vb[k + 1], c0[k]);
      h->timing.ms_host_gather +=
          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
      queue_rhs(k);
    }
    const int64_t a = c0[k], n = c0[k + 1] - c0[k];
    cudaStream_t ks = h->pipe[1 + (k & 1)];
    CSD_CUDA(cudaStreamWaitEvent(ks, h->pev[k], 0));
    h->stream = ks;
    h->sm_cap = (k + 1 < C) ? h->num_sms - plan.rhs_ctas : 0;
    h->sched_slot = 1 + k;
    h->sched_base = a;
    csd::FistaParams f = fp;
    f.list = h->iota.as<int64_t>() + a;
    f.n_work = n;
    f.queue = h->queue.as<unsigned long long>() + k;
    launch_fista(h, Kp / 8, f);
    h->sm_cap = 0;
    h->sched_slot = 0;
    h->sched_base = 0;
    csd::EpilogueParams e = ep;
    e.list = h->iota.as<int64_t>() + a;
    e.n_work = n;
    if (cout) e.vox = h->iota.as<int64_t>();  // rows in position order
    const bool direct = d_out_host && k == C - 1;
    if (direct) {
      e.coeffs = d_out_host;
      if (!cout) CSD_CUDA(cudaStreamWaitEvent(ks, h->pev[18], 0));  // after the slab's zero-fill
    }
    launch_epilogue(h, e);
    h->stream = st;
    if (!direct) {
      const int64_t lo = cout ? c0[k] : vb[k], hi = cout ? c0[k + 1] : vb[k + 1];
      CSD_CUDA(cudaMemcpyAsync(host_coeffs + lo * K, d_coeffs + lo * K,
                               sizeof(float) * static_cast<size_t>(hi - lo) * K, cudaMemcpyDeviceToHost, ks));
    }
    CSD_CUDA(cudaEventRecord(h->oev[k], ks));  // chunk k's slab is on the host
  }
  if (user_out) {
    // a caller's pageable output: each chunk's rows are copied into the
    // volume (the unmasked rows zeroed) as soon as they are on the host, so
    // the copies of the first chunks overlap the later chunks' iterations
    const size_t row = sizeof(float) * static_cast<size_t>(K);
    for (int k = 0; k < C; ++k) {
      CSD_CUDA(cudaEventSynchronize(h->oev[k]));
      const auto t0 = std::chrono::steady_clock::now();
      masked_rows(
          host_mask, vb[k], vb[k + 1], c0[k],
          [&](int64_t v, int64_t r) { std::memcpy(user_out + v * K, host_coeffs + r * K, row); },
          [&](int64_t v0, int64_t v1) { std::memset(user_out + v0 * K, 0, row * static_cast<size_t>(v1 - v0)); });
      h->timing.ms_host_copy_out +=
          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  }
  if (d_out_host && !cout) CSD_CUDA(cudaStreamWaitEvent(st, h->pev[18], 0));
  for (int j = 1; j <= 2; ++j) {
    CSD_CUDA(cudaEventRecord(h->pev[15 + j], h->pipe[j]));
    CSD_CUDA(cudaStreamWaitEvent(st, h->pev[15 + j], 0));
  }
  record(h, 7);
  record(h, 3);
  unsigned long long itot[3] = {0, 0, 0};
  CSD_CUDA(cudaMemcpyAsync(itot, h->itotal.p, sizeof itot, cudaMemcpyDeviceToHost, st));
  CSD_CUDA(cudaStreamSynchronize(st));
  info.total_iterations = itot[0];
  info.representative_alpha = spec->alpha;
  info.Xfinal = h->X.as<double>();
  info.conv_final = h->conv.as<uint8_t>();
  h->timing.tensor_flops = static_cast<double>(itot[1]) * (Kp / 8) * 512.0;
  h->timing.fista_parked = static_cast<int64_t>(itot[2]);
  h->timing.ms_mixed_kernel = 0.f;
  h->timing.int8_tensor_ops = 0.0;
  h->timing.fp64_rerun_voxels = 0;
  float ms = 0;
  h->timing.ms_setup = (cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]) == cudaSuccess) ? ms : 0.f;
  h->timing.ms_rhs = 0.f;  // overlapped with the iterations
  h->timing.ms_solve = (cudaEventElapsedTime(&ms, h->ev[2], h->ev[7]) == cudaSuccess) ? ms : 0.f;
  h->timing.ms_solve_kernel = h->timing.ms_solve;
  h->timing.ms_epilogue = 0.f;
  h->timing.ms_total = (cudaEventElapsedTime(&ms, h->ev[0], h->ev[3]) == cudaSuccess) ? ms : 0.f;
  h->timing.launches = h->launches;
  return info;
}

void fill_scalars(const HostGtab& g, const FitInfo& info, const csd_shore_spec* spec, csd_fit_result* out) {
  out->n_coeffs = n_coeffs(spec->radial_order);
  out->n_voxels = info.V;
  out->has_alpha_distribution = info.has_dist ? 1 : 0;
  for (int i = 0; i < 3; ++i) out->alpha_distribution[i] = info.dist[i];
  out->representative_alpha = info.representative_alpha;
  out->big_delta_seconds = g.big;
  out->small_delta_seconds = g.small;
  out->tau_seconds = g.tau;
  out->delta_source = g.delta_source;
  out->n_shells = static_cast<int32_t>(std::min<size_t>(g.shells.size(), 32));
  for (int i = 0; i < out->n_shells; ++i) out->dwi_shells[i] = g.shells[i];
  out->lmax = info.lmax;
  out->n_constraint_dirs = info.n_constraint_dirs;
  out->total_iterations = info.total_iterations;
}

}  // namespace

// ======================================================================
// C ABI
// ======================================================================

extern "C" {

const char* csd_version(void) { return "cs_dmri_b200 0.1.0 (sm_100a)"; }
int csd_abi_version(void) { return CSD_ABI_VERSION; }

void csd_default_spec(csd_shore_spec* s) {
  s->radial_order = 6;
  s->zeta = 700.0;
  s->regularization = CSD_REG_L1;
  s->alpha_mode = CSD_ALPHA_L2_ANCHORED;
  s->alpha = 1.0;
  s->alpha_ratio = 1e-3;
  s->path_n_alphas = 20;
  s->path_eps = 0.0;
  s->slack = 0.05;
  s->max_iter = 1000;
  s->tol = 1e-6;
  s->non_negative = 0;
  s->lambda_n = 1e-8;
  s->lambda_l = 1e-8;
  s->nonneg_max_iter = 200;
  s->nonneg_tol = 1e-9;
  s->nonneg_epsilon = 1e-10;
  s->diagnostics = 0;
  s->allow_single_shell = 0;
  s->precision = CSD_PRECISION_FP64;
}

int csd_shore_n_coeffs(int32_t radial_order) { return radial_order < 0 ? 0 : n_coeffs(radial_order); }

int csd_create(csd_handle** out, int32_t device, char* err, size_t err_len) {
  if (!out) {
    set_err(err, err_len, "null handle pointer");
    return CSD_ERR_INVALID;
  }
  *out = nullptr;
  csd_handle* h = new csd_handle();
  try {
    int count = 0;
    CSD_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count)
      throw Error{CSD_ERR_INVALID, "CUDA device " + std::to_string(device) + " not present (" +
                                       std::to_string(count) + " visible)"};
    CSD_CUDA(cudaSetDevice(device));
    h->device = device;
    cudaDeviceProp prop{};
    CSD_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
      throw Error{CSD_ERR_CUDA, std::string("this library is built for sm_100a (B200); device is ") +
                                    prop.name};
    h->num_sms = prop.multiProcessorCount;
    h->smem_optin = static_cast<int>(prop.sharedMemPerBlockOptin);
    CSD_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    for (auto& e : h->ev) CSD_CUDA(cudaEventCreate(&e));
    CSD_CUDA(cudaEventCreateWithFlags(&h->order_ev, cudaEventDisableTiming));
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    delete h;
    return e.code;
  }
  *out = h;
  return CSD_OK;
}

void csd_destroy(csd_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  DevBuf* bufs[] = {&h->bvals, &h->bvecs, &h->M, &h->Mt, &h->G, &h->A, &h->gfrag, &h->mfrag, &h->mtfrag, &h->sst_v, &h->mom, &h->scal, &h->ok, &h->dirs, &h->Cmat, &h->Le, &h->Wi, &h->Q1, &h->ovf,
                    &h->icls_gam, &h->icls_ut, &h->icls_ginv, &h->icls_y, &h->icls_pf, &h->icls_jcol,
                    &h->data, &h->mask, &h->coeffs, &h->r2, &h->resid, &h->iters_map, &h->kind_map,
                    &h->alpha_map, &h->bic_map, &h->rss_map, &h->blk, &h->total, &h->vox, &h->B, &h->X, &h->sig,
                    &h->iters, &h->conv, &h->queue, &h->itotal, &h->resid_v, &h->nnz_v, &h->amax,
                    &h->zero, &h->alpha_v, &h->Xsel, &h->Xfb, &h->Xl2, &h->rss_l2, &h->list, &h->active,
                    &h->pbest, &h->psel, &h->pact, &h->palpha_sel, &h->pit_sel, &h->pconv_sel,
                    &h->palpha_fb, &h->pit_fb, &h->pconv_fb, &h->pcode, &h->gdig, &h->gfexp, &h->flagged,
                    &h->mixstat, &h->pcoef, &h->pmat, &h->pout, &h->pgt, &h->pgv, &h->pdir, &h->pconst,
                    &h->iota, &h->adjW, &h->adjovf, &h->adjstat, &h->adjconst, &h->hinv,
                    &h->gdtab, &h->gdq, &h->tuneB, &h->tuneX, &h->tuneIt, &h->tuneConv, &h->tuneQ,
                    &h->schedY, &h->schedPend, &h->schedKey, &h->schedOrder, &h->schedCnt,
                    &h->schedD, &h->schedU, &h->schedN, &h->gtf32, &h->x32, &h->kktv, &h->kktovf,
                    &h->kktfail, &h->kktstat};
  for (auto s : h->pipe)
    if (s) cudaStreamSynchronize(s);
  for (DevBuf* b : bufs) b->release();
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->order_ev) cudaEventDestroy(h->order_ev);
  for (auto& e : h->pev)
    if (e) cudaEventDestroy(e);
  for (auto& e : h->oev)
    if (e) cudaEventDestroy(e);
  for (auto& e : h->kev)
    if (e) cudaEventDestroy(e);
  if (h->stage) cudaFreeHost(h->stage);
  if (h->ostage) cudaFreeHost(h->ostage);
  for (auto s : h->pipe)
    if (s) cudaStreamDestroy(s);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

static int check_common(csd_handle* h, const void* data, const void* mask, int64_t X, int64_t Y, int64_t Z,
                        const csd_gtab* gtab, const csd_shore_spec* spec, csd_fit_result* out) {
  if (!h || !data || !mask || !gtab || !spec || !out || !out->coefficients) return 1;
  if (X < 0 || Y < 0 || Z < 0 || gtab->n <= 0 || !gtab->bvals || !gtab->bvecs) return 1;
  return 0;
}

int csd_shore_fit_volume_device(csd_handle* h, const float* d_data, const uint8_t* d_mask, int64_t X,
                                int64_t Y, int64_t Z, const csd_gtab* gtab, const csd_shore_spec* spec,
                                csd_fit_result* out, void* stream, char* err, size_t err_len) {
  if (check_common(h, d_data, d_mask, X, Y, Z, gtab, spec, out)) {
    set_err(err, err_len, "invalid argument: null pointer or bad shape");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    HostGtab g = make_gtab(gtab);
    std::string warnings;
    const double path_eps = validate(spec, g, warnings);
    // Queue the whole fit on the caller's stream when one is given.
    struct StreamSwap {
      csd_handle* h;
      cudaStream_t saved;
      ~StreamSwap() { h->stream = saved; }
    } swap{h, h->stream};
    if (stream) h->stream = static_cast<cudaStream_t>(stream);
    HandleOrder call_order(h);
    DevOut d{out->coefficients, out->r2,  out->residual_l2, out->alpha, out->bic, out->rss_l2,
             out->iterations,   out->regularization_kind};
    FitInfo info = run_fit(h, d_data, d_mask, X * Y * Z, g, spec, path_eps, d);
    const int K = n_coeffs(spec->radial_order);
    if (out->coef64 && info.V > 0)
      CSD_CUDA(cudaMemcpy2DAsync(out->coef64, sizeof(double) * K, info.Xfinal, sizeof(double) * h->Kp,
                                 sizeof(double) * K, info.V, cudaMemcpyDeviceToDevice, h->stream));
    if (out->converged && info.V > 0)
      CSD_CUDA(cudaMemcpyAsync(out->converged, info.conv_final, info.V, cudaMemcpyDeviceToDevice, h->stream));
    CSD_CUDA(cudaStreamSynchronize(h->stream));
    fill_scalars(g, info, spec, out);
    warnings += info.warnings;
    std::snprintf(out->warnings, sizeof out->warnings, "%s", warnings.c_str());
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_fit_volume(csd_handle* h, const float* data, const uint8_t* mask, int64_t X, int64_t Y,
                         int64_t Z, const csd_gtab* gtab, const csd_shore_spec* spec, csd_fit_result* out,
                         char* err, size_t err_len) {
  if (check_common(h, data, mask, X, Y, Z, gtab, spec, out)) {
    set_err(err, err_len, "invalid argument: null pointer or bad shape");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    HandleOrder call_order(h);
    HostGtab g = make_gtab(gtab);
    std::string warnings;
    const double path_eps = validate(spec, g, warnings);
    const int64_t nvol = X * Y * Z;
    const int N = gtab->n;
    const int K = n_coeffs(spec->radial_order);
    cudaStream_t st = h->stream;
    h->mask.ensure(static_cast<size_t>(nvol));
    h->coeffs.ensure(sizeof(float) * static_cast<size_t>(nvol) * K);
    CSD_CUDA(cudaMemcpyAsync(h->mask.p, mask, static_cast<size_t>(nvol), cudaMemcpyHostToDevice, st));
    // Pinned (page-locked, mapped) input volumes are read in place by the
    // right-hand-side kernel, masked rows only; pageable ones are copied whole.
    const float* d_data = nullptr;
    bool on_host = false;
    {
      cudaPointerAttributes attr{};
      if (cudaPointerGetAttributes(&attr, data) == cudaSuccess && attr.type == cudaMemoryTypeHost &&
          attr.devicePointer && h->dmma_rhs_possible(N, K)) {
        d_data = static_cast<const float*>(attr.devicePointer);
        on_host = true;
      }
      cudaGetLastError();  // a pageable pointer may leave an error code behind
    }
    h->timing.ms_host_gather = 0.f;
    h->timing.ms_host_copy_out = 0.f;
    // Fixed-alpha FP64 L1 with nothing but the coefficients requested: the
    // pipelined path (transfers overlap the fit) when the volume is on the host.
    const bool pipe_ok = K == 72 && spec->regularization == CSD_REG_L1 && spec->alpha_mode == CSD_ALPHA_FIXED &&
                         spec->precision == CSD_PRECISION_FP64 && spec->diagnostics == 0 && !out->coef64 &&
                         !out->converged && spec->max_iter > 0 && (fista_variant(h) == 3 || fista_variant(h) == 4);
    int64_t v_host = -1;  // masked voxels, counted on the host when a compact buffer is sized
    auto masked_count = [&]() {
      if (v_host < 0) {
        std::atomic<int64_t> c{0};
        host_parallel(nvol, 1 << 16, [&](int64_t a, int64_t b) {
          int64_t k = 0;
          for (int64_t v = a; v < b; ++v) k += mask[v] != 0;
          c += k;
        });
        v_host = c.load();
      }
      return v_host;
    };
    bool staged = false, stage_compact = false;
    if (!on_host && h->dmma_rhs_possible(N, K)) {
      // A pageable volume: its masked rows are gathered on host threads into
      // the handle's page-locked staging buffer, which the device then reads
      // in place like a page-locked input.  For the pipelined fit the buffer
      // holds only the masked rows, in order (gathered chunk by chunk,
      // below); other fits use a buffer of the volume's shape (masked rows
      // only written and read) and gather everything first.
      stage_compact = pipe_ok;
      const int64_t rows = stage_compact ? std::max<int64_t>(masked_count(), 1) : nvol;
      float* stage = ensure_pinned(h->stage, h->stage_bytes, sizeof(float) * static_cast<size_t>(rows) * N);
      void* dp = nullptr;
      CSD_CUDA(cudaHostGetDevicePointer(&dp, stage, 0));
      d_data = static_cast<const float*>(dp);
      on_host = true;
      staged = true;
    }
    if (!on_host) {
      h->data.ensure(sizeof(float) * static_cast<size_t>(nvol) * N);
      CSD_CUDA(cudaMemcpyAsync(h->data.p, data, sizeof(float) * static_cast<size_t>(nvol) * N,
                               cudaMemcpyHostToDevice, st));
      d_data = h->data.as<float>();
    }
    const bool diag = spec->diagnostics != 0;
    auto map_f = [&](DevBuf& b, void* host) -> float* {
      if (!diag || !host) return nullptr;
      b.ensure(sizeof(float) * nvol);
      return b.as<float>();
    };
    DevOut d{};
    d.coeffs = h->coeffs.as<float>();
    d.r2 = map_f(h->r2, out->r2);
    d.resid = map_f(h->resid, out->residual_l2);
    d.alpha = map_f(h->alpha_map, out->alpha);
    d.bic = map_f(h->bic_map, out->bic);
    d.rss_l2 = map_f(h->rss_map, out->rss_l2);
    if (diag && out->iterations) {
      h->iters_map.ensure(sizeof(uint32_t) * nvol);
      d.iters = h->iters_map.as<uint32_t>();
    }
    if (diag && out->regularization_kind) {
      h->kind_map.ensure(nvol);
      d.kind = h->kind_map.as<uint8_t>();
    }
    const bool pipelined = on_host && pipe_ok;
    // A pageable output of the pipelined fit: the fit writes the masked
    // voxels' coefficients in position order into the handle's page-locked
    // buffer (V x K), and host threads copy each chunk's rows into the
    // caller's volume as soon as they are on the host, zeroing the others.
    float* host_out = out->coefficients;
    bool out_staged = false;
    if (pipelined) {
      cudaPointerAttributes attr{};
      const bool pinned_out = cudaPointerGetAttributes(&attr, out->coefficients) == cudaSuccess &&
                              attr.type == cudaMemoryTypeHost && attr.devicePointer;
      cudaGetLastError();
      if (!pinned_out) {
        host_out = ensure_pinned(h->ostage, h->ostage_bytes,
                                 sizeof(float) * static_cast<size_t>(std::max<int64_t>(masked_count(), 1)) * K);
        out_staged = true;
      }
    }
    HostGather hg;
    if (staged) {
      hg.data = data;
      hg.mask = mask;
      hg.stage = h->stage;
      hg.N = N;
      hg.compact = stage_compact;
      if (!pipelined) {
        const auto t0 = std::chrono::steady_clock::now();
        gather_rows(hg, 0, nvol);
        h->timing.ms_host_gather =
            std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
      }
    }
    FitInfo info = pipelined
                       ? run_fit_pipelined(h, d_data, h->mask.as<uint8_t>(), nvol, g, spec, d.coeffs, host_out,
                                           staged ? &hg : nullptr, out_staged ? out->coefficients : nullptr,
                                           mask)
                       : run_fit(h, d_data, h->mask.as<uint8_t>(), nvol, g, spec, path_eps, d, on_host);
    if (!pipelined)
      CSD_CUDA(cudaMemcpyAsync(out->coefficients, d.coeffs, sizeof(float) * static_cast<size_t>(nvol) * K,
                               cudaMemcpyDeviceToHost, st));
    const bool is_l1 = spec->regularization == CSD_REG_L1;
    if (diag) {
      if (d.r2) CSD_CUDA(cudaMemcpyAsync(out->r2, d.r2, sizeof(float) * nvol, cudaMemcpyDeviceToHost, st));
      if (d.resid)
        CSD_CUDA(cudaMemcpyAsync(out->residual_l2, d.resid, sizeof(float) * nvol, cudaMemcpyDeviceToHost, st));
      if (d.iters)
        CSD_CUDA(cudaMemcpyAsync(out->iterations, d.iters, sizeof(uint32_t) * nvol, cudaMemcpyDeviceToHost, st));
      if (d.kind)
        CSD_CUDA(cudaMemcpyAsync(out->regularization_kind, d.kind, nvol, cudaMemcpyDeviceToHost, st));
      if (d.alpha && is_l1)
        CSD_CUDA(cudaMemcpyAsync(out->alpha, d.alpha, sizeof(float) * nvol, cudaMemcpyDeviceToHost, st));
      if (d.bic && is_l1)
        CSD_CUDA(cudaMemcpyAsync(out->bic, d.bic, sizeof(float) * nvol, cudaMemcpyDeviceToHost, st));
      if (d.rss_l2 && is_l1 && spec->alpha_mode == CSD_ALPHA_L2_ANCHORED)
        CSD_CUDA(cudaMemcpyAsync(out->rss_l2, d.rss_l2, sizeof(float) * nvol, cudaMemcpyDeviceToHost, st));
    }
    if (out->coef64 && info.V > 0)
      CSD_CUDA(cudaMemcpy2DAsync(out->coef64, sizeof(double) * K, info.Xfinal, sizeof(double) * h->Kp,
                                 sizeof(double) * K, info.V, cudaMemcpyDeviceToHost, st));
    if (out->converged && info.V > 0)
      CSD_CUDA(cudaMemcpyAsync(out->converged, info.conv_final, info.V, cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
    fill_scalars(g, info, spec, out);
    warnings += info.warnings;
    std::snprintf(out->warnings, sizeof out->warnings, "%s", warnings.c_str());
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_design_matrix(csd_handle* h, const csd_gtab* gtab, int32_t radial_order, double zeta,
                            double* out, char* err, size_t err_len) {
  if (!h || !gtab || !out || gtab->n <= 0 || radial_order < 0) {
    set_err(err, err_len, "invalid argument");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    HandleOrder call_order(h);
    HostGtab g = make_gtab(gtab);
    ensure_setup(h, g, radial_order, zeta, false, 0.0, 0.0);
    CSD_CUDA(cudaMemcpyAsync(out, h->M.p, sizeof(double) * h->N * h->K, cudaMemcpyDeviceToHost, h->stream));
    CSD_CUDA(cudaStreamSynchronize(h->stream));
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

}  // extern "C"

namespace {

void check_coeff_args(int64_t X, int64_t Y, int64_t Z, int32_t radial_order) {
  if (X < 0 || Y < 0 || Z < 0) throw Error{CSD_ERR_INVALID, "volume dimensions must be non-negative"};
  if (radial_order < 0 || radial_order % 2 != 0 || radial_order > 14)
    throw Error{CSD_ERR_INVALID, "radial_order must be an even number <= 14, got " + std::to_string(radial_order)};
}

// Copy the coefficient volume to the device and launch k_apply_rows with AT
// (K x R, device) over it; the result comes back into `out`.
void apply_rows_volume(csd_handle* h, const float* coefficients, int64_t nvox, int K, const double* AT, int R,
                       const uint8_t* d_mask, bool skip_zero, float* out) {
  cudaStream_t st = h->stream;
  h->pcoef.ensure(sizeof(float) * std::max<int64_t>(nvox * K, 1));
  h->pout.ensure(sizeof(float) * std::max<int64_t>(nvox * R, 1));
  if (nvox == 0) return;
  CSD_CUDA(cudaMemcpyAsync(h->pcoef.p, coefficients, sizeof(float) * nvox * K, cudaMemcpyHostToDevice, st));
  const size_t smem = sizeof(double) * csd::kApplyTile * K;
  const int64_t tiles = (nvox + csd::kApplyTile - 1) / csd::kApplyTile;
  const int grid = static_cast<int>(std::min<int64_t>(tiles, static_cast<int64_t>(h->num_sms) * 8));
  csd::k_apply_rows<<<grid, 256, smem, st>>>(h->pcoef.as<float>(), nvox, K, AT, R, d_mask, skip_zero ? 1 : 0,
                                             h->pout.as<float>());
  CSD_LAUNCH();
  CSD_CUDA(cudaMemcpyAsync(out, h->pout.p, sizeof(float) * nvox * R, cudaMemcpyDeviceToHost, st));
  CSD_CUDA(cudaStreamSynchronize(st));
}

// Nearest-rank percentile of the finite values (io/microstructure.rs:303-313).
bool finite_percentile(const float* xs, int64_t n, double percentile, float* out) {
  std::vector<float> f;
  f.reserve(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i)
    if (std::isfinite(xs[i])) f.push_back(xs[i]);
  if (f.empty()) return false;
  const size_t m = f.size();
  const double p = std::min(std::max(percentile, 0.0), 100.0) / 100.0;
  const size_t idx = std::min(static_cast<size_t>(std::round(p * static_cast<double>(m - 1))), m - 1);
  std::nth_element(f.begin(), f.begin() + static_cast<std::ptrdiff_t>(idx), f.end());
  *out = f[idx];
  return true;
}

}  // namespace

extern "C" {

int csd_shore_predict(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                      int32_t radial_order, double zeta, const csd_gtab* target, float* signal_out, char* err,
                      size_t err_len) {
  if (!h || !target || target->n <= 0 || (!coefficients && X * Y * Z > 0) || (!signal_out && X * Y * Z > 0)) {
    set_err(err, err_len, "invalid argument");
    return CSD_ERR_INVALID;
  }
  try {
    check_coeff_args(X, Y, Z, radial_order);
    CSD_CUDA(cudaSetDevice(h->device));
    HandleOrder call_order(h);
    cudaStream_t st = h->stream;
    HostGtab g = make_gtab(target);
    const int N = static_cast<int>(g.bvals.size());
    const int K = n_coeffs(radial_order);
    h->pgv.ensure(sizeof(double) * 4 * N);
    CSD_CUDA(cudaMemcpyAsync(h->pgv.p, g.bvals.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
    CSD_CUDA(cudaMemcpyAsync(h->pgv.as<double>() + N, g.bvecs.data(), sizeof(double) * 3 * N,
                             cudaMemcpyHostToDevice, st));
    h->pmat.ensure(sizeof(double) * static_cast<size_t>(N) * K);
    h->pgt.ensure(sizeof(double) * static_cast<size_t>(K) * N);
    const double qdenom = 4.0 * kPi * kPi * g.tau;  // src/qspace.rs:384-385
    const long long nk = static_cast<long long>(N) * K;
    csd::k_design<<<static_cast<unsigned>((nk + 255) / 256), 256, 0, st>>>(
        h->pgv.as<double>(), h->pgv.as<double>() + N, N, K, radial_order, zeta, qdenom, g.b0, h->pmat.as<double>());
    CSD_LAUNCH();
    csd::k_transpose_design<<<(K * N + 255) / 256, 256, 0, st>>>(h->pmat.as<double>(), N, K, K, h->pgt.as<double>());
    CSD_LAUNCH();
    apply_rows_volume(h, coefficients, X * Y * Z, K, h->pgt.as<double>(), N, nullptr, true, signal_out);
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_odf_sh(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                     int32_t radial_order, double zeta, int32_t lmax, const uint8_t* mask, float* sh_out, char* err,
                     size_t err_len) {
  if (!h || (!coefficients && X * Y * Z > 0) || (!sh_out && X * Y * Z > 0)) {
    set_err(err, err_len, "invalid argument");
    return CSD_ERR_INVALID;
  }
  try {
    check_coeff_args(X, Y, Z, radial_order);
    if (lmax < 0 || lmax % 2 != 0 || lmax > radial_order)  // python/src/models.rs:212-214
      throw Error{CSD_ERR_INVALID, "lmax must be even and \xe2\x89\xa4 radial_order (" + std::to_string(radial_order) +
                                       "), got " + std::to_string(lmax)};
    CSD_CUDA(cudaSetDevice(h->device));
    HandleOrder call_order(h);
    cudaStream_t st = h->stream;
    const int K = n_coeffs(radial_order);
    const int R = (lmax + 1) * (lmax + 2) / 2;
    const int64_t nvox = X * Y * Z;
    h->pgt.ensure(sizeof(double) * static_cast<size_t>(K) * R);
    CSD_CUDA(cudaMemsetAsync(h->pgt.p, 0, sizeof(double) * static_cast<size_t>(K) * R, st));
    csd::k_tournier_projT<<<grid1(K), 256, 0, st>>>(K, radial_order, zeta, lmax, R, h->pgt.as<double>());
    CSD_LAUNCH();
    const uint8_t* d_mask = nullptr;
    if (mask && nvox > 0) {
      h->mask.ensure(std::max<int64_t>(nvox, 1));
      CSD_CUDA(cudaMemcpyAsync(h->mask.p, mask, nvox, cudaMemcpyHostToDevice, st));
      d_mask = h->mask.as<uint8_t>();
    }
    apply_rows_volume(h, coefficients, nvox, K, h->pgt.as<double>(), R, d_mask, false, sh_out);
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_microstructure(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                             int32_t radial_order, double zeta, const uint8_t* mask, const float* directions,
                             int32_t units, int32_t reject_outliers, float outlier_factor, float* rtop, float* rtap,
                             float* rtpp, float* msd, float* qiv, float* ng, char* err, size_t err_len) {
  float* maps[6] = {rtop, rtap, rtpp, msd, qiv, ng};
  const int64_t nvox = X * Y * Z;
  bool outs_ok = true;
  for (float* m : maps) outs_ok = outs_ok && (m || nvox == 0);
  if (!h || !outs_ok || ((!coefficients || !mask) && nvox > 0)) {
    set_err(err, err_len, "invalid argument");
    return CSD_ERR_INVALID;
  }
  try {
    check_coeff_args(X, Y, Z, radial_order);
    if (units != 0 && units != 1) throw Error{CSD_ERR_INVALID, "units must be 0 (um) or 1 (mm)"};
    CSD_CUDA(cudaSetDevice(h->device));
    HandleOrder call_order(h);
    cudaStream_t st = h->stream;
    const int K = n_coeffs(radial_order);
    for (float* m : maps)
      if (nvox > 0) std::fill(m, m + nvox, 0.0f);
    if (nvox == 0) return CSD_OK;
    h->mask.ensure(nvox);
    CSD_CUDA(cudaMemcpyAsync(h->mask.p, mask, nvox, cudaMemcpyHostToDevice, st));
    const int64_t V = compact(h, h->mask.as<uint8_t>(), nvox, h->vox);
    if (V == 0) return CSD_OK;
    h->pcoef.ensure(sizeof(float) * nvox * K);
    CSD_CUDA(cudaMemcpyAsync(h->pcoef.p, coefficients, sizeof(float) * nvox * K, cudaMemcpyHostToDevice, st));
    const float* d_dirs = nullptr;
    if (directions) {
      h->pdir.ensure(sizeof(float) * nvox * 3);
      CSD_CUDA(cudaMemcpyAsync(h->pdir.p, directions, sizeof(float) * nvox * 3, cudaMemcpyHostToDevice, st));
      d_dirs = h->pdir.as<float>();
    }
    h->pconst.ensure(sizeof(csd::MicroConsts));
    csd::k_micro_consts<<<1, 1, 0, st>>>(radial_order, zeta, h->pconst.as<csd::MicroConsts>());
    CSD_LAUNCH();
    // unit scales (io/microstructure.rs:162-173)
    const bool um = units == 0;
    h->pout.ensure(sizeof(float) * 6 * V);
    csd::k_microstructure<<<grid1(V, 128), 128, 0, st>>>(
        h->pcoef.as<float>(), h->vox.as<int64_t>(), V, d_dirs, h->pconst.as<csd::MicroConsts>(), um ? 1e-9f : 1.0f,
        um ? 1e-6f : 1.0f, um ? 1e-3f : 1.0f, um ? 1e6f : 1.0f, um ? 1e15f : 1.0f, 1.0f, h->pout.as<float>());
    CSD_LAUNCH();
    std::vector<float> s(static_cast<size_t>(6 * V));
    std::vector<int64_t> vox(static_cast<size_t>(V));
    CSD_CUDA(cudaMemcpyAsync(s.data(), h->pout.p, sizeof(float) * 6 * V, cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaMemcpyAsync(vox.data(), h->vox.p, sizeof(int64_t) * V, cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
    for (int m = 0; m < 6; ++m) {
      float* a = s.data() + static_cast<size_t>(m) * V;
      if (reject_outliers) {  // io/microstructure.rs:222-270, nan_above (:317-326)
        float p99;
        if (finite_percentile(a, V, 99.0, &p99)) {
          const float thr = outlier_factor * p99;
          for (int64_t i = 0; i < V; ++i)
            if (std::isfinite(a[i]) && a[i] > thr) a[i] = std::nanf("");
        }
      }
      for (int64_t i = 0; i < V; ++i) maps[m][vox[static_cast<size_t>(i)]] = a[i];
    }
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_set_option(csd_handle* h, int32_t option, int64_t value) {
  if (!h) return CSD_ERR_INVALID;
  switch (option) {
    case CSD_OPT_FISTA_SHAPE:
      if (value != 0 && value != 1 && value != 12 && value != 16) return CSD_ERR_INVALID;
      h->opt_shape = static_cast<int>(value);
      return CSD_OK;
    case CSD_OPT_FISTA_SCHEDULE:
      if (value < 0 || value > 100000) return CSD_ERR_INVALID;
      h->opt_schedule = static_cast<int>(value);
      return CSD_OK;
    case CSD_OPT_KKT_ITERATIONS:
      if (value < 0 || value > 100000) return CSD_ERR_INVALID;
      h->opt_kkt_iters = static_cast<int>(value);
      return CSD_OK;
    case CSD_OPT_KKT_ROUNDS:
      if (value < 1 || value > 4096) return CSD_ERR_INVALID;
      h->opt_kkt_rounds = static_cast<int>(value);
      return CSD_OK;
    case CSD_OPT_TENSOR_WAIT_NS:
      if (value < 1 || value > 2000000000LL) return CSD_ERR_INVALID;
      h->opt_wait_ns = static_cast<unsigned long long>(value);
      return CSD_OK;
    case CSD_OPT_ICLS:
      if (value != 0 && value != 1) return CSD_ERR_INVALID;
      h->opt_icls = static_cast<int>(value);
      return CSD_OK;
    default:
      return CSD_ERR_INVALID;
  }
}

int csd_last_timing(const csd_handle* h, csd_fit_timing* out) {
  if (!h || !out) return CSD_ERR_INVALID;
  *out = h->timing;
  out->fista_warps = h->fista_warps;
  out->fista_tune_ms12 = h->tune_ms[0];
  out->fista_tune_ms16 = h->tune_ms[1];
  return CSD_OK;
}

}  // extern "C"

// ======================================================================
// Allocation-free batch fit
// ======================================================================
//
// Some callers cannot let a library call cudaMalloc: applications that hand
// all device memory to their own pool allocator up front (a framework's
// caching allocator, an inference server with a fixed memory budget), and
// latency-critical pipelines for which cudaMalloc / cudaFree are unacceptable
// because cudaFree synchronises the whole device and either may fail once
// the pool owns the memory.  csd_shore_fista_batch_noalloc serves them: it
// runs the fixed-alpha FISTA fit of a batch of voxels with every piece of
// scratch (design matrix, Gram tiles, right-hand sides, iterates, work
// queue) placed in one statically sized device array that the library
// reserves when it is loaded.  The caller still provides the inputs and
// outputs in device memory.
//
// Limits: at most kNoAllocMaxVoxels voxels and kNoAllocMaxMeasurements
// measurements per call, radial order <= 6 (K <= 72).  The array is about
// 10.3 MB and every GPU that loads the library holds it until the process
// exits.  All calls share it and it keeps the last call's contents: each
// call rebuilds what it reads and clears the work-queue counter, but two
// calls that overlap on the GPU (different streams or threads) race on it.

namespace {

constexpr int64_t kNoAllocMaxVoxels = 8192;
constexpr int kNoAllocMaxMeasurements = 1024;
constexpr int kNoAllocMaxKp = 72;

constexpr size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }
constexpr size_t kNaBvals = 0;
constexpr size_t kNaBvecs = align256(kNaBvals + sizeof(double) * kNoAllocMaxMeasurements);
constexpr size_t kNaM = align256(kNaBvecs + sizeof(double) * 3 * kNoAllocMaxMeasurements);
constexpr size_t kNaG = align256(kNaM + sizeof(double) * kNoAllocMaxMeasurements * kNoAllocMaxKp);
constexpr size_t kNaGfrag = align256(kNaG + sizeof(double) * kNoAllocMaxKp * kNoAllocMaxKp);
constexpr size_t kNaScal = align256(kNaGfrag + sizeof(double) * kNoAllocMaxKp * kNoAllocMaxKp);
constexpr size_t kNaVox = align256(kNaScal + sizeof(double) * 4);
constexpr size_t kNaB = align256(kNaVox + sizeof(int64_t) * kNoAllocMaxVoxels);
constexpr size_t kNaX = align256(kNaB + sizeof(double) * kNoAllocMaxVoxels * kNoAllocMaxKp);
constexpr size_t kNaIters = align256(kNaX + sizeof(double) * kNoAllocMaxVoxels * kNoAllocMaxKp);
constexpr size_t kNaConv = align256(kNaIters + sizeof(uint32_t) * kNoAllocMaxVoxels);
constexpr size_t kNaQueue = align256(kNaConv + kNoAllocMaxVoxels);
constexpr size_t kNoAllocBytes = align256(kNaQueue + sizeof(unsigned long long));

__global__ void k_noalloc_iota(int64_t* vox, int64_t V) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v < V) vox[v] = v;
}

__global__ void k_noalloc_to_f32(const double* X, int64_t V, int K, int Kp, float* out) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= V * K) return;
  out[e] = static_cast<float>(X[(e / K) * Kp + (e % K)]);
}

}  // namespace

// The scratch of csd_shore_fista_batch_noalloc.  Host code must not use this
// name as an address: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[256] = {};

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached for the life of the
// process.  cudaDeviceReset unloads the module that holds the array, so the
// cached address is not valid across a reset: this entry point must not be
// called after the process has reset a device.
unsigned char* noalloc_scratch(int device) {
  if (device < 0 || device >= 256) throw Error{CSD_ERR_INVALID, "device index out of range"};
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error{CSD_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e)};
    g_noalloc_addr[device] = static_cast<unsigned char*>(p);
  }
  return g_noalloc_addr[device];
}

template <int MT>
void noalloc_fista(const csd::FistaParams& p, int num_sms, cudaStream_t st) {
  constexpr int KP = 8 * MT, KT = 2 * MT;
  const size_t smem = sizeof(double) * (static_cast<size_t>(MT) * KT * 32 + 8 * KP * 8);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_fista_fp64<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  int per_sm = 0;
  CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_fista_fp64<MT>, 256, smem));
  per_sm = std::max(per_sm, 1);
  const int64_t warps_needed = (p.n_work + 7) / 8;
  int64_t blocks = std::min<int64_t>(static_cast<int64_t>(num_sms) * per_sm, (warps_needed + 7) / 8);
  blocks = std::max<int64_t>(blocks, 1);
  csd::k_fista_fp64<MT><<<static_cast<unsigned>(blocks), 256, smem, st>>>(p);
  CSD_CUDA(cudaGetLastError());
}

template <int KP>
void noalloc_rhs(const float* d, const int64_t* vox, int64_t V, int N, const double* M, int K, double* B,
                 cudaStream_t st) {
  const size_t smem = sizeof(double) * (32 * KP + 64 * 33);
  CSD_CUDA(cudaFuncSetAttribute(csd::k_rhs<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  csd::k_rhs<KP><<<static_cast<unsigned>((V + 63) / 64), 256, smem, st>>>(d, vox, V, N, M, K, B);
  CSD_CUDA(cudaGetLastError());
}

}  // namespace

extern "C" int csd_shore_fista_batch_noalloc(const csd_gtab* gtab, const csd_shore_spec* spec,
                                             const float* d_signals, int64_t n_voxels, float* d_coeffs,
                                             uint32_t* d_iterations, void* stream, char* err,
                                             size_t err_len) {
  if (!gtab || !spec || !gtab->bvals || !gtab->bvecs || gtab->n <= 0 || n_voxels < 0 ||
      (n_voxels > 0 && (!d_signals || !d_coeffs))) {
    set_err(err, err_len, "invalid argument: null pointer or bad size");
    return CSD_ERR_INVALID;
  }
  try {
    if (spec->regularization != CSD_REG_L1 || spec->alpha_mode != CSD_ALPHA_FIXED)
      throw Error{CSD_ERR_INVALID, "the allocation-free batch fit supports L1 with a fixed alpha only"};
    if (spec->precision != CSD_PRECISION_FP64)
      throw Error{CSD_ERR_INVALID, "the allocation-free batch fit runs in FP64 only (precision fp64)"};
    if (spec->radial_order > 6)
      throw Error{CSD_ERR_INVALID, "the allocation-free batch fit supports radial order <= 6 (K <= 72), got " +
                                       std::to_string(spec->radial_order)};
    if (gtab->n > kNoAllocMaxMeasurements)
      throw Error{CSD_ERR_INVALID, "the allocation-free batch fit takes at most " +
                                       std::to_string(kNoAllocMaxMeasurements) + " measurements, got " +
                                       std::to_string(gtab->n)};
    if (n_voxels > kNoAllocMaxVoxels)
      throw Error{CSD_ERR_INVALID, "the allocation-free batch fit takes at most " +
                                       std::to_string(kNoAllocMaxVoxels) + " voxels per call, got " +
                                       std::to_string(n_voxels)};
    HostGtab g = make_gtab(gtab);
    std::string warnings;
    validate(spec, g, warnings);
    int device = 0;
    CSD_CUDA(cudaGetDevice(&device));
    int num_sms = 0;
    CSD_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    unsigned char* s = noalloc_scratch(device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int N = g.bvals.empty() ? 0 : static_cast<int>(g.bvals.size());
    const int K = n_coeffs(spec->radial_order);
    const int Kp = 8 * mt_for(K);
    const int MT = Kp / 8, KT = Kp / 4;
    double* bvals = reinterpret_cast<double*>(s + kNaBvals);
    double* bvecs = reinterpret_cast<double*>(s + kNaBvecs);
    double* M = reinterpret_cast<double*>(s + kNaM);
    double* G = reinterpret_cast<double*>(s + kNaG);
    double* gfrag = reinterpret_cast<double*>(s + kNaGfrag);
    double* scal = reinterpret_cast<double*>(s + kNaScal);
    int64_t* vox = reinterpret_cast<int64_t*>(s + kNaVox);
    double* B = reinterpret_cast<double*>(s + kNaB);
    double* X = reinterpret_cast<double*>(s + kNaX);
    uint32_t* iters = reinterpret_cast<uint32_t*>(s + kNaIters);
    uint8_t* conv = reinterpret_cast<uint8_t*>(s + kNaConv);
    unsigned long long* queue = reinterpret_cast<unsigned long long*>(s + kNaQueue);

    // Setup of this gradient table (rebuilt on every call).
    CSD_CUDA(cudaMemcpyAsync(bvals, g.bvals.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
    CSD_CUDA(cudaMemcpyAsync(bvecs, g.bvecs.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    const double qdenom = 4.0 * kPi * kPi * g.tau;
    const long long nk = static_cast<long long>(N) * K;
    csd::k_design<<<static_cast<unsigned>((nk + 255) / 256), 256, 0, st>>>(bvals, bvecs, N, K, spec->radial_order,
                                                                           spec->zeta, qdenom, g.b0, M);
    CSD_CUDA(cudaGetLastError());
    csd::k_gram<<<(Kp * Kp + 255) / 256, 256, 0, st>>>(M, N, K, Kp, spec->radial_order, 0.0, 0.0, G, nullptr);
    CSD_CUDA(cudaGetLastError());
    const size_t lsm = sizeof(double) * (static_cast<size_t>(Kp) * Kp + 2 * Kp);
    CSD_CUDA(cudaFuncSetAttribute(csd::k_lipschitz, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(lsm)));
    csd::k_lipschitz<<<1, 256, lsm, st>>>(G, Kp, N, 200000, scal, scal + 1);
    CSD_CUDA(cudaGetLastError());
    csd::k_pack_gfrag<<<(MT * KT * 32 + 255) / 256, 256, 0, st>>>(G, Kp, gfrag);
    CSD_CUDA(cudaGetLastError());
    double lipschitz = 0.0;
    CSD_CUDA(cudaMemcpyAsync(&lipschitz, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
    if (n_voxels == 0) return CSD_OK;

    // b = M^T s, then the FISTA iterations (the same kernels as the volume fit).
    k_noalloc_iota<<<grid1(n_voxels), 256, 0, st>>>(vox, n_voxels);
    CSD_CUDA(cudaGetLastError());
    switch (Kp) {
      case 8: noalloc_rhs<8>(d_signals, vox, n_voxels, N, M, K, B, st); break;
      case 32: noalloc_rhs<32>(d_signals, vox, n_voxels, N, M, K, B, st); break;
      case 72: noalloc_rhs<72>(d_signals, vox, n_voxels, N, M, K, B, st); break;
      default: throw Error{CSD_ERR_INVALID, "unsupported coefficient count"};
    }
    CSD_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st));
    csd::FistaParams fp{};
    fp.gfrag = gfrag;
    fp.B = B;
    fp.X = X;
    fp.warm = nullptr;
    fp.iters = iters;
    fp.conv = conv;
    fp.V = n_voxels;
    fp.n_inv = 1.0 / static_cast<double>(N);
    fp.step = 1.0 / lipschitz;
    fp.thr = fp.step * spec->alpha;
    fp.alpha_v = nullptr;
    fp.tol = spec->tol;
    fp.max_iter = spec->max_iter;
    fp.non_negative = spec->non_negative;
    fp.queue = queue;
    fp.list = nullptr;
    fp.n_work = n_voxels;
    fp.iter_total = nullptr;
    if (spec->max_iter <= 0) {
      csd::k_fista_noop<<<grid1(n_voxels * (Kp + 1)), 256, 0, st>>>(fp, Kp);
      CSD_CUDA(cudaGetLastError());
    } else {
      switch (MT) {
        case 1: noalloc_fista<1>(fp, num_sms, st); break;
        case 4: noalloc_fista<4>(fp, num_sms, st); break;
        case 9: noalloc_fista<9>(fp, num_sms, st); break;
        default: throw Error{CSD_ERR_INVALID, "unsupported coefficient count"};
      }
    }
    k_noalloc_to_f32<<<grid1(n_voxels * K), 256, 0, st>>>(X, n_voxels, K, Kp, d_coeffs);
    CSD_CUDA(cudaGetLastError());
    if (d_iterations)
      CSD_CUDA(cudaMemcpyAsync(d_iterations, iters, sizeof(uint32_t) * n_voxels, cudaMemcpyDeviceToDevice, st));
    CSD_CUDA(cudaStreamSynchronize(st));
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

#include "sphere_host.cuh"
#include "differentiable_host.cuh"
#include "peaks_host.cuh"
#include "graddev_host.cuh"
