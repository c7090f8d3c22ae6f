// Host side of the differentiable fit: a batch fit of device-resident voxel
// signals with FP64 coefficients out (fixed or per-voxel alpha, optional warm
// start), its adjoint, and the linear / ratio maps on coefficients (ODF
// amplitudes on a sphere, predicted signals, RTOP) with theirs.  Included once
// at the end of csd_shore.cu: it uses that file's handle and helpers.
#pragma once

namespace {

// Queue a call's work on the caller's stream; NULL is the legacy default
// stream (the calls return without waiting, so the work must be ordered with
// what the caller does next on that stream).
struct StreamScope {
  csd_handle* h;
  cudaStream_t saved;
  StreamScope(csd_handle* hh, void* stream) : h(hh), saved(hh->stream) {
    h->stream = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
  }
  ~StreamScope() { h->stream = saved; }
};

// b = M^T s for every row, then FISTA (fixed or per-voxel alpha, optional
// warm start) or the Tikhonov solve; FP64 coefficients (V x K) out.
void run_fit_batch(csd_handle* h, const float* d_sig, int64_t V, const HostGtab& g, const csd_shore_spec* spec,
                   const double* d_alpha, const double* d_warm, const int64_t* d_order, double* d_coef,
                   uint32_t* d_iters) {
  cudaStream_t st = h->stream;
  h->launches = 0;
  h->precision = spec->precision;
  const bool is_l1 = spec->regularization == CSD_REG_L1;
  ensure_setup(h, g, spec->radial_order, spec->zeta, !is_l1, spec->lambda_n, spec->lambda_l);
  const int N = h->N, K = h->K, Kp = h->Kp;
  if (V == 0) return;
  h->vox.ensure(sizeof(int64_t) * V);
  h->B.ensure(sizeof(double) * V * Kp);
  h->X.ensure(sizeof(double) * V * Kp);
  h->iters.ensure(sizeof(uint32_t) * V);
  h->conv.ensure(V);
  h->queue.ensure(sizeof(unsigned long long));
  csd::k_iota<<<grid1(V), 256, 0, st>>>(h->vox.as<int64_t>(), V);
  CSD_LAUNCH();
  // Tikhonov with the DMMA product c = P s, as the volume fit does
  const bool l2_operator = !is_l1 && h->dmma_rhs && h->pfrag_valid;
  launch_rhs(h, d_sig, V, nullptr, l2_operator ? h->pfrag.as<double>() : nullptr,
             l2_operator ? h->X.as<double>() : nullptr);
  if (is_l1) {
    ensure_mom(h, spec->max_iter);
    if (d_warm) {
      CSD_CUDA(cudaMemsetAsync(h->X.p, 0, sizeof(double) * V * Kp, st));
      CSD_CUDA(cudaMemcpy2DAsync(h->X.p, sizeof(double) * Kp, d_warm, sizeof(double) * K, sizeof(double) * K, V,
                                 cudaMemcpyDeviceToDevice, st));
    }
    csd::FistaParams fp{};
    fp.gfrag = h->gfrag.as<double>();
    fp.B = h->B.as<double>();
    fp.X = h->X.as<double>();
    fp.warm = d_warm ? h->X.as<double>() : nullptr;  // read at slot fill, before the slot's voxel is written
    fp.iters = h->iters.as<uint32_t>();
    fp.conv = h->conv.as<uint8_t>();
    fp.V = V;
    fp.n_inv = 1.0 / static_cast<double>(N);
    fp.step = 1.0 / h->lipschitz;
    fp.thr = fp.step * spec->alpha;
    fp.alpha_v = d_alpha;
    fp.tol = spec->tol;
    fp.max_iter = spec->max_iter;
    fp.non_negative = spec->non_negative;
    fp.queue = h->queue.as<unsigned long long>();
    fp.list = d_order;  // the order the persistent kernel takes voxels in (nullptr: 0 .. V-1)
    fp.n_work = V;
    CSD_CUDA(cudaMemsetAsync(h->queue.p, 0, sizeof(unsigned long long), st));
    if (d_order) {
      SchedOff single_pass(h);  // the caller's order replaces the two-pass schedule
      launch_fista(h, Kp / 8, fp);
    } else {
      launch_fista(h, Kp / 8, fp);
    }
    if (d_iters)
      CSD_CUDA(cudaMemcpyAsync(d_iters, h->iters.p, sizeof(uint32_t) * V, cudaMemcpyDeviceToDevice, st));
  } else {
    if (!l2_operator) launch_tikhonov(h, h->B.as<double>(), h->X.as<double>(), V);
    if (d_iters) {
      csd::k_fill_u32<<<grid1(V), 256, 0, st>>>(d_iters, V, 1u);
      CSD_LAUNCH();
    }
  }
  CSD_CUDA(cudaMemcpy2DAsync(d_coef, sizeof(double) * K, h->X.p, sizeof(double) * Kp, sizeof(double) * K, V,
                             cudaMemcpyDeviceToDevice, st));
}

// Shared memory per warp of the first L1 pass: supports of up to this many
// coefficients (larger ones go to the second pass).
constexpr int kAdjSmallCap = 40;

template <int RPL>
void launch_l1_adjoint_t(csd_handle* h, const csd::AdjointParams& p0) {
  cudaStream_t st = h->stream;
  csd::AdjointParams p = p0;
  // pass 1: every voxel, supports up to kAdjSmallCap in a small per-warp slice
  p.cap = std::min(p.K, kAdjSmallCap);
  p.list = nullptr;
  p.list_len = nullptr;
  {
    const size_t per_warp = sizeof(double) * static_cast<size_t>(csd::l1_adjoint_warp_doubles(p.cap, p.K));
    const int warps = 8;
    const size_t smem = per_warp * warps;
    CSD_CUDA(cudaFuncSetAttribute(csd::k_l1_adjoint<RPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(std::max(smem, per_warp * 8))));
    int per_sm = 0;
    CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_l1_adjoint<RPL>, 32 * warps, smem));
    const int64_t blocks = std::max<int64_t>(
        1, std::min<int64_t>((p.V + warps - 1) / warps, static_cast<int64_t>(h->num_sms) * std::max(per_sm, 1)));
    csd::k_l1_adjoint<RPL><<<static_cast<unsigned>(blocks), 32 * warps, smem, st>>>(p);
    CSD_LAUNCH();
  }
  if (p.cap >= p.K) return;
  // pass 2: the listed voxels with the full-size slice (count read on device)
  p.cap = p.K;
  p.list = p.overflow;
  p.list_len = p.n_overflow;
  p.overflow = nullptr;
  p.n_overflow = nullptr;
  const size_t per_warp = sizeof(double) * static_cast<size_t>(csd::l1_adjoint_warp_doubles(p.K, p.K));
  const int warps = static_cast<int>(std::min<size_t>(8, static_cast<size_t>(h->smem_optin) / per_warp));
  if (warps < 1) throw Error{CSD_ERR_INVALID, "coefficient count too large for the L1 adjoint"};
  const size_t smem = per_warp * warps;
  CSD_CUDA(cudaFuncSetAttribute(csd::k_l1_adjoint<RPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  csd::k_l1_adjoint<RPL><<<static_cast<unsigned>(h->num_sms), 32 * warps, smem, st>>>(p);
  CSD_LAUNCH();
}

void launch_apply64(csd_handle* h, const double* At, int rows, int cols, const double* in, int64_t ldin, int64_t V,
                    double* out, float* out32, int64_t ldout);

// H^{-1} (K x K, row k = H^{-1} e_k) for the current factor, by the factor's
// solves of the identity rows; kept until the factor changes.
void ensure_hinv(csd_handle* h) {
  if (h->hinv_valid && h->hinv_key == h->chol_key) return;
  const int K = h->K, Kp = h->Kp;
  cudaStream_t st = h->stream;
  h->ptmp.ensure(2 * sizeof(double) * static_cast<size_t>(K) * Kp);
  double* id = h->ptmp.as<double>();
  double* rows = id + static_cast<size_t>(K) * Kp;
  csd::k_identity_rows<<<(K * Kp + 255) / 256, 256, 0, st>>>(id, K, Kp);
  CSD_LAUNCH();
  launch_tikhonov(h, id, rows, K);
  h->hinv.ensure(sizeof(double) * static_cast<size_t>(K) * K);
  CSD_CUDA(cudaMemcpy2DAsync(h->hinv.p, sizeof(double) * K, rows, sizeof(double) * Kp, sizeof(double) * K, K,
                             cudaMemcpyDeviceToDevice, st));
  h->hinv_key = h->chol_key;
  h->hinv_valid = true;
}

// L2 adjoint: w = H^{-1} gc (the rows of H^{-1} are its columns, so they are
// the apply's transposed operand as they stand), then the hyper-parameter
// gradients from w and c.
template <int RPL>
void launch_l2_adjoint_t(csd_handle* h, const csd::AdjointParams& p) {
  ensure_hinv(h);
  launch_apply64(h, h->hinv.as<double>(), p.K, p.K, p.GC, p.ldg, p.V, p.W, nullptr, p.Kp);
  if (p.ghyper) {
    const int warps = 8;
    const int64_t blocks =
        std::max<int64_t>(1, std::min<int64_t>((p.V + warps - 1) / warps, static_cast<int64_t>(h->num_sms) * 8));
    csd::k_l2_hyper<RPL><<<static_cast<unsigned>(blocks), 32 * warps, 0, h->stream>>>(
        p.W, p.Kp, p.X, p.ldx, p.V, p.K, p.radial_order, p.ghyper);
    CSD_LAUNCH();
  }
}

template <template <int> class F>
void dispatch_rpl(int K, csd_handle* h, const csd::AdjointParams& p) {
  switch ((K + 31) / 32) {
    case 1: F<1>::run(h, p); break;
    case 2: F<2>::run(h, p); break;
    case 3: F<3>::run(h, p); break;
    case 4: F<4>::run(h, p); break;
    case 5: F<5>::run(h, p); break;
    default: throw Error{CSD_ERR_INVALID, "adjoint kernels support K <= 160"};
  }
}
template <int R>
struct L1Adj {
  static void run(csd_handle* h, const csd::AdjointParams& p) { launch_l1_adjoint_t<R>(h, p); }
};
template <int R>
struct L2Adj {
  static void run(csd_handle* h, const csd::AdjointParams& p) { launch_l2_adjoint_t<R>(h, p); }
};

void launch_apply64(csd_handle* h, const double* At, int rows, int cols, const double* in, int64_t ldin, int64_t V,
                    double* out, float* out32, int64_t ldout) {
  // tensor-core path when the matrix fits in one CTA's shared memory
  const size_t dmma_smem = sizeof(double) * 32 * static_cast<size_t>((rows + 7) / 8) * ((cols + 3) / 4);
  if (dmma_smem <= static_cast<size_t>(h->smem_optin)) {
    const int64_t groups = (V + 7) / 8;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((groups + 7) / 8, h->num_sms));
    auto go = [&](auto kern) {
      CSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dmma_smem)));
      kern<<<static_cast<unsigned>(blocks), 256, dmma_smem, h->stream>>>(At, rows, cols, in, ldin, V, out, out32,
                                                                         ldout);
      CSD_LAUNCH();
    };
    if ((cols + 3) / 4 <= csd::kApplyKtr)
      go(csd::k_apply_dmma<true>);
    else
      go(csd::k_apply_dmma<false>);
    return;
  }
  const size_t per_warp = sizeof(double) * 8 * static_cast<size_t>(cols);
  const int warps = static_cast<int>(std::max<size_t>(1, std::min<size_t>(8, (100u << 10) / per_warp)));
  const size_t smem = per_warp * warps;
  if (smem > static_cast<size_t>(h->smem_optin)) throw Error{CSD_ERR_INVALID, "matrix too wide to apply"};
  CSD_CUDA(cudaFuncSetAttribute(csd::k_apply64, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_apply64, 32 * warps, smem));
  const int64_t groups = (V + 7) / 8;
  const int64_t blocks = std::max<int64_t>(
      1, std::min<int64_t>((groups + warps - 1) / warps, static_cast<int64_t>(h->num_sms) * std::max(per_sm, 1)));
  csd::k_apply64<<<static_cast<unsigned>(blocks), 32 * warps, smem, h->stream>>>(At, rows, cols, in, ldin, V, out,
                                                                                 out32, ldout);
  CSD_LAUNCH();
}

// RTOP constants for (radial_order, zeta), built once and kept on the handle.
const csd::MicroConsts* micro_consts(csd_handle* h, int radial_order, double zeta) {
  if (radial_order < 0 || radial_order > csd::kMicroMaxN - 1 || radial_order % 2 != 0)
    throw Error{CSD_ERR_INVALID, "radial order must be even and at most 14 for the RTOP constants"};
  if (!(h->adjconst.p && h->adjconst_order == radial_order && h->adjconst_zeta == zeta)) {
    h->adjconst.ensure(sizeof(csd::MicroConsts));
    csd::k_micro_consts<<<1, 1, 0, h->stream>>>(radial_order, zeta, h->adjconst.as<csd::MicroConsts>());
    CSD_LAUNCH();
    h->adjconst_order = radial_order;
    h->adjconst_zeta = zeta;
  }
  return h->adjconst.as<csd::MicroConsts>();
}

}  // namespace

extern "C" {

int csd_geodesic_sphere(int32_t frequency, int32_t hemisphere, double* out, int32_t capacity) {
  if (frequency < 1 || frequency > 64) return -1;
  const SphereMesh m = geodesic_mesh(frequency);
  const std::vector<double> v = hemisphere ? m.hemisphere() : m.v;
  const int n = static_cast<int>(v.size() / 3);
  if (out && capacity >= n) std::memcpy(out, v.data(), sizeof(double) * v.size());
  return n;
}

int csd_shore_fit_batch_device(csd_handle* h, const float* d_signals, int64_t n_voxels, const csd_gtab* gtab,
                               const csd_shore_spec* spec, const double* d_alpha, const double* d_warm,
                               const int64_t* d_order, double* d_coef, uint32_t* d_iterations, void* stream,
                               char* err, size_t err_len) {
  if (!h || !gtab || !spec || n_voxels < 0 || (n_voxels > 0 && (!d_signals || !d_coef))) {
    set_err(err, err_len, "invalid argument: null pointer or negative voxel count");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    HostGtab g = make_gtab(gtab);
    std::string warnings;
    validate(spec, g, warnings);
    if (spec->regularization == CSD_REG_NONNEG)
      throw Error{CSD_ERR_INVALID, "the batch fit takes regularization l1 or l2"};
    if (spec->regularization == CSD_REG_L1 && spec->alpha_mode != CSD_ALPHA_FIXED)
      throw Error{CSD_ERR_INVALID, "the batch fit takes alpha_mode fixed (one alpha, or one per voxel)"};
    if (spec->precision == CSD_PRECISION_MIXED_KKT || spec->precision == CSD_PRECISION_FP64_KKT)
      throw Error{CSD_ERR_INVALID, "the batch fit takes precision fp64 or mixed"};
    StreamScope scope(h, stream);
    HandleOrder call_order(h);
    run_fit_batch(h, d_signals, n_voxels, g, spec, d_alpha, d_warm, d_order, d_coef, d_iterations);
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_fit_adjoint_device(csd_handle* h, const csd_gtab* gtab, const csd_shore_spec* spec,
                                 const double* d_coef, const double* d_grad_coef, int64_t n_voxels,
                                 float* d_grad_signal, double* d_grad_signal64, double* d_grad_hyper,
                                 uint64_t* d_n_singular, void* stream, char* err, size_t err_len) {
  if (!h || !gtab || !spec || n_voxels < 0 || (n_voxels > 0 && (!d_coef || !d_grad_coef))) {
    set_err(err, err_len, "invalid argument: null pointer or negative voxel count");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    HostGtab g = make_gtab(gtab);
    if (spec->regularization == CSD_REG_NONNEG)
      throw Error{CSD_ERR_INVALID, "the adjoint covers regularization l1 and l2"};
    StreamScope scope(h, stream);
    HandleOrder call_order(h);
    const bool is_l1 = spec->regularization == CSD_REG_L1;
    h->launches = 0;
    ensure_setup(h, g, spec->radial_order, spec->zeta, !is_l1, spec->lambda_n, spec->lambda_l);
    if (n_voxels == 0) return CSD_OK;
    const int N = h->N, K = h->K, Kp = h->Kp;
    h->adjW.ensure(sizeof(double) * static_cast<size_t>(n_voxels) * Kp);
    csd::AdjointParams p{};
    p.G = is_l1 ? h->G.as<double>() : h->A.as<double>();
    p.X = d_coef;
    p.ldx = K;
    p.GC = d_grad_coef;
    p.ldg = K;
    p.V = n_voxels;
    p.K = K;
    p.Kp = Kp;
    p.radial_order = spec->radial_order;
    p.n_samples = static_cast<double>(N);
    p.W = h->adjW.as<double>();
    p.ghyper = d_grad_hyper;
    p.n_singular = reinterpret_cast<unsigned long long*>(d_n_singular);
    if (is_l1) {
      h->adjovf.ensure(sizeof(int64_t) * static_cast<size_t>(n_voxels));
      h->adjstat.ensure(sizeof(unsigned long long));
      CSD_CUDA(cudaMemsetAsync(h->adjstat.p, 0, sizeof(unsigned long long), h->stream));
      p.overflow = h->adjovf.as<int64_t>();
      p.n_overflow = h->adjstat.as<unsigned long long>();
      dispatch_rpl<L1Adj>(K, h, p);
    } else {
      dispatch_rpl<L2Adj>(K, h, p);
    }
    if (d_grad_signal || d_grad_signal64)  // grad_s = M w
      launch_apply64(h, h->Mt.as<double>(), N, K, h->adjW.as<double>(), Kp, n_voxels, d_grad_signal64, d_grad_signal,
                     N);
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_apply_rows_device(csd_handle* h, const double* d_At, int32_t rows, int32_t cols, const double* d_in,
                          int64_t n_voxels, double* d_out, void* stream, char* err, size_t err_len) {
  if (!h || rows <= 0 || cols <= 0 || n_voxels < 0 || (n_voxels > 0 && (!d_At || !d_in || !d_out))) {
    set_err(err, err_len, "invalid argument: null pointer or bad shape");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    StreamScope scope(h, stream);
    HandleOrder call_order(h);
    h->launches = 0;
    if (n_voxels > 0) launch_apply64(h, d_At, rows, cols, d_in, cols, n_voxels, d_out, nullptr, rows);
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_odf_matrix(csd_handle* h, int32_t radial_order, double zeta, const double* dirs, int32_t n_dirs,
                         double* out, char* err, size_t err_len) {
  if (!h || !dirs || !out || n_dirs <= 0 || radial_order < 0 || radial_order % 2 != 0) {
    set_err(err, err_len, "invalid argument: null pointer, no directions or odd radial order");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    HandleOrder call_order(h);
    const int K = n_coeffs(radial_order);
    cudaStream_t st = h->stream;
    h->pdir.ensure(sizeof(double) * 3 * n_dirs);
    h->pmat.ensure(sizeof(double) * static_cast<size_t>(n_dirs) * K);
    CSD_CUDA(cudaMemcpyAsync(h->pdir.p, dirs, sizeof(double) * 3 * n_dirs, cudaMemcpyHostToDevice, st));
    h->launches = 0;
    csd::k_constraint<<<(n_dirs * K + 255) / 256, 256, 0, st>>>(h->pdir.as<double>(), n_dirs, K, radial_order, zeta,
                                                               h->pmat.as<double>());
    CSD_LAUNCH();
    CSD_CUDA(cudaMemcpyAsync(out, h->pmat.p, sizeof(double) * static_cast<size_t>(n_dirs) * K,
                             cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_rtop_device(csd_handle* h, int32_t radial_order, double zeta, const double* d_coef, int64_t n_voxels,
                          double* d_rtop, void* stream, char* err, size_t err_len) {
  if (!h || n_voxels < 0 || (n_voxels > 0 && (!d_coef || !d_rtop))) {
    set_err(err, err_len, "invalid argument: null pointer or negative voxel count");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    StreamScope scope(h, stream);
    HandleOrder call_order(h);
    h->launches = 0;
    const csd::MicroConsts* mc = micro_consts(h, radial_order, zeta);
    if (n_voxels > 0) {
      csd::k_rtop64<<<grid1(n_voxels), 256, 0, h->stream>>>(mc, d_coef, n_coeffs(radial_order), n_voxels, d_rtop);
      CSD_LAUNCH();
    }
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

int csd_shore_rtop_adjoint_device(csd_handle* h, int32_t radial_order, double zeta, const double* d_coef,
                                  int64_t n_voxels, const double* d_grad_rtop, double* d_grad_coef, void* stream,
                                  char* err, size_t err_len) {
  if (!h || n_voxels < 0 || (n_voxels > 0 && (!d_coef || !d_grad_rtop || !d_grad_coef))) {
    set_err(err, err_len, "invalid argument: null pointer or negative voxel count");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    StreamScope scope(h, stream);
    HandleOrder call_order(h);
    h->launches = 0;
    const csd::MicroConsts* mc = micro_consts(h, radial_order, zeta);
    const int K = n_coeffs(radial_order);
    if (n_voxels > 0) {
      csd::k_rtop64_adjoint<<<grid1(n_voxels), 256, 0, h->stream>>>(mc, d_coef, K, n_voxels, d_grad_rtop,
                                                                    d_grad_coef, K);
      CSD_LAUNCH();
    }
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}

}  // extern "C"
