// Host side of the per-voxel-design fit (gradient deviation, dropped
// samples).  Included once at the end of csd_shore.cu.
#pragma once

extern "C" int csd_shore_fit_graddev_device(csd_handle* h, const float* d_signals, int64_t n_voxels,
                                            const csd_gtab* gtab, const csd_shore_spec* spec,
                                            const double* d_graddev, const uint8_t* d_keep,
                                            const double* d_alpha, double* d_coef, uint32_t* d_iterations,
                                            uint8_t* d_converged, double* d_lipschitz, int32_t* d_n_rows,
                                            void* stream, char* err, size_t err_len) {
  if (!h || !gtab || !spec || n_voxels < 0 ||
      (n_voxels > 0 && (!d_signals || !d_coef || !d_iterations || !d_converged))) {
    set_err(err, err_len, "invalid argument: null pointer or negative voxel count");
    return CSD_ERR_INVALID;
  }
  try {
    CSD_CUDA(cudaSetDevice(h->device));
    HostGtab g = make_gtab(gtab);
    std::string warnings;
    if (spec->precision < CSD_PRECISION_FP64 || spec->precision > CSD_PRECISION_FP64_KKT)
      throw Error{CSD_ERR_INVALID, "unknown precision"};
    // the shared checks; the precisions this fit takes are checked below (its
    // converged-optimum mode also serves radial order 8)
    csd_shore_spec shared = *spec;
    shared.precision = CSD_PRECISION_FP64;
    validate(&shared, g, warnings);
    if (spec->regularization != CSD_REG_L1 || spec->alpha_mode != CSD_ALPHA_FIXED)
      throw Error{CSD_ERR_INVALID, "the per-voxel-design fit takes regularization l1 with alpha_mode fixed"};
    if (spec->radial_order != 6 && spec->radial_order != 8)
      throw Error{CSD_ERR_INVALID, "the per-voxel-design fit is built for radial orders 6 and 8"};
    if (spec->precision == CSD_PRECISION_MIXED)
      throw Error{CSD_ERR_INVALID, "the per-voxel-design fit takes precision fp64, fp64-kkt or mixed-kkt"};
    // converged-optimum modes: the polish and certificate are those of the
    // shared-design path.  Each voxel has its own Gram matrix, so there is no
    // shared tensor-core operand: "fp64-kkt" runs the support iterations in
    // FP64, "mixed-kkt" keeps G_v as FP32 planes hi + lo and runs the Lanczos
    // estimate and the support iterations in FP32 on hi (half the shared-memory
    // traffic of the products), the polish in FP64 on hi + lo
    const bool kkt = spec->precision == CSD_PRECISION_MIXED_KKT || spec->precision == CSD_PRECISION_FP64_KKT;
    StreamScope scope(h, stream);
    HandleOrder call_order(h);
    cudaStream_t st = h->stream;
    h->launches = 0;
    const int N = static_cast<int>(g.bvals.size());
    const int K = n_coeffs(spec->radial_order);
    const csd::GdLayout lay(K, spec->radial_order, N);
    if (lay.total_bytes + 64 > static_cast<size_t>(h->smem_optin))
      throw Error{CSD_ERR_INVALID, "gradient table too long for the per-voxel-design fit (shared memory)"};
    if (n_voxels == 0) return CSD_OK;
    // the table itself (not the per-table setup cache: the designs are per voxel)
    h->gdtab.ensure(sizeof(double) * 4 * static_cast<size_t>(N));
    CSD_CUDA(cudaMemcpyAsync(h->gdtab.p, g.bvals.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
    CSD_CUDA(cudaMemcpyAsync(h->gdtab.as<double>() + N, g.bvecs.data(), sizeof(double) * 3 * N,
                             cudaMemcpyHostToDevice, st));
    int kkt_iters = h->opt_kkt_iters > 0 ? h->opt_kkt_iters : 32;
    ensure_mom(h, std::max(spec->max_iter, 48));
    h->gdq.ensure(4 * sizeof(unsigned long long));
    CSD_CUDA(cudaMemsetAsync(h->gdq.p, 0, 4 * sizeof(unsigned long long), st));
    csd::GraddevParams p{};
    p.S = d_signals;
    p.T = d_graddev;
    p.keep = d_keep;
    p.bvals = h->gdtab.as<double>();
    p.bvecs = h->gdtab.as<double>() + N;
    p.N = N;
    p.K = K;
    p.radial_order = spec->radial_order;
    p.zeta = spec->zeta;
    p.qdenom = 4.0 * kPi * kPi * g.tau;  // src/qspace.rs:384-385
    p.b0_thr = g.b0;
    p.alpha = spec->alpha;
    p.alpha_v = d_alpha;
    p.tol = spec->tol;
    p.max_iter = spec->max_iter;
    p.non_negative = spec->non_negative;
    p.mom = h->mom.as<double>();
    p.V = n_voxels;
    p.queue = h->gdq.as<unsigned long long>();
    p.X = d_coef;
    p.iters = d_iterations;
    p.conv = d_converged;
    p.lipschitz = d_lipschitz;
    p.n_rows = d_n_rows;
    p.iter_total = h->gdq.as<unsigned long long>() + 1;
    p.kkt = kkt ? 1 : 0;
    p.mixed = spec->precision == CSD_PRECISION_MIXED_KKT ? 1 : 0;
    p.kkt_iters = kkt_iters;
    p.kkt_rounds = h->opt_kkt_rounds;
    p.kappa = kKktKappa;
    p.n_uncertified = h->gdq.as<unsigned long long>() + 2;
    p.round_total = h->gdq.as<unsigned long long>() + 3;
    auto go = [&](auto kern, const csd::GraddevParams& q) {
      CSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(lay.total_bytes)));
      const int grid = static_cast<int>(std::min<int64_t>(h->num_sms, q.V));
      kern<<<grid, 256, lay.total_bytes, st>>>(q);
      CSD_LAUNCH();
    };
    auto launch = [&](const csd::GraddevParams& q) {
      if (K == 72)
        go(csd::k_graddev_fit<9>, q);
      else
        go(csd::k_graddev_fit<19>, q);
    };
    // Autotuning of the certified modes' support-iteration count, once per
    // (table, radial order, mode): the whole fit of a prefix of this call's
    // own voxels (24 per SM: their deviation tensors and dropped samples are
    // what sets the cost) with 16, 24, 32 and 48 iterations, untimed and then
    // timed, and the fastest count serves this and later calls.  It runs only
    // for calls of at least four such prefixes (a smaller call takes 32 until
    // a larger one has tuned the table).  Every count ends at the certified
    // optimum, so the choice changes the time, not the result.
    float tune_ms[4] = {0.f, 0.f, 0.f, 0.f};
    if (kkt && h->opt_kkt_iters <= 0) {
      static constexpr int kCand[4] = {16, 24, 32, 48};
      uint64_t key = 1469598103934665603ull;
      key = fnv1a(key, g.bvals.data(), g.bvals.size() * sizeof(double));
      key = fnv1a(key, g.bvecs.data(), g.bvecs.size() * sizeof(double));
      const double sc[6] = {g.tau, g.b0, spec->zeta, static_cast<double>(spec->radial_order),
                            static_cast<double>(spec->precision), static_cast<double>(spec->non_negative)};
      key = fnv1a(key, sc, sizeof sc);
      const int64_t Vt = 24 * static_cast<int64_t>(h->num_sms);
      const auto hit = h->gd_tune_cache.find(key);
      if (hit != h->gd_tune_cache.end()) {
        kkt_iters = static_cast<int>(hit->second[0]);
        for (int i = 0; i < 4; ++i) tune_ms[i] = hit->second[1 + i];
      } else if (n_voxels >= 4 * Vt) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        CSD_CUDA(cudaEventCreate(&e0));
        CSD_CUDA(cudaEventCreate(&e1));
        csd::GraddevParams q = p;
        q.V = Vt;
        float best = 0.f;
        int best_k = 32;
        for (int c = 0; c < 4; ++c) {
          q.kkt_iters = kCand[c];
          float ms = 0.f;
          for (int pass = 0; pass < 2; ++pass) {
            CSD_CUDA(cudaMemsetAsync(h->gdq.p, 0, 4 * sizeof(unsigned long long), st));
            CSD_CUDA(cudaEventRecord(e0, st));
            launch(q);
            CSD_CUDA(cudaEventRecord(e1, st));
            CSD_CUDA(cudaEventSynchronize(e1));
            if (pass == 1 && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = 0.f;
          }
          tune_ms[c] = ms;
          if (ms > 0.f && (best == 0.f || ms < best)) {
            best = ms;
            best_k = kCand[c];
          }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        kkt_iters = best_k;
        h->gd_tune_cache[key] = {static_cast<float>(best_k), tune_ms[0], tune_ms[1], tune_ms[2], tune_ms[3]};
        CSD_CUDA(cudaMemsetAsync(h->gdq.p, 0, 4 * sizeof(unsigned long long), st));
      }
    }
    p.kkt_iters = kkt_iters;
    launch(p);
    if (kkt) {  // the certificate counters (this mode waits for its work)
      unsigned long long c[2] = {0, 0};
      CSD_CUDA(cudaMemcpyAsync(c, h->gdq.as<unsigned long long>() + 2, sizeof c, cudaMemcpyDeviceToHost, st));
      CSD_CUDA(cudaStreamSynchronize(st));
      h->timing.kkt_uncertified = static_cast<int64_t>(c[0]);
      h->timing.kkt_rounds = c[1];
      h->timing.kkt_iterations = kkt_iters;
      for (int i = 0; i < 4; ++i) h->timing.kkt_tune_ms[i] = tune_ms[i];
    }
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}
