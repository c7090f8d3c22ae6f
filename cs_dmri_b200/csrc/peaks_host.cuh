// Host side of the ODF maps: GFA and peaks of a coefficient volume on the
// hemisphere of a geodesic sphere.  Included once at the end of csd_shore.cu.
#pragma once

extern "C" int csd_shore_odf_peaks(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                                   int32_t radial_order, double zeta, const uint8_t* mask, int32_t sphere_frequency,
                                   int32_t npeaks, double relative_peak_threshold, double min_separation_angle_deg,
                                   float* gfa, float* peak_dirs, float* peak_values, float* peak_qa, char* err,
                                   size_t err_len) {
  const int64_t nvox = X * Y * Z;
  if (!h || ((!coefficients || !gfa || !peak_dirs || !peak_values || !peak_qa) && nvox > 0)) {
    set_err(err, err_len, "invalid argument");
    return CSD_ERR_INVALID;
  }
  try {
    check_coeff_args(X, Y, Z, radial_order);
    if (sphere_frequency < 1 || sphere_frequency > 10)
      throw Error{CSD_ERR_INVALID, "sphere_frequency must be in 1..10"};
    if (npeaks < 1 || npeaks > csd::kPeakMax)
      throw Error{CSD_ERR_INVALID, "npeaks must be in 1.." + std::to_string(csd::kPeakMax)};
    if (!(relative_peak_threshold >= 0.0 && relative_peak_threshold <= 1.0))
      throw Error{CSD_ERR_INVALID, "relative_peak_threshold must be in [0, 1]"};
    if (!(min_separation_angle_deg >= 0.0 && min_separation_angle_deg <= 90.0))
      throw Error{CSD_ERR_INVALID, "min_separation_angle must be in [0, 90] degrees"};
    CSD_CUDA(cudaSetDevice(h->device));
    HandleOrder call_order(h);
    cudaStream_t st = h->stream;
    h->launches = 0;
    const int K = n_coeffs(radial_order);
    std::fill(gfa, gfa + nvox, 0.0f);
    std::fill(peak_dirs, peak_dirs + nvox * npeaks * 3, 0.0f);
    std::fill(peak_values, peak_values + nvox * npeaks, 0.0f);
    std::fill(peak_qa, peak_qa + nvox * npeaks, 0.0f);
    if (nvox == 0) return CSD_OK;
    // hemisphere of the sampling sphere and its mesh, antipodes folded
    const SphereMesh m = geodesic_mesh(sphere_frequency);
    const std::vector<double> dirs = m.hemisphere();
    const int R = m.n_hemi;
    if (R > 32 * csd::kPeakMaxRows) throw Error{CSD_ERR_INVALID, "sphere too fine for the peak kernel"};
    std::vector<std::set<int>> adj(static_cast<size_t>(R));
    for (const auto& e : m.edges) {
      const int a = m.hemi_of[static_cast<size_t>(e[0])], b = m.hemi_of[static_cast<size_t>(e[1])];
      if (a < 0 || b < 0 || a == b) continue;
      adj[static_cast<size_t>(a)].insert(b);
      adj[static_cast<size_t>(b)].insert(a);
    }
    std::vector<int> off(static_cast<size_t>(R) + 1, 0), nb;
    for (int r = 0; r < R; ++r) {
      nb.insert(nb.end(), adj[static_cast<size_t>(r)].begin(), adj[static_cast<size_t>(r)].end());
      off[static_cast<size_t>(r) + 1] = static_cast<int>(nb.size());
    }
    // device buffers: directions, mesh, A (R x K) and its transpose
    h->pdir.ensure(sizeof(double) * dirs.size());
    h->pgv.ensure(sizeof(int) * (off.size() + nb.size()));
    h->pmat.ensure(sizeof(double) * static_cast<size_t>(R) * K);
    h->pgt.ensure(sizeof(double) * static_cast<size_t>(K) * R);
    CSD_CUDA(cudaMemcpyAsync(h->pdir.p, dirs.data(), sizeof(double) * dirs.size(), cudaMemcpyHostToDevice, st));
    CSD_CUDA(cudaMemcpyAsync(h->pgv.p, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, st));
    CSD_CUDA(cudaMemcpyAsync(h->pgv.as<int>() + off.size(), nb.data(), sizeof(int) * nb.size(),
                             cudaMemcpyHostToDevice, st));
    csd::k_constraint<<<(R * K + 255) / 256, 256, 0, st>>>(h->pdir.as<double>(), R, K, radial_order, zeta,
                                                          h->pmat.as<double>());
    CSD_LAUNCH();
    csd::k_transpose_design<<<(K * R + 255) / 256, 256, 0, st>>>(h->pmat.as<double>(), R, K, K, h->pgt.as<double>());
    CSD_LAUNCH();
    // masked voxels
    h->mask.ensure(nvox);
    if (mask) {
      CSD_CUDA(cudaMemcpyAsync(h->mask.p, mask, nvox, cudaMemcpyHostToDevice, st));
    } else {
      CSD_CUDA(cudaMemsetAsync(h->mask.p, 1, nvox, st));
    }
    const int64_t V = compact(h, h->mask.as<uint8_t>(), nvox, h->vox);
    if (V == 0) return CSD_OK;
    h->pcoef.ensure(sizeof(float) * nvox * K);
    CSD_CUDA(cudaMemcpyAsync(h->pcoef.p, coefficients, sizeof(float) * nvox * K, cudaMemcpyHostToDevice, st));
    const size_t per_v = static_cast<size_t>(1 + 3 * npeaks + 2 * npeaks);
    h->pout.ensure(sizeof(float) * per_v * V);
    float* o = h->pout.as<float>();
    csd::PeakParams pp{};
    pp.coeffs = h->pcoef.as<float>();
    pp.vox = h->vox.as<int64_t>();
    pp.V = V;
    pp.K = K;
    pp.R = R;
    pp.At = h->pgt.as<double>();
    pp.dirs = h->pdir.as<double>();
    pp.nb_off = h->pgv.as<int>();
    pp.nb = h->pgv.as<int>() + off.size();
    pp.npeaks = npeaks;
    pp.rel_thr = relative_peak_threshold;
    pp.cos_sep = std::cos(min_separation_angle_deg * kPi / 180.0);
    pp.gfa = o;
    pp.pdir = o + V;
    pp.pval = o + V + 3 * npeaks * V;
    pp.pqa = o + V + 4 * npeaks * V;
    // the amplitude matrix staged once per CTA when it fits next to the warp
    // slices (16 warps), else read through the caches (8 warps)
    const size_t at_bytes = sizeof(double) * static_cast<size_t>(K) * R;
    pp.at_in_smem = at_bytes + sizeof(double) * 16 * static_cast<size_t>(K + R) <= static_cast<size_t>(h->smem_optin);
    const int warps = pp.at_in_smem ? 16 : 8;
    const size_t smem = (pp.at_in_smem ? at_bytes : 0) + sizeof(double) * static_cast<size_t>(warps) * (K + R);
    CSD_CUDA(cudaFuncSetAttribute(csd::k_odf_peaks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    int per_sm = 0;
    CSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd::k_odf_peaks, 32 * warps, smem));
    const int64_t blocks =
        std::max<int64_t>(1, std::min<int64_t>((V + warps - 1) / warps, h->num_sms * std::max(per_sm, 1)));
    csd::k_odf_peaks<<<static_cast<unsigned>(blocks), 32 * warps, smem, st>>>(pp);
    CSD_LAUNCH();
    std::vector<float> hs(per_v * static_cast<size_t>(V));
    std::vector<int64_t> vox(static_cast<size_t>(V));
    CSD_CUDA(cudaMemcpyAsync(hs.data(), o, sizeof(float) * hs.size(), cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaMemcpyAsync(vox.data(), h->vox.p, sizeof(int64_t) * V, cudaMemcpyDeviceToHost, st));
    CSD_CUDA(cudaStreamSynchronize(st));
    const float* hg = hs.data();
    const float* hd = hg + V;
    const float* hv = hd + 3 * npeaks * V;
    const float* hq = hv + npeaks * V;
    for (int64_t i = 0; i < V; ++i) {
      const int64_t x = vox[static_cast<size_t>(i)];
      gfa[x] = hg[i];
      std::memcpy(peak_dirs + x * npeaks * 3, hd + i * npeaks * 3, sizeof(float) * 3 * npeaks);
      std::memcpy(peak_values + x * npeaks, hv + i * npeaks, sizeof(float) * npeaks);
      std::memcpy(peak_qa + x * npeaks, hq + i * npeaks, sizeof(float) * npeaks);
    }
  } catch (const Error& e) {
    set_err(err, err_len, e.msg);
    return e.code;
  }
  return CSD_OK;
}
