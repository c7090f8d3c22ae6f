// Sampling sphere for ODFs: a class I geodesic icosphere with its mesh.
// Included once at the end of csd_shore.cu.
#pragma once

namespace {

// Class I geodesic sphere of frequency f: every face of the icosahedron split
// into f^2 triangles on a flat barycentric grid, the grid points projected on
// the unit sphere, shared edge points kept once (first-seen order): 10 f^2 + 2
// vertices, 362 at f = 6.  `edges` are the sides of the small triangles.
// The vertex set is antipodally symmetric (the icosahedron is); `hemi_of[i]`
// maps vertex i to its index in the hemisphere (one vertex of each antipodal
// pair: z > 0, or z = 0 and y > 0, or z = y = 0 and x > 0).
struct SphereMesh {
  std::vector<double> v;                 // n x 3
  std::vector<std::array<int, 2>> edges;
  std::vector<int> hemi_of;              // n
  int n_hemi = 0;
  std::vector<double> hemisphere() const {
    std::vector<double> out(3 * static_cast<size_t>(n_hemi));
    for (size_t i = 0; i < hemi_of.size(); ++i)
      if (hemi_of[i] >= 0 && is_upper(i))
        for (int d = 0; d < 3; ++d) out[3 * hemi_of[i] + d] = v[3 * i + d];
    return out;
  }
  bool is_upper(size_t i) const {
    const double e = 1e-12, x = v[3 * i], y = v[3 * i + 1], z = v[3 * i + 2];
    return (z > e) || (std::fabs(z) <= e && y > e) || (std::fabs(z) <= e && std::fabs(y) <= e && x > 0.0);
  }
};

SphereMesh geodesic_mesh(int f) {
  const double ph = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<std::array<double, 3>> ico = {{-1, ph, 0}, {1, ph, 0},   {-1, -ph, 0}, {1, -ph, 0},
                                            {0, -1, ph}, {0, 1, ph},   {0, -1, -ph}, {0, 1, -ph},
                                            {ph, 0, -1}, {ph, 0, 1},   {-ph, 0, -1}, {-ph, 0, 1}};
  for (auto& a : ico) {
    const double n = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (auto& c : a) c /= n;
  }
  const int faces[20][3] = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                            {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                            {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                            {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
  SphereMesh m;
  std::map<std::array<long long, 3>, int> id_of;
  auto key = [](const std::array<double, 3>& p) {
    return std::array<long long, 3>{std::llround(p[0] * 1e9), std::llround(p[1] * 1e9), std::llround(p[2] * 1e9)};
  };
  std::set<std::pair<int, int>> edge_set;
  std::vector<int> grid(static_cast<size_t>((f + 1) * (f + 1)));
  for (const auto& t : faces) {
    for (int i = 0; i <= f; ++i)
      for (int j = 0; i + j <= f; ++j) {
        const double wa = static_cast<double>(f - i - j) / f, wb = static_cast<double>(i) / f,
                     wc = static_cast<double>(j) / f;
        std::array<double, 3> p;
        for (int d = 0; d < 3; ++d) p[d] = wa * ico[t[0]][d] + wb * ico[t[1]][d] + wc * ico[t[2]][d];
        const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        for (auto& c : p) c /= n;
        const auto k = key(p);
        auto it = id_of.find(k);
        int id;
        if (it == id_of.end()) {
          id = static_cast<int>(m.v.size() / 3);
          id_of[k] = id;
          m.v.insert(m.v.end(), p.begin(), p.end());
        } else {
          id = it->second;
        }
        grid[static_cast<size_t>(i * (f + 1) + j)] = id;
      }
    auto at = [&](int i, int j) { return grid[static_cast<size_t>(i * (f + 1) + j)]; };
    auto add = [&](int a, int b) { edge_set.insert({std::min(a, b), std::max(a, b)}); };
    for (int i = 0; i < f; ++i)
      for (int j = 0; i + j < f; ++j) {
        add(at(i, j), at(i + 1, j));
        add(at(i, j), at(i, j + 1));
        add(at(i + 1, j), at(i, j + 1));
      }
  }
  for (const auto& e : edge_set) m.edges.push_back({e.first, e.second});
  const int n = static_cast<int>(m.v.size() / 3);
  m.hemi_of.assign(static_cast<size_t>(n), -1);
  int h = 0;
  for (int i = 0; i < n; ++i)
    if (m.is_upper(static_cast<size_t>(i))) m.hemi_of[static_cast<size_t>(i)] = h++;
  m.n_hemi = h;
  for (int i = 0; i < n; ++i) {
    if (m.hemi_of[static_cast<size_t>(i)] >= 0) continue;
    const std::array<double, 3> q = {-m.v[3 * i], -m.v[3 * i + 1], -m.v[3 * i + 2]};
    const auto it = id_of.find(key(q));
    if (it != id_of.end()) m.hemi_of[static_cast<size_t>(i)] = m.hemi_of[static_cast<size_t>(it->second)];
  }
  return m;
}

}  // namespace
