// solve_cube.cpp -- the reference's call chain on the n^3 Kuhn-split cube,
// written against the C++ adapters (include/emagddm_b200.hpp) the way a
// reference caller would write it:
//   GlobalEdgeIDGenerator -> EMDOFManager::build/applyTreeGauge
//   -> GpuEMAssembly::assemble -> GpuCGSolver::set_matrix/solve,
// or (--direct) the GPU direct backend on the same gauged system.  --hex keeps
// the hexes as HEX8_EDGE elements; --wiggle moves every interior node by
// 0.2 h sin(...) per coordinate (a deterministic non-affine geometry) and
// --xyz writes the node coordinates used.
// Usage: solve_cube <n> [--numbering-only] [--direct] [--hex] [--wiggle] [--av]
//                       [--x out.bin] [--xyz out.bin]
// Prints one line of key=value pairs.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "emagddm_b200.hpp"

int main(int argc, char** argv) {
  const int n = argc > 1 ? std::atoi(argv[1]) : 4;
  bool numbering_only = false, direct = false, hex = false, wiggle = false, av = false;
  const char* xout = nullptr;
  const char* xyzout = nullptr;
  for (int i = 2; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--numbering-only")) numbering_only = true;
    if (!std::strcmp(argv[i], "--direct")) direct = true;
    if (!std::strcmp(argv[i], "--hex")) hex = true;
    if (!std::strcmp(argv[i], "--wiggle")) wiggle = true;
    if (!std::strcmp(argv[i], "--av")) av = true;
    if (!std::strcmp(argv[i], "--x") && i + 1 < argc) xout = argv[++i];
    if (!std::strcmp(argv[i], "--xyz") && i + 1 < argc) xyzout = argv[++i];
  }
  const int n1 = n + 1;
  std::vector<double> xyz;
  for (int k = 0; k < n1; ++k)
    for (int j = 0; j < n1; ++j)
      for (int i = 0; i < n1; ++i) {
        const bool interior = i > 0 && i < n && j > 0 && j < n && k > 0 && k < n;
        const double h = 0.2 / n, w = wiggle && interior ? 1.0 : 0.0;
        xyz.push_back(double(i) / n + w * h * std::sin(1.3 * i + 2.1 * j + 0.7 * k));
        xyz.push_back(double(j) / n + w * h * std::sin(0.4 * i + 1.7 * j + 2.9 * k));
        xyz.push_back(double(k) / n + w * h * std::sin(2.3 * i + 0.9 * j + 1.1 * k));
      }
  if (xyzout) {
    FILE* f = std::fopen(xyzout, "wb");
    if (f) {
      std::fwrite(xyz.data(), sizeof(double), xyz.size(), f);
      std::fclose(f);
    }
  }
  auto gid = [&](int i, int j, int k) { return i + n1 * (j + n1 * k); };
  const int kuhn[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  std::vector<int32_t> tets;
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        if (hex) {
          for (auto& o : off) tets.push_back(gid(i + o[0], j + o[1], k + o[2]));
          continue;
        }
        for (auto& t : kuhn)
          for (int a = 0; a < 4; ++a) {
            const int* o = off[t[a]];
            tets.push_back(gid(i + o[0], j + o[1], k + o[2]));
          }
      }
  // Dirichlet: every element edge lying in a boundary face (duplicates are fine)
  const int ge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  const int he[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  const int npe = hex ? 8 : 4, epe = hex ? 12 : 6;
  std::vector<int32_t> dir;
  auto coord = [&](int g, int c) { return c == 0 ? g % n1 : c == 1 ? (g / n1) % n1 : g / (n1 * n1); };
  for (size_t t = 0; t < tets.size() / npe; ++t)
    for (int q = 0; q < epe; ++q) {
      const int* e = hex ? he[q] : ge[q];
      const int a = tets[npe * t + e[0]], b = tets[npe * t + e[1]];
      for (int c = 0; c < 3; ++c)
        if (coord(a, c) == coord(b, c) && (coord(a, c) == 0 || coord(a, c) == n)) {
          dir.push_back(a);
          dir.push_back(b);
          break;
        }
    }
  emg::Mesh mesh(xyz, tets, std::vector<int32_t>(tets.size() / npe, 0), dir, 0,
                 hex ? EMG_ELEM_HEX8_EDGE : EMG_ELEM_TET4_EDGE);
  emg::GlobalEdgeIDGenerator gen(mesh);
  gen.generate();
  emg::EMDOFManager dofs(mesh);
  dofs.build();
  const int n_free = dofs.getNumFreeDOFs();
  dofs.applyTreeGauge(EMG_GAUGE_REF);
  long long l2g_sum = 0;
  for (int32_t v : dofs.getElemLocalToGlobal()) l2g_sum += v;
  std::printf("n=%d edges=%d free=%d dofs=%d l2g_sum=%lld", n, gen.getNumGlobalEdges(), n_free,
              dofs.getNumFreeDOFs(), l2g_sum);
  if (av) {
    // element DOF types SCALAR_ONLY / VECTOR_EDGE_ONLY / MIXED_AV in turn,
    // scalar Dirichlet on every boundary node
    std::vector<int32_t> types, phi;
    for (size_t t = 0; t < tets.size() / npe; ++t) types.push_back(static_cast<int32_t>(t % 3));
    for (int g = 0; g < n1 * n1 * n1; ++g)
      for (int c = 0; c < 3; ++c)
        if (coord(g, c) == 0 || coord(g, c) == n) { phi.push_back(g); break; }
    emg::EMDOFManager av_dofs(mesh);
    const auto rows = av_dofs.buildWithDofTypes(types, phi, EMG_GAUGE_REF);
    long long av_sum = 0, av_len = 0;
    for (const auto& r : rows)
      for (int32_t v : r) { av_sum += v; ++av_len; }
    std::printf(" av_dofs=%d av_scalar=%d av_sum=%lld av_len=%lld", av_dofs.getNumFreeDOFs(),
                av_dofs.getNumScalarFreeDOFs(), av_sum, av_len);
  }
  if (numbering_only) {
    std::printf("\n");
    return 0;
  }
  // nu = 1, J = (0,0,1) in the central box [0.375, 0.625]^3
  emg_source box{};
  box.kind = EMG_SRC_BOX;
  box.j[2] = 1.0;
  const double p[6] = {0.375, 0.625, 0.375, 0.625, 0.375, 0.625};
  std::memcpy(box.p, p, sizeof(p));
  if (direct) {
    emg::GpuDirectBackend ds(mesh, dofs);
    if (!ds.factor({1.0}, {0.0}, {box})) {
      std::printf(" factor_error=\"%s\"\n", ds.error_message().c_str());
      return 2;
    }
    const emg::SolverResult r = ds.solve({}, 1e-12, 6);
    double norm = 0.0;
    for (double v : r.x) norm += v * v;
    std::printf(" solver=%s status=%d residual=%.3e xnorm=%.12e\n", emg::GpuDirectBackend::name(),
                static_cast<int>(r.status), r.residual_norm, std::sqrt(norm));
    if (xout) {
      FILE* f = std::fopen(xout, "wb");
      if (f) {
        std::fwrite(r.x.data(), sizeof(double), r.x.size(), f);
        std::fclose(f);
      }
    }
    return r.status == emg::SolverStatus::SUCCESS ? 0 : 1;
  }
  emg::GpuEMAssembly as;
  if (!as.assemble(mesh, dofs.getElemLocalToGlobal(), {1.0}, {0.0}, {box})) {
    std::printf(" assemble_error=\"%s\"\n", as.error_message().c_str());
    return 2;
  }
  emg::GpuCGSolver cg(1e-10, 10000, /*jacobi=*/true);
  cg.set_matrix(as.getStiffnessMatrix());
  const emg::SolverResult r = cg.solve(as.getSourceVector());
  double norm = 0.0;
  for (double v : r.x) norm += v * v;
  std::printf(" solver=%s status=%d iterations=%d residual=%.3e xnorm=%.12e\n", cg.get_solver_name().c_str(),
              static_cast<int>(r.status), r.iterations, r.residual_norm, std::sqrt(norm));
  if (xout) {
    FILE* f = std::fopen(xout, "wb");
    if (f) {
      std::fwrite(r.x.data(), sizeof(double), r.x.size(), f);
      std::fclose(f);
    }
  }
  return r.status == emg::SolverStatus::SUCCESS ? 0 : 1;
}
