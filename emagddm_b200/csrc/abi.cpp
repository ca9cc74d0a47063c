// abi.cpp -- the extern "C" entry points declared in include/emagddm_b200.h.
// Handles wrap host C++ objects (numbering) and device objects (assembly,
// CSR, Krylov workspaces).  No exception crosses the ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "device.h"
#include "tune.h"
#include "fetidp_dev.h"
#include "internal.h"
#include "trace.h"

struct emg_mesh_t {
  emg::Mesh m;
  std::vector<int32_t> material_tags;  // physical tag of each material id (Gmsh input)
};
struct emg_dofmap_t {
  emg::DofMap d;
};
struct emg_csr_t {
  emg::DevCsr* csr = nullptr;
  bool owned = true;
};
struct emg_fetidp_t {
  emg::FetiDP fd;
};
struct emg_direct_t {
  emg::FetiDP fd;  // one subdomain: nested dissection + multifrontal Cholesky
};
struct emg_system_t {
  emg::System s;
  emg_csr_t k_handle, m_handle;
};

namespace emg {
namespace {
thread_local std::string g_error;
}
void set_error(const std::string& msg) { g_error = msg; }
}  // namespace emg

namespace {

using emg::set_error;

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return EMG_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_error(e.what());
    return EMG_ERR_INTERNAL;
  } catch (...) {
    set_error("unknown exception");
    return EMG_ERR_INTERNAL;
  }
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

template <class T>
int upload(T** dst, const T* src, int64_t count, bool src_on_device, cudaStream_t st) {
  size_t bytes = sizeof(T) * static_cast<size_t>(count > 0 ? count : 1);
  EMG_CK(cudaMallocAsync(reinterpret_cast<void**>(dst), bytes, st));
  if (count > 0 && src)
    EMG_CK(cudaMemcpyAsync(*dst, src, sizeof(T) * count,
                           src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  return EMG_SUCCESS;
}

int system_create_impl(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_elems,
                       const int32_t* elems, const int32_t* material, const int32_t* l2g, int64_t n_dofs,
                       void* stream, emg_system* out, bool on_device) {
  if (!out) { set_error("null output handle"); return EMG_INVALID_INPUT; }
  *out = nullptr;
  if (!emg::valid_elem_type(elem_type)) { set_error("unknown element type"); return EMG_INVALID_INPUT; }
  const int npe = emg::nodes_per_elem(elem_type), epe = emg::edges_per_elem(elem_type);
  if (n_nodes <= 0 || n_elems <= 0 || !xyz || !elems || !l2g) {
    set_error("mesh is empty");  // em_assembly.cpp:154-166
    return EMG_INVALID_INPUT;
  }
  if (n_dofs <= 0) {
    // matrix dimension = largest equation index + 1 (em_assembly.cpp:190-215)
    std::vector<int32_t> h;
    const int32_t* src = l2g;
    if (on_device) {
      h.resize(epe * n_elems);
      EMG_CK(cudaMemcpy(h.data(), l2g, sizeof(int32_t) * epe * n_elems, cudaMemcpyDeviceToHost));
      src = h.data();
    }
    int64_t mx = -1;
    for (int64_t i = 0; i < epe * n_elems; ++i) mx = std::max<int64_t>(mx, src[i]);
    n_dofs = mx + 1;
    if (n_dofs <= 0) { set_error("no free DOF (all constrained)"); return EMG_INVALID_INPUT; }
  }
  emg::keep_pool_memory();
  auto* h = new emg_system_t();
  emg::System& s = h->s;
  cudaStream_t st = as_stream(stream);
  s.elem_type = elem_type;
  s.n_nodes = n_nodes;
  s.n_elems = n_elems;
  s.n = n_dofs;
  int rc = EMG_SUCCESS;
  if (!rc) rc = upload(&s.xyz, xyz, 3 * n_nodes, on_device, st);
  if (!rc) rc = upload(&s.elems, elems, npe * n_elems, on_device, st);
  if (!rc) rc = upload(&s.l2g, l2g, epe * n_elems, on_device, st);
  if (!rc) {
    rc = upload(&s.material, material, n_elems, on_device, st);
    if (!rc && !material) {
      cudaError_t e = cudaMemsetAsync(s.material, 0, sizeof(int32_t) * n_elems, st);
      if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); rc = EMG_ERR_CUDA; }
    }
  }
  if (!rc) {
    cudaError_t e = cudaMallocAsync(&s.err, sizeof(int32_t), st);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); rc = EMG_ERR_CUDA; }
  }
  if (!rc) {
    emg::trace_mark(st, "create.upload");
    emg::TraceScope t("system_create.build");
    rc = emg::system_build(s, st);
  }
  if (rc) { delete h; return rc; }
  h->k_handle.csr = &s.K;
  h->k_handle.owned = false;
  h->m_handle.csr = &s.M;
  h->m_handle.owned = false;
  *out = h;
  return EMG_SUCCESS;
}

int csr_from_device(int64_t n, int64_t nnz, const int32_t* rp, const int32_t* col,
                    const double* val, bool src_dev, cudaStream_t st, emg_csr* out) {
  auto* h = new emg_csr_t();
  h->csr = new emg::DevCsr();
  emg::DevCsr& A = *h->csr;
  A.n = n;
  A.nnz = nnz;
  emg::keep_pool_memory();
  int rc = upload(&A.row_ptr, rp, n + 1, src_dev, st);
  if (!rc) rc = upload(&A.col, col, nnz, src_dev, st);
  if (!rc) rc = upload(&A.val, val, nnz, src_dev, st);
  if (!rc && src_dev) rc = emg::check_csr(n, A.row_ptr, A.col, nnz, st);
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); rc = EMG_ERR_CUDA; }
  }
  if (rc) { delete h->csr; delete h; return rc; }
  *out = h;
  return EMG_SUCCESS;
}

void feti_info(const emg::FetiPlan& p, int64_t* info, int32_t n) {
  int64_t v[22] = {0};
  v[0] = p.n_parts;
  v[1] = p.n_dofs;
  v[2] = p.n_union;
  v[3] = p.n_lambda;
  v[4] = p.n_coarse;
  v[5] = static_cast<int64_t>(p.fronts.size());
  v[6] = static_cast<int64_t>(p.level_ptr.size()) - 1;
  v[7] = p.max_front;
  v[8] = p.max_npiv;
  v[9] = p.fac_size;
  v[10] = p.upd_pool;
  v[11] = p.root_off.empty() ? 0 : p.root_off.back();
  for (int32_t s = 0; s < p.n_parts; ++s) {
    v[12] += p.nI[s];
    v[13] += p.nD[s];
    v[14] += p.nP[s];
    v[15] = std::max<int64_t>(v[15], p.nD[s]);
  }
  v[16] = p.max_children;
  // flops of the numeric phase: partial Cholesky of the fronts (panel part,
  // rank-npiv update of the update block), inverse factors of S_DD and the
  // three deluxe products per face
  double panel = 0.0, syrk = 0.0, other = 0.0;
  for (const emg::FetiFront& f : p.fronts) {
    const double np = f.npiv, nu = f.f - f.npiv;
    panel += np * np * np / 3.0 + nu * np * np;
    syrk += nu * nu * np;
  }
  for (int32_t s = 0; s < p.n_parts; ++s) other += static_cast<double>(p.nD[s]) * p.nD[s] * p.nD[s] / 3.0;
  for (int32_t f = 0; f < p.n_faces; ++f) {
    const double m = static_cast<double>(p.face_ptr[f + 1] - p.face_ptr[f]);
    other += 6.0 * m * m * m + m * m * m / 3.0 + m * m * m / 3.0;
  }
  v[17] = static_cast<int64_t>(panel);
  v[18] = static_cast<int64_t>(syrk);
  v[19] = static_cast<int64_t>(other);
  // entries of the S_DD blocks the symmetric products read (the 64 x 64
  // tiles on and below the diagonal) and of the deluxe face blocks (one of
  // each face's four n_F x n_F blocks)
  for (int32_t s = 0; s < p.n_parts; ++s) {
    const int64_t n = p.nD[s], nb = (n + 63) / 64;
    for (int64_t I = 0; I < nb; ++I)
      for (int64_t J = 0; J <= I; ++J) v[20] += std::min<int64_t>(64, n - 64 * I) * std::min<int64_t>(64, n - 64 * J);
  }
  for (int32_t f = 0; f < p.n_faces; ++f) {
    const int64_t m = p.face_ptr[f + 1] - p.face_ptr[f];
    v[21] += m * m;
  }
  for (int32_t i = 0; i < n && i < 22; ++i) info[i] = v[i];
}

// A DOF map viewed as one subdomain (the direct solver's plan).
emg::DofMap single_part(const emg::DofMap& d) {
  emg::DofMap s = d;
  s.n_parts = 1;
  s.tet_part.assign(d.n_elems, 0);
  s.dof_primal.assign(d.n_dofs, 0);
  s.n_primal_fix = 0;
  return s;
}

}  // namespace

extern "C" {

int32_t emg_abi_version(void) { return EMG_ABI_VERSION; }

const char* emg_last_error(void) { return emg::g_error.c_str(); }

int emg_mesh_create(int64_t n_nodes, const double* xyz, int64_t n_tets, const int32_t* tets,
                    const int32_t* material_id, int64_t n_dirichlet,
                    const int32_t* dirichlet_pairs, int32_t n_hole_markers, emg_mesh* out) {
  return emg_mesh_create_typed(EMG_ELEM_TET4_EDGE, n_nodes, xyz, n_tets, tets, material_id, n_dirichlet,
                               dirichlet_pairs, n_hole_markers, out);
}

int emg_mesh_create_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_elems,
                          const int32_t* elems, const int32_t* material_id, int64_t n_dirichlet,
                          const int32_t* dirichlet_pairs, int32_t n_hole_markers, emg_mesh* out) {
  return guarded([&]() -> int {
    if (!out) { set_error("null output handle"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    if (!emg::valid_elem_type(elem_type)) { set_error("unknown element type"); return EMG_INVALID_INPUT; }
    const int npe = emg::nodes_per_elem(elem_type);
    if (n_nodes <= 0 || n_elems <= 0 || !elems) { set_error("mesh is empty"); return EMG_INVALID_INPUT; }
    if (n_dirichlet < 0 || (n_dirichlet > 0 && !dirichlet_pairs)) {
      set_error("bad Dirichlet pair list");
      return EMG_INVALID_INPUT;
    }
    for (int64_t t = 0; t < n_elems; ++t)
      if (!emg::valid_row(elem_type, elems + npe * t, n_nodes)) {
        set_error("element " + std::to_string(t) + ": node index out of range or unknown element type");  // em_assembly.cpp:603-608
        return EMG_INVALID_INPUT;
      }
    auto* h = new emg_mesh_t();
    emg::Mesh& m = h->m;
    m.elem_type = elem_type;
    m.n_nodes = n_nodes;
    m.n_elems = n_elems;
    if (xyz) m.xyz.assign(xyz, xyz + 3 * n_nodes);
    m.elems.assign(elems, elems + npe * n_elems);
    if (material_id) m.material.assign(material_id, material_id + n_elems);
    else m.material.assign(n_elems, 0);
    if (n_dirichlet > 0) m.dirichlet.assign(dirichlet_pairs, dirichlet_pairs + 2 * n_dirichlet);
    m.n_hole_markers = n_hole_markers > 0 ? n_hole_markers : 0;
    *out = h;
    return EMG_SUCCESS;
  });
}

int emg_mesh_elem_type(emg_mesh mesh, int32_t* elem_type, int32_t* nodes_per_elem, int32_t* edges_per_elem) {
  if (!mesh) { set_error("null mesh"); return EMG_INVALID_INPUT; }
  if (elem_type) *elem_type = mesh->m.elem_type;
  if (nodes_per_elem) *nodes_per_elem = mesh->m.npe();
  if (edges_per_elem) *edges_per_elem = mesh->m.epe();
  return EMG_SUCCESS;
}

void emg_mesh_destroy(emg_mesh mesh) { delete mesh; }

int emg_mesh_read_gmsh(const char* path, const int32_t* dirichlet_tags, int32_t n_tags, emg_mesh* out) {
  return guarded([&]() -> int {
    if (!path || !out || n_tags < 0 || (n_tags > 0 && !dirichlet_tags)) {
      set_error("bad argument");
      return EMG_INVALID_INPUT;
    }
    *out = nullptr;
    auto* h = new emg_mesh_t();
    int rc = emg::read_gmsh(path, dirichlet_tags, n_tags, h->m, h->material_tags);
    if (rc) { delete h; return rc; }
    *out = h;
    return EMG_SUCCESS;
  });
}

int emg_mesh_info(emg_mesh mesh, int64_t* n_nodes, int64_t* n_elems, int64_t* n_dirichlet, int32_t* n_materials) {
  if (!mesh) { set_error("null mesh"); return EMG_INVALID_INPUT; }
  const emg::Mesh& m = mesh->m;
  if (n_nodes) *n_nodes = m.n_nodes;
  if (n_elems) *n_elems = m.n_elems;
  if (n_dirichlet) *n_dirichlet = static_cast<int64_t>(m.dirichlet.size() / 2);
  if (n_materials) {
    int32_t mx = -1;
    for (int32_t v : m.material) mx = std::max(mx, v);
    *n_materials = mx + 1;
  }
  return EMG_SUCCESS;
}

int emg_mesh_export(emg_mesh mesh, double* xyz, int32_t* tets, int32_t* material, int32_t* dirichlet_pairs) {
  if (!mesh) { set_error("null mesh"); return EMG_INVALID_INPUT; }
  const emg::Mesh& m = mesh->m;
  if (xyz && !m.xyz.empty()) std::memcpy(xyz, m.xyz.data(), sizeof(double) * m.xyz.size());
  if (tets) std::memcpy(tets, m.elems.data(), sizeof(int32_t) * m.elems.size());
  if (material) std::memcpy(material, m.material.data(), sizeof(int32_t) * m.material.size());
  if (dirichlet_pairs && !m.dirichlet.empty())
    std::memcpy(dirichlet_pairs, m.dirichlet.data(), sizeof(int32_t) * m.dirichlet.size());
  return EMG_SUCCESS;
}

int emg_mesh_material_tags(emg_mesh mesh, int32_t* tags) {
  if (!mesh) { set_error("null mesh"); return EMG_INVALID_INPUT; }
  if (tags && !mesh->material_tags.empty())
    std::memcpy(tags, mesh->material_tags.data(), sizeof(int32_t) * mesh->material_tags.size());
  return EMG_SUCCESS;
}

int emg_edge_ids(emg_mesh mesh, int32_t* elem_edge, int32_t* edge_nodes, int64_t* n_edges) {
  return guarded([&]() -> int {
    if (!mesh) { set_error("null mesh"); return EMG_INVALID_INPUT; }
    int rc = emg::build_edge_ids(mesh->m);
    if (rc) return rc;
    if (n_edges) *n_edges = mesh->m.n_edges;
    if (elem_edge) std::memcpy(elem_edge, mesh->m.elem_edge.data(), sizeof(int32_t) * mesh->m.elem_edge.size());
    if (edge_nodes) std::memcpy(edge_nodes, mesh->m.edge_nodes.data(), sizeof(int32_t) * mesh->m.edge_nodes.size());
    return EMG_SUCCESS;
  });
}

int emg_dof_build(emg_mesh mesh, int32_t gauge_mode, emg_dofmap* out) {
  return guarded([&]() -> int {
    if (!mesh || !out) { set_error("null handle"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    auto* h = new emg_dofmap_t();
    int rc = emg::build_dofmap(mesh->m, gauge_mode, h->d);
    if (rc) { delete h; return rc; }
    *out = h;
    return EMG_SUCCESS;
  });
}

int emg_dof_build_av(emg_mesh mesh, const int32_t* dof_type, int64_t n_scalar_dirichlet,
                     const int32_t* scalar_dirichlet, int32_t gauge_mode, int32_t* l2g,
                     int64_t* n_scalar_free, int64_t* n_free, int64_t* n_dofs) {
  return guarded([&]() -> int {
    if (!mesh) { set_error("null handle"); return EMG_INVALID_INPUT; }
    if (mesh->m.elem_type == EMG_ELEM_MIXED) { set_error("emg_dof_build_av: mixed-type meshes are numbered, assembled and solved by the Krylov solvers only"); return EMG_INVALID_INPUT; }
    std::vector<int32_t> rows;
    int64_t ns = 0, nf = 0, nd = 0;
    int rc = emg::build_dofmap_av(mesh->m, dof_type, n_scalar_dirichlet, scalar_dirichlet, gauge_mode, rows,
                                  ns, nf, nd);
    if (rc) return rc;
    if (l2g && !rows.empty()) std::memcpy(l2g, rows.data(), sizeof(int32_t) * rows.size());
    if (n_scalar_free) *n_scalar_free = ns;
    if (n_free) *n_free = nf;
    if (n_dofs) *n_dofs = nd;
    return EMG_SUCCESS;
  });
}

int emg_dof_build_device(int32_t elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* elems,
                         int64_t n_dir, const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge_mode,
                         int32_t* l2g, int64_t* n_edges, int64_t* n_free, int64_t* n_dofs, void* stream) {
  return guarded([&]() -> int {
    emg::keep_pool_memory();
    return emg::dof_build_gpu(elem_type, n_nodes, n_elems, elems, n_dir, dir_pairs, n_hole_markers, gauge_mode, l2g,
                              n_edges, n_free, n_dofs, as_stream(stream));
  });
}

int emg_dofmap_info(emg_dofmap map, int64_t* n_edges, int64_t* n_free, int64_t* n_dofs) {
  if (!map) { set_error("null dofmap"); return EMG_INVALID_INPUT; }
  if (n_edges) *n_edges = map->d.n_edges;
  if (n_free) *n_free = map->d.n_free;
  if (n_dofs) *n_dofs = map->d.n_dofs;
  return EMG_SUCCESS;
}

int emg_dofmap_export(emg_dofmap map, int32_t* l2g, int32_t* edge_dof) {
  if (!map) { set_error("null dofmap"); return EMG_INVALID_INPUT; }
  if (l2g) std::memcpy(l2g, map->d.l2g.data(), sizeof(int32_t) * map->d.l2g.size());
  if (edge_dof) std::memcpy(edge_dof, map->d.edge_dof.data(), sizeof(int32_t) * map->d.edge_dof.size());
  return EMG_SUCCESS;
}

int emg_dofmap_expand(emg_dofmap map, const double* reduced, double* full) {
  if (!map || !reduced || !full) { set_error("null argument"); return EMG_INVALID_INPUT; }
  for (int64_t e = 0; e < map->d.n_edges; ++e) {
    int32_t k = map->d.edge_dof[e];
    full[e] = k >= 0 ? reduced[k] : 0.0;
  }
  return EMG_SUCCESS;
}

void emg_dofmap_destroy(emg_dofmap map) { delete map; }

int emg_dof_build_partitioned(emg_mesh mesh, const int32_t* tet_part, int32_t n_parts,
                              emg_dofmap* out) {
  return guarded([&]() -> int {
    if (!mesh || !out) { set_error("null handle"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    auto* h = new emg_dofmap_t();
    int rc = emg::build_dofmap_partitioned(mesh->m, tet_part, n_parts, h->d);
    if (rc) { delete h; return rc; }
    *out = h;
    return EMG_SUCCESS;
  });
}

int emg_dofmap_partition_info(emg_dofmap map, int32_t* n_parts, int64_t* n_primal,
                              int64_t* n_primal_fix, int32_t* primal) {
  if (!map) { set_error("null dofmap"); return EMG_INVALID_INPUT; }
  const emg::DofMap& d = map->d;
  if (d.n_parts < 1) { set_error("dofmap has no partition"); return EMG_INVALID_INPUT; }
  if (n_parts) *n_parts = d.n_parts;
  int64_t np = 0;
  for (uint8_t f : d.dof_primal) np += f;
  if (n_primal) *n_primal = np;
  if (n_primal_fix) *n_primal_fix = d.n_primal_fix;
  if (primal)
    for (int64_t k = 0; k < d.n_dofs; ++k) primal[k] = d.dof_primal[k];
  return EMG_SUCCESS;
}

int emg_system_create(int64_t n_nodes, const double* xyz, int64_t n_tets, const int32_t* tets,
                      const int32_t* material, const int32_t* l2g, int64_t n_dofs, void* stream,
                      emg_system* out) {
  return guarded([&]() -> int {
    return system_create_impl(EMG_ELEM_TET4_EDGE, n_nodes, xyz, n_tets, tets, material, l2g, n_dofs, stream,
                              out, false);
  });
}

int emg_system_create_device(int64_t n_nodes, const double* xyz_d, int64_t n_tets,
                             const int32_t* tets_d, const int32_t* material_d,
                             const int32_t* l2g_d, int64_t n_dofs, void* stream, emg_system* out) {
  return guarded([&]() -> int {
    return system_create_impl(EMG_ELEM_TET4_EDGE, n_nodes, xyz_d, n_tets, tets_d, material_d, l2g_d, n_dofs,
                              stream, out, true);
  });
}

int emg_system_create_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_elems,
                            const int32_t* elems, const int32_t* material, const int32_t* l2g,
                            int64_t n_dofs, int32_t on_device, void* stream, emg_system* out) {
  return guarded([&]() -> int {
    return system_create_impl(elem_type, n_nodes, xyz, n_elems, elems, material, l2g, n_dofs, stream, out,
                              on_device != 0);
  });
}

int emg_system_assemble(emg_system sys, const double* nu, const double* sigma, int32_t n_materials,
                        const emg_source* sources, int32_t n_sources, int32_t flags, void* stream) {
  return guarded([&]() -> int {
    if (!sys) { set_error("null system"); return EMG_INVALID_INPUT; }
    return emg::system_assemble(sys->s, nu, sigma, n_materials, sources, n_sources, flags, as_stream(stream));
  });
}

int emg_system_set_source_map(emg_system sys, const int32_t* tet_source) {
  return guarded([&]() -> int {
    if (!sys) { set_error("null system"); return EMG_INVALID_INPUT; }
    emg::System& s = sys->s;
    if (s.src_map) { EMG_CK(cudaFreeAsync(s.src_map, 0)); s.src_map = nullptr; }
    if (!tet_source) return EMG_SUCCESS;
    EMG_CK(cudaMallocAsync(&s.src_map, sizeof(int32_t) * s.n_elems, 0));
    EMG_CK(cudaMemcpyAsync(s.src_map, tet_source, sizeof(int32_t) * s.n_elems, cudaMemcpyHostToDevice, 0));
    EMG_CK(cudaStreamSynchronize(0));
    return EMG_SUCCESS;
  });
}

int emg_system_info(emg_system sys, int64_t* n_rows, int64_t* nnz) {
  if (!sys) { set_error("null system"); return EMG_INVALID_INPUT; }
  if (n_rows) *n_rows = sys->s.n;
  if (nnz) *nnz = sys->s.K.nnz;
  return EMG_SUCCESS;
}

int emg_system_export(emg_system sys, int32_t* row_ptr, int32_t* col, double* kval, double* mval,
                      double* rhs) {
  return guarded([&]() -> int {
    if (!sys) { set_error("null system"); return EMG_INVALID_INPUT; }
    const emg::System& s = sys->s;
    if (row_ptr) EMG_CK(cudaMemcpy(row_ptr, s.K.row_ptr, sizeof(int32_t) * (s.n + 1), cudaMemcpyDeviceToHost));
    if (col) EMG_CK(cudaMemcpy(col, s.K.col, sizeof(int32_t) * s.K.nnz, cudaMemcpyDeviceToHost));
    if (kval) EMG_CK(cudaMemcpy(kval, s.K.val, sizeof(double) * s.K.nnz, cudaMemcpyDeviceToHost));
    if (mval) {
      if (!s.M.val) { set_error("mass matrix was not assembled"); return EMG_INVALID_INPUT; }
      EMG_CK(cudaMemcpy(mval, s.M.val, sizeof(double) * s.K.nnz, cudaMemcpyDeviceToHost));
    }
    if (rhs) EMG_CK(cudaMemcpy(rhs, s.rhs, sizeof(double) * s.n, cudaMemcpyDeviceToHost));
    return EMG_SUCCESS;
  });
}

int emg_system_combine(emg_system sys, double alpha, double beta, emg_csr* out) {
  return guarded([&]() -> int {
    if (!sys || !out) { set_error("null argument"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    const emg::System& s = sys->s;
    if (!s.M.val) { set_error("mass matrix was not assembled (EMG_FLAG_MASS)"); return EMG_INVALID_INPUT; }
    emg_csr h = nullptr;
    int rc = csr_from_device(s.n, s.K.nnz, s.K.row_ptr, s.K.col, s.K.val, true, nullptr, &h);
    if (rc) return rc;
    rc = emg::axpby_values(h->csr->val, alpha, s.K.val, beta, s.M.val, s.K.nnz, nullptr);
    if (rc) { emg_csr_destroy(h); return rc; }
    *out = h;
    return EMG_SUCCESS;
  });
}

emg_csr emg_system_matrix(emg_system sys, int32_t which) {
  if (!sys) return nullptr;
  if (which == 1) return sys->s.M.val ? &sys->m_handle : nullptr;
  return &sys->k_handle;
}

const double* emg_system_rhs_device(emg_system sys) { return sys ? sys->s.rhs : nullptr; }

void emg_system_destroy(emg_system sys) {
  if (!sys) return;
  emg::TraceScope t("emg_system_destroy");
  {
    emg::TraceScope t2("emg_system_destroy.sync");
    cudaDeviceSynchronize();
  }
  delete sys;
  // The destructors return their buffers with cudaFreeAsync on the legacy
  // stream; waiting for those frees here lets the next allocations reuse the
  // memory at once.  Without it a following create / solve now and then
  // stalled for 0.1-0.9 s inside CUDA calls on B200 (measured).
  cudaStreamSynchronize(0);
}

int emg_csr_create(int64_t n, const int32_t* row_ptr, const int32_t* col, const double* val,
                   void* stream, emg_csr* out) {
  return guarded([&]() -> int {
    if (!out) { set_error("null output handle"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    if (n <= 0 || !row_ptr || !col || !val) { set_error("empty matrix"); return EMG_INVALID_INPUT; }
    if (row_ptr[0] != 0) { set_error("row_ptr[0] != 0"); return EMG_INVALID_INPUT; }
    for (int64_t i = 0; i < n; ++i)
      if (row_ptr[i + 1] < row_ptr[i]) { set_error("row_ptr not monotone"); return EMG_INVALID_INPUT; }
    // Merge duplicates and sort columns per row, as SparseConverter::to_eigen
    // (setFromTriplets) does before the reference solvers see the matrix.
    std::vector<int32_t> rp(n + 1, 0), cc;
    std::vector<double> vv;
    cc.reserve(row_ptr[n]);
    vv.reserve(row_ptr[n]);
    std::vector<std::pair<int32_t, double>> row;
    for (int64_t i = 0; i < n; ++i) {
      row.clear();
      for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
        if (col[k] < 0 || col[k] >= n) { set_error("column index out of range"); return EMG_INVALID_INPUT; }
        row.emplace_back(col[k], val[k]);
      }
      std::stable_sort(row.begin(), row.end(),
                       [](const auto& a, const auto& b) { return a.first < b.first; });
      for (size_t k = 0; k < row.size(); ++k) {
        if (k > 0 && row[k].first == row[k - 1].first) vv.back() += row[k].second;
        else { cc.push_back(row[k].first); vv.push_back(row[k].second); }
      }
      rp[i + 1] = static_cast<int32_t>(cc.size());
    }
    return csr_from_device(n, static_cast<int64_t>(cc.size()), rp.data(), cc.data(), vv.data(), false,
                           as_stream(stream), out);
  });
}

int emg_csr_create_device(int64_t n, int64_t nnz, const int32_t* row_ptr_d, const int32_t* col_d,
                          const double* val_d, void* stream, emg_csr* out) {
  return guarded([&]() -> int {
    if (!out) { set_error("null output handle"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    if (n <= 0 || nnz < 0 || !row_ptr_d || !col_d || !val_d) { set_error("empty matrix"); return EMG_INVALID_INPUT; }
    return csr_from_device(n, nnz, row_ptr_d, col_d, val_d, true, as_stream(stream), out);
  });
}

int emg_csr_info(emg_csr A, int64_t* n, int64_t* nnz) {
  if (!A || !A->csr) { set_error("null matrix"); return EMG_INVALID_INPUT; }
  if (n) *n = A->csr->n;
  if (nnz) *nnz = A->csr->nnz;
  return EMG_SUCCESS;
}

void emg_csr_destroy(emg_csr A) {
  if (!A || !A->owned) return;  // borrowed handles belong to their system
  cudaDeviceSynchronize();
  delete A->csr;
  delete A;
  cudaStreamSynchronize(0);  // the frees above complete before the caller allocates again
}

int emg_spmv(emg_csr A, const double* x_d, double* y_d, void* stream) {
  return guarded([&]() -> int {
    if (!A || !A->csr) { set_error("null matrix"); return EMG_INVALID_INPUT; }
    return emg::csr_spmv(*A->csr, x_d, y_d, as_stream(stream));
  });
}

namespace {
int solve_host(emg_csr A, const double* b, double* x, const emg_krylov_config* cfg, emg_result* out,
               bool bicg) {
  return guarded([&]() -> int {
    emg_result dummy;
    if (!out) out = &dummy;
    std::memset(out, 0, sizeof(*out));
    out->status = EMG_INVALID_INPUT;
    if (!A || !A->csr || !cfg || !b || !x) { set_error("null argument"); return EMG_INVALID_INPUT; }
    const int64_t n = A->csr->n;
    // Stream-ordered buffers from the same pool as the solver's workspace
    // (a plain cudaMalloc cannot reuse memory that pool keeps reserved).
    double *bd = nullptr, *xd = nullptr;
    EMG_CK(cudaMallocAsync(&bd, sizeof(double) * n, 0));
    if (cudaError_t e = cudaMallocAsync(&xd, sizeof(double) * n, 0); e != cudaSuccess) {
      cudaFreeAsync(bd, 0);
      EMG_CK(e);
    }
    int rc = EMG_SUCCESS;
    if (cudaError_t e = cudaMemcpyAsync(bd, b, sizeof(double) * n, cudaMemcpyHostToDevice, 0);
        e != cudaSuccess) {
      set_error(cudaGetErrorString(e));
      rc = EMG_ERR_CUDA;
    }
    if (rc == EMG_SUCCESS)
      rc = bicg ? emg::bicgstab_solve(*A->csr, bd, xd, *cfg, nullptr, out)
                : emg::cg_solve(*A->csr, bd, xd, *cfg, nullptr, out);
    if (rc == EMG_SUCCESS || rc == EMG_NUMERICAL_ERROR || rc == EMG_DIVERGED || rc == EMG_MAX_ITER_REACHED) {
      if (cudaError_t e = cudaMemcpy(x, xd, sizeof(double) * n, cudaMemcpyDeviceToHost); e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        rc = EMG_ERR_CUDA;
      }
    }
    cudaFreeAsync(bd, 0);
    cudaFreeAsync(xd, 0);
    cudaStreamSynchronize(0);
    return rc;
  });
}
int solve_device(emg_csr A, const double* b, double* x, const emg_krylov_config* cfg, void* stream,
                 emg_result* out, bool bicg) {
  return guarded([&]() -> int {
    emg_result dummy;
    if (!out) out = &dummy;
    std::memset(out, 0, sizeof(*out));
    out->status = EMG_INVALID_INPUT;
    if (!A || !A->csr || !cfg) { set_error("null argument"); return EMG_INVALID_INPUT; }
    return bicg ? emg::bicgstab_solve(*A->csr, b, x, *cfg, as_stream(stream), out)
                : emg::cg_solve(*A->csr, b, x, *cfg, as_stream(stream), out);
  });
}
}  // namespace

int emg_cg_solve(emg_csr A, const double* b, double* x, const emg_krylov_config* cfg, emg_result* out) {
  return solve_host(A, b, x, cfg, out, false);
}
int emg_cg_solve_device(emg_csr A, const double* b_d, double* x_d, const emg_krylov_config* cfg,
                        void* stream, emg_result* out) {
  return solve_device(A, b_d, x_d, cfg, stream, out, false);
}
int emg_bicgstab_solve(emg_csr A, const double* b, double* x, const emg_krylov_config* cfg,
                       emg_result* out) {
  return solve_host(A, b, x, cfg, out, true);
}
int emg_bicgstab_solve_device(emg_csr A, const double* b_d, double* x_d, const emg_krylov_config* cfg,
                              void* stream, emg_result* out) {
  return solve_device(A, b_d, x_d, cfg, stream, out, true);
}

int emg_system_solve(emg_system sys, int32_t kind, const emg_krylov_config* cfg, double* x,
                     int32_t x_on_device, void* stream, emg_result* out) {
  return guarded([&]() -> int {
    emg_result dummy;
    if (!out) out = &dummy;
    std::memset(out, 0, sizeof(*out));
    out->status = EMG_INVALID_INPUT;
    if (!sys || !cfg || !x) { set_error("null argument"); return EMG_INVALID_INPUT; }
    emg::System& s = sys->s;
    cudaStream_t st = as_stream(stream);
    double* xd = x;
    if (!x_on_device) EMG_CK(cudaMallocAsync(&xd, sizeof(double) * s.n, st));
    int rc = kind == 1 ? emg::bicgstab_solve(s.K, s.rhs, xd, *cfg, st, out)
                       : emg::cg_solve(s.K, s.rhs, xd, *cfg, st, out);
    if (!x_on_device) {
      if (rc <= EMG_MAX_ITER_REACHED)
        EMG_CK(cudaMemcpyAsync(x, xd, sizeof(double) * s.n, cudaMemcpyDeviceToHost, st));
      EMG_CK(cudaFreeAsync(xd, st));
      EMG_CK(cudaStreamSynchronize(st));
    }
    return rc;
  });
}

int emg_cg_kernel_times(emg_csr A, int32_t iterations, void* stream, double* ms) {
  return guarded([&]() -> int {
    if (!A || !A->csr) { set_error("null matrix"); return EMG_INVALID_INPUT; }
    return emg::cg_kernel_times(*A->csr, iterations, as_stream(stream), ms);
  });
}

int emg_test_tc_tile(int32_t mr, int32_t mc, int32_t k, const double* a_d, int64_t lda, const double* b_d,
                     int64_t ldb, double* c_d, int64_t ldc, void* stream) {
  return guarded([&]() -> int { return emg::tc_tile_test(mr, mc, k, a_d, lda, b_d, ldb, c_d, ldc, as_stream(stream)); });
}

struct emg_aedt_t {
  emg::AedtProject p;
};

namespace {
void copy_str(const std::string& s, char* buf, int32_t cap) {
  if (!buf || cap <= 0) return;
  const size_t n = std::min<size_t>(s.size(), static_cast<size_t>(cap - 1));
  std::memcpy(buf, s.data(), n);
  buf[n] = '\0';
}
}  // namespace

int emg_aedt_read(const char* path, emg_aedt* out) {
  return guarded([&]() -> int {
    if (!path || !out) { set_error("null argument"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    auto* h = new emg_aedt_t();
    const int rc = emg::aedt_read(path, h->p);
    if (rc) { delete h; return rc; }
    *out = h;
    return EMG_SUCCESS;
  });
}

int emg_aedt_info(emg_aedt a, int32_t* n_materials, int32_t* n_objects, int32_t* n_boundaries) {
  if (!a) { set_error("null AEDT handle"); return EMG_INVALID_INPUT; }
  if (n_materials) *n_materials = static_cast<int32_t>(a->p.materials.size());
  if (n_objects) *n_objects = static_cast<int32_t>(a->p.objects.size());
  if (n_boundaries) *n_boundaries = static_cast<int32_t>(a->p.boundaries.size());
  return EMG_SUCCESS;
}

int emg_aedt_material(emg_aedt a, int32_t k, char* name, int32_t cap, double* mu_r, double* sigma,
                      int32_t* flags, int32_t* n_bh) {
  if (!a || k < 0 || k >= static_cast<int32_t>(a->p.materials.size())) {
    set_error("AEDT material index out of range");
    return EMG_INVALID_INPUT;
  }
  const auto& m = a->p.materials[k];
  copy_str(m.name, name, cap);
  if (mu_r) *mu_r = m.mu_r;
  if (sigma) *sigma = m.sigma;
  if (flags) *flags = m.flags;
  if (n_bh) *n_bh = static_cast<int32_t>(m.h.size());
  return EMG_SUCCESS;
}

int emg_aedt_bh_curve(emg_aedt a, int32_t k, double* h, double* b, int32_t cap) {
  if (!a || k < 0 || k >= static_cast<int32_t>(a->p.materials.size())) {
    set_error("AEDT material index out of range");
    return EMG_INVALID_INPUT;
  }
  const auto& m = a->p.materials[k];
  for (int32_t i = 0; i < cap && i < static_cast<int32_t>(m.h.size()); ++i) {
    if (h) h[i] = m.h[i];
    if (b) b[i] = m.b[i];
  }
  return EMG_SUCCESS;
}

int emg_aedt_object(emg_aedt a, int32_t k, char* name, int32_t cap, char* material, int32_t mcap,
                    int32_t* solve_inside) {
  if (!a || k < 0 || k >= static_cast<int32_t>(a->p.objects.size())) {
    set_error("AEDT object index out of range");
    return EMG_INVALID_INPUT;
  }
  const auto& o = a->p.objects[k];
  copy_str(o.name, name, cap);
  copy_str(o.material, material, mcap);
  if (solve_inside) *solve_inside = o.solve_inside;
  return EMG_SUCCESS;
}

int emg_aedt_boundary(emg_aedt a, int32_t k, char* name, int32_t cap, char* type, int32_t tcap, char* value,
                      int32_t vcap) {
  if (!a || k < 0 || k >= static_cast<int32_t>(a->p.boundaries.size())) {
    set_error("AEDT boundary index out of range");
    return EMG_INVALID_INPUT;
  }
  const auto& b = a->p.boundaries[k];
  copy_str(b.name, name, cap);
  copy_str(b.type, type, tcap);
  copy_str(b.value, value, vcap);
  return EMG_SUCCESS;
}

void emg_aedt_destroy(emg_aedt a) { delete a; }

int emg_tune_enable(int32_t on) {
  emg::tune::set_enabled(on != 0);
  return EMG_SUCCESS;
}

int32_t emg_tune_report(char* buf, int32_t cap) {
  const std::string r = emg::tune::report();
  if (buf && cap > 0) {
    const size_t n = std::min<size_t>(r.size(), static_cast<size_t>(cap - 1));
    std::memcpy(buf, r.data(), n);
    buf[n] = '\0';
  }
  return static_cast<int32_t>(r.size() + 1);
}

int emg_test_set_barrier_spins(int32_t spins) {
  return guarded([&]() -> int { return emg::set_barrier_spins(spins); });
}

int emg_batch_cg_solve_device(emg_csr A, int32_t n_blocks, const int64_t* block_row_ptr,
                              const double* b_d, double* x_d, const emg_krylov_config* cfg,
                              void* stream, emg_result* results) {
  return guarded([&]() -> int {
    if (!A || !A->csr || !cfg) { set_error("null argument"); return EMG_INVALID_INPUT; }
    return emg::batch_cg_solve(*A->csr, n_blocks, block_row_ptr, b_d, x_d, *cfg, as_stream(stream),
                               results);
  });
}

int emg_cg_solve_noalloc(int64_t n, int64_t nnz, const int32_t* row_ptr_d, const int32_t* col_d,
                         const double* val_d, const double* b_d, double* x_d,
                         const emg_krylov_config* cfg, void* stream, emg_result* out) {
  return guarded([&]() -> int {
    emg_result dummy;
    if (!out) out = &dummy;
    std::memset(out, 0, sizeof(*out));
    out->status = EMG_INVALID_INPUT;
    if (!cfg) { set_error("emg_cg_solve_noalloc: null config"); return EMG_INVALID_INPUT; }
    return emg::cg_solve_noalloc(n, nnz, row_ptr_d, col_d, val_d, b_d, x_d, *cfg, as_stream(stream), out);
  });
}

int emg_csr_solver_format(emg_csr A, int64_t* slots, int64_t* slices) {
  if (!A || !A->csr) { set_error("null matrix"); return EMG_INVALID_INPUT; }
  if (slots) *slots = emg::sell_slots(*A->csr);
  if (slices) *slices = emg::sell_slices(*A->csr);
  return EMG_SUCCESS;
}

int emg_last_history(emg_csr A, double* residuals, int32_t cap) {
  if (!A || !A->csr || !residuals || cap <= 0) return 0;
  int n = emg::csr_history(*A->csr, residuals, cap);
  return n < 0 ? 0 : n;
}

int emg_fetidp_plan_info(emg_mesh mesh, emg_dofmap map, int64_t* info, int32_t n_info) {
  return guarded([&]() -> int {
    if (!mesh || !map || (!info && n_info > 0)) { set_error("null argument"); return EMG_INVALID_INPUT; }
    emg::FetiPlan p;
    int rc = map->d.n_parts < 1 ? emg::build_feti_plan(mesh->m, single_part(map->d), p)
                                : emg::build_feti_plan(mesh->m, map->d, p);
    if (rc) return rc;
    feti_info(p, info, n_info);
    return EMG_SUCCESS;
  });
}

int emg_fetidp_create(emg_mesh mesh, emg_dofmap map, void* stream, emg_fetidp* out) {
  return guarded([&]() -> int {
    if (!mesh || !map || !out) { set_error("null argument"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    emg::keep_pool_memory();
    auto* h = new emg_fetidp_t();
    int rc = h->fd.create(mesh->m, map->d, as_stream(stream));
    if (rc) { delete h; return rc; }
    *out = h;
    return EMG_SUCCESS;
  });
}

int emg_fetidp_factor(emg_fetidp fd, const double* nu, const double* sigma, int32_t n_materials,
                      const emg_source* sources, int32_t n_sources, int32_t flags) {
  return guarded([&]() -> int {
    if (!fd) { set_error("null FETI-DP handle"); return EMG_INVALID_INPUT; }
    return fd->fd.factor(nu, sigma, n_materials, sources, n_sources, flags);
  });
}

namespace {
int fetidp_solve_impl(emg::FetiDP* fp, const emg_krylov_config* cfg, const double* b, double* x, int32_t on_device,
                      emg_result* out) {
  if (!fp || !cfg) { set_error("null argument"); return EMG_INVALID_INPUT; }
  if (cfg->max_iterations < 0 || !(cfg->tolerance > 0.0)) {
    set_error("bad tolerance or iteration limit");
    return EMG_INVALID_INPUT;
  }
  emg::FetiDP& F = *fp;
  const int64_t n = F.plan.n_dofs;
  const double* bd = nullptr;
  if (b) {
    if (on_device) bd = b;
    else {
      cudaError_t e = cudaMemcpyAsync(F.rglob_d, b, sizeof(double) * n, cudaMemcpyHostToDevice, F.st);
      if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return EMG_ERR_CUDA; }
      bd = F.rglob_d;  // copied into the solver's own right-hand side before use
    }
  }
  emg_result r{};
  int rc = F.solve(*cfg, bd, on_device ? x : nullptr, &r);
  if (rc == EMG_SUCCESS || rc == EMG_MAX_ITER_REACHED || rc == EMG_NUMERICAL_ERROR) {
    if (x && !on_device) {
      cudaError_t e = cudaMemcpy(x, F.xacc_d, sizeof(double) * n, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return EMG_ERR_CUDA; }
    }
    if (out) *out = r;
  }
  return rc;
}
}  // namespace

int emg_fetidp_solve(emg_fetidp fd, const emg_krylov_config* cfg, double* x, int32_t x_on_device,
                     emg_result* out) {
  return guarded([&]() -> int { return fetidp_solve_impl(fd ? &fd->fd : nullptr, cfg, nullptr, x, x_on_device, out); });
}

int emg_fetidp_solve_rhs(emg_fetidp fd, const emg_krylov_config* cfg, const double* b, double* x,
                         int32_t on_device, emg_result* out) {
  return guarded([&]() -> int {
    if (!b) { set_error("null right-hand side"); return EMG_INVALID_INPUT; }
    return fetidp_solve_impl(fd ? &fd->fd : nullptr, cfg, b, x, on_device, out);
  });
}

int emg_fetidp_info(emg_fetidp fd, int64_t* info, int32_t n_info) {
  if (!fd || (!info && n_info > 0)) { set_error("null argument"); return EMG_INVALID_INPUT; }
  feti_info(fd->fd.plan, info, n_info);
  return EMG_SUCCESS;
}

int emg_fetidp_stats(emg_fetidp fd, double* stats, int32_t n_stats) {
  if (!fd || (!stats && n_stats > 0)) { set_error("null argument"); return EMG_INVALID_INPUT; }
  const emg::FetiStats& s = fd->fd.stats;
  const double v[8] = {s.factor_ms, s.solve_ms, static_cast<double>(s.iterations), s.lambda_residual, s.residual,
                       static_cast<double>(s.refinements), s.lambda_ms, s.fronts_ms};
  for (int32_t i = 0; i < n_stats && i < 8; ++i) stats[i] = v[i];
  return EMG_SUCCESS;
}

void emg_fetidp_destroy(emg_fetidp fd) { delete fd; }

int emg_fetidp_learned_init(emg_fetidp fd, uint64_t seed) {
  return guarded([&]() -> int {
    if (!fd) { set_error("null FETI-DP handle"); return EMG_INVALID_INPUT; }
    return emg::learned_init(fd->fd, seed);
  });
}

int emg_fetidp_learned_train(emg_fetidp fd, int32_t batch, const double* r_d, const double* t_d, float lr,
                             double* loss) {
  return guarded([&]() -> int {
    if (!fd || !r_d || !t_d) { set_error("null argument"); return EMG_INVALID_INPUT; }
    return emg::learned_train(fd->fd, batch, r_d, t_d, lr, loss);
  });
}

int emg_fetidp_learned_params(emg_fetidp fd, float* params, int64_t* n, int32_t load) {
  return guarded([&]() -> int {
    if (!fd) { set_error("null FETI-DP handle"); return EMG_INVALID_INPUT; }
    return emg::learned_params(fd->fd, params, n, load);
  });
}

int emg_fetidp_apply(emg_fetidp fd, int32_t op, const double* in_d, double* out_d) {
  return guarded([&]() -> int {
    if (!fd || !in_d || !out_d) { set_error("null argument"); return EMG_INVALID_INPUT; }
    return fd->fd.apply_op(op, in_d, out_d);
  });
}

int emg_fetidp_duals(emg_fetidp fd, int64_t* dual_off, int32_t* dual_lam, int32_t* dual_sign, int32_t* lam_entry) {
  if (!fd) { set_error("null FETI-DP handle"); return EMG_INVALID_INPUT; }
  const emg::FetiPlan& p = fd->fd.plan;
  if (dual_off) std::memcpy(dual_off, p.dual_off.data(), sizeof(int64_t) * p.dual_off.size());
  if (dual_lam && !p.dual_lam.empty()) std::memcpy(dual_lam, p.dual_lam.data(), sizeof(int32_t) * p.dual_lam.size());
  if (dual_sign && !p.dual_sign.empty())
    std::memcpy(dual_sign, p.dual_sign.data(), sizeof(int32_t) * p.dual_sign.size());
  if (lam_entry && !p.lam_entry.empty())
    std::memcpy(lam_entry, p.lam_entry.data(), sizeof(int32_t) * p.lam_entry.size());
  return EMG_SUCCESS;
}

int emg_fetidp_lambda_rhs(emg_fetidp fd, const double* b_d, double* rhs_d) {
  return guarded([&]() -> int {
    if (!fd || !rhs_d) { set_error("null argument"); return EMG_INVALID_INPUT; }
    return fd->fd.lambda_rhs(b_d, rhs_d);
  });
}

int emg_direct_create(emg_mesh mesh, emg_dofmap map, void* stream, emg_direct* out) {
  return guarded([&]() -> int {
    if (!mesh || !map || !out) { set_error("null argument"); return EMG_INVALID_INPUT; }
    *out = nullptr;
    if (map->d.n_elems != mesh->m.n_elems || map->d.elem_type != mesh->m.elem_type ||
        map->d.l2g.size() != static_cast<size_t>(mesh->m.epe() * mesh->m.n_elems)) {
      set_error("DOF map does not belong to this mesh");
      return EMG_INVALID_INPUT;
    }
    emg::keep_pool_memory();
    auto* h = new emg_direct_t();
    int rc = h->fd.create(mesh->m, single_part(map->d), as_stream(stream));
    if (rc) { delete h; return rc; }
    *out = h;
    return EMG_SUCCESS;
  });
}

int emg_direct_factor(emg_direct d, const double* nu, const double* sigma, int32_t n_materials,
                      const emg_source* sources, int32_t n_sources, int32_t flags) {
  return guarded([&]() -> int {
    if (!d) { set_error("null direct-solver handle"); return EMG_INVALID_INPUT; }
    return d->fd.factor(nu, sigma, n_materials, sources, n_sources, flags);
  });
}

int emg_direct_solve(emg_direct d, const emg_krylov_config* cfg, const double* b, double* x, int32_t on_device,
                     emg_result* out) {
  return guarded([&]() -> int {
    if (!d) { set_error("null direct-solver handle"); return EMG_INVALID_INPUT; }
    return fetidp_solve_impl(&d->fd, cfg, b, x, on_device, out);
  });
}

int emg_direct_info(emg_direct d, int64_t* info, int32_t n_info) {
  if (!d || (!info && n_info > 0)) { set_error("null argument"); return EMG_INVALID_INPUT; }
  feti_info(d->fd.plan, info, n_info);
  return EMG_SUCCESS;
}

void emg_direct_destroy(emg_direct d) { delete d; }

}  // extern "C"
