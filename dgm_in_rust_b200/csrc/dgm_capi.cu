// dgm_capi.cu -- host side of the C ABI declared in include/dgm_b200.h.
//
// A dgm_ctx owns one CUDA stream, the device-resident state (U and the two RK stage buffers
// of TemperalDisc::temporary_solutions, temporal_disc.rs:9), the SoA mesh/geometry arrays and
// the control block through which the time-march loop runs on the device.  Whole time steps
// are captured into CUDA graphs (one launch per group of steps).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dgm_b200.h"
#include "dgm_device.cuh"

using dgm::Control;
using dgm::KParams;
using dgm::MeshDev;
using dgm::NEQ;

struct dgm_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  int P = 0, nb = 0, nq = 0, ng = 0;
  int64_t ne = 0, ld = 0, n_int = 0, n_bnd = 0, np = 0;
  int limiter = 1;
  double hcr = 1.4, cfl = 0.0, final_time = 0.0;
  int64_t final_step = 0;
  double current_time = 0.0;
  int64_t current_step = 0;
  std::vector<unsigned char> kparams;  // host image of KParams<P>
  // device buffers
  double *U = nullptr, *U1 = nullptr, *U2 = nullptr, *R = nullptr, *F = nullptr, *stage = nullptr;
  unsigned char* t0 = nullptr;
  unsigned int* status = nullptr;
  int* work = nullptr;
  Control* ctl = nullptr;
  std::vector<void*> allocs;
  int64_t bytes = 0;
  int coop_blocks = 1;
  bool coop_ok = true;
  // graphs[with_residual][g]: g = 0 captures graph_steps steps, g = 1 a single step
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int graph_steps = 8;
  bool graphs_broken = false;
  bool limits_dirty = false;
  int64_t err_where = -1;
  int64_t last_troubled = 0;
  int last_waves = 0;
};

namespace {

const int64_t kGraphSteps = 8;

#define CK(call)                                                                 \
  do {                                                                           \
    cudaError_t _e = (call);                                                     \
    if (_e != cudaSuccess) {                                                     \
      std::fprintf(stderr, "dgm_b200: %s failed: %s (%s:%d)\n", #call,           \
                   cudaGetErrorString(_e), __FILE__, __LINE__);                  \
      return DGM_CUDA_ERROR;                                                     \
    }                                                                            \
  } while (0)

template <class T>
int dev_alloc(dgm_ctx* c, T** p, size_t count) {
  void* ptr = nullptr;
  const size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
  if (cudaMalloc(&ptr, nbytes) != cudaSuccess) {
    cudaGetLastError();
    return DGM_OOM;
  }
  c->allocs.push_back(ptr);
  c->bytes += (int64_t)nbytes;
  *p = static_cast<T*>(ptr);
  return DGM_OK;
}

template <class T>
int upload(dgm_ctx* c, T** p, const std::vector<T>& h) {
  int st = dev_alloc(c, p, h.size());
  if (st) return st;
  if (!h.empty()) CK(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return DGM_OK;
}

template <int P>
KParams<P>& kp_of(dgm_ctx* c) {
  return *reinterpret_cast<KParams<P>*>(c->kparams.data());
}

// ---------------------------------------------------------------------------------------------
// Kernel launch helpers, one instantiation per supported order.
// ---------------------------------------------------------------------------------------------
template <int P>
struct Ops {
  using V = dgm::Variant<P>;

  static int edge_flux(dgm_ctx* c, const double* U) {
    const int64_t total = (c->n_int + c->n_bnd) * V::NG;
    const int threads = 256;
    const int blocks = (int)std::max<int64_t>(1, (total + threads - 1) / threads);
    dgm::k_edge_flux<P><<<blocks, threads, 0, c->stream>>>(kp_of<P>(c), U, c->F);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  template <int MODE>
  static int element(dgm_ctx* c, const double* Uin, const double* Ubase, double* Uout, const double* Rin,
                     double* Rout) {
    const int threads = 256;  // 8 warps x 8 elements, 4 threads (variables) per element
    const int blocks = (int)std::max<int64_t>(1, (c->ne + 63) / 64);
    dgm::k_element<P, MODE><<<blocks, threads, 0, c->stream>>>(kp_of<P>(c), Uin, Ubase, c->F, Uout, Rin, Rout);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int limiter(dgm_ctx* c, double* U) {
    if (!c->limiter) return DGM_OK;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c->coop_blocks);
    cfg.blockDim = dim3(dgm::kLimiterWarps * 32);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, dgm::k_limiter<P>, kp_of<P>(c), U, c->t0, c->status, c->work));
    return DGM_OK;
  }

  static int time_step(dgm_ctx* c, const double* U) {
    const int threads = 256;
    const int blocks = (int)std::max<int64_t>(1, (c->ne + threads - 1) / threads);
    dgm::k_time_step<P><<<blocks, threads, 0, c->stream>>>(kp_of<P>(c), U);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  // One SSP-RK3 step on the resident state (rk3.rs:7-26); dt is read from the control block.
  static int rk3(dgm_ctx* c, double* Rout) {
    int st;
    if ((st = edge_flux(c, c->U))) return st;
    if ((st = element<1>(c, c->U, nullptr, c->U1, nullptr, nullptr))) return st;
    if ((st = limiter(c, c->U1))) return st;
    if ((st = edge_flux(c, c->U1))) return st;
    if ((st = element<2>(c, c->U1, c->U, c->U2, nullptr, nullptr))) return st;
    if ((st = limiter(c, c->U2))) return st;
    if ((st = edge_flux(c, c->U2))) return st;
    if ((st = element<3>(c, c->U2, c->U, c->U, nullptr, Rout))) return st;
    return limiter(c, c->U);
  }

  // One iteration of time_march (temporal_disc.rs:22-33), fully on the device.
  static int step(dgm_ctx* c, double* Rout) {
    dgm::k_step_begin<<<1, 1, 0, c->stream>>>(c->ctl);
    CK(cudaGetLastError());
    int st;
    if ((st = time_step(c, c->U))) return st;
    dgm::k_step_dt<<<1, 1, 0, c->stream>>>(c->ctl);
    CK(cudaGetLastError());
    if ((st = rk3(c, Rout))) return st;
    dgm::k_step_end<<<1, 1, 0, c->stream>>>(c->ctl);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int to_soa(dgm_ctx* c, const double* src_aos, double* dst) {
    const int64_t n = c->ne * NEQ * V::NB;
    const int threads = 256;
    dgm::k_aos_to_soa<V::NB><<<(int)((n + threads - 1) / threads), threads, 0, c->stream>>>(src_aos, dst, (int)c->ne, (int)c->ld);
    CK(cudaGetLastError());
    return DGM_OK;
  }
  static int to_aos(dgm_ctx* c, const double* src, double* dst_aos) {
    const int64_t n = c->ne * NEQ * V::NB;
    const int threads = 256;
    dgm::k_soa_to_aos<V::NB><<<(int)((n + threads - 1) / threads), threads, 0, c->stream>>>(src, dst_aos, (int)c->ne, (int)c->ld);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int occupancy(dgm_ctx* c) {
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dgm::k_limiter<P>, dgm::kLimiterWarps * 32, 0));
    per_sm = std::max(1, per_sm);
    const int64_t want = std::max<int64_t>(1, (c->ne + 32 * dgm::kLimiterWarps - 1) / (32 * dgm::kLimiterWarps));
    c->coop_blocks = (int)std::min<int64_t>((int64_t)per_sm * c->num_sms, want);
    return DGM_OK;
  }

  static int fill_tables(dgm_ctx* c, const dgm_tables_desc* t) {
    c->kparams.assign(sizeof(KParams<P>), 0);
    auto& kp = kp_of<P>(c);
    auto& tb = kp.tab;
    const int NB = V::NB, NQ = V::NQ, NG = V::NG, NK = V::NK;
    const int nk_in = t->n_deriv_keys;
    if (nk_in < NK) return DGM_BAD_ARG;
    for (int q = 0; q < NQ; ++q)
      for (int b = 0; b < NB; ++b) {
        tb.phi_cell[q][b] = t->phi_cell[q * NB + b];
        tb.dxi[q][b] = t->dphi_cell_ref[((size_t)q * NB + b) * nk_in + 0];
        tb.deta[q][b] = t->dphi_cell_ref[((size_t)q * NB + b) * nk_in + 1];
        for (int k = 0; k < NK; ++k) tb.dref[q][b][k] = t->dphi_cell_ref[((size_t)q * NB + b) * nk_in + k];
      }
    for (int k = 0; k < 3; ++k)
      for (int g = 0; g < NG; ++g)
        for (int b = 0; b < NB; ++b) tb.phi_edge[k][g][b] = t->phi_edge[(k * NG + g) * NB + b];
    for (int q = 0; q < NQ; ++q) tb.cell_w[q] = t->cell_weights[q];
    for (int g = 0; g < NG; ++g) tb.edge_w[g] = t->edge_weights[g];
    for (int b = 0; b < NB; ++b) {
      tb.mass[b] = t->mass_diag[b];
      kp.inv_mass[b] = 1.0 / t->mass_diag[b];
    }
    // gas constants with the reference's expressions (flux.rs:76-77, 85, 96)
    dgm::Gas& gas = kp.gas;
    gas.hcr = c->hcr;
    gas.gm1 = c->hcr - 1.0;
    gas.zeta = (c->hcr - 1.0) / (2.0 * c->hcr);
    gas.inv_zeta = 1.0 / gas.zeta;
    gas.zm1h = (gas.zeta - 1.0) / 2.0;
    gas.gp1h = (c->hcr + 1.0) / (2.0 * c->hcr);
    const double n = std::nearbyint(gas.inv_zeta);
    gas.inv_zeta_int = (n >= 1.0 && n <= 16.0 && std::fabs(gas.inv_zeta - n) <= 1e-12 * n) ? (int)n : 0;
    kp.ctl = c->ctl;
    return DGM_OK;
  }
};

template <class F>
int dispatch(dgm_ctx* c, F&& f) {
  switch (c->P) {
    case 1: return f(Ops<1>{});
    case 2: return f(Ops<2>{});
    case 3: return f(Ops<3>{});
  }
  return DGM_BAD_ARG;
}

MeshDev& mesh_of(dgm_ctx* c) {
  switch (c->P) {
    case 1: return kp_of<1>(c).m;
    case 2: return kp_of<2>(c).m;
    default: return kp_of<3>(c).m;
  }
}

int read_control(dgm_ctx* c, Control* h) {
  CK(cudaMemcpyAsync(h, c->ctl, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

// Resets the device status word and returns the status raised since the last call.
int collect_status(dgm_ctx* c) {
  Control h;
  int st = read_control(c, &h);
  if (st) return st;
  c->current_time = h.t;
  c->current_step = h.step;
  c->last_troubled = h.troubled;
  c->last_waves = h.waves;
  if (h.status != 0) {
    c->err_where = h.err_where;
    const int zero = 0;
    CK(cudaMemcpyAsync(&c->ctl->status, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return h.status;
  }
  return DGM_OK;
}

int set_active(dgm_ctx* c, double dt, bool set_dt) {
  dgm::k_set_active<<<1, 1, 0, c->stream>>>(c->ctl, dt, set_dt ? 1 : 0);
  CK(cudaGetLastError());
  return DGM_OK;
}

int upload_state(dgm_ctx* c, const double* host, double* dst) {
  const size_t n = (size_t)c->ne * NEQ * c->nb;
  CK(cudaMemcpyAsync(c->stage, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return dispatch(c, [&](auto ops) { return decltype(ops)::to_soa(c, c->stage, dst); });
}

int download_state(dgm_ctx* c, const double* src, double* host) {
  const size_t n = (size_t)c->ne * NEQ * c->nb;
  int st = dispatch(c, [&](auto ops) { return decltype(ops)::to_aos(c, src, c->stage); });
  if (st) return st;
  CK(cudaMemcpyAsync(host, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return DGM_OK;
}

int write_clock(dgm_ctx* c) {
  Control h;
  int st = read_control(c, &h);
  if (st) return st;
  h.t = c->current_time;
  h.step = c->current_step;
  h.final_time = c->final_time;
  h.final_step = c->final_step;
  h.cfl = c->cfl;
  CK(cudaMemcpyAsync(c->ctl, &h, sizeof(Control), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->limits_dirty = false;
  return DGM_OK;
}

int build_graph(dgm_ctx* c, int with_residual, int single) {
  if (c->graph[with_residual][single] || c->graphs_broken) return DGM_OK;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    c->graphs_broken = true;
    return DGM_OK;
  }
  int st = DGM_OK;
  const int n = single ? 1 : c->graph_steps;
  for (int i = 0; i < n && st == DGM_OK; ++i)
    st = dispatch(c, [&](auto ops) { return decltype(ops)::step(c, with_residual ? c->R : nullptr); });
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (st != DGM_OK || e != cudaSuccess || g == nullptr) {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    c->graphs_broken = true;  // fall back to direct launches
    return DGM_OK;
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    c->graphs_broken = true;
    return DGM_OK;
  }
  c->graph[with_residual][single] = exec;
  return DGM_OK;
}

// Enqueue n time-march iterations on the resident state.
int enqueue_steps(dgm_ctx* c, int64_t n, int with_residual) {
  int st;
  while (n > 0) {
    const int single = n >= c->graph_steps ? 0 : 1;
    if ((st = build_graph(c, with_residual, single))) return st;
    if (!c->graphs_broken) {
      CK(cudaGraphLaunch(c->graph[with_residual][single], c->stream));
      n -= single ? 1 : c->graph_steps;
    } else {
      st = dispatch(c, [&](auto ops) { return decltype(ops)::step(c, with_residual ? c->R : nullptr); });
      if (st) return st;
      n -= 1;
    }
  }
  return DGM_OK;
}

int build_mesh(dgm_ctx* c, const dgm_mesh_desc* m) {
  const int64_t ne = m->n_elements, ned = m->n_edges;
  if (ne <= 0 || ned <= 0 || ne > (1ll << 30) || ned > (1ll << 29)) return DGM_BAD_ARG;
  const int64_t ld = (ne + 31) / 32 * 32;
  c->ne = ne;
  c->ld = ld;
  c->np = m->n_patches;
  auto X = [&](int64_t v) { return m->vertex_xy[2 * v]; };
  auto Y = [&](int64_t v) { return m->vertex_xy[2 * v + 1]; };
  auto in_range = [](int64_t i, int64_t n) { return i >= 0 && i < n; };
  // edge slots: internal edges in Mesh::internal_edge_indices order, then boundary edges
  std::vector<int64_t> slot_of(ned, -1), slot_ref;
  std::vector<int2> ie_lr;
  std::vector<int> ie_ic;
  std::vector<double4> ie_geo;
  for (int64_t i = 0; i < m->n_internal_edges; ++i) {
    const int64_t d = m->internal_edges[i];
    if (!in_range(d, ned) || slot_of[d] >= 0) return DGM_BAD_ARG;
    const int64_t L = m->edge_elements[2 * d], R = m->edge_elements[2 * d + 1];
    const int64_t il = m->edge_in_cell[2 * d], ir = m->edge_in_cell[2 * d + 1];
    if (!in_range(L, ne) || !in_range(R, ne) || L == R || !in_range(il, 3) || !in_range(ir, 3)) return DGM_BAD_ARG;
    slot_of[d] = (int64_t)slot_ref.size();
    slot_ref.push_back(d);
    ie_lr.push_back(make_int2((int)L, (int)R));
    ie_ic.push_back((int)(il | (ir << 2)));
    const double jd = m->edge_jacob_det[d];
    ie_geo.push_back(make_double4(m->edge_normal[2 * d], m->edge_normal[2 * d + 1], 0.5 * jd, jd));
  }
  c->n_int = (int64_t)slot_ref.size();
  std::vector<int> be_elem, be_info;
  std::vector<double4> be_geo;
  for (int64_t d = 0; d < ned; ++d) {
    if (m->edge_elements[2 * d + 1] != -1) continue;
    const int64_t e = m->edge_elements[2 * d], k = m->edge_in_cell[2 * d], patch = m->edge_patch[d];
    if (!in_range(e, ne) || !in_range(k, 3) || !in_range(patch, m->n_patches)) return DGM_BAD_ARG;
    slot_of[d] = (int64_t)slot_ref.size();
    slot_ref.push_back(d);
    const int type = m->patch_type[patch];
    if (type != DGM_WALL && type != DGM_FARFIELD) return DGM_BAD_ARG;
    be_elem.push_back((int)e);
    be_info.push_back((int)(k | (type << 2) | (patch << 3)));
    // outward orientation, boundary_condition.rs:22-28
    const bool same = m->elem_vertices[3 * e + k] == m->edge_vertices[2 * d];
    const double nx = same ? m->edge_normal[2 * d] : -m->edge_normal[2 * d];
    const double ny = same ? m->edge_normal[2 * d + 1] : -m->edge_normal[2 * d + 1];
    const double jd = m->edge_jacob_det[d];
    be_geo.push_back(make_double4(nx, ny, 0.5 * jd, jd));
  }
  c->n_bnd = (int64_t)be_elem.size();
  // far-field conserved state, boundary_condition.rs:50-55
  std::vector<double4> patch_q(std::max<int64_t>(1, m->n_patches));
  for (int64_t p = 0; p < m->n_patches; ++p) {
    const double* bq = &m->patch_quantity[4 * p];
    patch_q[p] = make_double4(bq[0], bq[0] * bq[1], bq[0] * bq[2],
                              bq[3] / (c->hcr - 1.0) + 0.5 * bq[0] * (bq[1] * bq[1] + bq[2] * bq[2]));
  }
  // element faces, neighbours, geometry (SoA)
  std::vector<int> face(3 * ld, 0), nbr(3 * ld, -1);
  std::vector<double> jac(ne), hmin(ne), h15(ne), dinv(4 * ld, 0.0);
  std::vector<unsigned char> in_list(ne, 0);
  for (int64_t i = 0; i < m->n_boundary_elements; ++i) {
    const int64_t e = m->boundary_elements[i];
    if (!in_range(e, ne)) return DGM_BAD_ARG;
    in_list[e] = 1;
  }
  for (int64_t e = 0; e < ne; ++e) {
    bool has_boundary = false;
    for (int k = 0; k < 3; ++k) {
      const int64_t d = m->elem_edges[3 * e + k];
      if (!in_range(d, ned) || slot_of[d] < 0) return DGM_BAD_ARG;
      int side;
      if (m->edge_elements[2 * d + 1] == -1) {
        if (m->edge_elements[2 * d] != e || m->edge_in_cell[2 * d] != k) return DGM_BAD_ARG;
        side = 0;
        has_boundary = true;
        if (m->elem_neighbours[3 * e + k] != -1) return DGM_BAD_ARG;
      } else {
        const bool same = m->elem_vertices[3 * e + k] == m->edge_vertices[2 * d];
        if (m->edge_elements[2 * d] == e && same && m->edge_in_cell[2 * d] == k) side = 0;
        else if (m->edge_elements[2 * d + 1] == e && !same && m->edge_in_cell[2 * d + 1] == k) side = 1;
        else return DGM_BAD_ARG;  // orientation inconsistent with process_mesh's left/right rule
        const int64_t other = m->edge_elements[2 * d + (side ? 0 : 1)];
        if (m->elem_neighbours[3 * e + k] != other) return DGM_BAD_ARG;
        nbr[k * ld + e] = (int)other;
      }
      face[k * ld + e] = (int)((slot_of[d] << 1) | side);
    }
    // every element is in exactly one of the internal / boundary element lists
    if (has_boundary != (in_list[e] != 0)) return DGM_BAD_ARG;
    const double J = m->elem_jacob_det[e];
    const int64_t v1 = m->elem_vertices[3 * e], v2 = m->elem_vertices[3 * e + 1], v3 = m->elem_vertices[3 * e + 2];
    if (!in_range(v1, m->n_vertices) || !in_range(v2, m->n_vertices) || !in_range(v3, m->n_vertices)) return DGM_BAD_ARG;
    jac[e] = J;
    // compute_dphi inverse Jacobian, mesh.rs:93-100
    dinv[0 * ld + e] = (Y(v3) - Y(v1)) / J;
    dinv[1 * ld + e] = -(X(v3) - X(v1)) / J;
    dinv[2 * ld + e] = -(Y(v2) - Y(v1)) / J;
    dinv[3 * ld + e] = (X(v2) - X(v1)) / J;
    hmin[e] = m->elem_minimum_height[e];
    h15[e] = std::pow(m->elem_circumradius[e], 1.5);  // weno.rs:81 h.powf(1.5)
  }
  MeshDev md{};
  md.ne = (int)ne;
  md.ld = (int)ld;
  md.n_int = (int)c->n_int;
  md.n_bnd = (int)c->n_bnd;
  int st;
  double *d_jac, *d_dinv, *d_hmin, *d_h15;
  int *d_face, *d_nbr, *d_ie_ic, *d_be_elem, *d_be_info;
  int2* d_ie_lr;
  double4 *d_ie_geo, *d_be_geo, *d_patch;
  int64_t* d_slot_ref;
  if ((st = upload(c, &d_jac, jac)) || (st = upload(c, &d_dinv, dinv)) || (st = upload(c, &d_hmin, hmin)) ||
      (st = upload(c, &d_h15, h15)) || (st = upload(c, &d_face, face)) || (st = upload(c, &d_nbr, nbr)) ||
      (st = upload(c, &d_ie_lr, ie_lr)) || (st = upload(c, &d_ie_ic, ie_ic)) || (st = upload(c, &d_ie_geo, ie_geo)) ||
      (st = upload(c, &d_be_elem, be_elem)) || (st = upload(c, &d_be_info, be_info)) ||
      (st = upload(c, &d_be_geo, be_geo)) || (st = upload(c, &d_patch, patch_q)) ||
      (st = upload(c, &d_slot_ref, slot_ref)))
    return st;
  md.jac = d_jac;
  md.dinv = d_dinv;
  md.hmin = d_hmin;
  md.h15 = d_h15;
  md.face = d_face;
  md.nbr = d_nbr;
  md.ie_lr = d_ie_lr;
  md.ie_ic = d_ie_ic;
  md.ie_geo = d_ie_geo;
  md.be_elem = d_be_elem;
  md.be_info = d_be_info;
  md.be_geo = d_be_geo;
  md.patch_q = d_patch;
  md.slot_ref = d_slot_ref;
  mesh_of(c) = md;
  return DGM_OK;
}

}  // namespace

extern "C" {

const char* dgm_version(void) { return "dgm_b200 0.1 (sm_100a, FP64 DG residual + SSP-RK3)"; }

const char* dgm_status_string(int32_t s) {
  switch (s) {
    case DGM_OK: return "ok";
    case DGM_NEG_DENSITY: return "Negative density found in HLLC!";
    case DGM_NEG_PRESSURE: return "Negative pressure found in HLLC!";
    case DGM_NONFINITE: return "Non-finite value";
    case DGM_TOO_MANY_BOUNDARY_EDGES: return "Invalid number of boundary neighbours!";
    case DGM_OOM: return "Device memory allocation failed";
    case DGM_TIMEOUT: return "Device wait timed out";
    case DGM_BAD_ARG: return "Invalid argument";
    case DGM_CUDA_ERROR: return "CUDA runtime error";
    case DGM_NO_DEVICE: return "No usable CUDA device";
  }
  return "unknown status";
}

void dgm_destroy(dgm_ctx* c) {
  if (!c) return;
  if (c->device >= 0) cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& row : c->graph)
    for (auto& g : row)
      if (g) cudaGraphExecDestroy(g);
  for (void* p : c->allocs) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

dgm_ctx* dgm_create(const dgm_mesh_desc* mesh, const dgm_tables_desc* tables, const dgm_params* params,
                    int32_t* status) {
  int32_t dummy;
  if (!status) status = &dummy;
  if (!mesh || !tables || !params) {
    *status = DGM_BAD_ARG;
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || params->device < 0 || params->device >= ndev) {
    cudaGetLastError();
    *status = DGM_NO_DEVICE;
    return nullptr;
  }
  const int P = tables->order;
  const bool ok_variant = (P == 1 && tables->n_basis == 3 && tables->n_cell_gp == 3 && tables->n_edge_gp == 2) ||
                          (P == 2 && tables->n_basis == 6 && tables->n_cell_gp == 6 && tables->n_edge_gp == 3) ||
                          (P == 3 && tables->n_basis == 10 && tables->n_cell_gp == 12 && tables->n_edge_gp == 4);
  if (!ok_variant) {
    *status = DGM_BAD_ARG;
    return nullptr;
  }
  auto* c = new dgm_ctx();
  c->device = params->device;
  c->P = P;
  c->nb = tables->n_basis;
  c->nq = tables->n_cell_gp;
  c->ng = tables->n_edge_gp;
  c->hcr = params->hcr;
  c->cfl = params->cfl;
  c->final_time = params->final_time;
  c->final_step = params->final_step;
  c->limiter = params->limiter ? 1 : 0;
  auto fail = [&](int st) {
    *status = st;
    dgm_destroy(c);
    return (dgm_ctx*)nullptr;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(DGM_NO_DEVICE);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) return fail(DGM_NO_DEVICE);
  c->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  int st;
  if ((st = dev_alloc(c, &c->ctl, 1))) return fail(st);
  if (cudaMemset(c->ctl, 0, sizeof(Control)) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  st = dispatch(c, [&](auto ops) { return decltype(ops)::fill_tables(c, tables); });
  if (st) return fail(st);
  if ((st = build_mesh(c, mesh))) return fail(st);
  const size_t n_state = (size_t)NEQ * c->nb * c->ld;
  const size_t n_flux = (size_t)(c->n_int + c->n_bnd) * c->ng * 4;
  if ((st = dev_alloc(c, &c->U, n_state)) || (st = dev_alloc(c, &c->U1, n_state)) ||
      (st = dev_alloc(c, &c->U2, n_state)) || (st = dev_alloc(c, &c->R, n_state)) ||
      (st = dev_alloc(c, &c->F, n_flux)) || (st = dev_alloc(c, &c->stage, (size_t)c->ne * NEQ * c->nb)) ||
      (st = dev_alloc(c, &c->t0, (size_t)c->ne)) || (st = dev_alloc(c, &c->status, (size_t)c->ne)) ||
      (st = dev_alloc(c, &c->work, (size_t)c->ne)))
    return fail(st);
  for (double* p : {c->U, c->U1, c->U2, c->R})
    if (cudaMemset(p, 0, n_state * sizeof(double)) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  if (cudaMemset(c->status, 0, (size_t)c->ne * sizeof(unsigned int)) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  if ((st = dispatch(c, [&](auto ops) { return decltype(ops)::occupancy(c); }))) return fail(st);
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
  if (!coop) return fail(DGM_NO_DEVICE);
  c->graph_steps = (int)kGraphSteps;
  if ((st = write_clock(c))) return fail(st);
  *status = DGM_OK;
  return c;
}

int32_t dgm_compute_residuals(dgm_ctx* c, double* residuals, const double* solutions) {
  if (!c || !residuals || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, solutions, c->U1))) return st;
  if ((st = upload_state(c, residuals, c->U2))) return st;
  if ((st = set_active(c, 0.0, false))) return st;
  st = dispatch(c, [&](auto ops) {
    using O = decltype(ops);
    int s2 = O::edge_flux(c, c->U1);
    if (s2) return s2;
    return O::template element<0>(c, c->U1, nullptr, nullptr, c->U2, c->R);
  });
  if (st) return st;
  if ((st = download_state(c, c->R, residuals))) return st;
  return collect_status(c);
}

int32_t dgm_apply_limiter(dgm_ctx* c, double* solutions, int64_t* troubled) {
  if (!c || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, solutions, c->U1))) return st;
  if ((st = set_active(c, 0.0, false))) return st;
  if ((st = dispatch(c, [&](auto ops) { return decltype(ops)::limiter(c, c->U1); }))) return st;
  if ((st = download_state(c, c->U1, solutions))) return st;
  st = collect_status(c);
  if (troubled) *troubled = c->last_troubled;
  return st;
}

int32_t dgm_compute_time_step(dgm_ctx* c, const double* solutions, double* time_step) {
  if (!c || !solutions || !time_step) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, solutions, c->U1))) return st;
  if ((st = set_active(c, 0.0, false))) return st;
  if ((st = dispatch(c, [&](auto ops) { return decltype(ops)::time_step(c, c->U1); }))) return st;
  Control h;
  if ((st = read_control(c, &h))) return st;
  unsigned long long bits = h.dt_bits;
  std::memcpy(time_step, &bits, sizeof(double));
  return collect_status(c);
}

int32_t dgm_rk3(dgm_ctx* c, double* residuals, double* solutions, double time_step) {
  if (!c || !residuals || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, solutions, c->U))) return st;
  if ((st = set_active(c, time_step, true))) return st;
  if ((st = dispatch(c, [&](auto ops) { return decltype(ops)::rk3(c, c->R); }))) return st;
  if ((st = download_state(c, c->U, solutions))) return st;
  if ((st = download_state(c, c->R, residuals))) return st;
  return collect_status(c);
}

int32_t dgm_time_march(dgm_ctx* c, double* residuals, double* solutions) {
  if (!c || !residuals || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = write_clock(c))) return st;
  if ((st = upload_state(c, solutions, c->U))) return st;
  const int64_t remaining = std::max<int64_t>(0, c->final_step - c->current_step);
  if ((st = enqueue_steps(c, remaining, 1))) return st;
  if ((st = download_state(c, c->U, solutions))) return st;
  if (remaining > 0)
    if ((st = download_state(c, c->R, residuals))) return st;
  return collect_status(c);
}

int32_t dgm_get_clock(dgm_ctx* c, double* t, int64_t* step) {
  if (!c) return DGM_BAD_ARG;
  if (t) *t = c->current_time;
  if (step) *step = c->current_step;
  return DGM_OK;
}

int32_t dgm_set_clock(dgm_ctx* c, double t, int64_t step) {
  if (!c) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  c->current_time = t;
  c->current_step = step;
  return write_clock(c);
}

int32_t dgm_set_limits(dgm_ctx* c, double final_time, int64_t final_step) {
  if (!c) return DGM_BAD_ARG;
  c->final_time = final_time;
  c->final_step = final_step;
  c->limits_dirty = true;
  return DGM_OK;
}

int32_t dgm_upload_solutions(dgm_ctx* c, const double* solutions) {
  if (!c || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = upload_state(c, solutions, c->U);
  if (st) return st;
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

int32_t dgm_download_solutions(dgm_ctx* c, double* solutions) {
  if (!c || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = download_state(c, c->U, solutions);
  if (st) return st;
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

int32_t dgm_advance(dgm_ctx* c, int64_t n_steps) {
  if (!c || n_steps < 0) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  if (c->limits_dirty) {
    int st = write_clock(c);
    if (st) return st;
  }
  return enqueue_steps(c, n_steps, 0);
}

int32_t dgm_synchronize(dgm_ctx* c) {
  if (!c) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  return collect_status(c);
}

void* dgm_stream(dgm_ctx* c) { return c ? (void*)c->stream : nullptr; }

int32_t dgm_launch_phase(dgm_ctx* c, int32_t phase) {
  if (!c || phase < 0 || phase > 3) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = set_active(c, 0.0, false);
  if (st) return st;
  return dispatch(c, [&](auto ops) {
    using O = decltype(ops);
    switch (phase) {
      case 0: return O::time_step(c, c->U);
      case 1: return O::edge_flux(c, c->U);
      case 2: return O::template element<2>(c, c->U, c->U, c->U2, nullptr, nullptr);
      default: return O::limiter(c, c->U2);
    }
  });
}

int32_t dgm_phase_launches_per_step(dgm_ctx* c, int32_t phase) {
  if (!c) return 0;
  static const int per_step[4] = {1, 3, 3, 3};
  if (phase < 0 || phase > 3) return 0;
  if (!c->limiter && phase == 3) return 0;
  return per_step[phase];
}

int32_t dgm_launches_per_step(dgm_ctx* c) {
  if (!c) return 0;
  return 3 /* step control */ + 1 /* time step */ + 3 * (2 + (c->limiter ? 1 : 0));
}

int64_t dgm_error_location(dgm_ctx* c) { return c ? c->err_where : -1; }

int32_t dgm_limiter_stats(dgm_ctx* c, int64_t* troubled, int32_t* waves) {
  if (!c) return DGM_BAD_ARG;
  if (troubled) *troubled = c->last_troubled;
  if (waves) *waves = c->last_waves;
  return DGM_OK;
}

int64_t dgm_device_bytes(dgm_ctx* c) { return c ? c->bytes : 0; }

}  // extern "C"
