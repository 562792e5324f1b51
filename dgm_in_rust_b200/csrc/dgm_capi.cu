// dgm_capi.cu -- host side of the C ABI declared in include/dgm_b200.h.
//
// A dgm_ctx owns one CUDA stream, the device-resident state (U and the two RK stage buffers
// of TemperalDisc::temporary_solutions, temporal_disc.rs:9), the SoA mesh/geometry arrays of
// one or more mesh instances (a disconnected union mesh), a control block per instance and the
// context-wide control block through which the time-march loop runs on the device.  Whole time
// steps are captured into CUDA graphs (one launch per group of steps).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "dgm_b200.h"
#include "dgm_device.cuh"
#include "dgm_mixed.cuh"
#include "dgm_tc.cuh"
#include "dgm_viscous.cuh"

using dgm::Control;
using dgm::InstCtl;
using dgm::KParams;
using dgm::MeshDev;
using dgm::NEQ;

struct HostInst {
  int64_t elem_off = 0, ne = 0;         // element range in the union mesh (the mesh's elements)
  int64_t bslot_off = 0, nb_slots = 0;  // boundary-slot range (relative to n_int)
  // capacity ranges (dgm_create_batch_slots): elements [elem_off, elem_off + elem_cap), internal
  // slots [int_off, int_off + int_cap), boundary slots [n_int + bnd_off, + bnd_cap), patches
  int64_t elem_cap = 0, int_off = 0, int_cap = 0, bnd_off = 0, bnd_cap = 0, patch_off = 0, patch_cap = 0;
  double cfl = 0.0, final_time = 0.0;
  int64_t final_step = 0;
  double t = 0.0;
  int64_t step = 0;
  int32_t status = 0;
  int64_t err_where = -1;
};

struct dgm_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;  // the device's context pool (held while the context lives)
  int P = 0, nb = 0, nq = 0, ng = 0;
  int prec = 0;       // storage: 0 FP64 state, 1 FP32 state and bulk arithmetic
  int prec_mode = 0;  // dgm_params::precision (0 fp64, 1 fp32, 2 tf32, 3 tf32x3, 4 fp32 arithmetic, fp64 state)
  int tc_split = 0;   // element pass on the tensor cores: 0 no (FP32 FMA), 1 TF32, 3 3xTF32
  int64_t ne = 0, ld = 0, n_int = 0, n_bnd = 0, np = 0, max_inst_ne = 0;
  int limiter = 1;
  double hcr = 1.4;
  std::vector<HostInst> inst;
  std::vector<unsigned char> kparams;  // host image of KParams<P, T>
  // Navier-Stokes residual (dgm_set_viscous): host image of NsParams<P>, the global lifts
  int viscous = 0;
  std::vector<unsigned char> nsparams;
  double* ns_lift = nullptr;
  std::vector<double> proj_phi, proj_w, proj_mass;  // FP64 tables of the initial projection
  // device buffers (state arrays are of the storage type)
  void *U = nullptr, *U1 = nullptr, *U2 = nullptr, *R = nullptr, *F = nullptr;
  double* stage = nullptr;  // FP64 staging in the reference layout (largest instance)
  unsigned char* t0 = nullptr;
  unsigned int* status = nullptr;
  int* work = nullptr;
  int* wl1 = nullptr;    // limiter: cells the detection enlists for wave 1 (entries of kEntryInts ints)
  int* pend = nullptr;   // limiter: elements the detection leaves for later waves
  int* order = nullptr;  // limiter: the detection's visiting order of the warp batches (breadth-first)
  int* d_elem_rng = nullptr;   // [2 n] first element, element count of each instance's mesh
  int* d_bslot_rng = nullptr;  // [2 n] first boundary slot (relative to n_int), boundary slot count
  bool padded = false;         // capacity ranges above the meshes' sizes: dead instance and null element
  int dead_inst = 0;           // index of the dead instance (padded contexts)
  int64_t null_elem = -1;      // the null element (padded contexts)
  double* d_diag = nullptr;
  double* h_diag = nullptr;         // pinned host copy of d_diag (dgm_enqueue_diagnostics)
  cudaEvent_t diag_ready = nullptr;  // recorded after the copy into h_diag
  double* gram = nullptr;   // WENO Gram matrices, [NB (NB + 1) / 2][ld] (limiter on)
  Control* ctl = nullptr;
  InstCtl* ic = nullptr;
  std::vector<void*> allocs;
  int64_t bytes = 0;
  int coop_blocks[2] = {1, 1};   // co-resident blocks of the limiter's wave kernel [schedule]
  int lim_one_per_sm = 0;        // wave kernel on one block per SM (cheaper grid barriers) instead of all
  int lim_staged = 0;            // limiter detector variant (dgm_set_limiter_variant / autotune)
  int lim_queue = 0;             // limiter schedule (dgm_set_limiter_schedule / autotune)
  int edge_pair = 0;             // edge pass form: 0 thread per (slot, point), 1 lane pair per slot,
                                 // 2 lane per point with the slots' records staged in shared memory,
                                 // 3 form 0 compiled for 64 registers
  float lim_us[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // last autotuned limiter times [detector][schedule]
  // launch configuration of the edge and element passes (dgm_set_launch_config / dgm_autotune):
  // edge_blocks = 0 launches one thread per (slot, Gauss point), else a grid-stride grid
  int edge_threads = 256, edge_blocks = 0, elem_threads = 256;
  // graphs[with_residual][g]: g = 0 captures graph_steps steps, g = 1 a single step
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int graph_steps = 8;
  bool graphs_broken = false;
  bool limits_dirty = false;
  bool dt_dirty = false;  // a host-driven time step left its minimum in the control blocks
  int64_t err_where = -1;
  int64_t last_troubled = 0;
  int last_waves = 0;
  bool owns_stream = true;
  // mixed batch (dgm_create_mixed): one child context per order present (kids[P - 1]), sharing
  // this context's stream; instance i of the batch is instance imap[i].second of kids[imap[i].first]
  bool mixed = false;
  dgm_ctx* kids[3] = {nullptr, nullptr, nullptr};
  std::vector<std::pair<int, int>> imap;
  int* mwork = nullptr;  // the mixed limiter's worklist of waves 2, 3, ... (all groups' elements)
  int mixed_blocks = 1;  // co-resident blocks of the mixed limiter's wave kernel
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

// Device memory of contexts comes from one stream-ordered pool per device, owned by the library
// and kept (release threshold: unlimited) while any context is alive: creating and destroying a
// context then costs no cudaMalloc/cudaFree, and in particular no device-wide synchronisation
// (cudaFree waits for every stream), so contexts created and retired while others run -- the
// serving loop's cohorts -- do not stall them.  The pool is trimmed when the last context of the
// device is destroyed.
constexpr int kMaxDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pool[kMaxDevices] = {};
int g_live[kMaxDevices] = {};

cudaMemPool_t pool_acquire(int device) {
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (device < 0 || device >= kMaxDevices) return nullptr;
  if (!g_pool[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&g_pool[device], &props) != cudaSuccess) {
      cudaGetLastError();
      g_pool[device] = nullptr;
      return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(g_pool[device], cudaMemPoolAttrReleaseThreshold, &keep);
  }
  ++g_live[device];
  return g_pool[device];
}

void pool_release(int device) {
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (device < 0 || device >= kMaxDevices || !g_pool[device]) return;
  if (--g_live[device] == 0) cudaMemPoolTrimTo(g_pool[device], 0);
}

int dev_alloc_bytes(dgm_ctx* c, void** p, size_t nbytes) {
  void* ptr = nullptr;
  if (!c->pool || cudaMallocFromPoolAsync(&ptr, std::max<size_t>(nbytes, 16), c->pool, c->stream) != cudaSuccess) {
    cudaGetLastError();
    return DGM_OOM;
  }
  c->allocs.push_back(ptr);
  c->bytes += (int64_t)nbytes;
  *p = ptr;
  return DGM_OK;
}

template <class T>
int dev_alloc(dgm_ctx* c, T** p, size_t count) {
  void* ptr = nullptr;
  const size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
  int st = dev_alloc_bytes(c, &ptr, nbytes);
  if (st) return st;
  *p = static_cast<T*>(ptr);
  return DGM_OK;
}

// Pageable source: cudaMemcpyAsync returns once the data is staged, so `h` may go out of scope.
template <class T>
int upload(dgm_ctx* c, T** p, const std::vector<T>& h) {
  int st = dev_alloc(c, p, h.size());
  if (st) return st;
  if (!h.empty()) CK(cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  return DGM_OK;
}

template <int P, typename T>
KParams<P, T>& kp_of(dgm_ctx* c) {
  return *reinterpret_cast<KParams<P, T>*>(c->kparams.data());
}

template <int P>
dgm::NsParams<P>& ns_of(dgm_ctx* c) {
  return *reinterpret_cast<dgm::NsParams<P>*>(c->nsparams.data());
}

// ---------------------------------------------------------------------------------------------
// Kernel launch helpers, one instantiation per (order, storage type).
// ---------------------------------------------------------------------------------------------
// T: the arithmetic type of the bulk kernels (and of the edge-flux array); St: the state's
// storage type (St = double, T = float: FP32 arithmetic on an FP64 state).
template <int P, typename T, typename St = T>
struct Ops {
  using V = dgm::Variant<P>;
  static St* S(void* p) { return static_cast<St*>(p); }
  static T* Fx(void* p) { return static_cast<T*>(p); }

  // The viscous residual's lift and edge passes (FP64 contexts only: dgm_set_viscous checks).
  static int ns_edge(dgm_ctx* c, const St* U) {
    if constexpr (std::is_same<T, double>::value && std::is_same<St, double>::value) {
      const int64_t nt = c->ne * NEQ;
      dgm::k_ns_lift<P><<<(int)std::max<int64_t>(1, (nt + 255) / 256), 256, 0, c->stream>>>(kp_of<P, T>(c),
                                                                                           ns_of<P>(c), U);
      CK(cudaGetLastError());
      const int64_t nt2 = (c->n_int + c->n_bnd) * 4;  // four lanes per edge slot
      constexpr int tpb = dgm::kNsEdgeThreads;
      dgm::k_edge_flux_ns<P><<<(int)std::max<int64_t>(1, (nt2 + tpb - 1) / tpb), tpb, 0, c->stream>>>(
          kp_of<P, T>(c), ns_of<P>(c), U, Fx(c->F));
      CK(cudaGetLastError());
      return DGM_OK;
    } else {
      return DGM_BAD_ARG;
    }
  }

  static int edge_flux(dgm_ctx* c, const St* U) {
    if (c->viscous) return ns_edge(c, U);
    const int threads = c->edge_threads;
    if (c->edge_pair == 2) {  // a warp covers 32 / NG slots per iteration; fixed 128-thread blocks
      constexpr int spw = 32 / V::NG, tpb = dgm::kEdgeStagedThreads;
      const int64_t warps = (c->n_int + c->n_bnd + spw - 1) / spw;
      const int64_t full = std::max<int64_t>(1, (warps * 32 + tpb - 1) / tpb);
      const int blocks = (int)(c->edge_blocks > 0 ? std::min<int64_t>(c->edge_blocks, full) : full);
      dgm::k_edge_flux_staged<P, T, St><<<blocks, tpb, 0, c->stream>>>(kp_of<P, T>(c), U, Fx(c->F));
    } else if (c->edge_pair == 1) {  // a warp covers 16 slots per iteration
      const int64_t warps = (c->n_int + c->n_bnd + 15) / 16;
      const int64_t full = std::max<int64_t>(1, (warps * 32 + threads - 1) / threads);
      const int blocks = (int)(c->edge_blocks > 0 ? std::min<int64_t>(c->edge_blocks, full) : full);
      dgm::k_edge_flux_pair<P, T, St><<<blocks, threads, 0, c->stream>>>(kp_of<P, T>(c), U, Fx(c->F));
    } else {
      const int64_t total = (c->n_int + c->n_bnd) * V::NG;
      const int64_t full = std::max<int64_t>(1, (total + threads - 1) / threads);
      const int blocks = (int)(c->edge_blocks > 0 ? std::min<int64_t>(c->edge_blocks, full) : full);
      if (c->edge_pair == 3)  // the point form at 64 registers
        dgm::k_edge_flux_r64<P, T, St><<<blocks, threads, 0, c->stream>>>(kp_of<P, T>(c), U, Fx(c->F));
      else
        dgm::k_edge_flux<P, T, St><<<blocks, threads, 0, c->stream>>>(kp_of<P, T>(c), U, Fx(c->F));
    }
    CK(cudaGetLastError());
    return DGM_OK;
  }

  template <int MODE, int SPLIT>
  static int element_tc(dgm_ctx* c, const float* Uin, const float* Ubase, float* Uout, const float* Rin,
                        float* Rout) {
    auto kern = dgm::k_element_tc<P, MODE, SPLIT>;
    const int smem = (int)dgm::tc::Plan<P, SPLIT>::bytes;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // Residency is left to the hardware: registers and shared memory allow several CTAs per SM,
    // and tensor memory at most 512 / 32 = 16 (the thread limit gives the same), so the grid is
    // the tile count capped at 16 CTAs per SM; every CTA loops over its share of tiles.
    const int64_t tiles = (c->ne + dgm::tc::kElems - 1) / dgm::tc::kElems;
    const int64_t cap = (int64_t)(512 / dgm::tc::kTmemCols) * c->num_sms;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, cap));
    kern<<<blocks, dgm::tc::kThreads, smem, c->stream>>>(kp_of<P, float>(c), Uin, Ubase,
                                                         static_cast<const float*>(c->F), Uout, Rin, Rout);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  template <int MODE>
  static int element(dgm_ctx* c, const St* Uin, const St* Ubase, St* Uout, const St* Rin, St* Rout) {
    if constexpr (std::is_same<T, double>::value && std::is_same<St, double>::value) {
      if (c->viscous) {  // the element pass with the viscous volume term
        const int threads = c->elem_threads, per_block = threads / 4;
        const int blocks = (int)std::max<int64_t>(1, (c->ne + per_block - 1) / per_block);
        dgm::k_element_ns<P, MODE><<<blocks, threads, 0, c->stream>>>(kp_of<P, T>(c), ns_of<P>(c), Uin, Ubase,
                                                                      Fx(c->F), Uout, Rin, Rout);
        CK(cudaGetLastError());
        return DGM_OK;
      }
    }
    if constexpr (std::is_same<T, float>::value && std::is_same<St, float>::value) {
      if (c->tc_split == 1) return element_tc<MODE, 1>(c, Uin, Ubase, Uout, Rin, Rout);
      if (c->tc_split == 3) return element_tc<MODE, 3>(c, Uin, Ubase, Uout, Rin, Rout);
    }
    const int threads = c->elem_threads;  // warps of 8 elements, 4 threads (variables) per element
    const int per_block = threads / 4;
    const int blocks = (int)std::max<int64_t>(1, (c->ne + per_block - 1) / per_block);
    dgm::k_element<P, T, MODE, St><<<blocks, threads, 0, c->stream>>>(kp_of<P, T>(c), Uin, Ubase, Fx(c->F), Uout, Rin,
                                                                   Rout);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int limiter(dgm_ctx* c, St* U) {
    if (!c->limiter) return DGM_OK;
    const int dblocks = (int)std::max<int64_t>(1, (c->ld / 32 + dgm::kDetectWarps - 1) / dgm::kDetectWarps);
    if (c->lim_staged)
      dgm::k_lim_detect<P, T, true, St><<<dblocks, dgm::kDetectThreads, 0, c->stream>>>(kp_of<P, T>(c), U, c->t0, c->status,
                                                                                   c->wl1, c->pend, c->order);
    else
      dgm::k_lim_detect<P, T, false, St><<<dblocks, dgm::kDetectThreads, 0, c->stream>>>(kp_of<P, T>(c), U, c->t0,
                                                                                    c->status, c->wl1, c->pend, c->order);
    CK(cudaGetLastError());
    cudaLaunchConfig_t cfg = {};
    const int full = c->coop_blocks[c->lim_queue];
    cfg.gridDim = dim3(c->lim_one_per_sm ? std::min(full, c->num_sms) : full);
    cfg.blockDim = dim3(dgm::kLimiterWarps * 32);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    auto kern = c->lim_queue ? dgm::k_limiter<P, T, true, St> : dgm::k_limiter<P, T, false, St>;
    CK(cudaLaunchKernelEx(&cfg, kern, kp_of<P, T>(c), U, (const unsigned char*)c->t0, c->status, c->work,
                          (const int*)c->wl1, (const int*)c->pend));
    return DGM_OK;
  }

  static int step_head(dgm_ctx* c, const St* U) {
    const int threads = 256;
    const int blocks = (int)std::max<int64_t>(1, (c->ne + threads - 1) / threads);
    dgm::k_step_head<P, T, St><<<blocks, threads, 0, c->stream>>>(kp_of<P, T>(c), U);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int time_step(dgm_ctx* c, const St* U) {
    const int threads = 256;
    const int blocks = (int)std::max<int64_t>(1, (c->ne + threads - 1) / threads);
    dgm::k_time_step<P, T, St><<<blocks, threads, 0, c->stream>>>(kp_of<P, T>(c), U);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int diagnostics(dgm_ctx* c, const St* R) {
    dgm::k_diagnostics<P, T, St><<<(int)c->inst.size(), 256, 0, c->stream>>>(kp_of<P, T>(c), S(c->U), R, c->d_elem_rng,
                                                                          c->d_bslot_rng, c->d_diag);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  // One SSP-RK3 step on the resident state (rk3.rs:7-26); dt is read from the control blocks.
  static int rk3(dgm_ctx* c, St* Rout) {
    St *U = S(c->U), *U1 = S(c->U1), *U2 = S(c->U2);
    int st;
    if ((st = edge_flux(c, U))) return st;
    if ((st = element<1>(c, U, nullptr, U1, nullptr, nullptr))) return st;
    if ((st = limiter(c, U1))) return st;
    if ((st = edge_flux(c, U1))) return st;
    if ((st = element<2>(c, U1, U, U2, nullptr, nullptr))) return st;
    if ((st = limiter(c, U2))) return st;
    if ((st = edge_flux(c, U2))) return st;
    if ((st = element<3>(c, U2, U, U, nullptr, Rout))) return st;
    return limiter(c, U);
  }

  // One iteration of time_march (temporal_disc.rs:22-33) for every instance, on the device.
  static int step(dgm_ctx* c, St* Rout) {
    const int n = (int)c->inst.size();
    const int tb = 128, nblk = (n + tb - 1) / tb;
    int st;
    if ((st = step_head(c, S(c->U)))) return st;
    if ((st = rk3(c, Rout))) return st;
    dgm::k_step_end<<<nblk, tb, 0, c->stream>>>(c->ic, n);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  // FP64 device array in the reference layout -> the state (FP32 contexts; FP64 copies directly)
  static int to_storage(dgm_ctx* c, const double* src, void* dst, int64_t elem_off, int64_t ne) {
    const long long n = (long long)ne * NEQ * V::NB;
    const int threads = 256;
    if constexpr (std::is_same<St, float>::value) {
      dgm::k_f64_to_f32<<<(int)((n + threads - 1) / threads), threads, 0, c->stream>>>(
          src, S(dst) + elem_off * NEQ * V::NB, n);
      CK(cudaGetLastError());
    }
    return DGM_OK;
  }
  static int cell_fields(dgm_ctx* c, int64_t i, double* dst) {
    const HostInst& h = c->inst[i];
    const int threads = 256;
    dgm::k_cell_fields<P, T, St><<<(int)((h.ne + threads - 1) / threads), threads, 0, c->stream>>>(
        kp_of<P, T>(c), S(c->U), (int)h.elem_off, (int)h.ne, dst);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  // WENO Gram matrices of the elements [e0, e0 + count)
  static int weno_gram(dgm_ctx* c, int64_t e0, int64_t count) {
    constexpr int NPAIR = V::NB * (V::NB + 1) / 2;
    const int64_t n = (int64_t)NPAIR * count;
    const int threads = 256;
    if (n > 0)
      dgm::k_weno_gram<P, T><<<(int)((n + threads - 1) / threads), threads, 0, c->stream>>>(kp_of<P, T>(c), c->gram,
                                                                                         (int)e0, (int)count);
    CK(cudaGetLastError());
    kp_of<P, T>(c).m.gram = c->gram;
    return DGM_OK;
  }

  static MeshDev& mesh(dgm_ctx* c) { return kp_of<P, T>(c).m; }

  static int project(dgm_ctx* c, int64_t i, const double q[NEQ]) {
    dgm::Projection<P> pr;
    for (int g = 0; g < V::NQ; ++g) {
      for (int b = 0; b < V::NB; ++b) pr.phi[g][b] = c->proj_phi[g * V::NB + b];
      pr.w[g] = c->proj_w[g];
    }
    for (int b = 0; b < V::NB; ++b) pr.mass[b] = c->proj_mass[b];
    for (int v = 0; v < NEQ; ++v) pr.q[v] = q[v];
    const HostInst& h = c->inst[i];
    const int threads = 256;
    dgm::k_project_uniform<P, St><<<(int)((h.ne + threads - 1) / threads), threads, 0, c->stream>>>(
        pr, kp_of<P, T>(c).m.jac, S(c->U), (int)h.elem_off, (int)h.ne, (int)c->ld);
    CK(cudaGetLastError());
    return DGM_OK;
  }
  static int from_storage(dgm_ctx* c, const void* src, double* dst, int64_t elem_off, int64_t ne) {
    const long long n = (long long)ne * NEQ * V::NB;
    const int threads = 256;
    if constexpr (std::is_same<St, float>::value) {
      dgm::k_f32_to_f64<<<(int)((n + threads - 1) / threads), threads, 0, c->stream>>>(
          static_cast<const float*>(src) + elem_off * NEQ * V::NB, dst, n);
      CK(cudaGetLastError());
    }
    return DGM_OK;
  }

  static int occupancy(dgm_ctx* c) {
    int per_sm[2] = {0, 0};
    const int threads = dgm::kLimiterWarps * 32;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], dgm::k_limiter<P, T, false, St>, threads, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], dgm::k_limiter<P, T, true, St>, threads, 0));
    const int64_t want = std::max<int64_t>(1, (c->ne + 32 * dgm::kLimiterWarps - 1) / (32 * dgm::kLimiterWarps));
    for (int q = 0; q < 2; ++q)
      c->coop_blocks[q] = (int)std::min<int64_t>((int64_t)std::max(1, per_sm[q]) * c->num_sms, want);
    return DGM_OK;
  }

  static int fill_tables(dgm_ctx* c, const dgm_tables_desc* t) {
    c->kparams.assign(sizeof(KParams<P, T>), 0);
    auto& kp = kp_of<P, T>(c);
    auto& tb = kp.t;
    auto& td = kp.d;
    const int NB = V::NB, NQ = V::NQ, NG = V::NG, NK = V::NK;
    const int nk_in = t->n_deriv_keys;
    if (nk_in < NK) return DGM_BAD_ARG;
    for (int q = 0; q < NQ; ++q)
      for (int b = 0; b < NB; ++b) {
        tb.phi_cell[q][b] = T(t->phi_cell[q * NB + b]);
        tb.dxi[q][b] = T(t->dphi_cell_ref[((size_t)q * NB + b) * nk_in + 0]);
        tb.deta[q][b] = T(t->dphi_cell_ref[((size_t)q * NB + b) * nk_in + 1]);
        for (int k = 0; k < NK; ++k) td.dref[q][b][k] = t->dphi_cell_ref[((size_t)q * NB + b) * nk_in + k];
      }
    for (int k = 0; k < 3; ++k)
      for (int g = 0; g < NG; ++g)
        for (int b = 0; b < NB; ++b) {
          tb.phi_edge[k][g][b] = T(t->phi_edge[(k * NG + g) * NB + b]);
          td.phi_edge[k][g][b] = t->phi_edge[(k * NG + g) * NB + b];
        }
    for (int q = 0; q < NQ; ++q) {
      tb.cell_w[q] = T(t->cell_weights[q]);
      td.cell_w[q] = t->cell_weights[q];
    }
    for (int g = 0; g < NG; ++g) {
      tb.edge_w[g] = T(t->edge_weights[g]);
      td.edge_w[g] = t->edge_weights[g];
    }
    for (int b = 0; b < NB; ++b) tb.inv_mass[b] = T(1.0 / t->mass_diag[b]);
    c->proj_phi.assign(t->phi_cell, t->phi_cell + NQ * NB);
    c->proj_w.assign(t->cell_weights, t->cell_weights + NQ);
    c->proj_mass.assign(t->mass_diag, t->mass_diag + NB);
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
    kp.ic = c->ic;
    return DGM_OK;
  }

  static int set_mesh(dgm_ctx* c, const MeshDev& md) {
    kp_of<P, T>(c).m = md;
    return DGM_OK;
  }

  // NsParams<P> from the reference-space edge derivative table [3][NG][NB][2] and the flow
  // parameters; the global-lift array is allocated once.
  static int set_viscous(dgm_ctx* c, double prandtl_number, double gas_constant, const double* dphi_edge) {
    c->nsparams.assign(sizeof(dgm::NsParams<P>), 0);
    auto& ns = ns_of<P>(c);
    for (int k = 0; k < 3; ++k)
      for (int g = 0; g < V::NG; ++g)
        for (int b = 0; b < V::NB; ++b)
          for (int d = 0; d < 2; ++d) ns.dphi_edge[k][g][b][d] = dphi_edge[((k * V::NG + g) * V::NB + b) * 2 + d];
    for (int b = 0; b < V::NB; ++b) ns.mass[b] = c->proj_mass[b];
    ns.hp = c->hcr / prandtl_number;
    ns.rgas = gas_constant;
    if (!c->ns_lift) {
      const int st = dev_alloc(c, &c->ns_lift, (size_t)c->ld * 2 * NEQ * V::NB);
      if (st) return st;
    }
    ns.lift = c->ns_lift;
    return DGM_OK;
  }
};

template <class F>
int dispatch(dgm_ctx* c, F&& f) {
  if (c->prec_mode == 4) {  // FP32 arithmetic on an FP64 state
    switch (c->P) {
      case 1: return f(Ops<1, float, double>{});
      case 2: return f(Ops<2, float, double>{});
      case 3: return f(Ops<3, float, double>{});
    }
    return DGM_BAD_ARG;
  }
  if (c->prec == 0) {
    switch (c->P) {
      case 1: return f(Ops<1, double>{});
      case 2: return f(Ops<2, double>{});
      case 3: return f(Ops<3, double>{});
    }
  } else {
    switch (c->P) {
      case 1: return f(Ops<1, float>{});
      case 2: return f(Ops<2, float>{});
      case 3: return f(Ops<3, float>{});
    }
  }
  return DGM_BAD_ARG;
}

// Bytes of one state coefficient (storage) and of one edge-flux value (arithmetic).
size_t elem_bytes(const dgm_ctx* c) { return (c->prec == 0 || c->prec_mode == 4) ? sizeof(double) : sizeof(float); }
size_t flux_bytes(const dgm_ctx* c) { return c->prec == 0 ? sizeof(double) : sizeof(float); }

int read_control(dgm_ctx* c, Control* h, std::vector<InstCtl>* hi) {
  CK(cudaMemcpyAsync(h, c->ctl, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
  if (hi) {
    hi->resize(c->inst.size());
    CK(cudaMemcpyAsync(hi->data(), c->ic, sizeof(InstCtl) * c->inst.size(), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

// Pulls the device clocks/statuses into the host mirrors; resets the device status words and
// returns the first status raised since the last call (DGM_OK if none).
int collect_status(dgm_ctx* c) {
  Control h;
  std::vector<InstCtl> hi;
  int st = read_control(c, &h, &hi);
  if (st) return st;
  for (size_t i = 0; i < c->inst.size(); ++i) {
    c->inst[i].t = hi[i].t;
    c->inst[i].step = hi[i].step;
    if (hi[i].status) {
      c->inst[i].status = hi[i].status;
      c->inst[i].err_where = hi[i].err_where;
    }
  }
  c->last_troubled = h.troubled;
  c->last_waves = h.waves;
  if (h.status != 0) {
    c->err_where = h.err_where;
    const int zero = 0;
    CK(cudaMemcpyAsync(&c->ctl->status, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (h.status == dgm::ST_TIMEOUT || h.status == dgm::ST_LIST_OVERFLOW) {
      // a limiter pass that gave up (or dropped a worklist entry) may have left queue slots,
      // counters and a half-passed grid barrier behind: clear them all
      CK(cudaMemsetAsync(c->work, 0, sizeof(int) * std::max<int64_t>(c->ne, 1), c->stream));
      Control z = h;
      z.status = 0;
      z.t0_count = 0;
      z.unknown[0] = z.unknown[1] = 0;
      z.wl_count[0] = z.wl_count[1] = 0;
      z.wl1_count = z.pend_count = 0;
      z.bar_word = 0u;
      for (auto& q : z.lq) dgm::reset_queue(q);
      CK(cudaMemcpyAsync(c->ctl, &z, sizeof(Control), cudaMemcpyHostToDevice, c->stream));
    }
    for (size_t i = 0; i < c->inst.size(); ++i)
      if (hi[i].status) CK(cudaMemcpyAsync(&c->ic[i].status, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return h.status;
  }
  return DGM_OK;
}

int set_active(dgm_ctx* c, double dt, bool set_dt) {
  const int n = (int)c->inst.size();
  dgm::k_set_active<<<(n + 127) / 128, 128, 0, c->stream>>>(c->ctl, c->ic, n, dt, set_dt ? 1 : 0);
  CK(cudaGetLastError());
  return DGM_OK;
}

// Host state ([element][variable][basis], FP64) of instance i -> device state array dst: the
// device layout is the same element-major order, so an FP64 state is one copy; an FP32 state goes
// through the FP64 staging buffer and a conversion.
int upload_state(dgm_ctx* c, int64_t i, const double* host, void* dst) {
  const HostInst& h = c->inst[i];
  const size_t n = (size_t)h.ne * NEQ * c->nb;
  if (elem_bytes(c) == sizeof(double)) {
    CK(cudaMemcpyAsync(static_cast<double*>(dst) + (size_t)h.elem_off * NEQ * c->nb, host, n * sizeof(double),
                       cudaMemcpyHostToDevice, c->stream));
    return DGM_OK;
  }
  CK(cudaMemcpyAsync(c->stage, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return dispatch(c, [&](auto ops) { return decltype(ops)::to_storage(c, c->stage, dst, h.elem_off, h.ne); });
}

int download_state(dgm_ctx* c, int64_t i, const void* src, double* host) {
  const HostInst& h = c->inst[i];
  const size_t n = (size_t)h.ne * NEQ * c->nb;
  if (elem_bytes(c) == sizeof(double)) {
    CK(cudaMemcpyAsync(host, static_cast<const double*>(src) + (size_t)h.elem_off * NEQ * c->nb, n * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream));
  } else {
    int st = dispatch(c, [&](auto ops) { return decltype(ops)::from_storage(c, src, c->stage, h.elem_off, h.ne); });
    if (st) return st;
    CK(cudaMemcpyAsync(host, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));  // the host reads the array; the staging buffer is reused
  return DGM_OK;
}

// Host clocks and loop bounds -> device control blocks (statuses and dt are kept).
int write_clock(dgm_ctx* c) {
  Control h;
  std::vector<InstCtl> hi;
  int st = read_control(c, &h, &hi);
  if (st) return st;
  for (size_t i = 0; i < c->inst.size(); ++i) {
    hi[i].t = c->inst[i].t;
    hi[i].step = c->inst[i].step;
    hi[i].final_time = c->inst[i].final_time;
    hi[i].final_step = c->inst[i].final_step;
    hi[i].cfl = c->inst[i].cfl;
    hi[i].status = c->inst[i].status;
    hi[i].err_where = c->inst[i].err_where;
    const double start = 1.0e10;  // the time step's start value, temporal_disc.rs:59
    std::memcpy(&hi[i].dt_bits, &start, sizeof(double));
  }
  h.head_done = 0u;
  CK(cudaMemcpyAsync(c->ic, hi.data(), sizeof(InstCtl) * hi.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(&c->ctl->head_done, &h.head_done, sizeof(unsigned int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->limits_dirty = false;
  c->dt_dirty = false;
  return DGM_OK;
}

int mixed_step(dgm_ctx* c, int with_residual);

// One time-march iteration of every instance, enqueued on the context's stream.
int step_once(dgm_ctx* c, int with_residual) {
  if (c->mixed) return mixed_step(c, with_residual);
  return dispatch(c, [&](auto ops) {
    using O = decltype(ops);
    return O::step(c, with_residual ? O::S(c->R) : nullptr);
  });
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
  for (int i = 0; i < n && st == DGM_OK; ++i) st = step_once(c, with_residual);
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

// Drop the captured step graphs (they hold the launch configuration of their capture).
void reset_graphs(dgm_ctx* c) {
  for (auto& row : c->graph)
    for (auto& g : row)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
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
      st = step_once(c, with_residual);
      if (st) return st;
      n -= 1;
    }
  }
  return DGM_OK;
}

// Union mesh of all instances.  Instance i owns fixed ranges of the union's arrays -- elements
// [elem_off, elem_off + elem_cap), internal edge slots [int_off, int_off + int_cap), boundary
// edge slots [n_int + bnd_off, n_int + bnd_off + bnd_cap) and patches [patch_off, patch_off +
// patch_cap) -- with its mesh's entries first (internal edges in Mesh::internal_edge_indices order,
// boundary edges in edge-id order) and padding after.  A context created with capacities above
// its meshes' sizes (dgm_create_batch_slots) can later take a different mesh into an instance's
// ranges (dgm_instance_replace).  Padding elements and every padding slot belong to a "dead"
// instance (index n_inst, never stepping: its loop bounds are zero), so every kernel skips them;
// padding slots refer to a null element (the last element of the union, also dead).  Without
// padding the layout is the plain concatenation, with no dead instance and no null element.

// One instance's part of the union mesh, in its capacity ranges (element-indexed rows have length
// elem_cap; element, slot and patch ids are global).
struct InstArrays {
  std::vector<double> jac, hmin, h15, dinv;  // dinv: [4][elem_cap]
  std::vector<int> face, nbr, inst;          // face, nbr: [3][elem_cap]
  std::vector<int2> ie_lr;
  std::vector<int> ie_ic;
  std::vector<double4> ie_geo;
  std::vector<int> be_elem, be_info;
  std::vector<double4> be_geo;
  std::vector<double4> patch_q;
  std::vector<int64_t> int_ref, bnd_ref;     // reference edge id of each slot (-1: padding)
};

int64_t boundary_edge_count(const dgm_mesh_desc* m) {
  int64_t n = 0;
  for (int64_t d = 0; d < m->n_edges; ++d) n += m->edge_elements[2 * d + 1] == -1 ? 1 : 0;
  return n;
}

// Builds instance i's arrays from mesh m into its ranges (HostInst offsets and capacities must be
// set, and c->n_int, c->dead_inst, c->null_elem).  Validates every index against process_mesh's
// conventions before anything reaches the device.
int fill_instance(const dgm_ctx* c, int i, const dgm_mesh_desc* m, InstArrays& a) {
  const HostInst& hi = c->inst[i];
  auto in_range = [](int64_t v, int64_t n) { return v >= 0 && v < n; };
  if (m->n_elements <= 0 || m->n_edges <= 0 || m->n_vertices <= 0 || m->n_patches < 0) return DGM_BAD_ARG;
  if (m->n_elements > hi.elem_cap || m->n_internal_edges > hi.int_cap || boundary_edge_count(m) > hi.bnd_cap ||
      m->n_patches > hi.patch_cap)
    return DGM_BAD_ARG;
  const int64_t ned = m->n_edges, nei = m->n_elements, cap = hi.elem_cap, eo = hi.elem_off;
  const int dead = c->dead_inst, null_e = (int)c->null_elem;
  a.jac.assign(cap, 1.0);
  a.hmin.assign(cap, 1.0);
  a.h15.assign(cap, 1.0);
  a.dinv.assign(4 * cap, 0.0);
  a.face.assign(3 * cap, (int)((hi.int_cap > 0 ? hi.int_off : c->n_int + hi.bnd_off) << 1));
  a.nbr.assign(3 * cap, -1);
  a.inst.assign(cap, dead);
  a.ie_lr.assign(hi.int_cap, make_int2(null_e, null_e));
  a.ie_ic.assign(hi.int_cap, 0);
  a.ie_geo.assign(hi.int_cap, make_double4(0.0, 0.0, 0.0, 0.0));
  a.int_ref.assign(hi.int_cap, -1);
  a.be_elem.assign(hi.bnd_cap, null_e);
  a.be_info.assign(hi.bnd_cap, (int)(hi.patch_off << 3));
  a.be_geo.assign(hi.bnd_cap, make_double4(0.0, 0.0, 0.0, 0.0));
  a.bnd_ref.assign(hi.bnd_cap, -1);
  a.patch_q.assign(std::max<int64_t>(hi.patch_cap, 0), make_double4(0.0, 0.0, 0.0, 0.0));
  std::vector<int64_t> slot_of(ned, -1);
  // internal edges
  for (int64_t k = 0; k < m->n_internal_edges; ++k) {
    const int64_t d = m->internal_edges[k];
    if (!in_range(d, ned) || slot_of[d] >= 0) return DGM_BAD_ARG;
    const int64_t L = m->edge_elements[2 * d], R = m->edge_elements[2 * d + 1];
    const int64_t il = m->edge_in_cell[2 * d], ir = m->edge_in_cell[2 * d + 1];
    if (!in_range(L, nei) || !in_range(R, nei) || L == R || !in_range(il, 3) || !in_range(ir, 3)) return DGM_BAD_ARG;
    slot_of[d] = hi.int_off + k;
    a.int_ref[k] = d;
    a.ie_lr[k] = make_int2((int)(eo + L), (int)(eo + R));
    a.ie_ic[k] = (int)(il | (ir << 2));
    const double jd = m->edge_jacob_det[d];
    a.ie_geo[k] = make_double4(m->edge_normal[2 * d], m->edge_normal[2 * d + 1], 0.5 * jd, jd);
  }
  // boundary edges, in edge-id order
  int64_t nbs = 0;
  for (int64_t d = 0; d < ned; ++d) {
    if (m->edge_elements[2 * d + 1] != -1) continue;
    const int64_t e = m->edge_elements[2 * d], k = m->edge_in_cell[2 * d], patch = m->edge_patch[d];
    if (!in_range(e, nei) || !in_range(k, 3) || !in_range(patch, m->n_patches)) return DGM_BAD_ARG;
    if (slot_of[d] >= 0) return DGM_BAD_ARG;
    slot_of[d] = c->n_int + hi.bnd_off + nbs;
    a.bnd_ref[nbs] = d;
    const int type = m->patch_type[patch];
    if (type != DGM_WALL && type != DGM_FARFIELD) return DGM_BAD_ARG;
    a.be_elem[nbs] = (int)(eo + e);
    a.be_info[nbs] = (int)(k | (type << 2) | ((hi.patch_off + patch) << 3));
    // outward orientation, boundary_condition.rs:22-28
    const bool same = m->elem_vertices[3 * e + k] == m->edge_vertices[2 * d];
    const double nx = same ? m->edge_normal[2 * d] : -m->edge_normal[2 * d];
    const double ny = same ? m->edge_normal[2 * d + 1] : -m->edge_normal[2 * d + 1];
    const double jd = m->edge_jacob_det[d];
    a.be_geo[nbs] = make_double4(nx, ny, 0.5 * jd, jd);
    ++nbs;
  }
  // far-field conserved state, boundary_condition.rs:50-55
  for (int64_t p = 0; p < m->n_patches; ++p) {
    const double* bq = &m->patch_quantity[4 * p];
    a.patch_q[p] = make_double4(bq[0], bq[0] * bq[1], bq[0] * bq[2],
                                bq[3] / (c->hcr - 1.0) + 0.5 * bq[0] * (bq[1] * bq[1] + bq[2] * bq[2]));
  }
  std::vector<unsigned char> in_list(nei, 0);
  for (int64_t k = 0; k < m->n_boundary_elements; ++k) {
    const int64_t e = m->boundary_elements[k];
    if (!in_range(e, nei)) return DGM_BAD_ARG;
    in_list[e] = 1;
  }
  auto X = [&](int64_t v) { return m->vertex_xy[2 * v]; };
  auto Y = [&](int64_t v) { return m->vertex_xy[2 * v + 1]; };
  for (int64_t e = 0; e < nei; ++e) {
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
        a.nbr[k * cap + e] = -1;
      } else {
        const bool same = m->elem_vertices[3 * e + k] == m->edge_vertices[2 * d];
        if (m->edge_elements[2 * d] == e && same && m->edge_in_cell[2 * d] == k) side = 0;
        else if (m->edge_elements[2 * d + 1] == e && !same && m->edge_in_cell[2 * d + 1] == k) side = 1;
        else return DGM_BAD_ARG;  // orientation inconsistent with process_mesh's left/right rule
        const int64_t other = m->edge_elements[2 * d + (side ? 0 : 1)];
        if (m->elem_neighbours[3 * e + k] != other) return DGM_BAD_ARG;
        a.nbr[k * cap + e] = (int)(eo + other);
      }
      a.face[k * cap + e] = (int)((slot_of[d] << 1) | side);
    }
    // every element is in exactly one of the internal / boundary element lists
    if (has_boundary != (in_list[e] != 0)) return DGM_BAD_ARG;
    const double J = m->elem_jacob_det[e];
    const int64_t v1 = m->elem_vertices[3 * e], v2 = m->elem_vertices[3 * e + 1], v3 = m->elem_vertices[3 * e + 2];
    if (!in_range(v1, m->n_vertices) || !in_range(v2, m->n_vertices) || !in_range(v3, m->n_vertices))
      return DGM_BAD_ARG;
    a.jac[e] = J;
    a.inst[e] = i;
    // compute_dphi inverse Jacobian, mesh.rs:93-100
    a.dinv[0 * cap + e] = (Y(v3) - Y(v1)) / J;
    a.dinv[1 * cap + e] = -(X(v3) - X(v1)) / J;
    a.dinv[2 * cap + e] = -(Y(v2) - Y(v1)) / J;
    a.dinv[3 * cap + e] = (X(v2) - X(v1)) / J;
    a.hmin[e] = m->elem_minimum_height[e];
    a.h15[e] = std::pow(m->elem_circumradius[e], 1.5);  // weno.rs:81 h.powf(1.5)
  }
  return DGM_OK;
}

// Instance ranges of the diagnostics: [2 n] (first element, element count) and (first boundary
// slot relative to n_int, boundary slot count) of each instance's mesh.
int upload_ranges(dgm_ctx* c) {
  const size_t n = c->inst.size();
  std::vector<int> er(2 * n), br(2 * n);
  for (size_t i = 0; i < n; ++i) {
    er[2 * i] = (int)c->inst[i].elem_off;
    er[2 * i + 1] = (int)c->inst[i].ne;
    br[2 * i] = (int)c->inst[i].bslot_off;
    br[2 * i + 1] = (int)c->inst[i].nb_slots;
  }
  if (!c->d_elem_rng) {
    int st;
    if ((st = dev_alloc(c, &c->d_elem_rng, 2 * n)) || (st = dev_alloc(c, &c->d_bslot_rng, 2 * n))) return st;
  }
  CK(cudaMemcpyAsync(c->d_elem_rng, er.data(), sizeof(int) * 2 * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_bslot_rng, br.data(), sizeof(int) * 2 * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));  // the host vectors go out of scope
  return DGM_OK;
}

int build_mesh(dgm_ctx* c, const dgm_mesh_desc* meshes, const dgm_slot_capacity* caps, int n_inst, MeshDev& md) {
  // capacity layout
  int64_t ne = 0, n_int = 0, n_bnd = 0, np = 0;
  bool padding = false;
  for (int i = 0; i < n_inst; ++i) {
    const dgm_mesh_desc* m = &meshes[i];
    if (m->n_elements <= 0 || m->n_edges <= 0 || m->n_vertices <= 0 || m->n_patches < 0) return DGM_BAD_ARG;
    const int64_t nbe = boundary_edge_count(m);
    HostInst& hi = c->inst[i];
    hi.elem_cap = caps ? caps[i].elements : m->n_elements;
    hi.int_cap = caps ? caps[i].internal_edges : m->n_internal_edges;
    hi.bnd_cap = caps ? caps[i].boundary_edges : nbe;
    hi.patch_cap = caps ? caps[i].patches : m->n_patches;
    if (hi.elem_cap < m->n_elements || hi.int_cap < m->n_internal_edges || hi.bnd_cap < nbe ||
        hi.patch_cap < m->n_patches || hi.elem_cap > (1ll << 30) || hi.int_cap > (1ll << 30) ||
        hi.bnd_cap > (1ll << 30) || hi.patch_cap > (1ll << 20))
      return DGM_BAD_ARG;
    padding = padding || hi.elem_cap > m->n_elements || hi.int_cap > m->n_internal_edges || hi.bnd_cap > nbe ||
              hi.patch_cap > m->n_patches;
    hi.elem_off = ne;
    hi.int_off = n_int;
    hi.bnd_off = n_bnd;
    hi.patch_off = np;
    hi.bslot_off = n_bnd;
    hi.ne = m->n_elements;
    hi.nb_slots = nbe;
    ne += hi.elem_cap;
    n_int += hi.int_cap;
    n_bnd += hi.bnd_cap;
    np += hi.patch_cap;
  }
  c->dead_inst = padding ? n_inst : 0;
  c->null_elem = padding ? ne : -1;
  if (padding) ne += 1;
  if (ne > (1ll << 30) || n_int + n_bnd > (1ll << 29)) return DGM_BAD_ARG;
  const int64_t ld = (ne + 31) / 32 * 32;
  c->ne = ne;
  c->ld = ld;
  c->np = np;
  c->n_int = n_int;
  c->n_bnd = n_bnd;
  c->padded = padding;
  std::vector<int64_t> slot_ref(n_int + n_bnd, -1);
  std::vector<int2> ie_lr(n_int);
  std::vector<int> ie_ic(n_int);
  std::vector<double4> ie_geo(n_int);
  std::vector<int> be_elem(n_bnd), be_info(n_bnd);
  std::vector<double4> be_geo(n_bnd);
  std::vector<double4> patch_q(std::max<int64_t>(1, np));
  std::vector<int> face(3 * ld, 0), nbr(3 * ld, -1), inst_of(ne, c->dead_inst);
  std::vector<double> jac(ne, 1.0), hmin(ne, 1.0), h15(ne, 1.0), dinv(4 * ld, 0.0);
  InstArrays a;
  for (int i = 0; i < n_inst; ++i) {
    int st = fill_instance(c, i, &meshes[i], a);
    if (st) return st;
    const HostInst& hi = c->inst[i];
    const int64_t eo = hi.elem_off, cap = hi.elem_cap;
    std::copy(a.jac.begin(), a.jac.end(), jac.begin() + eo);
    std::copy(a.hmin.begin(), a.hmin.end(), hmin.begin() + eo);
    std::copy(a.h15.begin(), a.h15.end(), h15.begin() + eo);
    std::copy(a.inst.begin(), a.inst.end(), inst_of.begin() + eo);
    for (int k = 0; k < 4; ++k) std::copy(a.dinv.begin() + k * cap, a.dinv.begin() + (k + 1) * cap, dinv.begin() + k * ld + eo);
    for (int k = 0; k < 3; ++k) {
      std::copy(a.face.begin() + k * cap, a.face.begin() + (k + 1) * cap, face.begin() + k * ld + eo);
      std::copy(a.nbr.begin() + k * cap, a.nbr.begin() + (k + 1) * cap, nbr.begin() + k * ld + eo);
    }
    std::copy(a.ie_lr.begin(), a.ie_lr.end(), ie_lr.begin() + hi.int_off);
    std::copy(a.ie_ic.begin(), a.ie_ic.end(), ie_ic.begin() + hi.int_off);
    std::copy(a.ie_geo.begin(), a.ie_geo.end(), ie_geo.begin() + hi.int_off);
    std::copy(a.int_ref.begin(), a.int_ref.end(), slot_ref.begin() + hi.int_off);
    std::copy(a.be_elem.begin(), a.be_elem.end(), be_elem.begin() + hi.bnd_off);
    std::copy(a.be_info.begin(), a.be_info.end(), be_info.begin() + hi.bnd_off);
    std::copy(a.be_geo.begin(), a.be_geo.end(), be_geo.begin() + hi.bnd_off);
    std::copy(a.bnd_ref.begin(), a.bnd_ref.end(), slot_ref.begin() + n_int + hi.bnd_off);
    std::copy(a.patch_q.begin(), a.patch_q.end(), patch_q.begin() + hi.patch_off);
  }
  // the limiter detection's visiting order of the warp batches (32 consecutive elements each):
  // breadth-first over the graph of batches that hold neighbouring elements, each connected piece
  // from its lowest unvisited batch, so that a batch and the batches holding its elements'
  // neighbours are processed at about the same time and their traces are mostly in cache.  Any
  // order gives the same results; this one only changes which loads hit.
  const int64_t nbatch = ld / 32;
  std::vector<int> order;
  {
    std::vector<int> deg(nbatch + 1, 0), adj;
    for (int64_t e = 0; e < ne; ++e)
      for (int k = 0; k < 3; ++k) {
        const int nb = nbr[k * ld + e];
        if (nb >= 0 && (nb >> 5) != (e >> 5)) ++deg[(e >> 5) + 1];
      }
    for (int64_t b = 0; b < nbatch; ++b) deg[b + 1] += deg[b];
    adj.resize(deg[nbatch]);
    std::vector<int> fill(deg.begin(), deg.end() - 1);
    for (int64_t e = 0; e < ne; ++e)
      for (int k = 0; k < 3; ++k) {
        const int nb = nbr[k * ld + e];
        if (nb >= 0 && (nb >> 5) != (e >> 5)) adj[fill[e >> 5]++] = nb >> 5;
      }
    order.reserve((size_t)nbatch);
    std::vector<unsigned char> seen((size_t)nbatch, 0);
    for (int64_t s0 = 0; s0 < nbatch; ++s0) {
      if (seen[s0]) continue;
      seen[s0] = 1;
      order.push_back((int)s0);
      for (size_t h = order.size() - 1; h < order.size(); ++h) {
        const int b = order[h];
        for (int j = deg[b]; j < deg[b + 1]; ++j)
          if (!seen[adj[j]]) {
            seen[adj[j]] = 1;
            order.push_back(adj[j]);
          }
      }
    }
  }
  md = MeshDev{};
  md.ne = (int)ne;
  md.ld = (int)ld;
  md.n_int = (int)n_int;
  md.n_bnd = (int)n_bnd;
  md.n_inst = n_inst + (padding ? 1 : 0);  // the dead instance is read from inst[] like the others
  int st;
  double *d_jac, *d_dinv, *d_hmin, *d_h15;
  int *d_face, *d_nbr, *d_inst, *d_ie_ic, *d_be_elem, *d_be_info;
  int2* d_ie_lr;
  double4 *d_ie_geo, *d_be_geo, *d_patch;
  int64_t* d_slot_ref;
  if ((st = upload(c, &d_jac, jac)) || (st = upload(c, &d_dinv, dinv)) || (st = upload(c, &d_hmin, hmin)) ||
      (st = upload(c, &d_h15, h15)) || (st = upload(c, &d_face, face)) || (st = upload(c, &d_nbr, nbr)) ||
      (st = upload(c, &d_inst, inst_of)) || (st = upload(c, &d_ie_lr, ie_lr)) || (st = upload(c, &d_ie_ic, ie_ic)) ||
      (st = upload(c, &d_ie_geo, ie_geo)) || (st = upload(c, &d_be_elem, be_elem)) ||
      (st = upload(c, &d_be_info, be_info)) || (st = upload(c, &d_be_geo, be_geo)) ||
      (st = upload(c, &d_patch, patch_q)) || (st = upload(c, &d_slot_ref, slot_ref)) ||
      (st = upload(c, &c->order, order)))
    return st;
  md.jac = d_jac;
  md.dinv = d_dinv;
  md.hmin = d_hmin;
  md.h15 = d_h15;
  md.face = d_face;
  md.nbr = d_nbr;
  md.inst = d_inst;
  md.ie_lr = d_ie_lr;
  md.ie_ic = d_ie_ic;
  md.ie_geo = d_ie_geo;
  md.be_elem = d_be_elem;
  md.be_info = d_be_info;
  md.be_geo = d_be_geo;
  md.patch_q = d_patch;
  md.slot_ref = d_slot_ref;
  if ((st = upload_ranges(c))) return st;
  int64_t mx = 0;
  for (auto& h : c->inst) mx = std::max(mx, h.elem_cap);
  c->max_inst_ne = mx;
  return DGM_OK;
}

bool variant_ok(const dgm_tables_desc* t) {
  const int P = t->order;
  return (P == 1 && t->n_basis == 3 && t->n_cell_gp == 3 && t->n_edge_gp == 2) ||
         (P == 2 && t->n_basis == 6 && t->n_cell_gp == 6 && t->n_edge_gp == 3) ||
         (P == 3 && t->n_basis == 10 && t->n_cell_gp == 12 && t->n_edge_gp == 4);
}

dgm_ctx* create(int n_inst, const dgm_mesh_desc* meshes, const dgm_slot_capacity* caps, const dgm_tables_desc* tables,
                const dgm_params* params, int32_t* status, cudaStream_t shared_stream = nullptr) {
  int32_t dummy;
  if (!status) status = &dummy;
  if (n_inst < 1 || !meshes || !tables || !params) {
    *status = DGM_BAD_ARG;
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || params->device < 0 || params->device >= ndev) {
    cudaGetLastError();
    *status = DGM_NO_DEVICE;
    return nullptr;
  }
  if (!variant_ok(tables) || params->precision < 0 || params->precision > 4) {
    *status = DGM_BAD_ARG;
    return nullptr;
  }
  for (int i = 1; i < n_inst; ++i)
    if (params[i].hcr != params[0].hcr) {  // the gas constants are shared by the whole context
      *status = DGM_BAD_ARG;
      return nullptr;
    }
  auto* c = new dgm_ctx();
  c->device = params->device;
  c->P = tables->order;
  c->nb = tables->n_basis;
  c->nq = tables->n_cell_gp;
  c->ng = tables->n_edge_gp;
  c->prec_mode = params->precision;
  c->prec = params->precision == 0 ? 0 : 1;
  c->tc_split = params->precision == 2 ? 1 : (params->precision == 3 ? 3 : 0);
  c->hcr = params->hcr;
  c->limiter = params->limiter ? 1 : 0;
  c->inst.resize(n_inst);
  for (int i = 0; i < n_inst; ++i) {
    c->inst[i].cfl = params[i].cfl;
    c->inst[i].final_time = params[i].final_time;
    c->inst[i].final_step = params[i].final_step;
  }
  auto fail = [&](int st) {
    *status = st;
    dgm_destroy(c);
    return (dgm_ctx*)nullptr;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(DGM_NO_DEVICE);
  if (cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess)
    return fail(DGM_NO_DEVICE);
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
  if (!coop) return fail(DGM_NO_DEVICE);
  if (shared_stream) {
    c->stream = shared_stream;
    c->owns_stream = false;
  } else if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    return fail(DGM_CUDA_ERROR);
  }
  c->pool = pool_acquire(c->device);
  if (!c->pool) return fail(DGM_CUDA_ERROR);
  int st;
  // one more instance control block than instances: the dead instance of padded contexts (all
  // zero: never stepping)
  if ((st = dev_alloc(c, &c->ctl, 1)) || (st = dev_alloc(c, &c->ic, (size_t)n_inst + 1))) return fail(st);
  if (cudaMemsetAsync(c->ctl, 0, sizeof(Control), c->stream) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  if (cudaMemsetAsync(c->ic, 0, sizeof(InstCtl) * (n_inst + 1), c->stream) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  st = dispatch(c, [&](auto ops) { return decltype(ops)::fill_tables(c, tables); });
  if (st) return fail(st);
  MeshDev md;
  if ((st = build_mesh(c, meshes, caps, n_inst, md))) return fail(st);
  dispatch(c, [&](auto ops) { return decltype(ops)::set_mesh(c, md); });
  const size_t n_state = (size_t)NEQ * c->nb * c->ld;
  const size_t n_flux = (size_t)(c->n_int + c->n_bnd) * c->ng * 4;
  const size_t eb = elem_bytes(c);
  if ((st = dev_alloc_bytes(c, &c->U, n_state * eb)) || (st = dev_alloc_bytes(c, &c->U1, n_state * eb)) ||
      (st = dev_alloc_bytes(c, &c->U2, n_state * eb)) || (st = dev_alloc_bytes(c, &c->R, n_state * eb)) ||
      (st = dev_alloc_bytes(c, &c->F, n_flux * flux_bytes(c))) ||
      (st = dev_alloc(c, &c->stage, (size_t)c->max_inst_ne * NEQ * c->nb)) ||
      (st = dev_alloc(c, &c->t0, (size_t)c->ne)) || (st = dev_alloc(c, &c->status, (size_t)c->ne)) ||
      (st = dev_alloc(c, &c->work, (size_t)c->ne)) || (st = dev_alloc(c, &c->wl1, (size_t)c->ne * dgm::kEntryInts)) ||
      (st = dev_alloc(c, &c->pend, (size_t)c->ne)) || (st = dev_alloc(c, &c->d_diag, (size_t)n_inst * 8)))
    return fail(st);
  for (void* p : {c->U, c->U1, c->U2, c->R})
    if (cudaMemsetAsync(p, 0, n_state * eb, c->stream) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  // the limiter's queue slots are zero between passes (each consumer clears its slot)
  if (cudaMemsetAsync(c->work, 0, sizeof(int) * std::max<int64_t>(c->ne, 1), c->stream) != cudaSuccess)
    return fail(DGM_CUDA_ERROR);
  if (c->limiter) {
    if ((st = dev_alloc(c, &c->gram, (size_t)(c->nb * (c->nb + 1) / 2) * c->ld))) return fail(st);
    if ((st = dispatch(c, [&](auto ops) { return decltype(ops)::weno_gram(c, 0, c->ne); }))) return fail(st);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  }
  if (cudaMemsetAsync(c->status, 0, (size_t)c->ne * sizeof(unsigned int), c->stream) != cudaSuccess)
    return fail(DGM_CUDA_ERROR);
  if ((st = dispatch(c, [&](auto ops) { return decltype(ops)::occupancy(c); }))) return fail(st);
  c->graph_steps = (int)kGraphSteps;
  if ((st = write_clock(c))) return fail(st);
  *status = DGM_OK;
  return c;
}


// ---------------------------------------------------------------------------------------------
// Mixed batches: one child context per order (its own union mesh, tables and arrays), one stream,
// and one launch per kernel of the step over all children (dgm_mixed.cuh).
// ---------------------------------------------------------------------------------------------
constexpr int kMixedEdgeThreads = 128, kMixedElemThreads = 128;

template <typename T, int MASK, typename St = T>
struct MixOps {
  using M = dgm::Mixed<T, MASK, St>;
  static St* S(void* p) { return static_cast<St*>(p); }
  static T* Fx(void* p) { return static_cast<T*>(p); }

  static void base(dgm_ctx* p, M& mp) {
    std::memset(static_cast<void*>(&mp), 0, sizeof(M));
    for (int g = 0; g < 3; ++g) {
      dgm_ctx* k = p->kids[g];
      if (!k) continue;
      if constexpr ((MASK & 1) != 0)
        if (g == 0) std::memcpy(static_cast<void*>(&mp.k1), k->kparams.data(), sizeof(mp.k1));
      if constexpr ((MASK & 2) != 0)
        if (g == 1) std::memcpy(static_cast<void*>(&mp.k2), k->kparams.data(), sizeof(mp.k2));
      if constexpr ((MASK & 4) != 0)
        if (g == 2) std::memcpy(static_cast<void*>(&mp.k3), k->kparams.data(), sizeof(mp.k3));
      auto& a = mp.g[g];
      a.n_inst = (int)k->inst.size();
      a.F = Fx(k->F);
      a.t0 = k->t0;
      a.status = k->status;
      a.wl1 = k->wl1;
      a.pend = k->pend;
      a.order = k->order;
    }
  }

  static int blocks_total(const M& mp) { return std::max(1, mp.g[0].blocks + mp.g[1].blocks + mp.g[2].blocks); }

  // which: 0 = U, 1 = U1, 2 = U2
  static St* arr(dgm_ctx* k, int which) { return S(which == 0 ? k->U : which == 1 ? k->U1 : k->U2); }

  static int step_head(dgm_ctx* p) {
    M mp;
    base(p, mp);
    for (int g = 0; g < 3; ++g)
      if (dgm_ctx* k = p->kids[g]) {
        mp.g[g].Uin = S(k->U);
        mp.g[g].blocks = (int)((k->ne + 255) / 256);
      }
    dgm::k_step_head_mixed<T, MASK, St><<<blocks_total(mp), 256, 0, p->stream>>>(mp);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int edge_flux(dgm_ctx* p, int which) {
    M mp;
    base(p, mp);
    for (int g = 0; g < 3; ++g)
      if (dgm_ctx* k = p->kids[g]) {
        mp.g[g].Uin = arr(k, which);
        mp.g[g].blocks = (int)(((k->n_int + k->n_bnd) * k->ng + kMixedEdgeThreads - 1) / kMixedEdgeThreads);
      }
    dgm::k_edge_flux_mixed<T, MASK, St><<<blocks_total(mp), kMixedEdgeThreads, 0, p->stream>>>(mp);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  template <int MODE>
  static int element(dgm_ctx* p, bool with_residual) {
    M mp;
    base(p, mp);
    for (int g = 0; g < 3; ++g)
      if (dgm_ctx* k = p->kids[g]) {
        auto& a = mp.g[g];
        a.Uin = arr(k, MODE == 1 ? 0 : MODE == 2 ? 1 : 2);
        a.Ubase = MODE == 1 ? nullptr : S(k->U);
        a.Uout = arr(k, MODE == 1 ? 1 : MODE == 2 ? 2 : 0);
        a.Rout = (MODE == 3 && with_residual) ? S(k->R) : nullptr;
        a.blocks = (int)((k->ne + kMixedElemThreads / 4 - 1) / (kMixedElemThreads / 4));
      }
    dgm::k_element_mixed<T, MASK, MODE, St><<<blocks_total(mp), kMixedElemThreads, 0, p->stream>>>(mp);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int limiter(dgm_ctx* p, int which) {
    if (!p->limiter) return DGM_OK;
    M mp;
    base(p, mp);
    for (int g = 0; g < 3; ++g)
      if (dgm_ctx* k = p->kids[g]) {
        mp.g[g].Uin = arr(k, which);
        mp.g[g].Uout = arr(k, which);
        mp.g[g].blocks = (int)((k->ld / 32 + dgm::kDetectWarps - 1) / dgm::kDetectWarps);
      }
    dgm::k_lim_detect_mixed<T, MASK, false, St><<<blocks_total(mp), dgm::kDetectThreads, 0, p->stream>>>(mp);
    CK(cudaGetLastError());
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p->mixed_blocks);
    cfg.blockDim = dim3(dgm::kLimiterWarps * 32);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = p->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, dgm::k_limiter_mixed<T, MASK, St>, mp, p->mwork));
    return DGM_OK;
  }

  static int step_end(dgm_ctx* p) {
    M mp;
    base(p, mp);
    const int n = mp.g[0].n_inst + mp.g[1].n_inst + mp.g[2].n_inst;
    dgm::k_step_end_mixed<T, MASK, St><<<(n + 127) / 128, 128, 0, p->stream>>>(mp);
    CK(cudaGetLastError());
    return DGM_OK;
  }

  static int step(dgm_ctx* p, bool with_residual) {
    int st;
    if ((st = step_head(p))) return st;
    if ((st = edge_flux(p, 0)) || (st = element<1>(p, false)) || (st = limiter(p, 1))) return st;
    if ((st = edge_flux(p, 1)) || (st = element<2>(p, false)) || (st = limiter(p, 2))) return st;
    if ((st = edge_flux(p, 2)) || (st = element<3>(p, with_residual)) || (st = limiter(p, 0))) return st;
    return step_end(p);
  }

  static int occupancy(dgm_ctx* p) {
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dgm::k_limiter_mixed<T, MASK, St>, dgm::kLimiterWarps * 32,
                                                     0));
    int64_t ne = 0;
    for (dgm_ctx* k : p->kids)
      if (k) ne += k->ne;
    const int64_t want = std::max<int64_t>(1, (ne + 32 * dgm::kLimiterWarps - 1) / (32 * dgm::kLimiterWarps));
    p->mixed_blocks = (int)std::min<int64_t>((int64_t)std::max(1, per_sm) * p->num_sms, want);
    return DGM_OK;
  }
};

// Sets of orders compiled for mixed launches: {1, 2} and {1, 2, 3} (any other set runs as the
// latter with empty groups).
template <class F>
int mixed_dispatch(dgm_ctx* p, F&& f) {
  const bool three = p->kids[2] != nullptr;
  if (p->prec_mode == 4) return three ? f(MixOps<float, 7, double>{}) : f(MixOps<float, 3, double>{});
  if (p->prec == 0) return three ? f(MixOps<double, 7>{}) : f(MixOps<double, 3>{});
  return three ? f(MixOps<float, 7>{}) : f(MixOps<float, 3>{});
}

int mixed_step(dgm_ctx* c, int with_residual) {
  return mixed_dispatch(c, [&](auto ops) { return decltype(ops)::step(c, with_residual != 0); });
}

dgm_ctx* create_mixed(int n, const dgm_mesh_desc* meshes, const int32_t* orders, const dgm_tables_desc* tables,
                      const dgm_params* params, const dgm_slot_capacity* caps, int32_t* status) {
  int32_t dummy;
  if (!status) status = &dummy;
  if (n < 1 || !meshes || !orders || !tables || !params) {
    *status = DGM_BAD_ARG;
    return nullptr;
  }
  for (int i = 0; i < n; ++i)
    if (orders[i] < 1 || orders[i] > 3 || params[i].hcr != params[0].hcr || params[i].precision != params[0].precision ||
        params[i].limiter != params[0].limiter || params[i].device != params[0].device) {
      *status = DGM_BAD_ARG;
      return nullptr;
    }
  if (params[0].precision != 0 && params[0].precision != 1 && params[0].precision != 4) {  // no tensor-core modes
    *status = DGM_BAD_ARG;
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || params->device < 0 || params->device >= ndev) {
    cudaGetLastError();
    *status = DGM_NO_DEVICE;
    return nullptr;
  }
  auto* p = new dgm_ctx();
  p->mixed = true;
  p->device = params->device;
  p->prec_mode = params->precision;
  p->prec = params->precision == 0 ? 0 : 1;
  p->hcr = params->hcr;
  p->limiter = params->limiter ? 1 : 0;
  auto fail = [&](int st) {
    *status = st;
    dgm_destroy(p);
    return (dgm_ctx*)nullptr;
  };
  if (cudaSetDevice(p->device) != cudaSuccess) return fail(DGM_NO_DEVICE);
  if (cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess)
    return fail(DGM_NO_DEVICE);
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  p->pool = pool_acquire(p->device);
  if (!p->pool) return fail(DGM_CUDA_ERROR);
  p->imap.resize(n);
  int64_t ne_all = 0;
  for (int g = 0; g < 3; ++g) {
    std::vector<dgm_mesh_desc> ms;
    std::vector<dgm_params> ps;
    std::vector<dgm_slot_capacity> cs;
    for (int i = 0; i < n; ++i)
      if (orders[i] == g + 1) {
        p->imap[i] = {g, (int)ms.size()};
        ms.push_back(meshes[i]);
        ps.push_back(params[i]);
        if (caps) cs.push_back(caps[i]);
      }
    if (ms.empty()) continue;
    if (tables[g].order != g + 1) return fail(DGM_BAD_ARG);
    int32_t st = DGM_OK;
    p->kids[g] = create((int)ms.size(), ms.data(), caps ? cs.data() : nullptr, &tables[g], ps.data(), &st, p->stream);
    if (!p->kids[g]) return fail(st ? st : DGM_CUDA_ERROR);
    ne_all += p->kids[g]->ne;
  }
  int st;
  if ((st = dev_alloc(p, &p->mwork, (size_t)ne_all))) return fail(st);
  if ((st = mixed_dispatch(p, [&](auto ops) { return decltype(ops)::occupancy(p); }))) return fail(st);
  if (cudaStreamSynchronize(p->stream) != cudaSuccess) return fail(DGM_CUDA_ERROR);
  p->graph_steps = (int)kGraphSteps;
  *status = DGM_OK;
  return p;
}

// The child context and its instance index of a mixed batch's instance i (the context itself and i
// for other contexts); false if i is out of range.
bool resolve(dgm_ctx*& c, int32_t& i) {
  if (!c) return false;
  if (!c->mixed) return i >= 0 && i < (int32_t)c->inst.size();
  if (i < 0 || i >= (int32_t)c->imap.size()) return false;
  const auto& m = c->imap[i];
  c = c->kids[m.first];
  i = m.second;
  return c != nullptr;
}

// Writes the clocks of children whose host mirrors changed (dgm_instance_set / replace).
int mixed_sync_clocks(dgm_ctx* p) {
  for (dgm_ctx* k : p->kids)
    if (k && (k->limits_dirty || k->dt_dirty)) {
      int st = write_clock(k);
      if (st) return st;
    }
  return DGM_OK;
}

int mixed_collect(dgm_ctx* p) {
  int first = DGM_OK;
  for (dgm_ctx* k : p->kids)
    if (k) {
      const int st = collect_status(k);
      if (st && !first) first = st;
    }
  return first;
}

}  // namespace

extern "C" {

const char* dgm_version(void) { return "dgm_b200 0.2 (sm_100a; FP64 and FP32 DG residual + SSP-RK3, batched)"; }

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
    case DGM_NOT_READY: return "Work still in flight";
    case DGM_LIST_OVERFLOW: return "Limiter worklist overflow";
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
  for (dgm_ctx* k : c->kids) dgm_destroy(k);
  if (c->h_diag) cudaFreeHost(c->h_diag);
  if (c->diag_ready) cudaEventDestroy(c->diag_ready);
  if (c->stream) {
    for (void* p : c->allocs) cudaFreeAsync(p, c->stream);  // back to the pool, in stream order
    cudaStreamSynchronize(c->stream);
    if (c->owns_stream) cudaStreamDestroy(c->stream);
  }
  if (c->pool) pool_release(c->device);
  delete c;
}

dgm_ctx* dgm_create(const dgm_mesh_desc* mesh, const dgm_tables_desc* tables, const dgm_params* params,
                    int32_t* status) {
  return create(1, mesh, nullptr, tables, params, status);
}

dgm_ctx* dgm_create_batch(int32_t n_instances, const dgm_mesh_desc* meshes, const dgm_tables_desc* tables,
                          const dgm_params* params, int32_t* status) {
  return create(n_instances, meshes, nullptr, tables, params, status);
}

dgm_ctx* dgm_create_batch_slots(int32_t n_instances, const dgm_mesh_desc* meshes, const dgm_slot_capacity* capacity,
                                const dgm_tables_desc* tables, const dgm_params* params, int32_t* status) {
  if (!capacity) {
    if (status) *status = DGM_BAD_ARG;
    return nullptr;
  }
  return create(n_instances, meshes, capacity, tables, params, status);
}

dgm_ctx* dgm_create_mixed(int32_t n_instances, const dgm_mesh_desc* meshes, const int32_t* orders,
                          const dgm_tables_desc* tables, const dgm_params* params, const dgm_slot_capacity* capacity,
                          int32_t* status) {
  return create_mixed(n_instances, meshes, orders, tables, params, capacity, status);
}

int32_t dgm_instance_capacity(dgm_ctx* c, int32_t i, dgm_slot_capacity* out) {
  if (!resolve(c, i) || !out) return DGM_BAD_ARG;
  const HostInst& h = c->inst[i];
  out->elements = h.elem_cap;
  out->internal_edges = h.int_cap;
  out->boundary_edges = h.bnd_cap;
  out->patches = h.patch_cap;
  return DGM_OK;
}

// Takes a new mesh into instance i's capacity ranges: rebuilds the instance's geometry,
// connectivity, edge slots, patches and limiter visiting order on the host, copies them into its
// ranges of the device arrays, recomputes its WENO Gram matrices, zeroes its state and resets its
// clock, loop bounds and status.  The other instances are untouched; the step graphs stay valid
// (they hold array addresses and sizes, which do not change).
int32_t dgm_instance_replace(dgm_ctx* c, int32_t i, const dgm_mesh_desc* mesh, const dgm_params* params) {
  if (!resolve(c, i) || !mesh || !params || params->hcr != c->hcr) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));  // nothing of this context may still read the old mesh
  InstArrays a;
  int st = fill_instance(c, i, mesh, a);
  if (st) return st;
  HostInst& h = c->inst[i];
  const int64_t eo = h.elem_off, cap = h.elem_cap, ld = c->ld;
  MeshDev* mdp = nullptr;
  dispatch(c, [&](auto ops) {
    mdp = &decltype(ops)::mesh(c);
    return DGM_OK;
  });
  if (!mdp) return DGM_BAD_ARG;
  const MeshDev& md = *mdp;
  auto put = [&](const void* dst, const void* src, size_t bytes) -> int {
    if (bytes) CK(cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, c->stream));
    return DGM_OK;
  };
  if ((st = put(md.jac + eo, a.jac.data(), cap * sizeof(double))) || (st = put(md.hmin + eo, a.hmin.data(), cap * sizeof(double))) ||
      (st = put(md.h15 + eo, a.h15.data(), cap * sizeof(double))) || (st = put(md.inst + eo, a.inst.data(), cap * sizeof(int))))
    return st;
  for (int k = 0; k < 4; ++k)
    if ((st = put(md.dinv + k * ld + eo, a.dinv.data() + k * cap, cap * sizeof(double)))) return st;
  for (int k = 0; k < 3; ++k)
    if ((st = put(md.face + k * ld + eo, a.face.data() + k * cap, cap * sizeof(int))) ||
        (st = put(md.nbr + k * ld + eo, a.nbr.data() + k * cap, cap * sizeof(int))))
      return st;
  if ((st = put(md.ie_lr + h.int_off, a.ie_lr.data(), h.int_cap * sizeof(int2))) ||
      (st = put(md.ie_ic + h.int_off, a.ie_ic.data(), h.int_cap * sizeof(int))) ||
      (st = put(md.ie_geo + h.int_off, a.ie_geo.data(), h.int_cap * sizeof(double4))) ||
      (st = put(md.slot_ref + h.int_off, a.int_ref.data(), h.int_cap * sizeof(int64_t))) ||
      (st = put(md.be_elem + h.bnd_off, a.be_elem.data(), h.bnd_cap * sizeof(int))) ||
      (st = put(md.be_info + h.bnd_off, a.be_info.data(), h.bnd_cap * sizeof(int))) ||
      (st = put(md.be_geo + h.bnd_off, a.be_geo.data(), h.bnd_cap * sizeof(double4))) ||
      (st = put(md.slot_ref + c->n_int + h.bnd_off, a.bnd_ref.data(), h.bnd_cap * sizeof(int64_t))) ||
      (st = put(md.patch_q + h.patch_off, a.patch_q.data(), h.patch_cap * sizeof(double4))))
    return st;
  const size_t rec = (size_t)NEQ * c->nb * elem_bytes(c);
  for (void* p : {c->U, c->U1, c->U2, c->R})
    CK(cudaMemsetAsync(static_cast<char*>(p) + (size_t)eo * rec, 0, (size_t)cap * rec, c->stream));
  if (c->limiter && (st = dispatch(c, [&](auto ops) { return decltype(ops)::weno_gram(c, eo, cap); }))) return st;
  h.ne = mesh->n_elements;
  h.nb_slots = boundary_edge_count(mesh);
  h.cfl = params->cfl;
  h.final_time = params->final_time;
  h.final_step = params->final_step;
  h.t = 0.0;
  h.step = 0;
  h.status = 0;
  h.err_where = -1;
  c->limits_dirty = true;
  if ((st = upload_ranges(c))) return st;  // synchronizes: the host arrays may go
  return DGM_OK;
}

int32_t dgm_instance_upload(dgm_ctx* c, int32_t i, const double* solutions) {
  if (!resolve(c, i) || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = upload_state(c, i, solutions, c->U);
  if (st) return st;
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

int32_t dgm_instance_download(dgm_ctx* c, int32_t i, double* solutions) {
  if (!resolve(c, i) || !solutions) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  return download_state(c, i, c->U, solutions);
}

int32_t dgm_instance_download_residual(dgm_ctx* c, int32_t i, double* residuals) {
  if (!resolve(c, i) || !residuals) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  return download_state(c, i, c->R, residuals);
}

int32_t dgm_instance_state(dgm_ctx* c, int32_t i, double* t, int64_t* step, int32_t* status, int64_t* where) {
  if (!resolve(c, i)) return DGM_BAD_ARG;
  const HostInst& h = c->inst[i];
  if (t) *t = h.t;
  if (step) *step = h.step;
  if (status) *status = h.status;
  if (where) *where = h.err_where;
  return DGM_OK;
}

int32_t dgm_instance_set(dgm_ctx* c, int32_t i, double t, int64_t step, double final_time, int64_t final_step) {
  if (!resolve(c, i)) return DGM_BAD_ARG;
  HostInst& h = c->inst[i];
  h.t = t;
  h.step = step;
  h.final_time = final_time;
  h.final_step = final_step;
  h.status = 0;
  h.err_where = -1;
  c->limits_dirty = true;
  return DGM_OK;
}

// Solver::set_initial_solution (solver.rs:45-79) on the device: the free-stream state of
// InitialSolution, with the reference's expressions, projected onto the basis of every element
// of instance i (all instances for dgm_set_initial_solution) in the resident state.
static int set_initial(dgm_ctx* c, int64_t i, double density, double angle_of_attack, double mach_number,
                       double pressure) {
  if (!(density > 0.0) || !(pressure > 0.0) || !std::isfinite(angle_of_attack) || !std::isfinite(mach_number))
    return DGM_BAD_ARG;
  const double sound_speed = std::sqrt(c->hcr * pressure / density);
  const double pi = 3.14159265358979323846;           // f64::consts::PI
  const double a = angle_of_attack * (pi / 180.0);   // f64::to_radians
  const double x_velocity = mach_number * std::cos(a) * sound_speed;
  const double y_velocity = mach_number * std::sin(a) * sound_speed;
  const double total_energy =
      pressure / (c->hcr - 1.0) + 0.5 * density * (x_velocity * x_velocity + y_velocity * y_velocity);
  const double q[NEQ] = {density, density * x_velocity, density * y_velocity, total_energy};
  return dispatch(c, [&](auto ops) { return decltype(ops)::project(c, i, q); });
}

int32_t dgm_instance_set_initial(dgm_ctx* c, int32_t i, double density, double angle_of_attack,
                                 double mach_number, double pressure) {
  if (!resolve(c, i)) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = set_initial(c, i, density, angle_of_attack, mach_number, pressure);
  if (st) return st;
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

int32_t dgm_set_initial_solution(dgm_ctx* c, double density, double angle_of_attack, double mach_number,
                                 double pressure) {
  if (!c) return DGM_BAD_ARG;
  if (c->mixed) {
    for (dgm_ctx* k : c->kids)
      if (k) {
        const int st = dgm_set_initial_solution(k, density, angle_of_attack, mach_number, pressure);
        if (st) return st;
      }
    return DGM_OK;
  }
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  for (size_t i = 0; i < c->inst.size(); ++i) {
    int st = set_initial(c, (int64_t)i, density, angle_of_attack, mach_number, pressure);
    if (st) return st;
  }
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

int32_t dgm_instance_count(dgm_ctx* c) { return c ? (int32_t)(c->mixed ? c->imap.size() : c->inst.size()) : 0; }

int32_t dgm_compute_residuals(dgm_ctx* c, double* residuals, const double* solutions) {
  if (!c || !residuals || !solutions || c->inst.size() != 1) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, 0, solutions, c->U1))) return st;
  if ((st = upload_state(c, 0, residuals, c->U2))) return st;
  if ((st = set_active(c, 0.0, false))) return st;
  st = dispatch(c, [&](auto ops) {
    using O = decltype(ops);
    int s2 = O::edge_flux(c, O::S(c->U1));
    if (s2) return s2;
    return O::template element<0>(c, O::S(c->U1), nullptr, nullptr, O::S(c->U2), O::S(c->R));
  });
  if (st) return st;
  if ((st = download_state(c, 0, c->R, residuals))) return st;
  return collect_status(c);
}

int32_t dgm_apply_limiter(dgm_ctx* c, double* solutions, int64_t* troubled) {
  if (!c || !solutions || c->inst.size() != 1) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, 0, solutions, c->U1))) return st;
  if ((st = set_active(c, 0.0, false))) return st;
  if ((st = dispatch(c, [&](auto ops) {
         using O = decltype(ops);
         return O::limiter(c, O::S(c->U1));
       })))
    return st;
  if ((st = download_state(c, 0, c->U1, solutions))) return st;
  st = collect_status(c);
  if (troubled) *troubled = c->last_troubled;
  return st;
}

int32_t dgm_compute_time_step(dgm_ctx* c, const double* solutions, double* time_step) {
  if (!c || !solutions || !time_step || c->inst.size() != 1) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, 0, solutions, c->U1))) return st;
  if ((st = set_active(c, 0.0, false))) return st;
  if ((st = dispatch(c, [&](auto ops) {
         using O = decltype(ops);
         return O::time_step(c, O::S(c->U1));
       })))
    return st;
  Control h;
  std::vector<InstCtl> hi;
  if ((st = read_control(c, &h, &hi))) return st;
  unsigned long long bits = hi[0].dt_bits;
  std::memcpy(time_step, &bits, sizeof(double));
  c->dt_dirty = true;
  return collect_status(c);
}

int32_t dgm_rk3(dgm_ctx* c, double* residuals, double* solutions, double time_step) {
  if (!c || !residuals || !solutions || c->inst.size() != 1) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = upload_state(c, 0, solutions, c->U))) return st;
  if ((st = set_active(c, time_step, true))) return st;
  if ((st = dispatch(c, [&](auto ops) {
         using O = decltype(ops);
         return O::rk3(c, O::S(c->R));
       })))
    return st;
  if ((st = download_state(c, 0, c->U, solutions))) return st;
  if ((st = download_state(c, 0, c->R, residuals))) return st;
  return collect_status(c);
}

int32_t dgm_time_march(dgm_ctx* c, double* residuals, double* solutions) {
  if (!c || !residuals || !solutions || c->inst.size() != 1) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st;
  if ((st = write_clock(c))) return st;
  if ((st = upload_state(c, 0, solutions, c->U))) return st;
  const int64_t remaining = std::max<int64_t>(0, c->inst[0].final_step - c->inst[0].step);
  if ((st = enqueue_steps(c, remaining, 1))) return st;
  if ((st = download_state(c, 0, c->U, solutions))) return st;
  if (remaining > 0)
    if ((st = download_state(c, 0, c->R, residuals))) return st;
  return collect_status(c);
}

int32_t dgm_get_clock(dgm_ctx* c, double* t, int64_t* step) {
  if (!c || c->inst.empty()) return DGM_BAD_ARG;
  if (t) *t = c->inst[0].t;
  if (step) *step = c->inst[0].step;
  return DGM_OK;
}

int32_t dgm_set_clock(dgm_ctx* c, double t, int64_t step) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  for (auto& h : c->inst) {
    h.t = t;
    h.step = step;
  }
  return write_clock(c);
}

int32_t dgm_set_limits(dgm_ctx* c, double final_time, int64_t final_step) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c) return DGM_BAD_ARG;
  for (auto& h : c->inst) {
    h.final_time = final_time;
    h.final_step = final_step;
  }
  c->limits_dirty = true;
  return DGM_OK;
}

int32_t dgm_upload_solutions(dgm_ctx* c, const double* solutions) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || !solutions || c->inst.size() != 1) return DGM_BAD_ARG;
  return dgm_instance_upload(c, 0, solutions);
}

int32_t dgm_download_solutions(dgm_ctx* c, double* solutions) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || !solutions || c->inst.size() != 1) return DGM_BAD_ARG;
  return dgm_instance_download(c, 0, solutions);
}

int32_t dgm_advance(dgm_ctx* c, int64_t n_steps) {
  if (!c || n_steps < 0) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  if (c->mixed) {
    const int st = mixed_sync_clocks(c);
    return st ? st : enqueue_steps(c, n_steps, 0);
  }
  if (c->limits_dirty || c->dt_dirty) {
    int st = write_clock(c);
    if (st) return st;
  }
  return enqueue_steps(c, n_steps, 0);
}

int32_t dgm_advance_with_residual(dgm_ctx* c, int64_t n_steps) {
  if (!c || n_steps < 0) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  if (c->mixed) {
    const int st = mixed_sync_clocks(c);
    return st ? st : enqueue_steps(c, n_steps, 1);
  }
  if (c->limits_dirty || c->dt_dirty) {
    int st = write_clock(c);
    if (st) return st;
  }
  return enqueue_steps(c, n_steps, 1);
}

int32_t dgm_synchronize(dgm_ctx* c) {
  if (!c) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  return c->mixed ? mixed_collect(c) : collect_status(c);
}

int32_t dgm_query(dgm_ctx* c) {
  if (!c) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  const cudaError_t e = cudaStreamQuery(c->stream);
  if (e == cudaErrorNotReady) return DGM_NOT_READY;
  CK(e);
  return c->mixed ? mixed_collect(c) : collect_status(c);
}

void* dgm_stream(dgm_ctx* c) { return c ? (void*)c->stream : nullptr; }

int32_t dgm_launch_phase(dgm_ctx* c, int32_t phase) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || phase < 0 || phase > 3) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = set_active(c, 0.0, false);
  if (st) return st;
  return dispatch(c, [&](auto ops) {
    using O = decltype(ops);
    switch (phase) {
      case 0: c->dt_dirty = true; return O::time_step(c, O::S(c->U));
      case 1: return O::edge_flux(c, O::S(c->U));
      case 2: return O::template element<2>(c, O::S(c->U), O::S(c->U), O::S(c->U2), nullptr, nullptr);
      default: return O::limiter(c, O::S(c->U2));
    }
  });
}

int32_t dgm_set_launch_config(dgm_ctx* c, int32_t edge_threads, int32_t edge_blocks, int32_t element_threads) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c) return DGM_BAD_ARG;
  auto threads_ok = [](int32_t t) { return t >= 32 && t <= 256 && t % 32 == 0; };
  if (!threads_ok(edge_threads) || !threads_ok(element_threads) || edge_blocks < 0 || edge_blocks > (1 << 24))
    return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  c->edge_threads = edge_threads;
  c->edge_blocks = edge_blocks;
  c->elem_threads = element_threads;
  reset_graphs(c);
  return DGM_OK;
}

int32_t dgm_set_limiter_variant(dgm_ctx* c, int32_t staged) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || (staged != 0 && staged != 1)) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  c->lim_staged = staged;
  reset_graphs(c);
  return DGM_OK;
}

// The queue schedule needs the worklist all zero when a pass starts (its consumers clear what
// they take); the barrier schedule leaves its entries behind, so a switch to the queue clears it.
static int set_schedule(dgm_ctx* c, int queue) {
  if (queue && !c->lim_queue)
    CK(cudaMemsetAsync(c->work, 0, sizeof(int) * std::max<int64_t>(c->ne, 1), c->stream));
  c->lim_queue = queue;
  return DGM_OK;
}

int32_t dgm_set_limiter_grid(dgm_ctx* c, int32_t one_per_sm) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || (one_per_sm != 0 && one_per_sm != 1)) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  c->lim_one_per_sm = one_per_sm;
  reset_graphs(c);
  return DGM_OK;
}

int32_t dgm_get_limiter_grid(dgm_ctx* c) { return c ? c->lim_one_per_sm : -1; }

int32_t dgm_set_limiter_schedule(dgm_ctx* c, int32_t queue) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || (queue != 0 && queue != 1)) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  int st = set_schedule(c, queue);
  if (st) return st;
  reset_graphs(c);
  return DGM_OK;
}

int32_t dgm_get_limiter_schedule(dgm_ctx* c, int32_t* queue, double* tuned_us) {
  if (!c) return DGM_BAD_ARG;
  if (queue) *queue = c->lim_queue;
  if (tuned_us)
    for (int q = 0; q < 2; ++q) tuned_us[q] = std::min(c->lim_us[0][q], c->lim_us[1][q]);
  return DGM_OK;
}

int32_t dgm_set_edge_variant(dgm_ctx* c, int32_t pair) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || pair < 0 || pair > 3) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  c->edge_pair = pair;
  reset_graphs(c);
  return DGM_OK;
}

int32_t dgm_get_edge_variant(dgm_ctx* c) { return c ? c->edge_pair : -1; }

int32_t dgm_set_viscous(dgm_ctx* c, int32_t enable, double prandtl_number, double gas_constant,
                        const double* dphi_edge_ref) {
  if (!c || c->mixed || (enable != 0 && enable != 1)) return DGM_BAD_ARG;
  if (enable && (c->prec_mode != 0 || !dphi_edge_ref || !(prandtl_number > 0.0) || !(gas_constant > 0.0) ||
                 !std::isfinite(prandtl_number) || !std::isfinite(gas_constant)))
    return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaStreamSynchronize(c->stream));
  if (enable) {
    const int st = dispatch(c, [&](auto ops) {
      return decltype(ops)::set_viscous(c, prandtl_number, gas_constant, dphi_edge_ref);
    });
    if (st) return st;
  }
  c->viscous = enable;
  reset_graphs(c);
  return DGM_OK;
}

int32_t dgm_get_viscous(dgm_ctx* c) { return c ? c->viscous : -1; }

int32_t dgm_get_limiter_variant(dgm_ctx* c, int32_t* staged, double* tuned_us) {
  if (!c) return DGM_BAD_ARG;
  if (staged) *staged = c->lim_staged;
  if (tuned_us)
    for (int v = 0; v < 2; ++v) tuned_us[v] = std::min(c->lim_us[v][0], c->lim_us[v][1]);
  return DGM_OK;
}

int32_t dgm_get_launch_config(dgm_ctx* c, int32_t* config) {
  if (!c || !config) return DGM_BAD_ARG;
  config[0] = c->edge_threads;
  config[1] = c->edge_blocks;
  config[2] = c->elem_threads;
  return DGM_OK;
}

// Times every candidate configuration of the edge and element passes on the resident state
// (CUDA events on the context's stream, after warm-up launches) and keeps the fastest.  The
// candidates only regroup independent per-slot / per-element work, so results are unchanged.
int32_t dgm_autotune(dgm_ctx* c, int32_t repeats, double* best_us) {
  if (c && c->mixed) return DGM_BAD_ARG;  // per-order settings and single-mesh calls
  if (!c || repeats < 1 || repeats > 1000) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = set_active(c, 0.0, false);
  if (st) return st;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return DGM_CUDA_ERROR;
  }
  const int sms = c->num_sms;
  // (form, threads, blocks): per-point (at two register budgets), lane-pair and staged edge
  // passes, one work item per thread or a grid-stride grid of 4-16 blocks per SM (the staged form
  // always runs 128-thread blocks)
  const int edge_cand[][3] = {{0, 256, 0},        {0, 128, 0},        {0, 64, 0},         {0, 256, 4 * sms},
                              {0, 256, 8 * sms},  {0, 128, 8 * sms},  {0, 128, 16 * sms}, {1, 256, 0},
                              {1, 128, 0},        {1, 64, 0},         {1, 128, 8 * sms},  {1, 128, 16 * sms},
                              {2, 128, 0},        {2, 128, 8 * sms},  {2, 128, 16 * sms}, {3, 256, 0},
                              {3, 128, 0},        {3, 256, 8 * sms},  {3, 128, 16 * sms}};
  const int elem_cand[] = {256, 128, 64};
  auto time_phase = [&](int phase, float* us) -> int {
    for (int w = 0; w < 2; ++w) {
      int s2 = dispatch(c, [&](auto ops) {
        using O = decltype(ops);
        return phase == 1 ? O::edge_flux(c, O::S(c->U))
                          : O::template element<2>(c, O::S(c->U), O::S(c->U), O::S(c->U2), nullptr, nullptr);
      });
      if (s2) return s2;
    }
    CK(cudaEventRecord(e0, c->stream));
    for (int r = 0; r < repeats; ++r) {
      int s2 = dispatch(c, [&](auto ops) {
        using O = decltype(ops);
        return phase == 1 ? O::edge_flux(c, O::S(c->U))
                          : O::template element<2>(c, O::S(c->U), O::S(c->U), O::S(c->U2), nullptr, nullptr);
      });
      if (s2) return s2;
    }
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *us = 1000.f * ms / repeats;
    return DGM_OK;
  };
  float best_edge = 1e30f, best_elem = 1e30f;
  int be_t = c->edge_threads, be_b = c->edge_blocks, bl_t = c->elem_threads, be_f = c->edge_pair;
  // limiter detector variant: each timed launch limits the same stage buffer, rebuilt by an edge
  // and an element pass before it (only the limiter sits between the events)
  auto time_limiter = [&](float* us) -> int {
    float tot = 0.f;
    for (int r = 0; r < repeats + 2; ++r) {
      int s2 = dispatch(c, [&](auto ops) {
        using O = decltype(ops);
        int s3 = O::edge_flux(c, O::S(c->U));
        if (!s3) s3 = O::template element<2>(c, O::S(c->U), O::S(c->U), O::S(c->U2), nullptr, nullptr);
        if (!s3) CK(cudaEventRecord(e0, c->stream));
        if (!s3) s3 = O::limiter(c, O::S(c->U2));
        if (!s3) CK(cudaEventRecord(e1, c->stream));
        return s3;
      });
      if (s2) return s2;
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (r >= 2) tot += ms;
    }
    *us = 1000.f * tot / repeats;
    return DGM_OK;
  };
  if (c->limiter) {
    // detector form x schedule x wave-kernel grid (all co-resident blocks, or one per SM)
    int bv = 0, bq = 0, bg = 0;
    float best = 1e30f;
    for (int v = 0; v < 2 && !st; ++v)
      for (int q = 0; q < 2 && !st; ++q) {
        c->lim_us[v][q] = 1e30f;
        for (int gsz = 0; gsz < 2 && !st; ++gsz) {
          c->lim_staged = v;
          c->lim_one_per_sm = gsz;
          st = set_schedule(c, q);
          float us = 0.f;
          if (!st) st = time_limiter(&us);
          if (!st && us < c->lim_us[v][q]) c->lim_us[v][q] = us;
          if (!st && us < best) best = us, bv = v, bq = q, bg = gsz;
        }
      }
    c->lim_staged = bv;
    c->lim_one_per_sm = bg;
    if (!st) st = set_schedule(c, bq);
  }
  for (auto& cand : edge_cand) {
    c->edge_pair = cand[0];
    c->edge_threads = cand[1];
    c->edge_blocks = cand[2];
    float us;
    if ((st = time_phase(1, &us))) break;
    if (us < best_edge) best_edge = us, be_f = cand[0], be_t = cand[1], be_b = cand[2];
  }
  for (int t : elem_cand) {
    if (st) break;
    c->elem_threads = t;
    float us;
    if ((st = time_phase(2, &us))) break;
    if (us < best_elem) best_elem = us, bl_t = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->edge_pair = be_f;
  c->edge_threads = be_t;
  c->edge_blocks = be_b;
  c->elem_threads = bl_t;
  reset_graphs(c);
  if (best_us) {
    best_us[0] = best_edge;
    best_us[1] = best_elem;
  }
  const int device_status = collect_status(c);
  return st ? st : device_status;
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
  return 1 /* step head: loop condition + time step */ + 1 /* step end */ +
         3 * (2 + (c->viscous ? 1 /* global lifts */ : 0) + (c->limiter ? 2 /* detection, waves */ : 0));
}

int64_t dgm_error_location(dgm_ctx* c) {
  if (!c) return -1;
  if (c->mixed)
    for (dgm_ctx* k : c->kids)
      if (k && k->err_where >= 0) return k->err_where;
  return c->err_where;
}

int32_t dgm_limiter_stats(dgm_ctx* c, int64_t* troubled, int32_t* waves) {
  if (!c) return DGM_BAD_ARG;
  if (c->mixed) {
    int64_t t = 0;
    int w = 0;
    for (dgm_ctx* k : c->kids)
      if (k) {
        t += k->last_troubled;
        w = std::max(w, k->last_waves);
      }
    if (troubled) *troubled = t;
    if (waves) *waves = w;
    return DGM_OK;
  }
  if (troubled) *troubled = c->last_troubled;
  if (waves) *waves = c->last_waves;
  return DGM_OK;
}

int64_t dgm_device_bytes(dgm_ctx* c) {
  if (!c) return 0;
  int64_t b = c->bytes;
  for (dgm_ctx* k : c->kids)
    if (k) b += k->bytes;
  return b;
}

int32_t dgm_diagnostics(dgm_ctx* c, int32_t use_residual, double* out) {
  if (!c || !out) return DGM_BAD_ARG;
  if (c->mixed) {  // each order's instances, scattered into the batch's instance order
    std::vector<double> part;
    for (int g = 0; g < 3; ++g) {
      dgm_ctx* k = c->kids[g];
      if (!k) continue;
      part.assign(8 * k->inst.size(), 0.0);
      const int st = dgm_diagnostics(k, use_residual, part.data());
      if (st) return st;
      for (size_t i = 0; i < c->imap.size(); ++i)
        if (c->imap[i].first == g) std::memcpy(out + 8 * i, part.data() + 8 * c->imap[i].second, 8 * sizeof(double));
    }
    return DGM_OK;
  }
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  int st = dispatch(c, [&](auto ops) {
    using O = decltype(ops);
    return O::diagnostics(c, use_residual ? O::S(c->R) : nullptr);
  });
  if (st) return st;
  CK(cudaMemcpyAsync(out, c->d_diag, sizeof(double) * 8 * c->inst.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

int32_t dgm_enqueue_diagnostics(dgm_ctx* c, int32_t use_residual) {
  if (!c || c->mixed) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  const size_t bytes = sizeof(double) * 8 * c->inst.size();
  if (!c->h_diag) {
    CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_diag), bytes));
    CK(cudaEventCreateWithFlags(&c->diag_ready, cudaEventDisableTiming));
  }
  int st = dispatch(c, [&](auto ops) {
    using O = decltype(ops);
    return O::diagnostics(c, use_residual ? O::S(c->R) : nullptr);
  });
  if (st) return st;
  CK(cudaMemcpyAsync(c->h_diag, c->d_diag, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(c->diag_ready, c->stream));
  return DGM_OK;
}

int32_t dgm_collected_diagnostics(dgm_ctx* c, double* out) {
  if (!c || !out || c->mixed || !c->h_diag) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  CK(cudaEventSynchronize(c->diag_ready));
  std::memcpy(out, c->h_diag, sizeof(double) * 8 * c->inst.size());
  return DGM_OK;
}

int32_t dgm_precision(dgm_ctx* c) { return c ? c->prec_mode : -1; }

int32_t dgm_cell_fields(dgm_ctx* c, int32_t i, double* fields) {
  if (!resolve(c, i) || !fields) return DGM_BAD_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return DGM_CUDA_ERROR;
  // the FP64 staging buffer holds a whole instance's state (ne x 4 x NB >= ne x 4 doubles)
  int st = dispatch(c, [&](auto ops) { return decltype(ops)::cell_fields(c, i, c->stage); });
  if (st) return st;
  CK(cudaMemcpyAsync(fields, c->stage, sizeof(double) * 4 * (size_t)c->inst[i].ne, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DGM_OK;
}

}  // extern "C"
