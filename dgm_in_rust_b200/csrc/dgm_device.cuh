// dgm_device.cuh -- device code of the B200 DG residual + SSP-RK3 path.
//
// One context holds one or more independent mesh instances as a single disconnected union
// mesh (element, edge and patch indices offset per instance), so every launch covers all
// instances; each instance has its own time-march control (time, dt, step, loop bounds, status).
//
// Data layout in HBM:
//   state      U[e][v][b]             element-major in the storage type T (double or float), the
//                                      reference's own [element][variable][basis] order: an
//                                      element's 4 NB coefficients are contiguous (48 to 320 bytes,
//                                      a multiple of 16), read with 16-byte loads; padded to ld
//                                      elements (element count rounded up to 32)
//   geometry   jac[ne], dinv[4][ld]   (dxi/dx, dxi/dy, deta/dx, deta/dy), hmin[ne], h15[ne]
//   faces      face[3][ld]            (edge slot << 1) | side, side 1 = element is the edge's
//                                      right element; slots [0, n_int) are internal edges,
//                                      [n_int, n_int + n_bnd) boundary edges
//   instance   inst[ne]               instance of each element
//   edge flux  F[slot][NG][4]          HLLC / boundary flux at the edge Gauss points times half
//                                      the edge length (type T); written by the edge pass,
//                                      gathered by the element pass (no atomics)
// Tables travel in the kernel parameter block (constant bank): every compile-time-indexed table
// read is a broadcast operand.  With T = float the volume/edge contractions, fluxes and stage
// updates run in FP32; the limiter (KXRCF detection, WENO indicators and weights), the
// positivity checks of HLLC and the time step stay in FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

namespace dgm {

constexpr int NEQ = 4;
constexpr double F64_EPS = 2.220446049250313e-16;  // f64::EPSILON, weno.rs:1

// Status codes (mirrors include/dgm_b200.h).
enum : int {
  ST_OK = 0,
  ST_NEG_DENSITY = 1,
  ST_NEG_PRESSURE = 2,
  ST_NONFINITE = 3,
  ST_TOO_MANY_BOUNDARY_EDGES = 4,
  ST_TIMEOUT = 6,
  ST_LIST_OVERFLOW = 12,
};

// Supported discretisations: (order, triangle rule, edge rule, derivative keys used by WENO).
template <int P> struct Variant;
template <> struct Variant<1> { static constexpr int NB = 3, NQ = 3, NG = 2, NK = 2; };
template <> struct Variant<2> { static constexpr int NB = 6, NQ = 6, NG = 3, NK = 5; };
template <> struct Variant<3> { static constexpr int NB = 10, NQ = 12, NG = 4, NK = 9; };

// Tables of the bulk kernels, in the storage type.
template <int P, typename T>
struct TablesT {
  using V = Variant<P>;
  T phi_cell[V::NQ][V::NB];          // phis_cell_gps
  T dxi[V::NQ][V::NB];               // d/dxi  at cell points
  T deta[V::NQ][V::NB];              // d/deta at cell points
  T phi_edge[3][V::NG][V::NB];       // phis_edge_gps
  T cell_w[V::NQ];
  T edge_w[V::NG];
  T inv_mass[V::NB];                 // 1 / mass_mat_diag
};

// FP64 tables of the limiter and the diagnostics.
template <int P>
struct TablesD {
  using V = Variant<P>;
  double phi_edge[3][V::NG][V::NB];
  double cell_w[V::NQ];
  double edge_w[V::NG];
  double dref[V::NQ][V::NB][V::NK];  // reference derivatives up to order P
};

struct MeshDev {
  int ne, ld, n_int, n_bnd, n_inst, _pad;
  const double* __restrict__ jac;     // [ne]
  const double* __restrict__ dinv;    // [4][ld]
  const double* __restrict__ hmin;    // [ne]
  const double* __restrict__ h15;     // [ne] circumradius^1.5
  const int* __restrict__ face;       // [3][ld]
  const int* __restrict__ nbr;        // [3][ld]  -1 on the boundary
  const int* __restrict__ inst;       // [ne] instance of each element
  const int2* __restrict__ ie_lr;     // [n_int] left, right element
  const int* __restrict__ ie_ic;      // [n_int] ilic | iric << 2
  const double4* __restrict__ ie_geo; // [n_int] nx, ny, half length, length
  const int* __restrict__ be_elem;    // [n_bnd]
  const int* __restrict__ be_info;    // [n_bnd] ic | type << 2 | patch << 3
  const double4* __restrict__ be_geo; // [n_bnd] outward nx, ny, half length, length
  const double4* __restrict__ patch_q;// [np] conserved far-field state
  const int64_t* __restrict__ slot_ref;  // [n_int + n_bnd] reference edge id of each slot
  const double* __restrict__ gram;    // [NB (NB + 1) / 2][ld] WENO Gram matrices (limiter on)
};

// Time-march state of one instance (TemperalDisc's current_time / current_step and the loop
// bounds of SolverParameters), advanced on the device.
struct InstCtl {
  double t, dt, final_time, cfl;
  long long step, final_step;
  unsigned long long dt_bits;  // atomicMin target of the instance's time step
  int active;                  // this step runs (loop condition of temporal_disc.rs:22)
  int status;                  // first error raised in this instance
  long long err_where;         // edge / element of that error
};

// Counters of one limiter wave, each on its own 128-byte line so that polling one does not slow
// the atomics on another: cells enlisted for reconstruction (tail), tickets handed to
// reconstructing warps (head), warps that finished the wave's scan (scanned) and cells left for a
// later wave (unknown).
struct alignas(128) LimQueue {
  int tail;
  int _pad0[31];
  int head;
  int _pad1[31];
  int scanned;
  int unknown;
  int _pad2[30];
};

__host__ __device__ __forceinline__ void reset_queue(LimQueue& q) {
  q.tail = 0;
  q.head = 0;
  q.scanned = 0;
  q.unknown = 0;
}

// Context-wide control block: first error, limiter counters, grid barrier.
struct Control {
  int status;                  // first error raised on the device (any instance)
  int _pad0;
  long long err_where;
  int t0_count;                // cells flagged by the parallel KXRCF pass
  int troubled;                // cells limited since the last step start
  int waves;                   // limiter waves of the last pass
  int unknown[2];              // barrier schedule: per-wave count of unsettled cells (double-buffered)
  int wl_count[2];             // barrier schedule: per-wave worklist length (double-buffered)
  int wl1_count;               // cells the detection enlisted for wave 1
  int pend_count;              // elements the detection left for later waves
  unsigned int bar_word;       // grid barrier of the limiter kernels: arrivals, top bit flips per barrier
  unsigned int head_done;      // blocks of k_step_head that have finished (last one closes the step head)
  LimQueue lq[3];              // queue schedule: per-wave queues, wave w uses lq[w % 3]
};

// Zeroes the counters, worklist lengths and queues of the limiter pass that follows.  Every launch
// that precedes a limiter pass calls it from one thread (the element passes, FMA and tensor-core,
// and k_set_active before host-driven passes): the detection's atomics then start from zero.
__device__ __forceinline__ void reset_limiter_pass(Control* ctl) {
  ctl->t0_count = 0;
  ctl->unknown[0] = ctl->unknown[1] = 0;
  ctl->wl_count[0] = ctl->wl_count[1] = 0;
  ctl->wl1_count = ctl->pend_count = 0;
  for (int w = 0; w < 3; ++w) reset_queue(ctl->lq[w]);
}

// Gas constants, computed once on the host from hcr with the reference's expressions.
struct Gas {
  double hcr;        // ratio of specific heats
  double gm1;        // hcr - 1
  double zeta;       // (hcr - 1) / (2 hcr)                      flux.rs:76
  double inv_zeta;   // 1 / zeta
  double zm1h;       // (zeta - 1) / 2                            flux.rs:77
  double gp1h;       // (hcr + 1) / (2 hcr)                       flux.rs:85,96
  int inv_zeta_int;  // 1/zeta when it is an integer to round-off (7 for hcr = 1.4), else 0
  int _pad;
};

template <int P, typename T>
struct KParams {
  TablesT<P, T> t;
  TablesD<P> d;
  MeshDev m;
  Gas gas;
  Control* ctl;
  InstCtl* ic;
};

__device__ __forceinline__ void raise_status(Control* ctl, InstCtl* ic, int code, long long where) {
  if (atomicCAS(&ic->status, 0, code) == 0) ic->err_where = where;
  if (atomicCAS(&ctl->status, 0, code) == 0) ctl->err_where = where;
}

// Stores v at list[i] when i is inside the list's capacity; otherwise drops it and reports
// ST_LIST_OVERFLOW (a worklist holds each element at most once per pass, so this only fires if
// its counter was not reset before the pass).
__device__ __forceinline__ void list_put(Control* ctl, int* __restrict__ list, int i, int cap, int v) {
  if (i < cap) {
    list[i] = v;
  } else if (atomicCAS(&ctl->status, 0, ST_LIST_OVERFLOW) == 0) {
    ctl->err_where = i;
  }
}

// Wave-1 worklist entries carry the element's faces and neighbours, so that the reconstruction
// that takes the entry needs no further dependent load before the states:
// list[8 i .. 8 i + 7] = {e, face[0..2], nbr[0..2], 0}.  Dropped and reported like list_put.
constexpr int kEntryInts = 8;
__device__ __forceinline__ void entry_put(Control* ctl, int* __restrict__ list, int i, int cap, int e,
                                          const int (&f)[3], const int (&n)[3]) {
  if (i < cap) {
    int4* p = reinterpret_cast<int4*>(list + (size_t)kEntryInts * i);
    p[0] = make_int4(e, f[0], f[1], f[2]);
    p[1] = make_int4(n[0], n[1], n[2], 0);
  } else if (atomicCAS(&ctl->status, 0, ST_LIST_OVERFLOW) == 0) {
    ctl->err_where = i;
  }
}

// Reads entry i of such a list into every lane of the warp (lanes 0-6 load one word each).
__device__ __forceinline__ int entry_get(const int* __restrict__ list, int i, int lane, int (&f)[3], int (&n)[3]) {
  const int v = lane < 7 ? __ldcg(&list[(size_t)kEntryInts * i + lane]) : 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    f[k] = __shfl_sync(0xffffffffu, v, 1 + k);
    n[k] = __shfl_sync(0xffffffffu, v, 4 + k);
  }
  return __shfl_sync(0xffffffffu, v, 0);
}

template <typename T>
__device__ __forceinline__ T ld_state(const T* p) { return __ldcg(p); }

// State load for a kernel that either only reads the array (RO: through L1, where neighbouring
// lanes' gathers reuse each other's lines) or writes it while reading (L2 only, always coherent).
template <bool RO, typename T>
__device__ __forceinline__ T ld_st(const T* p) {
  if constexpr (RO) return __ldg(p);
  else return __ldcg(p);
}

// An element's own coefficient: a plain load when the record is staged in shared memory.
template <bool RO, bool SHARED, typename T>
__device__ __forceinline__ T ld_own(const T* p) {
  if constexpr (SHARED) return *p;
  else return ld_st<RO>(p);
}

// Index of coefficient (v, b) of element e in an element-major state array.
template <int NB>
__host__ __device__ __forceinline__ size_t sx(int e, int v, int b) {
  return (size_t)e * (NEQ * NB) + (size_t)(v * NB + b);
}

// The NB modes of variable VAR of element e (L2 loads), converted to FP64, with the widest loads
// the block's alignment allows (its byte offset in the 16-byte aligned record is known at compile
// time): 16-byte loads for the density block and most others, 8- or 4-byte ones otherwise.
template <int NB, typename T, int VAR, bool RO = false>
__device__ __forceinline__ void load_var_modes(const T* __restrict__ U, int e, double (&out)[NB]) {
  constexpr int OFF = VAR * NB * (int)sizeof(T);  // byte offset of the block in the record
  constexpr int ALIGN = (OFF % 16 == 0) ? 16 : (OFF % 8 == 0) ? 8 : 4;
  const T* p = U + (size_t)e * (NEQ * NB) + VAR * NB;
  if constexpr (std::is_same<T, double>::value && ALIGN == 16) {
#pragma unroll
    for (int i = 0; i < NB / 2; ++i) {
      const double2 x = ld_st<RO>(reinterpret_cast<const double2*>(p) + i);
      out[2 * i] = x.x;
      out[2 * i + 1] = x.y;
    }
    if constexpr (NB % 2) out[NB - 1] = ld_st<RO>(p + NB - 1);
  } else if constexpr (std::is_same<T, float>::value && ALIGN == 16) {
#pragma unroll
    for (int i = 0; i < NB / 4; ++i) {
      const float4 x = ld_st<RO>(reinterpret_cast<const float4*>(p) + i);
      out[4 * i] = x.x;
      out[4 * i + 1] = x.y;
      out[4 * i + 2] = x.z;
      out[4 * i + 3] = x.w;
    }
#pragma unroll
    for (int i = NB / 4 * 4; i < NB; ++i) out[i] = ld_st<RO>(p + i);
  } else if constexpr (std::is_same<T, float>::value && ALIGN == 8) {
#pragma unroll
    for (int i = 0; i < NB / 2; ++i) {
      const float2 x = ld_st<RO>(reinterpret_cast<const float2*>(p) + i);
      out[2 * i] = x.x;
      out[2 * i + 1] = x.y;
    }
    if constexpr (NB % 2) out[NB - 1] = ld_st<RO>(p + NB - 1);
  } else {
#pragma unroll
    for (int i = 0; i < NB; ++i) out[i] = (double)ld_st<RO>(p + i);
  }
}

// All 4 NB coefficients of element e with 16-byte loads (the record is 16-byte aligned for every
// order and storage type).  L1 = true caches in L1 (for arrays no thread writes during the
// kernel); otherwise the loads go to L2 only.
template <int NB, typename T, bool L1 = false>
__device__ __forceinline__ void load_elem(const T* __restrict__ U, int e, T (&u)[NEQ * NB]) {
  constexpr int N = NEQ * NB;
  if constexpr (std::is_same<T, double>::value) {
    const double2* p = reinterpret_cast<const double2*>(U + (size_t)e * N);
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const double2 x = L1 ? p[i] : __ldcg(p + i);
      u[2 * i] = x.x;
      u[2 * i + 1] = x.y;
    }
  } else {
    const float4* p = reinterpret_cast<const float4*>(U + (size_t)e * N);
#pragma unroll
    for (int i = 0; i < N / 4; ++i) {
      const float4 x = L1 ? p[i] : __ldcg(p + i);
      u[4 * i] = x.x;
      u[4 * i + 1] = x.y;
      u[4 * i + 2] = x.z;
      u[4 * i + 3] = x.w;
    }
  }
}

// flux::flux, flux.rs:154-169 (one reciprocal of the density instead of three divisions)
template <typename T>
__device__ __forceinline__ void euler_flux(const T q[4], T gm1, T f[4], T g[4]) {
  const T rq = T(1) / q[0];
  const T u = q[1] * rq;
  const T v = q[2] * rq;
  const T p = gm1 * (q[3] - T(0.5) * (q[1] * q[1] + q[2] * q[2]) * rq);
  f[0] = q[1];
  f[1] = q[1] * u + p;
  f[2] = q[2] * u;
  f[3] = u * (q[3] + p);
  g[0] = q[2];
  g[1] = q[1] * v;
  g[2] = q[2] * v + p;
  g[3] = v * (q[3] + p);
}

template <typename T>
__device__ __forceinline__ T ipow(T x, int n) {
  T r = T(1);
  while (n) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}

// flux::hllc, flux.rs:28-153.  Returns ST_NEG_DENSITY / ST_NEG_PRESSURE like the reference's Err.
// Same formulas; densities enter through their reciprocals, x^zeta as exp(zeta log x), and
// (.)^(1/zeta) as an integer power when 1/zeta is an integer to round-off (hcr = 1.4: 7);
// both differ from the reference's libm pow only in the last bits.  In FP32 the density and
// pressure checks are evaluated in FP64.
template <typename T>
__device__ __forceinline__ int hllc(const T lv[4], const T rv[4], T nx, T ny, const Gas& gas, T flux[4]) {
  const T gm1 = T(gas.gm1), hcr = T(gas.hcr);
  const T ql0 = lv[0], ql1 = lv[1] * nx + lv[2] * ny, ql2 = -lv[1] * ny + lv[2] * nx, ql3 = lv[3];
  const T qr0 = rv[0], qr1 = rv[1] * nx + rv[2] * ny, qr2 = -rv[1] * ny + rv[2] * nx, qr3 = rv[3];
  const T rl = T(1) / ql0, rr = T(1) / qr0;
  const T ul = ql1 * rl, ur = qr1 * rr, vl = ql2 * rl, vr = qr2 * rr;
  const T pl = gm1 * (ql3 - T(0.5) * (ql1 * ql1 + ql2 * ql2) * rl);
  const T pr = gm1 * (qr3 - T(0.5) * (qr1 * qr1 + qr2 * qr2) * rr);
  if constexpr (std::is_same<T, double>::value) {
    if (ql0 < 0.0 || qr0 < 0.0) return ST_NEG_DENSITY;
    if (pl < 0.0 || pr < 0.0) return ST_NEG_PRESSURE;
  } else {
    // the sign of an FP32 density is the sign of its FP64 value: no FP64 arithmetic needed
    if (lv[0] < 0.0f || rv[0] < 0.0f) return ST_NEG_DENSITY;
    // The FP32 pressure is within a few FP32 ulps of max(E, kinetic energy) of the FP64 pressure of
    // the same traces, so where it exceeds 1e-4 |E| the FP64 pressure is positive as well; only
    // pressures that are small against the energy are decided in FP64 (same decisions as always
    // evaluating in FP64, at a fraction of the cost).
    if (!(pl > 1e-4f * fabsf(ql3)) || !(pr > 1e-4f * fabsf(qr3))) {
      const double dl0 = lv[0], dr0 = rv[0];
      const double dpl = gas.gm1 * ((double)lv[3] - 0.5 * ((double)lv[1] * lv[1] + (double)lv[2] * lv[2]) / dl0);
      const double dpr = gas.gm1 * ((double)rv[3] - 0.5 * ((double)rv[1] * rv[1] + (double)rv[2] * rv[2]) / dr0);
      if (dpl < 0.0 || dpr < 0.0) return ST_NEG_PRESSURE;
    }
  }
  const T cl = sqrt(hcr * pl * rl);
  const T cr = sqrt(hcr * pr * rr);
  const T fl0 = ql1, fl1 = ql1 * ul + pl, fl2 = ql2 * ul, fl3 = ul * (ql3 + pl);
  const T fr0 = qr1, fr1 = qr1 * ur + pr, fr2 = qr2 * ur, fr3 = ur * (qr3 + pr);
  // PVRS-type p*, flux.rs:75-78
  const T zeta = T(gas.zeta);
  const T base = (cl + cr - T(gas.zm1h) * (ur - ul)) / (cl * exp(-zeta * log(pl)) + cr * exp(-zeta * log(pr)));
  const T p_star = gas.inv_zeta_int ? ipow(base, gas.inv_zeta_int) : exp(T(gas.inv_zeta) * log(base));
  const T ql_lower = (p_star <= pl) ? T(1) : sqrt(T(1) + T(gas.gp1h) * (p_star / pl - T(1)));
  const T sl = ul - cl * ql_lower;
  const T qr_lower = (p_star <= pr) ? T(1) : sqrt(T(1) + T(gas.gp1h) * (p_star / pr - T(1)));
  const T sr = ur + cr * qr_lower;
  T f0, fn, ft, f3;
  if (sl >= T(0)) {
    f0 = fl0; fn = fl1; ft = fl2; f3 = fl3;
  } else if (sr <= T(0)) {
    f0 = fr0; fn = fr1; ft = fr2; f3 = fr3;
  } else {
    const T s_star = (pr - pl + ql0 * ul * (sl - ul) - qr0 * ur * (sr - ur)) / (ql0 * (sl - ul) - qr0 * (sr - ur));
    if (s_star >= T(0)) {
      const T dl = ql0 * (sl - ul);
      const T m = dl / (sl - s_star);
      const T qs0 = m, qs1 = m * s_star, qs2 = m * vl;
      const T qs3 = m * (ql3 * rl + (s_star - ul) * (s_star + pl / dl));
      f0 = fl0 + sl * (qs0 - ql0);
      fn = fl1 + sl * (qs1 - ql1);
      ft = fl2 + sl * (qs2 - ql2);
      f3 = fl3 + sl * (qs3 - ql3);
    } else {
      const T dr = qr0 * (sr - ur);
      const T m = dr / (sr - s_star);
      const T qs0 = m, qs1 = m * s_star, qs2 = m * vr;
      const T qs3 = m * (qr3 * rr + (s_star - ur) * (s_star + pr / dr));
      f0 = fr0 + sr * (qs0 - qr0);
      fn = fr1 + sr * (qs1 - qr1);
      ft = fr2 + sr * (qs2 - qr2);
      f3 = fr3 + sr * (qs3 - qr3);
    }
  }
  flux[0] = f0;
  flux[1] = fn * nx - ft * ny;
  flux[2] = fn * ny + ft * nx;
  flux[3] = f3;
  return ST_OK;
}

// compute_eigenmatrix, local_characteristics.rs:4-50 (reciprocals of rho and c)
template <typename T>
__device__ __forceinline__ void eigenmatrix(const T q[4], T nx, T ny, const Gas& gas, T L[4][4], T R[4][4]) {
  const T gm1 = T(gas.gm1), hcr = T(gas.hcr);
  const T rq = T(1) / q[0];
  const T u = q[1] * rq;
  const T v = q[2] * rq;
  const T p = gm1 * (q[3] - T(0.5) * (q[1] * q[1] + q[2] * q[2]) * rq);
  const T c = sqrt(hcr * p * rq);
  const T ic = T(1) / c;
  const T h = (q[3] + p) * rq;
  const T b1 = gm1 * (ic * ic);
  const T b2 = b1 * (u * u + v * v) * T(0.5);
  const T vn = u * nx + v * ny;
  L[0][0] = (b2 + vn * ic) * T(0.5);
  L[0][1] = -(b1 * u + nx * ic) * T(0.5);
  L[0][2] = -(b1 * v + ny * ic) * T(0.5);
  L[0][3] = b1 * T(0.5);
  L[1][0] = ny * u - nx * v;
  L[1][1] = -ny;
  L[1][2] = nx;
  L[1][3] = T(0);
  L[2][0] = T(1) - b2;
  L[2][1] = b1 * u;
  L[2][2] = b1 * v;
  L[2][3] = -b1;
  L[3][0] = (b2 - vn * ic) * T(0.5);
  L[3][1] = -(b1 * u - nx * ic) * T(0.5);
  L[3][2] = -(b1 * v - ny * ic) * T(0.5);
  L[3][3] = b1 * T(0.5);
  R[0][0] = T(1);
  R[0][1] = T(0);
  R[0][2] = T(1);
  R[0][3] = T(1);
  R[1][0] = u - c * nx;
  R[1][1] = -ny;
  R[1][2] = u;
  R[1][3] = u + c * nx;
  R[2][0] = v - c * ny;
  R[2][1] = nx;
  R[2][2] = v;
  R[2][3] = v + c * ny;
  R[3][0] = h - c * vn;
  R[3][1] = -u * ny + v * nx;
  R[3][2] = (u * u + v * v) * T(0.5);
  R[3][3] = h + c * vn;
}

// Physical derivative of a mode for key kk from reference derivatives r[] (mesh.rs:101-114;
// third order: the same chain rule expanded, p=3 extension).
template <int NK>
__device__ __forceinline__ double phys_deriv(const double (&r)[NK], double xx, double xy, double ex,
                                             double ey, int kk) {
  switch (kk) {
    case 0: return xx * r[0] + ex * r[1];
    case 1: return xy * r[0] + ey * r[1];
  }
  if constexpr (NK >= 5) {
    switch (kk) {
      case 2: return (xx * xx) * r[2] + 2.0 * xx * ex * r[3] + (ex * ex) * r[4];
      case 3: return xx * xy * r[2] + (xx * ey + ex * xy) * r[3] + ex * ey * r[4];
      case 4: return (xy * xy) * r[2] + 2.0 * xy * ey * r[3] + (ey * ey) * r[4];
    }
  }
  if constexpr (NK >= 9) {
    // (xx Dxi + ex Deta)^a (xy Dxi + ey Deta)^c, a + c = 3, c = kk - 5
    switch (kk) {
      case 5: return xx * xx * xx * r[5] + 3.0 * xx * xx * ex * r[6] + 3.0 * xx * ex * ex * r[7] + ex * ex * ex * r[8];
      case 6: return xx * xx * xy * r[5] + (xx * xx * ey + 2.0 * xx * ex * xy) * r[6] +
                     (2.0 * xx * ex * ey + ex * ex * xy) * r[7] + ex * ex * ey * r[8];
      case 7: return xx * xy * xy * r[5] + (2.0 * xx * xy * ey + ex * xy * xy) * r[6] +
                     (xx * ey * ey + 2.0 * ex * xy * ey) * r[7] + ex * ey * ey * r[8];
      case 8: return xy * xy * xy * r[5] + 3.0 * xy * xy * ey * r[6] + 3.0 * xy * ey * ey * r[7] + ey * ey * ey * r[8];
    }
  }
  return 0.0;
}

// Boundary flux at one Gauss point of a boundary slot, from the interior trace lv (times
// nothing: the caller scales by half the edge length).  Slip wall: the pressure flux
// [0, p nx, p ny, 0] (boundary_condition.rs:31-47); far field: characteristic upwinding between
// the interior trace and the patch's free stream, then the physical normal flux of the blended
// state (boundary_condition.rs:48-94).  (nx, ny) is the element's outward normal.
// The far-field boundary state (boundary_condition.rs:64-73): the characteristic variables of the
// interior trace lv where the wave leaves the domain (eigenvalue >= 0), of the free stream bq
// (conserved) where it enters, mapped back to conserved variables.
template <typename T>
__device__ __forceinline__ void far_field_state(const T lv[4], T nx, T ny, const double4 bq, const Gas& gas, T q[4]) {
  const T gm1 = T(gas.gm1);
  const T bc[4] = {T(bq.x), T(bq.y), T(bq.z), T(bq.w)};
  const T u = lv[1] / lv[0];
  const T v = lv[2] / lv[0];
  const T p = gm1 * (lv[3] - T(0.5) * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
  const T c = sqrt(T(gas.hcr) * p / lv[0]);
  const T vn = u * nx + v * ny;
  T Lm[4][4], Rm[4][4];
  eigenmatrix<T>(lv, nx, ny, gas, Lm, Rm);
  const T lam[4] = {vn - c, vn, vn, vn + c};
  T mix[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    T alpha = T(0), beta = T(0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      alpha += Lm[i][j] * lv[j];
      beta += Lm[i][j] * bc[j];
    }
    mix[i] = lam[i] >= T(0) ? alpha : beta;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    T sum = T(0);
#pragma unroll
    for (int j = 0; j < 4; ++j) sum += Rm[i][j] * mix[j];
    q[i] = sum;
  }
}

template <typename T>
__device__ __forceinline__ void boundary_flux(const T lv[4], int info, T nx, T ny, const MeshDev& m, const Gas& gas,
                                              T out[4]) {
  const T gm1 = T(gas.gm1);
  if (((info >> 2) & 1) == 0) {
    const T pressure = gm1 * (lv[3] - T(0.5) * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
    out[0] = T(0);
    out[1] = pressure * nx;
    out[2] = pressure * ny;
    out[3] = T(0);
    return;
  }
  T q[4];
  far_field_state<T>(lv, nx, ny, m.patch_q[info >> 3], gas, q);
  const T un = q[1] / q[0];
  const T vv = q[2] / q[0];
  const T vn_new = un * nx + vv * ny;
  const T p_new = gm1 * (q[3] - T(0.5) * (q[1] * q[1] + q[2] * q[2]) / q[0]);
  const T h_new = q[3] + p_new;
  out[0] = q[0] * vn_new;
  out[1] = q[1] * vn_new + p_new * nx;
  out[2] = q[2] * vn_new + p_new * ny;
  out[3] = h_new * vn_new;
}

template <typename T>
__device__ __forceinline__ void store_flux(T* F, size_t s, int NG, int g, const T out[4]) {
  T* dst = &F[(s * NG + g) * 4];
  if constexpr (std::is_same<T, double>::value) {
    reinterpret_cast<double2*>(dst)[0] = make_double2(out[0], out[1]);
    reinterpret_cast<double2*>(dst)[1] = make_double2(out[2], out[3]);
  } else {
    reinterpret_cast<float4*>(dst)[0] = make_float4(out[0], out[1], out[2], out[3]);
  }
}

// ------------------------------------------------------------------------------------------
// Edge pass: one thread per (edge slot, Gauss point).  Internal slots: traces of both
// elements + HLLC (integrate_over_edges_euler, spatial_disc.rs:161-211).  Boundary slots:
// slip-wall pressure flux or characteristic far-field flux (apply_bc_euler,
// boundary_condition.rs:19-97).  Writes F[slot][g][v] * half length.  Slots of instances that
// are not stepping are skipped.
// An element's record loaded from storage type S and converted to the arithmetic type T (FP64
// storage with FP32 arithmetic; the plain load when the types agree).
template <int NB, typename S, typename T, bool L1 = false>
__device__ __forceinline__ void load_elem_as(const S* __restrict__ U, int e, T (&u)[NEQ * NB]) {
  if constexpr (std::is_same<S, T>::value) {
    load_elem<NB, T, L1>(U, e, u);
  } else {
    S w[NEQ * NB];
    load_elem<NB, S, L1>(U, e, w);
#pragma unroll
    for (int i = 0; i < NEQ * NB; ++i) u[i] = T(w[i]);
  }
}

// ------------------------------------------------------------------------------------------
// The kernels' bodies take their block index and block count within the launch (bid, nblk) as
// arguments, so that a launch over several meshes of different orders (a mixed batch) can give each
// order's body its own range of blocks; the single-order kernels pass blockIdx.x and gridDim.x.
// S is the state's storage type (FP64 storage with FP32 arithmetic: S = double, T = float).
template <int P, typename T, typename S = T>
__device__ __forceinline__ void edge_flux_body(const KParams<P, T>& kp, const S* __restrict__ U, T* __restrict__ F,
                                               int bid, int nblk) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  __shared__ T s_pe[3 * NG * NB];
  for (int i = threadIdx.x; i < 3 * NG * NB; i += blockDim.x) s_pe[i] = (&kp.t.phi_edge[0][0][0])[i];
  __syncthreads();
  const MeshDev& m = kp.m;
  const Gas& gas = kp.gas;
  const int total = (m.n_int + m.n_bnd) * NG;
  for (int t = bid * blockDim.x + threadIdx.x; t < total; t += nblk * blockDim.x) {
    const int s = t / NG, g = t - s * NG;
    T out[4];
    if (s < m.n_int) {
      const int2 lr = m.ie_lr[s];
      const int inst = m.n_inst > 1 ? m.inst[lr.x] : 0;
      if (!kp.ic[inst].active) continue;
      const int ic = m.ie_ic[s];
      const T* pl = &s_pe[((ic & 3) * NG + g) * NB];
      const T* pr = &s_pe[((ic >> 2) * NG + (NG - 1 - g)) * NB];
      T ul[NEQ * NB], ur[NEQ * NB];
      load_elem_as<NB, S, T>(U, lr.x, ul);
      load_elem_as<NB, S, T>(U, lr.y, ur);
      T lv[4], rv[4];
#pragma unroll
      for (int v = 0; v < NEQ; ++v) {
        T a = T(0), c = T(0);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          a += ul[v * NB + b] * pl[b];
          c += ur[v * NB + b] * pr[b];
        }
        lv[v] = a;
        rv[v] = c;
      }
      const double4 geo = m.ie_geo[s];
      const int st = hllc<T>(lv, rv, T(geo.x), T(geo.y), gas, out);
      if (st != ST_OK) raise_status(kp.ctl, &kp.ic[inst], st, m.slot_ref[s]);
#pragma unroll
      for (int v = 0; v < NEQ; ++v) out[v] *= T(geo.z);
    } else {
      const int sb = s - m.n_int;
      const int e = m.be_elem[sb];
      const int inst = m.n_inst > 1 ? m.inst[e] : 0;
      if (!kp.ic[inst].active) continue;
      const int info = m.be_info[sb];
      const T* pe = &s_pe[((info & 3) * NG + g) * NB];
      T ue[NEQ * NB];
      load_elem_as<NB, S, T>(U, e, ue);
      T lv[4];
#pragma unroll
      for (int v = 0; v < NEQ; ++v) {
        T a = T(0);
#pragma unroll
        for (int b = 0; b < NB; ++b) a += ue[v * NB + b] * pe[b];
        lv[v] = a;
      }
      const double4 geo = m.be_geo[sb];
      boundary_flux<T>(lv, info, T(geo.x), T(geo.y), m, gas, out);
#pragma unroll
      for (int v = 0; v < NEQ; ++v) out[v] *= T(geo.z);
    }
    store_flux<T>(F, (size_t)s, NG, g, out);
  }
}

template <int P, typename T, typename S = T>
__global__ void __launch_bounds__(256, 3) k_edge_flux(const __grid_constant__ KParams<P, T> kp,
                                                      const S* __restrict__ U, T* __restrict__ F) {
  edge_flux_body<P, T, S>(kp, U, F, blockIdx.x, gridDim.x);
}

// The same kernel compiled for 4 blocks of 256 threads per SM (at most 64 registers, a few bytes
// of spills) instead of 3: more warps in flight for the latency-bound gathers, more local-memory
// traffic; the autotuner picks one of the two per context.
template <int P, typename T, typename S = T>
__global__ void __launch_bounds__(256, 4) k_edge_flux_r64(const __grid_constant__ KParams<P, T> kp,
                                                          const S* __restrict__ U, T* __restrict__ F) {
  edge_flux_body<P, T, S>(kp, U, F, blockIdx.x, gridDim.x);
}

// The same edge pass with two lanes per edge slot, one per side: each lane loads its element's
// modes once, evaluates the traces at all NG points (the right side at the reversed points,
// spatial_disc.rs:185), the pair swaps traces with shuffles, and the two lanes split the points
// for HLLC / the boundary flux.  Each element's state is loaded once per slot instead of once per
// point; every trace and flux is the same expression in the same order as in k_edge_flux, so the
// results are bitwise identical.  A warp covers 16 consecutive slots per iteration.
template <int P, typename T, typename S = T>
__device__ __forceinline__ void edge_flux_pair_body(const KParams<P, T>& kp, const S* __restrict__ U,
                                                    T* __restrict__ F, int bid, int nblk) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  constexpr int G0 = (NG + 1) / 2;  // points of the left lane: [0, G0); right lane: [G0, NG)
  __shared__ T s_pe[3 * NG * NB];
  for (int i = threadIdx.x; i < 3 * NG * NB; i += blockDim.x) s_pe[i] = (&kp.t.phi_edge[0][0][0])[i];
  __syncthreads();
  const MeshDev& m = kp.m;
  const Gas& gas = kp.gas;
  const int total = m.n_int + m.n_bnd;
  const int lane = threadIdx.x & 31, side = lane & 1;
  const int gwarp = (bid * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (nblk * blockDim.x) >> 5;
  for (int base = gwarp * 16; base < total; base += nwarps * 16) {
    const int s = base + (lane >> 1);
    bool valid = s < total, internal = false, has = false;
    int e = 0, k = 0, inst = 0, info = 0;
    if (valid) {
      if (s < m.n_int) {
        internal = true;
        const int2 lr = m.ie_lr[s];
        const int ic = m.ie_ic[s];
        e = side ? lr.y : lr.x;
        k = side ? (ic >> 2) : (ic & 3);
        inst = m.n_inst > 1 ? m.inst[lr.x] : 0;
        has = true;
      } else {
        const int sb = s - m.n_int;
        e = m.be_elem[sb];
        info = m.be_info[sb];
        k = info & 3;
        inst = m.n_inst > 1 ? m.inst[e] : 0;
        has = side == 0;
      }
      if (!kp.ic[inst].active) valid = has = false;
    }
    T u[NEQ * NB];
    if (has) {
      load_elem_as<NB, S, T>(U, e, u);
    } else {
#pragma unroll
      for (int i = 0; i < NEQ * NB; ++i) u[i] = T(0);
    }
    T tr[NEQ][NG];
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        const T* pe = &s_pe[(k * NG + (side ? NG - 1 - g : g)) * NB];
        T a = T(0);
#pragma unroll
        for (int b = 0; b < NB; ++b) a += u[v * NB + b] * pe[b];
        tr[v][g] = a;
      }
    }
    T ot[NEQ][NG];
#pragma unroll
    for (int v = 0; v < NEQ; ++v)
#pragma unroll
      for (int g = 0; g < NG; ++g) ot[v][g] = __shfl_xor_sync(0xffffffffu, tr[v][g], 1);
    if (!valid) continue;
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      if ((g < G0) != (side == 0)) continue;
      T lv[4], rv[4], out[4];
#pragma unroll
      for (int v = 0; v < NEQ; ++v) {
        lv[v] = side ? ot[v][g] : tr[v][g];
        rv[v] = side ? tr[v][g] : ot[v][g];
      }
      if (internal) {
        const double4 geo = m.ie_geo[s];
        const int st = hllc<T>(lv, rv, T(geo.x), T(geo.y), gas, out);
        if (st != ST_OK) raise_status(kp.ctl, &kp.ic[inst], st, m.slot_ref[s]);
#pragma unroll
        for (int v = 0; v < NEQ; ++v) out[v] *= T(geo.z);
      } else {
        const double4 geo = m.be_geo[s - m.n_int];
        boundary_flux<T>(lv, info, T(geo.x), T(geo.y), m, gas, out);
#pragma unroll
        for (int v = 0; v < NEQ; ++v) out[v] *= T(geo.z);
      }
      store_flux<T>(F, (size_t)s, NG, g, out);
    }
  }
}

template <int P, typename T, typename S = T>
__global__ void __launch_bounds__(256, 2) k_edge_flux_pair(const __grid_constant__ KParams<P, T> kp,
                                                           const S* __restrict__ U, T* __restrict__ F) {
  edge_flux_pair_body<P, T, S>(kp, U, F, blockIdx.x, gridDim.x);
}

// Element records staged in shared memory are padded to an odd number of 16-byte units:
// consecutive lanes reading the same coefficient of their own records then spread over the banks
// (2-way conflicts for FP64, 4-way for FP32, the least 16-byte granularity allows; unpadded
// records of 48-320 bytes map most lanes to the same few banks).
template <int NB, typename T>
struct Staged {
  static constexpr int kRecBytes = NEQ * NB * (int)sizeof(T);
  static constexpr int kStrideBytes = kRecBytes + ((kRecBytes / 16) % 2 == 0 ? 16 : 32);
  static constexpr int kStride = kStrideBytes / (int)sizeof(T);  // record stride in T
  static constexpr int kCpr = kRecBytes / 16;                          // 16-byte chunks per record
  static_assert(kRecBytes % 16 == 0, "element records are a multiple of 16 bytes");
};

// The edge pass with the records of a warp's slots staged in shared memory: NG lanes per slot (one
// per Gauss point), 32 / NG slots per warp iteration.  The warp first copies both sides' records of
// its slots with coalesced 16-byte loads -- each record once per slot, where the per-point form
// loads it NG times -- and then every lane evaluates its point's traces from shared memory and the
// HLLC / boundary flux.  The traces, fluxes and stores are the same expressions in the same order
// as in k_edge_flux, so the results are bitwise identical.  Blocks of kEdgeStagedThreads.
constexpr int kEdgeStagedThreads = 128;

template <int P, typename T, typename S = T>
__device__ __forceinline__ void edge_flux_staged_body(const KParams<P, T>& kp, const S* __restrict__ U,
                                                      T* __restrict__ F, int bid, int nblk) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  constexpr int SPW = 32 / NG;                    // slots per warp iteration
  constexpr int STRIDE = Staged<NB, S>::kStride;  // record stride in S: an odd number of 16-byte units
  constexpr int CPR = Staged<NB, S>::kCpr;        // 16-byte chunks per record
  constexpr int WARPS = kEdgeStagedThreads / 32;
  __shared__ T s_pe[3 * NG * NB];
  __shared__ __align__(16) S s_rec[WARPS][2][SPW * STRIDE];  // [side][slot record]
  for (int i = threadIdx.x; i < 3 * NG * NB; i += blockDim.x) s_pe[i] = (&kp.t.phi_edge[0][0][0])[i];
  __syncthreads();
  const MeshDev& m = kp.m;
  const Gas& gas = kp.gas;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int sl = lane / NG, g = lane - sl * NG;
  const int gwarp = bid * WARPS + wib, nwarps = nblk * WARPS;
  const int total = m.n_int + m.n_bnd;
  for (int base = gwarp * SPW; base < total; base += nwarps * SPW) {
    const int s = base + sl;
    bool valid = sl < SPW && s < total, internal = false;
    int eL = -1, eR = -1, inst = 0, ic = 0, info = 0;
    if (valid) {
      if (s < m.n_int) {
        const int2 lr = m.ie_lr[s];
        eL = lr.x;
        eR = lr.y;
        internal = true;
        ic = m.ie_ic[s];
      } else {
        const int sb = s - m.n_int;
        eL = m.be_elem[sb];
        info = m.be_info[sb];
      }
      inst = m.n_inst > 1 ? m.inst[eL] : 0;
      if (!kp.ic[inst].active) valid = false;
    }
    // stage the records: chunk c of record r = side * SPW + slot
    constexpr int TOT = 2 * SPW * CPR, IT = (TOT + 31) / 32;
    const int myL = valid ? eL : -1, myR = (valid && internal) ? eR : -1;
    __syncwarp();
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int c = lane + 32 * it;
      const int r = c / CPR, k = c - r * CPR;
      const int side = r / SPW, slot = r - side * SPW;
      const int src = (slot < SPW ? slot : 0) * NG;
      const int eLs = __shfl_sync(0xffffffffu, myL, src);
      const int eRs = __shfl_sync(0xffffffffu, myR, src);
      const int e = side ? eRs : eLs;
      if (c < TOT && e >= 0) {
        const uint4* gsrc = reinterpret_cast<const uint4*>(U + (size_t)e * (NEQ * NB));
        *reinterpret_cast<uint4*>(&s_rec[wib][side][slot * STRIDE + k * (16 / (int)sizeof(S))]) = __ldcg(gsrc + k);
      }
    }
    __syncwarp();
    if (!valid) continue;
    T out[4];
    const S* recL = &s_rec[wib][0][sl * STRIDE];
    if (internal) {
      const S* recR = &s_rec[wib][1][sl * STRIDE];
      const T* pl = &s_pe[((ic & 3) * NG + g) * NB];
      const T* pr = &s_pe[((ic >> 2) * NG + (NG - 1 - g)) * NB];
      T lv[4], rv[4];
#pragma unroll
      for (int v = 0; v < NEQ; ++v) {
        T a = T(0), c = T(0);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          a += T(recL[v * NB + b]) * pl[b];
          c += T(recR[v * NB + b]) * pr[b];
        }
        lv[v] = a;
        rv[v] = c;
      }
      const double4 geo = m.ie_geo[s];
      const int st = hllc<T>(lv, rv, T(geo.x), T(geo.y), gas, out);
      if (st != ST_OK) raise_status(kp.ctl, &kp.ic[inst], st, m.slot_ref[s]);
#pragma unroll
      for (int v = 0; v < NEQ; ++v) out[v] *= T(geo.z);
    } else {
      const T* pe = &s_pe[((info & 3) * NG + g) * NB];
      T lv[4];
#pragma unroll
      for (int v = 0; v < NEQ; ++v) {
        T a = T(0);
#pragma unroll
        for (int b = 0; b < NB; ++b) a += T(recL[v * NB + b]) * pe[b];
        lv[v] = a;
      }
      const double4 geo = m.be_geo[s - m.n_int];
      boundary_flux<T>(lv, info, T(geo.x), T(geo.y), m, gas, out);
#pragma unroll
      for (int v = 0; v < NEQ; ++v) out[v] *= T(geo.z);
    }
    store_flux<T>(F, (size_t)s, NG, g, out);
  }
}

template <int P, typename T, typename S = T>
__global__ void __launch_bounds__(kEdgeStagedThreads, 4) k_edge_flux_staged(const __grid_constant__ KParams<P, T> kp,
                                                                         const S* __restrict__ U, T* __restrict__ F) {
  edge_flux_staged_body<P, T, S>(kp, U, F, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------------------------------------
// Element pass: volume integral (integrate_over_cell_euler, spatial_disc.rs:40-69, and
// boundary_condition.rs:98-117 for boundary elements), gather of the three faces' edge fluxes
// with the left/right sign and Gauss-point reversal of spatial_disc.rs:202-206, inverse mass
// (spatial_disc.rs:349-357), then the SSP-RK3 stage combination of rk3.rs:10,16,22.
//   MODE 0: out = (Rin + terms) / mass            (compute_residuals semantics)
//   MODE 1: out = Uin + dt R
//   MODE 2: out = 0.75 Ubase + 0.25 (Uin + dt R)
//   MODE 3: out = 1/3 Ubase + 2/3 (Uin + dt R)
// Four threads per element, one per conserved variable: lane = v * 8 + i within a warp that
// covers 8 elements.  The quadrature-point states are exchanged with shuffles, so a thread
// holds only its variable's NB modes and residuals.  The warp's 8 element records are one
// contiguous block of the element-major arrays: it moves them between global and shared memory
// with 16-byte accesses (coalesced), and each thread reads and writes its variable's modes in
// shared memory.  Elements of instances that are not stepping are left untouched (their records
// are not stored).
// ------------------------------------------------------------------------------------------
constexpr int kElemMaxWarps = 8;  // element pass: at most 256 threads per block

// Copies the NR element records starting at e0 (always inside the arrays, which are padded to a
// multiple of 32 elements, with e0 a multiple of NR) into the warp's shared buffer (record r at
// sbuf + r * Staged::kStride), with coalesced 16-byte loads through L2.
template <int NB, typename T, int NR = 8>
__device__ __forceinline__ void warp_load_records(const T* __restrict__ src, int e0, T* sbuf, int lane) {
  using S = Staged<NB, T>;
  constexpr int C = NR * S::kCpr;
  const uint4* g = reinterpret_cast<const uint4*>(src + (size_t)e0 * NEQ * NB);
  __syncwarp();
#pragma unroll
  for (int c = lane; c < C; c += 32)
    *reinterpret_cast<uint4*>(sbuf + (c / S::kCpr) * S::kStride + (c % S::kCpr) * (16 / (int)sizeof(T))) = __ldcg(g + c);
  __syncwarp();
}

// Stores the warp's shared buffer to the 8 element records starting at e0, skipping the records
// of elements whose bit in `keep` is clear.
template <int NB, typename T>
__device__ __forceinline__ void warp_store_records(T* dst, int e0, const T* sbuf, unsigned int keep, int lane) {
  using S = Staged<NB, T>;
  constexpr int C = 8 * S::kCpr;
  uint4* g = reinterpret_cast<uint4*>(dst + (size_t)e0 * NEQ * NB);
  __syncwarp();
#pragma unroll
  for (int c = lane; c < C; c += 32)
    if ((keep >> (c / S::kCpr)) & 1u)
      g[c] = *reinterpret_cast<const uint4*>(sbuf + (c / S::kCpr) * S::kStride + (c % S::kCpr) * (16 / (int)sizeof(T)));
  __syncwarp();
}

// S is the state's storage type: with S = double and T = float the contractions, fluxes and the
// residual are FP32 and the stage combination is evaluated in FP64 on the FP64 state.
template <int P, typename T, int MODE, typename S = T>
__device__ __forceinline__ void element_body(const KParams<P, T>& kp, const S* __restrict__ Uin, const S* Ubase,
                                             const T* __restrict__ F, S* Uout, const S* Rin, S* Rout, int bid) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NQ = V::NQ, NG = V::NG;
  constexpr int STRIDE = Staged<NB, S>::kStride;
  __shared__ __align__(16) S s_rec[kElemMaxWarps][8 * STRIDE];
  Control* ctl = kp.ctl;
  if (bid == 0 && threadIdx.x == 0) reset_limiter_pass(ctl);  // for the limiter pass that follows
  const MeshDev& m = kp.m;
  const int lane = threadIdx.x & 31;
  const int var = lane >> 3, i = lane & 7;
  const int e0 = (bid * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 8;
  const int e_raw = e0 + i;
  if (e0 >= m.ne) return;  // whole warp past the end
  const int e = e_raw < m.ne ? e_raw : m.ne - 1;
  const int inst = m.n_inst > 1 ? m.inst[e] : 0;
  const bool valid = e_raw < m.ne && kp.ic[inst].active;
  const unsigned int keep = __ballot_sync(0xffffffffu, valid) & 0xffu;  // lanes 0-7: var 0 of each element
  if (!keep) return;  // no element of this warp is stepping (finished instances, slot padding)
  const size_t ld = m.ld;
  S* sbuf = s_rec[threadIdx.x >> 5];
  S* mine_rec = sbuf + i * STRIDE + var * NB;
  warp_load_records<NB, S>(Uin, e0, sbuf, lane);
  S us[NB];
  T u[NB], r[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    us[b] = mine_rec[b];
    u[b] = T(us[b]);
    r[b] = T(0);
  }
  const T J = T(m.jac[e]);
  const T xx = T(m.dinv[0 * ld + e]), xy = T(m.dinv[1 * ld + e]), ex = T(m.dinv[2 * ld + e]),
          ey = T(m.dinv[3 * ld + e]);
  const T gm1 = T(kp.gas.gm1);
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    T mine = T(0);
#pragma unroll
    for (int b = 0; b < NB; ++b) mine += u[b] * kp.t.phi_cell[q][b];
    T uq[NEQ];
#pragma unroll
    for (int w = 0; w < NEQ; ++w) uq[w] = __shfl_sync(0xffffffffu, mine, w * 8 + i);
    T f[NEQ], g[NEQ];
    euler_flux<T>(uq, gm1, f, g);
    const T fv = var == 0 ? f[0] : var == 1 ? f[1] : var == 2 ? f[2] : f[3];
    const T gv = var == 0 ? g[0] : var == 1 ? g[1] : var == 2 ? g[2] : g[3];
    const T sc = kp.t.cell_w[q] * T(0.5) * J;
    const T fx = sc * (fv * xx + gv * xy);
    const T fe = sc * (fv * ex + gv * ey);
#pragma unroll
    for (int b = 0; b < NB; ++b) r[b] += fx * kp.t.dxi[q][b] + fe * kp.t.deta[q][b];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int fw = m.face[k * ld + e];
    const int slot = fw >> 1;
    const bool right = fw & 1;
    const T* Fs = &F[(size_t)slot * NG * 4 + var];
#pragma unroll
    for (int gp = 0; gp < NG; ++gp) {
      const int src = right ? (NG - 1 - gp) : gp;
      const T coef = right ? kp.t.edge_w[gp] : -kp.t.edge_w[gp];
      const T fv = coef * __ldcg(&Fs[src * 4]);
#pragma unroll
      for (int b = 0; b < NB; ++b) r[b] += fv * kp.t.phi_edge[k][gp][b];
    }
  }
  const S dt = S(kp.ic[inst].dt);
  const T inv_half_j = T(1) / (T(0.5) * J);
  if constexpr (MODE == 0) {  // compute_residuals adds to the residual it is given
    warp_load_records<NB, S>(Rin, e0, sbuf, lane);
#pragma unroll
    for (int b = 0; b < NB; ++b) r[b] = T(mine_rec[b]) + r[b];
  }
#pragma unroll
  for (int b = 0; b < NB; ++b) r[b] = r[b] * kp.t.inv_mass[b] * inv_half_j;  // divide_residual_by_mass_mat_diag
  if (Rout) {
#pragma unroll
    for (int b = 0; b < NB; ++b) mine_rec[b] = S(r[b]);
    warp_store_records<NB, S>(Rout, e0, sbuf, keep, lane);
  }
  if constexpr (MODE != 0) {
    S base[NB];
    if constexpr (MODE >= 2) {
      warp_load_records<NB, S>(Ubase, e0, sbuf, lane);
#pragma unroll
      for (int b = 0; b < NB; ++b) base[b] = mine_rec[b];
      __syncwarp();
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const S rr = S(r[b]);
      S out;
      if constexpr (MODE == 1) {
        out = us[b] + dt * rr;
      } else if constexpr (MODE == 2) {
        out = S(0.75) * base[b] + S(0.25) * (us[b] + dt * rr);
      } else {
        out = S(1.0 / 3.0) * base[b] + S(2.0 / 3.0) * (us[b] + dt * rr);
      }
      mine_rec[b] = out;
    }
    warp_store_records<NB, S>(Uout, e0, sbuf, keep, lane);
  }
}

template <int P, typename T, int MODE, typename S = T>
__global__ void __launch_bounds__(256, 3) k_element(const __grid_constant__ KParams<P, T> kp,
                                                    const S* __restrict__ Uin, const S* Ubase,
                                                    const T* __restrict__ F, S* Uout, const S* Rin, S* Rout) {
  element_body<P, T, MODE, S>(kp, Uin, Ubase, F, Uout, Rin, Rout, blockIdx.x);
}

// ------------------------------------------------------------------------------------------
// modified_kxrcf, weno.rs:7-85, for element e on state U (FP64 arithmetic).  Keeps the
// reference's exterior-trace indexing: the neighbour's modes are evaluated with this element's
// own local edge index k (weno.rs:21-27 pick in_cell_indices[side], always this element's).
// `own` is e's record (the limiter stages its warp's records in shared memory); the
// neighbours' modes are read from U through L2.
// ------------------------------------------------------------------------------------------
// RO: U is only read during the kernel (neighbour traces through L1); OWN_SHARED: `own` is staged
// in shared memory (plain loads), else it is e's record in U (loaded like the neighbours').
template <int P, typename T, bool RO = false, bool OWN_SHARED = false, typename S = T>
__device__ __forceinline__ bool kxrcf(const KParams<P, T>& kp, const S* __restrict__ U, int e, const S* own) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  const MeshDev& m = kp.m;
  const size_t ld = m.ld;
  double density_jump = 0.0, total_energy_jump = 0.0, surface = 0.0;
  double min_density = 1.0e10, min_total_energy = 1.0e10;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int fw = m.face[k * ld + e];
    const int slot = fw >> 1;
    if (slot >= m.n_int) continue;
    const int nb = m.nbr[k * ld + e];
    const double4 geo = m.ie_geo[slot];
    const double nx = (fw & 1) ? -geo.x : geo.x;
    const double ny = (fw & 1) ? -geo.y : geo.y;
    double own_rho[NG], own_rhoe[NG];
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      double rho = 0.0, rho_e = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        rho += (double)ld_own<RO, OWN_SHARED>(&own[0 * NB + b]) * kp.d.phi_edge[k][g][b];
        rho_e += (double)ld_own<RO, OWN_SHARED>(&own[3 * NB + b]) * kp.d.phi_edge[k][g][b];
      }
      own_rho[g] = rho;
      own_rhoe[g] = rho_e;
      if (rho < min_density) min_density = rho;
      if (rho_e < min_total_energy) min_total_energy = rho_e;
    }
    constexpr int cg = NG / 2;
    double rho_u = 0.0, rho_v = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      rho_u += (double)ld_own<RO, OWN_SHARED>(&own[1 * NB + b]) * kp.d.phi_edge[k][cg][b];
      rho_v += (double)ld_own<RO, OWN_SHARED>(&own[2 * NB + b]) * kp.d.phi_edge[k][cg][b];
    }
    if (rho_u * nx + rho_v * ny < 0.0) {
      double rho_jump = 0.0, rho_e_jump = 0.0;
      const double jd = geo.w;
      double nrho[NB], nrhoe[NB];
      load_var_modes<NB, S, 0, RO>(U, nb, nrho);
      load_var_modes<NB, S, 3, RO>(U, nb, nrhoe);
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        double er = 0.0, ere = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          er += nrho[b] * kp.d.phi_edge[k][NG - 1 - g][b];
          ere += nrhoe[b] * kp.d.phi_edge[k][NG - 1 - g][b];
        }
        rho_jump += 0.5 * jd * kp.d.edge_w[g] * (own_rho[g] - er);
        rho_e_jump += 0.5 * jd * kp.d.edge_w[g] * (own_rhoe[g] - ere);
      }
      density_jump += rho_jump;
      total_energy_jump += rho_e_jump;
      surface += jd;
    }
  }
  const double h15 = m.h15[e];
  const double ind_d = fabs(density_jump) / (h15 * surface * min_density);
  const double ind_e = fabs(total_energy_jump) / (h15 * surface * min_total_energy);
  return (ind_d >= 1.0) || (ind_e >= 1.0);
}

// The same detector with its loads in three rounds, each issued in full before it is used: the
// element's faces and neighbours, then its own state, the face normals and h^1.5, then the
// neighbours' density and energy modes of the inflow faces.  Fewer dependent memory round trips
// than kxrcf (which walks the faces one after another) at the price of registers: faster when
// a pass is latency-bound (small meshes), slower when occupancy matters (large batches); the
// autotuner picks one per context.  Same arithmetic in the same order, so the same flags.
template <int P, typename T, bool RO = false, bool OWN_SHARED = false, typename S = T>
__device__ __forceinline__ bool kxrcf_staged(const KParams<P, T>& kp, const S* __restrict__ U, int e,
                                             const S* own_rec) {
  int fw[3], nb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    fw[k] = kp.m.face[k * kp.m.ld + e];
    nb[k] = kp.m.nbr[k * kp.m.ld + e];
  }
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  const MeshDev& m = kp.m;
  double own[NEQ][NB];
#pragma unroll
  for (int v = 0; v < NEQ; ++v)
#pragma unroll
    for (int b = 0; b < NB; ++b) own[v][b] = (double)ld_own<RO, OWN_SHARED>(&own_rec[v * NB + b]);
  double nx[3], ny[3], jd[3];
  bool interior[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int slot = fw[k] >> 1;
    interior[k] = slot < m.n_int;
    const double4 geo = interior[k] ? m.ie_geo[slot] : make_double4(0.0, 0.0, 0.0, 0.0);
    nx[k] = (fw[k] & 1) ? -geo.x : geo.x;
    ny[k] = (fw[k] & 1) ? -geo.y : geo.y;
    jd[k] = geo.w;
  }
  const double h15 = m.h15[e];
  // inflow test at the centre Gauss point (weno.rs:42-52)
  constexpr int cg = NG / 2;
  bool inflow[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double rho_u = 0.0, rho_v = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      rho_u += own[1][b] * kp.d.phi_edge[k][cg][b];
      rho_v += own[2][b] * kp.d.phi_edge[k][cg][b];
    }
    inflow[k] = interior[k] && (rho_u * nx[k] + rho_v * ny[k] < 0.0);
  }
  double ext_rho[3][NB], ext_rhoe[3][NB];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      ext_rho[k][b] = inflow[k] ? (double)ld_st<RO>(&U[sx<NB>(nb[k], 0, b)]) : 0.0;
      ext_rhoe[k][b] = inflow[k] ? (double)ld_st<RO>(&U[sx<NB>(nb[k], 3, b)]) : 0.0;
    }
  double density_jump = 0.0, total_energy_jump = 0.0, surface = 0.0;
  double min_density = 1.0e10, min_total_energy = 1.0e10;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (!interior[k]) continue;
    double own_rho[NG], own_rhoe[NG];
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      double rho = 0.0, rho_e = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        rho += own[0][b] * kp.d.phi_edge[k][g][b];
        rho_e += own[3][b] * kp.d.phi_edge[k][g][b];
      }
      own_rho[g] = rho;
      own_rhoe[g] = rho_e;
      if (rho < min_density) min_density = rho;
      if (rho_e < min_total_energy) min_total_energy = rho_e;
    }
    if (inflow[k]) {
      double rho_jump = 0.0, rho_e_jump = 0.0;
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        double er = 0.0, ere = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          er += ext_rho[k][b] * kp.d.phi_edge[k][NG - 1 - g][b];
          ere += ext_rhoe[k][b] * kp.d.phi_edge[k][NG - 1 - g][b];
        }
        rho_jump += 0.5 * jd[k] * kp.d.edge_w[g] * (own_rho[g] - er);
        rho_e_jump += 0.5 * jd[k] * kp.d.edge_w[g] * (own_rhoe[g] - ere);
      }
      density_jump += rho_jump;
      total_energy_jump += rho_e_jump;
      surface += jd[k];
    }
  }
  const double ind_d = fabs(density_jump) / (h15 * surface * min_density);
  const double ind_e = fabs(total_energy_jump) / (h15 * surface * min_total_energy);
  return (ind_d >= 1.0) || (ind_e >= 1.0);
}

// ------------------------------------------------------------------------------------------
// weno, weno.rs:86-269: characteristic WENO reconstruction of element e by one warp (FP64).
//
// The smoothness indicator of a projected polynomial P (weno.rs:125-143, 156-174),
//   beta = sum_{l=1..p} sum_{l1+l2=l} J^(l-1) int_e (sum_b P_b d^{l1,l2} phi_b)^2,
// is the quadratic form P^T Q P with the element's Gram matrix
//   Q[b][b'] = sum_keys J^(l-1) sum_q 0.5 J w_q D_{q,b,key} D_{q,b',key},
// which depends on the geometry only: k_weno_gram computes it once per context, and it serves
// the 3 faces x 4 polynomials x 4 variables of every limiting pass (the reference re-evaluates
// the derivative sums for each of those 48 indicators).  The three
// faces are processed concurrently (lane -> (face, poly, variable, mode)); projections,
// normalisation, recombination and the area average keep the reference's summation order.
// ------------------------------------------------------------------------------------------
// Entry (b, c) of an element's WENO Gram matrix,
//   Q[b][c] = sum_{l=1..p} J^(l-1) sum_{l1+l2=l} sum_q 0.5 J w_q D_{q,b,(l1,l2)} D_{q,c,(l1,l2)},
// with D the physical derivatives of the modes at the cell points (compute_dphi, mesh.rs:66-147):
// P^T Q P is the smoothness indicator of weno.rs:125-143, 156-174.
template <int P>
__device__ __forceinline__ double gram_entry(const double* __restrict__ dref, const double* __restrict__ cell_w,
                                             double J, double xx, double xy, double ex, double ey, int b, int c) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NQ = V::NQ, NK = V::NK;
  double acc = 0.0;
#pragma unroll
  for (int l = 1; l <= P; ++l) {
    const double jp = (l == 1) ? 1.0 : (l == 2 ? J : J * J);
#pragma unroll
    for (int l1 = 0; l1 <= l; ++l1) {
      const int kk = l * (l + 1) / 2 - 1 + (l - l1);
      double integral = 0.0;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const double(&rb)[NK] = *reinterpret_cast<const double(*)[NK]>(&dref[(q * NB + b) * NK]);
        const double(&rc)[NK] = *reinterpret_cast<const double(*)[NK]>(&dref[(q * NB + c) * NK]);
        const double db = phys_deriv<NK>(rb, xx, xy, ex, ey, kk);
        const double dc = phys_deriv<NK>(rc, xx, xy, ex, ey, kk);
        integral += 0.5 * J * cell_w[q] * (db * dc);
      }
      acc += jp * integral;
    }
  }
  return acc;
}

// Setup kernel: the Gram matrices of elements [e0, e0 + count) (upper triangle, pair-major), one
// thread per (pair, element); a warp shares its pair, so the table reads are uniform.
template <int P, typename T>
__global__ void k_weno_gram(const __grid_constant__ KParams<P, T> kp, double* __restrict__ gram, int e0, int count) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NPAIR = NB * (NB + 1) / 2;
  const MeshDev& m = kp.m;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)NPAIR * count) return;
  const int pr = (int)(i / count), e = e0 + (int)(i - (long long)pr * count);
  int b = 0, c = pr;
  while (c >= NB - b) {
    c -= NB - b;
    ++b;
  }
  c += b;
  const size_t ld = m.ld;
  gram[(size_t)pr * ld + e] = gram_entry<P>(&kp.d.dref[0][0][0], kp.d.cell_w, m.jac[e], m.dinv[0 * ld + e],
                                            m.dinv[1 * ld + e], m.dinv[2 * ld + e], m.dinv[3 * ld + e], b, c);
}

template <int P>
struct WenoScratch {
  using V = Variant<P>;
  double Q[V::NB][V::NB];
  double pol[4][NEQ][V::NB];           // pol[0] = target, pol[j+1] = neighbour j, mode 0 <- target's
  double L[3][4][4], R[3][4][4];
  double proj[3][4][NEQ][V::NB];
  double nlw[3][4][NEQ];
  double pol_new[3][NEQ][V::NB];
};

template <int P, typename T, typename Sto = T>
__device__ __forceinline__ int weno_reconstruct(const KParams<P, T>& kp, Sto* __restrict__ U, int e,
                                                const int (&faces)[3], const int (&nbrs)[3], int lane,
                                                WenoScratch<P>& S) {
  using V = Variant<P>;
  constexpr int NB = V::NB;
  const MeshDev& m = kp.m;
  const size_t ld = m.ld;
  bool interior[3];
  int nbd = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    interior[k] = (faces[k] >> 1) < m.n_int;
    if (!interior[k]) ++nbd;
  }
  if (nbd > 2) return ST_TOO_MANY_BOUNDARY_EDGES;
  // linear weights with the reference's indexing (weno.rs:93-110)
  double lw[4] = {0.997, 0.001, 0.001, 0.001};
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (!interior[k]) lw[k] = 0.0;
  if (nbd == 0) lw[0] = 0.997;
  else if (nbd == 1) lw[1] = 0.998;
  else lw[2] = 0.999;
  // one round of global loads: the state of e and of its interior neighbours, e's Gram matrix
  // (geometry only: precomputed by k_weno_gram), the face normals (lanes 0-2) and the
  // neighbours' Jacobians
  constexpr int NLD = (NEQ * NB + 31) / 32, NPAIR = NB * (NB + 1) / 2, NQL = (NPAIR + 31) / 32;
  double own[NLD], nbv[NLD][3], qv[NQL];
#pragma unroll
  for (int it = 0; it < NLD; ++it) {
    const int i = lane + 32 * it;
    const bool ok = i < NEQ * NB;
    const int b = i % NB;
    own[it] = ok ? (double)ld_state(&U[(size_t)e * (NEQ * NB) + i]) : 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      nbv[it][k] = (ok && interior[k] && b > 0) ? (double)ld_state(&U[(size_t)nbrs[k] * (NEQ * NB) + i]) : 0.0;
  }
#pragma unroll
  for (int it = 0; it < NQL; ++it) {
    const int pr = lane + 32 * it;
    qv[it] = pr < NPAIR ? m.gram[(size_t)pr * ld + e] : 0.0;
  }
  const int my_face = lane == 0 ? faces[0] : (lane == 1 ? faces[1] : faces[2]);
  const bool my_interior = lane < 3 && (lane == 0 ? interior[0] : (lane == 1 ? interior[1] : interior[2]));
  const double4 geo = my_interior ? m.ie_geo[my_face >> 1] : make_double4(0.0, 0.0, 0.0, 0.0);
  double Jn[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) Jn[k] = interior[k] ? m.jac[nbrs[k]] : 0.0;
#pragma unroll
  for (int it = 0; it < NLD; ++it) {
    const int i = lane + 32 * it;
    if (i < NEQ * NB) {
      const int v = i / NB, b = i - v * NB;
      S.pol[0][v][b] = own[it];
#pragma unroll
      for (int k = 0; k < 3; ++k) S.pol[k + 1][v][b] = nbv[it][k];
    }
  }
#pragma unroll
  for (int it = 0; it < NQL; ++it) {
    const int pr = lane + 32 * it;
    if (pr < NPAIR) {
      int b = 0, c = pr;
      while (c >= NB - b) {
        c -= NB - b;
        ++b;
      }
      c += b;
      S.Q[b][c] = qv[it];
      S.Q[c][b] = qv[it];
    }
  }
  __syncwarp();
  if (lane < NEQ) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (interior[k]) S.pol[k + 1][lane][0] = S.pol[0][lane][0];
  }
  if (my_interior) {  // unoriented normal (weno.rs:121-122)
    double mean[4];
#pragma unroll
    for (int v = 0; v < NEQ; ++v) mean[v] = S.pol[0][v][0];
    eigenmatrix<double>(mean, geo.x, geo.y, kp.gas, S.L[lane], S.R[lane]);
  }
  __syncwarp();
  // projections onto the characteristic fields of each face (weno.rs:123-124, 155)
#pragma unroll
  for (int it = 0; it < (3 * 4 * NEQ * NB + 31) / 32; ++it) {
    const int idx = lane + 32 * it;
    if (idx >= 3 * 4 * NEQ * NB) break;
    const int f = idx / (4 * NEQ * NB), r1 = idx - f * 4 * NEQ * NB;
    const int j = r1 / (NEQ * NB), r2 = r1 - j * NEQ * NB, r = r2 / NB, b = r2 - r * NB;
    double sum = 0.0;
    if (interior[f] && (j == 0 || interior[j - 1])) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sum += S.L[f][r][k] * S.pol[j][k][b];
    }
    S.proj[f][j][r][b] = sum;
  }
  __syncwarp();
  // nonlinear weights (weno.rs:142, 173)
#pragma unroll
  for (int it = 0; it < (3 * 4 * NEQ + 31) / 32; ++it) {
    const int idx = lane + 32 * it;
    if (idx >= 3 * 4 * NEQ) break;
    const int f = idx >> 4, j = (idx >> 2) & 3, v = idx & 3;
    double w = 0.0;
    if (interior[f] && (j == 0 || interior[j - 1])) {
      double pv[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) pv[b] = S.proj[f][j][v][b];
      double beta = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        double t = 0.0;
#pragma unroll
        for (int c = 0; c < NB; ++c) t += S.Q[b][c] * pv[c];
        beta += pv[b] * t;
      }
      w = lw[j] / ((beta + F64_EPS) * (beta + F64_EPS));
    }
    S.nlw[f][j][v] = w;
  }
  __syncwarp();
  // normalise and combine (weno.rs:180-194)
#pragma unroll
  for (int it = 0; it < (3 * NEQ * NB + 31) / 32; ++it) {
    const int idx = lane + 32 * it;
    if (idx >= 3 * NEQ * NB) break;
    const int f = idx / (NEQ * NB), r1 = idx - f * NEQ * NB, v = r1 / NB, b = r1 - v * NB;
    double acc = 0.0;
    if (interior[f]) {
      const double inv_den = 1.0 / (((S.nlw[f][0][v] + S.nlw[f][1][v]) + S.nlw[f][2][v]) + S.nlw[f][3][v]);
#pragma unroll
      for (int j = 0; j < 4; ++j) acc += (S.nlw[f][j][v] * inv_den) * S.proj[f][j][v][b];
    }
    S.pol_new[f][v][b] = acc;
  }
  __syncwarp();
  // back to conserved variables, area-weighted average over the faces in order (weno.rs:195-263)
  double neighbour_area = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (interior[k]) neighbour_area += Jn[k] * 0.5;
  const double inv_area = 1.0 / neighbour_area;
  for (int idx = lane; idx < NEQ * NB; idx += 32) {
    const int r = idx / NB, b = idx - r * NB;
    double recon = 0.0;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (!interior[f]) continue;
      double sum = 0.0;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sum += S.R[f][r][k] * S.pol_new[f][k][b];
      recon = recon + sum * Jn[f] * 0.5;
    }
    U[sx<NB>(e, r, b)] = Sto(recon * inv_area);
  }
  __syncwarp();
  return ST_OK;
}

// Release add and acquire load at GPU scope (the PTX memory model's synchronisation pair).
__device__ __forceinline__ unsigned int atom_add_release_gpu(unsigned int* p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Bounded grid barrier for the co-resident (cooperative) limiter kernels: a sense-reversing
// arrival word.  Thread 0 of every block adds 1, block 0 adds 2^31 - (nblocks - 1), so that a
// barrier adds exactly 2^31 in all -- the top bit flips with the last arrival, whatever the order,
// and the low bits return to their value (nothing to reset, no second word to publish).  A block
// waits until the top bit differs from the one its own arrival saw.  The arrival is a release
// (the block's writes, ordered by __syncthreads, before it) and the polling an acquire (every
// arrival's writes before the block's next reads): no separate fences.
__device__ __forceinline__ bool grid_barrier(Control* ctl, unsigned int nblocks) {
  __syncthreads();
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_fail = 0;
    const unsigned int inc = blockIdx.x == 0 ? 0x80000000u - (nblocks - 1u) : 1u;
    const unsigned int seen = atom_add_release_gpu(&ctl->bar_word, inc);
    long long it = 0;
    while (((seen ^ ld_acquire_gpu(&ctl->bar_word)) & 0x80000000u) == 0u) {
      if (++it > (1ll << 25)) {  // ~ seconds: co-residency is guaranteed, so this is a fault
        if (atomicCAS(&ctl->status, 0, ST_TIMEOUT) == 0) ctl->err_where = -1;
        s_fail = 1;
        break;
      }
    }
  }
  __syncthreads();
  return s_fail == 0;
}

constexpr int kLimiterWarps = 4;

// Release/acquire fence at GPU scope: orders this thread's earlier accesses before its later ones
// as seen by other blocks (what the limiter's queue hand-offs need; lighter than a sequentially
// consistent __threadfence).
__device__ __forceinline__ void fence_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Queue schedule.  Lane 0 of a reconstructing warp: returns the next cell enlisted in a wave's
// queue, or -1 once
// every warp has finished the wave's scan and every enlisted cell has been taken.  The warp first
// waits, reading only, until the queue shows an untaken slot (so idle warps take no ticket and do
// not queue up on the ticket counter), then takes a ticket.  A ticket inside the queue whose slot
// is not yet written waits for its producer, which has reserved it; a ticket that overshot the
// queue waits until the queue grows past it or closes.  Slots hold cell + 1 and are cleared by
// their consumer, so the whole queue is zero again when a pass ends.  Every wait is bounded.
__device__ __forceinline__ int limiter_ticket(Control* ctl, LimQueue* q, int* __restrict__ work, int cap,
                                              int nwarps) {
  volatile int* tail = &q->tail;
  volatile int* head = &q->head;
  volatile int* scanned = &q->scanned;
  constexpr long long kSpin = 1ll << 23;
  unsigned int ns = 64;
  long long it = 0;
  for (;; ++it) {
    if (*head < *tail) break;
    if (*scanned >= nwarps) {
      fence_gpu();
      if (*head >= *tail) return -1;
      break;
    }
    if (it > kSpin) goto timeout;
    __nanosleep(ns);
    ns = ns < 1024u ? 2u * ns : 1024u;
  }
  {
    const int i = atomicAdd(&q->head, 1);
    ns = 32;
    for (; it <= 2 * kSpin; ++it) {
      if (i < cap) {
        volatile int* slot = work + i;
        const int v = *slot;
        if (v != 0) {
          *slot = 0;
          return v - 1;
        }
      }
      if (*scanned >= nwarps) {
        fence_gpu();
        if (i >= *tail) return -1;
        ns = 32;  // reserved by a producer: its store is on the way
      }
      __nanosleep(ns);
      ns = ns < 1024u ? 2u * ns : 1024u;
    }
  }
timeout:
  if (atomicCAS(&ctl->status, 0, ST_TIMEOUT) == 0) ctl->err_where = -1;
  return -1;
}

// The limiter (apply_limiter -> weno, limiter.rs:7, weno.rs:86-269), exact in the reference's
// sequential, in-place element order, run in parallel waves:
//   * an element settles in wave w once every lower-index neighbour settled in an earlier
//     wave; it is limited iff modified_kxrcf flags it on the values the sequential loop would
//     see at that point: the parallel flag of wave 1 when no lower neighbour was rewritten,
//     else recomputed;
//   * a limited element is reconstructed from final lower neighbours and untouched higher
//     neighbours -- again what the sequential loop reads;
//   * elements that settle in the same wave never read one another, so in-place writes are
//     race free.
// Status word per element: (wave << 2) | kind, kind 1 clean, 2 limited, 0 not settled yet.  Wave
// count = longest chain of increasing-index neighbours through unsettled elements: 2 on the
// O-grid's 2-colour numbering.  Instances never share neighbours, so one pass limits all of them;
// elements of instances that are not stepping settle clean without evaluation.
//
// Two launches per pass.  k_lim_detect evaluates modified_kxrcf on every element (the parallel
// flags t0 of wave 1), one warp per batch of 32 consecutive elements (their records staged in
// shared memory), one lane per element, at full occupancy, visiting the batches in a
// breadth-first order of the batch graph so that the neighbour traces it gathers are mostly in
// cache; it settles the clean elements without a lower-index neighbour, enlists the troubled ones
// for wave 1 (wl1) and lists the elements that wait for a lower neighbour (pend).  k_limiter, a
// cooperative persistent kernel, then reconstructs wave 1's cells (one warp each), and runs waves
// 2, 3, ... over the pending list: each wave scans it, settles clean ready elements, enlists
// troubled ready ones and reconstructs them, with a grid barrier between waves.  Within a wave,
// two schedules join the scan and the reconstruction, with bitwise identical results:
//   * QUEUE = false: a grid barrier separates the scan from the reconstruction, warps take the
//     worklist's entries in a fixed stride (the entries stay behind after the pass);
//   * QUEUE = true: a warp that has finished its scan takes tickets from the queue and
//     reconstructs while other warps still scan.  That overlap is safe: a reconstruction in wave
//     w rewrites an element all of whose lower neighbours settled before wave w, so the only
//     concurrent reads of it are wave-1 flags of its higher neighbours, and those flags are never
//     used (a higher neighbour of a rewritten element is re-evaluated in a later wave).
constexpr int kDetectWarps = 4;
constexpr int kDetectThreads = kDetectWarps * 32;

// Shared memory of one detection block: each warp's 32 staged records.
template <int P, typename T>
struct DetectSmem {
  static constexpr int kStride = Staged<Variant<P>::NB, T>::kStride;
  static constexpr size_t kBytes = (size_t)kDetectWarps * 32 * kStride * sizeof(T);
};

template <int P, typename T, bool STAGED, typename S = T>
__device__ __forceinline__ void lim_detect_body(const KParams<P, T>& kp, const S* __restrict__ U,
                                                unsigned char* __restrict__ t0, unsigned int* __restrict__ status,
                                                int* __restrict__ wl1, int* __restrict__ pend,
                                                const int* __restrict__ order, int bid, S* s_det) {
  using V = Variant<P>;
  constexpr int STRIDE = DetectSmem<P, S>::kStride;
  Control* ctl = kp.ctl;
  const MeshDev& m = kp.m;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int w = bid * kDetectWarps + wib;  // position in the batch order
  if (w >= m.ld / 32) return;              // the whole warp
  const int e0 = order[w] * 32;            // the warp's batch: 32 consecutive elements
  const int e = e0 + lane;
  bool flag = false, enlist = false, wait = false, active = false;
  if (e < m.ne) {
    const int inst = m.n_inst > 1 ? m.inst[e] : 0;
    active = kp.ic[inst].active != 0;
  }
  if (__any_sync(0xffffffffu, active)) {
    // the batch's records are contiguous: staged with coalesced 16-byte loads (arrays are padded
    // to whole batches)
    S* recs = s_det + (size_t)wib * 32 * STRIDE;
    warp_load_records<V::NB, S, 32>(U, e0, recs, lane);
    if (active) {
      const S* own = recs + lane * STRIDE;
      flag = STAGED ? kxrcf_staged<P, T, true, true, S>(kp, U, e, own) : kxrcf<P, T, true, true, S>(kp, U, e, own);
      bool ready = true;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int nb = m.nbr[k * m.ld + e];
        if (nb >= 0 && nb < e) ready = false;
      }
      wait = !ready;
      enlist = ready && flag;
    }
  }
  if (e < m.ne) {
    t0[e] = flag ? 1 : 0;
    status[e] = (wait || enlist) ? 0u : ((1u << 2) | 1u);  // not stepping or clean and ready: settled
  }
  const unsigned int below = (1u << lane) - 1u;
  const unsigned int fm = __ballot_sync(0xffffffffu, flag);
  if (fm && lane == 0) atomicAdd(&ctl->t0_count, __popc(fm));
  const unsigned int em = __ballot_sync(0xffffffffu, enlist);
  if (em) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&ctl->wl1_count, __popc(em));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (enlist) {
      int f[3], n[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        f[k] = m.face[k * m.ld + e];
        n[k] = m.nbr[k * m.ld + e];
      }
      entry_put(ctl, wl1, base + __popc(em & below), m.ne, e, f, n);
    }
  }
  const unsigned int wm = __ballot_sync(0xffffffffu, wait);
  if (wm) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&ctl->pend_count, __popc(wm));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (wait) list_put(ctl, pend, base + __popc(wm & below), m.ne, e);
  }
}

// The compact detector at 6 blocks per SM (80 registers); the staged one keeps its registers.
template <int P, typename T, bool STAGED, typename S = T>
__global__ void __launch_bounds__(kDetectThreads, STAGED ? 1 : 6) k_lim_detect(const __grid_constant__ KParams<P, T> kp,
                                                               const S* __restrict__ U,
                                                               unsigned char* __restrict__ t0,
                                                               unsigned int* __restrict__ status,
                                                               int* __restrict__ wl1, int* __restrict__ pend,
                                                               const int* __restrict__ order) {
  __shared__ __align__(16) unsigned char s_det[DetectSmem<P, S>::kBytes];
  lim_detect_body<P, T, STAGED, S>(kp, U, t0, status, wl1, pend, order, blockIdx.x, reinterpret_cast<S*>(s_det));
}

template <int P, typename T, bool QUEUE, typename S = T>
__global__ void __launch_bounds__(kLimiterWarps * 32) k_limiter(const __grid_constant__ KParams<P, T> kp,
                                                                S* __restrict__ U,
                                                                const unsigned char* __restrict__ t0,
                                                                unsigned int* __restrict__ status,
                                                                int* __restrict__ work,
                                                                const int* __restrict__ wl1,
                                                                const int* __restrict__ pend) {
  Control* ctl = kp.ctl;
  const MeshDev& m = kp.m;
  constexpr size_t kWarpBytes = (sizeof(WenoScratch<P>) + 127) / 128 * 128;
  __shared__ __align__(128) unsigned char s_warp[kLimiterWarps][kWarpBytes];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  WenoScratch<P>* scratch_w = reinterpret_cast<WenoScratch<P>*>(s_warp[wib]);
  const int gwarp = blockIdx.x * kLimiterWarps + wib;
  const int nwarps = gridDim.x * kLimiterWarps;
  // the detection launch has finished: its counts are final
  const int flagged = ctl->t0_count;
  const int n_wl1 = min(ctl->wl1_count, m.ne);  // larger only after an overflow (reported)
  const int n_pend = min(ctl->pend_count, m.ne);
  int troubled_local = 0;
  int wave = 1;
  // reconstruction of one enlisted element by the whole warp
  auto reconstruct_with = [&](int et, const int (&fwt)[3], const int (&nbt)[3]) {
    const int rs = weno_reconstruct<P, T, S>(kp, U, et, fwt, nbt, lane, *scratch_w);
    if (rs != ST_OK && lane == 0) {
      const int inst = m.n_inst > 1 ? m.inst[et] : 0;
      raise_status(ctl, &kp.ic[inst], rs, et);
    }
  };
  auto reconstruct = [&](int et) {
    int fwt[3], nbt[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      fwt[k] = m.face[k * m.ld + et];
      nbt[k] = m.nbr[k * m.ld + et];
    }
    reconstruct_with(et, fwt, nbt);
  };
  if (flagged > 0) {  // else no element is limited: every block leaves at once
    // ---- wave 1: the cells enlisted by the detection (the list is complete) ----
    for (int i = gwarp; i < n_wl1; i += nwarps) {
      int fwt[3], nbt[3];
      const int et = entry_get(wl1, i, lane, fwt, nbt);
      reconstruct_with(et, fwt, nbt);
      if (lane == 0) status[et] = (1u << 2) | 2u;
      ++troubled_local;
    }
    // ---- waves 2, 3, ...: the elements that waited for a lower neighbour ----
    bool more = n_pend > 0;
    if (more && !grid_barrier(ctl, gridDim.x)) more = false;
    for (wave = 2; more; ++wave) {
      LimQueue* q = &ctl->lq[wave % 3];
      // the queue of wave w + 1 was last used by wave w - 2, whose readers all passed a barrier since
      if (QUEUE && blockIdx.x == 0 && threadIdx.x == 0) reset_queue(ctl->lq[(wave + 1) % 3]);
      int unknown_local = 0;
      for (int base = gwarp * 32; base < n_pend; base += nwarps * 32) {
        const int i = base + lane;
        const int e = i < n_pend ? __ldcg(&pend[i]) : 0;
        bool pending = false, ready = false, trouble = false, any_mod = false;
        if (i < n_pend) {
          pending = (__ldcg(&status[e]) & 3u) == 0u;
          if (pending) {
            ready = true;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              const int nb = m.nbr[k * m.ld + e];
              if (nb >= 0 && nb < e) {
                const unsigned int sn = __ldcg(&status[nb]);
                if ((sn & 3u) == 0u || (int)(sn >> 2) >= wave) ready = false;
                else if ((sn & 3u) == 2u) any_mod = true;
              }
            }
          }
        }
        // modified_kxrcf again only next to rewritten cells, each element reading its own record
        // (it is still pending, so nothing has rewritten it in this pass)
        if (pending && ready) {
          if (any_mod) {
            const S* own = U + (size_t)e * (NEQ * Variant<P>::NB);
            trouble = kxrcf<P, T, false, false, S>(kp, U, e, own);
          } else {
            trouble = t0[e] != 0;
          }
          if (!trouble) status[e] = ((unsigned int)wave << 2) | 1u;
        }
        const unsigned int tb = __ballot_sync(0xffffffffu, ready && trouble);
        if (tb) {
          int slot0 = 0;
          if (lane == 0) slot0 = atomicAdd(QUEUE ? &q->tail : &ctl->wl_count[wave & 1], __popc(tb));
          slot0 = __shfl_sync(0xffffffffu, slot0, 0);
          if (ready && trouble) list_put(ctl, work, slot0 + __popc(tb & ((1u << lane) - 1u)), m.ne, QUEUE ? e + 1 : e);
        }
        unknown_local += (pending && !ready) ? 1 : 0;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) unknown_local += __shfl_xor_sync(0xffffffffu, unknown_local, o);
      int remaining = 0;
      if (!QUEUE) {
        if (lane == 0 && unknown_local) atomicAdd(&ctl->unknown[wave & 1], unknown_local);
        if (!grid_barrier(ctl, gridDim.x)) break;
        const int n_work = min(*((volatile int*)&ctl->wl_count[wave & 1]), m.ne);
        remaining = *((volatile int*)&ctl->unknown[wave & 1]);
        // the other parity's counters were last read before the previous wave's second barrier
        if (blockIdx.x == 0 && threadIdx.x == 0) {
          ctl->wl_count[(wave + 1) & 1] = 0;
          ctl->unknown[(wave + 1) & 1] = 0;
        }
        // ---- reconstruct the enlisted elements, one warp each, in a fixed stride ----
        for (int i = gwarp; i < n_work; i += nwarps) {
          const int et = __ldcg(&work[i]);
          reconstruct(et);
          __threadfence();
          if (lane == 0) status[et] = ((unsigned int)wave << 2) | 2u;
          ++troubled_local;
        }
      } else {
        __syncwarp();
        if (lane == 0) {
          if (unknown_local) atomicAdd(&q->unknown, unknown_local);
          fence_gpu();  // the count before the report that this warp's scan is done
          atomicAdd(&q->scanned, 1);
        }
        // ---- reconstruct enlisted elements from the queue while other warps still scan ----
        for (;;) {
          int et = -1;
          if (lane == 0) et = limiter_ticket(ctl, q, work, m.ne, nwarps);
          et = __shfl_sync(0xffffffffu, et, 0);
          if (et < 0) break;
          reconstruct(et);
          // no fence: nothing reads this element or its status before the wave's barrier
          if (lane == 0) status[et] = ((unsigned int)wave << 2) | 2u;
          ++troubled_local;
        }
        // every warp's scan has been reported (the ticket loop ends only then): the count is final
        if (lane == 0) {
          fence_gpu();
          remaining = *((volatile int*)&q->unknown);
        }
        remaining = __shfl_sync(0xffffffffu, remaining, 0);
      }
      if (remaining == 0) break;  // no further wave: nothing reads what this one wrote
      if (!grid_barrier(ctl, gridDim.x)) break;
      if (wave > m.ne + 2) break;
    }
  }
  // statistics; the pass's counters and queues are reset before the next pass by the element
  // pass that precedes every limiter pass (or by the host-driven entry points)
  __shared__ int s_troubled;
  if (threadIdx.x == 0) s_troubled = 0;
  __syncthreads();
  if (lane == 0 && troubled_local) atomicAdd_block(&s_troubled, troubled_local);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_troubled) atomicAdd(&ctl->troubled, s_troubled);
    if (blockIdx.x == 0) ctl->waves = wave;  // every block leaves after the same wave
  }
}

// compute_time_step, temporal_disc.rs:58-88: each instance's minimum over its elements
// (FP64 arithmetic, deterministic: min of IEEE bit patterns of non-negative doubles).
template <int P, typename T, typename S = T>
__global__ void __launch_bounds__(256) k_time_step(const __grid_constant__ KParams<P, T> kp, const S* __restrict__ U) {
  using V = Variant<P>;
  constexpr int NB = V::NB;
  const MeshDev& m = kp.m;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int ec = e < m.ne ? e : m.ne - 1;
  const int inst = m.n_inst > 1 ? m.inst[ec] : 0;
  unsigned long long bits = 0x7ff0000000000000ull;  // +inf never wins against 1e10
  if (e < m.ne && kp.ic[inst].active) {
    S rec[NEQ * NB];
    load_elem<NB, S, true>(U, e, rec);
    double s[NEQ];
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      double a = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) a += (double)rec[v * NB + b];
      s[v] = a;
    }
    const double hcr = kp.gas.hcr;
    const double rho = s[0];
    const double u = s[1] / rho;
    const double v = s[2] / rho;
    const double p = (hcr - 1.0) * (s[3] - 0.5 * rho * (u * u + v * v));
    const double c = sqrt(hcr * p / rho);
    const double speed = sqrt(u * u + v * v) + c;
    const double dt = kp.ic[inst].cfl * m.hmin[e] / speed;
    if (dt < 1.0e10) bits = (unsigned long long)__double_as_longlong(dt);  // NaN never passes
  }
  const int inst0 = __shfl_sync(0xffffffffu, inst, 0);
  if (__all_sync(0xffffffffu, inst == inst0)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, o);
      bits = other < bits ? other : bits;
    }
    if ((threadIdx.x & 31) == 0 && bits != 0x7ff0000000000000ull) atomicMin(&kp.ic[inst0].dt_bits, bits);
  } else if (bits != 0x7ff0000000000000ull) {
    atomicMin(&kp.ic[inst].dt_bits, bits);  // warp straddles two instances
  }
}

// Head of one time_march iteration (temporal_disc.rs:22-26) in one launch: the loop condition of
// every instance, its CFL time step (compute_time_step, temporal_disc.rs:58-88, as k_time_step)
// and the clamp to final_time.  Every thread evaluates the loop condition of its element's
// instance from the clock it reads (nothing writes the clocks during this kernel); the last block
// to finish (counted in Control::head_done) publishes `active` and the clamped dt.  dt_bits must
// hold the bits of 1e10 (the reference's start value) on entry: the last block restores it after
// reading the minimum, and the host restores it after host-driven time steps.
__device__ __forceinline__ bool step_runs(const InstCtl& c) {
  return c.status == 0 && c.step < c.final_step && c.t < c.final_time;
}

template <int P, typename T, typename S = T>
__device__ __forceinline__ void step_head_elems(const KParams<P, T>& kp, const S* __restrict__ U, int bid) {
  using V = Variant<P>;
  constexpr int NB = V::NB;
  const MeshDev& m = kp.m;
  InstCtl* ic = kp.ic;
  const int e = bid * blockDim.x + threadIdx.x;
  const int ec = e < m.ne ? e : m.ne - 1;
  const int inst = m.n_inst > 1 ? m.inst[ec] : 0;
  unsigned long long bits = 0x7ff0000000000000ull;
  if (e < m.ne && step_runs(ic[inst])) {
    S rec[NEQ * NB];
    load_elem<NB, S, true>(U, e, rec);
    double s[NEQ];
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      double a = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) a += (double)rec[v * NB + b];
      s[v] = a;
    }
    const double hcr = kp.gas.hcr;
    const double rho = s[0];
    const double u = s[1] / rho;
    const double v = s[2] / rho;
    const double p = (hcr - 1.0) * (s[3] - 0.5 * rho * (u * u + v * v));
    const double c = sqrt(hcr * p / rho);
    const double speed = sqrt(u * u + v * v) + c;
    const double dt = ic[inst].cfl * m.hmin[e] / speed;
    if (dt < 1.0e10) bits = (unsigned long long)__double_as_longlong(dt);  // NaN never passes
  }
  const int inst0 = __shfl_sync(0xffffffffu, inst, 0);
  if (__all_sync(0xffffffffu, inst == inst0)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, o);
      bits = other < bits ? other : bits;
    }
    if ((threadIdx.x & 31) == 0 && bits != 0x7ff0000000000000ull) atomicMin(&ic[inst0].dt_bits, bits);
  } else if (bits != 0x7ff0000000000000ull) {
    atomicMin(&ic[inst].dt_bits, bits);
  }
}

// True in the last block of the launch to get here (counted in ctl->head_done, reset by it).
__device__ __forceinline__ bool last_block_in(Control* ctl, unsigned int nblocks) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&ctl->head_done, 1u) == nblocks - 1;
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  if (threadIdx.x == 0) ctl->head_done = 0u;
  return true;
}

// Closes the step head of the instances ic[0, n_inst): loop condition and clamped dt.
__device__ __forceinline__ void step_head_close(Control* ctl, InstCtl* ic, int n_inst) {
  if (threadIdx.x == 0) ctl->troubled = 0;
  for (int i = threadIdx.x; i < n_inst; i += blockDim.x) {
    InstCtl& c = ic[i];
    const int act = step_runs(c) ? 1 : 0;
    c.active = act;
    const unsigned long long start = (unsigned long long)__double_as_longlong(1.0e10);
    const unsigned long long mn = atomicExch(&c.dt_bits, start);
    if (act) {
      double dt = __longlong_as_double((long long)mn);
      if (c.t + dt > c.final_time) dt = c.final_time - c.t;  // temporal_disc.rs:23-26
      c.dt = dt;
    }
  }
}

template <int P, typename T, typename S = T>
__global__ void __launch_bounds__(256) k_step_head(const __grid_constant__ KParams<P, T> kp, const S* __restrict__ U) {
  step_head_elems<P, T, S>(kp, U, blockIdx.x);
  // the last block closes the head: loop condition and clamped dt of every instance
  if (last_block_in(kp.ctl, gridDim.x)) step_head_close(kp.ctl, kp.ic, kp.m.n_inst);
}

// temporal_disc.rs:32-33
__global__ void k_step_end(InstCtl* ic, int n_inst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst || !ic[i].active) return;
  ic[i].t += ic[i].dt;
  ic[i].step += 1;
}
// Host-driven calls (compute_residuals / apply_limiter / rk3 with a given dt): every instance
// steps; set_dt writes the given dt into every instance.
__global__ void k_set_active(Control* ctl, InstCtl* ic, int n_inst, double dt, int set_dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    ctl->troubled = 0;
    reset_limiter_pass(ctl);
  }
  if (i >= n_inst) return;
  ic[i].active = 1;
  if (set_dt) ic[i].dt = dt;
  ic[i].dt_bits = (unsigned long long)__double_as_longlong(1.0e10);
}


// FP64 diagnostics of each instance, one block per instance (deterministic: fixed per-thread
// order, fixed tree): out[i] = { integral of rho, rho u, rho v, rho E over the mesh (mode-0
// coefficient times the element area), pressure force (Fx, Fy) exerted on the wall patches
// (sum over wall edges and Gauss points of w p n |e|/2 with the element's outward normal,
// i.e. the force on the body), sum of squares of the density residual's modal coefficients
// (from R, when given), number of elements }.  Not part of the reference, which computes no
// forces or norms.
template <int P, typename T, typename S = T>
__global__ void __launch_bounds__(256) k_diagnostics(const __grid_constant__ KParams<P, T> kp, const S* __restrict__ U,
                                                     const S* __restrict__ R, const int* __restrict__ elem_rng,
                                                     const int* __restrict__ bslot_rng, double* __restrict__ out) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG, NQ = V::NQ;
  const MeshDev& m = kp.m;
  const int inst = blockIdx.x;
  const int e0 = elem_rng[2 * inst], e1 = e0 + elem_rng[2 * inst + 1];
  const int b0 = bslot_rng[2 * inst], b1 = b0 + bslot_rng[2 * inst + 1];  // boundary slots, relative to n_int
  double wsum = 0.0;
#pragma unroll
  for (int q = 0; q < NQ; ++q) wsum += kp.d.cell_w[q];
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const double area = 0.5 * m.jac[e] * wsum;
#pragma unroll
    for (int v = 0; v < NEQ; ++v) acc[v] += area * (double)U[sx<NB>(e, v, 0)];
    if (R) {
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const double r = (double)R[sx<NB>(e, 0, b)];
        acc[6] += r * r;
      }
    }
  }
  for (int sb = b0 + threadIdx.x; sb < b1; sb += blockDim.x) {
    const int info = m.be_info[sb];
    if (((info >> 2) & 1) != 0) continue;  // far field
    const int e = m.be_elem[sb], k = info & 3;
    const double4 geo = m.be_geo[sb];
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      double q[4];
#pragma unroll
      for (int v = 0; v < NEQ; ++v) {
        double a = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) a += (double)U[sx<NB>(e, v, b)] * kp.d.phi_edge[k][g][b];
        q[v] = a;
      }
      const double p = kp.gas.gm1 * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
      acc[4] += kp.d.edge_w[g] * p * geo.x * geo.z;
      acc[5] += kp.d.edge_w[g] * p * geo.y * geo.z;
    }
  }
  __shared__ double red[7][256];
#pragma unroll
  for (int k = 0; k < 7; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 7; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 7; ++k) out[inst * 8 + k] = red[k][0];
    out[inst * 8 + 7] = (double)(e1 - e0);
  }
}

// Cell fields of write_to_vtk (write_results.rs:33-61) for the elements [e0, e0 + ne): density,
// x and y velocity and pressure from the mode-0 coefficients, in FP64 with the reference's
// expressions and operation order (no contraction into FMAs): velocity = momentum / density,
// pressure = (hcr - 1) (energy - 0.5 density (u^2 + v^2)).  out is [ne][4].
template <int P, typename T, typename S = T>
__global__ void k_cell_fields(const __grid_constant__ KParams<P, T> kp, const S* __restrict__ U, int e0, int ne,
                              double* __restrict__ out) {
  constexpr int NB = Variant<P>::NB;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  const int e = e0 + i;
  const double density = (double)U[sx<NB>(e, 0, 0)];
  const double x_momentum = (double)U[sx<NB>(e, 1, 0)];
  const double y_momentum = (double)U[sx<NB>(e, 2, 0)];
  const double energy = (double)U[sx<NB>(e, 3, 0)];
  const double x_velocity = x_momentum / density;
  const double y_velocity = y_momentum / density;
  const double kinetic = __dadd_rn(__dmul_rn(x_velocity, x_velocity), __dmul_rn(y_velocity, y_velocity));
  const double pressure = __dmul_rn(kp.gas.gm1, __dsub_rn(energy, __dmul_rn(__dmul_rn(0.5, density), kinetic)));
  out[4 * i + 0] = density;
  out[4 * i + 1] = x_velocity;
  out[4 * i + 2] = y_velocity;
  out[4 * i + 3] = pressure;
}

// Conversions between the reference's FP64 arrays and an FP32 state (same element-major
// layout; FP64 states are copied directly).
__global__ void k_f64_to_f32(const double* __restrict__ src, float* __restrict__ dst, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}
__global__ void k_f32_to_f64(const float* __restrict__ src, double* __restrict__ dst, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}

// Initial L2 projection of a uniform state onto the basis (Solver::set_initial_solution,
// solver.rs:45-79): U[e][v][b] = (sum_g 0.5 J_e w_g q_v phi_gb) / (m_b 0.5 J_e), with the
// reference's operation order and no contraction into FMAs, so the result is bit-identical to
// the reference loop.  One thread per element of one instance.
template <int P>
struct Projection {
  using V = Variant<P>;
  double phi[V::NQ][V::NB];
  double w[V::NQ];
  double mass[V::NB];
  double q[NEQ];
};

template <int P, typename T>
__global__ void k_project_uniform(const __grid_constant__ Projection<P> pr, const double* __restrict__ jac,
                                  T* __restrict__ U, int e0, int ne, int ld) {
  using V = Variant<P>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  const int e = e0 + i;
  const double J = jac[e];
  const double hj = __dmul_rn(0.5, J);
#pragma unroll
  for (int v = 0; v < NEQ; ++v) {
#pragma unroll
    for (int b = 0; b < V::NB; ++b) {
      double acc = 0.0;
#pragma unroll
      for (int g = 0; g < V::NQ; ++g)
        acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(__dmul_rn(hj, pr.w[g]), pr.q[v]), pr.phi[g][b]));
      U[sx<V::NB>(e, v, b)] = T(acc / __dmul_rn(__dmul_rn(pr.mass[b], 0.5), J));
    }
  }
}

}  // namespace dgm
