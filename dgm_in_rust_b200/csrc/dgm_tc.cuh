// dgm_tc.cuh -- the element pass with its two basis contractions on the tensor cores (tcgen05).
//
// A CTA of 128 threads owns a tile of 32 elements: row r = 4 * (element slot) + variable, one
// thread and one tensor-memory lane per row.  Per tile:
//   MMA 1 (basis -> quadrature points):  Uq[r][q] = sum_b U[r][b] phi_cell[q][b]
//          A = the tile's modal coefficients (K = NB padded to 8), B = phi_cell (N = NQ -> 16);
//   the thread of row r reads its variable at the NQ points from tensor memory, gathers the other
//   three variables of its element by shuffles, forms the Euler fluxes (flux::flux, flux.rs:154-169)
//   and the edge-flux terms of its faces (spatial_disc.rs:202-206);
//   MMA 2 (quadrature points and edge points -> basis):
//          R[r][b] = sum_q Fx[r][q] dphi/dxi[q][b] + Fe[r][q] dphi/deta[q][b]
//                  + sum_{k,g} Fedge[r][k][g] phi_edge[k][g][b]
//          A = [Fx | Fe | Fedge] (K = 2 NQ + 3 NG padded to 8), B = the stacked tables (N = NB -> 16);
//   then inverse mass and the SSP-RK3 stage update as in k_element.
// Operands are staged in shared memory in the K-major, unswizzled canonical layout (8-row x
// 16-byte core matrices), one elected thread issues tcgen05.mma (kind::tf32, FP32 accumulation
// in tensor memory) and commits to an mbarrier, and every thread reads its accumulator row with
// tcgen05.ld.  SPLIT = 1 feeds TF32-rounded operands (about 1e-3 relative per product); SPLIT = 3
// splits each operand into a TF32 head and tail and sums head*head + tail*head + head*tail,
// which recovers FP32-level products (the 3xTF32 scheme) at three times the MMA work.
// The storage type is FP32; the limiter, time step and positivity checks are unchanged (FP64).
#pragma once
#include <cstdint>

#include "dgm_device.cuh"

namespace dgm {
namespace tc {

constexpr int kRows = 128;           // MMA M
constexpr int kElems = kRows / NEQ;  // elements per tile
constexpr int kThreads = kRows;      // one thread per accumulator row
constexpr int kN = 16;               // MMA N: NQ <= 12 and NB <= 10, padded
constexpr uint32_t kTmemCols = 32;   // accumulator 1 in columns [0, 16), accumulator 2 in [16, 32)
constexpr long long kWaitPolls = 1ll << 24;

template <int P>
struct Dims {
  using V = Variant<P>;
  static constexpr int K1 = (V::NB + 7) / 8 * 8;                  // contraction 1
  static constexpr int KV2 = 2 * V::NQ + 3 * V::NG;                // contraction 2 (valid)
  static constexpr int K2 = (KV2 + 7) / 8 * 8;
};

// Shared-memory plan of one CTA (bytes), dynamic shared memory.
template <int P, int SPLIT>
struct Plan {
  using D = Dims<P>;
  static constexpr int KA = (D::K1 > D::K2 ? D::K1 : D::K2) * SPLIT;
  static constexpr uint32_t a_bytes = kRows * KA * 4;
  static constexpr uint32_t b1_off = a_bytes;
  static constexpr uint32_t b1_bytes = kN * D::K1 * SPLIT * 4;
  static constexpr uint32_t b2_off = b1_off + b1_bytes;
  static constexpr uint32_t b2_bytes = kN * D::K2 * SPLIT * 4;
  static constexpr uint32_t bar_off = (b2_off + b2_bytes + 15) / 16 * 16;
  static constexpr uint32_t bytes = bar_off + 16;  // mbarrier (8 B) + tensor-memory address (4 B)
};

// Byte offset of (row, k) in a K-major, unswizzled operand of `rows` rows: core matrices of
// 8 rows x 16 bytes (4 TF32 values), row groups 128 bytes apart, 4-wide K chunks rows * 16 bytes
// apart.
__host__ __device__ constexpr uint32_t off(int row, int k, int rows) {
  return (uint32_t)(((((k >> 2) * (rows >> 3)) + (row >> 3)) << 7) + ((row & 7) << 4) + ((k & 3) << 2));
}

// Shared-memory matrix descriptor: start address, leading byte offset (K-chunk stride), stride
// byte offset (row-group stride), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Writes operand value x for (row, k) of a K-major operand of K columns: SPLIT 1 stores the TF32
// rounding; SPLIT 3 stores [head | tail | head] (A) or [head | head | tail] (B) along K.
template <int SPLIT, bool IS_A>
__device__ __forceinline__ void put(unsigned char* base, int row, int k, int K, int rows, float x) {
  const float hi = tf32_round(x);
  if constexpr (SPLIT == 1) {
    *reinterpret_cast<float*>(base + off(row, k, rows)) = hi;
  } else {
    const float lo = x - hi;
    *reinterpret_cast<float*>(base + off(row, k, rows)) = hi;
    *reinterpret_cast<float*>(base + off(row, K + k, rows)) = IS_A ? lo : hi;
    *reinterpret_cast<float*>(base + off(row, 2 * K + k, rows)) = IS_A ? hi : lo;
  }
}

// Writes the 4-wide K chunk c (k = 4c .. 4c+3) of row `row` of the A operand with one 16-byte
// store per part (a warp's 32 rows then fill 512 contiguous bytes: no bank conflicts).
template <int SPLIT>
__device__ __forceinline__ void put_a4(unsigned char* base, int row, int c, int K, const float (&x)[4]) {
  float4 hi, lo;
  hi.x = tf32_round(x[0]);
  hi.y = tf32_round(x[1]);
  hi.z = tf32_round(x[2]);
  hi.w = tf32_round(x[3]);
  *reinterpret_cast<float4*>(base + off(row, 4 * c, kRows)) = hi;
  if constexpr (SPLIT == 3) {
    lo = make_float4(x[0] - hi.x, x[1] - hi.y, x[2] - hi.z, x[3] - hi.w);
    *reinterpret_cast<float4*>(base + off(row, K + 4 * c, kRows)) = lo;
    *reinterpret_cast<float4*>(base + off(row, 2 * K + 4 * c, kRows)) = hi;
  }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A * B^T over one K-step of 8, issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1 : 0)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// Bounded wait for the mbarrier phase with parity `phase`; false if the bound ran out.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
  for (long long it = 0; it < kWaitPolls; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// This thread's accumulator row: 16 consecutive FP32 columns starting at `col`.
__device__ __forceinline__ void tmem_row16(uint32_t tmem, int warp, int col, float (&v)[16]) {
  const uint32_t addr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)col;
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc

// Element pass (as k_element<P, float, MODE>) with both contractions on the tensor cores.
// Persistent: each CTA allocates its 32 tensor-memory columns once and loops over tiles.
template <int P, int MODE, int SPLIT>
__global__ void __launch_bounds__(tc::kThreads, 8) k_element_tc(const __grid_constant__ KParams<P, float> kp,
                                                              const float* __restrict__ Uin, const float* Ubase,
                                                              const float* __restrict__ F, float* Uout,
                                                              const float* Rin, float* Rout) {
  using V = Variant<P>;
  using D = tc::Dims<P>;
  using PL = tc::Plan<P, SPLIT>;
  constexpr int NB = V::NB, NQ = V::NQ, NG = V::NG;
  constexpr int K1 = D::K1, K2 = D::K2;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sa = smem;
  unsigned char* sb1 = smem + PL::b1_off;
  unsigned char* sb2 = smem + PL::b2_off;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + PL::bar_off);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + PL::bar_off + 8);
  Control* ctl = kp.ctl;
  const MeshDev& m = kp.m;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (blockIdx.x == 0 && t == 0) reset_limiter_pass(ctl);  // for the limiter pass that follows
  // constant operands: B1[q][b] = phi_cell, B2[b][k] = [dxi | deta | phi_edge] (zero padded)
  for (int i = t; i < tc::kN * K1; i += tc::kThreads) {
    const int n = i / K1, k = i - n * K1;
    const float x = (n < NQ && k < NB) ? kp.t.phi_cell[n][k] : 0.f;
    tc::put<SPLIT, false>(sb1, n, k, K1, tc::kN, x);
  }
  for (int i = t; i < tc::kN * K2; i += tc::kThreads) {
    const int n = i / K2, k = i - n * K2;
    float x = 0.f;
    if (n < NB) {
      if (k < NQ) x = kp.t.dxi[k][n];
      else if (k < 2 * NQ) x = kp.t.deta[k - NQ][n];
      else if (k < D::KV2) {
        const int kk = (k - 2 * NQ) / NG, g = (k - 2 * NQ) - kk * NG;
        x = kp.t.phi_edge[kk][g][n];
      }
    }
    tc::put<SPLIT, false>(sb2, n, k, K2, tc::kN, x);
  }
  const uint32_t bar_a = tc::smem_addr(bar);
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_addr(tmem_slot)),
                 "r"(tc::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc::fence_async_smem();
  tc::tc_before_sync();
  __syncthreads();
  tc::tc_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tc::idesc_tf32(tc::kRows, tc::kN);
  const uint32_t a_s = tc::smem_addr(sa), b1_s = tc::smem_addr(sb1), b2_s = tc::smem_addr(sb2);
  uint32_t phase = 0;
  const int slot_e = t >> 2, var = t & 3;
  const size_t ld = m.ld;
  for (int tile = blockIdx.x; tile * tc::kElems < m.ne; tile += gridDim.x) {
    const int e_raw = tile * tc::kElems + slot_e;
    const int e = e_raw < m.ne ? e_raw : m.ne - 1;
    const int inst = m.n_inst > 1 ? m.inst[e] : 0;
    const bool valid = e_raw < m.ne && kp.ic[inst].active;
    float u[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) u[b] = ld_state(&Uin[sx<NB>(e, var, b)]);
    // geometry and the faces' edge fluxes: loaded now, used after the first contraction
    const float J = (float)m.jac[e];
    const float xx = (float)m.dinv[0 * ld + e], xy = (float)m.dinv[1 * ld + e], ex = (float)m.dinv[2 * ld + e],
                ey = (float)m.dinv[3 * ld + e];
    float a2[D::K2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int fw = m.face[k * ld + e];
      const int slot = fw >> 1;
      const bool right = fw & 1;
      const float* Fs = &F[(size_t)slot * NG * 4 + var];
#pragma unroll
      for (int gp = 0; gp < NG; ++gp) {
        const int src = right ? (NG - 1 - gp) : gp;
        const float coef = right ? kp.t.edge_w[gp] : -kp.t.edge_w[gp];
        a2[2 * NQ + k * NG + gp] = coef * __ldcg(&Fs[src * 4]);
      }
    }
#pragma unroll
    for (int k = D::KV2; k < K2; ++k) a2[k] = 0.f;
    // ---- contraction 1: modal coefficients -> values at the quadrature points ----
#pragma unroll
    for (int c = 0; c < K1 / 4; ++c) {
      float x[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) x[j] = 4 * c + j < NB ? u[4 * c + j] : 0.f;
      tc::put_a4<SPLIT>(sa, t, c, K1, x);
    }
    tc::fence_async_smem();
    tc::tc_before_sync();
    __syncthreads();
    if (t == 0) {
      tc::tc_after_sync();
#pragma unroll
      for (int s = 0; s < K1 * SPLIT / 8; ++s)
        tc::mma_tf32(tmem, tc::sdesc(a_s + s * 2 * tc::kRows * 16, tc::kRows * 16, 128),
                     tc::sdesc(b1_s + s * 2 * tc::kN * 16, tc::kN * 16, 128), idesc, s > 0);
      tc::mma_commit(bar_a);
    }
    bool ok = tc::bar_wait(bar_a, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      if (t == 0 && atomicCAS(&ctl->status, 0, ST_TIMEOUT) == 0) ctl->err_where = -1;
      break;
    }
    tc::tc_after_sync();
    float uq[16];
    tc::tmem_row16(tmem, warp, 0, uq);
    // ---- fluxes at the quadrature points (flux::flux) ----
    const float gm1 = (float)kp.gas.gm1;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      float qs[NEQ];
#pragma unroll
      for (int w = 0; w < NEQ; ++w) qs[w] = __shfl_sync(0xffffffffu, uq[q], (lane & ~3) + w);
      float f[NEQ], g[NEQ];
      euler_flux<float>(qs, gm1, f, g);
      const float fv = var == 0 ? f[0] : var == 1 ? f[1] : var == 2 ? f[2] : f[3];
      const float gv = var == 0 ? g[0] : var == 1 ? g[1] : var == 2 ? g[2] : g[3];
      const float sc = kp.t.cell_w[q] * 0.5f * J;
      a2[q] = sc * (fv * xx + gv * xy);
      a2[NQ + q] = sc * (fv * ex + gv * ey);
    }
    // ---- contraction 2: volume and face terms -> modal residual ----
#pragma unroll
    for (int c = 0; c < K2 / 4; ++c) {
      const float x[4] = {a2[4 * c], a2[4 * c + 1], a2[4 * c + 2], a2[4 * c + 3]};
      tc::put_a4<SPLIT>(sa, t, c, K2, x);
    }
    tc::fence_async_smem();
    tc::tc_before_sync();
    __syncthreads();
    if (t == 0) {
      tc::tc_after_sync();
#pragma unroll
      for (int s = 0; s < K2 * SPLIT / 8; ++s)
        tc::mma_tf32(tmem + (uint32_t)tc::kN, tc::sdesc(a_s + s * 2 * tc::kRows * 16, tc::kRows * 16, 128),
                     tc::sdesc(b2_s + s * 2 * tc::kN * 16, tc::kN * 16, 128), idesc, s > 0);
      tc::mma_commit(bar_a);
    }
    ok = tc::bar_wait(bar_a, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      if (t == 0 && atomicCAS(&ctl->status, 0, ST_TIMEOUT) == 0) ctl->err_where = -1;
      break;
    }
    tc::tc_after_sync();
    float r[16];
    tc::tmem_row16(tmem, warp, tc::kN, r);
    // ---- inverse mass and stage update (as k_element) ----
    if (valid) {
      const float dt = (float)kp.ic[inst].dt;
      const float inv_half_j = 1.f / (0.5f * J);
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const size_t idx = sx<NB>(e, var, b);
        float rr = r[b];
        if constexpr (MODE == 0) rr = Rin[idx] + rr;
        rr = rr * kp.t.inv_mass[b] * inv_half_j;
        if (Rout) Rout[idx] = rr;
        if constexpr (MODE == 1) {
          Uout[idx] = u[b] + dt * rr;
        } else if constexpr (MODE == 2) {
          Uout[idx] = 0.75f * Ubase[idx] + 0.25f * (u[b] + dt * rr);
        } else if constexpr (MODE == 3) {
          Uout[idx] = (1.f / 3.f) * Ubase[idx] + (2.f / 3.f) * (u[b] + dt * rr);
        }
      }
    }
    tc::tc_before_sync();  // this tile's accumulator reads precede the next tile's MMAs
  }
  // after a wait that ran out, give the tensor cores a second bounded wait before the columns
  // are freed (on the normal exit the last phase is complete and this returns at once)
  if (t == 0) tc::bar_wait(bar_a, phase ^ 1u);
  tc::tc_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::tc_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::kTmemCols) : "memory");
  }
}

}  // namespace dgm
