// dgm_mixed.cuh -- kernels of a mixed batch: meshes of different polynomial orders advanced by the
// same launches.
//
// A mixed batch holds one group per order (its own union mesh, tables and state arrays, as a
// single-order batch has them).  Every kernel of a step is ONE launch over all groups: the blocks
// of a launch are split into consecutive ranges, one per group, and each block runs the body of
// its group's order (the same bodies as the single-order kernels, compiled for that order), so
// each group computes exactly what it computes alone.  The limiter's wave kernel, a cooperative
// launch with grid barriers, takes its work items from all groups' lists in one index space and
// dispatches each to its group's order.  MASK is the set of orders the launch is compiled for
// (bit P-1 for order P); a group without meshes gets no blocks and no work.
#pragma once
#include <type_traits>

#include "dgm_device.cuh"

namespace dgm {

struct NoParams {};
template <int P, typename T, bool ON>
using KParamsIf = typename std::conditional<ON, KParams<P, T>, NoParams>::type;

// The device arrays one launch uses of one group, and the group's share of the launch's blocks
// (states of storage type S, edge fluxes of the arithmetic type T).
template <typename T, typename S = T>
struct GroupArgs {
  const S* Uin;
  const S* Ubase;
  S* Uout;
  const S* Rin;
  S* Rout;
  T* F;
  unsigned char* t0;
  unsigned int* status;
  int* wl1;
  int* pend;
  const int* order;
  int blocks;
  int n_inst;  // instances of the group (without the dead instance of padded groups); 0 = no group
};

template <typename T, int MASK, typename S = T>
struct Mixed {
  KParamsIf<1, T, (MASK & 1) != 0> k1;
  KParamsIf<2, T, (MASK & 2) != 0> k2;
  KParamsIf<3, T, (MASK & 4) != 0> k3;
  GroupArgs<T, S> g[3];
};

template <class K>
struct OrderOf;
template <int P, typename T>
struct OrderOf<KParams<P, T>> {
  static constexpr int value = P;
};

// Calls f(kparams, group args, block index within the group, the group's block count) for the
// group that owns this block.
template <typename T, int MASK, typename S, class F>
__device__ __forceinline__ void on_block(const Mixed<T, MASK, S>& mp, F&& f) {
  int b = blockIdx.x;
  if constexpr ((MASK & 1) != 0) {
    if (b < mp.g[0].blocks) {
      f(mp.k1, mp.g[0], b, mp.g[0].blocks);
      return;
    }
    b -= mp.g[0].blocks;
  }
  if constexpr ((MASK & 2) != 0) {
    if (b < mp.g[1].blocks) {
      f(mp.k2, mp.g[1], b, mp.g[1].blocks);
      return;
    }
    b -= mp.g[1].blocks;
  }
  if constexpr ((MASK & 4) != 0) {
    if (b < mp.g[2].blocks) f(mp.k3, mp.g[2], b, mp.g[2].blocks);
  }
}

// Calls f(kparams, group args) for group index g (0, 1, 2 = order 1, 2, 3) if that group has
// meshes (a group without meshes has no parameters to read).
template <typename T, int MASK, typename S, class F>
__device__ __forceinline__ void with_group(const Mixed<T, MASK, S>& mp, int g, F&& f) {
  if constexpr ((MASK & 1) != 0) {
    if (g == 0) {
      if (mp.g[0].n_inst > 0) f(mp.k1, mp.g[0]);
      return;
    }
  }
  if constexpr ((MASK & 2) != 0) {
    if (g == 1) {
      if (mp.g[1].n_inst > 0) f(mp.k2, mp.g[1]);
      return;
    }
  }
  if constexpr ((MASK & 4) != 0) {
    if (g == 2 && mp.g[2].n_inst > 0) f(mp.k3, mp.g[2]);
  }
}

// The control block of the first group with meshes: grid barrier, block counters and the wave
// counters of the mixed limiter.
template <typename T, int MASK, typename S>
__device__ __forceinline__ Control* lead_ctl(const Mixed<T, MASK, S>& mp) {
  if constexpr ((MASK & 1) != 0) {
    if (mp.g[0].n_inst > 0) return mp.k1.ctl;
  }
  if constexpr ((MASK & 2) != 0) {
    if (mp.g[1].n_inst > 0) return mp.k2.ctl;
  }
  if constexpr ((MASK & 4) != 0) return mp.k3.ctl;
  return nullptr;
}

template <typename T, int MASK, typename S = T>
__global__ void __launch_bounds__(256, 3) k_edge_flux_mixed(const __grid_constant__ Mixed<T, MASK, S> mp) {
  on_block(mp, [&](const auto& kp, const GroupArgs<T, S>& g, int b, int nb) {
    constexpr int P = OrderOf<std::decay_t<decltype(kp)>>::value;
    edge_flux_body<P, T, S>(kp, g.Uin, g.F, b, nb);
  });
}

template <typename T, int MASK, int MODE, typename S = T>
__global__ void __launch_bounds__(256, 3) k_element_mixed(const __grid_constant__ Mixed<T, MASK, S> mp) {
  on_block(mp, [&](const auto& kp, const GroupArgs<T, S>& g, int b, int) {
    constexpr int P = OrderOf<std::decay_t<decltype(kp)>>::value;
    element_body<P, T, MODE, S>(kp, g.Uin, g.Ubase, g.F, g.Uout, g.Rin, g.Rout, b);
  });
}

// Shared bytes of the largest order of the set (the detection blocks' staged records).
template <typename S, int MASK>
struct MixedDetectSmem {
  static constexpr size_t b1 = (MASK & 1) ? DetectSmem<1, S>::kBytes : 0;
  static constexpr size_t b2 = (MASK & 2) ? DetectSmem<2, S>::kBytes : 0;
  static constexpr size_t b3 = (MASK & 4) ? DetectSmem<3, S>::kBytes : 0;
  static constexpr size_t m12 = b1 > b2 ? b1 : b2;
  static constexpr size_t bytes = m12 > b3 ? m12 : b3;
};

template <typename T, int MASK, bool STAGED, typename S = T>
__global__ void __launch_bounds__(kDetectThreads) k_lim_detect_mixed(const __grid_constant__ Mixed<T, MASK, S> mp) {
  __shared__ __align__(16) unsigned char s_det[MixedDetectSmem<S, MASK>::bytes];
  on_block(mp, [&](const auto& kp, const GroupArgs<T, S>& g, int b, int) {
    constexpr int P = OrderOf<std::decay_t<decltype(kp)>>::value;
    lim_detect_body<P, T, STAGED, S>(kp, g.Uin, g.t0, g.status, g.wl1, g.pend, g.order, b, reinterpret_cast<S*>(s_det));
  });
}

template <typename T, int MASK, typename S = T>
__global__ void __launch_bounds__(256) k_step_head_mixed(const __grid_constant__ Mixed<T, MASK, S> mp) {
  on_block(mp, [&](const auto& kp, const GroupArgs<T, S>& g, int b, int) {
    constexpr int P = OrderOf<std::decay_t<decltype(kp)>>::value;
    step_head_elems<P, T, S>(kp, g.Uin, b);
  });
  if (!last_block_in(lead_ctl(mp), gridDim.x)) return;
  for (int gi = 0; gi < 3; ++gi)
    with_group(mp, gi, [&](const auto& kp, const GroupArgs<T, S>&) { step_head_close(kp.ctl, kp.ic, kp.m.n_inst); });
}

template <typename T, int MASK, typename S = T>
__global__ void k_step_end_mixed(const __grid_constant__ Mixed<T, MASK, S> mp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int gi = 0; gi < 3; ++gi) {
    bool mine = false;
    with_group(mp, gi, [&](const auto& kp, const GroupArgs<T, S>& g) {
      if (i < g.n_inst) {
        mine = true;
        InstCtl& c = kp.ic[i];
        if (c.active) {
          c.t += c.dt;
          c.step += 1;
        }
      } else {
        i -= g.n_inst;
      }
    });
    if (mine) return;
  }
}

// WENO scratch of the largest order of the set.
template <int MASK>
struct MixedScratch {
  static constexpr size_t b1 = (MASK & 1) ? sizeof(WenoScratch<1>) : 0;
  static constexpr size_t b2 = (MASK & 2) ? sizeof(WenoScratch<2>) : 0;
  static constexpr size_t b3 = (MASK & 4) ? sizeof(WenoScratch<3>) : 0;
  static constexpr size_t m12 = b1 > b2 ? b1 : b2;
  static constexpr size_t bytes = ((m12 > b3 ? m12 : b3) + 127) / 128 * 128;
};

// The limiter's wave kernel over all groups (k_limiter of each group, in one cooperative launch):
// wave 1 reconstructs the cells every group's detection enlisted; waves 2, 3, ... scan the
// groups' pending lists together, enlist ready troubled elements of any group in one worklist
// (`work`, entries (group << 30) | element) and reconstruct them, a grid barrier between the
// phases (the barrier schedule of k_limiter).  Elements only neighbour elements of their own
// group, so each group settles exactly as in its own pass.  The lead group's control block holds
// the grid barrier and the wave counters; the element pass of the next stage resets every group's
// counters.
// Held at 3 blocks per SM (168 registers) when the batch has orders 1 and 2 only -- the occupancy
// of the order-2 kernel; with order 3 (whose kernel alone needs 222 registers), 2 blocks per SM.
template <typename T, int MASK, typename S = T>
__global__ void __launch_bounds__(kLimiterWarps * 32, (MASK & 4) ? 2 : 3) k_limiter_mixed(const __grid_constant__ Mixed<T, MASK, S> mp,
                                                                      int* __restrict__ work) {
  Control* ctl = lead_ctl(mp);
  constexpr size_t kWarpBytes = MixedScratch<MASK>::bytes;
  __shared__ __align__(128) unsigned char s_warp[kLimiterWarps][kWarpBytes];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * kLimiterWarps + wib;
  const int nwarps = gridDim.x * kLimiterWarps;
  // the detection launch has finished: its counts are final
  int flagged = 0, n1[3] = {0, 0, 0}, np[3] = {0, 0, 0}, cap = 0;  // cap: the worklist's length
  for (int gi = 0; gi < 3; ++gi)
    with_group(mp, gi, [&](const auto& kp, const GroupArgs<T, S>&) {
      flagged += kp.ctl->t0_count;
      n1[gi] = min(kp.ctl->wl1_count, kp.m.ne);  // larger only after an overflow (reported)
      np[gi] = min(kp.ctl->pend_count, kp.m.ne);
      cap += kp.m.ne;
    });
  const int n1_all = n1[0] + n1[1] + n1[2], np_all = np[0] + np[1] + np[2];
  int troubled_local[3] = {0, 0, 0};
  int wave = 1;
  // reconstruction of element et of group gi; faces and neighbours from its worklist entry
  // (have_ids) or loaded here
  auto reconstruct = [&](int gi, int et, bool have_ids, const int (&fin)[3], const int (&nin)[3]) {
    with_group(mp, gi, [&](const auto& kp, const GroupArgs<T, S>& g) {
      constexpr int P = OrderOf<std::decay_t<decltype(kp)>>::value;
      const MeshDev& m = kp.m;
      int fwt[3], nbt[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        fwt[k] = have_ids ? fin[k] : m.face[k * m.ld + et];
        nbt[k] = have_ids ? nin[k] : m.nbr[k * m.ld + et];
      }
      const int rs = weno_reconstruct<P, T, S>(kp, g.Uout, et, fwt, nbt, lane,
                                            *reinterpret_cast<WenoScratch<P>*>(s_warp[wib]));
      if (rs != ST_OK && lane == 0) {
        const int inst = m.n_inst > 1 ? m.inst[et] : 0;
        raise_status(kp.ctl, &kp.ic[inst], rs, et);
      }
    });
  };
  auto split = [&](const int (&n)[3], int i, int& gi) {  // global list index -> (group, index)
    gi = 0;
    while (gi < 2 && i >= n[gi]) i -= n[gi++];
    return i;
  };
  if (flagged > 0) {
    // ---- wave 1: the cells enlisted by the detections ----
    for (int i = gwarp; i < n1_all; i += nwarps) {
      int gi;
      const int li = split(n1, i, gi);
      int et = 0, fwt[3], nbt[3];
      with_group(mp, gi, [&](const auto&, const GroupArgs<T, S>& g) { et = entry_get(g.wl1, li, lane, fwt, nbt); });
      reconstruct(gi, et, true, fwt, nbt);
      with_group(mp, gi, [&](const auto&, const GroupArgs<T, S>& g) {
        if (lane == 0) g.status[et] = (1u << 2) | 2u;
      });
      ++troubled_local[gi];
    }
    // ---- waves 2, 3, ...: the elements that waited for a lower neighbour, all groups ----
    bool more = np_all > 0;
    if (more && !grid_barrier(ctl, gridDim.x)) more = false;
    for (wave = 2; more; ++wave) {
      int unknown_local = 0;
      for (int base = gwarp * 32; base < np_all; base += nwarps * 32) {
        const int i = base + lane;
        bool pending = false, ready = false, trouble = false;
        int gi = 0, e = 0;
        if (i < np_all) {
          const int li = split(np, i, gi);
          with_group(mp, gi, [&](const auto& kp, const GroupArgs<T, S>& g) {
            constexpr int P = OrderOf<std::decay_t<decltype(kp)>>::value;
            const MeshDev& m = kp.m;
            e = __ldcg(&g.pend[li]);
            pending = (__ldcg(&g.status[e]) & 3u) == 0u;
            if (!pending) return;
            bool any_mod = false;
            ready = true;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              const int nb = m.nbr[k * m.ld + e];
              if (nb >= 0 && nb < e) {
                const unsigned int sn = __ldcg(&g.status[nb]);
                if ((sn & 3u) == 0u || (int)(sn >> 2) >= wave) ready = false;
                else if ((sn & 3u) == 2u) any_mod = true;
              }
            }
            if (!ready) return;
            if (any_mod) {
              const S* own = g.Uout + (size_t)e * (NEQ * Variant<P>::NB);
              trouble = kxrcf<P, T, false, false, S>(kp, g.Uout, e, own);
            } else {
              trouble = g.t0[e] != 0;
            }
            if (!trouble) g.status[e] = ((unsigned int)wave << 2) | 1u;
          });
        }
        const unsigned int tb = __ballot_sync(0xffffffffu, ready && trouble);
        if (tb) {
          int slot0 = 0;
          if (lane == 0) slot0 = atomicAdd(&ctl->wl_count[wave & 1], __popc(tb));
          slot0 = __shfl_sync(0xffffffffu, slot0, 0);
          if (ready && trouble) list_put(ctl, work, slot0 + __popc(tb & ((1u << lane) - 1u)), cap, (gi << 30) | e);
        }
        unknown_local += (pending && !ready) ? 1 : 0;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) unknown_local += __shfl_xor_sync(0xffffffffu, unknown_local, o);
      if (lane == 0 && unknown_local) atomicAdd(&ctl->unknown[wave & 1], unknown_local);
      if (!grid_barrier(ctl, gridDim.x)) break;
      const int n_work = min(*((volatile int*)&ctl->wl_count[wave & 1]), cap);
      const int remaining = *((volatile int*)&ctl->unknown[wave & 1]);
      // the other parity's counters were last read before the previous wave's second barrier
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->wl_count[(wave + 1) & 1] = 0;
        ctl->unknown[(wave + 1) & 1] = 0;
      }
      for (int i = gwarp; i < n_work; i += nwarps) {
        const int entry = __ldcg(&work[i]);
        const int gi = entry >> 30, et = entry & ((1 << 30) - 1);
        const int none[3] = {0, 0, 0};
        reconstruct(gi, et, false, none, none);
        __threadfence();
        with_group(mp, gi, [&](const auto&, const GroupArgs<T, S>& g) {
          if (lane == 0) g.status[et] = ((unsigned int)wave << 2) | 2u;
        });
        ++troubled_local[gi];
      }
      if (remaining == 0) break;  // no further wave: nothing reads what this one wrote
      if (!grid_barrier(ctl, gridDim.x)) break;
      if (wave > (1 << 29)) break;
    }
  }
  // statistics; every group's counters are reset before the next pass by the element pass
  __shared__ int s_troubled[3];
  if (threadIdx.x < 3) s_troubled[threadIdx.x] = 0;
  __syncthreads();
  for (int gi = 0; gi < 3; ++gi)
    if (lane == 0 && troubled_local[gi]) atomicAdd_block(&s_troubled[gi], troubled_local[gi]);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int gi = 0; gi < 3; ++gi)
      with_group(mp, gi, [&](const auto& kp, const GroupArgs<T, S>&) {
        if (s_troubled[gi]) atomicAdd(&kp.ctl->troubled, s_troubled[gi]);
        if (blockIdx.x == 0) kp.ctl->waves = wave;
      });
  }
}

}  // namespace dgm
