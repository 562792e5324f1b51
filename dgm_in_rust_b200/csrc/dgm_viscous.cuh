// dgm_viscous.cuh -- the Navier-Stokes (BR2) residual that the reference keeps disabled
// (spatial_disc.rs:34-36): integrate_over_cell_ns (spatial_disc.rs:70-160), integrate_over_edges_ns
// (:212-348) and apply_bc_ns (boundary_condition.rs:121-413), with Sutherland's viscosity and the
// viscous Jacobians of viscous.rs:6-64.  FP64 only.  A context switched to it (dgm_set_viscous)
// runs, per stage, three launches in place of the Euler edge and element passes:
//
//   k_ns_lift      a thread per (element, variable): the element's global lifting operator --
//                  the jumps across its faces (the neighbour chosen by the reference's in-cell index
//                  test, spatial_disc.rs:86-93), plus on boundary faces the wall / far-field local
//                  lifts (boundary_condition.rs:181-302) -- divided by the mass diagonal;
//   k_edge_flux_ns four lanes per edge slot (the lifts once per slot, a point per lane): HLLC minus
//                  the viscous flux of both sides, each with its own gradient and its local lift
//                  (the left one scaled by 3, the right one not, spatial_disc.rs:298-299,
//                  326-327), stored like the Euler fluxes; boundary slots: the wall / far-field
//                  inviscid flux minus the viscous one;
//   k_element_ns   the Euler element pass with the volume term (F - Fv, G - Gv), the viscous
//                  fluxes from the state's gradient plus the global lift at each cell point.
//
// Everything the reference evaluates per (variable, mode) is evaluated here in its order within
// each term; the sums over edges and elements are gathered as in the Euler passes (the reference
// folds them in a run-dependent order), so results agree with the oracle to round-off.
#pragma once

#include "dgm_device.cuh"

namespace dgm {

template <int P>
struct NsParams {
  using V = Variant<P>;
  double dphi_edge[3][V::NG][V::NB][2];  // reference-space d/dxi, d/deta at the edge points
  double mass[V::NB];                    // mass_mat_diag
  double hp;                             // hcr / prandtl_number
  double rgas;                           // gas_constant
  double* lift;                          // [ld][2][4][NB]: x and y global lifts (k_ns_lift)
};

// compute_dynamic_viscosity (viscous.rs:6-12) of a state: p, T = p / (R rho), Sutherland's law.
__device__ __forceinline__ double ns_viscosity(const double q[4], const Gas& gas, double rgas) {
  const double pressure = gas.gm1 * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
  const double temperature = pressure / (rgas * q[0]);
  const double mu_ref = 1.716e-5, sutherland_constant = 110.4, t_ref = 273.15;
  return mu_ref * pow(temperature / t_ref, 1.5) * (t_ref + sutherland_constant) / (temperature + sutherland_constant);
}

// Entry (i, j) of g11 (m = 0), g12 (1), g21 (2), g22 (3) of viscous_jacobian (viscous.rs:13-57)
// before the scaling by mu / rho; u, v, e = q[1..3] / q[0], hp = hcr / prandtl_number.
__device__ __forceinline__ double ns_g(int m, int i, int j, double u, double v, double e, double hp) {
  switch (m * 16 + i * 4 + j) {
    case 0 * 16 + 1 * 4 + 0: return -4.0 / 3.0 * u;
    case 0 * 16 + 1 * 4 + 1: return 4.0 / 3.0;
    case 0 * 16 + 2 * 4 + 0: return -v;
    case 0 * 16 + 2 * 4 + 2: return 1.0;
    case 0 * 16 + 3 * 4 + 0: return -(4.0 / 3.0 * (u * u) + v * v + hp * (e - u * u - v * v));
    case 0 * 16 + 3 * 4 + 1: return (4.0 / 3.0 - hp) * u;
    case 0 * 16 + 3 * 4 + 2: return (1.0 - hp) * v;
    case 0 * 16 + 3 * 4 + 3: return hp;
    case 1 * 16 + 1 * 4 + 0: return 2.0 / 3.0 * v;
    case 1 * 16 + 1 * 4 + 2: return -2.0 / 3.0;
    case 1 * 16 + 2 * 4 + 0: return -u;
    case 1 * 16 + 2 * 4 + 1: return 1.0;
    case 1 * 16 + 3 * 4 + 0: return -1.0 / 3.0 * u * v;
    case 1 * 16 + 3 * 4 + 1: return v;
    case 1 * 16 + 3 * 4 + 2: return -2.0 / 3.0 * u;
    case 2 * 16 + 1 * 4 + 0: return -v;
    case 2 * 16 + 1 * 4 + 2: return 1.0;
    case 2 * 16 + 2 * 4 + 0: return 2.0 / 3.0 * u;
    case 2 * 16 + 2 * 4 + 1: return -2.0 / 3.0;
    case 2 * 16 + 3 * 4 + 0: return -1.0 / 3.0 * u * v;
    case 2 * 16 + 3 * 4 + 1: return -2.0 / 3.0 * v;
    case 2 * 16 + 3 * 4 + 2: return u;
    case 3 * 16 + 1 * 4 + 0: return -u;
    case 3 * 16 + 1 * 4 + 1: return 1.0;
    case 3 * 16 + 2 * 4 + 0: return -4.0 / 3.0 * v;
    case 3 * 16 + 2 * 4 + 2: return 4.0 / 3.0;
    case 3 * 16 + 3 * 4 + 0: return -(u * u + 4.0 / 3.0 * (v * v) + hp * (e - u * u - v * v));
    case 3 * 16 + 3 * 4 + 1: return (1.0 - hp) * u;
    case 3 * 16 + 3 * 4 + 2: return (4.0 / 3.0 - hp) * v;
    case 3 * 16 + 3 * 4 + 3: return hp;
    default: return 0.0;
  }
}

// Rows i of (fv, gv) = G (gradient + lift) at state q (the iflux loop of spatial_disc.rs:131-146):
// gx[j], gy[j] are dsol_dx + lift_x and dsol_dy + lift_y of variable j.
__device__ __forceinline__ void ns_viscous_row(int i, const double q[4], double mu, double hp, const double gx[4],
                                               const double gy[4], double& fv, double& gv) {
  const double u = q[1] / q[0], v = q[2] / q[0], e = q[3] / q[0];
  const double scale = mu / q[0];
  fv = 0.0;
  gv = 0.0;
#pragma unroll
  for (int j = 0; j < NEQ; ++j) {
    const double g11 = ns_g(0, i, j, u, v, e, hp) * scale, g12 = ns_g(1, i, j, u, v, e, hp) * scale;
    const double g21 = ns_g(2, i, j, u, v, e, hp) * scale, g22 = ns_g(3, i, j, u, v, e, hp) * scale;
    fv += g11 * gx[j] + g12 * gy[j];
    gv += g21 * gx[j] + g22 * gy[j];
  }
}

// The local lift of variable w on boundary slot sb (boundary_condition.rs:181-302): the wall's
// momentum and energy jumps with the cell tables at the point index, the far field's jumps to the
// characteristic state with the edge tables.
template <int P>
__device__ __noinline__ void ns_boundary_lift(const KParams<P, double>& kp, const double* __restrict__ Ue, int sb,
                                              int w, double J, double (&llx)[Variant<P>::NB],
                                              double (&lly)[Variant<P>::NB]) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  const MeshDev& m = kp.m;
  const int info = m.be_info[sb];
  const int ic = info & 3;
  const double4 geo = m.be_geo[sb];
  const bool wall = ((info >> 2) & 1) == 0;
  for (int b = 0; b < NB; ++b) llx[b] = lly[b] = 0.0;
  if (wall && w == 0) return;
  for (int g = 0; g < NG; ++g) {
    double lv[4];
    for (int v = 0; v < NEQ; ++v) {
      double a = 0.0;
      for (int b = 0; b < NB; ++b) a += Ue[v * NB + b] * kp.d.phi_edge[ic][g][b];
      lv[v] = a;
    }
    double comp;
    if (wall) {  // boundary_condition.rs:183-201: momentum and energy jumps, cell tables at g
      const double pressure = kp.gas.gm1 * (lv[3] - 0.5 * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
      const double boundary_energy = pressure / kp.gas.gm1;
      comp = w == 1 ? lv[1] : w == 2 ? lv[2] : lv[3] - boundary_energy;
    } else {  // boundary_condition.rs:264-289
      double q[4];
      far_field_state<double>(lv, geo.x, geo.y, m.patch_q[info >> 3], kp.gas, q);
      comp = lv[w] - q[w];
    }
    const double jx = comp * geo.x, jy = comp * geo.y;
    for (int b = 0; b < NB; ++b) {
      if (wall) {
        llx[b] -= 0.5 * jx * kp.t.phi_cell[g][b] * kp.d.cell_w[g] * 0.5 * J;
        lly[b] -= 0.5 * jy * kp.t.phi_cell[g][b] * kp.d.cell_w[g] * 0.5 * J;
      } else {
        llx[b] -= 0.5 * jx * kp.d.phi_edge[ic][g][b] * kp.d.edge_w[g] * 0.5 * geo.w;
        lly[b] -= 0.5 * jy * kp.d.phi_edge[ic][g][b] * kp.d.edge_w[g] * 0.5 * geo.w;
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// Global lifts: a thread per (element, variable).
// ------------------------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(256) k_ns_lift(const __grid_constant__ KParams<P, double> kp,
                                                 const __grid_constant__ NsParams<P> ns, const double* __restrict__ U) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  const MeshDev& m = kp.m;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int e = (int)(t >> 2), w = (int)(t & 3);
  if (e >= m.ne) return;
  const int inst = m.n_inst > 1 ? m.inst[e] : 0;
  if (!kp.ic[inst].active) return;
  const size_t ld = m.ld;
  const double* Ue = U + (size_t)e * NEQ * NB;
  const double J = m.jac[e];
  double lx[NB], ly[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) lx[b] = ly[b] = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int fw = m.face[k * ld + e];
    const int slot = fw >> 1;
    if (slot < m.n_int) {
      // the neighbour and normal of the reference's test on the edge's first in-cell index
      const int ic = m.ie_ic[slot];
      const int2 lr = m.ie_lr[slot];
      const double4 geo = m.ie_geo[slot];
      const bool first = (ic & 3) == k;
      const int iric = first ? (ic >> 2) : (ic & 3);
      const int nbe = first ? lr.y : lr.x;
      const double nx = first ? geo.x : -geo.x, ny = first ? geo.y : -geo.y;
      const double* Un = U + (size_t)nbe * NEQ * NB + w * NB;
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        double lv = 0.0, rv = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          lv += Ue[w * NB + b] * kp.d.phi_edge[k][g][b];
          rv += Un[b] * kp.d.phi_edge[iric][NG - 1 - g][b];
        }
        const double jump_x = (lv - rv) * nx, jump_y = (lv - rv) * ny;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          lx[b] -= 0.5 * jump_x * kp.d.phi_edge[k][g][b] * kp.d.edge_w[g] * 0.5 * geo.w;
          ly[b] -= 0.5 * jump_y * kp.d.phi_edge[k][g][b] * kp.d.edge_w[g] * 0.5 * geo.w;
        }
      }
    } else {
      // boundary face: its local lift, added whole (global_lift + local_lift); out of line, so
      // that the rare far-field arithmetic does not hold registers in the common path
      double llx[NB], lly[NB];
      ns_boundary_lift<P>(kp, Ue, slot - m.n_int, w, J, llx, lly);
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        lx[b] = lx[b] + llx[b];
        ly[b] = ly[b] + lly[b];
      }
    }
  }
  double* out = ns.lift + (size_t)e * 2 * NEQ * NB + w * NB;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    out[b] = lx[b] / (ns.mass[b] * 0.5 * J);
    out[NEQ * NB + b] = ly[b] / (ns.mass[b] * 0.5 * J);
  }
}

// ------------------------------------------------------------------------------------------
// Edge pass: four lanes per edge slot.  Lane w first evaluates, for variable w, the traces at
// every point of the edge, the local lifts of every mode and the gradient plus lift at every point
// (the work a point needs of all variables, done once per slot instead of once per point); the
// four lanes then exchange them by shuffles, and lane g < NG evaluates HLLC and the viscous fluxes
// at point g.  Every value is the same expression in the same order as in the reference's loops.
// ------------------------------------------------------------------------------------------
// Physical first derivatives of mode b at point g of local edge k (mesh.rs:115-127) with the
// element's inverse Jacobian (dxi/dx, dxi/dy, deta/dx, deta/dy).
template <int P>
__device__ __forceinline__ void ns_dphi_edge(const NsParams<P>& ns, int k, int g, int b, double xx, double xy,
                                             double ex, double ey, double& dx, double& dy) {
  dx = xx * ns.dphi_edge[k][g][b][0] + ex * ns.dphi_edge[k][g][b][1];
  dy = xy * ns.dphi_edge[k][g][b][0] + ey * ns.dphi_edge[k][g][b][1];
}

// The four lanes' values a[h] at point `me`: out[j] = lane j's a[me] (all lanes take part).
template <int NG>
__device__ __forceinline__ void ns_gather(unsigned int mask, const double (&a)[NG], int me, double out[4]) {
#pragma unroll
  for (int h = 0; h < NG; ++h)
#pragma unroll
    for (int j = 0; j < NEQ; ++j) {
      const double v = __shfl_sync(mask, a[h], j, 4);
      if (h == me) out[j] = v;
    }
}

constexpr int kNsEdgeThreads = 128;  // 32 slots per block

template <int P>
__global__ void __launch_bounds__(kNsEdgeThreads) k_edge_flux_ns(const __grid_constant__ KParams<P, double> kp,
                                                                 const __grid_constant__ NsParams<P> ns,
                                                                 const double* __restrict__ U, double* __restrict__ F) {
  using V = Variant<P>;
  constexpr int NB = V::NB, NG = V::NG;
  const MeshDev& m = kp.m;
  const Gas& gas = kp.gas;
  const size_t ld = m.ld;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if ((t >> 2) >= (long long)(m.n_int + m.n_bnd)) return;  // the slot's four lanes together
  const int s = (int)(t >> 2), w = (int)(t & 3);
  const unsigned int mask = 0xFu << (threadIdx.x & 28);     // the slot's four lanes
  double out[4];
  if (s < m.n_int) {  // integrate_over_edges_ns, spatial_disc.rs:212-348
    const int2 lr = m.ie_lr[s];
    const int inst = m.n_inst > 1 ? m.inst[lr.x] : 0;
    if (!kp.ic[inst].active) return;
    const int ic = m.ie_ic[s], ilic = ic & 3, iric = ic >> 2;
    const double4 geo = m.ie_geo[s];
    const double nx = geo.x, ny = geo.y, jd = geo.w;
    const double* UL = U + (size_t)lr.x * NEQ * NB + w * NB;
    const double* UR = U + (size_t)lr.y * NEQ * NB + w * NB;
    const double JL = m.jac[lr.x], JR = m.jac[lr.y];
    const double lxx = m.dinv[0 * ld + lr.x], lxy = m.dinv[1 * ld + lr.x], lex = m.dinv[2 * ld + lr.x],
                 ley = m.dinv[3 * ld + lr.x];
    const double rxx = m.dinv[0 * ld + lr.y], rxy = m.dinv[1 * ld + lr.y], rex = m.dinv[2 * ld + lr.y],
                 rey = m.dinv[3 * ld + lr.y];
    // variable w: traces at every point (the jumps of the local lifts)
    double tl[NG], tr[NG];
#pragma unroll
    for (int h = 0; h < NG; ++h) {
      double a = 0.0, c = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        a += UL[b] * kp.d.phi_edge[ilic][h][b];
        c += UR[b] * kp.d.phi_edge[iric][NG - 1 - h][b];
      }
      tl[h] = a;
      tr[h] = c;
    }
    // gradient and local lift of variable w at every point, each side (spatial_disc.rs:290-300,
    // 318-328); the right side at the reversed point
    double dxl[NG], dyl[NG], llx[NG], lly[NG], dxr[NG], dyr[NG], rlx[NG], rly[NG];
#pragma unroll
    for (int g = 0; g < NG; ++g) dxl[g] = dyl[g] = llx[g] = lly[g] = dxr[g] = dyr[g] = rlx[g] = rly[g] = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      double ax = 0.0, ay = 0.0, cx = 0.0, cy = 0.0;  // local lifts of mode b (:233-249)
#pragma unroll
      for (int h = 0; h < NG; ++h) {
        const double jump_x = (tl[h] - tr[h]) * nx, jump_y = (tl[h] - tr[h]) * ny;
        ax -= 0.5 * jump_x * kp.d.phi_edge[ilic][h][b] * kp.d.edge_w[h] * 0.5 * jd;
        ay -= 0.5 * jump_y * kp.d.phi_edge[ilic][h][b] * kp.d.edge_w[h] * 0.5 * jd;
        cx += 0.5 * jump_x * kp.d.phi_edge[iric][NG - 1 - h][b] * kp.d.edge_w[NG - 1 - h] * 0.5 * jd;
        cy += 0.5 * jump_y * kp.d.phi_edge[iric][NG - 1 - h][b] * kp.d.edge_w[NG - 1 - h] * 0.5 * jd;
      }
      ax /= ns.mass[b] * 0.5 * JL;
      ay /= ns.mass[b] * 0.5 * JL;
      cx /= ns.mass[b] * 0.5 * JR;
      cy /= ns.mass[b] * 0.5 * JR;
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        const int gr = NG - 1 - g;
        double dpx, dpy;
        ns_dphi_edge<P>(ns, ilic, g, b, lxx, lxy, lex, ley, dpx, dpy);
        dxl[g] += UL[b] * dpx;
        dyl[g] += UL[b] * dpy;
        llx[g] += 3.0 * ax * kp.d.phi_edge[ilic][g][b];
        lly[g] += 3.0 * ay * kp.d.phi_edge[ilic][g][b];
        ns_dphi_edge<P>(ns, iric, gr, b, rxx, rxy, rex, rey, dpx, dpy);
        dxr[g] += UR[b] * dpx;
        dyr[g] += UR[b] * dpy;
        rlx[g] += cx * kp.d.phi_edge[iric][gr][b];
        rly[g] += cy * kp.d.phi_edge[iric][gr][b];
      }
    }
    double gl_x[NG], gl_y[NG], gr_x[NG], gr_y[NG];
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      gl_x[g] = dxl[g] + llx[g];
      gl_y[g] = dyl[g] + lly[g];
      gr_x[g] = dxr[g] + rlx[g];
      gr_y[g] = dyr[g] + rly[g];
    }
    // lane g: every variable's values at point g
    double lv[4], rv[4], gxL[4], gyL[4], gxR[4], gyR[4];
    ns_gather<NG>(mask, tl, w, lv);
    ns_gather<NG>(mask, tr, w, rv);
    ns_gather<NG>(mask, gl_x, w, gxL);
    ns_gather<NG>(mask, gl_y, w, gyL);
    ns_gather<NG>(mask, gr_x, w, gxR);
    ns_gather<NG>(mask, gr_y, w, gyR);
    if (w >= NG) return;
    const int st = hllc<double>(lv, rv, nx, ny, gas, out);
    if (st != ST_OK) raise_status(kp.ctl, &kp.ic[inst], st, m.slot_ref[s]);
    const double muL = ns_viscosity(lv, gas, ns.rgas), muR = ns_viscosity(rv, gas, ns.rgas);
#pragma unroll
    for (int i = 0; i < NEQ; ++i) {
      double fv, gv, visc = 0.0;
      ns_viscous_row(i, lv, muL, ns.hp, gxL, gyL, fv, gv);
      visc = visc + 0.5 * (nx * fv + ny * gv);
      ns_viscous_row(i, rv, muR, ns.hp, gxR, gyR, fv, gv);
      visc = visc + 0.5 * (nx * fv + ny * gv);
      out[i] = (out[i] - visc) * geo.z;
    }
  } else {  // the boundary faces of apply_bc_ns, boundary_condition.rs:169-371
    const int sb = s - m.n_int;
    const int e = m.be_elem[sb];
    const int inst = m.n_inst > 1 ? m.inst[e] : 0;
    if (!kp.ic[inst].active) return;
    const int info = m.be_info[sb], ic = info & 3;
    const bool wall = ((info >> 2) & 1) == 0;
    const double4 geo = m.be_geo[sb];
    const double nx = geo.x, ny = geo.y, jd = geo.w;
    const double* Ue = U + (size_t)e * NEQ * NB;
    const double J = m.jac[e];
    const double xx = m.dinv[0 * ld + e], xy = m.dinv[1 * ld + e], ex = m.dinv[2 * ld + e], ey = m.dinv[3 * ld + e];
    // every variable's traces at every point (lane w evaluates variable w), and the far-field
    // states there
    double tw[NG];
#pragma unroll
    for (int h = 0; h < NG; ++h) {
      double a = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) a += Ue[w * NB + b] * kp.d.phi_edge[ic][h][b];
      tw[h] = a;
    }
    double tv[NG][4], qn[NG][4];
#pragma unroll
    for (int h = 0; h < NG; ++h) {
#pragma unroll
      for (int j = 0; j < NEQ; ++j) tv[h][j] = __shfl_sync(mask, tw[h], j, 4);
      if (!wall) far_field_state<double>(tv[h], nx, ny, m.patch_q[info >> 3], gas, qn[h]);
    }
    // variable w: local lift (wall :181-201, with the cell tables at the point index; far field
    // :264-302), gradient plus 3 x lift at every point
    double gxw[NG], gyw[NG], dx[NG], dy[NG], lx[NG], ly[NG];
#pragma unroll
    for (int g = 0; g < NG; ++g) dx[g] = dy[g] = lx[g] = ly[g] = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      double ax = 0.0, ay = 0.0;
      if (!wall || w > 0) {
#pragma unroll
        for (int h = 0; h < NG; ++h) {
          double comp;
          if (wall) {
            const double pressure =
                gas.gm1 * (tv[h][3] - 0.5 * (tv[h][1] * tv[h][1] + tv[h][2] * tv[h][2]) / tv[h][0]);
            comp = w == 3 ? tv[h][3] - pressure / gas.gm1 : tw[h];
            ax -= 0.5 * (comp * nx) * kp.t.phi_cell[h][b] * kp.d.cell_w[h] * 0.5 * J;
            ay -= 0.5 * (comp * ny) * kp.t.phi_cell[h][b] * kp.d.cell_w[h] * 0.5 * J;
          } else {
            const double qw = w == 0 ? qn[h][0] : w == 1 ? qn[h][1] : w == 2 ? qn[h][2] : qn[h][3];
            comp = tw[h] - qw;
            ax -= 0.5 * (comp * nx) * kp.d.phi_edge[ic][h][b] * kp.d.edge_w[h] * 0.5 * jd;
            ay -= 0.5 * (comp * ny) * kp.d.phi_edge[ic][h][b] * kp.d.edge_w[h] * 0.5 * jd;
          }
        }
        ax /= ns.mass[b] * 0.5 * J;
        ay /= ns.mass[b] * 0.5 * J;
      }
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        double dpx, dpy;
        ns_dphi_edge<P>(ns, ic, g, b, xx, xy, ex, ey, dpx, dpy);
        dx[g] += Ue[w * NB + b] * dpx;
        dy[g] += Ue[w * NB + b] * dpy;
        lx[g] += 3.0 * ax * kp.d.phi_edge[ic][g][b];
        ly[g] += 3.0 * ay * kp.d.phi_edge[ic][g][b];
      }
    }
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      gxw[g] = dx[g] + lx[g];
      gyw[g] = dy[g] + ly[g];
    }
    double gx[4], gy[4];
    ns_gather<NG>(mask, gxw, w, gx);
    ns_gather<NG>(mask, gyw, w, gy);
    if (w >= NG) return;
    double tg[4], qg[4];  // the trace and far-field state at this lane's point
#pragma unroll
    for (int h = 0; h < NG; ++h)
      if (h == w)
#pragma unroll
        for (int j = 0; j < NEQ; ++j) {
          tg[j] = tv[h][j];
          qg[j] = qn[h][j];
        }
    double inv[4];
    if (wall) {
      const double pressure = gas.gm1 * (tg[3] - 0.5 * (tg[1] * tg[1] + tg[2] * tg[2]) / tg[0]);
      inv[0] = 0.0;
      inv[1] = pressure * nx;
      inv[2] = pressure * ny;
      inv[3] = 0.0;
    } else {
      const double u_new = qg[1] / qg[0], v_new = qg[2] / qg[0];
      const double vn_new = u_new * nx + v_new * ny;
      const double p_new = gas.gm1 * (qg[3] - 0.5 * (qg[1] * qg[1] + qg[2] * qg[2]) / qg[0]);
      const double h_new = qg[3] + p_new;
      inv[0] = qg[0] * vn_new;
      inv[1] = qg[1] * vn_new + p_new * nx;
      inv[2] = qg[2] * vn_new + p_new * ny;
      inv[3] = h_new * vn_new;
    }
    const double mu = ns_viscosity(tg, gas, ns.rgas);
#pragma unroll
    for (int i = 0; i < NEQ; ++i) {
      double fv, gv;
      ns_viscous_row(i, tg, mu, ns.hp, gx, gy, fv, gv);
      out[i] = (inv[i] - (nx * fv + ny * gv)) * geo.z;
    }
  }
  store_flux<double>(F, (size_t)s, NG, w, out);
}

// ------------------------------------------------------------------------------------------
// Element pass: the Euler element pass (element_body) with the viscous volume term.
// ------------------------------------------------------------------------------------------
template <int P, int MODE>
__global__ void __launch_bounds__(256) k_element_ns(const __grid_constant__ KParams<P, double> kp,
                                                       const __grid_constant__ NsParams<P> ns,
                                                       const double* __restrict__ Uin, const double* Ubase,
                                                       const double* __restrict__ F, double* Uout,
                                                       const double* Rin, double* Rout) {
  using V = Variant<P>;
  using S = double;
  using T = double;
  constexpr int NB = V::NB, NQ = V::NQ, NG = V::NG;
  constexpr int STRIDE = Staged<NB, S>::kStride;
  __shared__ __align__(16) S s_rec[kElemMaxWarps][8 * STRIDE];
  Control* ctl = kp.ctl;
  if (blockIdx.x == 0 && threadIdx.x == 0) reset_limiter_pass(ctl);  // for the limiter pass that follows
  const MeshDev& m = kp.m;
  const int lane = threadIdx.x & 31;
  const int var = lane >> 3, i = lane & 7;
  const int e0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 8;
  const int e_raw = e0 + i;
  if (e0 >= m.ne) return;
  const int e = e_raw < m.ne ? e_raw : m.ne - 1;
  const int inst = m.n_inst > 1 ? m.inst[e] : 0;
  const bool valid = e_raw < m.ne && kp.ic[inst].active;
  const unsigned int keep = __ballot_sync(0xffffffffu, valid) & 0xffu;
  if (!keep) return;
  const size_t ld = m.ld;
  S* sbuf = s_rec[threadIdx.x >> 5];
  S* mine_rec = sbuf + i * STRIDE + var * NB;
  warp_load_records<NB, S>(Uin, e0, sbuf, lane);
  double u[NB], r[NB], lfx[NB], lfy[NB];
  const double* lift = ns.lift + (size_t)e * 2 * NEQ * NB + var * NB;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    u[b] = mine_rec[b];
    r[b] = 0.0;
    lfx[b] = lift[b];
    lfy[b] = lift[NEQ * NB + b];
  }
  const double J = m.jac[e];
  const double xx = m.dinv[0 * ld + e], xy = m.dinv[1 * ld + e], ex = m.dinv[2 * ld + e], ey = m.dinv[3 * ld + e];
  const double gm1 = kp.gas.gm1;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double mine = 0.0, dx = 0.0, dy = 0.0, lx = 0.0, ly = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      mine += u[b] * kp.t.phi_cell[q][b];
      dx += u[b] * (xx * kp.t.dxi[q][b] + ex * kp.t.deta[q][b]);
      dy += u[b] * (xy * kp.t.dxi[q][b] + ey * kp.t.deta[q][b]);
      lx += lfx[b] * kp.t.phi_cell[q][b];
      ly += lfy[b] * kp.t.phi_cell[q][b];
    }
    double uq[NEQ], gx[NEQ], gy[NEQ];
#pragma unroll
    for (int w = 0; w < NEQ; ++w) {
      uq[w] = __shfl_sync(0xffffffffu, mine, w * 8 + i);
      gx[w] = __shfl_sync(0xffffffffu, dx + lx, w * 8 + i);
      gy[w] = __shfl_sync(0xffffffffu, dy + ly, w * 8 + i);
    }
    double f[NEQ], g[NEQ];
    euler_flux<double>(uq, gm1, f, g);
    double fvis, gvis;
    ns_viscous_row(var, uq, ns_viscosity(uq, kp.gas, ns.rgas), ns.hp, gx, gy, fvis, gvis);
    const double fv = (var == 0 ? f[0] : var == 1 ? f[1] : var == 2 ? f[2] : f[3]) - fvis;
    const double gv = (var == 0 ? g[0] : var == 1 ? g[1] : var == 2 ? g[2] : g[3]) - gvis;
    const double sc = kp.t.cell_w[q] * 0.5 * J;
    const double fx = sc * (fv * xx + gv * xy);
    const double fe = sc * (fv * ex + gv * ey);
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
  if constexpr (MODE == 0) {
    warp_load_records<NB, S>(Rin, e0, sbuf, lane);
#pragma unroll
    for (int b = 0; b < NB; ++b) r[b] = T(mine_rec[b]) + r[b];
  }
#pragma unroll
  for (int b = 0; b < NB; ++b) r[b] = r[b] * kp.t.inv_mass[b] * inv_half_j;
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
      S out;
      if constexpr (MODE == 1) {
        out = u[b] + dt * r[b];
      } else if constexpr (MODE == 2) {
        out = S(0.75) * base[b] + S(0.25) * (u[b] + dt * r[b]);
      } else {
        out = S(1.0 / 3.0) * base[b] + S(2.0 / 3.0) * (u[b] + dt * r[b]);
      }
      mine_rec[b] = out;
    }
    warp_store_records<NB, S>(Uout, e0, sbuf, keep, lane);
  }
}

}  // namespace dgm
