// fdtd_adjoint.cuh -- exact discrete adjoint as two deterministic gathers.
//
// Reverse step `it` of the reference (src/DeepGPR/lib/deepgpr_cpu.c:2054-2107):
//   receivers^T, source^T (waveform gradient), imaging condition,
//   (E CPML + E update)^T  -> lambda_H,  (H CPML + H update)^T -> lambda_E.
//
// Here one reverse step is two grid kernels:
//   k_adj_e(it): sums the staged source-gradient terms of step it; gathers
//                the transposed backward differences of the E channels into
//                lambda_H; then computes the H-CPML adjoint weights of step it
//                at its own cell (they only need the new lambda_H).
//   k_adj_h(it): imaging condition of step it (needs lambda_E before the
//                ce_hist scaling); lambda_E <- ce_hist lambda_E + gathers of
//                the H channels; then the head of step it-1 at its own cell:
//                receiver cotangents, staged source-gradient terms and the
//                E-CPML adjoint weights.
// A prologue launch of k_adj_h (PROLOGUE=true) performs that head for step
// nt-1.  Every value is produced by exactly one thread, in the reference's
// summation order, so the result is independent of the launch shape.
#pragma once

#include "fdtd_common.cuh"

namespace dg {

template <typename T> struct Phys;
template <> struct Phys<float> {
  static __device__ __forceinline__ float eps0() { return 8.8541878128e-12f; }
  static __device__ __forceinline__ float pec() { return 100.0f; }
};
template <> struct Phys<double> {
  static __device__ __forceinline__ double eps0() { return 8.8541878128e-12; }
  static __device__ __forceinline__ double pec() { return 100.0; }
};

template <typename T>
struct AdjArgs {
  Grid g;
  T dx, dy, dz;
  T inv_dx, inv_dy, inv_dz;         // 1/spacing as the reference forms it
  FixedDiv<T> ddt;                  // division by dt (imaging condition)
  FixedDiv<T> ddy, ddz;             // division by dy, dz (curl scaling c dx / d)
  int dy_eq, dz_eq;
  T *lEx, *lEy, *lEz, *lHx, *lHy, *lHz;
  const T *ce_hist, *ce_curl, *ce_rhs, *ch_curl, *ch_rhs;
  Face<T> eF[6], hF[6];             // psi = psi cotangents, w1/w2 = weight scratch
  int has_cpml;
  Control* ctrl;
  int k_in_chunk;                   // time step = ctrl->cur - k_in_chunk
  int nt;
  // receivers^T
  PointTable rcv;
  const T* data_grad;               // (nshot, nt, nrx)
  int rx_comp, nrx;
  // sources^T
  PointTable src;
  T* srcv;                          // (nshot, nsrc) staged terms of one step
  T* grad_source;                   // (nsrc, nt)
  int want_src, nsrc, src_comp;
  T src_geo;                        // dl / ((dx*dy)*dz)
  // imaging condition
  int want_eps, want_sig, acc64;
  T* g_eps;
  T* g_sig;
  double* g_eps64;
  double* g_sig64;
  const T* sigma;
  T dt;
  int S, mode, kind, e_only, nt_saved;
  HBox box;
  long long frame, comp_stride;
  const void* E_saved;
  const void* R_saved;
  const float* e_scales;
  const float* r_scales;
  int ntiles;
};

// Adjoint of one CPML auxiliary update (deepgpr_cpu.c:518-527): returns the
// transposed-curl weight and advances the psi cotangent.
template <typename T>
__device__ __forceinline__ T pml_weight(T lam, T inv_h, T up, T sign, const Prof<T>& pr, T* lpsi) {
  const T ph = *lpsi;
  const T w = (sign * up * pr.ra1 * lam - pr.rf * ph) * inv_h;
  *lpsi = sign * up * pr.rb * lam + pr.re * ph;
  return w;
}

// Transpose of d_back gathered at target coordinate c (deepgpr_cpu.c:429-467).
// W(d) returns the channel weight of the source point at offset d.
// Full-radius form: every source point of the target is inside the grid.
template <typename T, int R, typename WF>
__device__ __forceinline__ T gather_back_full(const WF& W) {
  if (R == 1) {
    T acc = W(0);
    acc -= W(1);
    return acc;
  }
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    const T t = tap<T>(R, r);
    acc += t * W(-(r - 1));
    acc -= t * W(r);
  }
  return acc;
}

template <typename T, int R, typename WF>
__device__ __forceinline__ T gather_back(const WF& W, int c, int n) {
  if (R == 1) {
    T acc = W(0);
    if (c + 1 < n) acc -= W(1);
    return acc;
  }
  if (c >= 2 * R - 1 && c + 2 * R - 1 < n) return gather_back_full<T, R>(W);
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    const int up = c - (r - 1);
    if (up >= 0) {
      const int rr = rad_back(up, n, R);
      if (r <= rr) acc += tap<T>(rr, r) * W(-(r - 1));
    }
    const int dn = c + r;
    if (dn < n) {
      const int rr = rad_back(dn, n, R);
      if (r <= rr) acc -= tap<T>(rr, r) * W(r);
    }
  }
  return acc;
}

// Transpose of d_fwd gathered at target coordinate c (deepgpr_cpu.c:470-507).
template <typename T, int R, typename WF>
__device__ __forceinline__ T gather_fwd_full(const WF& W) {
  if (R == 1) {
    T acc = T(0);
    acc += W(-1);
    acc -= W(0);
    return acc;
  }
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    const T t = tap<T>(R, r);
    acc += t * W(-r);
    acc -= t * W(r - 1);
  }
  return acc;
}

template <typename T, int R, typename WF>
__device__ __forceinline__ T gather_fwd(const WF& W, int c, int n) {
  if (R == 1) {
    T acc = T(0);
    if (c >= 1) acc += W(-1);
    acc -= W(0);
    return acc;
  }
  if (c >= 2 * R - 1 && c + 2 * R <= n) return gather_fwd_full<T, R>(W);
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    const int up = c - r;
    if (up >= 0) {
      const int rr = rad_fwd(up, n, R);
      if (r <= rr) acc += tap<T>(rr, r) * W(-r);
    }
    const int dn = c + (r - 1);
    if (dn < n) {
      const int rr = rad_fwd(dn, n, R);
      if (r <= rr) acc -= tap<T>(rr, r) * W(r - 1);
    }
  }
  return acc;
}

template <typename T>
__device__ __forceinline__ T scaled(T c1, T dx, T d, int eq) {
  return eq ? c1 : c1 * dx / d;
}

// CPML part of a channel weight at a source point: faces f_lo then f_hi of
// one axis, slot `slot`, in the reference's summation order.
template <typename T, bool EFACE>
__device__ __forceinline__ void add_pml(T& w, const Face<T>& Flo, const Face<T>& Fhi, const Grid& g, int axis,
                                        int slot, int s, int i, int j, int k) {
  const int c = axis == 0 ? i : (axis == 1 ? j : k);
  const int n = axis == 0 ? g.NX : (axis == 1 ? g.NY : g.NZ);
  if (EFACE && c == 0) return;
  const int q0 = EFACE ? q_low_e(Flo.p, c) : q_low_h(Flo.p, c);
  if (q0 >= 0) {
    const PsiDims d = EFACE ? psi_dims_e(g, axis, slot, Flo.p) : psi_dims_h(g, axis, slot, Flo.p);
    w += (slot == 1 ? Flo.w1 : Flo.w2)[psi_index(d, axis, s, q0, i, j, k)];
  }
  const int q1 = q_high(Fhi.p, c, n);
  if (q1 >= 0) {
    const PsiDims d = EFACE ? psi_dims_e(g, axis, slot, Fhi.p) : psi_dims_h(g, axis, slot, Fhi.p);
    w += (slot == 1 ? Fhi.w1 : Fhi.w2)[psi_index(d, axis, s, q1, i, j, k)];
  }
}

// ---------------------------------------------------------------------------
// k_adj_e: lambda_H += curl^T of the E channels; H-CPML weights of step it.
// Channels (source = E cell): A_X = -c lambda_ey, A_Y = c_y lambda_ex -> lambda_hz;
// B_X = c lambda_ez, B_Z = -c_z lambda_ex -> lambda_hy; C_Y = -c_y lambda_ez,
// C_Z = c_z lambda_ey -> lambda_hx (deepgpr_cpu.c:1236-1270).
// ---------------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(kBlock) k_adj_e(AdjArgs<T> a) {
  const Grid& g = a.g;
  const int it = a.ctrl->cur - a.k_in_chunk;
  if (a.want_src && blockIdx.x == 0 && blockIdx.y == 0) {
    // waveform gradient of step it: shots summed in order (deepgpr_cpu.c:1524-1533)
    for (int m = threadIdx.x; m < a.nsrc; m += blockDim.x) {
      T acc = a.grad_source[(long long)m * a.nt + it];
      for (int s = 0; s < g.nshot; ++s) acc += a.srcv[(long long)s * a.nsrc + m];
      a.grad_source[(long long)m * a.nt + it] = acc;
    }
  }
  const int c = blockIdx.x * kBlock + threadIdx.x;
  if (c >= g.cells) return;
  int i, j, k;
  cell_ijk(g, c, i, j, k);
  const bool pml = a.has_cpml != 0;
  const int sx = g.sx, sy = g.NZ;
  int qh[6] = {-1, -1, -1, -1, -1, -1};
  bool any_h = false;
  T up_h = T(0);
  if (pml) {
    qh[0] = q_low_h(a.hF[0].p, i);
    qh[1] = q_high(a.hF[1].p, i, g.NX);
    qh[2] = q_low_h(a.hF[2].p, j);
    qh[3] = q_high(a.hF[3].p, j, g.NY);
    qh[4] = q_low_h(a.hF[4].p, k);
    qh[5] = q_high(a.hF[5].p, k, g.NZ);
    any_h = qh[0] >= 0 || qh[1] >= 0 || qh[2] >= 0 || qh[3] >= 0 || qh[4] >= 0 || qh[5] >= 0;
    if (any_h) up_h = a.ch_rhs[c];
  }
  const int s0 = blockIdx.y * g.shots_per_group;
  const int s1 = min(s0 + g.shots_per_group, g.nshot);
  for (int s = s0; s < s1; ++s) {
    const long long base = (long long)s * g.cells + c;
    const T* lex = a.lEx + base;
    const T* ley = a.lEy + base;
    const T* lez = a.lEz + base;
    auto wAX = [&](int d) -> T {
      const int x = i + d;
      T w = T(0);
      if (pml && j < g.NY - 1) add_pml<T, true>(w, a.eF[0], a.eF[1], g, 0, 1, s, x, j, k);
      if (upd_ey(g, x, j, k)) w += (-a.ce_curl[c + d * sx]) * ley[(long long)d * sx];
      return w;
    };
    auto wBX = [&](int d) -> T {
      const int x = i + d;
      T w = T(0);
      if (pml && k < g.NZ - 1) add_pml<T, true>(w, a.eF[0], a.eF[1], g, 0, 2, s, x, j, k);
      if (upd_ez(g, x, j, k)) w += a.ce_curl[c + d * sx] * lez[(long long)d * sx];
      return w;
    };
    auto wAY = [&](int d) -> T {
      const int y = j + d;
      T w = T(0);
      if (pml && i < g.NX - 1) add_pml<T, true>(w, a.eF[2], a.eF[3], g, 1, 1, s, i, y, k);
      if (upd_ex(g, i, y, k)) w += scaled(a.ce_curl[c + d * sy], a.dx, a.dy, a.dy_eq) * lex[d * sy];
      return w;
    };
    auto wCY = [&](int d) -> T {
      const int y = j + d;
      T w = T(0);
      if (pml && k < g.NZ - 1) add_pml<T, true>(w, a.eF[2], a.eF[3], g, 1, 2, s, i, y, k);
      if (upd_ez(g, i, y, k)) w += (-scaled(a.ce_curl[c + d * sy], a.dx, a.dy, a.dy_eq)) * lez[d * sy];
      return w;
    };
    auto wBZ = [&](int d) -> T {
      const int z = k + d;
      T w = T(0);
      if (pml && i < g.NX - 1) add_pml<T, true>(w, a.eF[4], a.eF[5], g, 2, 1, s, i, j, z);
      if (upd_ex(g, i, j, z)) w += (-scaled(a.ce_curl[c + d], a.dx, a.dz, a.dz_eq)) * lex[d];
      return w;
    };
    auto wCZ = [&](int d) -> T {
      const int z = k + d;
      T w = T(0);
      if (pml && j < g.NY - 1) add_pml<T, true>(w, a.eF[4], a.eF[5], g, 2, 2, s, i, j, z);
      if (upd_ey(g, i, j, z)) w += scaled(a.ce_curl[c + d], a.dx, a.dz, a.dz_eq) * ley[d];
      return w;
    };
    T hx = a.lHx[base], hy = a.lHy[base], hz = a.lHz[base];
    hz += gather_back<T, R>(wAX, i, g.NX);
    hz += gather_back<T, R>(wAY, j, g.NY);
    hy += gather_back<T, R>(wBX, i, g.NX);
    hy += gather_back<T, R>(wBZ, k, g.NZ);
    hx += gather_back<T, R>(wCY, j, g.NY);
    hx += gather_back<T, R>(wCZ, k, g.NZ);
    a.lHx[base] = hx;
    a.lHy[base] = hy;
    a.lHz[base] = hz;
    if (any_h) {
      // H-CPML adjoint weights of step it (deepgpr_cpu.c:1331-1396)
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int q = qh[f];
        if (q < 0) continue;
        const Face<T>& F = a.hF[f];
        const Prof<T> pr = prof(F, q);
        const int axis = f >> 1;
        if (axis == 0) {
          if (k < g.NZ - 1) {
            const long long pi = psi_index(psi_dims_h(g, 0, 1, F.p), 0, s, q, i, j, k);
            F.w1[pi] = pml_weight(hy, a.inv_dx, up_h, T(1), pr, &F.psi1[pi]);
          }
          if (j < g.NY - 1) {
            const long long pi = psi_index(psi_dims_h(g, 0, 2, F.p), 0, s, q, i, j, k);
            F.w2[pi] = pml_weight(hz, a.inv_dx, up_h, T(-1), pr, &F.psi2[pi]);
          }
        } else if (axis == 1) {
          if (k < g.NZ - 1) {
            const long long pi = psi_index(psi_dims_h(g, 1, 1, F.p), 1, s, q, i, j, k);
            F.w1[pi] = pml_weight(hx, a.inv_dy, up_h, T(-1), pr, &F.psi1[pi]);
          }
          if (i < g.NX - 1) {
            const long long pi = psi_index(psi_dims_h(g, 1, 2, F.p), 1, s, q, i, j, k);
            F.w2[pi] = pml_weight(hz, a.inv_dy, up_h, T(1), pr, &F.psi2[pi]);
          }
        } else {
          if (j < g.NY - 1) {
            const long long pi = psi_index(psi_dims_h(g, 2, 1, F.p), 2, s, q, i, j, k);
            F.w1[pi] = pml_weight(hx, a.inv_dz, up_h, T(1), pr, &F.psi1[pi]);
          }
          if (i < g.NX - 1) {
            const long long pi = psi_index(psi_dims_h(g, 2, 2, F.p), 2, s, q, i, j, k);
            F.w2[pi] = pml_weight(hy, a.inv_dz, up_h, T(-1), pr, &F.psi2[pi]);
          }
        }
      }
    }
  }
}

// Head of reverse step `st` at one cell: receiver cotangents, staged source
// terms and E-CPML adjoint weights (deepgpr_cpu.c:1479-1534, 1155-1234).
template <typename T>
__device__ __forceinline__ void reverse_head(const AdjArgs<T>& a, int st, int s, int c, int i, int j, int k,
                                             int rrow, int srow, T& ex, T& ey, T& ez, const int* qe, bool any_e,
                                             T up_e) {
  const Grid& g = a.g;
  if (rrow >= 0) {
    for (int e = a.rcv.off[rrow]; e < a.rcv.off[rrow + 1]; ++e) {
      if (a.rcv.shot[e] != s) continue;
      const T d = a.data_grad[((long long)s * a.nt + st) * a.nrx + a.rcv.idx[e]];
      if (a.rx_comp == 0) ex += d;
      else if (a.rx_comp == 1) ey += d;
      else ez += d;
    }
  }
  if (a.want_src && srow >= 0) {
    const T lam = a.src_comp == 0 ? ex : (a.src_comp == 1 ? ey : ez);
    for (int e = a.src.off[srow]; e < a.src.off[srow + 1]; ++e)
      if (a.src.shot[e] == s) a.srcv[(long long)s * a.nsrc + a.src.idx[e]] = -a.ce_rhs[c] * a.src_geo * lam;
  }
  if (any_e) {
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int q = qe[f];
      if (q < 0) continue;
      const Face<T>& F = a.eF[f];
      const Prof<T> pr = prof(F, q);
      const int axis = f >> 1;
      if (axis == 0) {
        if (j < g.NY - 1) {
          const long long pi = psi_index(psi_dims_e(g, 0, 1, F.p), 0, s, q, i, j, k);
          F.w1[pi] = pml_weight(ey, a.inv_dx, up_e, T(-1), pr, &F.psi1[pi]);
        }
        if (k < g.NZ - 1) {
          const long long pi = psi_index(psi_dims_e(g, 0, 2, F.p), 0, s, q, i, j, k);
          F.w2[pi] = pml_weight(ez, a.inv_dx, up_e, T(1), pr, &F.psi2[pi]);
        }
      } else if (axis == 1) {
        if (i < g.NX - 1) {
          const long long pi = psi_index(psi_dims_e(g, 1, 1, F.p), 1, s, q, i, j, k);
          F.w1[pi] = pml_weight(ex, a.inv_dy, up_e, T(1), pr, &F.psi1[pi]);
        }
        if (k < g.NZ - 1) {
          const long long pi = psi_index(psi_dims_e(g, 1, 2, F.p), 1, s, q, i, j, k);
          F.w2[pi] = pml_weight(ez, a.inv_dy, up_e, T(-1), pr, &F.psi2[pi]);
        }
      } else {
        if (i < g.NX - 1) {
          const long long pi = psi_index(psi_dims_e(g, 2, 1, F.p), 2, s, q, i, j, k);
          F.w1[pi] = pml_weight(ex, a.inv_dz, up_e, T(-1), pr, &F.psi1[pi]);
        }
        if (j < g.NY - 1) {
          const long long pi = psi_index(psi_dims_e(g, 2, 2, F.p), 2, s, q, i, j, k);
          F.w2[pi] = pml_weight(ey, a.inv_dz, up_e, T(1), pr, &F.psi2[pi]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// k_adj_h: imaging of step it, lambda_E update, head of step it-1.
// H channels (source = H cell): A_X = c lambda_hy, A_Y = -c_y lambda_hx -> lambda_ez;
// B_X = -c lambda_hz, B_Z = c_z lambda_hx -> lambda_ey; C_Y = c_y lambda_hz,
// C_Z = -c_z lambda_hy -> lambda_ex (deepgpr_cpu.c:1400-1424).
// ---------------------------------------------------------------------------
template <typename T, int R, bool PROLOGUE>
__global__ void __launch_bounds__(kBlock) k_adj_h(AdjArgs<T> a) {
  __shared__ int smap[kBlock];
  __shared__ int rmap[kBlock];
  const Grid& g = a.g;
  const int c0 = blockIdx.x * kBlock;
  const int c = c0 + threadIdx.x;
  build_block_map(a.src, c0, smap);
  build_block_map(a.rcv, c0, rmap);
  if (c >= g.cells) return;
  const int srow = a.want_src ? smap[threadIdx.x] : -1;
  const int rrow = rmap[threadIdx.x];
  const int it = a.ctrl->cur - a.k_in_chunk;
  const int head = PROLOGUE ? it : it - 1;
  int i, j, k;
  cell_ijk(g, c, i, j, k);
  const bool pml = a.has_cpml != 0;
  const int sx = g.sx, sy = g.NZ;

  // imaging condition setup (deepgpr_cpu.c:1659-1745)
  const bool want_model = (a.want_eps || a.want_sig) && !PROLOGUE;
  const bool image = want_model && (it % a.S == 0);
  const int slot = it / a.S;
  long long h = 0;
  const bool inbox = image && in_box(a.box, i, j, k, h);
  T ca = T(0), cbv = T(0), wgt = T(0), dca_e = T(0), dcb_e = T(0), dca_s = T(0), dcb_s = T(0);
  bool pec_ok = false;
  if (inbox) {
    ca = a.ce_hist[c];
    cbv = a.ce_rhs[c];
    int w = a.S;
    if (it + w > a.nt) w = a.nt - it;
    wgt = T(w);
    pec_ok = a.sigma[c] <= Phys<T>::pec();
    dca_e = div_fixed(Phys<T>::eps0() * (T(1) - ca) * cbv, a.ddt);
    dcb_e = div_fixed(-Phys<T>::eps0() * cbv * cbv, a.ddt);
    dca_s = T(-0.5) * (T(1) + ca) * cbv;
    dcb_s = T(-0.5) * cbv * cbv;
  }
  T loc_e = T(0), loc_s = T(0);
  double loc_e64 = 0.0, loc_s64 = 0.0;

  const bool dex = upd_ex(g, i, j, k), dey = upd_ey(g, i, j, k), dez = upd_ez(g, i, j, k);
  const T chist = a.ce_hist[c];
  int qe[6] = {-1, -1, -1, -1, -1, -1};
  bool any_e = false;
  T up_e = T(0);
  if (pml && head >= 0) {
    qe[0] = i > 0 ? q_low_e(a.eF[0].p, i) : -1;
    qe[1] = i > 0 ? q_high(a.eF[1].p, i, g.NX) : -1;
    qe[2] = j > 0 ? q_low_e(a.eF[2].p, j) : -1;
    qe[3] = j > 0 ? q_high(a.eF[3].p, j, g.NY) : -1;
    qe[4] = k > 0 ? q_low_e(a.eF[4].p, k) : -1;
    qe[5] = k > 0 ? q_high(a.eF[5].p, k, g.NZ) : -1;
    any_e = qe[0] >= 0 || qe[1] >= 0 || qe[2] >= 0 || qe[3] >= 0 || qe[4] >= 0 || qe[5] >= 0;
    if (any_e) up_e = a.ce_rhs[c];
  }
  const int ncomp = a.mode == 3 ? 3 : 1;
  const long long bc = a.box.cells();

  const int s0 = blockIdx.y * g.shots_per_group;
  const int s1 = min(s0 + g.shots_per_group, g.nshot);
  for (int s = s0; s < s1; ++s) {
    const long long base = (long long)s * g.cells + c;
    T ex = a.lEx[base], ey = a.lEy[base], ez = a.lEz[base];
    if (inbox) {
      const T lam3[3] = {ex, ey, ez};
      for (int q = 0; q < ncomp; ++q) {
        const int fc = a.mode == 3 ? q : 2;
        const bool du = fc == 0 ? dex : (fc == 1 ? dey : dez);
        const long long hi = q * a.comp_stride + slot * a.frame + s * bc + h;
        const int tile = c / kBlock;
        float esc = 1.0f, rsc = 1.0f;
        if (a.kind == kFP8) {
          esc = a.e_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + tile];
          if (!a.e_only) rsc = a.r_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + tile];
        }
        const T eo = hist_load<T>(a.E_saved, hi, a.kind, esc);
        T rhs;
        if (!a.e_only) {
          rhs = hist_load<T>(a.R_saved, hi, a.kind, rsc);
        } else {
          const T nxt = slot + 1 < a.nt_saved ? hist_load<T>(a.E_saved, hi + a.frame, a.kind, 1.0f)
                                              : hist_load<T>(a.R_saved, q * a.frame + s * bc + h, a.kind, 1.0f);
          const T aeff = du ? ca : T(1);
          rhs = cbv != T(0) ? (nxt - aeff * eo) / cbv : T(0);
        }
        T lam = lam3[fc];
        if (eo == T(0) && rhs == T(0)) lam = T(0);
        const T gca = du ? lam * eo * wgt : T(0);
        const T gcb = lam * rhs * wgt;
        if (pec_ok) {
          if (a.want_eps) {
            const T term = gca * dca_e + gcb * dcb_e;
            if (a.acc64) loc_e64 += double(term); else loc_e += term;
          }
          if (a.want_sig) {
            const T term = gca * dca_s + gcb * dcb_s;
            if (a.acc64) loc_s64 += double(term); else loc_s += term;
          }
        }
      }
    }
    if (!PROLOGUE) {
      if (dex) ex = chist * ex;
      if (dey) ey = chist * ey;
      if (dez) ez = chist * ez;
      const T* lhx = a.lHx + base;
      const T* lhy = a.lHy + base;
      const T* lhz = a.lHz + base;
      auto wAX = [&](int d) -> T {
        const int x = i + d;
        T w = T(0);
        if (pml && k < g.NZ - 1) add_pml<T, false>(w, a.hF[0], a.hF[1], g, 0, 1, s, x, j, k);
        if (upd_hy(g, x, j, k)) w += a.ch_curl[c + d * sx] * lhy[(long long)d * sx];
        return w;
      };
      auto wBX = [&](int d) -> T {
        const int x = i + d;
        T w = T(0);
        if (pml && j < g.NY - 1) add_pml<T, false>(w, a.hF[0], a.hF[1], g, 0, 2, s, x, j, k);
        if (upd_hz(g, x, j, k)) w += (-a.ch_curl[c + d * sx]) * lhz[(long long)d * sx];
        return w;
      };
      auto wAY = [&](int d) -> T {
        const int y = j + d;
        T w = T(0);
        if (pml && k < g.NZ - 1) add_pml<T, false>(w, a.hF[2], a.hF[3], g, 1, 1, s, i, y, k);
        if (upd_hx(g, i, y, k)) w += (-scaled(a.ch_curl[c + d * sy], a.dx, a.dy, a.dy_eq)) * lhx[d * sy];
        return w;
      };
      auto wCY = [&](int d) -> T {
        const int y = j + d;
        T w = T(0);
        if (pml && i < g.NX - 1) add_pml<T, false>(w, a.hF[2], a.hF[3], g, 1, 2, s, i, y, k);
        if (upd_hz(g, i, y, k)) w += scaled(a.ch_curl[c + d * sy], a.dx, a.dy, a.dy_eq) * lhz[d * sy];
        return w;
      };
      auto wBZ = [&](int d) -> T {
        const int z = k + d;
        T w = T(0);
        if (pml && j < g.NY - 1) add_pml<T, false>(w, a.hF[4], a.hF[5], g, 2, 1, s, i, j, z);
        if (upd_hx(g, i, j, z)) w += scaled(a.ch_curl[c + d], a.dx, a.dz, a.dz_eq) * lhx[d];
        return w;
      };
      auto wCZ = [&](int d) -> T {
        const int z = k + d;
        T w = T(0);
        if (pml && i < g.NX - 1) add_pml<T, false>(w, a.hF[4], a.hF[5], g, 2, 2, s, i, j, z);
        if (upd_hy(g, i, j, z)) w += (-scaled(a.ch_curl[c + d], a.dx, a.dz, a.dz_eq)) * lhy[d];
        return w;
      };
      ez += gather_fwd<T, R>(wAX, i, g.NX);
      ez += gather_fwd<T, R>(wAY, j, g.NY);
      ey += gather_fwd<T, R>(wBX, i, g.NX);
      ey += gather_fwd<T, R>(wBZ, k, g.NZ);
      ex += gather_fwd<T, R>(wCY, j, g.NY);
      ex += gather_fwd<T, R>(wCZ, k, g.NZ);
    }
    if (head >= 0) reverse_head(a, head, s, c, i, j, k, rrow, srow, ex, ey, ez, qe, any_e, up_e);
    a.lEx[base] = ex;
    a.lEy[base] = ey;
    a.lEz[base] = ez;
  }
  if (inbox) {
    const long long gi = ((long long)i * (g.NY - 1) + j) * (g.NZ - 1) + k;
    if (a.want_eps) {
      if (a.acc64) a.g_eps64[gi] += loc_e64; else a.g_eps[gi] += loc_e;
    }
    if (a.want_sig) {
      if (a.acc64) a.g_sig64[gi] += loc_s64; else a.g_sig[gi] += loc_s;
    }
  }
}

// grad += (T) acc64 after the reverse loop.
template <typename T>
__global__ void k_fold_acc64(T* __restrict__ g, const double* __restrict__ acc, long long n) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x)
    g[w] = g[w] + T(acc[w]);
}

}  // namespace dg
