// fdtd_adjoint.cuh -- adjoint-step arguments and helpers shared by the 2D TM
// and 3D adjoint kernels.
//
// Reverse step `it` of the reference (src/DeepGPR/lib/deepgpr_cpu.c:2054-2107):
//   receivers^T, source^T (waveform gradient), imaging condition,
//   (E CPML + E update)^T  -> lambda_H,  (H CPML + H update)^T -> lambda_E.
// The helpers here are the per-cell pieces of that step: the CPML adjoint
// weight (pml_weight), the transposed staggered differences near the grid
// ends (gather_back / gather_fwd), the per-face weight lookup (add_pml), the
// head of a reverse step at one cell (reverse_head) and the FP64 gradient fold
// (k_fold_acc64).  Every value is produced by exactly one thread, in the
// reference's summation order, so results do not depend on launch shapes.
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

// grad += (T) acc64 after the reverse loop.
template <typename T>
__global__ void k_fold_acc64(T* __restrict__ g, const double* __restrict__ acc, long long n) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x)
    g[w] = g[w] + T(acc[w]);
}

}  // namespace dg
