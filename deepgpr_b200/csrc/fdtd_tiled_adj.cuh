// fdtd_tiled_adj.cuh -- adjoint pieces shared by the 2D and 3D kernels.
//
// The argument block of the adjoint kernels (TiledAdj), gather wrappers, the
// per-cell head of a reverse step (receiver cotangents and staged source
// terms through the point bitmaps; E-CPML adjoint weights), and the general
// one-thread-per-cell imaging kernel k_image (used for history boxes of
// 2^31 cells or more; k3_image covers the rest).  The per-cell arithmetic is
// that of fdtd_adjoint.cuh (reference: src/DeepGPR/lib/deepgpr_cpu.c:1112-1534,
// 1659-1745).
#pragma once

#include "fdtd_adjoint.cuh"
#include "fdtd_tiled.cuh"

namespace dg {

template <typename T>
struct TiledAdj {
  AdjArgs<T> a;
  PointSet src, rcv;
  int xchunk;
};

// Gathers on an accessor W(d) = weight of the source at offset d.
template <typename T, int R, typename WF>
__device__ __forceinline__ T gback(const WF& W, int c, int n) {
  return gather_back<T, R>(W, c, n);
}
template <typename T, int R, typename WF>
__device__ __forceinline__ T gfwd(const WF& W, int c, int n) {
  return gather_fwd<T, R>(W, c, n);
}

// Head of reverse step st at one cell, bitmap-driven variant of reverse_head.
template <typename T>
__device__ __forceinline__ void tiled_head(const TiledAdj<T>& P, int st, int s, int c, T& ex, T& ey, T& ez) {
  const AdjArgs<T>& a = P.a;
  if (point_hit(P.rcv, s, c)) {
    const int row = point_row(P.rcv, c);
    for (int e = a.rcv.off[row]; e < a.rcv.off[row + 1]; ++e) {
      if (a.rcv.shot[e] != s) continue;
      const T d = a.data_grad[((long long)s * a.nt + st) * a.nrx + a.rcv.idx[e]];
      if (a.rx_comp == 0) ex += d;
      else if (a.rx_comp == 1) ey += d;
      else ez += d;
    }
  }
  if (a.want_src && point_hit(P.src, s, c)) {
    const int row = point_row(P.src, c);
    const T lam = a.src_comp == 0 ? ex : (a.src_comp == 1 ? ey : ez);
    for (int e = a.src.off[row]; e < a.src.off[row + 1]; ++e)
      if (a.src.shot[e] == s) a.srcv[(long long)s * a.nsrc + a.src.idx[e]] = -a.ce_rhs[c] * a.src_geo * lam;
  }
}

// E-CPML adjoint weights of a cell for the next reverse step.
template <typename T>
__device__ __forceinline__ void e_pml_head(const AdjArgs<T>& a, int s, int i, int j, int k, int c, T ex, T ey,
                                           T ez) {
  const Grid& g = a.g;
  int qe[6];
  qe[0] = i > 0 ? q_low_e(a.eF[0].p, i) : -1;
  qe[1] = i > 0 ? q_high(a.eF[1].p, i, g.NX) : -1;
  qe[2] = j > 0 ? q_low_e(a.eF[2].p, j) : -1;
  qe[3] = j > 0 ? q_high(a.eF[3].p, j, g.NY) : -1;
  qe[4] = k > 0 ? q_low_e(a.eF[4].p, k) : -1;
  qe[5] = k > 0 ? q_high(a.eF[5].p, k, g.NZ) : -1;
  if (qe[0] < 0 && qe[1] < 0 && qe[2] < 0 && qe[3] < 0 && qe[4] < 0 && qe[5] < 0) return;
  const T up_e = a.ce_rhs[c];
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

// ---------------------------------------------------------------------------
// Imaging condition of one saved step (deepgpr_cpu.c:1659-1745).
// One thread per history-box cell; shots and components summed inside the
// thread in the reference's order.  lam_* point at lambda_E before the
// ce_hist scaling of this step, element (s, i, j, k) at
// s * ls + i * lp + j * lr + k.  3D grids (the 2D TM path uses tm_image).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_image(AdjArgs<T> a, const T* lam_x, const T* lam_y, const T* lam_z,
                                               long long ls, int lp, int lr) {
  const Grid& g = a.g;
  const int it = a.ctrl->cur - a.k_in_chunk;
  if (it % a.S != 0) return;
  const int slot = it / a.S;
  const long long bc = a.box.cells();
  const long long hidx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (hidx >= bc) return;
  const int hi = int(hidx / ((long long)a.box.ny * a.box.nz));
  const int rem = int(hidx % ((long long)a.box.ny * a.box.nz));
  const int i = hi + a.box.x0, j = rem / a.box.nz + a.box.y0, k = rem % a.box.nz + a.box.z0;
  const int c = i * g.sx + j * g.NZ + k;
  const long long cl = (long long)i * lp + (long long)j * lr + k;
  const T ca = a.ce_hist[c], cbv = a.ce_rhs[c];
  int w = a.S;
  if (it + w > a.nt) w = a.nt - it;
  const T wgt = T(w);
  const bool pec_ok = a.sigma[c] <= Phys<T>::pec();
  const T dca_e = div_fixed(Phys<T>::eps0() * (T(1) - ca) * cbv, a.ddt);
  const T dcb_e = div_fixed(-Phys<T>::eps0() * cbv * cbv, a.ddt);
  const FixedDiv<T> dcb = fixed_div_dev(cbv);   // shared by the shots
  const T dca_s = T(-0.5) * (T(1) + ca) * cbv;
  const T dcb_s = T(-0.5) * cbv * cbv;
  const bool dex = upd_ex(g, i, j, k), dey = upd_ey(g, i, j, k), dez = upd_ez(g, i, j, k);
  const int ncomp = a.mode == 3 ? 3 : 1;
  const long long tile = fp8_tile3(g, i, j, k);
  T loc_e = T(0), loc_s = T(0);
  double loc_e64 = 0.0, loc_s64 = 0.0;
  for (int s = 0; s < g.nshot; ++s) {
    const long long lf = (long long)s * ls + cl;
    for (int q = 0; q < ncomp; ++q) {
      const int fc = a.mode == 3 ? q : 2;
      const bool du = fc == 0 ? dex : (fc == 1 ? dey : dez);
      const long long hix = q * a.comp_stride + slot * a.frame + s * bc + hidx;
      float esc = 1.0f, rsc = 1.0f;
      if (is_tiled(a.kind)) {
        const long long si = (((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + tile;
        esc = a.e_scales[si];
        if (!a.e_only) rsc = a.r_scales[si];
      }
      const T eo = hist_load<T>(a.E_saved, hix, a.kind, esc);
      T rhs;
      if (!a.e_only) {
        rhs = hist_load<T>(a.R_saved, hix, a.kind, rsc);
      } else {
        const T nxt = slot + 1 < a.nt_saved ? hist_load<T>(a.E_saved, hix + a.frame, a.kind, 1.0f)
                                            : hist_load<T>(a.R_saved, q * a.frame + s * bc + hidx, a.kind, 1.0f);
        const T aeff = du ? ca : T(1);
        rhs = cbv != T(0) ? div_fixed(nxt - aeff * eo, dcb) : T(0);
      }
      T lam = fc == 0 ? lam_x[lf] : (fc == 1 ? lam_y[lf] : lam_z[lf]);
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
  const long long gi = ((long long)i * (g.NY - 1) + j) * (g.NZ - 1) + k;
  if (a.want_eps) {
    if (a.acc64) a.g_eps64[gi] += loc_e64; else a.g_eps[gi] += loc_e;
  }
  if (a.want_sig) {
    if (a.acc64) a.g_sig64[gi] += loc_s64; else a.g_sig[gi] += loc_s;
  }
}

}  // namespace dg
