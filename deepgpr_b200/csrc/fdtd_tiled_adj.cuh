// fdtd_tiled_adj.cuh -- bandwidth-oriented adjoint kernels.
//
// Same tiling as fdtd_tiled.cuh.  A transposed-curl channel weight W of a
// source cell is formed once per plane (x channels go into the register
// queue, y/z channels into shared memory together with their halo) and the
// target gathers read them; the per-cell arithmetic is that of
// fdtd_adjoint.cuh (reference: src/DeepGPR/lib/deepgpr_cpu.c:1112-1459).
//
// The imaging condition runs as its own kernel (k_image) before the E step:
// it sums the shots of a cell inside one thread, in the reference's order,
// and reads lambda_E, the history frames and the coefficients coalesced.
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

// E-step channel weight of source cell (ii, jj, kk) of shot s (E faces first,
// then the interior term).  ch: 0 AX, 1 AY, 2 BX, 3 BZ, 4 CY, 5 CZ.
template <typename T>
__device__ __forceinline__ T e_channel(const AdjArgs<T>& a, int ch, int s, int ii, int jj, int kk) {
  const Grid& g = a.g;
  if (ii < 0 || jj < 0 || kk < 0 || ii >= g.NX || jj >= g.NY || kk >= g.NZ) return T(0);
  const int c = ii * g.sx + jj * g.NZ + kk;
  const long long f = (long long)s * g.cells + c;
  const bool pml = a.has_cpml != 0;
  T w = T(0);
  switch (ch) {
    case 0:  // A_X: x faces psi1 (Ey), -c lambda_ey
      if (pml && jj < g.NY - 1) add_pml<T, true>(w, a.eF[0], a.eF[1], g, 0, 1, s, ii, jj, kk);
      if (upd_ey(g, ii, jj, kk)) w += (-a.ce_curl[c]) * a.lEy[f];
      break;
    case 1:  // A_Y: y faces psi1 (Ex), c_y lambda_ex
      if (pml && ii < g.NX - 1) add_pml<T, true>(w, a.eF[2], a.eF[3], g, 1, 1, s, ii, jj, kk);
      if (upd_ex(g, ii, jj, kk)) w += scaled(a.ce_curl[c], a.dx, a.dy, a.dy_eq) * a.lEx[f];
      break;
    case 2:  // B_X: x faces psi2 (Ez), c lambda_ez
      if (pml && kk < g.NZ - 1) add_pml<T, true>(w, a.eF[0], a.eF[1], g, 0, 2, s, ii, jj, kk);
      if (upd_ez(g, ii, jj, kk)) w += a.ce_curl[c] * a.lEz[f];
      break;
    case 3:  // B_Z: z faces psi1 (Ex), -c_z lambda_ex
      if (pml && ii < g.NX - 1) add_pml<T, true>(w, a.eF[4], a.eF[5], g, 2, 1, s, ii, jj, kk);
      if (upd_ex(g, ii, jj, kk)) w += (-scaled(a.ce_curl[c], a.dx, a.dz, a.dz_eq)) * a.lEx[f];
      break;
    case 4:  // C_Y: y faces psi2 (Ez), -c_y lambda_ez
      if (pml && kk < g.NZ - 1) add_pml<T, true>(w, a.eF[2], a.eF[3], g, 1, 2, s, ii, jj, kk);
      if (upd_ez(g, ii, jj, kk)) w += (-scaled(a.ce_curl[c], a.dx, a.dy, a.dy_eq)) * a.lEz[f];
      break;
    default:  // C_Z: z faces psi2 (Ey), c_z lambda_ey
      if (pml && jj < g.NY - 1) add_pml<T, true>(w, a.eF[4], a.eF[5], g, 2, 2, s, ii, jj, kk);
      if (upd_ey(g, ii, jj, kk)) w += scaled(a.ce_curl[c], a.dx, a.dz, a.dz_eq) * a.lEy[f];
      break;
  }
  return w;
}

// H-step channel weight of source cell (ii, jj, kk).
template <typename T>
__device__ __forceinline__ T h_channel(const AdjArgs<T>& a, int ch, int s, int ii, int jj, int kk) {
  const Grid& g = a.g;
  if (ii < 0 || jj < 0 || kk < 0 || ii >= g.NX || jj >= g.NY || kk >= g.NZ) return T(0);
  const int c = ii * g.sx + jj * g.NZ + kk;
  const long long f = (long long)s * g.cells + c;
  const bool pml = a.has_cpml != 0;
  T w = T(0);
  switch (ch) {
    case 0:  // A_X (ez_x): x faces psi1 (Hy), c lambda_hy
      if (pml && kk < g.NZ - 1) add_pml<T, false>(w, a.hF[0], a.hF[1], g, 0, 1, s, ii, jj, kk);
      if (upd_hy(g, ii, jj, kk)) w += a.ch_curl[c] * a.lHy[f];
      break;
    case 1:  // A_Y (ez_y): y faces psi1 (Hx), -c_y lambda_hx
      if (pml && kk < g.NZ - 1) add_pml<T, false>(w, a.hF[2], a.hF[3], g, 1, 1, s, ii, jj, kk);
      if (upd_hx(g, ii, jj, kk)) w += (-scaled(a.ch_curl[c], a.dx, a.dy, a.dy_eq)) * a.lHx[f];
      break;
    case 2:  // B_X (ey_x): x faces psi2 (Hz), -c lambda_hz
      if (pml && jj < g.NY - 1) add_pml<T, false>(w, a.hF[0], a.hF[1], g, 0, 2, s, ii, jj, kk);
      if (upd_hz(g, ii, jj, kk)) w += (-a.ch_curl[c]) * a.lHz[f];
      break;
    case 3:  // B_Z (ey_z): z faces psi1 (Hx), c_z lambda_hx
      if (pml && jj < g.NY - 1) add_pml<T, false>(w, a.hF[4], a.hF[5], g, 2, 1, s, ii, jj, kk);
      if (upd_hx(g, ii, jj, kk)) w += scaled(a.ch_curl[c], a.dx, a.dz, a.dz_eq) * a.lHx[f];
      break;
    case 4:  // C_Y (ex_y): y faces psi2 (Hz), c_y lambda_hz
      if (pml && ii < g.NX - 1) add_pml<T, false>(w, a.hF[2], a.hF[3], g, 1, 2, s, ii, jj, kk);
      if (upd_hz(g, ii, jj, kk)) w += scaled(a.ch_curl[c], a.dx, a.dy, a.dy_eq) * a.lHz[f];
      break;
    default:  // C_Z (ex_z): z faces psi2 (Hy), -c_z lambda_hy
      if (pml && ii < g.NX - 1) add_pml<T, false>(w, a.hF[4], a.hF[5], g, 2, 2, s, ii, jj, kk);
      if (upd_hy(g, ii, jj, kk)) w += (-scaled(a.ch_curl[c], a.dx, a.dz, a.dz_eq)) * a.lHy[f];
      break;
  }
  return w;
}

// Gathers on an accessor W(d) = weight of the source at offset d.
template <typename T, int R, typename WF>
__device__ __forceinline__ T gback(const WF& W, int c, int n) {
  return gather_back<T, R>(W, c, n);
}
template <typename T, int R, typename WF>
__device__ __forceinline__ T gfwd(const WF& W, int c, int n) {
  return gather_fwd<T, R>(W, c, n);
}

// Fill a channel plane (own + y or z halo) in shared memory.
template <typename T, int R, typename CF>
__device__ __forceinline__ void fill_channel(T* sm, int own, const Halo3<R>& h, int i, int j0, int k0, bool want_y,
                                             bool want_z, T own_val, const CF& chan) {
  sm[own] = own_val;
#pragma unroll
  for (int p = 0; p < Halo3<R>::PER_THREAD; ++p) {
    if (h.sidx[p] < 0) continue;
    if (h.yslot[p] ? !want_y : !want_z) continue;
    // recover (jj, kk) of the slot from its smem index
    const int sy = h.sidx[p] / Halo3<R>::W, sz = h.sidx[p] % Halo3<R>::W;
    sm[h.sidx[p]] = h.ok[p] ? chan(i, j0 + sy - R, k0 + sz - R) : T(0);
  }
}

// ---------------------------------------------------------------------------
// 3D E step: lambda_H += curl^T(E channels); H-CPML weights of step it.
// ---------------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(256) k3_adj_e(TiledAdj<T> P) {
  using HL = Halo3<R>;
  constexpr int W = HL::W;
  constexpr int NS = (TY + 2 * R) * W;
  __shared__ T sAY[2][NS], sCY[2][NS], sBZ[2][NS], sCZ[2][NS];
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int it = a.ctrl->cur - a.k_in_chunk;
  if (a.want_src && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0) {
    for (int m = threadIdx.x; m < a.nsrc; m += blockDim.x) {
      T acc = a.grad_source[(long long)m * a.nt + it];
      for (int s = 0; s < g.nshot; ++s) acc += a.srcv[(long long)s * a.nsrc + m];
      a.grad_source[(long long)m * a.nt + it] = acc;
    }
  }
  const int nzt = (g.NZ + TZ - 1) / TZ;
  const int tz = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int k0 = (blockIdx.x % nzt) * TZ, j0 = (blockIdx.x / nzt) * TY;
  const int k = k0 + tz, j = j0 + ty;
  const bool colv = k < g.NZ && j < g.NY;
  const int x0 = blockIdx.y * P.xchunk, x1 = min(x0 + P.xchunk, g.NX);
  const int s = blockIdx.z;
  const long long sb = (long long)s * g.cells;
  const int col = colv ? j * g.NZ + k : 0;
  const int own = (ty + R) * W + tz + R;
  HL halo;
  halo.init(g, j0, k0);
  int qh[6] = {-1, -1, -1, -1, -1, -1};
  if (colv && a.has_cpml) {
    qh[2] = q_low_h(a.hF[2].p, j);
    qh[3] = q_high(a.hF[3].p, j, g.NY);
    qh[4] = q_low_h(a.hF[4].p, k);
    qh[5] = q_high(a.hF[5].p, k, g.NZ);
  }
  T qA[2 * R], qB[2 * R];   // A_X, B_X at planes i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = x0 - R + 1 + m;
    qA[m] = colv ? e_channel(a, 0, s, pl, j, k) : T(0);
    qB[m] = colv ? e_channel(a, 2, s, pl, j, k) : T(0);
  }
  for (int i = x0; i < x1; ++i) {
    const int b = (i - x0) & 1;
    qA[2 * R - 1] = colv ? e_channel(a, 0, s, i + R, j, k) : T(0);
    qB[2 * R - 1] = colv ? e_channel(a, 2, s, i + R, j, k) : T(0);
    fill_channel<T, R>(sAY[b], own, halo, i, j0, k0, true, false, colv ? e_channel(a, 1, s, i, j, k) : T(0),
                       [&](int ii, int jj, int kk) { return e_channel(a, 1, s, ii, jj, kk); });
    fill_channel<T, R>(sCY[b], own, halo, i, j0, k0, true, false, colv ? e_channel(a, 4, s, i, j, k) : T(0),
                       [&](int ii, int jj, int kk) { return e_channel(a, 4, s, ii, jj, kk); });
    fill_channel<T, R>(sBZ[b], own, halo, i, j0, k0, false, true, colv ? e_channel(a, 3, s, i, j, k) : T(0),
                       [&](int ii, int jj, int kk) { return e_channel(a, 3, s, ii, jj, kk); });
    fill_channel<T, R>(sCZ[b], own, halo, i, j0, k0, false, true, colv ? e_channel(a, 5, s, i, j, k) : T(0),
                       [&](int ii, int jj, int kk) { return e_channel(a, 5, s, ii, jj, kk); });
    __syncthreads();
    if (colv) {
      const long long f = sb + (long long)i * g.sx + col;
      const T* say = sAY[b];
      const T* scy = sCY[b];
      const T* sbz = sBZ[b];
      const T* scz = sCZ[b];
      T hx = a.lHx[f], hy = a.lHy[f], hz = a.lHz[f];
      hz += gback<T, R>([&](int d) { return qA[R - 1 + d]; }, i, g.NX);
      hz += gback<T, R>([&](int d) { return say[own + d * W]; }, j, g.NY);
      hy += gback<T, R>([&](int d) { return qB[R - 1 + d]; }, i, g.NX);
      hy += gback<T, R>([&](int d) { return sbz[own + d]; }, k, g.NZ);
      hx += gback<T, R>([&](int d) { return scy[own + d * W]; }, j, g.NY);
      hx += gback<T, R>([&](int d) { return scz[own + d]; }, k, g.NZ);
      a.lHx[f] = hx;
      a.lHy[f] = hy;
      a.lHz[f] = hz;
      if (a.has_cpml) {
        qh[0] = q_low_h(a.hF[0].p, i);
        qh[1] = q_high(a.hF[1].p, i, g.NX);
        const bool any_h = qh[0] >= 0 || qh[1] >= 0 || qh[2] >= 0 || qh[3] >= 0 || qh[4] >= 0 || qh[5] >= 0;
        if (any_h) {
          const T up_h = a.ch_rhs[i * g.sx + col];
#pragma unroll
          for (int fc = 0; fc < 6; ++fc) {
            const int q = qh[fc];
            if (q < 0) continue;
            const Face<T>& F = a.hF[fc];
            const Prof<T> pr = prof(F, q);
            const int axis = fc >> 1;
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
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) {
      qA[m] = qA[m + 1];
      qB[m] = qB[m + 1];
    }
  }
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
// 3D H step: lambda_E <- ce_hist lambda_E + curl^T(H channels); head of it-1.
// PROLOGUE: only the head of step it (= nt-1).
// ---------------------------------------------------------------------------
template <typename T, int R, bool PROLOGUE>
__global__ void __launch_bounds__(256) k3_adj_h(TiledAdj<T> P) {
  using HL = Halo3<R>;
  constexpr int W = HL::W;
  constexpr int NS = PROLOGUE ? 1 : (TY + 2 * R) * W;
  __shared__ T sAY[2][NS], sCY[2][NS], sBZ[2][NS], sCZ[2][NS];
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int it = a.ctrl->cur - a.k_in_chunk;
  const int head = PROLOGUE ? it : it - 1;
  const int nzt = (g.NZ + TZ - 1) / TZ;
  const int tz = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int k0 = (blockIdx.x % nzt) * TZ, j0 = (blockIdx.x / nzt) * TY;
  const int k = k0 + tz, j = j0 + ty;
  const bool colv = k < g.NZ && j < g.NY;
  const int x0 = blockIdx.y * P.xchunk, x1 = min(x0 + P.xchunk, g.NX);
  const int s = blockIdx.z;
  const long long sb = (long long)s * g.cells;
  const int col = colv ? j * g.NZ + k : 0;
  const int own = (ty + R) * W + tz + R;
  HL halo;
  if (!PROLOGUE) halo.init(g, j0, k0);
  T qA[2 * R], qB[2 * R];   // A_X, B_X at planes i-R .. i+R-1
  if (!PROLOGUE) {
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) {
      const int pl = x0 - R + m;
      qA[m] = colv ? h_channel(a, 0, s, pl, j, k) : T(0);
      qB[m] = colv ? h_channel(a, 2, s, pl, j, k) : T(0);
    }
  }
  for (int i = x0; i < x1; ++i) {
    const int b = (i - x0) & 1;
    if (!PROLOGUE) {
      qA[2 * R - 1] = colv ? h_channel(a, 0, s, i + R - 1, j, k) : T(0);
      qB[2 * R - 1] = colv ? h_channel(a, 2, s, i + R - 1, j, k) : T(0);
      fill_channel<T, R>(sAY[b], own, halo, i, j0, k0, true, false, colv ? h_channel(a, 1, s, i, j, k) : T(0),
                         [&](int ii, int jj, int kk) { return h_channel(a, 1, s, ii, jj, kk); });
      fill_channel<T, R>(sCY[b], own, halo, i, j0, k0, true, false, colv ? h_channel(a, 4, s, i, j, k) : T(0),
                         [&](int ii, int jj, int kk) { return h_channel(a, 4, s, ii, jj, kk); });
      fill_channel<T, R>(sBZ[b], own, halo, i, j0, k0, false, true, colv ? h_channel(a, 3, s, i, j, k) : T(0),
                         [&](int ii, int jj, int kk) { return h_channel(a, 3, s, ii, jj, kk); });
      fill_channel<T, R>(sCZ[b], own, halo, i, j0, k0, false, true, colv ? h_channel(a, 5, s, i, j, k) : T(0),
                         [&](int ii, int jj, int kk) { return h_channel(a, 5, s, ii, jj, kk); });
      __syncthreads();
    }
    if (colv) {
      const int c = i * g.sx + col;
      const long long f = sb + c;
      T ex = a.lEx[f], ey = a.lEy[f], ez = a.lEz[f];
      if (!PROLOGUE) {
        const T chist = a.ce_hist[c];
        if (upd_ex(g, i, j, k)) ex = chist * ex;
        if (upd_ey(g, i, j, k)) ey = chist * ey;
        if (upd_ez(g, i, j, k)) ez = chist * ez;
        const T* say = sAY[b];
        const T* scy = sCY[b];
        const T* sbz = sBZ[b];
        const T* scz = sCZ[b];
        ez += gfwd<T, R>([&](int d) { return qA[R + d]; }, i, g.NX);
        ez += gfwd<T, R>([&](int d) { return say[own + d * W]; }, j, g.NY);
        ey += gfwd<T, R>([&](int d) { return qB[R + d]; }, i, g.NX);
        ey += gfwd<T, R>([&](int d) { return sbz[own + d]; }, k, g.NZ);
        ex += gfwd<T, R>([&](int d) { return scy[own + d * W]; }, j, g.NY);
        ex += gfwd<T, R>([&](int d) { return scz[own + d]; }, k, g.NZ);
      }
      if (head >= 0) {
        tiled_head(P, head, s, c, ex, ey, ez);
        if (a.has_cpml) e_pml_head(a, s, i, j, k, c, ex, ey, ez);
      }
      a.lEx[f] = ex;
      a.lEy[f] = ey;
      a.lEz[f] = ez;
    }
    if (!PROLOGUE) {
#pragma unroll
      for (int m = 0; m < 2 * R - 1; ++m) {
        qA[m] = qA[m + 1];
        qB[m] = qB[m + 1];
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
      if (a.kind == kFP8) {
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
