// fdtd_forward.cuh -- forward time step as two fused kernels.
//
//   k_fwd_h : E^n history frame  +  H update  +  H CPML (psi recurrences)
//   k_fwd_e : E update  +  E CPML  +  source injection  +  R^n history frame
//             +  receiver sampling
//
// Reference step order (src/DeepGPR/lib/deepgpr_cpu.c:1862-1917): save E^n,
// update H, CPML H, update E, CPML E, inject sources, save R^n, sample
// receivers.  Within one half step a cell's CPML correction depends only on
// that cell, so it is applied in registers right after the base update.
#pragma once

#include "fdtd_common.cuh"

namespace dg {

template <typename T>
struct FwdArgs {
  Grid g;
  T dx, dy, dz;
  FixedDiv<T> ddx, ddy, ddz;        // division by dx, dy, dz (CPML differences, curl scaling)
  int dy_eq, dz_eq;                 // dy == dx, dz == dx (selects the curl scaling)
  T *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
  const T *ce_hist, *ce_curl, *ce_rhs, *ch_curl, *ch_rhs;
  Face<T> eF[6], hF[6];
  int has_cpml;
  Control* ctrl;
  int k_in_chunk;                   // time step = ctrl->cur + k_in_chunk
  int nt;
  // sources: E[c] -= ce_rhs[c] * (w * dl / (dx*dy*dz)), per shot in source order
  PointTable src;
  const T* wave;                    // (nsrc, nt)
  int src_comp;
  T src_dl, src_vol;                // dipole length, (dx*dy)*dz
  // receivers: rx[(s*nt + t)*nrx + r] = E_comp after injection
  PointTable rcv;
  T* rx;
  int rx_comp, nrx;
  // histories (layout (comp, slot, shot, box cells))
  int save_e, keep_r, S, mode, kind, nt_saved;
  HBox box;
  long long frame, comp_stride;
  void* E_saved;
  void* R_saved;
  float* e_scales;                  // FP8: one scale per (comp, slot, shot, tile)
  float* r_scales;
  int ntiles;
};

template <typename T>
__device__ __forceinline__ T curl_scale(T c1, T dx, T d, int eq) {
  return eq ? c1 : c1 * dx / d;
}

// E^n history frame (fused into the H kernel, which reads E anyway).
template <typename T>
__device__ __forceinline__ void store_e_frame(const FwdArgs<T>& a, int s, long long base, bool inbox,
                                              long long h, int slot, float* red) {
  const int ncomp = a.mode == 3 ? 3 : 1;
  for (int q = 0; q < ncomp; ++q) {
    const int fc = a.mode == 3 ? q : 2;
    const T* E = fc == 0 ? a.Ex : (fc == 1 ? a.Ey : a.Ez);
    T v = inbox ? E[base] : T(0);
    float inv = 1.0f;
    if (a.kind == kFP8) {
      float am = block_absmax(inbox ? fabsf(float(v)) : 0.0f, red);
      float sc = fp8_scale_of(am);
      inv = 1.0f / sc;
      if (threadIdx.x == 0)
        a.e_scales[(((long long)q * a.nt_saved + slot) * a.g.nshot + s) * a.ntiles + blockIdx.x] = sc;
    }
    if (inbox)
      hist_store<T>(a.E_saved, q * a.comp_stride + slot * a.frame + s * a.box.cells() + h, v, a.kind, inv);
  }
}

template <typename T, int R>
__global__ void __launch_bounds__(kBlock) k_fwd_h(FwdArgs<T> a) {
  __shared__ float red[33];
  const Grid& g = a.g;
  const int c = blockIdx.x * kBlock + threadIdx.x;
  const bool live = c < g.cells;
  int i = 0, j = 0, k = 0;
  if (live) cell_ijk(g, c, i, j, k);
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save = a.save_e && (it % a.S == 0);
  const int slot = it / a.S;
  long long h = 0;
  const bool inbox = live && save && in_box(a.box, i, j, k, h);

  const bool dhx = live && upd_hx(g, i, j, k);
  const bool dhy = live && upd_hy(g, i, j, k);
  const bool dhz = live && upd_hz(g, i, j, k);
  T c1 = T(0), up = T(0);
  if (live) c1 = a.ch_curl[c];
  const T cy = curl_scale(c1, a.dx, a.dy, a.dy_eq);
  const T cz = curl_scale(c1, a.dx, a.dz, a.dz_eq);
  int qf[6] = {-1, -1, -1, -1, -1, -1};
  bool any_pml = false;
  if (live && a.has_cpml) {
    qf[0] = q_low_h(a.hF[0].p, i);
    qf[1] = q_high(a.hF[1].p, i, g.NX);
    qf[2] = q_low_h(a.hF[2].p, j);
    qf[3] = q_high(a.hF[3].p, j, g.NY);
    qf[4] = q_low_h(a.hF[4].p, k);
    qf[5] = q_high(a.hF[5].p, k, g.NZ);
    any_pml = qf[0] >= 0 || qf[1] >= 0 || qf[2] >= 0 || qf[3] >= 0 || qf[4] >= 0 || qf[5] >= 0;
    if (any_pml) up = a.ch_rhs[c];
  }
  const int s0 = blockIdx.y * g.shots_per_group;
  const int s1 = min(s0 + g.shots_per_group, g.nshot);
  for (int s = s0; s < s1; ++s) {
    const long long base = (long long)s * g.cells + c;
    if (save) store_e_frame(a, s, base, inbox, h, slot, red);
    if (!live) continue;
    const T* ex = a.Ex + base;
    const T* ey = a.Ey + base;
    const T* ez = a.Ez + base;
    T hx = a.Hx[base], hy = a.Hy[base], hz = a.Hz[base];
    // derivatives shared by the base update and the CPML correction
    T dEz_dy = T(0), dEy_dz = T(0), dEx_dz = T(0), dEz_dx = T(0), dEy_dx = T(0), dEx_dy = T(0);
    const bool in_x = qf[0] >= 0 || qf[1] >= 0;
    const bool in_y = qf[2] >= 0 || qf[3] >= 0;
    const bool in_z = qf[4] >= 0 || qf[5] >= 0;
    if (dhx || (in_y && k < g.NZ - 1)) dEz_dy = d_fwd<T, R>(ez, g.NZ, j, g.NY);
    if (dhx || (in_z && j < g.NY - 1)) dEy_dz = d_fwd<T, R>(ey, 1, k, g.NZ);
    if (dhy || (in_z && i < g.NX - 1)) dEx_dz = d_fwd<T, R>(ex, 1, k, g.NZ);
    if (dhy || (in_x && k < g.NZ - 1)) dEz_dx = d_fwd<T, R>(ez, g.sx, i, g.NX);
    if (dhz || (in_x && j < g.NY - 1)) dEy_dx = d_fwd<T, R>(ey, g.sx, i, g.NX);
    if (dhz || (in_y && i < g.NX - 1)) dEx_dy = d_fwd<T, R>(ex, g.NZ, j, g.NY);
    // base update (deepgpr_cpu.c:917-931); ch_hist == 1 on every updated cell
    if (dhx) hx = hx - cy * dEz_dy + cz * dEy_dz;
    if (dhy) hy = hy - cz * dEx_dz + c1 * dEz_dx;
    if (dhz) hz = hz - c1 * dEy_dx + cy * dEx_dy;
    if (any_pml) {
      // CPML H, faces x0 xm y0 ym z0 zm (deepgpr_cpu.c:980-1097)
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int q = qf[f];
        if (q < 0) continue;
        const Face<T>& F = a.hF[f];
        const Prof<T> pr = prof(F, q);
        const int axis = f >> 1;
        if (axis == 0) {
          if (k < g.NZ - 1) {
            const long long pi = psi_index(psi_dims_h(g, 0, 1, F.p), 0, s, q, i, j, k);
            const T d = div_fixed(dEz_dx, a.ddx), ph = F.psi1[pi];
            hy += up * (pr.ra1 * d + pr.rb * ph);
            F.psi1[pi] = pr.re * ph - pr.rf * d;
          }
          if (j < g.NY - 1) {
            const long long pi = psi_index(psi_dims_h(g, 0, 2, F.p), 0, s, q, i, j, k);
            const T d = div_fixed(dEy_dx, a.ddx), ph = F.psi2[pi];
            hz -= up * (pr.ra1 * d + pr.rb * ph);
            F.psi2[pi] = pr.re * ph - pr.rf * d;
          }
        } else if (axis == 1) {
          if (k < g.NZ - 1) {
            const long long pi = psi_index(psi_dims_h(g, 1, 1, F.p), 1, s, q, i, j, k);
            const T d = div_fixed(dEz_dy, a.ddy), ph = F.psi1[pi];
            hx -= up * (pr.ra1 * d + pr.rb * ph);
            F.psi1[pi] = pr.re * ph - pr.rf * d;
          }
          if (i < g.NX - 1) {
            const long long pi = psi_index(psi_dims_h(g, 1, 2, F.p), 1, s, q, i, j, k);
            const T d = div_fixed(dEx_dy, a.ddy), ph = F.psi2[pi];
            hz += up * (pr.ra1 * d + pr.rb * ph);
            F.psi2[pi] = pr.re * ph - pr.rf * d;
          }
        } else {
          if (j < g.NY - 1) {
            const long long pi = psi_index(psi_dims_h(g, 2, 1, F.p), 2, s, q, i, j, k);
            const T d = div_fixed(dEy_dz, a.ddz), ph = F.psi1[pi];
            hx += up * (pr.ra1 * d + pr.rb * ph);
            F.psi1[pi] = pr.re * ph - pr.rf * d;
          }
          if (i < g.NX - 1) {
            const long long pi = psi_index(psi_dims_h(g, 2, 2, F.p), 2, s, q, i, j, k);
            const T d = div_fixed(dEx_dz, a.ddz), ph = F.psi2[pi];
            hy -= up * (pr.ra1 * d + pr.rb * ph);
            F.psi2[pi] = pr.re * ph - pr.rf * d;
          }
        }
      }
    }
    a.Hx[base] = hx;
    a.Hy[base] = hy;
    a.Hz[base] = hz;
  }
}

template <typename T, int R>
__global__ void __launch_bounds__(kBlock) k_fwd_e(FwdArgs<T> a) {
  __shared__ float red[33];
  __shared__ int smap[kBlock];
  __shared__ int rmap[kBlock];
  const Grid& g = a.g;
  const int c0 = blockIdx.x * kBlock;
  const int c = c0 + threadIdx.x;
  const bool live = c < g.cells;
  int i = 0, j = 0, k = 0;
  if (live) cell_ijk(g, c, i, j, k);
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save_r = a.keep_r && (it % a.S == 0);
  const int slot = it / a.S;
  long long h = 0;
  const bool inbox = live && save_r && in_box(a.box, i, j, k, h);

  build_block_map(a.src, c0, smap);
  build_block_map(a.rcv, c0, rmap);
  const int srow = smap[threadIdx.x];
  const int rrow = rmap[threadIdx.x];

  const bool dex = live && upd_ex(g, i, j, k);
  const bool dey = live && upd_ey(g, i, j, k);
  const bool dez = live && upd_ez(g, i, j, k);
  T c0e = T(0), c1 = T(0), cb = T(0);
  if (live) {
    c0e = a.ce_hist[c];
    c1 = a.ce_curl[c];
  }
  const T cy = curl_scale(c1, a.dx, a.dy, a.dy_eq);
  const T cz = curl_scale(c1, a.dx, a.dz, a.dz_eq);
  int qf[6] = {-1, -1, -1, -1, -1, -1};
  bool any_pml = false;
  if (live && a.has_cpml) {
    qf[0] = i > 0 ? q_low_e(a.eF[0].p, i) : -1;
    qf[1] = i > 0 ? q_high(a.eF[1].p, i, g.NX) : -1;
    qf[2] = j > 0 ? q_low_e(a.eF[2].p, j) : -1;
    qf[3] = j > 0 ? q_high(a.eF[3].p, j, g.NY) : -1;
    qf[4] = k > 0 ? q_low_e(a.eF[4].p, k) : -1;
    qf[5] = k > 0 ? q_high(a.eF[5].p, k, g.NZ) : -1;
    any_pml = qf[0] >= 0 || qf[1] >= 0 || qf[2] >= 0 || qf[3] >= 0 || qf[4] >= 0 || qf[5] >= 0;
  }
  if (live && (any_pml || srow >= 0 || save_r)) cb = a.ce_rhs[c];
  const bool in_x = qf[0] >= 0 || qf[1] >= 0;
  const bool in_y = qf[2] >= 0 || qf[3] >= 0;
  const bool in_z = qf[4] >= 0 || qf[5] >= 0;

  const int s0 = blockIdx.y * g.shots_per_group;
  const int s1 = min(s0 + g.shots_per_group, g.nshot);
  for (int s = s0; s < s1; ++s) {
    const long long base = (long long)s * g.cells + c;
    T ex = T(0), ey = T(0), ez = T(0), ox = T(0), oy = T(0), oz = T(0);
    if (live) {
      const T* hx = a.Hx + base;
      const T* hy = a.Hy + base;
      const T* hz = a.Hz + base;
      ox = ex = a.Ex[base];
      oy = ey = a.Ey[base];
      oz = ez = a.Ez[base];
      T dHz_dy = T(0), dHy_dz = T(0), dHx_dz = T(0), dHz_dx = T(0), dHy_dx = T(0), dHx_dy = T(0);
      if (dex || (in_y && i < g.NX - 1)) dHz_dy = d_back<T, R>(hz, g.NZ, j, g.NY);
      if (dex || (in_z && i < g.NX - 1)) dHy_dz = d_back<T, R>(hy, 1, k, g.NZ);
      if (dey || (in_z && j < g.NY - 1)) dHx_dz = d_back<T, R>(hx, 1, k, g.NZ);
      if (dey || (in_x && j < g.NY - 1)) dHz_dx = d_back<T, R>(hz, g.sx, i, g.NX);
      if (dez || (in_x && k < g.NZ - 1)) dHy_dx = d_back<T, R>(hy, g.sx, i, g.NX);
      if (dez || (in_y && k < g.NZ - 1)) dHx_dy = d_back<T, R>(hx, g.NZ, j, g.NY);
      // base update (deepgpr_cpu.c:700-715)
      if (dex) ex = c0e * ex + cy * dHz_dy - cz * dHy_dz;
      if (dey) ey = c0e * ey + cz * dHx_dz - c1 * dHz_dx;
      if (dez) ez = c0e * ez + c1 * dHy_dx - cy * dHx_dy;
      if (any_pml) {
        // CPML E, faces x0 xm y0 ym z0 zm (deepgpr_cpu.c:765-880)
#pragma unroll
        for (int f = 0; f < 6; ++f) {
          const int q = qf[f];
          if (q < 0) continue;
          const Face<T>& F = a.eF[f];
          const Prof<T> pr = prof(F, q);
          const int axis = f >> 1;
          if (axis == 0) {
            if (j < g.NY - 1) {
              const long long pi = psi_index(psi_dims_e(g, 0, 1, F.p), 0, s, q, i, j, k);
              const T d = div_fixed(dHz_dx, a.ddx), ph = F.psi1[pi];
              ey -= cb * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (k < g.NZ - 1) {
              const long long pi = psi_index(psi_dims_e(g, 0, 2, F.p), 0, s, q, i, j, k);
              const T d = div_fixed(dHy_dx, a.ddx), ph = F.psi2[pi];
              ez += cb * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          } else if (axis == 1) {
            if (i < g.NX - 1) {
              const long long pi = psi_index(psi_dims_e(g, 1, 1, F.p), 1, s, q, i, j, k);
              const T d = div_fixed(dHz_dy, a.ddy), ph = F.psi1[pi];
              ex += cb * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (k < g.NZ - 1) {
              const long long pi = psi_index(psi_dims_e(g, 1, 2, F.p), 1, s, q, i, j, k);
              const T d = div_fixed(dHx_dy, a.ddy), ph = F.psi2[pi];
              ez -= cb * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          } else {
            if (i < g.NX - 1) {
              const long long pi = psi_index(psi_dims_e(g, 2, 1, F.p), 2, s, q, i, j, k);
              const T d = div_fixed(dHy_dz, a.ddz), ph = F.psi1[pi];
              ex -= cb * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (j < g.NY - 1) {
              const long long pi = psi_index(psi_dims_e(g, 2, 2, F.p), 2, s, q, i, j, k);
              const T d = div_fixed(dHx_dz, a.ddz), ph = F.psi2[pi];
              ey += cb * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          }
        }
      }
      // sources of this shot at this cell, in source order (deepgpr_cpu.c:655-666)
      if (srow >= 0) {
        for (int e = a.src.off[srow]; e < a.src.off[srow + 1]; ++e) {
          if (a.src.shot[e] != s) continue;
          const T scale = a.wave[(long long)a.src.idx[e] * a.nt + it] * a.src_dl / a.src_vol;
          if (a.src_comp == 0) ex -= cb * scale;
          else if (a.src_comp == 1) ey -= cb * scale;
          else ez -= cb * scale;
        }
      }
    }
    // R^n = (E^(n+1) - a E^n) / cb over the history box (deepgpr_cpu.c:1559-1592)
    if (save_r) {
      const int ncomp = a.mode == 3 ? 3 : 1;
      for (int q = 0; q < ncomp; ++q) {
        const int fc = a.mode == 3 ? q : 2;
        T rv = T(0);
        if (inbox) {
          const T en = fc == 0 ? ex : (fc == 1 ? ey : ez);
          const T eo = fc == 0 ? ox : (fc == 1 ? oy : oz);
          const bool du = fc == 0 ? dex : (fc == 1 ? dey : dez);
          const T aeff = du ? c0e : T(1);
          rv = cb != T(0) ? (en - aeff * eo) / cb : T(0);
        }
        float inv = 1.0f;
        if (a.kind == kFP8) {
          float am = block_absmax(inbox ? fabsf(float(rv)) : 0.0f, red);
          float sc = fp8_scale_of(am);
          inv = 1.0f / sc;
          if (threadIdx.x == 0)
            a.r_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + blockIdx.x] = sc;
        }
        if (inbox)
          hist_store<T>(a.R_saved, q * a.comp_stride + slot * a.frame + s * a.box.cells() + h, rv, a.kind, inv);
      }
    }
    if (!live) continue;
    // receivers of this shot at this cell (deepgpr_cpu.c:600-623)
    if (rrow >= 0) {
      const T v = a.rx_comp == 0 ? ex : (a.rx_comp == 1 ? ey : ez);
      for (int e = a.rcv.off[rrow]; e < a.rcv.off[rrow + 1]; ++e)
        if (a.rcv.shot[e] == s) a.rx[((long long)s * a.nt + it) * a.nrx + a.rcv.idx[e]] = v;
    }
    a.Ex[base] = ex;
    a.Ey[base] = ey;
    a.Ez[base] = ez;
  }
}

// Copy of E (one frame, all shots) into a history buffer: the closing E^nt
// frame of an E-only history (deepgpr_cpu.c:1919-1930).
template <typename T>
__global__ void k_final_frame(const T* __restrict__ E, void* dst, Grid g, HBox box, int kind) {
  const long long bc = box.cells();
  const long long n = (long long)g.nshot * bc;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
    const long long s = w / bc, hh = w % bc;
    const int hi = int(hh / ((long long)box.ny * box.nz));
    const int rem = int(hh % ((long long)box.ny * box.nz));
    const int c = (hi + box.x0) * g.sx + (rem / box.nz + box.y0) * g.NZ + (rem % box.nz + box.z0);
    hist_store<T>(dst, w, E[s * g.cells + c], kind, 1.0f);
  }
}

}  // namespace dg
