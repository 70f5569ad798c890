// fdtd_tm2d.cuh -- 2D TM (Ez, Hx, Hy) kernels: 32-column warp strips.
//
// Layout inside a call: compact (shot, NX, NYP) arrays, NYP = NY rounded up to
// a multiple of 32 (zero padding, never written), so every row starts on a
// 128-byte boundary and a warp's row load is one fully used 128-byte line.
//
// Execution: every warp is independent.  A warp owns one 32-column strip of
// one shot (lane l holds column base + l) and streams along x over a chunk of
// rows:
//   * x-stencils read a register queue of the 2R rows around the current one
//     (each row is loaded once per strip);
//   * y-stencils take the neighbouring columns from the other lanes with warp
//     shuffles; lanes 0..2R-1 also hold the R halo columns on each side;
//   * the operands of row i+1 are loaded before row i is computed, so one
//     row of loads is always in flight behind the arithmetic;
//   * strips away from the CPML frame and the grid ends run a branch-free
//     interior path; the frame runs the general per-cell path;
//   * sources / receivers are looked up only on rows flagged for the shot.
// Chunk lengths are chosen from the kernels' occupancy so a launch is about
// one full wave of warps (see tm_geometry in fdtd_api.cu).
// Per-cell arithmetic is that of the reference (src/DeepGPR/lib/deepgpr_cpu.c:
// 670-1100 forward, 1112-1459 adjoint), in the same order.
#pragma once

#include "fdtd_tiled_adj.cuh"

namespace dg {

constexpr int TMW = 32;                // columns per warp strip = FP8 scale tile width
constexpr int TM_WARPS = 4;            // warps per CTA (neighbouring strips of one row chunk)
constexpr unsigned kFullMask = 0xffffffffu;

// Frame kinds of the general kernels: kFrameGeneral makes no assumption;
// kFrameXLean rows satisfy tm_lean_ok along x (no x CPML, full x stencils,
// x parts of the update predicates true); kFrameYLean strips lie in tiles
// where tm_lean_ok holds along y for every column.
constexpr int kFrameGeneral = 0, kFrameXLean = 1, kFrameYLean = 2;
constexpr int kTmMaxRects = 12;

// A rectangle of work: nseg warp strips of `width` columns from column
// 32 seg0, rows [row0, row1), every shot, cut into row chunks of xc rows;
// its warps are numbered from warp0.
struct TmRect {
  int seg0, nseg, row0, row1, xc, nchunk;
  int width;          // columns per warp: 32 (general kernels) or 128 (interior kernels)
  int kind;           // general kernels: frame kind of the rectangle (kFrameGeneral ...)
  long long warp0;
};

struct TmGeom {
  int NYP;            // padded row pitch
  int nseg;           // 32-column strips per row (NYP / 32)
  int nrect;          // rectangles of this launch (at most kTmMaxRects)
  int col1;           // interior kernels: end of the interior columns (a multiple of 32)
  int sum_source;     // adjoint E frame: this launch adds the step's source gradient
  TmRect rect[kTmMaxRects];
  long long nwarps;   // warps of all rectangles
  const unsigned char* src_rows;   // (nshot, NX): row holds a source of the shot
  const unsigned char* rcv_rows;   // (nshot, NX): row holds a receiver of the shot
};

template <typename T>
struct TmBuf {
  T *Ez, *Hx, *Hy;                                          // (nshot, NX, NYP)
  const T *ce_hist, *ce_curl, *ce_rhs, *ch_curl, *ch_rhs;   // (NX, NYP)
  // y-derivative curl coefficients c * dx / dy (the planes ce_curl / ch_curl
  // themselves when dy == dx), computed once per call
  const T *ce_curl_y, *ch_curl_y;
};

__device__ __forceinline__ float warp_absmax(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFullMask, v, o));
  return v;
}

struct WarpPos {
  int lane, seg, chunk, s, base, x0, x1, kind;
  bool live;
};

// Warp w -> (rectangle, strip, chunk, shot), strip fastest, so the warps of
// a CTA are neighbouring strips of the same rows.
// blk: the CTA's index within this geometry's part of the launch.
__device__ __forceinline__ WarpPos warp_pos(const TmGeom& tg, int nshot, unsigned blk) {
  WarpPos p;
  p.lane = threadIdx.x;
  // warp counts stay below 2^31 (checked on the host): 32-bit index arithmetic
  const unsigned w = blk * TM_WARPS + threadIdx.y;
  p.live = w < (unsigned)tg.nwarps;
  TmRect rc = tg.rect[0];
#pragma unroll
  for (int q = 1; q < kTmMaxRects; ++q)
    if (q < tg.nrect && w >= (unsigned)tg.rect[q].warp0) rc = tg.rect[q];
  const unsigned ww = p.live ? w - (unsigned)rc.warp0 : 0u;
  const unsigned nsg = (unsigned)rc.nseg, nch = (unsigned)rc.nchunk;
  const unsigned rest = ww / nsg;
  p.base = rc.seg0 * TMW + int(ww - rest * nsg) * rc.width;
  p.seg = p.base / TMW;
  const unsigned sh = rest / nch;
  p.chunk = int(rest - sh * nch);
  p.s = int(sh);
  p.live = p.live && p.s < nshot;
  p.kind = rc.kind;
  p.x0 = rc.row0 + p.chunk * rc.xc;
  p.x1 = min(p.x0 + rc.xc, rc.row1);
  return p;
}

// Halo column held by a lane: lanes [0, R) hold base - R + lane, lanes
// [R, 2R) hold base + 32 + lane - R.
template <int R>
__device__ __forceinline__ int halo_col(int base, int lane) {
  return lane < R ? base - R + lane : base + TMW + lane - R;
}

// Value at column base + lane + d (|d| <= R) from the lanes' own values and
// the halo lanes.  All 32 lanes must call it with the same d.
template <typename T, int R>
__device__ __forceinline__ T ynb(T own, T halo, int lane, int d) {
  const int src = lane + d;
  const T a = __shfl_sync(kFullMask, own, src & 31);
  const int hl = src < 0 ? src + R : src - TMW + R;
  const T b = __shfl_sync(kFullMask, halo, hl & 31);
  return (src >= 0 && src < TMW) ? a : b;
}

// ---------------------------------------------------------------------------
// Forward H (E^n history + Hx, Hy update + x/y CPML).
// ---------------------------------------------------------------------------
template <typename T, int R, int FK>
__device__ __forceinline__ void tm_fwd_h_body(const TiledFwd<T>& P, const TmBuf<T>& f, const TmGeom& tg, const WarpPos& wp) {
  constexpr bool XL = FK == kFrameXLean, YL = FK == kFrameYLean;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const int lane = wp.lane, s = wp.s;
  const int j = wp.base + lane;
  const bool cv = j < NY;
  const int hj = halo_col<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  const T* __restrict__ Ez = f.Ez + s * plane;
  T* __restrict__ Hx = f.Hx + s * plane;
  T* __restrict__ Hy = f.Hy + s * plane;
  const T* __restrict__ cc = f.ch_curl;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save = a.save_e && (it % a.S == 0);
  const int slot = it / a.S;
  const int qy0 = (!YL && cv && a.has_cpml) ? q_low_h(a.hF[2].p, j) : -1;
  const int qy1 = (!YL && cv && a.has_cpml) ? q_high(a.hF[3].p, j, NY) : -1;
  // warp-uniform: the strip is clear of the y CPML slabs and the clamped ends
  const int ylo = max(a.has_cpml ? a.hF[2].p : 0, R), yhi = NY - 1 - max(a.has_cpml ? a.hF[3].p : 0, R);
  const bool seg_int = YL || (wp.base >= ylo && wp.base + TMW - 1 < yhi);
  T q[2 * R];   // Ez at rows i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int r = wp.x0 - R + 1 + m;
    q[m] = (r >= 0 && r < NX) ? Ez[(long long)r * NYP + j] : T(0);
  }
  const T* __restrict__ ccy = f.ch_curl_y;
  T n_e, n_h, n_hx, n_hy, n_c, n_cy;   // operands of the next row
  auto fetch = [&](int i) {
    const long long rw = (long long)i * NYP;
    n_e = i + R < NX ? Ez[rw + (long long)R * NYP + j] : T(0);
    n_h = hok ? Ez[rw + hj] : T(0);
    n_hx = Hx[rw + j];
    n_hy = Hy[rw + j];
    n_c = cc[rw + j];
    n_cy = ccy[rw + j];
  };
  fetch(wp.x0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    q[2 * R - 1] = n_e;
    const T halo = n_h, hx0 = n_hx, hy0 = n_hy, c1 = n_c, cy = n_cy;
    if (i + 1 < wp.x1) fetch(i + 1);
    const long long rw = (long long)i * NYP;
    const T cur = q[R - 1];
    T yv[2 * R];   // Ez at columns j + d, d = -(R-1) .. R
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) yv[d + R - 1] = d == 0 ? cur : ynb<T, R>(cur, halo, lane, d);
    if (save) {
      long long hk = 0;
      const bool ib = cv && in_box(a.box, i, j, 0, hk);
      float inv = 1.0f;
      if (is_tiled(a.kind)) {
        // one scale per warp strip row: tile i * nseg + seg
        const float sc = tile_scale_of(a.kind, warp_absmax(ib ? fabsf(float(cur)) : 0.0f));
        inv = 1.0f / sc;
        if (lane == 0) a.e_scales[((long long)slot * g.nshot + s) * a.ntiles + (long long)i * tg.nseg + wp.seg] = sc;
      }
      if (ib) hist_store<T>(a.E_saved, slot * a.frame + s * a.box.cells() + hk, cur, a.kind, inv);
    }
    const int qx0 = (!XL && a.has_cpml) ? q_low_h(a.hF[0].p, i) : -1;
    const int qx1 = (!XL && a.has_cpml) ? q_high(a.hF[1].p, i, NX) : -1;
    const bool in_x = !XL && (qx0 >= 0 || qx1 >= 0);
    const bool row_int = XL || (!in_x && i > 0 && i < NX - 1 && i - R + 1 >= 0 && i + R < NX);
    if (row_int && seg_int) {
      T dEz_dy = T(0), dEz_dx = T(0);
      if (R == 1) {
        dEz_dy = yv[1] - yv[0];
        dEz_dx = q[1] - q[0];
      } else {
#pragma unroll
        for (int r = 1; r <= R; ++r) dEz_dy += tap<T>(R, r) * (yv[R - 1 + r] - yv[R - 1 - (r - 1)]);
#pragma unroll
        for (int r = 1; r <= R; ++r) dEz_dx += tap<T>(R, r) * (q[R - 1 + r] - q[R - 1 - (r - 1)]);
      }
      Hx[rw + j] = hx0 - cy * dEz_dy;
      Hy[rw + j] = hy0 + c1 * dEz_dx;
    } else if (cv) {
      // tm_upd_hx / tm_upd_hy split into row and column parts (true on lean rows / tiles)
      const bool dhx = (XL || (g.NX - 1 != 1 && i > 0 && i < g.NX - 1)) && (YL || j < g.NY - 1);
      const bool dhy = (XL || i < g.NX - 1) && (YL || (g.NY - 1 != 1 && j > 0 && j < g.NY - 1));
      const bool in_y = !YL && (qy0 >= 0 || qy1 >= 0);
      T dEz_dy = T(0), dEz_dx = T(0);
      const auto fy = [&](int d) { return yv[d + R - 1]; };
      const auto fx = [&](int d) { return q[R - 1 + d]; };
      if (dhx || in_y) dEz_dy = YL ? dfwd_full<T, R>(fy) : dfwd_f<T, R>(fy, j, NY);
      if (dhy || in_x) dEz_dx = XL ? dfwd_full<T, R>(fx) : dfwd_f<T, R>(fx, i, NX);
      T hxv = hx0, hyv = hy0;
      if (dhx) hxv = hxv - cy * dEz_dy;
      if (dhy) hyv = hyv + c1 * dEz_dx;
      if (in_x || in_y) {
        const T up = f.ch_rhs[rw + j];
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qx0 : qx1;
          if (XL || qq < 0) continue;
          const Face<T>& F = a.hF[fc];
          const Prof<T> pr = prof(F, qq);
          const long long pi = ((long long)s * F.p + qq) * NY + j;
          const T d = div_fixed(dEz_dx, a.ddx), ph = F.psi1[pi];
          hyv += up * (pr.ra1 * d + pr.rb * ph);
          F.psi1[pi] = pr.re * ph - pr.rf * d;
        }
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qy0 : qy1;
          if (YL || qq < 0) continue;
          const Face<T>& F = a.hF[2 + fc];
          const Prof<T> pr = prof(F, qq);
          const long long pi = ((long long)s * NX + i) * F.p + qq;
          const T d = div_fixed(dEz_dy, a.ddy), ph = F.psi1[pi];
          hxv -= up * (pr.ra1 * d + pr.rb * ph);
          F.psi1[pi] = pr.re * ph - pr.rf * d;
        }
      }
      Hx[rw + j] = hxv;
      Hy[rw + j] = hyv;
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) q[m] = q[m + 1];
  }
}

template <typename T, int R>
__device__ __forceinline__ void tm_fwd_h_run(const TiledFwd<T>& P, const TmBuf<T>& f, const TmGeom& tg, unsigned blk) {
  const WarpPos wp = warp_pos(tg, P.a.g.nshot, blk);
  if (!wp.live) return;
  if (wp.kind == kFrameXLean) tm_fwd_h_body<T, R, kFrameXLean>(P, f, tg, wp);
  else if (wp.kind == kFrameYLean) tm_fwd_h_body<T, R, kFrameYLean>(P, f, tg, wp);
  else tm_fwd_h_body<T, R, kFrameGeneral>(P, f, tg, wp);
}

template <typename T, int R>
__global__ void __launch_bounds__(32 * TM_WARPS) tm_fwd_h(TiledFwd<T> P, TmBuf<T> f, TmGeom tg) {
  tm_fwd_h_run<T, R>(P, f, tg, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Forward E (Ez update + x/y CPML + sources + R^n history + receivers).
// ---------------------------------------------------------------------------
template <typename T, int R, int FK>
__device__ __forceinline__ void tm_fwd_e_body(const TiledFwd<T>& P, const TmBuf<T>& f, const TmGeom& tg, const WarpPos& wp) {
  constexpr bool XL = FK == kFrameXLean, YL = FK == kFrameYLean;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const int lane = wp.lane, s = wp.s;
  const int j = wp.base + lane;
  const bool cv = j < NY;
  const int hj = halo_col<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  T* __restrict__ Ez = f.Ez + s * plane;
  const T* __restrict__ Hx = f.Hx + s * plane;
  const T* __restrict__ Hy = f.Hy + s * plane;
  const T* __restrict__ c0p = f.ce_hist;
  const T* __restrict__ c1p = f.ce_curl;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save_r = a.keep_r && (it % a.S == 0);
  const int slot = it / a.S;
  const int qy0 = (!YL && cv && a.has_cpml && j > 0) ? q_low_e(a.eF[2].p, j) : -1;
  const int qy1 = (!YL && cv && a.has_cpml && j > 0) ? q_high(a.eF[3].p, j, NY) : -1;
  const int ylo = max(a.has_cpml ? a.eF[2].p + 1 : 1, R), yhi = NY - 1 - max(a.has_cpml ? a.eF[3].p + 1 : 1, R);
  const bool seg_int = YL || (wp.base >= ylo && wp.base + TMW - 1 < yhi);
  T q[2 * R];   // Hy at rows i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int r = wp.x0 - R + m;
    q[m] = (r >= 0 && r < NX) ? Hy[(long long)r * NYP + j] : T(0);
  }
  const T* __restrict__ cyp = f.ce_curl_y;
  T n_y, n_x, n_h, n_ez, n_c0, n_c1, n_cy;   // operands of the next row
  auto fetch = [&](int i) {
    const long long rw = (long long)i * NYP;
    n_y = i + R - 1 < NX ? Hy[rw + (long long)(R - 1) * NYP + j] : T(0);
    n_x = Hx[rw + j];
    n_h = hok ? Hx[rw + hj] : T(0);
    n_ez = Ez[rw + j];
    n_c0 = c0p[rw + j];
    n_c1 = c1p[rw + j];
    n_cy = cyp[rw + j];
  };
  fetch(wp.x0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    q[2 * R - 1] = n_y;
    const T hxo = n_x, halo = n_h, ez0 = n_ez, c0 = n_c0, c1 = n_c1, cy = n_cy;
    if (i + 1 < wp.x1) fetch(i + 1);
    const long long rw = (long long)i * NYP;
    T yv[2 * R];   // Hx at columns j + d, d = -R .. R-1
#pragma unroll
    for (int d = -R; d <= R - 1; ++d) yv[d + R] = d == 0 ? hxo : ynb<T, R>(hxo, halo, lane, d);
    const int qx0 = (!XL && a.has_cpml && i > 0) ? q_low_e(a.eF[0].p, i) : -1;
    const int qx1 = (!XL && a.has_cpml && i > 0) ? q_high(a.eF[1].p, i, NX) : -1;
    const bool in_x = !XL && (qx0 >= 0 || qx1 >= 0);
    const bool row_pts = (tg.src_rows && tg.src_rows[(long long)s * NX + i]) ||
                         (tg.rcv_rows && tg.rcv_rows[(long long)s * NX + i]);
    const bool row_int = XL || (!in_x && i >= R && i + R - 1 < NX && i > 0 && i < NX - 1);
    if (row_int && seg_int && !row_pts && !save_r) {
      T dHy_dx = T(0), dHx_dy = T(0);
      if (R == 1) {
        dHy_dx = q[R] - q[R - 1];
        dHx_dy = yv[R] - yv[R - 1];
      } else {
#pragma unroll
        for (int r = 1; r <= R; ++r) dHy_dx += tap<T>(R, r) * (q[R + r - 1] - q[R - r]);
#pragma unroll
        for (int r = 1; r <= R; ++r) dHx_dy += tap<T>(R, r) * (yv[R + r - 1] - yv[R - r]);
      }
      Ez[rw + j] = c0 * ez0 + c1 * dHy_dx - cy * dHx_dy;
    } else {
      T ez = ez0, cb = T(0);
      bool dez = false;
      if (cv) {
        // tm_upd_ez split into row and column parts (true on lean rows / tiles)
        dez = (XL || YL || g.NX - 1 != 1 || g.NY - 1 != 1) && (XL || (i > 0 && i < NX - 1)) &&
              (YL || (j > 0 && j < NY - 1));
        const bool in_y = !YL && (qy0 >= 0 || qy1 >= 0);
        T dHy_dx = T(0), dHx_dy = T(0);
        const auto fx = [&](int d) { return q[R + d]; };
        const auto fy = [&](int d) { return yv[d + R]; };
        if (dez || in_x) dHy_dx = XL ? dback_full<T, R>(fx) : dback_f<T, R>(fx, i, NX);
        if (dez || in_y) dHx_dy = YL ? dback_full<T, R>(fy) : dback_f<T, R>(fy, j, NY);
        if (dez) ez = c0 * ez + c1 * dHy_dx - cy * dHx_dy;
        const int cfull = i * g.sx + j * g.NZ;
        const bool src_hit = row_pts && point_hit(P.src, s, cfull);
        if (in_x || in_y || src_hit || save_r) cb = f.ce_rhs[rw + j];
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qx0 : qx1;
          if (XL || qq < 0) continue;
          const Face<T>& F = a.eF[fc];
          const Prof<T> pr = prof(F, qq);
          const long long pi = ((long long)s * (F.p + 1) + qq) * NY + j;
          const T d = div_fixed(dHy_dx, a.ddx), ph = F.psi2[pi];
          ez += cb * (pr.ra1 * d + pr.rb * ph);
          F.psi2[pi] = pr.re * ph - pr.rf * d;
        }
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qy0 : qy1;
          if (YL || qq < 0) continue;
          const Face<T>& F = a.eF[2 + fc];
          const Prof<T> pr = prof(F, qq);
          const long long pi = ((long long)s * NX + i) * (F.p + 1) + qq;
          const T d = div_fixed(dHx_dy, a.ddy), ph = F.psi2[pi];
          ez -= cb * (pr.ra1 * d + pr.rb * ph);
          F.psi2[pi] = pr.re * ph - pr.rf * d;
        }
        if (src_hit) {
          T ex = T(0), ey = T(0);
          inject_at(P, s, cfull, it, cb, ex, ey, ez);
        }
      }
      if (save_r) {
        // R^n = (E^{n+1} - a_eff E^n) / cb (deepgpr_cpu.c:1850-1875); warp-uniform branch
        long long h = 0;
        const bool inbox = cv && in_box(a.box, i, j, 0, h);
        T rv = T(0);
        if (inbox) {
          const T aeff = dez ? c0 : T(1);
          rv = cb != T(0) ? (ez - aeff * ez0) / cb : T(0);
        }
        float inv = 1.0f;
        if (is_tiled(a.kind)) {
          const float sc = tile_scale_of(a.kind, warp_absmax(inbox ? fabsf(float(rv)) : 0.0f));
          if (lane == 0) a.r_scales[((long long)slot * g.nshot + s) * a.ntiles + (long long)i * tg.nseg + wp.seg] = sc;
          inv = 1.0f / sc;
        }
        if (inbox) hist_store<T>(a.R_saved, slot * a.frame + s * a.box.cells() + h, rv, a.kind, inv);
      }
      if (cv) {
        if (row_pts) sample_at(P, s, i * g.sx + j * g.NZ, it, T(0), T(0), ez);
        Ez[rw + j] = ez;
      }
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) q[m] = q[m + 1];
  }
}

template <typename T, int R>
__device__ __forceinline__ void tm_fwd_e_run(const TiledFwd<T>& P, const TmBuf<T>& f, const TmGeom& tg, unsigned blk) {
  const WarpPos wp = warp_pos(tg, P.a.g.nshot, blk);
  if (!wp.live) return;
  if (wp.kind == kFrameXLean) tm_fwd_e_body<T, R, kFrameXLean>(P, f, tg, wp);
  else if (wp.kind == kFrameYLean) tm_fwd_e_body<T, R, kFrameYLean>(P, f, tg, wp);
  else tm_fwd_e_body<T, R, kFrameGeneral>(P, f, tg, wp);
}

template <typename T, int R>
__global__ void __launch_bounds__(32 * TM_WARPS) tm_fwd_e(TiledFwd<T> P, TmBuf<T> f, TmGeom tg) {
  tm_fwd_e_run<T, R>(P, f, tg, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Adjoint channel weights of a source cell (ii, jj), general form with CPML.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T tmw_e_chan(const AdjArgs<T>& a, const TmBuf<T>& t, int NYP, int ch, int s, int ii,
                                        int jj) {
  const Grid& g = a.g;
  if (ii < 0 || jj < 0 || ii >= g.NX || jj >= g.NY) return T(0);
  const long long c = (long long)ii * NYP + jj;
  const long long f = (long long)s * g.NX * NYP + c;
  T w = T(0);
  if (ch == 2) {
    if (a.has_cpml) add_pml<T, true>(w, a.eF[0], a.eF[1], g, 0, 2, s, ii, jj, 0);
    if (tm_upd_ez(g, ii, jj)) w += t.ce_curl[c] * t.Ez[f];
  } else {
    if (a.has_cpml) add_pml<T, true>(w, a.eF[2], a.eF[3], g, 1, 2, s, ii, jj, 0);
    if (tm_upd_ez(g, ii, jj)) w += (-t.ce_curl_y[c]) * t.Ez[f];
  }
  return w;
}

template <typename T>
__device__ __forceinline__ T tmw_h_chan(const AdjArgs<T>& a, const TmBuf<T>& t, int NYP, int ch, int s, int ii,
                                        int jj) {
  const Grid& g = a.g;
  if (ii < 0 || jj < 0 || ii >= g.NX || jj >= g.NY) return T(0);
  const long long c = (long long)ii * NYP + jj;
  const long long f = (long long)s * g.NX * NYP + c;
  T w = T(0);
  if (ch == 0) {
    if (a.has_cpml) add_pml<T, false>(w, a.hF[0], a.hF[1], g, 0, 1, s, ii, jj, 0);
    if (tm_upd_hy(g, ii, jj)) w += t.ch_curl[c] * t.Hy[f];
  } else {
    if (a.has_cpml) add_pml<T, false>(w, a.hF[2], a.hF[3], g, 1, 1, s, ii, jj, 0);
    if (tm_upd_hx(g, ii, jj)) w += (-t.ch_curl_y[c]) * t.Hx[f];
  }
  return w;
}

// ---------------------------------------------------------------------------
// Adjoint E step: lambda_Hy += gather_x(B_X), lambda_Hx += gather_y(C_Y);
// H-CPML weights of step it.  B_X = c lambda_Ez, C_Y = -c_y lambda_Ez.
// ---------------------------------------------------------------------------
template <typename T, int R, int FK>
__device__ __forceinline__ void tm_adj_e_body(const TiledAdj<T>& P, const TmBuf<T>& t, const TmGeom& tg, const WarpPos& wp) {
  constexpr bool XL = FK == kFrameXLean, YL = FK == kFrameYLean;
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const int lane = wp.lane, s = wp.s;
  const int j = wp.base + lane;
  const bool cv = j < NY;
  const int hj = halo_col<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  const T* __restrict__ lEz = t.Ez + s * plane;
  T* __restrict__ lHx = t.Hx + s * plane;
  T* __restrict__ lHy = t.Hy + s * plane;
  const T* __restrict__ cc = t.ce_curl;
  const int qy0 = (!YL && cv && a.has_cpml) ? q_low_h(a.hF[2].p, j) : -1;
  const int qy1 = (!YL && cv && a.has_cpml) ? q_high(a.hF[3].p, j, NY) : -1;
  // strip (with its gather halo) away from the y ends and the E y-slabs:
  // C_Y has no CPML part and the full interior gather applies
  const int pyl = a.has_cpml ? a.eF[2].p : 0, pyh = a.has_cpml ? a.eF[3].p : 0;
  const bool seg_int = YL || (wp.base - (R - 1) > pyl && wp.base >= 2 * R - 1 &&
                              wp.base + TMW - 1 + R < NY - 1 - pyh && wp.base + TMW - 1 + 2 * R - 1 < NY);
  const bool colz = j > 0 && j < NY - 1;   // column part of tm_upd_ez
  T qB[2 * R];   // B_X at rows i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) qB[m] = cv ? tmw_e_chan(a, t, NYP, 2, s, wp.x0 - R + 1 + m, j) : T(0);
  T n_bz, n_bc, n_z, n_c, n_hz, n_hc, n_hx, n_hy;   // operands of the next row
  auto fetch = [&](int i) {
    const long long rw = (long long)i * NYP;
    const bool nb = i + R < NX;
    n_bz = nb ? lEz[rw + (long long)R * NYP + j] : T(0);
    n_bc = nb ? cc[rw + (long long)R * NYP + j] : T(0);
    n_z = lEz[rw + j];
    n_c = t.ce_curl_y[rw + j];
    n_hz = hok ? lEz[rw + hj] : T(0);
    n_hc = hok ? t.ce_curl_y[rw + hj] : T(0);
    n_hx = lHx[rw + j];
    n_hy = lHy[rw + j];
  };
  fetch(wp.x0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    const T bz = n_bz, bcc = n_bc, z = n_z, c = n_c, hz = n_hz, hc = n_hc;
    T hxv = n_hx, hyv = n_hy;
    if (i + 1 < wp.x1) fetch(i + 1);
    const long long rw = (long long)i * NYP;
    // B_X of row i+R: E x-face slab position of that row (its CPML part)
    const int qx0 = (!XL && a.has_cpml) ? q_low_e(a.eF[0].p, i + R) : -1;
    const int qx1 = (!XL && a.has_cpml) ? q_high(a.eF[1].p, i + R, NX) : -1;
    if (seg_int && (XL || (i + R < NX - 1 && i + R > 0 && qx0 < 0 && qx1 < 0))) {
      qB[2 * R - 1] = bcc * bz;
    } else if (XL) {
      // row i+R has no x CPML and updates Ez: the general weight without the face lookups
      T w = T(0);
      if (cv && colz) w += bcc * bz;
      qB[2 * R - 1] = w;
    } else {
      qB[2 * R - 1] = cv ? tmw_e_chan(a, t, NYP, 2, s, i + R, j) : T(0);
    }
    T cy_own, cy_halo;
    if (seg_int && i > 0 && i < NX - 1) {
      cy_own = (-c) * z;
      cy_halo = hok ? (-hc) * hz : T(0);
    } else {
      cy_own = cv ? tmw_e_chan(a, t, NYP, 4, s, i, j) : T(0);
      cy_halo = hok ? tmw_e_chan(a, t, NYP, 4, s, i, hj) : T(0);
    }
    T yv[2 * R];   // C_Y at columns j + d, d = -(R-1) .. R
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) yv[d + R - 1] = d == 0 ? cy_own : ynb<T, R>(cy_own, cy_halo, lane, d);
    if (cv) {
      const auto wx = [&](int d) { return qB[R - 1 + d]; };
      const auto wy = [&](int d) { return yv[d + R - 1]; };
      hyv += XL ? gather_back_full<T, R>(wx) : gback<T, R>(wx, i, NX);
      hxv += YL ? gather_back_full<T, R>(wy) : gback<T, R>(wy, j, NY);
      lHx[rw + j] = hxv;
      lHy[rw + j] = hyv;
      const int qh0 = (!XL && a.has_cpml) ? q_low_h(a.hF[0].p, i) : -1;
      const int qh1 = (!XL && a.has_cpml) ? q_high(a.hF[1].p, i, NX) : -1;
      if (qh0 >= 0 || qh1 >= 0 || qy0 >= 0 || qy1 >= 0) {
        const T up_h = t.ch_rhs[rw + j];
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qh0 : qh1;
          if (qq < 0) continue;
          const Face<T>& F = a.hF[fc];
          const long long pi = ((long long)s * F.p + qq) * NY + j;
          F.w1[pi] = pml_weight(hyv, a.inv_dx, up_h, T(1), prof(F, qq), &F.psi1[pi]);
        }
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qy0 : qy1;
          if (qq < 0) continue;
          const Face<T>& F = a.hF[2 + fc];
          const long long pi = ((long long)s * NX + i) * F.p + qq;
          F.w1[pi] = pml_weight(hxv, a.inv_dy, up_h, T(-1), prof(F, qq), &F.psi1[pi]);
        }
      }
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) qB[m] = qB[m + 1];
  }
}

template <typename T, int R>
__device__ __forceinline__ void tm_adj_e_run(const TiledAdj<T>& P, const TmBuf<T>& t, const TmGeom& tg, unsigned blk) {
  const AdjArgs<T>& a = P.a;
  if (a.want_src && tg.sum_source && blk == 0 && threadIdx.y == 0) {
    // waveform gradient of step it: shots summed in order (deepgpr_cpu.c:1524-1533)
    const int it = a.ctrl->cur - a.k_in_chunk;
    for (int m = threadIdx.x; m < a.nsrc; m += 32) {
      T acc = a.grad_source[(long long)m * a.nt + it];
      for (int s = 0; s < a.g.nshot; ++s) acc += a.srcv[(long long)s * a.nsrc + m];
      a.grad_source[(long long)m * a.nt + it] = acc;
    }
  }
  const WarpPos wp = warp_pos(tg, a.g.nshot, blk);
  if (!wp.live) return;
  if (wp.kind == kFrameXLean) tm_adj_e_body<T, R, kFrameXLean>(P, t, tg, wp);
  else if (wp.kind == kFrameYLean) tm_adj_e_body<T, R, kFrameYLean>(P, t, tg, wp);
  else tm_adj_e_body<T, R, kFrameGeneral>(P, t, tg, wp);
}

template <typename T, int R>
__global__ void __launch_bounds__(32 * TM_WARPS) tm_adj_e(TiledAdj<T> P, TmBuf<T> t, TmGeom tg) {
  tm_adj_e_run<T, R>(P, t, tg, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Adjoint H step: lambda_Ez <- ce_hist lambda_Ez + gather_x(A_X) + gather_y(A_Y);
// head of step it-1 (receivers^T, staged source terms, E-CPML weights).
// A_X = c lambda_Hy, A_Y = -c_y lambda_Hx.  PROLOGUE runs only the head of
// step nt-1.
// ---------------------------------------------------------------------------
template <typename T, int R, bool PROLOGUE, int FK>
__device__ __forceinline__ void tm_adj_h_body(const TiledAdj<T>& P, const TmBuf<T>& t, const TmGeom& tg,
                                              const WarpPos& wp) {
  constexpr bool XL = FK == kFrameXLean, YL = FK == kFrameYLean;
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const int lane = wp.lane, s = wp.s;
  const int j = wp.base + lane;
  const bool cv = j < NY;
  const int hj = halo_col<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  T* __restrict__ lEz = t.Ez + s * plane;
  const T* __restrict__ lHx = t.Hx + s * plane;
  const T* __restrict__ lHy = t.Hy + s * plane;
  const T* __restrict__ hc = t.ch_curl;
  const T* __restrict__ c0p = t.ce_hist;
  const int it = a.ctrl->cur - a.k_in_chunk;
  const int head = PROLOGUE ? it : it - 1;
  const int qy0 = (!YL && cv && a.has_cpml && j > 0) ? q_low_e(a.eF[2].p, j) : -1;
  const int qy1 = (!YL && cv && a.has_cpml && j > 0) ? q_high(a.eF[3].p, j, NY) : -1;
  const int pyl = a.has_cpml ? a.hF[2].p : 0, pyh = a.has_cpml ? a.hF[3].p : 0;
  const bool seg_int = YL || (wp.base - R >= pyl && wp.base >= 2 * R - 1 && wp.base > 0 &&
                              wp.base + TMW - 1 + R - 1 < NY - 1 - pyh && wp.base + TMW - 1 + 2 * R <= NY);
  const bool colhy = NY - 1 != 1 && j > 0 && j < NY - 1;   // column part of tm_upd_hy
  T qA[2 * R];   // A_X at rows i-R .. i+R-1
  if (!PROLOGUE) {
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) qA[m] = cv ? tmw_h_chan(a, t, NYP, 0, s, wp.x0 - R + m, j) : T(0);
  }
  T n_ay = T(0), n_ac = T(0), n_x = T(0), n_c = T(0), n_hx = T(0), n_hc = T(0), n_ez, n_c0 = T(0);   // next row
  auto fetch = [&](int i) {
    const long long rw = (long long)i * NYP;
    n_ez = lEz[rw + j];
    if (!PROLOGUE) {
      const bool nb = i + R - 1 < NX;
      n_ay = nb ? lHy[rw + (long long)(R - 1) * NYP + j] : T(0);
      n_ac = nb ? hc[rw + (long long)(R - 1) * NYP + j] : T(0);
      n_x = lHx[rw + j];
      n_c = t.ch_curl_y[rw + j];
      n_hx = hok ? lHx[rw + hj] : T(0);
      n_hc = hok ? t.ch_curl_y[rw + hj] : T(0);
      n_c0 = c0p[rw + j];
    }
  };
  fetch(wp.x0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    const T ay = n_ay, ac = n_ac, x = n_x, c = n_c, hx = n_hx, hcc = n_hc, c0 = n_c0;
    T ez = n_ez;
    if (i + 1 < wp.x1) fetch(i + 1);
    const long long rw = (long long)i * NYP;
    if (!PROLOGUE) {
      const int r1 = i + R - 1;
      const int qh0 = (!XL && a.has_cpml) ? q_low_h(a.hF[0].p, r1) : -1;
      const int qh1 = (!XL && a.has_cpml) ? q_high(a.hF[1].p, r1, NX) : -1;
      if (seg_int && (XL || (r1 < NX - 1 && qh0 < 0 && qh1 < 0))) {
        qA[2 * R - 1] = ac * ay;
      } else if (XL) {
        // row r1 has no x CPML and updates Hy: the general weight without the face lookups
        T w = T(0);
        if (cv && colhy) w += ac * ay;
        qA[2 * R - 1] = w;
      } else {
        qA[2 * R - 1] = cv ? tmw_h_chan(a, t, NYP, 0, s, r1, j) : T(0);
      }
      T ay_own, ay_halo;
      if (seg_int && i > 0 && i < NX - 1) {
        ay_own = (-c) * x;
        ay_halo = hok ? (-hcc) * hx : T(0);
      } else {
        ay_own = cv ? tmw_h_chan(a, t, NYP, 1, s, i, j) : T(0);
        ay_halo = hok ? tmw_h_chan(a, t, NYP, 1, s, i, hj) : T(0);
      }
      T yv[2 * R];   // A_Y at columns j + d, d = -R .. R-1
#pragma unroll
      for (int d = -R; d <= R - 1; ++d) yv[d + R] = d == 0 ? ay_own : ynb<T, R>(ay_own, ay_halo, lane, d);
      if (cv) {
        // tm_upd_ez split into row and column parts (true on lean rows / tiles)
        const bool dez = (XL || YL || g.NX - 1 != 1 || g.NY - 1 != 1) && (XL || (i > 0 && i < NX - 1)) &&
                         (YL || (j > 0 && j < NY - 1));
        if (dez) ez = c0 * ez;
        const auto wx = [&](int d) { return qA[R + d]; };
        const auto wy = [&](int d) { return yv[d + R]; };
        ez += XL ? gather_fwd_full<T, R>(wx) : gfwd<T, R>(wx, i, NX);
        ez += YL ? gather_fwd_full<T, R>(wy) : gfwd<T, R>(wy, j, NY);
      }
    }
    if (head >= 0 && cv) {
      const bool row_pts = (tg.rcv_rows && a.rx_comp == 2 && tg.rcv_rows[(long long)s * NX + i]) ||
                           (tg.src_rows && a.want_src && tg.src_rows[(long long)s * NX + i]);
      if (row_pts) {
        const int cfull = i * g.sx + j * g.NZ;
        if (a.rx_comp == 2 && point_hit(P.rcv, s, cfull)) {
          const int row = point_row(P.rcv, cfull);
          for (int e = a.rcv.off[row]; e < a.rcv.off[row + 1]; ++e)
            if (a.rcv.shot[e] == s) ez += a.data_grad[((long long)s * a.nt + head) * a.nrx + a.rcv.idx[e]];
        }
        if (a.want_src && point_hit(P.src, s, cfull)) {
          const int row = point_row(P.src, cfull);
          for (int e = a.src.off[row]; e < a.src.off[row + 1]; ++e)
            if (a.src.shot[e] == s)
              a.srcv[(long long)s * a.nsrc + a.src.idx[e]] = -t.ce_rhs[rw + j] * a.src_geo * ez;
        }
      }
      const int qx0 = (!XL && a.has_cpml && i > 0) ? q_low_e(a.eF[0].p, i) : -1;
      const int qx1 = (!XL && a.has_cpml && i > 0) ? q_high(a.eF[1].p, i, NX) : -1;
      if (qx0 >= 0 || qx1 >= 0 || qy0 >= 0 || qy1 >= 0) {
        const T up_e = t.ce_rhs[rw + j];
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qx0 : qx1;
          if (qq < 0) continue;
          const Face<T>& F = a.eF[fc];
          const long long pi = ((long long)s * (F.p + 1) + qq) * NY + j;
          F.w2[pi] = pml_weight(ez, a.inv_dx, up_e, T(1), prof(F, qq), &F.psi2[pi]);
        }
#pragma unroll
        for (int fc = 0; fc < 2; ++fc) {
          const int qq = fc == 0 ? qy0 : qy1;
          if (qq < 0) continue;
          const Face<T>& F = a.eF[2 + fc];
          const long long pi = ((long long)s * NX + i) * (F.p + 1) + qq;
          F.w2[pi] = pml_weight(ez, a.inv_dy, up_e, T(-1), prof(F, qq), &F.psi2[pi]);
        }
      }
    }
    if (cv) lEz[rw + j] = ez;
    if (!PROLOGUE) {
#pragma unroll
      for (int m = 0; m < 2 * R - 1; ++m) qA[m] = qA[m + 1];
    }
  }
}

template <typename T, int R, bool PROLOGUE>
__device__ __forceinline__ void tm_adj_h_run(const TiledAdj<T>& P, const TmBuf<T>& t, const TmGeom& tg, unsigned blk) {
  const WarpPos wp = warp_pos(tg, P.a.g.nshot, blk);
  if (!wp.live) return;
  if (PROLOGUE) {
    tm_adj_h_body<T, R, true, kFrameGeneral>(P, t, tg, wp);
  } else {
    if (wp.kind == kFrameXLean) tm_adj_h_body<T, R, false, kFrameXLean>(P, t, tg, wp);
    else if (wp.kind == kFrameYLean) tm_adj_h_body<T, R, false, kFrameYLean>(P, t, tg, wp);
    else tm_adj_h_body<T, R, false, kFrameGeneral>(P, t, tg, wp);
  }
}

template <typename T, int R, bool PROLOGUE>
__global__ void __launch_bounds__(32 * TM_WARPS) tm_adj_h(TiledAdj<T> P, TmBuf<T> t, TmGeom tg) {
  tm_adj_h_run<T, R, PROLOGUE>(P, t, tg, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Imaging condition of one saved step, 2D TM (deepgpr_cpu.c:1659-1745),
// lambda_Ez compact with pitch NYP.  One thread per history-box cell sums
// every shot in order (FP32 in the reference's order, or FP64 when ACC64).
// Shots are read in batches of four, the next batch's loads issued before
// the current batch is consumed; the per-shot work is branch-free (the PEC
// and wanted-gradient conditions are per cell and applied once at the end).
// KIND / EONLY fix the history format at compile time.
// ---------------------------------------------------------------------------
constexpr int kImageThreads = 128;

template <typename T, int KIND, bool EONLY, bool ACC64>
__global__ void __launch_bounds__(kImageThreads) tm_image(AdjArgs<T> a, const T* __restrict__ lam, int NYP,
                                                          int nseg) {
  constexpr int U = 4;
  const Grid& g = a.g;
  const int it = a.ctrl->cur - a.k_in_chunk;
  if (it % a.S != 0) return;
  const int slot = it / a.S;
  const long long bc = a.box.cells();
  const long long hidx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (hidx >= bc) return;
  const int i = int(hidx / a.box.ny) + a.box.x0, j = int(hidx % a.box.ny) + a.box.y0;
  const int c = i * g.sx + j * g.NZ;
  const long long gi = (long long)i * (g.NY - 1) + j;
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
  const bool dez = upd_ez(g, i, j, 0);
  const T aeff = dez ? ca : T(1);
  const int nshot = g.nshot;
  const bool last = slot + 1 >= a.nt_saved;   // E-only: E^(n+1) of the last frame is in R_saved
  const T* __restrict__ pl = lam + (long long)i * NYP + j;
  const long long lstride = (long long)g.NX * NYP;
  const void* nbase = (EONLY && !last) ? a.E_saved : a.R_saved;
  const long long ie0 = (long long)slot * a.frame + hidx;
  const long long in0 = EONLY ? (last ? hidx : ie0 + a.frame) : ie0;
  const long long sc0 = (long long)slot * nshot * a.ntiles + (long long)i * nseg + j / TMW;
  T acc_e = T(0), acc_s = T(0);
  double acc_e64 = 0.0, acc_s64 = 0.0;
  auto term = [&](T lv, T eo, T sec) {
    T rhs = sec;
    if (EONLY) rhs = cbv != T(0) ? div_fixed(sec - aeff * eo, dcb) : T(0);
    const T lamx = (eo == T(0) && rhs == T(0)) ? T(0) : lv;
    const T gca = dez ? lamx * eo * wgt : T(0);
    const T gcb = lamx * rhs * wgt;
    const T te = gca * dca_e + gcb * dcb_e;
    const T ts = gca * dca_s + gcb * dcb_s;
    if (ACC64) {
      acc_e64 += double(te);
      acc_s64 += double(ts);
    } else {
      acc_e += te;
      acc_s += ts;
    }
  };
  auto load1 = [&](long long so, T& l, T& e, T& n) {
    float esc = 1.0f, rsc = 1.0f;
    if (is_tiled(KIND)) {
      esc = a.e_scales[sc0 + so * a.ntiles];
      if (!EONLY) rsc = a.r_scales[sc0 + so * a.ntiles];
    }
    l = pl[so * lstride];
    e = hist_load<T>(a.E_saved, ie0 + so * bc, KIND, esc);
    n = hist_load<T>(nbase, in0 + so * bc, KIND, rsc);
  };
  T la[U], ea[U], na[U], lb[U], eb[U], nb[U];
  const int nfull = nshot / U * U;
#pragma unroll
  for (int u = 0; u < U; ++u)
    if (nfull > 0) load1(u, la[u], ea[u], na[u]);
  for (int s0 = 0; s0 < nfull; s0 += 2 * U) {
    if (s0 + U < nfull) {
#pragma unroll
      for (int u = 0; u < U; ++u) load1(s0 + U + u, lb[u], eb[u], nb[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) term(la[u], ea[u], na[u]);
    if (s0 + U >= nfull) break;
    if (s0 + 2 * U < nfull) {
#pragma unroll
      for (int u = 0; u < U; ++u) load1(s0 + 2 * U + u, la[u], ea[u], na[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) term(lb[u], eb[u], nb[u]);
  }
  for (int s = nfull; s < nshot; ++s) {
    T l, e, n;
    load1(s, l, e, n);
    term(l, e, n);
  }
  if (!pec_ok) {
    acc_e = acc_s = T(0);
    acc_e64 = acc_s64 = 0.0;
  }
  if (a.want_eps) {
    if (ACC64) a.g_eps64[gi] += acc_e64; else a.g_eps[gi] += acc_e;
  }
  if (a.want_sig) {
    if (ACC64) a.g_sig64[gi] += acc_s64; else a.g_sig[gi] += acc_s;
  }
}

// ===========================================================================
// Interior kernels (tmi_*).  Every cell of the launch's single rectangle
// takes the full-stencil, CPML-free form of its half step: the host picks the
// rectangle with tm_lean_ok, which states for each kernel the conditions
// under which the general kernel's per-cell code reduces to that form.  So
// these kernels carry no boundary logic.  Two rows per iteration; the
// operands of the next pair are loaded before the current pair is computed.
// Rows holding a source or receiver of any shot are left to the general
// kernels; history frames are written inline in the general kernels' order.
// ===========================================================================

// CPML thickness of the x (rows) and y (columns) faces, 0 without CPML.
struct TmFaces {
  int hx0, hx1, hy0, hy1, ex0, ex1, ey0, ey1;
};

__host__ __device__ inline bool tm_no_e_pml(int p0, int p1, int c, int n) {
  return !(c > 0 && (q_low_e(p0, c) >= 0 || q_high(p1, c, n) >= 0));
}
__host__ __device__ inline bool tm_no_h_pml(int p0, int p1, int c, int n) {
  return q_low_h(p0, c) < 0 && q_high(p1, c, n) < 0;
}

// kind 0 forward H, 1 forward E, 2 adjoint E step, 3 adjoint H step;
// axis 0: row c of n = NX rows (x faces), axis 1: column c of n = NY.
__host__ __device__ inline bool tm_lean_ok(int kind, int axis, int c, int n, int R, const TmFaces& f) {
  const int h0 = axis == 0 ? f.hx0 : f.hy0, h1 = axis == 0 ? f.hx1 : f.hy1;
  const int e0 = axis == 0 ? f.ex0 : f.ey0, e1 = axis == 0 ? f.ex1 : f.ey1;
  if (n - 1 == 1) return false;
  switch (kind) {
    case 0:   // Hx, Hy update (tm_upd_hx/hy), dfwd full, no H-CPML
      return c > 0 && c < n - 1 && tm_no_h_pml(h0, h1, c, n) && c - R + 1 >= 0 && c + R < n;
    case 1:   // Ez update (tm_upd_ez), dback full, no E-CPML
      return c > 0 && c < n - 1 && tm_no_e_pml(e0, e1, c, n) && c >= R && c + R - 1 < n;
    case 2: {   // gather_back full of E channels (sources c-R+1 .. c+R), no H-CPML weights
      if (!(c >= 2 * R - 1 && c + 2 * R - 1 < n && c > 0 && c < n - 1 && tm_no_h_pml(h0, h1, c, n))) return false;
      for (int r = c - R + 1; r <= c + R; ++r)
        if (!(r > 0 && r < n - 1 && tm_no_e_pml(e0, e1, r, n))) return false;
      return true;
    }
    default: {   // gather_fwd full of H channels (sources c-R .. c+R-1), Ez scaling, no E-CPML head
      if (!(c >= 2 * R - 1 && c + 2 * R <= n && c > 0 && c < n - 1 && tm_no_e_pml(e0, e1, c, n))) return false;
      for (int r = c - R; r <= c + R - 1; ++r)
        if (!(r < n - 1 && tm_no_h_pml(h0, h1, r, n))) return false;
      return true;
    }
  }
}

// Four columns per lane: lane l of a 128-column interior strip holds columns
// base + 4l .. base + 4l + 3 (one 16-byte access per array and row for FP32).
template <typename T>
__device__ __forceinline__ void ld4(const T* p, T (&o)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  } else {
    const double2 v0 = reinterpret_cast<const double2*>(p)[0], v1 = reinterpret_cast<const double2*>(p)[1];
    o[0] = v0.x; o[1] = v0.y; o[2] = v1.x; o[3] = v1.y;
  }
}
template <typename T>
__device__ __forceinline__ void st4(T* p, const T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
  }
}

// Halo column of a lane of a 128-column strip: lanes [0, R) hold
// base - R + lane, lanes [R, 2R) hold base + 128 + lane - R.
template <int R>
__device__ __forceinline__ int halo_col4(int base, int lane) {
  return lane < R ? base - R + lane : base + 4 * TMW + lane - R;
}

// Value at column base + 4 lane + m (-R <= m <= R + 3) from the lanes' own
// quadruples v and the halo lanes.  All lanes call it with the same m.
template <typename T, int R>
__device__ __forceinline__ T ynb4(const T (&v)[4], T halo, int lane, int m) {
  if (m >= 0 && m <= 3) return v[m];
  if (m < 0) {
    const T a = __shfl_up_sync(kFullMask, v[(4 + m) & 3], 1);
    const T b = __shfl_sync(kFullMask, halo, m + R);
    return lane == 0 ? b : a;
  }
  const T a = __shfl_down_sync(kFullMask, v[(m - 4) & 3], 1);
  const T b = __shfl_sync(kFullMask, halo, R + m - 4);
  return lane == 31 ? b : a;
}

// absmax over the 8 lanes of one 32-column FP8 tile
__device__ __forceinline__ float tile8_absmax(float v) {
  for (int o = 4; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFullMask, v, o));
  return v;
}

// Interior forward H.
template <typename T, int R>
__device__ __forceinline__ void tmi_fwd_h_run(const TiledFwd<T>& P, const TmBuf<T>& f, const TmGeom& tg, unsigned blk) {
  constexpr int MLO = -(R - 1), MHI = R + 3, NM = MHI - MLO + 1;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const WarpPos wp = warp_pos(tg, g.nshot, blk);
  if (!wp.live) return;
  const int lane = wp.lane, s = wp.s, x0 = wp.x0, x1 = wp.x1;
  const int j = wp.base + 4 * lane;
  const bool act = wp.base + TMW * (lane >> 3) < tg.col1;   // this lane's 32-column tile is interior
  const int hj = halo_col4<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  const T* __restrict__ Ezj = f.Ez + s * plane + j;
  const T* __restrict__ Ezh = f.Ez + s * plane + (hok ? hj : 0);
  T* __restrict__ Hxj = f.Hx + s * plane + j;
  T* __restrict__ Hyj = f.Hy + s * plane + j;
  const T* __restrict__ ccj = f.ch_curl + j;
  const T* __restrict__ cyj = f.ch_curl_y + j;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save = a.save_e && (it % a.S == 0);
  const int slot = it / a.S;
  const long long hbase = (long long)slot * a.frame + s * a.box.cells();
  const int bj = j - a.box.y0;
  const int RN = R * NYP;
  T q[2 * R][4];   // Ez at rows i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) ld4(Ezj + (x0 - R + 1 + m) * NYP, q[m]);
  T ne[4], nhx[4], nhy[4], nc[4], ncy[4], nh = T(0);
  auto fetch = [&](int o) {   // o = offset of the row
    ld4(Ezj + o + RN, ne);
    if (hok) nh = Ezh[o];
    ld4(Hxj + o, nhx);
    ld4(Hyj + o, nhy);
    ld4(ccj + o, nc);
    ld4(cyj + o, ncy);
  };
  fetch(x0 * NYP);
  for (int i = x0; i < x1; ++i) {
    const int o = i * NYP;
    T hx[4], hy[4], c1[4], cy[4];
    const T hl = nh;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      q[2 * R - 1][e] = ne[e];
      hx[e] = nhx[e];
      hy[e] = nhy[e];
      c1[e] = nc[e];
      cy[e] = ncy[e];
    }
    if (i + 1 < x1) fetch(o + NYP);
    T y[NM];   // Ez at columns j + m
#pragma unroll
    for (int m = MLO; m <= MHI; ++m) y[m - MLO] = ynb4<T, R>(q[R - 1], hl, lane, m);
    if (save) {
      const int bi = i - a.box.x0;
      const bool rin = act && bi >= 0 && bi < a.box.nx;
      bool ib[4];
      float am = 0.0f;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        ib[e] = rin && bj + e >= 0 && bj + e < a.box.ny;
        if (ib[e]) am = fmaxf(am, fabsf(float(q[R - 1][e])));
      }
      float inv = 1.0f;
      if (is_tiled(a.kind)) {
        const float sc = tile_scale_of(a.kind, tile8_absmax(am));
        inv = 1.0f / sc;
        if (act && (lane & 7) == 0)
          a.e_scales[((long long)slot * g.nshot + s) * a.ntiles + (long long)i * tg.nseg + wp.seg + (lane >> 3)] = sc;
      }
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (ib[e]) hist_store<T>(a.E_saved, hbase + (long long)bi * a.box.ny + bj + e, q[R - 1][e], a.kind, inv);
    }
    T ox[4], oy[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const T dEz_dy = dfwd_full<T, R>([&](int d) { return y[e + d - MLO]; });
      const T dEz_dx = dfwd_full<T, R>([&](int d) { return q[R - 1 + d][e]; });
      ox[e] = hx[e] - cy[e] * dEz_dy;
      oy[e] = hy[e] + c1[e] * dEz_dx;
    }
    if (act) {
      st4(Hxj + o, ox);
      st4(Hyj + o, oy);
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 4; ++e) q[m][e] = q[m + 1][e];
  }
}

// Interior forward E (+ R^n history).  Rows holding sources or receivers are
// frame rows.
template <typename T, int R>
__device__ __forceinline__ void tmi_fwd_e_run(const TiledFwd<T>& P, const TmBuf<T>& f, const TmGeom& tg, unsigned blk) {
  constexpr int MLO = -R, MHI = R + 2, NM = MHI - MLO + 1;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const WarpPos wp = warp_pos(tg, g.nshot, blk);
  if (!wp.live) return;
  const int lane = wp.lane, s = wp.s, x0 = wp.x0, x1 = wp.x1;
  const int j = wp.base + 4 * lane;
  const bool act = wp.base + TMW * (lane >> 3) < tg.col1;
  const int hj = halo_col4<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  T* __restrict__ Ezj = f.Ez + s * plane + j;
  const T* __restrict__ Hxj = f.Hx + s * plane + j;
  const T* __restrict__ Hxh = f.Hx + s * plane + (hok ? hj : 0);
  const T* __restrict__ Hyj = f.Hy + s * plane + j;
  const T* __restrict__ c0j = f.ce_hist + j;
  const T* __restrict__ c1j = f.ce_curl + j;
  const T* __restrict__ cyj = f.ce_curl_y + j;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save_r = a.keep_r && (it % a.S == 0);
  const int slot = it / a.S;
  const long long hbase = (long long)slot * a.frame + s * a.box.cells();
  const int bj = j - a.box.y0;
  const int RN = (R - 1) * NYP;
  T q[2 * R][4];   // Hy at rows i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) ld4(Hyj + (x0 - R + m) * NYP, q[m]);
  T ny[4], nx[4], nez[4], nc0[4], nc1[4], ncy[4], nh = T(0);
  auto fetch = [&](int o) {
    ld4(Hyj + o + RN, ny);
    ld4(Hxj + o, nx);
    if (hok) nh = Hxh[o];
    ld4(Ezj + o, nez);
    ld4(c0j + o, nc0);
    ld4(c1j + o, nc1);
    ld4(cyj + o, ncy);
  };
  fetch(x0 * NYP);
  for (int i = x0; i < x1; ++i) {
    const int o = i * NYP;
    T hxo[4], ez0[4], c0[4], c1[4], cy[4];
    const T hl = nh;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      q[2 * R - 1][e] = ny[e];
      hxo[e] = nx[e];
      ez0[e] = nez[e];
      c0[e] = nc0[e];
      c1[e] = nc1[e];
      cy[e] = ncy[e];
    }
    if (i + 1 < x1) fetch(o + NYP);
    T y[NM];   // Hx at columns j + m
#pragma unroll
    for (int m = MLO; m <= MHI; ++m) y[m - MLO] = ynb4<T, R>(hxo, hl, lane, m);
    T ez[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const T dHy_dx = dback_full<T, R>([&](int d) { return q[R + d][e]; });
      const T dHx_dy = dback_full<T, R>([&](int d) { return y[e + d - MLO]; });
      ez[e] = c0[e] * ez0[e] + c1[e] * dHy_dx - cy[e] * dHx_dy;
    }
    if (save_r) {
      // R^n = (E^{n+1} - ce_hist E^n) / cb (deepgpr_cpu.c:1850-1875)
      const int bi = i - a.box.x0;
      const bool rin = act && bi >= 0 && bi < a.box.nx;
      T cb[4], rv[4];
      bool ib[4];
      float am = 0.0f;
      ld4(f.ce_rhs + j + o, cb);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        ib[e] = rin && bj + e >= 0 && bj + e < a.box.ny;
        rv[e] = T(0);
        if (ib[e]) {
          rv[e] = cb[e] != T(0) ? (ez[e] - c0[e] * ez0[e]) / cb[e] : T(0);
          am = fmaxf(am, fabsf(float(rv[e])));
        }
      }
      float inv = 1.0f;
      if (is_tiled(a.kind)) {
        const float sc = tile_scale_of(a.kind, tile8_absmax(am));
        if (act && (lane & 7) == 0)
          a.r_scales[((long long)slot * g.nshot + s) * a.ntiles + (long long)i * tg.nseg + wp.seg + (lane >> 3)] = sc;
        inv = 1.0f / sc;
      }
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (ib[e]) hist_store<T>(a.R_saved, hbase + (long long)bi * a.box.ny + bj + e, rv[e], a.kind, inv);
    }
    if (act) st4(Ezj + o, ez);
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 4; ++e) q[m][e] = q[m + 1][e];
  }
}

// Interior adjoint E step.
template <typename T, int R>
__device__ __forceinline__ void tmi_adj_e_run(const TiledAdj<T>& P, const TmBuf<T>& t, const TmGeom& tg, unsigned blk) {
  constexpr int MLO = -(R - 1), MHI = R + 3, NM = MHI - MLO + 1;
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const WarpPos wp = warp_pos(tg, g.nshot, blk);
  if (!wp.live) return;
  const int lane = wp.lane, s = wp.s, x0 = wp.x0, x1 = wp.x1;
  const int j = wp.base + 4 * lane;
  const bool act = wp.base + TMW * (lane >> 3) < tg.col1;
  const int hj = halo_col4<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  const T* __restrict__ lEzj = t.Ez + s * plane + j;
  const T* __restrict__ lEzh = t.Ez + s * plane + (hok ? hj : 0);
  T* __restrict__ lHxj = t.Hx + s * plane + j;
  T* __restrict__ lHyj = t.Hy + s * plane + j;
  const T* __restrict__ ccj = t.ce_curl + j;
  const T* __restrict__ cyj = t.ce_curl_y + j;
  const T* __restrict__ cyh = t.ce_curl_y + (hok ? hj : 0);
  const int RN = R * NYP;
  T qB[2 * R][4];   // B_X = c lambda_Ez at rows i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int o = (x0 - R + 1 + m) * NYP;
    T z[4], c[4];
    ld4(lEzj + o, z);
    ld4(ccj + o, c);
#pragma unroll
    for (int e = 0; e < 4; ++e) qB[m][e] = c[e] * z[e];
  }
  T nbz[4], nbc[4], nz[4], ncy[4], nhx[4], nhy[4], nhz = T(0), nhc = T(0);
  auto fetch = [&](int o) {
    ld4(lEzj + o + RN, nbz);
    ld4(ccj + o + RN, nbc);
    ld4(lEzj + o, nz);
    ld4(cyj + o, ncy);
    if (hok) {
      nhz = lEzh[o];
      nhc = cyh[o];
    }
    ld4(lHxj + o, nhx);
    ld4(lHyj + o, nhy);
  };
  fetch(x0 * NYP);
  for (int i = x0; i < x1; ++i) {
    const int o = i * NYP;
    T cy[4], hx[4], hy[4];
    const T hcy = hok ? (-nhc) * nhz : T(0);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      qB[2 * R - 1][e] = nbc[e] * nbz[e];
      cy[e] = (-ncy[e]) * nz[e];
      hx[e] = nhx[e];
      hy[e] = nhy[e];
    }
    if (i + 1 < x1) fetch(o + NYP);
    T y[NM];   // C_Y at columns j + m
#pragma unroll
    for (int m = MLO; m <= MHI; ++m) y[m - MLO] = ynb4<T, R>(cy, hcy, lane, m);
    T ox[4], oy[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      oy[e] = hy[e] + gather_back_full<T, R>([&](int d) { return qB[R - 1 + d][e]; });
      ox[e] = hx[e] + gather_back_full<T, R>([&](int d) { return y[e + d - MLO]; });
    }
    if (act) {
      st4(lHyj + o, oy);
      st4(lHxj + o, ox);
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 4; ++e) qB[m][e] = qB[m + 1][e];
  }
}

// Interior adjoint H step.  Rows holding receivers or sources are frame rows
// (the head of step it-1 has nothing else to do in the interior).
template <typename T, int R>
__device__ __forceinline__ void tmi_adj_h_run(const TiledAdj<T>& P, const TmBuf<T>& t, const TmGeom& tg, unsigned blk) {
  constexpr int MLO = -R, MHI = R + 2, NM = MHI - MLO + 1;
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NYP = tg.NYP;
  const WarpPos wp = warp_pos(tg, g.nshot, blk);
  if (!wp.live) return;
  const int lane = wp.lane, s = wp.s, x0 = wp.x0, x1 = wp.x1;
  const int j = wp.base + 4 * lane;
  const bool act = wp.base + TMW * (lane >> 3) < tg.col1;
  const int hj = halo_col4<R>(wp.base, lane);
  const bool hok = lane < 2 * R && hj >= 0 && hj < NY;
  const long long plane = (long long)NX * NYP;
  T* __restrict__ lEzj = t.Ez + s * plane + j;
  const T* __restrict__ lHxj = t.Hx + s * plane + j;
  const T* __restrict__ lHxh = t.Hx + s * plane + (hok ? hj : 0);
  const T* __restrict__ lHyj = t.Hy + s * plane + j;
  const T* __restrict__ hcj = t.ch_curl + j;
  const T* __restrict__ cyj = t.ch_curl_y + j;
  const T* __restrict__ cyh = t.ch_curl_y + (hok ? hj : 0);
  const T* __restrict__ c0j = t.ce_hist + j;
  const int RN = (R - 1) * NYP;
  T qA[2 * R][4];   // A_X = c lambda_Hy at rows i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int o = (x0 - R + m) * NYP;
    T y[4], c[4];
    ld4(lHyj + o, y);
    ld4(hcj + o, c);
#pragma unroll
    for (int e = 0; e < 4; ++e) qA[m][e] = c[e] * y[e];
  }
  T nay[4], nac[4], nx[4], ncy[4], nez[4], nc0[4], nhx = T(0), nhc = T(0);
  auto fetch = [&](int o) {
    ld4(lHyj + o + RN, nay);
    ld4(hcj + o + RN, nac);
    ld4(lHxj + o, nx);
    ld4(cyj + o, ncy);
    if (hok) {
      nhx = lHxh[o];
      nhc = cyh[o];
    }
    ld4(lEzj + o, nez);
    ld4(c0j + o, nc0);
  };
  fetch(x0 * NYP);
  for (int i = x0; i < x1; ++i) {
    const int o = i * NYP;
    T ay[4], ezv[4], c0[4];
    const T hay = hok ? (-nhc) * nhx : T(0);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      qA[2 * R - 1][e] = nac[e] * nay[e];
      ay[e] = (-ncy[e]) * nx[e];
      ezv[e] = nez[e];
      c0[e] = nc0[e];
    }
    if (i + 1 < x1) fetch(o + NYP);
    T y[NM];   // A_Y at columns j + m
#pragma unroll
    for (int m = MLO; m <= MHI; ++m) y[m - MLO] = ynb4<T, R>(ay, hay, lane, m);
    T ez[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      ez[e] = c0[e] * ezv[e];
      ez[e] += gather_fwd_full<T, R>([&](int d) { return qA[R + d][e]; });
      ez[e] += gather_fwd_full<T, R>([&](int d) { return y[e + d - MLO]; });
    }
    if (act) st4(lEzj + o, ez);
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 4; ++e) qA[m][e] = qA[m + 1][e];
  }
}

// Resident CTAs per SM of the interior kernels: 6 (80 registers a thread)
// measured 1 % faster per gradient of a 400 x 800 grid (32 shots, order 4)
// than the unconstrained build (93-126 registers); 8 (64 registers) spills
// and is 15 % slower.
constexpr int kTmiMinBlocks = 6;

#define DG_TMI_WRAPPER(NAME, ARGS, BUF)                                                               \
  template <typename T, int R>                                                                       \
  __global__ void __launch_bounds__(32 * TM_WARPS, kTmiMinBlocks) NAME(ARGS<T> P, TmBuf<T> t, TmGeom tg) { \
    NAME##_run<T, R>(P, t, tg, blockIdx.x);                                                          \
  }
DG_TMI_WRAPPER(tmi_fwd_h, TiledFwd, f)
DG_TMI_WRAPPER(tmi_fwd_e, TiledFwd, f)
DG_TMI_WRAPPER(tmi_adj_e, TiledAdj, t)
DG_TMI_WRAPPER(tmi_adj_h, TiledAdj, t)
#undef DG_TMI_WRAPPER

// ---------------------------------------------------------------------------
// Fused half steps: one launch of nfb frame CTAs (the general kernels on the
// frame geometry fg) and gridDim.x - nfb interior CTAs (the interior kernels
// on ig), dealt evenly through the launch: CTA b is a frame CTA when
// floor((b+1) nfb / n) > floor(b nfb / n), n = gridDim.x.  The CTAs of a launch
// start in index order, so every SM runs the frame's latency-bound warps
// beside the interior's bandwidth-bound ones, where two launches on two
// streams mostly ran one after the other.  The two parts touch disjoint
// cells and read only fields the half step does not write.
// ---------------------------------------------------------------------------
struct FusedBlock {
  bool frame;
  unsigned idx;   // CTA index within its part
};
__device__ __forceinline__ FusedBlock fused_block(unsigned nfb) {
  const unsigned long long b = blockIdx.x, n = gridDim.x;
  const unsigned f1 = (unsigned)((b + 1) * nfb / n), f0 = (unsigned)(b * nfb / n);
  FusedBlock r;
  r.frame = f1 > f0;
  r.idx = r.frame ? f0 : (unsigned)b - f1;
  return r;
}

template <typename T, int R>
__global__ void __launch_bounds__(32 * TM_WARPS) tmf_fwd_h(TiledFwd<T> P, TmBuf<T> f, TmGeom fg, TmGeom ig,
                                                           unsigned nfb) {
  const FusedBlock fb = fused_block(nfb);
  if (fb.frame) tm_fwd_h_run<T, R>(P, f, fg, fb.idx);
  else tmi_fwd_h_run<T, R>(P, f, ig, fb.idx);
}
template <typename T, int R>
__global__ void __launch_bounds__(32 * TM_WARPS) tmf_fwd_e(TiledFwd<T> P, TmBuf<T> f, TmGeom fg, TmGeom ig,
                                                           unsigned nfb) {
  const FusedBlock fb = fused_block(nfb);
  if (fb.frame) tm_fwd_e_run<T, R>(P, f, fg, fb.idx);
  else tmi_fwd_e_run<T, R>(P, f, ig, fb.idx);
}
template <typename T, int R>
__global__ void __launch_bounds__(32 * TM_WARPS) tmf_adj_e(TiledAdj<T> P, TmBuf<T> t, TmGeom fg, TmGeom ig,
                                                           unsigned nfb) {
  const FusedBlock fb = fused_block(nfb);
  if (fb.frame) tm_adj_e_run<T, R>(P, t, fg, fb.idx);
  else tmi_adj_e_run<T, R>(P, t, ig, fb.idx);
}
template <typename T, int R>
__global__ void __launch_bounds__(32 * TM_WARPS) tmf_adj_h(TiledAdj<T> P, TmBuf<T> t, TmGeom fg, TmGeom ig,
                                                           unsigned nfb) {
  const FusedBlock fb = fused_block(nfb);
  if (fb.frame) tm_adj_h_run<T, R, false>(P, t, fg, fb.idx);
  else tmi_adj_h_run<T, R>(P, t, ig, fb.idx);
}

// (nshot, NX, NY, 2) plane k = 0  <->  (nshot, NX, NYP) with zero padding.
template <typename T>
__global__ void k_pack2d_pitch(const T* __restrict__ src, T* __restrict__ dst, long long rows, int NY, int NYP) {
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += nw) {
    const T* __restrict__ s = src + 2 * (r * NY);
    T* __restrict__ d = dst + r * NYP;
    for (int j = lane; j < NYP; j += 32) d[j] = j < NY ? s[2 * j] : T(0);
  }
}
// As k_pack2d_pitch for a curl coefficient, scaled to the y difference:
// c * dx / dy, the reference's order of operations.
template <typename T>
__global__ void k_pack2d_pitch_ys(const T* __restrict__ src, T* __restrict__ dst, long long rows, int NY, int NYP,
                                  T dx, T dy) {
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += nw) {
    const T* __restrict__ s = src + 2 * (r * NY);
    T* __restrict__ d = dst + r * NYP;
    for (int j = lane; j < NYP; j += 32) d[j] = j < NY ? s[2 * j] * dx / dy : T(0);
  }
}
template <typename T>
__global__ void k_unpack2d_pitch(const T* __restrict__ src, T* __restrict__ dst, long long rows, int NY, int NYP) {
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += nw) {
    const T* __restrict__ s = src + r * NYP;
    T* __restrict__ d = dst + 2 * (r * NY);
    for (int j = lane; j < NY; j += 32) d[2 * j] = s[j];
  }
}

}  // namespace dg
