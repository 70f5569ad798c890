// fdtd_tiled.cuh -- bandwidth-oriented forward kernels.
//
// 3D: a CTA owns a TZ x TY = 32 x 8 column tile of the (y, z) plane and one
// shot, and streams along x over a chunk of planes.  x-derivatives read a
// per-thread register queue of the 2R planes around the current one (each
// plane value is loaded from HBM once); y/z-derivatives read the current
// plane from double-buffered shared memory with an R-cell halo (coalesced
// loads, the halo comes from L2).  One __syncthreads per plane.
//
// The 2D TM path (nz = 1, Ez/Hx/Hy only) has its own kernels in fdtd_tm2d.cuh.
//
// Per-cell arithmetic is identical to the reference order (see
// fdtd_forward.cuh for the line references); only where the operands come
// from differs.
#pragma once

#include "fdtd_forward.cuh"

namespace dg {

constexpr int TZ = 32, TY = 8;       // 3D tile (threads = 256)

// Stencils on an accessor f(d) = value at offset d along the axis.
// Full-radius forms (the stencil lies inside the grid).
template <typename T, int R, typename F>
__device__ __forceinline__ T dfwd_full(const F& f) {
  if (R == 1) return f(1) - f(0);
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) acc += tap<T>(R, r) * (f(r) - f(-(r - 1)));
  return acc;
}
template <typename T, int R, typename F>
__device__ __forceinline__ T dback_full(const F& f) {
  if (R == 1) return f(0) - f(-1);
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) acc += tap<T>(R, r) * (f(r - 1) - f(-r));
  return acc;
}

template <typename T, int R, typename F>
__device__ __forceinline__ T dfwd_f(const F& f, int c, int n) {
  if (R == 1) return f(1) - f(0);
  if (c - R + 1 >= 0 && c + R < n) return dfwd_full<T, R>(f);
  T acc = T(0);
  const int rr = rad_fwd(c, n, R);
#pragma unroll
  for (int r = 1; r <= R; ++r)
    if (r <= rr) acc += tap<T>(rr, r) * (f(r) - f(-(r - 1)));
  return acc;
}

template <typename T, int R, typename F>
__device__ __forceinline__ T dback_f(const F& f, int c, int n) {
  if (R == 1) return f(0) - f(-1);
  if (c >= R && c + R - 1 < n) return dback_full<T, R>(f);
  T acc = T(0);
  const int rr = rad_back(c, n, R);
#pragma unroll
  for (int r = 1; r <= R; ++r)
    if (r <= rr) acc += tap<T>(rr, r) * (f(r - 1) - f(-r));
  return acc;
}

// Per-shot membership bitmaps of the source / receiver cells, plus the
// sorted table for the (rare) lookups.
struct PointSet {
  PointTable tb;
  const unsigned* bits;   // nshot * ceil(cells / 32) words
  int words_per_shot;
};

__device__ __forceinline__ bool point_hit(const PointSet& ps, int s, int c) {
  if (ps.tb.n == 0) return false;
  const unsigned w = ps.bits[(long long)s * ps.words_per_shot + (c >> 5)];
  return (w >> (c & 31)) & 1u;
}

__device__ __forceinline__ int point_row(const PointSet& ps, int c) {
  int lo = 0, hi = ps.tb.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ps.tb.cells[mid] < c) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Halo slots of a 3D tile: y-halo rows (2R x TZ) and z-halo columns (2R x TY).
template <int R>
struct Halo3 {
  static constexpr int W = TZ + 2 * R;            // smem row pitch
  static constexpr int NY_SLOTS = 2 * R * TZ;
  static constexpr int TOTAL = NY_SLOTS + 2 * R * TY;
  static constexpr int PER_THREAD = (TOTAL + 255) / 256;
  int sidx[PER_THREAD];   // smem index, -1 unused
  int goff[PER_THREAD];   // offset within a plane (j * NZ + k), valid only if ok
  bool ok[PER_THREAD];
  bool yslot[PER_THREAD];

  __device__ __forceinline__ void init(const Grid& g, int j0, int k0) {
#pragma unroll
    for (int p = 0; p < PER_THREAD; ++p) {
      const int h = threadIdx.x + 256 * p;
      sidx[p] = -1;
      ok[p] = false;
      yslot[p] = false;
      goff[p] = 0;
      if (h >= TOTAL) continue;
      int yy, zz, sy, sz;
      if (h < NY_SLOTS) {
        const int r = h / TZ, z = h % TZ;
        const int yo = r < R ? r - R : TY + r - R;
        yy = j0 + yo; zz = k0 + z; sy = yo + R; sz = z + R;
        yslot[p] = true;
      } else {
        const int h2 = h - NY_SLOTS;
        const int r = h2 / TY, y = h2 % TY;
        const int zo = r < R ? r - R : TZ + r - R;
        yy = j0 + y; zz = k0 + zo; sy = y + R; sz = zo + R;
      }
      sidx[p] = sy * W + sz;
      ok[p] = yy >= 0 && yy < g.NY && zz >= 0 && zz < g.NZ;
      if (ok[p]) goff[p] = yy * g.NZ + zz;
    }
  }
};

// Fill one smem plane: own value plus the y and/or z halo of `plane`.
template <typename T, int R>
__device__ __forceinline__ void fill_plane(T* s, const T* plane, T own, int own_idx, const Halo3<R>& h, bool want_y,
                                           bool want_z) {
  s[own_idx] = own;
#pragma unroll
  for (int p = 0; p < Halo3<R>::PER_THREAD; ++p) {
    if (h.sidx[p] < 0) continue;
    if (h.yslot[p] ? !want_y : !want_z) continue;
    s[h.sidx[p]] = h.ok[p] ? plane[h.goff[p]] : T(0);
  }
}

// FP8 tile index of a 3D cell (the forward CTA plane tile that wrote it).
__device__ __forceinline__ long long fp8_tile3(const Grid& g, int i, int j, int k) {
  const int nzt = (g.NZ + TZ - 1) / TZ, nyt = (g.NY + TY - 1) / TY;
  return ((long long)i * nyt + j / TY) * nzt + k / TZ;
}

template <typename T>
struct TiledFwd {
  FwdArgs<T> a;
  PointSet src, rcv;
  int xchunk;
  int tm2d;
};

// ---------------------------------------------------------------------------
// 3D H half step.
// ---------------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(256) k3_fwd_h(TiledFwd<T> P) {
  using HL = Halo3<R>;
  constexpr int W = HL::W;
  constexpr int NS = (TY + 2 * R) * W;
  __shared__ T sEx[2][NS], sEy[2][NS], sEz[2][NS];
  __shared__ float red[33];
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
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
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save = a.save_e && (it % a.S == 0);
  const int slot = it / a.S;
  // y / z CPML faces depend on the column only
  int qy0 = -1, qy1 = -1, qz0 = -1, qz1 = -1;
  if (colv && a.has_cpml) {
    qy0 = q_low_h(a.hF[2].p, j);
    qy1 = q_high(a.hF[3].p, j, g.NY);
    qz0 = q_low_h(a.hF[4].p, k);
    qz1 = q_high(a.hF[5].p, k, g.NZ);
  }
  T qy[2 * R], qz[2 * R];   // Ey, Ez at planes i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = x0 - R + 1 + m;
    const bool v = colv && pl >= 0 && pl < g.NX;
    qy[m] = v ? a.Ey[sb + (long long)pl * g.sx + col] : T(0);
    qz[m] = v ? a.Ez[sb + (long long)pl * g.sx + col] : T(0);
  }
  for (int i = x0; i < x1; ++i) {
    const int b = (i - x0) & 1;
    {
      const int pl = i + R;
      const bool v = colv && pl < g.NX;
      qy[2 * R - 1] = v ? a.Ey[sb + (long long)pl * g.sx + col] : T(0);
      qz[2 * R - 1] = v ? a.Ez[sb + (long long)pl * g.sx + col] : T(0);
    }
    const long long pb = sb + (long long)i * g.sx;
    const T exo = colv ? a.Ex[pb + col] : T(0);
    fill_plane<T, R>(sEx[b], a.Ex + pb, exo, own, halo, true, true);
    fill_plane<T, R>(sEy[b], a.Ey + pb, qy[R - 1], own, halo, false, true);
    fill_plane<T, R>(sEz[b], a.Ez + pb, qz[R - 1], own, halo, true, false);
    __syncthreads();
    if (save) {
      long long h = 0;
      const bool inbox = colv && in_box(a.box, i, j, k, h);
      const int ncomp = a.mode == 3 ? 3 : 1;
      for (int q = 0; q < ncomp; ++q) {
        const int fc = a.mode == 3 ? q : 2;
        const T v = fc == 0 ? exo : (fc == 1 ? qy[R - 1] : qz[R - 1]);
        float inv = 1.0f;
        if (a.kind == kFP8) {
          const float am = block_absmax(inbox ? fabsf(float(v)) : 0.0f, red);
          const float sc = fp8_scale_of(am);
          inv = 1.0f / sc;
          if (threadIdx.x == 0)
            a.e_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j0, k0)] = sc;
        }
        if (inbox) hist_store<T>(a.E_saved, q * a.comp_stride + slot * a.frame + s * a.box.cells() + h, v, a.kind, inv);
      }
    }
    if (colv) {
      const T* ex_ = sEx[b];
      const T* ey_ = sEy[b];
      const T* ez_ = sEz[b];
      const bool dhx = upd_hx(g, i, j, k), dhy = upd_hy(g, i, j, k), dhz = upd_hz(g, i, j, k);
      const int qx0 = a.has_cpml ? q_low_h(a.hF[0].p, i) : -1;
      const int qx1 = a.has_cpml ? q_high(a.hF[1].p, i, g.NX) : -1;
      const bool in_x = qx0 >= 0 || qx1 >= 0, in_y = qy0 >= 0 || qy1 >= 0, in_z = qz0 >= 0 || qz1 >= 0;
      const int c = i * g.sx + col;
      const T c1 = a.ch_curl[c];
      const T cy = curl_scale(c1, a.dx, a.dy, a.dy_eq);
      const T cz = curl_scale(c1, a.dx, a.dz, a.dz_eq);
      auto fy = [&](const T* sp) { return [=](int d) { return sp[own + d * W]; }; };
      auto fz = [&](const T* sp) { return [=](int d) { return sp[own + d]; }; };
      T dEz_dy = T(0), dEy_dz = T(0), dEx_dz = T(0), dEz_dx = T(0), dEy_dx = T(0), dEx_dy = T(0);
      if (dhx || (in_y && k < g.NZ - 1)) dEz_dy = dfwd_f<T, R>(fy(ez_), j, g.NY);
      if (dhx || (in_z && j < g.NY - 1)) dEy_dz = dfwd_f<T, R>(fz(ey_), k, g.NZ);
      if (dhy || (in_z && i < g.NX - 1)) dEx_dz = dfwd_f<T, R>(fz(ex_), k, g.NZ);
      if (dhy || (in_x && k < g.NZ - 1)) dEz_dx = dfwd_f<T, R>([&](int d) { return qz[R - 1 + d]; }, i, g.NX);
      if (dhz || (in_x && j < g.NY - 1)) dEy_dx = dfwd_f<T, R>([&](int d) { return qy[R - 1 + d]; }, i, g.NX);
      if (dhz || (in_y && i < g.NX - 1)) dEx_dy = dfwd_f<T, R>(fy(ex_), j, g.NY);
      T hx = a.Hx[pb + col], hy = a.Hy[pb + col], hz = a.Hz[pb + col];
      if (dhx) hx = hx - cy * dEz_dy + cz * dEy_dz;
      if (dhy) hy = hy - cz * dEx_dz + c1 * dEz_dx;
      if (dhz) hz = hz - c1 * dEy_dx + cy * dEx_dy;
      if (in_x || in_y || in_z) {
        const T up = a.ch_rhs[c];
        const int qf[6] = {qx0, qx1, qy0, qy1, qz0, qz1};
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
              const T d = dEz_dx / a.dx, ph = F.psi1[pi];
              hy += up * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (j < g.NY - 1) {
              const long long pi = psi_index(psi_dims_h(g, 0, 2, F.p), 0, s, q, i, j, k);
              const T d = dEy_dx / a.dx, ph = F.psi2[pi];
              hz -= up * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          } else if (axis == 1) {
            if (k < g.NZ - 1) {
              const long long pi = psi_index(psi_dims_h(g, 1, 1, F.p), 1, s, q, i, j, k);
              const T d = dEz_dy / a.dy, ph = F.psi1[pi];
              hx -= up * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (i < g.NX - 1) {
              const long long pi = psi_index(psi_dims_h(g, 1, 2, F.p), 1, s, q, i, j, k);
              const T d = dEx_dy / a.dy, ph = F.psi2[pi];
              hz += up * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          } else {
            if (j < g.NY - 1) {
              const long long pi = psi_index(psi_dims_h(g, 2, 1, F.p), 2, s, q, i, j, k);
              const T d = dEy_dz / a.dz, ph = F.psi1[pi];
              hx += up * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (i < g.NX - 1) {
              const long long pi = psi_index(psi_dims_h(g, 2, 2, F.p), 2, s, q, i, j, k);
              const T d = dEx_dz / a.dz, ph = F.psi2[pi];
              hy -= up * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          }
        }
      }
      a.Hx[pb + col] = hx;
      a.Hy[pb + col] = hy;
      a.Hz[pb + col] = hz;
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) {
      qy[m] = qy[m + 1];
      qz[m] = qz[m + 1];
    }
  }
}

// Sources of shot s at cell c (sequential in source order), then the R^n
// history and receiver samples of that cell -- shared by the 3D and 2D E kernels.
template <typename T>
__device__ __forceinline__ void inject_at(const TiledFwd<T>& P, int s, int c, int it, T cb, T& ex, T& ey, T& ez) {
  const FwdArgs<T>& a = P.a;
  if (!point_hit(P.src, s, c)) return;
  const int row = point_row(P.src, c);
  for (int e = a.src.off[row]; e < a.src.off[row + 1]; ++e) {
    if (a.src.shot[e] != s) continue;
    const T scale = a.wave[(long long)a.src.idx[e] * a.nt + it] * a.src_dl / a.src_vol;
    if (a.src_comp == 0) ex -= cb * scale;
    else if (a.src_comp == 1) ey -= cb * scale;
    else ez -= cb * scale;
  }
}

template <typename T>
__device__ __forceinline__ void sample_at(const TiledFwd<T>& P, int s, int c, int it, T ex, T ey, T ez) {
  const FwdArgs<T>& a = P.a;
  if (!point_hit(P.rcv, s, c)) return;
  const int row = point_row(P.rcv, c);
  const T v = a.rx_comp == 0 ? ex : (a.rx_comp == 1 ? ey : ez);
  for (int e = a.rcv.off[row]; e < a.rcv.off[row + 1]; ++e)
    if (a.rcv.shot[e] == s) a.rx[((long long)s * a.nt + it) * a.nrx + a.rcv.idx[e]] = v;
}

// ---------------------------------------------------------------------------
// 3D E half step (+ sources, R^n history, receivers).
// ---------------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(256) k3_fwd_e(TiledFwd<T> P) {
  using HL = Halo3<R>;
  constexpr int W = HL::W;
  constexpr int NS = (TY + 2 * R) * W;
  __shared__ T sHx[2][NS], sHy[2][NS], sHz[2][NS];
  __shared__ float red[33];
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
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
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save_r = a.keep_r && (it % a.S == 0);
  const int slot = it / a.S;
  int qy0 = -1, qy1 = -1, qz0 = -1, qz1 = -1;
  if (colv && a.has_cpml) {
    qy0 = j > 0 ? q_low_e(a.eF[2].p, j) : -1;
    qy1 = j > 0 ? q_high(a.eF[3].p, j, g.NY) : -1;
    qz0 = k > 0 ? q_low_e(a.eF[4].p, k) : -1;
    qz1 = k > 0 ? q_high(a.eF[5].p, k, g.NZ) : -1;
  }
  T qy[2 * R], qz[2 * R];   // Hy, Hz at planes i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = x0 - R + m;
    const bool v = colv && pl >= 0 && pl < g.NX;
    qy[m] = v ? a.Hy[sb + (long long)pl * g.sx + col] : T(0);
    qz[m] = v ? a.Hz[sb + (long long)pl * g.sx + col] : T(0);
  }
  for (int i = x0; i < x1; ++i) {
    const int b = (i - x0) & 1;
    {
      const int pl = i + R - 1;
      const bool v = colv && pl < g.NX;
      qy[2 * R - 1] = v ? a.Hy[sb + (long long)pl * g.sx + col] : T(0);
      qz[2 * R - 1] = v ? a.Hz[sb + (long long)pl * g.sx + col] : T(0);
    }
    const long long pb = sb + (long long)i * g.sx;
    const T hxo = colv ? a.Hx[pb + col] : T(0);
    fill_plane<T, R>(sHx[b], a.Hx + pb, hxo, own, halo, true, true);
    fill_plane<T, R>(sHy[b], a.Hy + pb, qy[R], own, halo, false, true);
    fill_plane<T, R>(sHz[b], a.Hz + pb, qz[R], own, halo, true, false);
    __syncthreads();
    T ex = T(0), ey = T(0), ez = T(0), ox = T(0), oy = T(0), oz = T(0), c0e = T(0), cb = T(0);
    bool dex = false, dey = false, dez = false;
    const int c = i * g.sx + col;
    if (colv) {
      dex = upd_ex(g, i, j, k);
      dey = upd_ey(g, i, j, k);
      dez = upd_ez(g, i, j, k);
      const int qx0 = (a.has_cpml && i > 0) ? q_low_e(a.eF[0].p, i) : -1;
      const int qx1 = (a.has_cpml && i > 0) ? q_high(a.eF[1].p, i, g.NX) : -1;
      const bool in_x = qx0 >= 0 || qx1 >= 0, in_y = qy0 >= 0 || qy1 >= 0, in_z = qz0 >= 0 || qz1 >= 0;
      const bool any_pml = in_x || in_y || in_z;
      const T* hx_ = sHx[b];
      const T* hy_ = sHy[b];
      const T* hz_ = sHz[b];
      auto fy = [&](const T* sp) { return [=](int d) { return sp[own + d * W]; }; };
      auto fz = [&](const T* sp) { return [=](int d) { return sp[own + d]; }; };
      c0e = a.ce_hist[c];
      const T c1 = a.ce_curl[c];
      const T cy = curl_scale(c1, a.dx, a.dy, a.dy_eq);
      const T cz = curl_scale(c1, a.dx, a.dz, a.dz_eq);
      ox = ex = a.Ex[pb + col];
      oy = ey = a.Ey[pb + col];
      oz = ez = a.Ez[pb + col];
      T dHz_dy = T(0), dHy_dz = T(0), dHx_dz = T(0), dHz_dx = T(0), dHy_dx = T(0), dHx_dy = T(0);
      if (dex || (in_y && i < g.NX - 1)) dHz_dy = dback_f<T, R>(fy(hz_), j, g.NY);
      if (dex || (in_z && i < g.NX - 1)) dHy_dz = dback_f<T, R>(fz(hy_), k, g.NZ);
      if (dey || (in_z && j < g.NY - 1)) dHx_dz = dback_f<T, R>(fz(hx_), k, g.NZ);
      if (dey || (in_x && j < g.NY - 1)) dHz_dx = dback_f<T, R>([&](int d) { return qz[R + d]; }, i, g.NX);
      if (dez || (in_x && k < g.NZ - 1)) dHy_dx = dback_f<T, R>([&](int d) { return qy[R + d]; }, i, g.NX);
      if (dez || (in_y && k < g.NZ - 1)) dHx_dy = dback_f<T, R>(fy(hx_), j, g.NY);
      if (dex) ex = c0e * ex + cy * dHz_dy - cz * dHy_dz;
      if (dey) ey = c0e * ey + cz * dHx_dz - c1 * dHz_dx;
      if (dez) ez = c0e * ez + c1 * dHy_dx - cy * dHx_dy;
      const bool src_hit = point_hit(P.src, s, c);
      if (any_pml || src_hit || save_r) cb = a.ce_rhs[c];
      if (any_pml) {
        const int qf[6] = {qx0, qx1, qy0, qy1, qz0, qz1};
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
              const T d = dHz_dx / a.dx, ph = F.psi1[pi];
              ey -= cb * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (k < g.NZ - 1) {
              const long long pi = psi_index(psi_dims_e(g, 0, 2, F.p), 0, s, q, i, j, k);
              const T d = dHy_dx / a.dx, ph = F.psi2[pi];
              ez += cb * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          } else if (axis == 1) {
            if (i < g.NX - 1) {
              const long long pi = psi_index(psi_dims_e(g, 1, 1, F.p), 1, s, q, i, j, k);
              const T d = dHz_dy / a.dy, ph = F.psi1[pi];
              ex += cb * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (k < g.NZ - 1) {
              const long long pi = psi_index(psi_dims_e(g, 1, 2, F.p), 1, s, q, i, j, k);
              const T d = dHx_dy / a.dy, ph = F.psi2[pi];
              ez -= cb * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          } else {
            if (i < g.NX - 1) {
              const long long pi = psi_index(psi_dims_e(g, 2, 1, F.p), 2, s, q, i, j, k);
              const T d = dHy_dz / a.dz, ph = F.psi1[pi];
              ex -= cb * (pr.ra1 * d + pr.rb * ph);
              F.psi1[pi] = pr.re * ph - pr.rf * d;
            }
            if (j < g.NY - 1) {
              const long long pi = psi_index(psi_dims_e(g, 2, 2, F.p), 2, s, q, i, j, k);
              const T d = dHx_dz / a.dz, ph = F.psi2[pi];
              ey += cb * (pr.ra1 * d + pr.rb * ph);
              F.psi2[pi] = pr.re * ph - pr.rf * d;
            }
          }
        }
      }
      if (src_hit) inject_at(P, s, c, it, cb, ex, ey, ez);
    }
    if (save_r) {
      long long h = 0;
      const bool inbox = colv && in_box(a.box, i, j, k, h);
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
          const float am = block_absmax(inbox ? fabsf(float(rv)) : 0.0f, red);
          const float sc = fp8_scale_of(am);
          inv = 1.0f / sc;
          if (threadIdx.x == 0)
            a.r_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j0, k0)] = sc;
        }
        if (inbox) hist_store<T>(a.R_saved, q * a.comp_stride + slot * a.frame + s * a.box.cells() + h, rv, a.kind, inv);
      }
    }
    if (colv) {
      sample_at(P, s, c, it, ex, ey, ez);
      a.Ex[pb + col] = ex;
      a.Ey[pb + col] = ey;
      a.Ez[pb + col] = ez;
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m) {
      qy[m] = qy[m + 1];
      qz[m] = qz[m + 1];
    }
  }
}

// 2D Yee predicates (NZ = 2, k = 0): Ez, Hx, Hy of the general rules.
__device__ __forceinline__ bool tm_upd_ez(const Grid& g, int i, int j) {
  return (g.NX - 1 != 1 || g.NY - 1 != 1) && i > 0 && i < g.NX - 1 && j > 0 && j < g.NY - 1;
}
__device__ __forceinline__ bool tm_upd_hx(const Grid& g, int i, int j) {
  return g.NX - 1 != 1 && i > 0 && i < g.NX - 1 && j < g.NY - 1;
}
__device__ __forceinline__ bool tm_upd_hy(const Grid& g, int i, int j) {
  return g.NY - 1 != 1 && i < g.NX - 1 && j > 0 && j < g.NY - 1;
}

}  // namespace dg
