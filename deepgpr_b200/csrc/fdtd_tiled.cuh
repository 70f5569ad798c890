// fdtd_tiled.cuh -- stencil helpers shared by the streaming kernels: full and
// radius-clamped staggered differences on accessors, point tables, the
// shared-memory halo slots of the 3D adjoint kernels, source injection and
// receiver sampling.  The 3D forward kernels are in fdtd_3d.cuh, the 2D TM
// kernels in fdtd_tm2d.cuh.
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

// FP8 scale tile of a 3D cell: one per (x plane, y row, 32 z columns).
__device__ __forceinline__ long long fp8_tile3(const Grid& g, int i, int j, int k) {
  const int nzt = (g.NZ + 31) / 32;
  return ((long long)i * g.NY + j) * nzt + k / 32;
}

template <typename T>
struct TiledFwd {
  FwdArgs<T> a;
  PointSet src, rcv;
  int xchunk;
  int tm2d;
};

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
