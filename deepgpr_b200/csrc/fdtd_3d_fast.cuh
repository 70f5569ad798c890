// fdtd_3d_fast.cuh -- 3D forward half steps on bulk-tensor (TMA) staged tiles.
//
// A CTA of 128 threads owns an (8 row x 64 column) tile of the (y, z) plane
// of one shot and streams it along x over a chunk of planes.  Per plane:
//   * the stencil operands (the other field's three components) arrive in a
//     shared-memory ring by TMA as a box of rows j0-R .. j0+7+R and columns
//     k0-4 .. k0+67 (zero outside the grid), a window of 2R planes plus
//     three planes in flight;
//   * the updated field's three components and its coefficients arrive by
//     TMA as the bare 8 x 64 tile, three planes ahead;
//   * warp w updates rows 2w, 2w+1; lane l columns 2l, 2l+1: x-, y- and
//     z-taps are shared-memory reads at fixed offsets, so a cell costs no
//     address arithmetic beyond its slot base;
//   * results go straight to global memory (the updated field, psi, history).
// Every cell evaluates the reference's expressions in the reference's order
// (src/DeepGPR/lib/deepgpr_cpu.c:670-1100: base update, CPML faces x, y, z,
// sources, R^n, receivers): difference taps of the clamped radius near the
// grid ends (zero beyond it), the Yee update predicates, and the single-face
// CPML form (faces of an axis at least 4 cells apart).  Sources, receivers
// and R^n run only on planes that hold them.  FP32 only; the FP64 runs and
// the general CPML form use the z-streamed kernels of fdtd_3d.cuh.
#pragma once

#include "fdtd_3d.cuh"
#include "fdtd_tma.cuh"

namespace dg {

constexpr int KT_TY = 8;          // rows of a tile
constexpr int KT_TZ = 64;         // columns of a tile (two per lane)
constexpr int KT_BZ = 72;         // columns of a staged box: k0 - 4 .. k0 + 67
constexpr int KT_THREADS = 128;   // four warps, two rows each
constexpr int KT_D = 3;           // planes in flight beyond the stencil window
constexpr int KT_NO = 3;          // slots of the own-tile ring

// NOWN: arrays staged per own-tile slot (the updated field's three
// components and its coefficients: 4 for H, 5 for E).
template <int R, int NOWN>
struct KtShape {
  static constexpr int BY = KT_TY + 2 * R;                        // rows of a staged box
  static constexpr int HALO = (BY * KT_BZ + 31) / 32 * 32;        // floats per staged component (128-byte slots)
  static constexpr int NS = 2 * R - 1 + KT_D;                     // stencil ring slots
  static constexpr int OWN = KT_TY * KT_TZ;                       // floats per own-tile array
  static constexpr size_t BYTES =
      (size_t)(NS * 3 * HALO + KT_NO * NOWN * OWN) * 4 + (NS + KT_NO) * sizeof(uint64_t);
};
template <int R>
__host__ __device__ constexpr int kt_min_blocks() {
  return R >= 4 ? 1 : (R >= 2 ? 2 : 3);
}

struct K3TGeom {
  int zp;                          // z pitch of the working copy
  int nyt, nzs;                    // tiles along y, strips along z
  int xc, nchunk;                  // x chunk length, chunks
  long long nblocks;
  const unsigned char* src_rows;   // (nshot, NX): the plane holds a source of the shot
  const unsigned char* rcv_rows;
  Control* ctrl;                   // error bits of a wait that ran out
};

// Tensor maps of one half step: the stencil operands with halo, the updated
// field's tile and up to two coefficient tiles.
struct K3TMaps {
  CUtensorMap halo[3];
  CUtensorMap own[3];
  CUtensorMap coef[2];
};

constexpr int kErrWaitTimeout = 4;

// ---------------------------------------------------------------------------
// Ring bookkeeping shared by both half steps.  Stencil window of plane i:
// planes i + LO .. i + HI; plane p lives in slot (p - x0 - LO) % NS.
// ---------------------------------------------------------------------------
template <int R, int LO, int HI, int NOWN>
struct KtRing {
  using Sh = KtShape<R, NOWN>;
  static constexpr int NS = HI - LO + KT_D;
  static_assert(NS == Sh::NS, "stencil window of 2R planes");
  float* ring;        // NS x 3 x HALO
  float* own;         // KT_NO x NOWN x OWN
  uint64_t* bar;      // NS stencil barriers, then KT_NO own barriers
  int x0, x1, NX, plane0, j0, k0;
  bool bad = false;

  __device__ float* slot(int p) const { return ring + ((p - x0 - LO) % NS) * 3 * Sh::HALO; }
  __device__ float* own_slot(int p) const { return own + ((p - x0) % KT_NO) * NOWN * Sh::OWN; }

  // thread 0: stencil plane p (zero-filled by all threads beforehand when outside the grid)
  __device__ void issue(const K3TMaps& m, int p) {
    const int sl = (p - x0 - LO) % NS;
    uint64_t* b = &bar[sl];
    if (p < 0 || p >= NX) {
      mbar_arrive(b);
      return;
    }
    float* dst = ring + sl * 3 * Sh::HALO;
    mbar_expect_tx(b, 3u * Sh::BY * KT_BZ * 4u);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma_load_3d(dst + c * Sh::HALO, &m.halo[c], k0 - 4, j0 - R, plane0 + p, b);
  }
  __device__ void issue_own(const K3TMaps& m, int p) {
    const int sl = (p - x0) % KT_NO;
    uint64_t* b = &bar[NS + sl];
    float* dst = own + sl * NOWN * Sh::OWN;
    mbar_expect_tx(b, (unsigned)NOWN * Sh::OWN * 4u);
#pragma unroll
    for (int c = 0; c < 3; ++c) tma_load_3d(dst + c * Sh::OWN, &m.own[c], k0, j0, plane0 + p, b);
#pragma unroll
    for (int c = 0; c < NOWN - 3; ++c) tma_load_3d(dst + (3 + c) * Sh::OWN, &m.coef[c], k0, j0, p, b);
  }
  // all threads: zero the slot of an out-of-grid plane
  __device__ void zero(int p) {
    float* dst = slot(p);
    for (int t = threadIdx.x; t < 3 * Sh::HALO; t += KT_THREADS) dst[t] = 0.0f;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __device__ void wait(int p) {
    const unsigned par = (unsigned)((p - x0 - LO) / NS) & 1u;
    if (!mbar_wait(&bar[(p - x0 - LO) % NS], par)) bad = true;
  }
  __device__ void wait_own(int p) {
    const unsigned par = (unsigned)((p - x0) / KT_NO) & 1u;
    if (!mbar_wait(&bar[NS + (p - x0) % KT_NO], par)) bad = true;
  }
  // planes issued so far (the same on every thread)
  int s_issued = 0, o_issued = 0;

  // prologue: barriers, first window and own planes
  __device__ void start(const K3TMaps& m) {
    const int last = x1 - 1 + HI;   // last stencil plane the chunk reads
    if (threadIdx.x == 0) {
      for (int q = 0; q < NS + KT_NO; ++q) mbar_init(&bar[q], 1);
      fence_barrier_init();
    }
    for (int p = x0 + LO; p < x0 + LO + NS && p <= last; ++p)
      if (p < 0 || p >= NX) zero(p);
    __syncthreads();
    s_issued = min(x0 + LO + NS, last + 1);
    o_issued = min(x0 + KT_NO, x1);
    if (threadIdx.x == 0) {
      for (int p = x0 + LO; p < s_issued; ++p) issue(m, p);
      for (int p = x0; p < o_issued; ++p) issue_own(m, p);
    }
    for (int p = x0 + LO; p < x0 + HI; ++p) wait(p);
  }
  __device__ void wait_plane(int i) {
    wait(i + HI);
    wait_own(i);
  }
  // end of plane i: frees the slot of plane i + LO and the own slot of plane i
  __device__ bool advance(const K3TMaps& m, int i) {
    if (__syncthreads_or(bad)) return false;
    const int p = i + HI + KT_D, last = x1 - 1 + HI;
    if (p <= last && (p < 0 || p >= NX)) zero(p);
    if (threadIdx.x == 0) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      if (p <= last) issue(m, p);
      if (i + KT_NO < x1) issue_own(m, i + KT_NO);
    }
    if (p <= last) s_issued = p + 1;
    if (i + KT_NO < x1) o_issued = i + KT_NO + 1;
    return true;
  }
  // after a wait ran out: bounded waits for the copies still in flight, then report
  __device__ void fail(Control* ctrl) {
    if (threadIdx.x == 0) {
      // the last NS stencil and KT_NO own planes issued (older slots were reused, so waited)
      for (int p = max(x0 + LO, s_issued - NS); p < s_issued; ++p) {
        const unsigned par = (unsigned)((p - x0 - LO) / NS) & 1u;
        for (unsigned n = 0; n < (1u << 20) && !mbar_try_wait(&bar[(p - x0 - LO) % NS], par); ++n) {
        }
      }
      for (int p = max(x0, o_issued - KT_NO); p < o_issued; ++p) {
        const unsigned par = (unsigned)((p - x0) / KT_NO) & 1u;
        for (unsigned n = 0; n < (1u << 20) && !mbar_try_wait(&bar[NS + (p - x0) % KT_NO], par); ++n) {
        }
      }
      atomicOr(&ctrl->error, kErrWaitTimeout);
    }
  }
};

// z window of a lane's column pair: v[m - MLO] = value at column k + m
// (k = k0 + 2 lane) for MLO <= m <= MHI + 1, from even-aligned pairs of one
// staged row (row pointer at column k0 - 4).
template <int MLO, int MHI>
struct ZWin {
  static constexpr int PLO = (MLO >= 0 ? MLO : MLO - 1) / 2;   // floor(MLO / 2)
  static constexpr int PHI = (MHI + 1 >= 0 ? MHI + 1 : MHI) / 2;
  static constexpr int N = 2 * (PHI - PLO + 1);
  float v[N];
  __device__ __forceinline__ void load(const float* row, int lane) {
    const float2* p = reinterpret_cast<const float2*>(row + 4 + 2 * lane);
#pragma unroll
    for (int q = PLO; q <= PHI; ++q) {
      const float2 t = p[q];
      v[2 * (q - PLO)] = t.x;
      v[2 * (q - PLO) + 1] = t.y;
    }
  }
  // value at column k + e + m
  __device__ __forceinline__ float at(int e, int m) const { return v[e + m - 2 * PLO]; }
};

// Forward / backward staggered difference with per-target taps (zero beyond
// the clamped radius); radius 1 is the plain difference.
template <int R, typename F>
__device__ __forceinline__ float kt_dfwd(const F& f, const float (&t)[R]) {
  if (R == 1) return f(1) - f(0);
  float acc = 0.0f;
#pragma unroll
  for (int r = 1; r <= R; ++r) acc += t[r - 1] * (f(r) - f(-(r - 1)));
  return acc;
}
template <int R, typename F>
__device__ __forceinline__ float kt_dback(const F& f, const float (&t)[R]) {
  if (R == 1) return f(0) - f(-1);
  float acc = 0.0f;
#pragma unroll
  for (int r = 1; r <= R; ++r) acc += t[r - 1] * (f(r - 1) - f(-r));
  return acc;
}

__device__ __forceinline__ void kt_cpml(float* psi, long long pi, const Prof<float>& pr, float dv,
                                        const FixedDiv<float>& h, float c, bool plus, float& u) {
  const float ph = psi[pi];
  const float d = div_fixed(dv, h);
  if (plus) u += c * (pr.ra1 * d + pr.rb * ph);
  else u -= c * (pr.ra1 * d + pr.rb * ph);
  psi[pi] = pr.re * ph - pr.rf * d;
}

// Tile position of the CTA: block -> (y tile fastest, z strip, shot, x chunk).
struct KtPos {
  int j0, k0, s, x0, x1;
  bool live;
};
__device__ __forceinline__ KtPos kt_pos(const K3TGeom& tg, const Grid& g) {
  KtPos p;
  unsigned b = blockIdx.x;
  const unsigned ny = (unsigned)tg.nyt, nz = (unsigned)tg.nzs, ns = (unsigned)g.nshot;
  unsigned q = b / ny;
  p.j0 = int(b - q * ny) * KT_TY;
  b = q;
  q = b / nz;
  p.k0 = int(b - q * nz) * KT_TZ;
  b = q;
  q = b / ns;
  p.s = int(b - q * ns);
  p.x0 = int(q) * tg.xc;
  p.x1 = min(p.x0 + tg.xc, g.NX);
  p.live = int(q) < tg.nchunk;
  return p;
}

// ---------------------------------------------------------------------------
// H half step (+ E^n history).  Stencil operands Ex, Ey, Ez at offsets
// -(R-1) .. R; own tiles Hx, Hy, Hz and ch_curl.
// ---------------------------------------------------------------------------
template <int R, bool EQ>
__global__ void __launch_bounds__(KT_THREADS, kt_min_blocks<R>())
    k3t_fwd_h(const __grid_constant__ K3TMaps maps, const __grid_constant__ TiledFwd<float> P, K3Buf<float> f,
              K3TGeom tg) {
  using T = float;
  constexpr int LO = -(R - 1), HI = R, BZ = KT_BZ, NOWN = 4;
  using Sh = KtShape<R, NOWN>;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const KtPos pos = kt_pos(tg, g);
  if (!pos.live) return;
  extern __shared__ __align__(128) float smem[];
  KtRing<R, LO, HI, NOWN> rg;
  rg.ring = smem;
  rg.own = smem + Sh::NS * 3 * Sh::HALO;
  rg.bar = reinterpret_cast<uint64_t*>(rg.own + KT_NO * NOWN * Sh::OWN);
  rg.x0 = pos.x0;
  rg.x1 = pos.x1;
  rg.NX = g.NX;
  rg.plane0 = pos.s * g.NX;
  rg.j0 = pos.j0;
  rg.k0 = pos.k0;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = tg.zp, s = pos.s;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int PS = NY * zp;
  T* __restrict__ Hx = f.Hx + (long long)s * NX * PS;
  T* __restrict__ Hy = f.Hy + (long long)s * NX * PS;
  T* __restrict__ Hz = f.Hz + (long long)s * NX * PS;
  const bool pml = a.has_cpml != 0;
  // per-column state (fixed along x)
  int kc[2];
  bool kv[2], hxz[2], hzz[2], onk[2];
  int zq[2];
  int fz = 5;
  T tz[2][R];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = pos.k0 + 2 * lane + e;
    kc[e] = k;
    kv[e] = k < NZ;
    hxz[e] = k < NZ - 1;
    hzz[e] = NZ - 1 != 1 && k > 0 && k < NZ - 1;
    onk[e] = kv[e] && k < NZ - 1;
    const int q0 = (kv[e] && pml) ? q_low_h(a.hF[4].p, k) : -1;
    const int q1 = (kv[e] && pml) ? q_high(a.hF[5].p, k, NZ) : -1;
    if (q0 >= 0) fz = 4;
    zq[e] = q0 >= 0 ? q0 : q1;
    taps_fwd<T, R>(k, NZ, tz[e]);
  }
  Prof<T> pz[2];
  const Face<T>& FZ = fz == 4 ? a.hF[4] : a.hF[5];
#pragma unroll
  for (int e = 0; e < 2; ++e) pz[e] = zq[e] >= 0 ? prof(FZ, zq[e]) : Prof<T>{0.0f, 0.0f, 0.0f, 0.0f};
  // per-row state (rows 2w, 2w + 1 of the tile)
  int jrow[2], qy[2];
  bool jv[2], hxy[2], hyy[2], jl[2];
  T ty[2][R];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int j = pos.j0 + 2 * w + r;
    jrow[r] = j;
    jv[r] = j < NY;
    hxy[r] = j < NY - 1;
    hyy[r] = NY - 1 != 1 && j > 0 && j < NY - 1;
    jl[r] = j < NY - 1;
    const int q0 = (jv[r] && pml) ? q_low_h(a.hF[2].p, j) : -1;
    const int q1 = (jv[r] && pml) ? q_high(a.hF[3].p, j, NY) : -1;
    qy[r] = q0 >= 0 ? q0 : (q1 >= 0 ? q1 + 1024 : -1);   // +1024: high face
    taps_fwd<T, R>(j, NY, ty[r]);
  }
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save = a.save_e && (it % a.S == 0);
  const int hslot = it / a.S;
  const int ncomp = a.mode == 3 ? 3 : 1;

  rg.start(maps);
  for (int i = pos.x0; i < pos.x1; ++i) {
    rg.wait_plane(i);
    const float* own = rg.own_slot(i);
    T tx[R];
    taps_fwd<T, R>(i, NX, tx);
    const bool hxx = NX - 1 != 1 && i > 0 && i < NX - 1, hyx = i < NX - 1, il = i < NX - 1;
    int qx = -1, fx = 0;
    if (pml) {
      const int q0 = q_low_h(a.hF[0].p, i), q1 = q_high(a.hF[1].p, i, NX);
      qx = q0 >= 0 ? q0 : q1;
      fx = q0 >= 0 ? 0 : 1;
    }
    const int bi = i - a.box.x0;
    const bool xin_box = save && bi >= 0 && bi < a.box.nx;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int jr = 2 * w + r, j = jrow[r];
      if (!jv[r]) continue;
      const int srow = (R + jr) * BZ;   // own row in a staged box
      // z windows of Ex, Ey (offsets -(R-1) .. R of each column)
      ZWin<LO, HI> zx, zy;
      const float* p0 = rg.slot(i);
      zx.load(p0 + srow, lane);
      zy.load(p0 + Sh::HALO + srow, lane);
      // y windows of Ex, Ez; x windows of Ey, Ez (column pairs)
      float2 yx[HI - LO + 1], yz[HI - LO + 1], xy[HI - LO + 1], xz[HI - LO + 1];
#pragma unroll
      for (int d = LO; d <= HI; ++d) {
        yx[d - LO] = *reinterpret_cast<const float2*>(p0 + (R + jr + d) * BZ + 4 + 2 * lane);
        yz[d - LO] = *reinterpret_cast<const float2*>(p0 + 2 * Sh::HALO + (R + jr + d) * BZ + 4 + 2 * lane);
        const float* pd = rg.slot(i + d);
        xy[d - LO] = *reinterpret_cast<const float2*>(pd + Sh::HALO + srow + 4 + 2 * lane);
        xz[d - LO] = *reinterpret_cast<const float2*>(pd + 2 * Sh::HALO + srow + 4 + 2 * lane);
      }
      const int oo = jr * KT_TZ + 2 * lane;
      const float2 h0 = *reinterpret_cast<const float2*>(own + oo);
      const float2 h1 = *reinterpret_cast<const float2*>(own + Sh::OWN + oo);
      const float2 h2 = *reinterpret_cast<const float2*>(own + 2 * Sh::OWN + oo);
      const float2 c2 = *reinterpret_cast<const float2*>(own + 3 * Sh::OWN + oo);
      T hx[2] = {h0.x, h0.y}, hy[2] = {h1.x, h1.y}, hz[2] = {h2.x, h2.y}, cc[2] = {c2.x, c2.y};
      T dEz_dy[2], dEx_dy[2], dEz_dx[2], dEy_dx[2], dEy_dz[2], dEx_dz[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const auto sel = [e](const float2& v) { return e == 0 ? v.x : v.y; };
        dEz_dy[e] = kt_dfwd<R>([&](int d) { return sel(yz[d - LO]); }, ty[r]);
        dEx_dy[e] = kt_dfwd<R>([&](int d) { return sel(yx[d - LO]); }, ty[r]);
        dEz_dx[e] = kt_dfwd<R>([&](int d) { return sel(xz[d - LO]); }, tx);
        dEy_dx[e] = kt_dfwd<R>([&](int d) { return sel(xy[d - LO]); }, tx);
        dEy_dz[e] = kt_dfwd<R>([&](int d) { return zy.at(e, d); }, tz[e]);
        dEx_dz[e] = kt_dfwd<R>([&](int d) { return zx.at(e, d); }, tz[e]);
        const T cx = cc[e];
        const T cy = (EQ || a.dy_eq) ? cx : div_fixed(cx * a.dx, a.ddy);
        const T cz = (EQ || a.dz_eq) ? cx : div_fixed(cx * a.dx, a.ddz);
        if (hxx && hxy[r] && hxz[e]) hx[e] = hx[e] - cy * dEz_dy[e] + cz * dEy_dz[e];
        if (hyx && hyy[r] && hxz[e]) hy[e] = hy[e] - cz * dEx_dz[e] + cx * dEz_dx[e];
        if (hyx && hxy[r] && hzz[e]) hz[e] = hz[e] - cx * dEy_dx[e] + cy * dEx_dy[e];
      }
      const long long go = (long long)i * PS + (long long)j * zp + kc[0];
      if (pml && (qx >= 0 || qy[r] >= 0 || zq[0] >= 0 || zq[1] >= 0)) {
        // CPML corrections in the reference order: x, y, z faces
        T up[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) up[e] = kv[e] ? f.ch_rhs[(long long)i * PS + (long long)j * zp + kc[e]] : 0.0f;
        if (qx >= 0) {
          const Face<T>& F = a.hF[fx];
          const Prof<T> pr = prof(F, qx);
          const long long b1 = ((long long)(s * F.p + qx) * NY + j) * (NZ - 1);
          const long long b2 = ((long long)(s * F.p + qx) * (NY - 1) + j) * NZ;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (onk[e]) kt_cpml(F.psi1, b1 + kc[e], pr, dEz_dx[e], a.ddx, up[e], true, hy[e]);
            if (kv[e] && jl[r]) kt_cpml(F.psi2, b2 + kc[e], pr, dEy_dx[e], a.ddx, up[e], false, hz[e]);
          }
        }
        if (qy[r] >= 0) {
          const int q = qy[r] & 1023;
          const Face<T>& F = qy[r] >= 1024 ? a.hF[3] : a.hF[2];
          const Prof<T> pr = prof(F, q);
          const long long b1 = (((long long)s * NX + i) * F.p + q) * (NZ - 1);
          const long long b2 = (((long long)s * (NX - 1) + i) * F.p + q) * NZ;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (onk[e]) kt_cpml(F.psi1, b1 + kc[e], pr, dEz_dy[e], a.ddy, up[e], false, hx[e]);
            if (kv[e] && il) kt_cpml(F.psi2, b2 + kc[e], pr, dEx_dy[e], a.ddy, up[e], true, hz[e]);
          }
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (zq[e] < 0) continue;
          if (jl[r]) kt_cpml(FZ.psi1, (((long long)s * NX + i) * (NY - 1) + j) * FZ.p + zq[e], pz[e], dEy_dz[e],
                             a.ddz, up[e], true, hx[e]);
          if (il) kt_cpml(FZ.psi2, (((long long)s * (NX - 1) + i) * NY + j) * FZ.p + zq[e], pz[e], dEx_dz[e],
                          a.ddz, up[e], false, hy[e]);
        }
      }
      if (kv[1]) {
        *reinterpret_cast<float2*>(Hx + go) = make_float2(hx[0], hx[1]);
        *reinterpret_cast<float2*>(Hy + go) = make_float2(hy[0], hy[1]);
        *reinterpret_cast<float2*>(Hz + go) = make_float2(hz[0], hz[1]);
      } else if (kv[0]) {
        Hx[go] = hx[0];
        Hy[go] = hy[0];
        Hz[go] = hz[0];
      }
      if (save) {
        // E^n history (before this step's update of E), deepgpr_cpu.c:1559-1590
        const bool rin = xin_box && j - a.box.y0 >= 0 && j - a.box.y0 < a.box.ny;
        bool ib[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) ib[e] = rin && kv[e] && kc[e] - a.box.z0 >= 0 && kc[e] - a.box.z0 < a.box.nz;
        const long long hoff = hslot * a.frame + s * a.box.cells() +
                               ((long long)bi * a.box.ny + (j - a.box.y0)) * a.box.nz + (kc[0] - a.box.z0);
        with_hist_kind(a.kind, [&](auto K) {
          constexpr int KIND = decltype(K)::value;
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            if (q >= ncomp) break;
            const int fc = a.mode == 3 ? q : 2;
            T v[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) v[e] = fc == 0 ? zx.at(e, 0) : (fc == 1 ? zy.at(e, 0) : (e == 0 ? yz[-LO].x : yz[-LO].y));
            float inv = 1.0f;
            if (is_tiled(KIND)) {
              float am = 0.0f;
#pragma unroll
              for (int e = 0; e < 2; ++e)
                if (ib[e]) am = fmaxf(am, fabsf(v[e]));
              const float sc = tile_scale_of(KIND, half_absmax(am));
              inv = 1.0f / sc;
              if ((lane & 15) == 0 && kc[0] < NZ)
                a.e_scales[(((long long)q * a.nt_saved + hslot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j, kc[0])] =
                    sc;
            }
            const long long hq = q * a.comp_stride + hoff;
            if (ib[0]) hist_store<T>(a.E_saved, hq, v[0], KIND, inv);
            if (ib[1]) hist_store<T>(a.E_saved, hq + 1, v[1], KIND, inv);
          }
        });
      }
    }
    if (!rg.advance(maps, i)) {
      rg.fail(tg.ctrl);
      return;
    }
  }
}

// ---------------------------------------------------------------------------
// E half step (+ sources, R^n history, receivers).  Stencil operands Hx, Hy,
// Hz at offsets -R .. R-1; own tiles Ex, Ey, Ez with ce_hist and ce_curl.
// ---------------------------------------------------------------------------
template <int R, bool EQ>
__global__ void __launch_bounds__(KT_THREADS, kt_min_blocks<R>())
    k3t_fwd_e(const __grid_constant__ K3TMaps maps, const __grid_constant__ TiledFwd<float> P, K3Buf<float> f,
              K3TGeom tg) {
  using T = float;
  constexpr int LO = -R, HI = R - 1, BZ = KT_BZ, NOWN = 5;
  using Sh = KtShape<R, NOWN>;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const KtPos pos = kt_pos(tg, g);
  if (!pos.live) return;
  extern __shared__ __align__(128) float smem[];
  KtRing<R, LO, HI, NOWN> rg;
  rg.ring = smem;
  rg.own = smem + Sh::NS * 3 * Sh::HALO;
  rg.bar = reinterpret_cast<uint64_t*>(rg.own + KT_NO * NOWN * Sh::OWN);
  rg.x0 = pos.x0;
  rg.x1 = pos.x1;
  rg.NX = g.NX;
  rg.plane0 = pos.s * g.NX;
  rg.j0 = pos.j0;
  rg.k0 = pos.k0;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = tg.zp, s = pos.s;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int PS = NY * zp;
  T* __restrict__ Ex = f.Ex + (long long)s * NX * PS;
  T* __restrict__ Ey = f.Ey + (long long)s * NX * PS;
  T* __restrict__ Ez = f.Ez + (long long)s * NX * PS;
  const bool pml = a.has_cpml != 0;
  int kc[2], zq[2];
  bool kv[2], exz[2], ezz[2], onk[2];
  int fz = 5;
  T tz[2][R];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = pos.k0 + 2 * lane + e;
    kc[e] = k;
    kv[e] = k < NZ;
    exz[e] = k > 0 && k < NZ - 1;
    ezz[e] = k < NZ - 1;
    onk[e] = kv[e] && k < NZ - 1;
    const int q0 = (kv[e] && pml && k > 0) ? q_low_e(a.eF[4].p, k) : -1;
    const int q1 = (kv[e] && pml && k > 0) ? q_high(a.eF[5].p, k, NZ) : -1;
    if (q0 >= 0) fz = 4;
    zq[e] = q0 >= 0 ? q0 : q1;
    taps_back<T, R>(k, NZ, tz[e]);
  }
  Prof<T> pz[2];
  const Face<T>& FZ = fz == 4 ? a.eF[4] : a.eF[5];
#pragma unroll
  for (int e = 0; e < 2; ++e) pz[e] = zq[e] >= 0 ? prof(FZ, zq[e]) : Prof<T>{0.0f, 0.0f, 0.0f, 0.0f};
  int jrow[2], qy[2];
  bool jv[2], exy[2], eyy[2], jl[2];
  T ty[2][R];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int j = pos.j0 + 2 * w + r;
    jrow[r] = j;
    jv[r] = j < NY;
    exy[r] = j > 0 && j < NY - 1;
    eyy[r] = j < NY - 1;
    jl[r] = j < NY - 1;
    const int q0 = (jv[r] && pml && j > 0) ? q_low_e(a.eF[2].p, j) : -1;
    const int q1 = (jv[r] && pml && j > 0) ? q_high(a.eF[3].p, j, NY) : -1;
    qy[r] = q0 >= 0 ? q0 : (q1 >= 0 ? q1 + 1024 : -1);
    taps_back<T, R>(j, NY, ty[r]);
  }
  const bool degx = NY - 1 != 1 || NZ - 1 != 1, degy = NX - 1 != 1 || NZ - 1 != 1, degz = NX - 1 != 1 || NY - 1 != 1;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save_r = a.keep_r && (it % a.S == 0);
  const int hslot = it / a.S;
  const int ncomp = a.mode == 3 ? 3 : 1;

  rg.start(maps);
  for (int i = pos.x0; i < pos.x1; ++i) {
    rg.wait_plane(i);
    const float* own = rg.own_slot(i);
    T tx[R];
    taps_back<T, R>(i, NX, tx);
    const bool exx = i < NX - 1, eyx = i > 0 && i < NX - 1, il = i < NX - 1;
    int qx = -1, fx = 0;
    if (pml && i > 0) {
      const int q0 = q_low_e(a.eF[0].p, i), q1 = q_high(a.eF[1].p, i, NX);
      qx = q0 >= 0 ? q0 : q1;
      fx = q0 >= 0 ? 0 : 1;
    }
    const bool pts = (tg.src_rows && tg.src_rows[(long long)s * NX + i]) ||
                     (tg.rcv_rows && tg.rcv_rows[(long long)s * NX + i]);
    const int bi = i - a.box.x0;
    const bool xin_box = save_r && bi >= 0 && bi < a.box.nx;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int jr = 2 * w + r, j = jrow[r];
      if (!jv[r]) continue;
      const int srow = (R + jr) * BZ;
      ZWin<LO, HI> zhx, zhy;
      const float* p0 = rg.slot(i);
      zhx.load(p0 + srow, lane);
      zhy.load(p0 + Sh::HALO + srow, lane);
      float2 yhx[HI - LO + 1], yhz[HI - LO + 1], xhy[HI - LO + 1], xhz[HI - LO + 1];
#pragma unroll
      for (int d = LO; d <= HI; ++d) {
        yhx[d - LO] = *reinterpret_cast<const float2*>(p0 + (R + jr + d) * BZ + 4 + 2 * lane);
        yhz[d - LO] = *reinterpret_cast<const float2*>(p0 + 2 * Sh::HALO + (R + jr + d) * BZ + 4 + 2 * lane);
        const float* pd = rg.slot(i + d);
        xhy[d - LO] = *reinterpret_cast<const float2*>(pd + Sh::HALO + srow + 4 + 2 * lane);
        xhz[d - LO] = *reinterpret_cast<const float2*>(pd + 2 * Sh::HALO + srow + 4 + 2 * lane);
      }
      const int oo = jr * KT_TZ + 2 * lane;
      const float2 e0v = *reinterpret_cast<const float2*>(own + oo);
      const float2 e1v = *reinterpret_cast<const float2*>(own + Sh::OWN + oo);
      const float2 e2v = *reinterpret_cast<const float2*>(own + 2 * Sh::OWN + oo);
      const float2 cav = *reinterpret_cast<const float2*>(own + 3 * Sh::OWN + oo);
      const float2 cbv = *reinterpret_cast<const float2*>(own + 4 * Sh::OWN + oo);
      T ex[2] = {e0v.x, e0v.y}, ey[2] = {e1v.x, e1v.y}, ez[2] = {e2v.x, e2v.y};
      const T c0[2] = {cav.x, cav.y}, c1[2] = {cbv.x, cbv.y};
      T ox[2], oy[2], oz[2];
      T dHz_dy[2], dHx_dy[2], dHz_dx[2], dHy_dx[2], dHy_dz[2], dHx_dz[2];
      bool dex[2], dey[2], dez[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const auto sel = [e](const float2& v) { return e == 0 ? v.x : v.y; };
        dHz_dy[e] = kt_dback<R>([&](int d) { return sel(yhz[d - LO]); }, ty[r]);
        dHx_dy[e] = kt_dback<R>([&](int d) { return sel(yhx[d - LO]); }, ty[r]);
        dHz_dx[e] = kt_dback<R>([&](int d) { return sel(xhz[d - LO]); }, tx);
        dHy_dx[e] = kt_dback<R>([&](int d) { return sel(xhy[d - LO]); }, tx);
        dHy_dz[e] = kt_dback<R>([&](int d) { return zhy.at(e, d); }, tz[e]);
        dHx_dz[e] = kt_dback<R>([&](int d) { return zhx.at(e, d); }, tz[e]);
        dex[e] = degx && exx && exy[r] && exz[e];
        dey[e] = degy && eyx && eyy[r] && exz[e];
        dez[e] = degz && eyx && exy[r] && ezz[e];
        const T cx = c1[e];
        const T cy = (EQ || a.dy_eq) ? cx : div_fixed(cx * a.dx, a.ddy);
        const T cz = (EQ || a.dz_eq) ? cx : div_fixed(cx * a.dx, a.ddz);
        ox[e] = ex[e];
        oy[e] = ey[e];
        oz[e] = ez[e];
        if (dex[e]) ex[e] = c0[e] * ex[e] + cy * dHz_dy[e] - cz * dHy_dz[e];
        if (dey[e]) ey[e] = c0[e] * ey[e] + cz * dHx_dz[e] - cx * dHz_dx[e];
        if (dez[e]) ez[e] = c0[e] * ez[e] + cx * dHy_dx[e] - cy * dHx_dy[e];
      }
      const long long go = (long long)i * PS + (long long)j * zp + kc[0];
      const bool cpml_cell = pml && (qx >= 0 || qy[r] >= 0 || zq[0] >= 0 || zq[1] >= 0);
      bool src_hit[2];
      int cell[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        cell[e] = (i * NY + j) * NZ + kc[e];
        src_hit[e] = kv[e] && pts && point_hit(P.src, s, cell[e]);
      }
      T cb[2] = {0.0f, 0.0f};
      if (cpml_cell || save_r || src_hit[0] || src_hit[1]) {
#pragma unroll
        for (int e = 0; e < 2; ++e) cb[e] = kv[e] ? f.ce_rhs[go + e] : 0.0f;
      }
      if (cpml_cell) {
        if (qx >= 0) {
          const Face<T>& F = a.eF[fx];
          const Prof<T> pr = prof(F, qx);
          const long long b1 = ((long long)(s * (F.p + 1) + qx) * (NY - 1) + j) * NZ;
          const long long b2 = ((long long)(s * (F.p + 1) + qx) * NY + j) * (NZ - 1);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (kv[e] && jl[r]) kt_cpml(F.psi1, b1 + kc[e], pr, dHz_dx[e], a.ddx, cb[e], false, ey[e]);
            if (onk[e]) kt_cpml(F.psi2, b2 + kc[e], pr, dHy_dx[e], a.ddx, cb[e], true, ez[e]);
          }
        }
        if (qy[r] >= 0) {
          const int q = qy[r] & 1023;
          const Face<T>& F = qy[r] >= 1024 ? a.eF[3] : a.eF[2];
          const Prof<T> pr = prof(F, q);
          const long long b1 = (((long long)s * (NX - 1) + i) * (F.p + 1) + q) * NZ;
          const long long b2 = (((long long)s * NX + i) * (F.p + 1) + q) * (NZ - 1);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (kv[e] && il) kt_cpml(F.psi1, b1 + kc[e], pr, dHz_dy[e], a.ddy, cb[e], true, ex[e]);
            if (onk[e]) kt_cpml(F.psi2, b2 + kc[e], pr, dHx_dy[e], a.ddy, cb[e], false, ez[e]);
          }
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (zq[e] < 0) continue;
          if (il) kt_cpml(FZ.psi1, (((long long)s * (NX - 1) + i) * NY + j) * (FZ.p + 1) + zq[e], pz[e], dHy_dz[e],
                          a.ddz, cb[e], false, ex[e]);
          if (jl[r]) kt_cpml(FZ.psi2, (((long long)s * NX + i) * (NY - 1) + j) * (FZ.p + 1) + zq[e], pz[e],
                             dHx_dz[e], a.ddz, cb[e], true, ey[e]);
        }
      }
      if (pts) {
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (src_hit[e]) inject_at(P, s, cell[e], it, cb[e], ex[e], ey[e], ez[e]);
      }
      if (save_r) {
        const bool rin = xin_box && j - a.box.y0 >= 0 && j - a.box.y0 < a.box.ny;
        bool ib[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) ib[e] = rin && kv[e] && kc[e] - a.box.z0 >= 0 && kc[e] - a.box.z0 < a.box.nz;
        const long long hoff = hslot * a.frame + s * a.box.cells() +
                               ((long long)bi * a.box.ny + (j - a.box.y0)) * a.box.nz + (kc[0] - a.box.z0);
        with_hist_kind(a.kind, [&](auto K) {
          constexpr int KIND = decltype(K)::value;
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            if (q >= ncomp) break;
            const int fc = a.mode == 3 ? q : 2;
            T rv[2];
            float am = 0.0f;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              rv[e] = 0.0f;
              if (ib[e]) {
                // R^n = (E^{n+1} - a_eff E^n) / cb (deepgpr_cpu.c:1850-1875)
                const T en = fc == 0 ? ex[e] : (fc == 1 ? ey[e] : ez[e]);
                const T eo = fc == 0 ? ox[e] : (fc == 1 ? oy[e] : oz[e]);
                const bool du = fc == 0 ? dex[e] : (fc == 1 ? dey[e] : dez[e]);
                const T aeff = du ? c0[e] : 1.0f;
                rv[e] = cb[e] != 0.0f ? (en - aeff * eo) / cb[e] : 0.0f;
                am = fmaxf(am, fabsf(rv[e]));
              }
            }
            float inv = 1.0f;
            if (is_tiled(KIND)) {
              const float sc = tile_scale_of(KIND, half_absmax(am));
              inv = 1.0f / sc;
              if ((lane & 15) == 0 && kc[0] < NZ)
                a.r_scales[(((long long)q * a.nt_saved + hslot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j, kc[0])] =
                    sc;
            }
            const long long hq = q * a.comp_stride + hoff;
            if (ib[0]) hist_store<T>(a.R_saved, hq, rv[0], KIND, inv);
            if (ib[1]) hist_store<T>(a.R_saved, hq + 1, rv[1], KIND, inv);
          }
        });
      }
      if (pts) {
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (kv[e]) sample_at(P, s, cell[e], it, ex[e], ey[e], ez[e]);
      }
      if (kv[1]) {
        *reinterpret_cast<float2*>(Ex + go) = make_float2(ex[0], ex[1]);
        *reinterpret_cast<float2*>(Ey + go) = make_float2(ey[0], ey[1]);
        *reinterpret_cast<float2*>(Ez + go) = make_float2(ez[0], ez[1]);
      } else if (kv[0]) {
        Ex[go] = ex[0];
        Ey[go] = ey[0];
        Ez[go] = ez[0];
      }
    }
    if (!rg.advance(maps, i)) {
      rg.fail(tg.ctrl);
      return;
    }
  }
}

}  // namespace dg
