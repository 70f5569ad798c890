// fdtd_3d.cuh -- 3D kernels: 64-column warp strips streaming along x.
//
// Layout inside a call: a z-pitched working copy (shot, NX, NY, zp) of the six
// field components and (NX, NY, zp) copies of the coefficients, zp = NZ
// rounded up to 32 (zero padding, never written), so every z row starts on a
// 128-byte boundary.  CPML psi arrays, histories and point tables keep the
// caller's logical layout.
//
// Execution: a CTA holds K3_WARPS warps on consecutive y rows of one
// 64-column z strip, one shot and one x chunk; every warp streams along x:
//   * lane l holds columns k0 + 2l, k0 + 2l + 1 (one 8-byte access per row);
//   * x-stencils read register queues of the 2R planes around the current one;
//   * y-stencils read the neighbouring rows directly (the CTA's own rows come
//     from L1, the halo rows from L2);
//   * z-stencils take the neighbouring columns from the other lanes with warp
//     shuffles; lanes 0..2R-1 also hold the R halo columns on each side;
//   * the next plane's operands are loaded before the current plane is
//     computed.
// Every derivative is first formed with the full stencil (neighbours outside
// the grid read as zero); the x and y boundary work (clamped stencils, CPML
// faces, update predicates) is uniform over a warp and runs only on the
// planes / rows that need it; only the first and last z strips carry per-lane
// z boundary work.  In FP32 the H z-face CPML corrections (k3z_fwd_h) and,
// without a stored R^n history, the E CPML frame (k3p_fwd_e) are finished by
// per-cell passes after the streamed kernel.  Per-cell arithmetic is that of
// the reference (src/DeepGPR/lib/deepgpr_cpu.c:670-1100) in the same order.
#pragma once

#include "fdtd_tm2d.cuh"

namespace dg {

constexpr int K3W = 64;       // z columns per warp strip (two per lane)
constexpr int K3_WARPS = 4;   // warps (y rows) per CTA
// Resident CTAs per SM the 3D kernels are built for: 12 warps per SM in FP32
// at radius <= 2 (<= 168 registers a thread), 8 otherwise.
template <typename T, int R>
__host__ __device__ constexpr int k3_min_blocks() {
  return (((R >= 4 || sizeof(T) == 8) ? 8 : 12) + K3_WARPS - 1) / K3_WARPS;
}
// The adjoint kernels fit 128 registers a thread without spilling at radius
// <= 2 in FP32: 16 warps per SM (measured 7-9 % faster than 12 on
// 320 x 320 x 160 + CPML; the forward kernels spill at 128 and lose).
template <typename T, int R>
__host__ __device__ constexpr int k3_adj_min_blocks() {
  return (((R >= 4 || sizeof(T) == 8) ? 8 : 16) + K3_WARPS - 1) / K3_WARPS;
}

// CPML forms of the z-streamed forward kernels: the staged single-face form
// (faces of an axis at least 4 cells apart), the general per-face form, and
// none in the streamed kernel: every cell gets its base update there and the
// CPML frame is finished by a per-cell pass kernel (k3p_fwd_e; E half step).
constexpr int kCpmSingle = 0, kCpmGeneral = 1, kCpmPass = 2;

// CPML frame of the pass form: along each axis the cells 0 .. lo-1 and
// hi .. n-1 (each face's CPML cells plus the cell at the grid end), as six
// disjoint boxes (x low, x high, y low and high within x's interior, z low
// and high within x's and y's interior): origin o, extents n, cumulative cell
// counts over one shot.
struct K3Frame {
  int lo[3], hi[3];
  int o[6][3], n[6][3];
  unsigned cum[6];
};

struct K3Geom {
  int zp;                          // z pitch of the working copy (multiple of 32)
  int nzs, nyt;                    // z strips per row, y tiles (of K3_WARPS rows) per plane
  int xc, nchunk;                  // x chunk length, chunks
  long long nblocks;               // nshot * nzs * nyt * nchunk
  const unsigned char* src_rows;   // (nshot, NX): the plane holds a source of the shot
  const unsigned char* rcv_rows;   // (nshot, NX): the plane holds a receiver of the shot
  int cpml_single;                 // along every axis the two CPML faces are >= 4 cells apart
  K3Frame fr;                      // CPML frame of the pass form (E half step)
  int zpost_h;                     // H z-face corrections in k3z_fwd_h after k3v_fwd_h
};

// (rows, n) <-> (rows, pitch) with zero padding: one warp per row, lanes over
// the columns (no integer division per element).
template <typename T>
__global__ void k_pack_rows(const T* __restrict__ src, T* __restrict__ dst, long long rows, int n, int pitch) {
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += nw) {
    const T* __restrict__ s = src + r * n;
    T* __restrict__ d = dst + r * pitch;
    for (int c = lane; c < pitch; c += 32) d[c] = c < n ? s[c] : T(0);
  }
}
template <typename T>
__global__ void k_unpack_rows(const T* __restrict__ src, T* __restrict__ dst, long long rows, int n, int pitch) {
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += nw) {
    const T* __restrict__ s = src + r * pitch;
    T* __restrict__ d = dst + r * n;
    for (int c = lane; c < n; c += 32) d[c] = s[c];
  }
}

template <typename T>
struct K3Buf {
  T *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;                            // (nshot, NX, NY, zp)
  const T *ce_hist, *ce_curl, *ce_rhs, *ch_curl, *ch_rhs;   // (NX, NY, zp)
};

template <typename T>
__device__ __forceinline__ void ld2(const T* p, T (&o)[2]) {
  if constexpr (sizeof(T) == 4) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    o[0] = v.x;
    o[1] = v.y;
  } else {
    const double2 v = *reinterpret_cast<const double2*>(p);
    o[0] = v.x;
    o[1] = v.y;
  }
}
template <typename T>
__device__ __forceinline__ void st2(T* p, const T (&v)[2]) {
  if constexpr (sizeof(T) == 4) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  else *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}

// absmax over the 16 lanes holding one 32-column FP8 tile
__device__ __forceinline__ float half_absmax(float v) {
  for (int o = 8; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFullMask, v, o));
  return v;
}

struct K3Pos {
  int lane, s, j, k0, kk, x0, x1;
  bool live;
};

// block -> (shot fastest, z strip, y tile, x chunk); CTAs of the same tile
// and different shots run together and share the coefficient rows in L2.
__device__ __forceinline__ K3Pos k3_pos(const K3Geom& kg, const Grid& g) {
  K3Pos p;
  p.lane = threadIdx.x;
  unsigned b = blockIdx.x;
  const unsigned ns = (unsigned)g.nshot, nz = (unsigned)kg.nzs, ny = (unsigned)kg.nyt;
  unsigned q = b / ns;
  p.s = int(b - q * ns);
  b = q;
  q = b / nz;
  const int zs = int(b - q * nz);
  b = q;
  q = b / ny;
  const int yt = int(b - q * ny);
  const int chunk = int(q);
  p.j = yt * K3_WARPS + threadIdx.y;
  p.live = p.j < g.NY && chunk < kg.nchunk;
  p.k0 = zs * K3W;
  p.kk = p.k0 + 2 * p.lane;
  p.x0 = chunk * kg.xc;
  p.x1 = min(p.x0 + kg.xc, g.NX);
  return p;
}

// Halo column of a lane (see halo_col2 in the 2D kernels): lanes [0, R) hold
// k0 - R + lane, lanes [R, 2R) hold k0 + 64 + lane - R.
template <int R>
__device__ __forceinline__ int k3_halo(int k0, int lane) {
  return lane < R ? k0 - R + lane : k0 + K3W + lane - R;
}

// z[m - MLO] = value at column kk + m (MLO <= m <= MHI, |m| <= R + 1), from
// the lanes' own pairs (constant-distance shuffles) and, for the lanes at the
// strip ends, the halo lanes.  All lanes call it.
template <typename T, int R, int MLO, int MHI>
__device__ __forceinline__ void znb(const T (&v)[2], T halo, int lane, T (&z)[MHI - MLO + 1]) {
#pragma unroll
  for (int m = MLO; m <= MHI; ++m) {
    if (m == 0 || m == 1) {
      z[m - MLO] = v[m];
    } else if (m < 0) {
      const int sh = (1 - m) / 2;   // -floor(m / 2)
      const T x = __shfl_up_sync(kFullMask, v[m & 1], sh);
      const T h = __shfl_sync(kFullMask, halo, (2 * lane + m + R) & 31);
      z[m - MLO] = lane >= sh ? x : h;
    } else {
      const int sh = m / 2;
      const T x = __shfl_down_sync(kFullMask, v[m & 1], sh);
      const T h = __shfl_sync(kFullMask, halo, (2 * lane + m - K3W + R) & 31);
      z[m - MLO] = lane + sh <= 31 ? x : h;
    }
  }
}

// Taps of the forward / backward staggered difference at coordinate c of an
// axis of n points: tap(rr, r) for r <= rr and zero beyond, rr the largest
// radius whose stencil fits (deepgpr_cpu.c:287-407).  With them a difference
// needs no branch near the ends; where the full stencil fits the taps are
// those of dfwd_full / dback_full and the result is the same.
template <typename T, int R>
__device__ __forceinline__ void taps_fwd(int c, int n, T (&t)[R]) {
  const int rr = rad_fwd(c, n, R);
#pragma unroll
  for (int r = 1; r <= R; ++r) t[r - 1] = r <= rr ? tap<T>(rr, r) : T(0);
}
template <typename T, int R>
__device__ __forceinline__ void taps_back(int c, int n, T (&t)[R]) {
  const int rr = rad_back(c, n, R);
#pragma unroll
  for (int r = 1; r <= R; ++r) t[r - 1] = r <= rr ? tap<T>(rr, r) : T(0);
}
template <typename T, int R, typename F>
__device__ __forceinline__ T dfwd_t(const F& f, const T (&t)[R]) {
  if (R == 1) return f(1) - f(0);
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) acc += t[r - 1] * (f(r) - f(-(r - 1)));
  return acc;
}
template <typename T, int R, typename F>
__device__ __forceinline__ T dback_t(const F& f, const T (&t)[R]) {
  if (R == 1) return f(0) - f(-1);
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) acc += t[r - 1] * (f(r - 1) - f(-r));
  return acc;
}

// Calls f(std::integral_constant<int, KIND>) for the history kind (one
// uniform switch, so the stores inside f compile for that kind only).
template <typename F>
__device__ __forceinline__ void with_hist_kind(int kind, F f) {
  switch (kind) {
    case kF16: f(std::integral_constant<int, kF16>()); break;
    case kBF16: f(std::integral_constant<int, kBF16>()); break;
    case kFP8: f(std::integral_constant<int, kFP8>()); break;
    case kI8: f(std::integral_constant<int, kI8>()); break;
    case kF64: f(std::integral_constant<int, kF64>()); break;
    default: f(std::integral_constant<int, kF32>()); break;
  }
}

// CPML correction of one face for the lane's pair: psi at index base + off[e]
// (off = k for x / y faces, q for z faces); u[e] += sgn * c[e] (ra1 d + rb psi),
// psi <- re psi - rf d, d = dv[e] / h (deepgpr_cpu.c:939-1100 order).
template <typename T>
__device__ __forceinline__ void cpml_pair(T* psi, long long base, const int (&off)[2], const bool (&on)[2],
                                          const Prof<T>& pr, const T (&dv)[2], const FixedDiv<T>& h, const T (&c)[2], T sgn,
                                          T (&u)[2]) {
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    if (!on[e]) continue;
    const long long pi = base + off[e];
    const T d = div_fixed(dv[e], h), ph = psi[pi];
    if (sgn > T(0)) u[e] += c[e] * (pr.ra1 * d + pr.rb * ph);
    else u[e] -= c[e] * (pr.ra1 * d + pr.rb * ph);
    psi[pi] = pr.re * ph - pr.rf * d;
  }
}

// One CPML recurrence with psi already loaded: u +-= c (ra1 d + rb psi),
// psi <- re psi - rf d, d = dv / h (deepgpr_cpu.c:939-1100 order).
template <typename T>
__device__ __forceinline__ void cpml_one(T* psi, long long pi, T ph, const Prof<T>& pr, T dv, const FixedDiv<T>& h,
                                         T c, bool plus, T& u) {
  const T d = div_fixed(dv, h);
  if (plus) u += c * (pr.ra1 * d + pr.rb * ph);
  else u -= c * (pr.ra1 * d + pr.rb * ph);
  psi[pi] = pr.re * ph - pr.rf * d;
}

// psi rows of a y or z CPML face at plane 0 of shot s and row j; plane i
// adds i * stride (psi extents from psi_dims_e / psi_dims_h).
template <typename T>
struct FaceRows {
  T* p1;
  T* p2;
  int s1, s2;
};

// (the low face lo when `low`, else hi; fields are selected one by one so that
// the kernel parameter array is never indexed at run time)
template <typename T, bool EFIELD>
__device__ __forceinline__ FaceRows<T> face_rows(const Face<T>& lo, const Face<T>& hi, bool low, const Grid& g,
                                                 int axis, int s, int j, int q) {
  const int p = low ? lo.p : hi.p;
  const PsiDims d1 = EFIELD ? psi_dims_e(g, axis, 1, p) : psi_dims_h(g, axis, 1, p);
  const PsiDims d2 = EFIELD ? psi_dims_e(g, axis, 2, p) : psi_dims_h(g, axis, 2, p);
  FaceRows<T> r;
  r.p1 = (low ? lo.psi1 : hi.psi1) + psi_index(d1, axis, s, q, 0, j, 0);
  r.p2 = (low ? lo.psi2 : hi.psi2) + psi_index(d2, axis, s, q, 0, j, 0);
  r.s1 = d1.b * d1.c;
  r.s2 = d2.b * d2.c;
  return r;
}

// x CPML face of plane i (-1: none) and its psi offsets of row j, column 0
template <typename T, bool EFIELD>
__device__ __forceinline__ int xface_at(const Face<T>* F, const Grid& g, int s, int i, int j, long long& b1,
                                        long long& b2) {
  const int q0 = EFIELD ? (i > 0 ? q_low_e(F[0].p, i) : -1) : q_low_h(F[0].p, i);
  const int q1 = (EFIELD && i == 0) ? -1 : q_high(F[1].p, i, g.NX);
  const int fx = q0 >= 0 ? 0 : (q1 >= 0 ? 1 : -1);
  const int q = q0 >= 0 ? q0 : q1, p = q0 >= 0 ? F[0].p : F[1].p;
  const PsiDims d1 = EFIELD ? psi_dims_e(g, 0, 1, p) : psi_dims_h(g, 0, 1, p);
  const PsiDims d2 = EFIELD ? psi_dims_e(g, 0, 2, p) : psi_dims_h(g, 0, 2, p);
  b1 = psi_index(d1, 0, s, q, i, j, 0);
  b2 = psi_index(d2, 0, s, q, i, j, 0);
  return fx;
}

// 4- or 8-byte global -> shared copy that bypasses the registers (sm_80+ cp.async)
template <typename T>
__device__ __forceinline__ void cp_async(T* smem, const T* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(sizeof(T)));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// all but the most recent group of this thread have landed and are visible to it
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Staged CPML operands of one plane, per warp: [stage][slot][cell][lane];
// slots x psi1, x psi2, y psi1, y psi2, z psi1, z psi2, curl-rhs coefficient.
constexpr int kStageSlots = 7;

// ---------------------------------------------------------------------------
// 3D H half step (+ E^n history).  EQ: dx == dy == dz (curl scale 1); CPM:
// CPML form (kCpmSingle, kCpmGeneral, kCpmPass).
// ---------------------------------------------------------------------------
template <typename T, int R, bool EQ, int CPM>
__global__ void __launch_bounds__(32 * K3_WARPS, k3_min_blocks<T, R>()) k3v_fwd_h(TiledFwd<T> P, K3Buf<T> f, K3Geom kg) {
  constexpr int ZLO = -(R - 1), ZHI = R + 1, NZN = ZHI - ZLO + 1;   // z neighbours of the pair, dfwd
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const K3Pos wp = k3_pos(kg, g);
  if (!wp.live) return;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const int PS = NY * zp;                                  // plane stride
  const long long sbase = (long long)s * NX * PS;
  const T* __restrict__ Ex = f.Ex + sbase;
  const T* __restrict__ Ey = f.Ey + sbase;
  const T* __restrict__ Ez = f.Ez + sbase;
  T* __restrict__ Hx = f.Hx + sbase;
  T* __restrict__ Hy = f.Hy + sbase;
  T* __restrict__ Hz = f.Hz + sbase;
  const T* __restrict__ cc = f.ch_curl;
  const bool pml = CPM != kCpmPass && a.has_cpml;   // CPML handled in this kernel
  const int hk = k3_halo<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;                              // offset of the lane's pair in a plane
  const int hrow = j * zp + (hok ? hk : 0);
  bool kv[2], hxz[2], hzz[2], kl[2];
  int qz0[2], qz1[2], kof[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = kk + e;
    kv[e] = k < NZ;
    kof[e] = k;
    hxz[e] = k < NZ - 1;                          // z part of upd_hx and upd_hy
    hzz[e] = NZ - 1 != 1 && k > 0 && k < NZ - 1;  // z part of upd_hz
    kl[e] = kv[e] && k < NZ - 1;
    qz0[e] = (kv[e] && pml && !kg.zpost_h) ? q_low_h(a.hF[4].p, k) : -1;
    qz1[e] = (kv[e] && pml && !kg.zpost_h) ? q_high(a.hF[5].p, k, NZ) : -1;
  }
  const bool zpml = qz0[0] >= 0 || qz1[0] >= 0 || qz0[1] >= 0 || qz1[1] >= 0;
  const bool any_zpml = __any_sync(kFullMask, zpml);
  T tz[2][R], ty[R];   // difference taps along z (per column) and y (per row)
  taps_fwd<T, R>(kk, NZ, tz[0]);
  taps_fwd<T, R>(kk + 1, NZ, tz[1]);
  taps_fwd<T, R>(j, NY, ty);
  // y parts (uniform over the warp)
  const bool hxy = j < NY - 1, hyy = NY - 1 != 1 && j > 0 && j < NY - 1;
  const int qy0 = pml ? q_low_h(a.hF[2].p, j) : -1;
  const int qy1 = pml ? q_high(a.hF[3].p, j, NY) : -1;
  const bool in_y = qy0 >= 0 || qy1 >= 0;
  // CPML rows of the row's y face and the lane's z face (faces of one axis apart)
  const bool cps = CPM == kCpmSingle && pml;
  const int fz = (qz0[0] >= 0 || qz0[1] >= 0) ? 4 : 5;
  int zq[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) zq[e] = fz == 4 ? qz0[e] : qz1[e];
  const FaceRows<T> yr = face_rows<T, false>(a.hF[2], a.hF[3], qy0 >= 0, g, 1, s, 0, qy0 >= 0 ? qy0 : qy1);
  const FaceRows<T> zr = face_rows<T, false>(a.hF[4], a.hF[5], fz == 4, g, 2, s, j, 0);
  Prof<T> pz[2];   // CPML profile of the lane's z-face cells (fixed along x)
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    pz[e] = Prof<T>{T(0), T(0), T(0), T(0)};
    if (cps && zq[e] >= 0) pz[e] = fz == 4 ? prof(a.hF[4], zq[e]) : prof(a.hF[5], zq[e]);
  }
  __shared__ T stg[K3_WARPS][2][kStageSlots][2][32];
  T(*const sg)[kStageSlots][2][32] = stg[threadIdx.y];
  const bool onk[2] = {kl[0], kl[1]}, jl = j < NY - 1;
  // issues the CPML operands of plane i into stage b (one commit group per plane)
  auto stage = [&](int i, int b) {
    long long bx1 = 0, bx2 = 0;
    int fx = -1;
    if (cps && (q_low_h(a.hF[0].p, i) >= 0 || q_high(a.hF[1].p, i, NX) >= 0))
      fx = xface_at<T, false>(a.hF, g, s, i, j, bx1, bx2);
    if (cps && (fx >= 0 || in_y || any_zpml)) {
      const bool il = i < NX - 1;
      const T* X1 = fx == 0 ? a.hF[0].psi1 : a.hF[1].psi1;
      const T* X2 = fx == 0 ? a.hF[0].psi2 : a.hF[1].psi2;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const bool zon = zq[e] >= 0;
        if (kv[e] && (fx >= 0 || in_y || zon)) cp_async(&sg[b][6][e][lane], f.ch_rhs + i * PS + row + e);
        if (fx >= 0 && onk[e]) cp_async(&sg[b][0][e][lane], X1 + bx1 + kof[e]);
        if (fx >= 0 && kv[e] && jl) cp_async(&sg[b][1][e][lane], X2 + bx2 + kof[e]);
        if (in_y && onk[e]) cp_async(&sg[b][2][e][lane], yr.p1 + (long long)i * yr.s1 + kof[e]);
        if (in_y && kv[e] && il) cp_async(&sg[b][3][e][lane], yr.p2 + (long long)i * yr.s2 + kof[e]);
        if (zon && jl) cp_async(&sg[b][4][e][lane], zr.p1 + (long long)i * zr.s1 + zq[e]);
        if (zon && il) cp_async(&sg[b][5][e][lane], zr.p2 + (long long)i * zr.s2 + zq[e]);
      }
    }
    cp_async_commit();
  };
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save = a.save_e && (it % a.S == 0);
  const int slot = it / a.S;
  const int ncomp = a.mode == 3 ? 3 : 1;
  // history box position of the lane's cells (the x part is added per plane)
  const bool brow = j - a.box.y0 >= 0 && j - a.box.y0 < a.box.ny;
  const bool bok[2] = {kv[0] && kk - a.box.z0 >= 0 && kk - a.box.z0 < a.box.nz,
                       kv[1] && kk + 1 - a.box.z0 >= 0 && kk + 1 - a.box.z0 < a.box.nz};
  const long long bplane = (long long)a.box.ny * a.box.nz;
  const long long h0 = (long long)(j - a.box.y0) * a.box.nz + (kk - a.box.z0);
  const long long hb = slot * a.frame + s * a.box.cells();
  T qEy[2 * R][2], qEz[2 * R][2];   // Ey, Ez at planes i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = wp.x0 - R + 1 + m;
    if (pl >= 0 && pl < NX) {
      ld2(Ey + pl * PS + row, qEy[m]);
      ld2(Ez + pl * PS + row, qEz[m]);
    } else {
      qEy[m][0] = qEy[m][1] = qEz[m][0] = qEz[m][1] = T(0);
    }
  }
  // operands of the next plane
  T nEx[2], nEyq[2], nEzq[2], nhx[2], nhy[2], nhz[2], nc[2], nhEx = T(0), nhEy = T(0);
  T nExy[2 * R][2], nEzy[2 * R][2];   // Ex, Ez at rows j + d, d = -(R-1) .. R (own row slot unused)
  auto fetch = [&](int i) {
    const int o = i * PS;
    ld2(Ex + o + row, nEx);
    if (i + R < NX) {
      ld2(Ey + o + R * PS + row, nEyq);
      ld2(Ez + o + R * PS + row, nEzq);
    } else {
      nEyq[0] = nEyq[1] = nEzq[0] = nEzq[1] = T(0);
    }
    if (hok) {
      nhEx = Ex[o + hrow];
      nhEy = Ey[o + hrow];
    }
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) {
      if (d == 0) continue;
      if (j + d >= 0 && j + d < NY) {
        ld2(Ex + o + row + d * zp, nExy[d + R - 1]);
        ld2(Ez + o + row + d * zp, nEzy[d + R - 1]);
      } else {
        nExy[d + R - 1][0] = nExy[d + R - 1][1] = nEzy[d + R - 1][0] = nEzy[d + R - 1][1] = T(0);
      }
    }
    ld2(Hx + o + row, nhx);
    ld2(Hy + o + row, nhy);
    ld2(Hz + o + row, nhz);
    ld2(cc + o + row, nc);
  };
  fetch(wp.x0);
  stage(wp.x0, 0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    T ex[2], hx[2], hy[2], hz[2], c1[2], exy[2 * R][2], ezy[2 * R][2];
    const T hEx = nhEx, hEy = nhEy;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      ex[e] = nEx[e];
      qEy[2 * R - 1][e] = nEyq[e];
      qEz[2 * R - 1][e] = nEzq[e];
      hx[e] = nhx[e];
      hy[e] = nhy[e];
      hz[e] = nhz[e];
      c1[e] = nc[e];
#pragma unroll
      for (int m = 0; m < 2 * R; ++m) {
        exy[m][e] = nExy[m][e];
        ezy[m][e] = nEzy[m][e];
      }
    }
    if (i + 1 < wp.x1) {
      fetch(i + 1);
      stage(i + 1, (i + 1 - wp.x0) & 1);
    } else {
      cp_async_commit();
    }
    const int o = i * PS;
    T zx[NZN], zy[NZN];   // Ex, Ey at columns kk + m of this plane
    znb<T, R, ZLO, ZHI>(ex, hEx, lane, zx);
    znb<T, R, ZLO, ZHI>(qEy[R - 1], hEy, lane, zy);
    if (save) {
      const int bi = i - a.box.x0;
      const bool rin = brow && bi >= 0 && bi < a.box.nx;
      const bool ib[2] = {rin && bok[0], rin && bok[1]};
      const long long hoff = hb + (long long)bi * bplane + h0;   // history index of the lane's first cell
      with_hist_kind(a.kind, [&](auto K) {
        constexpr int KIND = decltype(K)::value;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (q >= ncomp) break;
          const int fc = a.mode == 3 ? q : 2;
          T v[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) v[e] = fc == 0 ? ex[e] : (fc == 1 ? qEy[R - 1][e] : qEz[R - 1][e]);
          float inv = 1.0f;
          if (is_tiled(KIND)) {
            float am = 0.0f;
#pragma unroll
            for (int e = 0; e < 2; ++e)
              if (ib[e]) am = fmaxf(am, fabsf(float(v[e])));
            const float sc = tile_scale_of(KIND, half_absmax(am));
            inv = 1.0f / sc;
            if ((lane & 15) == 0 && kk < NZ)
              a.e_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j, kk)] = sc;
          }
          const long long hq = q * a.comp_stride + hoff;
          if (ib[0]) hist_store<T>(a.E_saved, hq, v[0], KIND, inv);
          if (ib[1]) hist_store<T>(a.E_saved, hq + 1, v[1], KIND, inv);
        }
      });
    }
    // x parts (uniform over the warp)
    T tx[R];
    taps_fwd<T, R>(i, NX, tx);
    const bool hxx = NX - 1 != 1 && i > 0 && i < NX - 1, hyx = i < NX - 1;
    const int qx0 = pml ? q_low_h(a.hF[0].p, i) : -1;
    const int qx1 = pml ? q_high(a.hF[1].p, i, NX) : -1;
    const bool in_x = qx0 >= 0 || qx1 >= 0;
    T dEz_dy[2], dEx_dy[2], dEz_dx[2], dEy_dx[2], dEy_dz[2], dEx_dz[2], cyv[2], czv[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const auto fzx = [&](int d) { return zx[e + d - ZLO]; };
      const auto fzy = [&](int d) { return zy[e + d - ZLO]; };
      const auto fyz = [&](int d) { return d == 0 ? qEz[R - 1][e] : ezy[d + R - 1][e]; };
      const auto fyx = [&](int d) { return d == 0 ? ex[e] : exy[d + R - 1][e]; };
      const auto fxz = [&](int d) { return qEz[R - 1 + d][e]; };
      const auto fxy = [&](int d) { return qEy[R - 1 + d][e]; };
      dEz_dy[e] = dfwd_t<T, R>(fyz, ty);
      dEx_dy[e] = dfwd_t<T, R>(fyx, ty);
      dEz_dx[e] = dfwd_t<T, R>(fxz, tx);
      dEy_dx[e] = dfwd_t<T, R>(fxy, tx);
      dEy_dz[e] = dfwd_t<T, R>(fzy, tz[e]);
      dEx_dz[e] = dfwd_t<T, R>(fzx, tz[e]);
      const T cx = c1[e];
      cyv[e] = (EQ || a.dy_eq) ? cx : div_fixed(cx * a.dx, a.ddy);   // per-axis scale, as curl_scale
      czv[e] = (EQ || a.dz_eq) ? cx : div_fixed(cx * a.dx, a.ddz);
      if (hxx && hxy && hxz[e]) hx[e] = hx[e] - cyv[e] * dEz_dy[e] + czv[e] * dEy_dz[e];
      if (hyx && hyy && hxz[e]) hy[e] = hy[e] - czv[e] * dEx_dz[e] + cx * dEz_dx[e];
      if (hyx && hxy && hzz[e]) hz[e] = hz[e] - cx * dEy_dx[e] + cyv[e] * dEx_dy[e];
    }
    if (cps && (in_x || in_y || any_zpml)) {
      // staged operands of this plane; faces update in the reference order x, y, z
      cp_async_wait_prev();
      const int b = (i - wp.x0) & 1;
      const bool il = i < NX - 1;
      T up[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) up[e] = (kv[e] && (in_x || in_y || zq[e] >= 0)) ? sg[b][6][e][lane] : T(0);
      if (in_x) {
        long long bx1, bx2;
        const int fx = xface_at<T, false>(a.hF, g, s, i, j, bx1, bx2);
        const Prof<T> pr = fx == 0 ? prof(a.hF[0], qx0) : prof(a.hF[1], qx1);
        T* X1 = fx == 0 ? a.hF[0].psi1 : a.hF[1].psi1;
        T* X2 = fx == 0 ? a.hF[0].psi2 : a.hF[1].psi2;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (onk[e]) cpml_one<T>(X1, bx1 + kof[e], sg[b][0][e][lane], pr, dEz_dx[e], a.ddx, up[e], true, hy[e]);
          if (kv[e] && jl) cpml_one<T>(X2, bx2 + kof[e], sg[b][1][e][lane], pr, dEy_dx[e], a.ddx, up[e], false, hz[e]);
        }
      }
      if (in_y) {
        const Prof<T> pr = qy0 >= 0 ? prof(a.hF[2], qy0) : prof(a.hF[3], qy1);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (onk[e])
            cpml_one<T>(yr.p1, (long long)i * yr.s1 + kof[e], sg[b][2][e][lane], pr, dEz_dy[e], a.ddy, up[e], false,
                        hx[e]);
          if (kv[e] && il)
            cpml_one<T>(yr.p2, (long long)i * yr.s2 + kof[e], sg[b][3][e][lane], pr, dEx_dy[e], a.ddy, up[e], true,
                        hz[e]);
        }
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (zq[e] < 0) continue;
        const Prof<T>& pr = pz[e];
        if (jl)
          cpml_one<T>(zr.p1, (long long)i * zr.s1 + zq[e], sg[b][4][e][lane], pr, dEy_dz[e], a.ddz, up[e], true, hx[e]);
        if (il)
          cpml_one<T>(zr.p2, (long long)i * zr.s2 + zq[e], sg[b][5][e][lane], pr, dEx_dz[e], a.ddz, up[e], false,
                      hy[e]);
      }
    } else if (CPM == kCpmGeneral && (in_x || in_y || any_zpml)) {
      // faces of one axis meet: the general per-face form
      T up[2];
      bool zon[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        zon[e] = qz0[e] >= 0 || qz1[e] >= 0;
        up[e] = (kv[e] && (in_x || in_y || zon[e])) ? f.ch_rhs[o + row + e] : T(0);
      }
      const bool jl = j < NY - 1, il = i < NX - 1;
      const bool onk[2] = {kl[0], kl[1]}, onj[2] = {kv[0] && jl, kv[1] && jl}, oni[2] = {kv[0] && il, kv[1] && il};
#pragma unroll
      for (int fc = 0; fc < 2; ++fc) {
        const int q = fc == 0 ? qx0 : qx1;
        if (q < 0) continue;
        const Face<T>& F = a.hF[fc];
        const Prof<T> pr = prof(F, q);
        cpml_pair<T>(F.psi1, psi_index(psi_dims_h(g, 0, 1, F.p), 0, s, q, i, j, 0), kof, onk, pr, dEz_dx, a.ddx, up,
                     T(1), hy);
        cpml_pair<T>(F.psi2, psi_index(psi_dims_h(g, 0, 2, F.p), 0, s, q, i, j, 0), kof, onj, pr, dEy_dx, a.ddx, up,
                     T(-1), hz);
      }
#pragma unroll
      for (int fc = 2; fc < 4; ++fc) {
        const int q = fc == 2 ? qy0 : qy1;
        if (q < 0) continue;
        const Face<T>& F = a.hF[fc];
        const Prof<T> pr = prof(F, q);
        cpml_pair<T>(F.psi1, psi_index(psi_dims_h(g, 1, 1, F.p), 1, s, q, i, j, 0), kof, onk, pr, dEz_dy, a.ddy, up,
                     T(-1), hx);
        cpml_pair<T>(F.psi2, psi_index(psi_dims_h(g, 1, 2, F.p), 1, s, q, i, j, 0), kof, oni, pr, dEx_dy, a.ddy, up,
                     T(1), hz);
      }
      if (any_zpml) {
#pragma unroll
        for (int fc = 4; fc < 6; ++fc) {
          const Face<T>& F = a.hF[fc];
          int qq[2];
          bool o1[2], o2[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            qq[e] = fc == 4 ? qz0[e] : qz1[e];
            o1[e] = qq[e] >= 0 && jl;
            o2[e] = qq[e] >= 0 && il;
          }
          if (!(o1[0] || o1[1] || o2[0] || o2[1])) continue;
          Prof<T> pr[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) pr[e] = prof(F, qq[e] >= 0 ? qq[e] : 0);
          const long long b1 = psi_index(psi_dims_h(g, 2, 1, F.p), 2, s, 0, i, j, 0);
          const long long b2 = psi_index(psi_dims_h(g, 2, 2, F.p), 2, s, 0, i, j, 0);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (o1[e]) {
              const T d = div_fixed(dEy_dz[e], a.ddz), ph = F.psi1[b1 + qq[e]];
              hx[e] += up[e] * (pr[e].ra1 * d + pr[e].rb * ph);
              F.psi1[b1 + qq[e]] = pr[e].re * ph - pr[e].rf * d;
            }
            if (o2[e]) {
              const T d = div_fixed(dEx_dz[e], a.ddz), ph = F.psi2[b2 + qq[e]];
              hy[e] -= up[e] * (pr[e].ra1 * d + pr[e].rb * ph);
              F.psi2[b2 + qq[e]] = pr[e].re * ph - pr[e].rf * d;
            }
          }
        }
      }
    }
    if (kv[1]) {
      st2(Hx + o + row, hx);
      st2(Hy + o + row, hy);
      st2(Hz + o + row, hz);
    } else if (kv[0]) {
      Hx[o + row] = hx[0];
      Hy[o + row] = hy[0];
      Hz[o + row] = hz[0];
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        qEy[m][e] = qEy[m + 1][e];
        qEz[m][e] = qEz[m + 1][e];
      }
  }
}

// ---------------------------------------------------------------------------
// 3D E half step (+ sources, R^n history, receivers).  With CPM == kCpmPass
// the CPML frame's cells are stored after their base update; their
// corrections, sources and receivers follow in k3p_fwd_e (no R^n kept).
// ---------------------------------------------------------------------------
template <typename T, int R, bool EQ, int CPM>
__global__ void __launch_bounds__(32 * K3_WARPS, k3_min_blocks<T, R>()) k3v_fwd_e(TiledFwd<T> P, K3Buf<T> f, K3Geom kg) {
  constexpr int ZLO = -R, ZHI = R, NZN = ZHI - ZLO + 1;   // z neighbours of the pair, dback
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const K3Pos wp = k3_pos(kg, g);
  if (!wp.live) return;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const int PS = NY * zp;
  const long long sbase = (long long)s * NX * PS;
  T* __restrict__ Ex = f.Ex + sbase;
  T* __restrict__ Ey = f.Ey + sbase;
  T* __restrict__ Ez = f.Ez + sbase;
  const T* __restrict__ Hx = f.Hx + sbase;
  const T* __restrict__ Hy = f.Hy + sbase;
  const T* __restrict__ Hz = f.Hz + sbase;
  const bool pml = CPM != kCpmPass && a.has_cpml;   // CPML handled in this kernel
  const int hk = k3_halo<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;
  const int hrow = j * zp + (hok ? hk : 0);
  bool kv[2], exz[2], ezz[2], kl[2], zfin[2];
  int qz0[2], qz1[2], kof[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = kk + e;
    kv[e] = k < NZ;
    kof[e] = k;
    exz[e] = k > 0 && k < NZ - 1;   // z part of upd_ex and upd_ey
    ezz[e] = k < NZ - 1;            // z part of upd_ez
    kl[e] = kv[e] && k < NZ - 1;
    qz0[e] = (kv[e] && pml && k > 0) ? q_low_e(a.eF[4].p, k) : -1;
    qz1[e] = (kv[e] && pml && k > 0) ? q_high(a.eF[5].p, k, NZ) : -1;
    // cells of the CPML frame, finished by k3p_fwd_e (corrections, sources, receivers)
    zfin[e] = CPM == kCpmPass && (k < kg.fr.lo[2] || k >= kg.fr.hi[2]);
  }
  const bool zpml = qz0[0] >= 0 || qz1[0] >= 0 || qz0[1] >= 0 || qz1[1] >= 0;
  const bool any_zpml = __any_sync(kFullMask, zpml);
  T tz[2][R], ty[R];   // difference taps along z (per column) and y (per row)
  taps_back<T, R>(kk, NZ, tz[0]);
  taps_back<T, R>(kk + 1, NZ, tz[1]);
  taps_back<T, R>(j, NY, ty);
  const bool exy = j > 0 && j < NY - 1, eyy = j < NY - 1;   // y parts of upd_ex / upd_ez and upd_ey
  const int qy0 = (pml && j > 0) ? q_low_e(a.eF[2].p, j) : -1;
  const int qy1 = (pml && j > 0) ? q_high(a.eF[3].p, j, NY) : -1;
  const bool yfin = CPM == kCpmPass && (j < kg.fr.lo[1] || j >= kg.fr.hi[1]);
  const bool in_y = qy0 >= 0 || qy1 >= 0;
  const bool degx = NY - 1 != 1 || NZ - 1 != 1, degy = NX - 1 != 1 || NZ - 1 != 1, degz = NX - 1 != 1 || NY - 1 != 1;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save_r = a.keep_r && (it % a.S == 0);
  const int slot = it / a.S;
  const int ncomp = a.mode == 3 ? 3 : 1;
  const bool brow = j - a.box.y0 >= 0 && j - a.box.y0 < a.box.ny;
  const bool bok[2] = {kv[0] && kk - a.box.z0 >= 0 && kk - a.box.z0 < a.box.nz,
                       kv[1] && kk + 1 - a.box.z0 >= 0 && kk + 1 - a.box.z0 < a.box.nz};
  const long long bplane = (long long)a.box.ny * a.box.nz;
  const long long h0 = (long long)(j - a.box.y0) * a.box.nz + (kk - a.box.z0);
  const long long hb = slot * a.frame + s * a.box.cells();
  const bool cps = CPM == kCpmSingle && pml;
  const int fz = (qz0[0] >= 0 || qz0[1] >= 0) ? 4 : 5;
  int zq[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) zq[e] = fz == 4 ? qz0[e] : qz1[e];
  const FaceRows<T> yr = face_rows<T, true>(a.eF[2], a.eF[3], qy0 >= 0, g, 1, s, 0, qy0 >= 0 ? qy0 : qy1);
  const FaceRows<T> zr = face_rows<T, true>(a.eF[4], a.eF[5], fz == 4, g, 2, s, j, 0);
  Prof<T> pz[2];   // CPML profile of the lane's z-face cells (fixed along x)
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    pz[e] = Prof<T>{T(0), T(0), T(0), T(0)};
    if (cps && zq[e] >= 0) pz[e] = fz == 4 ? prof(a.eF[4], zq[e]) : prof(a.eF[5], zq[e]);
  }
  __shared__ T stg[K3_WARPS][2][kStageSlots][2][32];
  T(*const sg)[kStageSlots][2][32] = stg[threadIdx.y];
  const bool onk[2] = {kl[0], kl[1]}, jl = j < NY - 1;
  // issues the CPML operands and the curl-rhs coefficient of plane i into stage b
  auto stage = [&](int i, int b) {
    long long bx1 = 0, bx2 = 0;
    int fx = -1;
    if (cps && i > 0 && (q_low_e(a.eF[0].p, i) >= 0 || q_high(a.eF[1].p, i, NX) >= 0))
      fx = xface_at<T, true>(a.eF, g, s, i, j, bx1, bx2);
    if (save_r || (cps && (fx >= 0 || in_y || any_zpml))) {
      const bool il = i < NX - 1;
      const T* X1 = fx == 0 ? a.eF[0].psi1 : a.eF[1].psi1;
      const T* X2 = fx == 0 ? a.eF[0].psi2 : a.eF[1].psi2;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const bool zon = cps && zq[e] >= 0;
        if (kv[e] && (save_r || fx >= 0 || (cps && in_y) || zon))
          cp_async(&sg[b][6][e][lane], f.ce_rhs + i * PS + row + e);
        if (!cps) continue;
        if (fx >= 0 && kv[e] && jl) cp_async(&sg[b][0][e][lane], X1 + bx1 + kof[e]);
        if (fx >= 0 && onk[e]) cp_async(&sg[b][1][e][lane], X2 + bx2 + kof[e]);
        if (in_y && kv[e] && il) cp_async(&sg[b][2][e][lane], yr.p1 + (long long)i * yr.s1 + kof[e]);
        if (in_y && onk[e]) cp_async(&sg[b][3][e][lane], yr.p2 + (long long)i * yr.s2 + kof[e]);
        if (zon && il) cp_async(&sg[b][4][e][lane], zr.p1 + (long long)i * zr.s1 + zq[e]);
        if (zon && jl) cp_async(&sg[b][5][e][lane], zr.p2 + (long long)i * zr.s2 + zq[e]);
      }
    }
    cp_async_commit();
  };
  T qHy[2 * R][2], qHz[2 * R][2];   // Hy, Hz at planes i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = wp.x0 - R + m;
    if (pl >= 0 && pl < NX) {
      ld2(Hy + pl * PS + row, qHy[m]);
      ld2(Hz + pl * PS + row, qHz[m]);
    } else {
      qHy[m][0] = qHy[m][1] = qHz[m][0] = qHz[m][1] = T(0);
    }
  }
  T nHx[2], nHyq[2], nHzq[2], nex[2], ney[2], nez[2], nc0[2], nc1[2], nhHx = T(0), nhHy = T(0);
  T nHxy[2 * R][2], nHzy[2 * R][2];   // Hx, Hz at rows j + d, d = -R .. R-1 (own row slot unused)
  auto fetch = [&](int i) {
    const int o = i * PS;
    ld2(Hx + o + row, nHx);
    if (i + R - 1 < NX) {
      ld2(Hy + o + (R - 1) * PS + row, nHyq);
      ld2(Hz + o + (R - 1) * PS + row, nHzq);
    } else {
      nHyq[0] = nHyq[1] = nHzq[0] = nHzq[1] = T(0);
    }
    if (hok) {
      nhHx = Hx[o + hrow];
      nhHy = Hy[o + hrow];
    }
#pragma unroll
    for (int d = -R; d <= R - 1; ++d) {
      if (d == 0) continue;
      if (j + d >= 0 && j + d < NY) {
        ld2(Hx + o + row + d * zp, nHxy[d + R]);
        ld2(Hz + o + row + d * zp, nHzy[d + R]);
      } else {
        nHxy[d + R][0] = nHxy[d + R][1] = nHzy[d + R][0] = nHzy[d + R][1] = T(0);
      }
    }
    ld2(Ex + o + row, nex);
    ld2(Ey + o + row, ney);
    ld2(Ez + o + row, nez);
    ld2(f.ce_hist + o + row, nc0);
    ld2(f.ce_curl + o + row, nc1);
  };
  fetch(wp.x0);
  stage(wp.x0, 0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    T hxo[2], ex[2], ey[2], ez[2], c0[2], c1[2], hxy[2 * R][2], hzy[2 * R][2];
    const T hHx = nhHx, hHy = nhHy;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      hxo[e] = nHx[e];
      qHy[2 * R - 1][e] = nHyq[e];
      qHz[2 * R - 1][e] = nHzq[e];
      ex[e] = nex[e];
      ey[e] = ney[e];
      ez[e] = nez[e];
      c0[e] = nc0[e];
      c1[e] = nc1[e];
#pragma unroll
      for (int m = 0; m < 2 * R; ++m) {
        hxy[m][e] = nHxy[m][e];
        hzy[m][e] = nHzy[m][e];
      }
    }
    if (i + 1 < wp.x1) {
      fetch(i + 1);
      stage(i + 1, (i + 1 - wp.x0) & 1);
    } else {
      cp_async_commit();
    }
    const int o = i * PS;
    T zx[NZN], zy[NZN];   // Hx, Hy at columns kk + m of this plane
    znb<T, R, ZLO, ZHI>(hxo, hHx, lane, zx);
    znb<T, R, ZLO, ZHI>(qHy[R], hHy, lane, zy);
    T tx[R];
    taps_back<T, R>(i, NX, tx);
    const bool exx = i < NX - 1, eyx = i > 0 && i < NX - 1;   // x parts of upd_ex and upd_ey / upd_ez
    const int qx0 = (pml && i > 0) ? q_low_e(a.eF[0].p, i) : -1;
    const int qx1 = (pml && i > 0) ? q_high(a.eF[1].p, i, NX) : -1;
    const bool xfin = yfin || (CPM == kCpmPass && (i < kg.fr.lo[0] || i >= kg.fr.hi[0]));
    const bool in_x = qx0 >= 0 || qx1 >= 0;
    const bool pts = (kg.src_rows && kg.src_rows[(long long)s * NX + i]) ||
                     (kg.rcv_rows && kg.rcv_rows[(long long)s * NX + i]);
    T dHz_dy[2], dHx_dy[2], dHz_dx[2], dHy_dx[2], dHy_dz[2], dHx_dz[2], ox[2], oy[2], oz[2];
    bool dex[2], dey[2], dez[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const auto fzx = [&](int d) { return zx[e + d - ZLO]; };
      const auto fzy = [&](int d) { return zy[e + d - ZLO]; };
      const auto fyz = [&](int d) { return d == 0 ? qHz[R][e] : hzy[d + R][e]; };
      const auto fyx = [&](int d) { return d == 0 ? hxo[e] : hxy[d + R][e]; };
      const auto fxz = [&](int d) { return qHz[R + d][e]; };
      const auto fxy = [&](int d) { return qHy[R + d][e]; };
      dHz_dy[e] = dback_t<T, R>(fyz, ty);
      dHx_dy[e] = dback_t<T, R>(fyx, ty);
      dHz_dx[e] = dback_t<T, R>(fxz, tx);
      dHy_dx[e] = dback_t<T, R>(fxy, tx);
      dHy_dz[e] = dback_t<T, R>(fzy, tz[e]);
      dHx_dz[e] = dback_t<T, R>(fzx, tz[e]);
      dex[e] = degx && exx && exy && exz[e];
      dey[e] = degy && eyx && eyy && exz[e];
      dez[e] = degz && eyx && exy && ezz[e];
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
    bool zon[2], src_hit[2];
    int cell[2];
    T cb[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      zon[e] = qz0[e] >= 0 || qz1[e] >= 0;
      cell[e] = (i * NY + j) * NZ + kk + e;   // logical cell (point tables)
      src_hit[e] = kv[e] && !xfin && !zfin[e] && pts && point_hit(P.src, s, cell[e]);
    }
    cp_async_wait_prev();
    const int b = (i - wp.x0) & 1;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      if (kv[e] && (save_r || (cps && (in_x || in_y || zq[e] >= 0)))) cb[e] = sg[b][6][e][lane];
      else cb[e] = (kv[e] && (src_hit[e] || (!cps && (in_x || in_y || zon[e])))) ? f.ce_rhs[o + row + e] : T(0);
    }
    if (cps && (in_x || in_y || any_zpml)) {
      // staged operands of this plane; faces update in the reference order x, y, z
      const bool il = i < NX - 1;
      if (in_x) {
        long long bx1, bx2;
        const int fx = xface_at<T, true>(a.eF, g, s, i, j, bx1, bx2);
        const Prof<T> pr = fx == 0 ? prof(a.eF[0], qx0) : prof(a.eF[1], qx1);
        T* X1 = fx == 0 ? a.eF[0].psi1 : a.eF[1].psi1;
        T* X2 = fx == 0 ? a.eF[0].psi2 : a.eF[1].psi2;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (kv[e] && jl) cpml_one<T>(X1, bx1 + kof[e], sg[b][0][e][lane], pr, dHz_dx[e], a.ddx, cb[e], false, ey[e]);
          if (onk[e]) cpml_one<T>(X2, bx2 + kof[e], sg[b][1][e][lane], pr, dHy_dx[e], a.ddx, cb[e], true, ez[e]);
        }
      }
      if (in_y) {
        const Prof<T> pr = qy0 >= 0 ? prof(a.eF[2], qy0) : prof(a.eF[3], qy1);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (kv[e] && il)
            cpml_one<T>(yr.p1, (long long)i * yr.s1 + kof[e], sg[b][2][e][lane], pr, dHz_dy[e], a.ddy, cb[e], true,
                        ex[e]);
          if (onk[e])
            cpml_one<T>(yr.p2, (long long)i * yr.s2 + kof[e], sg[b][3][e][lane], pr, dHx_dy[e], a.ddy, cb[e], false,
                        ez[e]);
        }
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (zq[e] < 0) continue;
        const Prof<T>& pr = pz[e];
        if (il)
          cpml_one<T>(zr.p1, (long long)i * zr.s1 + zq[e], sg[b][4][e][lane], pr, dHy_dz[e], a.ddz, cb[e], false,
                      ex[e]);
        if (jl)
          cpml_one<T>(zr.p2, (long long)i * zr.s2 + zq[e], sg[b][5][e][lane], pr, dHx_dz[e], a.ddz, cb[e], true,
                      ey[e]);
      }
    } else if (CPM == kCpmGeneral && (in_x || in_y || any_zpml)) {
      // faces of one axis meet: the general per-face form
      const bool jl = j < NY - 1, il = i < NX - 1;
      const bool onk[2] = {kl[0], kl[1]}, onj[2] = {kv[0] && jl, kv[1] && jl}, oni[2] = {kv[0] && il, kv[1] && il};
#pragma unroll
      for (int fc = 0; fc < 2; ++fc) {
        const int q = fc == 0 ? qx0 : qx1;
        if (q < 0) continue;
        const Face<T>& F = a.eF[fc];
        const Prof<T> pr = prof(F, q);
        cpml_pair<T>(F.psi1, psi_index(psi_dims_e(g, 0, 1, F.p), 0, s, q, i, j, 0), kof, onj, pr, dHz_dx, a.ddx, cb,
                     T(-1), ey);
        cpml_pair<T>(F.psi2, psi_index(psi_dims_e(g, 0, 2, F.p), 0, s, q, i, j, 0), kof, onk, pr, dHy_dx, a.ddx, cb,
                     T(1), ez);
      }
#pragma unroll
      for (int fc = 2; fc < 4; ++fc) {
        const int q = fc == 2 ? qy0 : qy1;
        if (q < 0) continue;
        const Face<T>& F = a.eF[fc];
        const Prof<T> pr = prof(F, q);
        cpml_pair<T>(F.psi1, psi_index(psi_dims_e(g, 1, 1, F.p), 1, s, q, i, j, 0), kof, oni, pr, dHz_dy, a.ddy, cb,
                     T(1), ex);
        cpml_pair<T>(F.psi2, psi_index(psi_dims_e(g, 1, 2, F.p), 1, s, q, i, j, 0), kof, onk, pr, dHx_dy, a.ddy, cb,
                     T(-1), ez);
      }
      if (any_zpml) {
#pragma unroll
        for (int fc = 4; fc < 6; ++fc) {
          const Face<T>& F = a.eF[fc];
          int qq[2];
          bool o1[2], o2[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            qq[e] = fc == 4 ? qz0[e] : qz1[e];
            o1[e] = qq[e] >= 0 && il;
            o2[e] = qq[e] >= 0 && jl;
          }
          if (!(o1[0] || o1[1] || o2[0] || o2[1])) continue;
          Prof<T> pr[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) pr[e] = prof(F, qq[e] >= 0 ? qq[e] : 0);
          const long long b1 = psi_index(psi_dims_e(g, 2, 1, F.p), 2, s, 0, i, j, 0);
          const long long b2 = psi_index(psi_dims_e(g, 2, 2, F.p), 2, s, 0, i, j, 0);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (o1[e]) {
              const T d = div_fixed(dHy_dz[e], a.ddz), ph = F.psi1[b1 + qq[e]];
              ex[e] -= cb[e] * (pr[e].ra1 * d + pr[e].rb * ph);
              F.psi1[b1 + qq[e]] = pr[e].re * ph - pr[e].rf * d;
            }
            if (o2[e]) {
              const T d = div_fixed(dHx_dz[e], a.ddz), ph = F.psi2[b2 + qq[e]];
              ey[e] += cb[e] * (pr[e].ra1 * d + pr[e].rb * ph);
              F.psi2[b2 + qq[e]] = pr[e].re * ph - pr[e].rf * d;
            }
          }
        }
      }
    }
    if (pts) {
#pragma unroll
      for (int e = 0; e < 2; ++e)
        if (src_hit[e]) inject_at(P, s, cell[e], it, cb[e], ex[e], ey[e], ez[e]);
    }
    if (save_r) {
      const int bi = i - a.box.x0;
      const bool rin = brow && bi >= 0 && bi < a.box.nx;
      const bool ib[2] = {rin && bok[0], rin && bok[1]};
      const long long hoff = hb + (long long)bi * bplane + h0;
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
            rv[e] = T(0);
            if (ib[e]) {
              // R^n = (E^{n+1} - a_eff E^n) / cb (deepgpr_cpu.c:1850-1875)
              const T en = fc == 0 ? ex[e] : (fc == 1 ? ey[e] : ez[e]);
              const T eo = fc == 0 ? ox[e] : (fc == 1 ? oy[e] : oz[e]);
              const bool du = fc == 0 ? dex[e] : (fc == 1 ? dey[e] : dez[e]);
              const T aeff = du ? c0[e] : T(1);
              rv[e] = cb[e] != T(0) ? (en - aeff * eo) / cb[e] : T(0);
              am = fmaxf(am, fabsf(float(rv[e])));
            }
          }
          float inv = 1.0f;
          if (is_tiled(KIND)) {
            const float sc = tile_scale_of(KIND, half_absmax(am));
            inv = 1.0f / sc;
            if ((lane & 15) == 0 && kk < NZ)
              a.r_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j, kk)] = sc;
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
        if (kv[e] && !xfin && !zfin[e]) sample_at(P, s, cell[e], it, ex[e], ey[e], ez[e]);
    }
    if (kv[1]) {
      st2(Ex + o + row, ex);
      st2(Ey + o + row, ey);
      st2(Ez + o + row, ez);
    } else if (kv[0]) {
      Ex[o + row] = ex[0];
      Ey[o + row] = ey[0];
      Ez[o + row] = ez[0];
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        qHy[m][e] = qHy[m + 1][e];
        qHz[m][e] = qHz[m + 1][e];
      }
  }
}

// ---------------------------------------------------------------------------
// H z-face CPML corrections (single-face form) in their own pass after
// k3v_fwd_h, which then skips them: only a few lanes of a z-streamed warp lie
// in a z face.  The z faces are the last correction of a cell in the
// reference order (x, y, z; deepgpr_cpu.c:980-1097) and E is not written
// during the H half step, so correcting the stored H here with the same
// derivative (same taps, same order) gives the same values.
// Block (32, kZfRowsF): x strides over the candidate z columns of a row (the
// low face's p, then the high face's p + 1), y = row within the block; grid
// (NX * ceil(NY / kZfRowsF), nshot).
// ---------------------------------------------------------------------------
constexpr int kZfRowsF = 8;
// Resident CTAs per SM of the forward CPML passes (k3z_fwd_h, k3p_fwd_e):
// latency-bound per-cell work, so residency counts more than registers
// (8: 32 registers a thread; measured on 320 x 320 x 160 + CPML 10 the E
// half step 7 % and the H half step 3 % faster than at 44-47 registers).
constexpr int kPassMinBlocks = 8;

template <typename T, int R>
__global__ void __launch_bounds__(32 * kZfRowsF, kPassMinBlocks) k3z_fwd_h(TiledFwd<T> P, K3Buf<T> f, K3Geom kg, int nyb) {
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ;
  const int p4 = a.hF[4].p, p5 = a.hF[5].p, nlo = p4, nk = nlo + p5 + 1;
  const int i = blockIdx.x / nyb;
  const int j = (blockIdx.x - i * nyb) * kZfRowsF + threadIdx.y;
  if (j >= NY) return;
  const int s = blockIdx.y, zp = kg.zp, PS = NY * zp;
  const long long rbase = (long long)s * NX * PS + (long long)i * PS + j * zp;   // (s, i, j, 0)
  const T* __restrict__ ex = f.Ex + rbase;
  const T* __restrict__ ey = f.Ey + rbase;
  for (int kc = threadIdx.x; kc < nk; kc += 32) {
    const int k = kc < nlo ? kc : NZ - 1 - p5 + (kc - nlo);
    const int q0 = q_low_h(p4, k), q1 = q_high(p5, k, NZ);
    if (q0 < 0 && q1 < 0) continue;
    const bool lo = q0 >= 0;
    const int q = lo ? q0 : q1;
    const Face<T>& F = lo ? a.hF[4] : a.hF[5];
    const Prof<T> pr = prof(F, q);
    T tz[R];
    taps_fwd<T, R>(k, NZ, tz);
    // columns outside the axis only meet zero taps
    const auto at = [&](const T* v, int d) { return (k + d >= 0 && k + d < NZ) ? v[k + d] : T(0); };
    const T up = f.ch_rhs[(long long)i * PS + j * zp + k];
    if (j < NY - 1) {
      const T d = dfwd_t<T, R>([&](int dd) { return at(ey, dd); }, tz);
      const long long pi = psi_index(psi_dims_h(g, 2, 1, F.p), 2, s, q, i, j, 0);
      T h = f.Hx[rbase + k];
      cpml_one<T>(F.psi1, pi, F.psi1[pi], pr, d, a.ddz, up, true, h);
      f.Hx[rbase + k] = h;
    }
    if (i < NX - 1) {
      const T d = dfwd_t<T, R>([&](int dd) { return at(ex, dd); }, tz);
      const long long pi = psi_index(psi_dims_h(g, 2, 2, F.p), 2, s, q, i, j, 0);
      T h = f.Hy[rbase + k];
      cpml_one<T>(F.psi2, pi, F.psi2[pi], pr, d, a.ddz, up, false, h);
      f.Hy[rbase + k] = h;
    }
  }
}

// ---------------------------------------------------------------------------
// CPML frame pass of the E half step's kCpmPass form, one thread per frame
// cell, launched on the same stream right after the streamed kernel, which
// stored every cell's base update.  A cell's CPML corrections come after its base update
// in the reference order (faces x0 xm y0 ym z0 zm, deepgpr_cpu.c:765-880,
// 980-1097), and the field the derivatives read is not written during the
// half step, so correcting the stored value here with the same derivatives
// (d_fwd / d_back: the streamed kernels' tap tables without their zero taps)
// gives the same values.  The pass then applies the cell's sources and
// receivers (deepgpr_cpu.c:655-666, 600-623); it runs only when no R^n history
// is kept (R^n needs E^n, which the streamed kernel has overwritten).  Only
// the lanes in a face need this work (in an edge z strip 5 of 32), so the
// streamed kernel carries none of it.  (For the H half step the same pass
// measured slower than the streamed kernel's own x and y corrections; there
// only the z faces move out, to k3z_fwd_h.)
// ---------------------------------------------------------------------------

// (i, j, k) of frame cell t of one shot, or false past the last one
__device__ __forceinline__ bool k3_frame_cell(const K3Frame& fr, unsigned t, int& i, int& j, int& k) {
  if (t >= fr.cum[5]) return false;
  int b = 0;
#pragma unroll
  for (int q = 0; q < 5; ++q) b += t >= fr.cum[q];
  const unsigned loc = t - (b > 0 ? fr.cum[b - 1] : 0u);
  const unsigned nz = (unsigned)fr.n[b][2], ny = (unsigned)fr.n[b][1];
  const unsigned rest = loc / nz, ri = rest / ny;
  k = fr.o[b][2] + int(loc - rest * nz);
  j = fr.o[b][1] + int(rest - ri * ny);
  i = fr.o[b][0] + int(ri);
  return true;
}

template <typename T, int R>
__global__ void __launch_bounds__(kBlock, kPassMinBlocks) k3p_fwd_e(TiledFwd<T> P, K3Buf<T> f, K3Geom kg) {
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  int i, j, k;
  if (!k3_frame_cell(kg.fr, blockIdx.x * kBlock + threadIdx.x, i, j, k)) return;
  const int s = blockIdx.y, zp = kg.zp, PS = g.NY * zp;
  const int it = a.ctrl->cur + a.k_in_chunk;
  int qf[6];
  qf[0] = i > 0 ? q_low_e(a.eF[0].p, i) : -1;
  qf[1] = i > 0 ? q_high(a.eF[1].p, i, g.NX) : -1;
  qf[2] = j > 0 ? q_low_e(a.eF[2].p, j) : -1;
  qf[3] = j > 0 ? q_high(a.eF[3].p, j, g.NY) : -1;
  qf[4] = k > 0 ? q_low_e(a.eF[4].p, k) : -1;
  qf[5] = k > 0 ? q_high(a.eF[5].p, k, g.NZ) : -1;
  const bool any_pml = qf[0] >= 0 || qf[1] >= 0 || qf[2] >= 0 || qf[3] >= 0 || qf[4] >= 0 || qf[5] >= 0;
  // the plane's point flags are loaded here and read after the corrections:
  // a CPML cell (nearly every frame cell) does not wait for them
  const unsigned char fsrc = kg.src_rows ? kg.src_rows[(long long)s * g.NX + i] : (unsigned char)0;
  const unsigned char frcv = kg.rcv_rows ? kg.rcv_rows[(long long)s * g.NX + i] : (unsigned char)0;
  if (!any_pml && (fsrc | frcv) == 0) return;
  const bool pts = (fsrc | frcv) != 0;
  const int cc = i * PS + j * zp + k;
  const long long base = (long long)s * g.NX * PS + cc;
  const T cb = f.ce_rhs[cc];
  const T* hx = f.Hx + base;
  const T* hy = f.Hy + base;
  const T* hz = f.Hz + base;
  T ex = f.Ex[base], ey = f.Ey[base], ez = f.Ez[base];
#pragma unroll
  for (int fc = 0; fc < 6; ++fc) {
    const int q = qf[fc];
    if (q < 0) continue;
    const Face<T>& F = a.eF[fc];
    const Prof<T> pr = prof(F, q);
    const int axis = fc >> 1;
    // psi slot 1 or 2 of this face: u +-= cb (ra1 d + rb psi), d = dv / h
    auto corr = [&](int slot, T dv, const FixedDiv<T>& hd, bool plus, T& u) {
      T* psi = slot == 1 ? F.psi1 : F.psi2;
      const long long pi = psi_index(psi_dims_e(g, axis, slot, F.p), axis, s, q, i, j, k);
      cpml_one<T>(psi, pi, psi[pi], pr, dv, hd, cb, plus, u);
    };
    if (axis == 0) {
      if (j < g.NY - 1) corr(1, d_back<T, R>(hz, PS, i, g.NX), a.ddx, false, ey);
      if (k < g.NZ - 1) corr(2, d_back<T, R>(hy, PS, i, g.NX), a.ddx, true, ez);
    } else if (axis == 1) {
      if (i < g.NX - 1) corr(1, d_back<T, R>(hz, zp, j, g.NY), a.ddy, true, ex);
      if (k < g.NZ - 1) corr(2, d_back<T, R>(hx, zp, j, g.NY), a.ddy, false, ez);
    } else {
      if (i < g.NX - 1) corr(1, d_back<T, R>(hy, 1, k, g.NZ), a.ddz, false, ex);
      if (j < g.NY - 1) corr(2, d_back<T, R>(hx, 1, k, g.NZ), a.ddz, true, ey);
    }
  }
  if (pts) {
    const int cell = (i * g.NY + j) * g.NZ + k;   // logical cell (point tables)
    inject_at(P, s, cell, it, cb, ex, ey, ez);
    sample_at(P, s, cell, it, ex, ey, ez);
  }
  f.Ex[base] = ex;
  f.Ey[base] = ey;
  f.Ez[base] = ez;
}

}  // namespace dg
