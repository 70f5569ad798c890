// fdtd_3d_wide_adj.cuh -- FP32 3D adjoint steps on 128-column warp strips.
//
// The adjoint E and H steps of fdtd_3d_adj.cuh (z-streamed, two columns per
// lane) in the layout of the wide forward kernels (fdtd_3d_wide.cuh): a warp
// owns 128 z columns of one (shot, y row), four per lane, and streams x
// planes; the plane's own rows and the entering x plane are staged into
// shared memory one plane ahead (cp.async, zero fill outside the grid); the
// neighbour rows of the y channels are loaded at the top of the plane; the
// z-face CPML weights of the lane's columns and of its halo column are
// prefetched one plane ahead into registers, the x- and y-face weights are
// read where they are used (planes and rows of a face, uniform over the
// warp).  Channels, gathers (per-target tap tables) and their order are those
// of the z-streamed kernels, which follow the reference
// (src/DeepGPR/lib/deepgpr_cpu.c:1112-1459, 1479-1534), so the results are
// the same bit for bit.  With one CPML face per axis (k3_cpml_single) the
// step's own CPML weights are formed by k3p_adj_w after each kernel, as for
// the z-streamed kernels.
#pragma once

#include "fdtd_3d_adj.cuh"
#include "fdtd_3d_wide.cuh"

namespace dg {

// Staged rows of one plane: the cell's own lambda_E, lambda_H and
// coefficients, then the entering x plane's two lambda components and curl
// coefficient (x channels).
constexpr int KWA_SLOTS = 11;
constexpr int kw_adj_smem_bytes() { return KW_WARPS * 2 * KWA_SLOTS * 32 * 16; }
constexpr int KWA_MIN_BLOCKS = 3;

// Face position along an axis for the E (EF) or H faces: q and whether it is
// the low face; -1 outside both.
template <bool EF>
__device__ __forceinline__ int kwa_face(const Face<float>* F, int axis, int c, int n, bool& lo) {
  int q0, q1;
  face_q<EF>(F[2 * axis].p, F[2 * axis + 1].p, c, n, q0, q1);
  lo = q0 >= 0;
  return q0 >= 0 ? q0 : q1;
}

// ---------------------------------------------------------------------------
// Adjoint E step (channels of the E sources gathered into lambda_H), as
// k3v_adj_e:   A_X = x w1 + (-c) lambda_ey,  A_Y = y w1 + c_y lambda_ex  -> lambda_hz
//              B_X = x w2 + c lambda_ez,     B_Z = z w1 + (-c_z) lambda_ex -> lambda_hy
//              C_Y = y w2 + (-c_y) lambda_ez, C_Z = z w2 + c_z lambda_ey  -> lambda_hx
// ---------------------------------------------------------------------------
template <int R, bool EQ>
__global__ void __launch_bounds__(32 * KW_WARPS, KWA_MIN_BLOCKS)
    k3w_adj_e(const __grid_constant__ TiledAdj<float> P, K3Buf<float> f, K3WGeom kg) {
  using T = float;
  constexpr int ZLO = -(R - 1), ZHI = R + 3, NZN = ZHI - ZLO + 1;   // z sources of the quadruple, gather_back
  constexpr int SEX = 0, SEY = 1, SEZ = 2, SC = 3, SHX = 4, SHY = 5, SHZ = 6, SLY = 7, SLZ = 8, SLC = 9;
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const int it = a.ctrl->cur - a.k_in_chunk;
  if (a.want_src && blockIdx.x == 0 && threadIdx.y == 0) {
    // waveform gradient of step it: shots summed in order (deepgpr_cpu.c:1524-1533)
    for (int m = threadIdx.x; m < a.nsrc; m += 32) {
      T acc = a.grad_source[(long long)m * a.nt + it];
      for (int s = 0; s < g.nshot; ++s) acc += a.srcv[(long long)s * a.nsrc + m];
      a.grad_source[(long long)m * a.nt + it] = acc;
    }
  }
  const KwPos wp = kw_pos(kg, g);
  if (!wp.live) return;
  extern __shared__ float4 kw_smem[];
  float4* const sb = kw_smem + threadIdx.y * 2 * KWA_SLOTS * 32 + threadIdx.x;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const bool lv = wp.lv;
  const int PS = NY * zp;
  const int hk = halo_col4<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;
  const long long srow = (long long)s * NX * PS + j * zp;
  const long long rb = srow + kk, rs = lv ? rb : srow;
  const int rowc = lv ? row : j * zp;
  const long long hrb = srow + (hok ? hk : 0);
  const int hrc = j * zp + (hok ? hk : 0);
  const bool pml = a.has_cpml != 0;
  const bool dxo = NY - 1 != 1 || NZ - 1 != 1, dyo = NX - 1 != 1 || NZ - 1 != 1, dzo = NX - 1 != 1 || NY - 1 != 1;
  const bool jm = j > 0 && j < NY - 1, jl = j < NY - 1;
  bool kv[4], km[4], kl[4];
  T zup[4][R], zdn[4][R], yup[R], ydn[R];
  int ezq[4];   // E z-face position of the lane's cells (-1: none)
  bool ezlo[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kk + e;
    kv[e] = k < NZ;
    km[e] = k > 0 && k < NZ - 1;
    kl[e] = k < NZ - 1;
    gtaps_back<T, R>(k, NZ, zup[e], zdn[e]);
    ezq[e] = (pml && kv[e]) ? kwa_face<true>(a.eF, 2, k, NZ, ezlo[e]) : -1;
  }
  gtaps_back<T, R>(j, NY, yup, ydn);
  bool ehlo = true;
  const int ehq = (pml && hok) ? kwa_face<true>(a.eF, 2, hk, NZ, ehlo) : -1;
  const bool hkm = hok && hk > 0 && hk < NZ - 1;
  const bool any_ez = __any_sync(kFullMask, ezq[0] >= 0 || ezq[1] >= 0 || ezq[2] >= 0 || ezq[3] >= 0 || ehq >= 0);
  unsigned ymask = 0;   // E y faces of the neighbour rows j + d (bit d + R - 1)
  if (pml) {
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) {
      bool lo;
      const int y = j + d;
      if (y >= 0 && y < NY && kwa_face<true>(a.eF, 1, y, NY, lo) >= 0) ymask |= 1u << (d + R - 1);
    }
  }
  // z-face weight of the lane's cell e (slot 1 or 2) at plane i
  auto zw = [&](int slot, int e, int i) -> T {
    const Face<T>& F = ezlo[e] ? a.eF[4] : a.eF[5];
    const T* W = slot == 1 ? F.w1 : F.w2;
    return W[cpml_at32<true>(g, 2, slot, F.p, s, ezq[e], i, j, kk + e)];
  };
  auto hzw = [&](int slot, int i) -> T {
    const Face<T>& F = ehlo ? a.eF[4] : a.eF[5];
    const T* W = slot == 1 ? F.w1 : F.w2;
    return W[cpml_at32<true>(g, 2, slot, F.p, s, ehq, i, j, hk)];
  };
  // x channels of plane x from its lambda_ey, lambda_ez, c
  auto xchan = [&](int x, const T (&ly)[4], const T (&lz)[4], const T (&c)[4], T (&A)[4], T (&B)[4]) {
    const bool xm = x > 0 && x < NX - 1;
    bool lo = true;
    const int qx = (pml && x >= 0 && x < NX) ? kwa_face<true>(a.eF, 0, x, NX, lo) : -1;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      T wa = T(0), wb = T(0);
      if (qx >= 0) {
        const Face<T>& F = lo ? a.eF[0] : a.eF[1];
        if (jl && kv[e]) wa += F.w1[cpml_at32<true>(g, 0, 1, F.p, s, qx, x, j, kk + e)];
        if (kl[e]) wb += F.w2[cpml_at32<true>(g, 0, 2, F.p, s, qx, x, j, kk + e)];
      }
      if (dyo && xm && jl && km[e]) wa += (-c[e]) * ly[e];
      if (dzo && xm && jm && kl[e]) wb += c[e] * lz[e];
      A[e] = wa;
      B[e] = wb;
    }
  };
  const int x0 = wp.x0;
  T qA[2 * R][4], qB[2 * R][4];   // A_X, B_X at planes i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = x0 - R + 1 + m;
    const bool in = pl >= 0 && pl < NX;
    T ly[4], lz[4], c[4];
    ld4m(f.Ey + rs + (in ? pl : 0) * PS, in && lv, ly);
    ld4m(f.Ez + rs + (in ? pl : 0) * PS, in && lv, lz);
    ld4m(f.ce_curl + rowc + (in ? pl : 0) * PS, in && lv, c);
    xchan(pl, ly, lz, c, qA[m], qB[m]);
  }
  T nhex = 0.0f, nhey = 0.0f, nhc = 0.0f, nzw1[4], nzw2[4], nhw1 = 0.0f, nhw2 = 0.0f;
  auto stage = [&](int i, int bf) {
    const int o = i * PS;
    float4* d = sb + bf * KWA_SLOTS * 32;
    const bool lead = i + R < NX;
    const int lo = lead ? R * PS : 0;
    cp16<true>(d + SEX * 32, f.Ex + rs + o, lv);
    cp16<true>(d + SEY * 32, f.Ey + rs + o, lv);
    cp16<true>(d + SEZ * 32, f.Ez + rs + o, lv);
    cp16<true>(d + SC * 32, f.ce_curl + rowc + o, lv);
    cp16<false>(d + SHX * 32, f.Hx + rs + o, lv);
    cp16<false>(d + SHY * 32, f.Hy + rs + o, lv);
    cp16<false>(d + SHZ * 32, f.Hz + rs + o, lv);
    cp16<true>(d + SLY * 32, f.Ey + rs + o + lo, lead && lv);
    cp16<true>(d + SLZ * 32, f.Ez + rs + o + lo, lead && lv);
    cp16<true>(d + SLC * 32, f.ce_curl + rowc + o + lo, lead && lv);
    cp_async_commit();
    if (hok) {
      nhex = f.Ex[hrb + o];
      nhey = f.Ey[hrb + o];
      nhc = f.ce_curl[hrc + o];
    }
    if (any_ez) {
      const bool il = i < NX - 1;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        nzw1[e] = (ezq[e] >= 0 && il) ? zw(1, e, i) : 0.0f;
        nzw2[e] = (ezq[e] >= 0 && jl) ? zw(2, e, i) : 0.0f;
      }
      nhw1 = (ehq >= 0 && il) ? hzw(1, i) : 0.0f;
      nhw2 = (ehq >= 0 && jl) ? hzw(2, i) : 0.0f;
    }
  };
  stage(x0, 0);
  for (int i = x0; i < wp.x1; ++i) {
    const T hex = nhex, hey = nhey, hc = nhc, hw1 = nhw1, hw2 = nhw2;
    T zw1[4], zw2[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      zw1[e] = nzw1[e];
      zw2[e] = nzw2[e];
    }
    const int bf = (i - x0) & 1;
    if (i + 1 < wp.x1) stage(i + 1, bf ^ 1);
    else cp_async_commit();
    const int o = i * PS;
    // neighbour rows of the y channels (lambda_ex, lambda_ez, c of rows j + d)
    T nx_[2 * R][4], nz_[2 * R][4], nc_[2 * R][4];
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) {
      if (d == 0) continue;
      const bool in = j + d >= 0 && j + d < NY;
      const int m = d + R - 1;
      ld4m(f.Ex + rs + o + (in ? d * zp : 0), in && lv, nx_[m]);
      ld4m(f.Ez + rs + o + (in ? d * zp : 0), in && lv, nz_[m]);
      ld4m(f.ce_curl + rowc + o + (in ? d * zp : 0), in && lv, nc_[m]);
    }
    cp_async_wait_prev();
    const float4* cur = sb + bf * KWA_SLOTS * 32;
    const bool il = i < NX - 1, im = i > 0 && i < NX - 1;
    {
      T ly[4], lz[4], c[4];
      from4(cur[SLY * 32], ly);
      from4(cur[SLZ * 32], lz);
      from4(cur[SLC * 32], c);
      xchan(i + R, ly, lz, c, qA[2 * R - 1], qB[2 * R - 1]);
    }
    T ex[4], ey[4], ez[4], c[4];
    from4(cur[SEX * 32], ex);
    from4(cur[SEY * 32], ey);
    from4(cur[SEZ * 32], ez);
    from4(cur[SC * 32], c);
    // z channels of the lane's columns and of the halo column
    T bz[4], cz[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      T w1 = T(0), w2 = T(0);
      if (ezq[e] >= 0 && il) w1 += zw1[e];
      if (ezq[e] >= 0 && jl) w2 += zw2[e];
      const T cze = curl_z<EQ>(a, c[e]);
      if (dxo && il && jm && km[e]) w1 += (-cze) * ex[e];
      if (dyo && im && jl && km[e]) w2 += cze * ey[e];
      bz[e] = w1;
      cz[e] = w2;
    }
    T hbz = T(0), hcz = T(0);
    if (hok) {
      if (ehq >= 0 && il) hbz += hw1;
      if (ehq >= 0 && jl) hcz += hw2;
      const T czh = curl_z<EQ>(a, hc);
      if (dxo && il && jm && hkm) hbz += (-czh) * hex;
      if (dyo && im && jl && hkm) hcz += czh * hey;
    }
    // y channels of rows j + d (own row from the stage)
    T ay[2 * R][4], cy[2 * R][4];
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) {
      const int y = j + d;
      const int m = d + R - 1;
      const bool ym = y > 0 && y < NY - 1;
      const bool yf = (ymask >> m) & 1u;
      bool ylo = true;
      const int qy = yf ? kwa_face<true>(a.eF, 1, y, NY, ylo) : -1;
      const Face<T>& FY = ylo ? a.eF[2] : a.eF[3];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const T lx = d == 0 ? ex[e] : nx_[m][e];
        const T lz = d == 0 ? ez[e] : nz_[m][e];
        const T cv = d == 0 ? c[e] : nc_[m][e];
        T w1 = T(0), w2 = T(0);
        if (yf) {
          if (il && kv[e]) w1 += FY.w1[cpml_at32<true>(g, 1, 1, FY.p, s, qy, i, y, kk + e)];
          if (kl[e]) w2 += FY.w2[cpml_at32<true>(g, 1, 2, FY.p, s, qy, i, y, kk + e)];
        }
        const T cye = curl_y<EQ>(a, cv);
        if (dxo && il && ym && km[e]) w1 += cye * lx;
        if (dzo && im && ym && kl[e]) w2 += (-cye) * lz;
        ay[m][e] = w1;
        cy[m][e] = w2;
      }
    }
    T zb[NZN], zc[NZN];
#pragma unroll
    for (int m = ZLO; m <= ZHI; ++m) {
      zb[m - ZLO] = ynb4<T, R>(bz, hbz, lane, m);
      zc[m - ZLO] = ynb4<T, R>(cz, hcz, lane, m);
    }
    // gathers, in the reference order
    T xup[R], xdn[R];
    xtaps<T, R, true>(i, NX, xup, xdn);
    T hx[4], hy[4], hz[4];
    from4(cur[SHX * 32], hx);
    from4(cur[SHY * 32], hy);
    from4(cur[SHZ * 32], hz);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      hz[e] += gback_t<T, R>([&](int d) { return qA[R - 1 + d][e]; }, xup, xdn);
      hz[e] += gback_t<T, R>([&](int d) { return ay[d + R - 1][e]; }, yup, ydn);
      hy[e] += gback_t<T, R>([&](int d) { return qB[R - 1 + d][e]; }, xup, xdn);
      hy[e] += gback_t<T, R>([&](int d) { return zb[e + d - ZLO]; }, zup[e], zdn[e]);
      hx[e] += gback_t<T, R>([&](int d) { return cy[d + R - 1][e]; }, yup, ydn);
      hx[e] += gback_t<T, R>([&](int d) { return zc[e + d - ZLO]; }, zup[e], zdn[e]);
    }
    if (lv) {
      st4(f.Hx + rb + o, hx);
      st4(f.Hy + rb + o, hy);
      st4(f.Hz + rb + o, hz);
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        qA[m][e] = qA[m + 1][e];
        qB[m][e] = qB[m + 1][e];
      }
  }
}

// ---------------------------------------------------------------------------
// Adjoint H step (channels of the H sources gathered into lambda_E, after the
// ce_hist scaling), then the head of step it-1 (receiver cotangents, staged
// source terms), as k3v_adj_h:
//   A_X = x w1 + c lambda_hy,      A_Y = y w1 + (-c_y) lambda_hx -> lambda_ez
//   B_X = x w2 + (-c) lambda_hz,   B_Z = z w1 + c_z lambda_hx    -> lambda_ey
//   C_Y = y w2 + c_y lambda_hz,    C_Z = z w2 + (-c_z) lambda_hy -> lambda_ex
// ---------------------------------------------------------------------------
template <int R, bool EQ>
__global__ void __launch_bounds__(32 * KW_WARPS, KWA_MIN_BLOCKS)
    k3w_adj_h(const __grid_constant__ TiledAdj<float> P, K3Buf<float> f, K3WGeom kg) {
  using T = float;
  constexpr int ZLO = -R, ZHI = R + 2, NZN = ZHI - ZLO + 1;   // z sources of the quadruple, gather_fwd
  constexpr int SHX = 0, SHY = 1, SHZ = 2, SC = 3, SEX = 4, SEY = 5, SEZ = 6, SCA = 7, SLY = 8, SLZ = 9, SLC = 10;
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const KwPos wp = kw_pos(kg, g);
  if (!wp.live) return;
  extern __shared__ float4 kw_smem[];
  float4* const sb = kw_smem + threadIdx.y * 2 * KWA_SLOTS * 32 + threadIdx.x;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const bool lv = wp.lv;
  const int PS = NY * zp;
  const int it = a.ctrl->cur - a.k_in_chunk;
  const int head = it - 1;
  const int hk = halo_col4<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;
  const long long srow = (long long)s * NX * PS + j * zp;
  const long long rb = srow + kk, rs = lv ? rb : srow;
  const int rowc = lv ? row : j * zp;
  const long long hrb = srow + (hok ? hk : 0);
  const int hrc = j * zp + (hok ? hk : 0);
  const bool pml = a.has_cpml != 0;
  // parts of upd_h*: hx: NX-1 != 1, mid(i), lo(j), lo(k); hy: NY-1 != 1, lo(i),
  // mid(j), lo(k); hz: NZ-1 != 1, lo(i), lo(j), mid(k); and of upd_e* for ce_hist
  const bool hxo = NX - 1 != 1, hyo = NY - 1 != 1, hzo = NZ - 1 != 1;
  const bool dxo = NY - 1 != 1 || NZ - 1 != 1, dyo = NX - 1 != 1 || NZ - 1 != 1, dzo = NX - 1 != 1 || NY - 1 != 1;
  const bool jm = j > 0 && j < NY - 1, jl = j < NY - 1;
  bool kv[4], km[4], kl[4];
  T zup[4][R], zdn[4][R], yup[R], ydn[R];
  int hzq[4];
  bool hzlo[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kk + e;
    kv[e] = k < NZ;
    km[e] = k > 0 && k < NZ - 1;
    kl[e] = k < NZ - 1;
    gtaps_fwd<T, R>(k, NZ, zup[e], zdn[e]);
    hzq[e] = (pml && kv[e]) ? kwa_face<false>(a.hF, 2, k, NZ, hzlo[e]) : -1;
  }
  gtaps_fwd<T, R>(j, NY, yup, ydn);
  bool hhlo = true;
  const int hhq = (pml && hok) ? kwa_face<false>(a.hF, 2, hk, NZ, hhlo) : -1;
  const bool hkl = hok && hk < NZ - 1;
  const bool any_hz = __any_sync(kFullMask, hzq[0] >= 0 || hzq[1] >= 0 || hzq[2] >= 0 || hzq[3] >= 0 || hhq >= 0);
  unsigned ymask = 0;   // H y faces of rows j + d (bit d + R)
  if (pml) {
#pragma unroll
    for (int d = -R; d <= R - 1; ++d) {
      bool lo;
      const int y = j + d;
      if (y >= 0 && y < NY && kwa_face<false>(a.hF, 1, y, NY, lo) >= 0) ymask |= 1u << (d + R);
    }
  }
  auto zw = [&](int slot, int e, int i) -> T {
    const Face<T>& F = hzlo[e] ? a.hF[4] : a.hF[5];
    const T* W = slot == 1 ? F.w1 : F.w2;
    return W[cpml_at32<false>(g, 2, slot, F.p, s, hzq[e], i, j, kk + e)];
  };
  auto hzw = [&](int slot, int i) -> T {
    const Face<T>& F = hhlo ? a.hF[4] : a.hF[5];
    const T* W = slot == 1 ? F.w1 : F.w2;
    return W[cpml_at32<false>(g, 2, slot, F.p, s, hhq, i, j, hk)];
  };
  auto xchan = [&](int x, const T (&ly)[4], const T (&lz)[4], const T (&c)[4], T (&A)[4], T (&B)[4]) {
    const bool xl = x >= 0 && x < NX - 1;
    bool lo = true;
    const int qx = (pml && x >= 0 && x < NX) ? kwa_face<false>(a.hF, 0, x, NX, lo) : -1;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      T wa = T(0), wb = T(0);
      if (qx >= 0) {
        const Face<T>& F = lo ? a.hF[0] : a.hF[1];
        if (kl[e]) wa += F.w1[cpml_at32<false>(g, 0, 1, F.p, s, qx, x, j, kk + e)];
        if (jl && kv[e]) wb += F.w2[cpml_at32<false>(g, 0, 2, F.p, s, qx, x, j, kk + e)];
      }
      if (hyo && xl && jm && kl[e]) wa += c[e] * ly[e];
      if (hzo && xl && jl && km[e]) wb += (-c[e]) * lz[e];
      A[e] = wa;
      B[e] = wb;
    }
  };
  const int x0 = wp.x0;
  T qA[2 * R][4], qB[2 * R][4];   // A_X, B_X at planes i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = x0 - R + m;
    const bool in = pl >= 0 && pl < NX;
    T ly[4], lz[4], c[4];
    ld4m(f.Hy + rs + (in ? pl : 0) * PS, in && lv, ly);
    ld4m(f.Hz + rs + (in ? pl : 0) * PS, in && lv, lz);
    ld4m(f.ch_curl + rowc + (in ? pl : 0) * PS, in && lv, c);
    xchan(pl, ly, lz, c, qA[m], qB[m]);
  }
  T nhhx = 0.0f, nhhy = 0.0f, nhc = 0.0f, nzw1[4], nzw2[4], nhw1 = 0.0f, nhw2 = 0.0f;
  auto stage = [&](int i, int bf) {
    const int o = i * PS;
    float4* d = sb + bf * KWA_SLOTS * 32;
    const bool lead = i + R - 1 < NX;
    const int lo = lead ? (R - 1) * PS : 0;
    cp16<true>(d + SHX * 32, f.Hx + rs + o, lv);
    cp16<true>(d + SHY * 32, f.Hy + rs + o, lv);
    cp16<true>(d + SHZ * 32, f.Hz + rs + o, lv);
    cp16<true>(d + SC * 32, f.ch_curl + rowc + o, lv);
    cp16<false>(d + SEX * 32, f.Ex + rs + o, lv);
    cp16<false>(d + SEY * 32, f.Ey + rs + o, lv);
    cp16<false>(d + SEZ * 32, f.Ez + rs + o, lv);
    cp16<false>(d + SCA * 32, f.ce_hist + rowc + o, lv);
    cp16<true>(d + SLY * 32, f.Hy + rs + o + lo, lead && lv);
    cp16<true>(d + SLZ * 32, f.Hz + rs + o + lo, lead && lv);
    cp16<true>(d + SLC * 32, f.ch_curl + rowc + o + lo, lead && lv);
    cp_async_commit();
    if (hok) {
      nhhx = f.Hx[hrb + o];
      nhhy = f.Hy[hrb + o];
      nhc = f.ch_curl[hrc + o];
    }
    if (any_hz) {
      const bool il = i < NX - 1;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        nzw1[e] = (hzq[e] >= 0 && jl) ? zw(1, e, i) : 0.0f;
        nzw2[e] = (hzq[e] >= 0 && il) ? zw(2, e, i) : 0.0f;
      }
      nhw1 = (hhq >= 0 && jl) ? hzw(1, i) : 0.0f;
      nhw2 = (hhq >= 0 && il) ? hzw(2, i) : 0.0f;
    }
  };
  stage(x0, 0);
  for (int i = x0; i < wp.x1; ++i) {
    const T hhx = nhhx, hhy = nhhy, hc = nhc, hw1 = nhw1, hw2 = nhw2;
    T zw1[4], zw2[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      zw1[e] = nzw1[e];
      zw2[e] = nzw2[e];
    }
    const int bf = (i - x0) & 1;
    if (i + 1 < wp.x1) stage(i + 1, bf ^ 1);
    else cp_async_commit();
    const int o = i * PS;
    // neighbour rows of the y channels (lambda_hx, lambda_hz, c of rows j + d)
    T nx_[2 * R][4], nz_[2 * R][4], nc_[2 * R][4];
#pragma unroll
    for (int d = -R; d <= R - 1; ++d) {
      if (d == 0) continue;
      const bool in = j + d >= 0 && j + d < NY;
      const int m = d + R;
      ld4m(f.Hx + rs + o + (in ? d * zp : 0), in && lv, nx_[m]);
      ld4m(f.Hz + rs + o + (in ? d * zp : 0), in && lv, nz_[m]);
      ld4m(f.ch_curl + rowc + o + (in ? d * zp : 0), in && lv, nc_[m]);
    }
    cp_async_wait_prev();
    const float4* cur = sb + bf * KWA_SLOTS * 32;
    const bool il = i < NX - 1, im = i > 0 && i < NX - 1;
    {
      T ly[4], lz[4], c[4];
      from4(cur[SLY * 32], ly);
      from4(cur[SLZ * 32], lz);
      from4(cur[SLC * 32], c);
      xchan(i + R - 1, ly, lz, c, qA[2 * R - 1], qB[2 * R - 1]);
    }
    T hx[4], hy[4], hz[4], c[4];
    from4(cur[SHX * 32], hx);
    from4(cur[SHY * 32], hy);
    from4(cur[SHZ * 32], hz);
    from4(cur[SC * 32], c);
    T bz[4], cz[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      T w1 = T(0), w2 = T(0);
      if (hzq[e] >= 0 && jl) w1 += zw1[e];
      if (hzq[e] >= 0 && il) w2 += zw2[e];
      const T cze = curl_z<EQ>(a, c[e]);
      if (hxo && im && jl && kl[e]) w1 += cze * hx[e];
      if (hyo && il && jm && kl[e]) w2 += (-cze) * hy[e];
      bz[e] = w1;
      cz[e] = w2;
    }
    T hbz = T(0), hcz = T(0);
    if (hok) {
      if (hhq >= 0 && jl) hbz += hw1;
      if (hhq >= 0 && il) hcz += hw2;
      const T czh = curl_z<EQ>(a, hc);
      if (hxo && im && jl && hkl) hbz += czh * hhx;
      if (hyo && il && jm && hkl) hcz += (-czh) * hhy;
    }
    T ay[2 * R][4], cy[2 * R][4];   // A_Y, C_Y at rows j + d, d = -R .. R-1
#pragma unroll
    for (int d = -R; d <= R - 1; ++d) {
      const int y = j + d;
      const int m = d + R;
      const bool yl = y >= 0 && y < NY - 1;
      const bool yf = (ymask >> m) & 1u;
      bool ylo = true;
      const int qy = yf ? kwa_face<false>(a.hF, 1, y, NY, ylo) : -1;
      const Face<T>& FY = ylo ? a.hF[2] : a.hF[3];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const T lx = d == 0 ? hx[e] : nx_[m][e];
        const T lz = d == 0 ? hz[e] : nz_[m][e];
        const T cv = d == 0 ? c[e] : nc_[m][e];
        T w1 = T(0), w2 = T(0);
        if (yf) {
          if (kl[e]) w1 += FY.w1[cpml_at32<false>(g, 1, 1, FY.p, s, qy, i, y, kk + e)];
          if (il && kv[e]) w2 += FY.w2[cpml_at32<false>(g, 1, 2, FY.p, s, qy, i, y, kk + e)];
        }
        const T cye = curl_y<EQ>(a, cv);
        if (hxo && im && yl && kl[e]) w1 += (-cye) * lx;
        if (hzo && il && yl && km[e]) w2 += cye * lz;
        ay[m][e] = w1;
        cy[m][e] = w2;
      }
    }
    T zb[NZN], zc[NZN];
#pragma unroll
    for (int m = ZLO; m <= ZHI; ++m) {
      zb[m - ZLO] = ynb4<T, R>(bz, hbz, lane, m);
      zc[m - ZLO] = ynb4<T, R>(cz, hcz, lane, m);
    }
    T xup[R], xdn[R];
    xtaps<T, R, false>(i, NX, xup, xdn);
    T ex[4], ey[4], ez[4], ca[4];
    from4(cur[SEX * 32], ex);
    from4(cur[SEY * 32], ey);
    from4(cur[SEZ * 32], ez);
    from4(cur[SCA * 32], ca);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (dxo && il && jm && km[e]) ex[e] = ca[e] * ex[e];
      if (dyo && im && jl && km[e]) ey[e] = ca[e] * ey[e];
      if (dzo && im && jm && kl[e]) ez[e] = ca[e] * ez[e];
      ez[e] += gfwd_t<T, R>([&](int d) { return qA[R + d][e]; }, xup, xdn);
      ez[e] += gfwd_t<T, R>([&](int d) { return ay[d + R][e]; }, yup, ydn);
      ey[e] += gfwd_t<T, R>([&](int d) { return qB[R + d][e]; }, xup, xdn);
      ey[e] += gfwd_t<T, R>([&](int d) { return zb[e + d - ZLO]; }, zup[e], zdn[e]);
      ex[e] += gfwd_t<T, R>([&](int d) { return cy[d + R][e]; }, yup, ydn);
      ex[e] += gfwd_t<T, R>([&](int d) { return zc[e + d - ZLO]; }, zup[e], zdn[e]);
    }
    if (head >= 0) {
      // receiver cotangents and staged source terms of step it-1 (the E-CPML
      // weights of that step: k3p_adj_w after this kernel)
      const bool pts = (kg.src_rows && kg.src_rows[(long long)s * NX + i]) ||
                       (kg.rcv_rows && kg.rcv_rows[(long long)s * NX + i]);
      if (pts) {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (kv[e]) head_gen(P, head, s, i, j, kk + e, true, false, ex[e], ey[e], ez[e]);
      }
    }
    if (lv) {
      st4(f.Ex + rb + o, ex);
      st4(f.Ey + rb + o, ey);
      st4(f.Ez + rb + o, ez);
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        qA[m][e] = qA[m + 1][e];
        qB[m][e] = qB[m + 1][e];
      }
  }
}

}  // namespace dg
