// fdtd_3d_adj.cuh -- 3D adjoint kernels on the z-pitched working copy.
//
// Same decomposition as the 3D forward kernels (fdtd_3d.cuh): a warp owns
// 64 z columns (two per lane) of one (shot, y row) and streams x planes; a
// CTA holds four rows.  One reverse step is
//   k3v_adj_e: lambda_H += curl^T of the E channels, then the H-CPML
//              adjoint weights of the step at the cell;
//   k3v_adj_h: lambda_E <- ce_hist lambda_E + curl^T of the H channels, then
//              the head of the next reverse step at the cell (receiver
//              cotangents, staged source terms, E-CPML adjoint weights).
// The arithmetic of every value is that of fdtd_adjoint.cuh, which follows
// the reference (src/DeepGPR/lib/deepgpr_cpu.c:1112-1459, 1479-1534): a
// channel weight W of a source cell is its CPML weight(s) plus the interior
// term; a target gathers the transposed difference of W along each axis in
// the reference order.  Channels along x come from a register queue (the
// entering plane's weights are formed once), along y from direct loads of
// the neighbouring rows, along z from constant-distance shuffles plus halo
// lanes.  Near the axis ends the gathers use per-target tap tables (zero
// where the source point is outside the axis or its clamped stencil does not
// reach the target), so the same code covers the whole grid.
//
// CPML channel weights of the next plane (of the entering x plane, of the
// lane's z columns and of the neighbour rows' y faces) are staged into shared
// memory with cp.async while the current plane is computed (the forward
// kernels' scheme).  With one CPML face per axis the weights of the step
// itself (k3v_adj_e: H faces; k3v_adj_h: E faces of the next step) are formed
// by k3p_adj_w after the kernel.
#pragma once

#include "fdtd_3d.cuh"
#include "fdtd_tiled_adj.cuh"

namespace dg {

// Gather taps at target c of an axis of n points.  gather_back: up[r-1]
// multiplies W(-(r-1)), dn[r-1] multiplies W(r); gather_fwd: up[r-1]
// multiplies W(-r), dn[r-1] multiplies W(r-1) (deepgpr_cpu.c:429-507).
template <typename T, int R>
__device__ __forceinline__ void gtaps_back(int c, int n, T (&up)[R], T (&dn)[R]) {
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    const int u = c - (r - 1), d = c + r;
    const int ru = u >= 0 ? rad_back(u, n, R) : 0, rd = d < n ? rad_back(d, n, R) : 0;
    up[r - 1] = r <= ru ? tap<T>(ru, r) : T(0);
    dn[r - 1] = r <= rd ? tap<T>(rd, r) : T(0);
  }
}
template <typename T, int R>
__device__ __forceinline__ void gtaps_fwd(int c, int n, T (&up)[R], T (&dn)[R]) {
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    const int u = c - r, d = c + r - 1;
    const int ru = u >= 0 ? rad_fwd(u, n, R) : 0, rd = d < n ? rad_fwd(d, n, R) : 0;
    up[r - 1] = r <= ru ? tap<T>(ru, r) : T(0);
    dn[r - 1] = r <= rd ? tap<T>(rd, r) : T(0);
  }
}
// x taps of a plane: the constant full-stencil taps away from the ends
template <typename T, int R, bool BACK>
__device__ __forceinline__ void xtaps(int i, int n, T (&up)[R], T (&dn)[R]) {
  const bool full = BACK ? (i >= 2 * R - 1 && i + 2 * R - 1 < n) : (i >= 2 * R - 1 && i + 2 * R <= n);
  if (full) {
#pragma unroll
    for (int r = 1; r <= R; ++r) up[r - 1] = dn[r - 1] = tap<T>(R, r);
  } else if (BACK) {
    gtaps_back<T, R>(i, n, up, dn);
  } else {
    gtaps_fwd<T, R>(i, n, up, dn);
  }
}
template <typename T, int R, typename WF>
__device__ __forceinline__ T gback_t(const WF& W, const T (&up)[R], const T (&dn)[R]) {
  if (R == 1) {
    T acc = W(0);
    acc -= dn[0] * W(1);
    return acc;
  }
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    acc += up[r - 1] * W(-(r - 1));
    acc -= dn[r - 1] * W(r);
  }
  return acc;
}
template <typename T, int R, typename WF>
__device__ __forceinline__ T gfwd_t(const WF& W, const T (&up)[R], const T (&dn)[R]) {
  T acc = T(0);
#pragma unroll
  for (int r = 1; r <= R; ++r) {
    acc += up[r - 1] * W(-r);
    acc -= dn[r - 1] * W(r - 1);
  }
  return acc;
}

// Face q of coordinate c on the low / high face of an axis (E faces skip c == 0).
template <bool EFACE>
__device__ __forceinline__ void face_q(int plo, int phi, int c, int n, int& q0, int& q1) {
  q0 = EFACE ? (c > 0 ? q_low_e(plo, c) : -1) : q_low_h(plo, c);
  q1 = (EFACE && c == 0) ? -1 : q_high(phi, c, n);
}

// Element offset of a CPML array entry (psi / weight shapes of psi_dims_e/h).
template <bool EFACE>
__device__ __forceinline__ long long cpml_at(const Grid& g, int axis, int slot, int p, int s, int q, int i, int j,
                                             int k) {
  const PsiDims d = EFACE ? psi_dims_e(g, axis, slot, p) : psi_dims_h(g, axis, slot, p);
  return psi_index(d, axis, s, q, i, j, k);
}

// The same in 32-bit arithmetic: the staged (single-face) kernels run only
// when every CPML array has fewer than 2^31 elements.
template <bool EFACE>
__device__ __forceinline__ int cpml_at32(const Grid& g, int axis, int slot, int p, int s, int q, int i, int j, int k) {
  const PsiDims d = EFACE ? psi_dims_e(g, axis, slot, p) : psi_dims_h(g, axis, slot, p);
  const int u = axis == 0 ? q : i, v = axis == 1 ? q : j, w = axis == 2 ? q : k;
  return ((s * d.a + u) * d.b + v) * d.c + w;
}

// Adjoint CPML weight with psi already loaded: returns w, stores psi
// (pml_weight of fdtd_adjoint.cuh).
template <typename T>
__device__ __forceinline__ T pml_weight_v(T lam, T inv_h, T up, T sign, const Prof<T>& pr, T ph, T* psi) {
  const T w = (sign * up * pr.ra1 * lam - pr.rf * ph) * inv_h;
  *psi = sign * up * pr.rb * lam + pr.re * ph;
  return w;
}

// curl scale along y / z (scaled() of fdtd_adjoint.cuh); EQ: dy == dz == dx
template <bool EQ, typename T>
__device__ __forceinline__ T curl_y(const AdjArgs<T>& a, T c) {
  return (EQ || a.dy_eq) ? c : div_fixed(c * a.dx, a.ddy);
}
template <bool EQ, typename T>
__device__ __forceinline__ T curl_z(const AdjArgs<T>& a, T c) {
  return (EQ || a.dz_eq) ? c : div_fixed(c * a.dx, a.ddz);
}

// General-form CPML pieces, out of line: a call is never predicated, so
// these lookups cost nothing on the planes and rows that do not take them
// (the kernels' parameter block is __grid_constant__, so references into it
// are passed without a copy).
// CPML weight of a source cell from the faces lo, hi of an axis (0 + lo + hi,
// add_pml of fdtd_adjoint.cuh).
template <typename T, bool EFACE>
__device__ __noinline__ T pml_w_gen(const Face<T>& lo, const Face<T>& hi, const Grid& g, int axis, int slot, int s,
                                    int i, int j, int k) {
  T w = T(0);
  add_pml<T, EFACE>(w, lo, hi, g, axis, slot, s, i, j, k);
  return w;
}
// H-CPML adjoint weights of one cell, every face in turn (deepgpr_cpu.c:1331-1396)
template <typename T>
__device__ __noinline__ void h_weights_gen(const AdjArgs<T>& a, int s, int i, int j, int k, T up, T hx, T hy,
                                           T hz) {
  const Grid& g = a.g;
  int qh[6];
  face_q<false>(a.hF[0].p, a.hF[1].p, i, g.NX, qh[0], qh[1]);
  face_q<false>(a.hF[2].p, a.hF[3].p, j, g.NY, qh[2], qh[3]);
  face_q<false>(a.hF[4].p, a.hF[5].p, k, g.NZ, qh[4], qh[5]);
  const bool il = i < g.NX - 1, jl = j < g.NY - 1, kl = k < g.NZ - 1;
#pragma unroll
  for (int fc = 0; fc < 6; ++fc) {
    const int q = qh[fc];
    if (q < 0) continue;
    const Face<T>& F = a.hF[fc];
    const Prof<T> pr = prof(F, q);
    const int axis = fc >> 1;
    const bool on1 = axis == 2 ? jl : kl;
    const bool on2 = axis == 0 ? jl : il;
    const T l1 = axis == 0 ? hy : hx;
    const T l2 = axis == 2 ? hy : hz;
    const T ih = axis == 0 ? a.inv_dx : (axis == 1 ? a.inv_dy : a.inv_dz);
    const T s1 = axis == 1 ? T(-1) : T(1);
    const T s2 = axis == 1 ? T(1) : T(-1);
    if (on1) {
      const long long pi = cpml_at<false>(g, axis, 1, F.p, s, q, i, j, k);
      F.w1[pi] = pml_weight(l1, ih, up, s1, pr, &F.psi1[pi]);
    }
    if (on2) {
      const long long pi = cpml_at<false>(g, axis, 2, F.p, s, q, i, j, k);
      F.w2[pi] = pml_weight(l2, ih, up, s2, pr, &F.psi2[pi]);
    }
  }
}
// head of a reverse step at one cell: receivers, sources, E-CPML weights
template <typename T>
__device__ __noinline__ void head_gen(const TiledAdj<T>& P, int st, int s, int i, int j, int k, bool pts, bool epml,
                                      T& ex, T& ey, T& ez) {
  const Grid& g = P.a.g;
  const int c = (i * g.NY + j) * g.NZ + k;
  if (pts) tiled_head(P, st, s, c, ex, ey, ez);
  if (epml) e_pml_head(P.a, s, i, j, k, c, ex, ey, ez);
}

// stage slots of the adjoint kernels: 6 fixed ones, then w1, w2 of the
// y-face weights of the 2R neighbour rows of the gathers along y
constexpr int kAdjSlots0 = 6;
template <int R>
__host__ __device__ constexpr int adj_slots() {
  return kAdjSlots0 + 4 * R;
}
enum : int {
  kStXw1 = 0, kStXw2 = 1,      // weights of the entering x plane's channels
  kStZw1 = 2, kStZw2 = 3,      // z-face weights of the lane's columns
  kStHw1 = 4, kStHw2 = 5,      // z-face weights of the halo column (cell 0)
  kStY = 6                     // row m: kStY + 2 m (w1), kStY + 2 m + 1 (w2)
};
// dynamic shared memory of k3v_adj_e / k3v_adj_h: two stages per warp
template <typename T, int R>
__host__ __device__ constexpr int k3_adj_smem_bytes() {
  return K3_WARPS * 2 * adj_slots<R>() * 2 * 32 * (int)sizeof(T);
}

// ---------------------------------------------------------------------------
// Adjoint E step.  Channels (source = E cell), deepgpr_cpu.c:1236-1270:
//   A_X = x faces w1 + (-c) lambda_ey,  A_Y = y faces w1 + c_y lambda_ex  -> lambda_hz
//   B_X = x faces w2 + c lambda_ez,     B_Z = z faces w1 + (-c_z) lambda_ex -> lambda_hy
//   C_Y = y faces w2 + (-c_y) lambda_ez, C_Z = z faces w2 + c_z lambda_ey  -> lambda_hx
// then the H-CPML weights of step it at the cell (deepgpr_cpu.c:1331-1396).
// ---------------------------------------------------------------------------
template <typename T, int R, bool EQ, bool GEN>
__global__ void __launch_bounds__(32 * K3_WARPS, k3_adj_min_blocks<T, R>())
    k3v_adj_e(const __grid_constant__ TiledAdj<T> P, K3Buf<T> f, K3Geom kg) {
  constexpr int ZLO = -(R - 1), ZHI = R + 1, NZN = ZHI - ZLO + 1;   // z sources of the pair, gather_back
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
  const K3Pos wp = k3_pos(kg, g);
  if (!wp.live) return;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const int PS = NY * zp;
  const long long sbase = (long long)s * NX * PS;
  const T* __restrict__ lEx = f.Ex + sbase;
  const T* __restrict__ lEy = f.Ey + sbase;
  const T* __restrict__ lEz = f.Ez + sbase;
  T* __restrict__ lHx = f.Hx + sbase;
  T* __restrict__ lHy = f.Hy + sbase;
  T* __restrict__ lHz = f.Hz + sbase;
  const T* __restrict__ cc = f.ce_curl;
  const int hk = k3_halo<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;
  const int hrow = j * zp + (hok ? hk : 0);
  // GEN: faces of an axis may meet (general form); else one face per axis (staged)
  const bool pml = a.has_cpml != 0, cps = !GEN && pml;
  // parts of the interior predicates (upd_e*): mid = 0 < c < n-1, lo = c < n-1
  const bool dxo = NY - 1 != 1 || NZ - 1 != 1, dyo = NX - 1 != 1 || NZ - 1 != 1, dzo = NX - 1 != 1 || NY - 1 != 1;
  const bool jm = j > 0 && j < NY - 1, jl = j < NY - 1;
  bool kv[2], km[2], kl[2];
  int kof[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = kk + e;
    kof[e] = k;
    kv[e] = k < NZ;
    km[e] = k > 0 && k < NZ - 1;
    kl[e] = k < NZ - 1;
  }
  const bool hkm = hok && hk > 0 && hk < NZ - 1;
  T zup[2][R], zdn[2][R], yup[R], ydn[R];
  gtaps_back<T, R>(kk, NZ, zup[0], zdn[0]);
  gtaps_back<T, R>(kk + 1, NZ, zup[1], zdn[1]);
  gtaps_back<T, R>(j, NY, yup, ydn);
  // CPML positions fixed for the warp / lane: E y faces of the neighbour rows
  // (bit d + R - 1), E z face of the lane's columns and of its halo column,
  // With the faces of an axis apart (cps), both columns of a lane lie in the
  // same face or none, and the H-CPML weights of the step are formed after this
  // kernel by k3p_adj_w.
  unsigned ymask = 0;
  if (pml) {
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) {
      const int y = j + d;
      int q0, q1;
      face_q<true>(a.eF[2].p, a.eF[3].p, y, NY, q0, q1);
      if (y >= 0 && y < NY && (q0 >= 0 || q1 >= 0)) ymask |= 1u << (d + R - 1);
    }
  }
  int ezq[2], ehq = -1;
  bool ezlo = false;   // the lane's z face is the low one
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    int q0, q1;
    face_q<true>(a.eF[4].p, a.eF[5].p, kk + e, NZ, q0, q1);
    ezq[e] = (cps && kv[e]) ? (q0 >= 0 ? q0 : q1) : -1;
    ezlo |= q0 >= 0;
  }
  bool ehlo = true;
  if (cps && hok) {
    int q0, q1;
    face_q<true>(a.eF[4].p, a.eF[5].p, hk, NZ, q0, q1);
    ehq = q0 >= 0 ? q0 : q1;
    ehlo = q0 >= 0;
  }
  const bool any_ez = __any_sync(kFullMask, ezq[0] >= 0 || ezq[1] >= 0 || ehq >= 0);

  constexpr int NSL = adj_slots<R>();
  extern __shared__ __align__(16) unsigned char k3_adj_smem[];   // k3_adj_smem_bytes<T, R>()
  T(*const sg)[NSL][2][32] = reinterpret_cast<T(*)[NSL][2][32]>(k3_adj_smem) + 2 * threadIdx.y;
  // stages the CPML operands of plane i into stage b (one commit group per plane)
  auto stage = [&](int i, int b) {
    if (cps) {
      const int xi = i + R;   // entering plane of the x channels
      int qa, qb;
      face_q<true>(a.eF[0].p, a.eF[1].p, xi, NX, qa, qb);
      const bool xin = xi < NX && (qa >= 0 || qb >= 0);
      const bool il = i < NX - 1;
      if (xin || any_ez || ymask) {
        // E y-face weights of the neighbour rows (A_Y, C_Y sources)
#pragma unroll
        for (int d = -(R - 1); d <= R; ++d) {
          const int m = d + R - 1;
          if (!((ymask >> m) & 1u)) continue;
          const int y = j + d;
          int q0, q1;
          face_q<true>(a.eF[2].p, a.eF[3].p, y, NY, q0, q1);
          const bool lo = q0 >= 0;
          const int q = lo ? q0 : q1, py = lo ? a.eF[2].p : a.eF[3].p;
          const T* YW1 = lo ? a.eF[2].w1 : a.eF[3].w1;
          const T* YW2 = lo ? a.eF[2].w2 : a.eF[3].w2;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (il && kv[e]) cp_async(&sg[b][kStY + 2 * m][e][lane], YW1 + cpml_at32<true>(g, 1, 1, py, s, q, i, y, kof[e]));
            if (kl[e]) cp_async(&sg[b][kStY + 2 * m + 1][e][lane], YW2 + cpml_at32<true>(g, 1, 2, py, s, q, i, y, kof[e]));
          }
        }
        const bool xlo = qa >= 0;
        const int qx = xlo ? qa : qb, px = xlo ? a.eF[0].p : a.eF[1].p;
        const T* XW1 = xlo ? a.eF[0].w1 : a.eF[1].w1;
        const T* XW2 = xlo ? a.eF[0].w2 : a.eF[1].w2;
        const int pez = ezlo ? a.eF[4].p : a.eF[5].p;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int k = kof[e];
          if (xin && jl && kv[e]) cp_async(&sg[b][kStXw1][e][lane], XW1 + cpml_at32<true>(g, 0, 1, px, s, qx, xi, j, k));
          if (xin && kl[e]) cp_async(&sg[b][kStXw2][e][lane], XW2 + cpml_at32<true>(g, 0, 2, px, s, qx, xi, j, k));
          if (ezq[e] >= 0) {
            if (il)
              cp_async(&sg[b][kStZw1][e][lane],
                       (ezlo ? a.eF[4].w1 : a.eF[5].w1) + cpml_at32<true>(g, 2, 1, pez, s, ezq[e], i, j, k));
            if (jl)
              cp_async(&sg[b][kStZw2][e][lane],
                       (ezlo ? a.eF[4].w2 : a.eF[5].w2) + cpml_at32<true>(g, 2, 2, pez, s, ezq[e], i, j, k));
          }
        }
        if (ehq >= 0) {
          const int pe = ehlo ? a.eF[4].p : a.eF[5].p;
          if (il)
            cp_async(&sg[b][kStHw1][0][lane],
                     (ehlo ? a.eF[4].w1 : a.eF[5].w1) + cpml_at32<true>(g, 2, 1, pe, s, ehq, i, j, hk));
          if (jl)
            cp_async(&sg[b][kStHw2][0][lane],
                     (ehlo ? a.eF[4].w2 : a.eF[5].w2) + cpml_at32<true>(g, 2, 2, pe, s, ehq, i, j, hk));
        }
      }
    }
    cp_async_commit();
  };

  // x channels of plane x from its lambda_ey, lambda_ez, c (and the staged
  // weights when the plane has an E x face)
  auto xchan = [&](int x, const T (&ly)[2], const T (&lz)[2], const T (&c)[2], int b, T (&A)[2], T (&B)[2]) {
    const bool xm = x > 0 && x < NX - 1;
    int qa = -1, qb = -1;
    if (pml) face_q<true>(a.eF[0].p, a.eF[1].p, x, NX, qa, qb);
    const bool xin = x >= 0 && x < NX && (qa >= 0 || qb >= 0);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      T wa = T(0), wb = T(0);
      if (xin) {
        if (cps) {
          if (jl && kv[e]) wa += sg[b][kStXw1][e][lane];
          if (kl[e]) wb += sg[b][kStXw2][e][lane];
        } else if (GEN) {
          if (jl && kv[e]) wa = pml_w_gen<T, true>(a.eF[0], a.eF[1], g, 0, 1, s, x, j, kof[e]);
          if (kl[e]) wb = pml_w_gen<T, true>(a.eF[0], a.eF[1], g, 0, 2, s, x, j, kof[e]);
        }
      }
      if (dyo && xm && jl && km[e]) wa += (-c[e]) * ly[e];
      if (dzo && xm && jm && kl[e]) wb += c[e] * lz[e];
      A[e] = wa;
      B[e] = wb;
    }
  };

  const int x0 = wp.x0;
  T qA[2 * R][2], qB[2 * R][2];   // A_X, B_X at planes i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = x0 - R + 1 + m;
    T ly[2] = {T(0), T(0)}, lz[2] = {T(0), T(0)}, c[2] = {T(0), T(0)};
    if (pl >= 0 && pl < NX) {
      ld2(lEy + pl * PS + row, ly);
      ld2(lEz + pl * PS + row, lz);
      ld2(cc + pl * PS + row, c);
    }
    // staged weights are not available for these planes: general form
    const bool xm = pl > 0 && pl < NX - 1;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      T wa = T(0), wb = T(0);
      if (pml && pl >= 0 && pl < NX) {
        if (jl && kv[e]) wa = pml_w_gen<T, true>(a.eF[0], a.eF[1], g, 0, 1, s, pl, j, kof[e]);
        if (kl[e]) wb = pml_w_gen<T, true>(a.eF[0], a.eF[1], g, 0, 2, s, pl, j, kof[e]);
      }
      if (dyo && xm && jl && km[e]) wa += (-c[e]) * ly[e];
      if (dzo && xm && jm && kl[e]) wb += c[e] * lz[e];
      qA[m][e] = wa;
      qB[m][e] = wb;
    }
  }
  // operands of the next plane
  T nyR[2], nzR[2], ncR[2];           // plane i+R: lambda_ey, lambda_ez, c
  T nx[2], ny[2], nz[2], nc[2];       // plane i: lambda_ex, lambda_ey, lambda_ez, c
  T nhx[2], nhy[2], nhz[2];           // plane i: lambda_H
  T nhex = T(0), nhey = T(0), nhc = T(0);   // halo column: lambda_ex, lambda_ey, c
  auto fetch = [&](int i) {
    const int o = i * PS;
    if (i + R < NX) {
      ld2(lEy + o + R * PS + row, nyR);
      ld2(lEz + o + R * PS + row, nzR);
      ld2(cc + o + R * PS + row, ncR);
    } else {
      nyR[0] = nyR[1] = nzR[0] = nzR[1] = ncR[0] = ncR[1] = T(0);
    }
    ld2(lEx + o + row, nx);
    ld2(lEy + o + row, ny);
    ld2(lEz + o + row, nz);
    ld2(cc + o + row, nc);
    ld2(lHx + o + row, nhx);
    ld2(lHy + o + row, nhy);
    ld2(lHz + o + row, nhz);
    if (hok) {
      nhex = lEx[o + hrow];
      nhey = lEy[o + hrow];
      nhc = cc[o + hrow];
    }
  };
  fetch(x0);
  stage(x0, 0);
  for (int i = x0; i < wp.x1; ++i) {
    T yR[2], zR[2], cR[2], ex[2], ey[2], ez[2], c[2], hx[2], hy[2], hz[2];
    const T hex = nhex, hey = nhey, hc = nhc;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      yR[e] = nyR[e];
      zR[e] = nzR[e];
      cR[e] = ncR[e];
      ex[e] = nx[e];
      ey[e] = ny[e];
      ez[e] = nz[e];
      c[e] = nc[e];
      hx[e] = nhx[e];
      hy[e] = nhy[e];
      hz[e] = nhz[e];
    }
    if (i + 1 < wp.x1) {
      fetch(i + 1);
      stage(i + 1, (i + 1 - x0) & 1);
    } else {
      cp_async_commit();
    }
    cp_async_wait_prev();
    const int b = (i - x0) & 1;
    const int o = i * PS;
    const bool il = i < NX - 1, im = i > 0 && i < NX - 1;
    xchan(i + R, yR, zR, cR, b, qA[2 * R - 1], qB[2 * R - 1]);
    // z channels of the lane's columns and of the halo column
    T bz[2], cz[2], hbz = T(0), hcz = T(0);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      T w1 = T(0), w2 = T(0);
      if (cps) {
        if (ezq[e] >= 0 && il) w1 += sg[b][kStZw1][e][lane];
        if (ezq[e] >= 0 && jl) w2 += sg[b][kStZw2][e][lane];
      } else if (GEN && pml && kv[e]) {
        if (il) w1 = pml_w_gen<T, true>(a.eF[4], a.eF[5], g, 2, 1, s, i, j, kof[e]);
        if (jl) w2 = pml_w_gen<T, true>(a.eF[4], a.eF[5], g, 2, 2, s, i, j, kof[e]);
      }
      const T cze = curl_z<EQ>(a, c[e]);
      if (dxo && il && jm && km[e]) w1 += (-cze) * ex[e];
      if (dyo && im && jl && km[e]) w2 += cze * ey[e];
      bz[e] = w1;
      cz[e] = w2;
    }
    if (hok) {
      if (cps) {
        if (ehq >= 0 && il) hbz += sg[b][kStHw1][0][lane];
        if (ehq >= 0 && jl) hcz += sg[b][kStHw2][0][lane];
      } else if (GEN && pml) {
        if (il) hbz = pml_w_gen<T, true>(a.eF[4], a.eF[5], g, 2, 1, s, i, j, hk);
        if (jl) hcz = pml_w_gen<T, true>(a.eF[4], a.eF[5], g, 2, 2, s, i, j, hk);
      }
      const T czh = curl_z<EQ>(a, hc);
      if (dxo && il && jm && hkm) hbz += (-czh) * hex;
      if (dyo && im && jl && hkm) hcz += czh * hey;
    }
    T zb[NZN], zc[NZN];
    znb<T, R, ZLO, ZHI>(bz, hbz, lane, zb);
    znb<T, R, ZLO, ZHI>(cz, hcz, lane, zc);
    // y channels of rows j + d (own row from the registers)
    T ay[2 * R][2], cy[2 * R][2];
#pragma unroll
    for (int d = -(R - 1); d <= R; ++d) {
      const int y = j + d;
      const int m = d + R - 1;
      T lx[2], lz[2], cv[2];
      if (d == 0) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          lx[e] = ex[e];
          lz[e] = ez[e];
          cv[e] = c[e];
        }
      } else if (y >= 0 && y < NY) {
        ld2(lEx + o + row + d * zp, lx);
        ld2(lEz + o + row + d * zp, lz);
        ld2(cc + o + row + d * zp, cv);
      } else {
        lx[0] = lx[1] = lz[0] = lz[1] = cv[0] = cv[1] = T(0);
      }
      const bool ym = y > 0 && y < NY - 1;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        T w1 = T(0), w2 = T(0);
        if ((ymask >> m) & 1u) {
          if (cps) {
            if (il && kv[e]) w1 += sg[b][kStY + 2 * m][e][lane];
            if (kl[e]) w2 += sg[b][kStY + 2 * m + 1][e][lane];
          } else if (GEN) {
            if (il && kv[e]) w1 = pml_w_gen<T, true>(a.eF[2], a.eF[3], g, 1, 1, s, i, y, kof[e]);
            if (kl[e]) w2 = pml_w_gen<T, true>(a.eF[2], a.eF[3], g, 1, 2, s, i, y, kof[e]);
          }
        }
        const T cye = curl_y<EQ>(a, cv[e]);
        if (dxo && il && ym && km[e]) w1 += cye * lx[e];
        if (dzo && im && ym && kl[e]) w2 += (-cye) * lz[e];
        ay[m][e] = w1;
        cy[m][e] = w2;
      }
    }
    // gathers, in the reference order
    T xup[R], xdn[R];
    xtaps<T, R, true>(i, NX, xup, xdn);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      hz[e] += gback_t<T, R>([&](int d) { return qA[R - 1 + d][e]; }, xup, xdn);
      hz[e] += gback_t<T, R>([&](int d) { return ay[d + R - 1][e]; }, yup, ydn);
      hy[e] += gback_t<T, R>([&](int d) { return qB[R - 1 + d][e]; }, xup, xdn);
      hy[e] += gback_t<T, R>([&](int d) { return zb[e + d - ZLO]; }, zup[e], zdn[e]);
      hx[e] += gback_t<T, R>([&](int d) { return cy[d + R - 1][e]; }, yup, ydn);
      hx[e] += gback_t<T, R>([&](int d) { return zc[e + d - ZLO]; }, zup[e], zdn[e]);
    }
    if (kv[1]) {
      st2(lHx + o + row, hx);
      st2(lHy + o + row, hy);
      st2(lHz + o + row, hz);
    } else if (kv[0]) {
      lHx[o + row] = hx[0];
      lHy[o + row] = hy[0];
      lHz[o + row] = hz[0];
    }
    // H-CPML adjoint weights of step it at the cell: with one face per axis
    // (cps) in k3p_adj_w after this kernel
    if (GEN && pml) {
      // faces of one axis meet: every face in turn, direct loads
#pragma unroll
      for (int e = 0; e < 2; ++e)
        if (kv[e]) h_weights_gen(a, s, i, j, kof[e], f.ch_rhs[o + row + e], hx[e], hy[e], hz[e]);
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        qA[m][e] = qA[m + 1][e];
        qB[m][e] = qB[m + 1][e];
      }
  }
}

// ---------------------------------------------------------------------------
// Adjoint H step.  Channels (source = H cell), deepgpr_cpu.c:1400-1424:
//   A_X = x faces w1 + c lambda_hy,      A_Y = y faces w1 + (-c_y) lambda_hx -> lambda_ez
//   B_X = x faces w2 + (-c) lambda_hz,   B_Z = z faces w1 + c_z lambda_hx    -> lambda_ey
//   C_Y = y faces w2 + c_y lambda_hz,    C_Z = z faces w2 + (-c_z) lambda_hy -> lambda_ex
// then the head of step it-1 at the cell.
// ---------------------------------------------------------------------------
template <typename T, int R, bool EQ, bool GEN>
__global__ void __launch_bounds__(32 * K3_WARPS, k3_adj_min_blocks<T, R>())
    k3v_adj_h(const __grid_constant__ TiledAdj<T> P, K3Buf<T> f, K3Geom kg) {
  constexpr int ZLO = -R, ZHI = R, NZN = ZHI - ZLO + 1;   // z sources of the pair, gather_fwd
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const K3Pos wp = k3_pos(kg, g);
  if (!wp.live) return;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const int PS = NY * zp;
  const long long sbase = (long long)s * NX * PS;
  T* __restrict__ lEx = f.Ex + sbase;
  T* __restrict__ lEy = f.Ey + sbase;
  T* __restrict__ lEz = f.Ez + sbase;
  const T* __restrict__ lHx = f.Hx + sbase;
  const T* __restrict__ lHy = f.Hy + sbase;
  const T* __restrict__ lHz = f.Hz + sbase;
  const T* __restrict__ hcf = f.ch_curl;
  const int it = a.ctrl->cur - a.k_in_chunk;
  const int head = it - 1;
  const int hk = k3_halo<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;
  const int hrow = j * zp + (hok ? hk : 0);
  // GEN: faces of an axis may meet (general form); else one face per axis (staged)
  const bool pml = a.has_cpml != 0, cps = !GEN && pml;
  // parts of upd_h*: hx: NX-1 != 1, mid(i), lo(j), lo(k); hy: NY-1 != 1, lo(i),
  // mid(j), lo(k); hz: NZ-1 != 1, lo(i), lo(j), mid(k); and of upd_e* for ce_hist
  const bool hxo = NX - 1 != 1, hyo = NY - 1 != 1, hzo = NZ - 1 != 1;
  const bool dxo = NY - 1 != 1 || NZ - 1 != 1, dyo = NX - 1 != 1 || NZ - 1 != 1, dzo = NX - 1 != 1 || NY - 1 != 1;
  const bool jm = j > 0 && j < NY - 1, jl = j < NY - 1;
  bool kv[2], km[2], kl[2];
  int kof[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = kk + e;
    kof[e] = k;
    kv[e] = k < NZ;
    km[e] = k > 0 && k < NZ - 1;
    kl[e] = k < NZ - 1;
  }
  const bool hkl = hok && hk < NZ - 1;
  T zup[2][R], zdn[2][R], yup[R], ydn[R];
  gtaps_fwd<T, R>(kk, NZ, zup[0], zdn[0]);
  gtaps_fwd<T, R>(kk + 1, NZ, zup[1], zdn[1]);
  gtaps_fwd<T, R>(j, NY, yup, ydn);
  unsigned ymask = 0;   // H y faces of rows j + d (bit d + R)
  if (pml) {
#pragma unroll
    for (int d = -R; d <= R - 1; ++d) {
      const int y = j + d;
      int q0, q1;
      face_q<false>(a.hF[2].p, a.hF[3].p, y, NY, q0, q1);
      if (y >= 0 && y < NY && (q0 >= 0 || q1 >= 0)) ymask |= 1u << (d + R);
    }
  }
  // (E-CPML weights of the next reverse step: k3p_adj_w, after this kernel)
  int hzq[2], hhq = -1;
  bool hzlo = false;
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    int q0, q1;
    face_q<false>(a.hF[4].p, a.hF[5].p, kk + e, NZ, q0, q1);
    hzq[e] = (cps && kv[e]) ? (q0 >= 0 ? q0 : q1) : -1;
    hzlo |= q0 >= 0;
  }
  bool hhlo = true;
  if (cps && hok) {
    int q0, q1;
    face_q<false>(a.hF[4].p, a.hF[5].p, hk, NZ, q0, q1);
    hhq = q0 >= 0 ? q0 : q1;
    hhlo = q0 >= 0;
  }
  const bool any_hz = __any_sync(kFullMask, hzq[0] >= 0 || hzq[1] >= 0 || hhq >= 0);
  const bool heads = head >= 0;

  constexpr int NSL = adj_slots<R>();
  extern __shared__ __align__(16) unsigned char k3_adj_smem[];   // k3_adj_smem_bytes<T, R>()
  T(*const sg)[NSL][2][32] = reinterpret_cast<T(*)[NSL][2][32]>(k3_adj_smem) + 2 * threadIdx.y;
  auto stage = [&](int i, int b) {
    if (cps) {
      const int xi = i + R - 1;   // entering plane of the x channels
      int qa, qb;
      face_q<false>(a.hF[0].p, a.hF[1].p, xi, NX, qa, qb);
      const bool xin = xi < NX && (qa >= 0 || qb >= 0);
      const bool il = i < NX - 1;
      if (xin || any_hz || ymask) {
        // H y-face weights of the neighbour rows (A_Y, C_Y sources)
#pragma unroll
        for (int d = -R; d <= R - 1; ++d) {
          const int m = d + R;
          if (!((ymask >> m) & 1u)) continue;
          const int y = j + d;
          int q0, q1;
          face_q<false>(a.hF[2].p, a.hF[3].p, y, NY, q0, q1);
          const bool lo = q0 >= 0;
          const int q = lo ? q0 : q1, py = lo ? a.hF[2].p : a.hF[3].p;
          const T* YW1 = lo ? a.hF[2].w1 : a.hF[3].w1;
          const T* YW2 = lo ? a.hF[2].w2 : a.hF[3].w2;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (kl[e]) cp_async(&sg[b][kStY + 2 * m][e][lane], YW1 + cpml_at32<false>(g, 1, 1, py, s, q, i, y, kof[e]));
            if (il && kv[e]) cp_async(&sg[b][kStY + 2 * m + 1][e][lane], YW2 + cpml_at32<false>(g, 1, 2, py, s, q, i, y, kof[e]));
          }
        }
        const bool xlo = qa >= 0;
        const int qx = xlo ? qa : qb, px = xlo ? a.hF[0].p : a.hF[1].p;
        const T* XW1 = xlo ? a.hF[0].w1 : a.hF[1].w1;
        const T* XW2 = xlo ? a.hF[0].w2 : a.hF[1].w2;
        const int phz = hzlo ? a.hF[4].p : a.hF[5].p;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int k = kof[e];
          if (xin && kl[e]) cp_async(&sg[b][kStXw1][e][lane], XW1 + cpml_at32<false>(g, 0, 1, px, s, qx, xi, j, k));
          if (xin && jl && kv[e]) cp_async(&sg[b][kStXw2][e][lane], XW2 + cpml_at32<false>(g, 0, 2, px, s, qx, xi, j, k));
          if (hzq[e] >= 0) {
            if (jl)
              cp_async(&sg[b][kStZw1][e][lane],
                       (hzlo ? a.hF[4].w1 : a.hF[5].w1) + cpml_at32<false>(g, 2, 1, phz, s, hzq[e], i, j, k));
            if (il)
              cp_async(&sg[b][kStZw2][e][lane],
                       (hzlo ? a.hF[4].w2 : a.hF[5].w2) + cpml_at32<false>(g, 2, 2, phz, s, hzq[e], i, j, k));
          }
          if (!heads) continue;
        }
        if (hhq >= 0) {
          const int ph = hhlo ? a.hF[4].p : a.hF[5].p;
          if (jl)
            cp_async(&sg[b][kStHw1][0][lane],
                     (hhlo ? a.hF[4].w1 : a.hF[5].w1) + cpml_at32<false>(g, 2, 1, ph, s, hhq, i, j, hk));
          if (il)
            cp_async(&sg[b][kStHw2][0][lane],
                     (hhlo ? a.hF[4].w2 : a.hF[5].w2) + cpml_at32<false>(g, 2, 2, ph, s, hhq, i, j, hk));
        }
      }
    }
    cp_async_commit();
  };

  auto xchan = [&](int x, const T (&ly)[2], const T (&lz)[2], const T (&c)[2], int b, T (&A)[2], T (&B)[2]) {
    const bool xl = x >= 0 && x < NX - 1;
    int qa = -1, qb = -1;
    if (pml) face_q<false>(a.hF[0].p, a.hF[1].p, x, NX, qa, qb);
    const bool xin = x >= 0 && x < NX && (qa >= 0 || qb >= 0);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      T wa = T(0), wb = T(0);
      if (xin) {
        if (cps) {
          if (kl[e]) wa += sg[b][kStXw1][e][lane];
          if (jl && kv[e]) wb += sg[b][kStXw2][e][lane];
        } else if (GEN) {
          if (kl[e]) wa = pml_w_gen<T, false>(a.hF[0], a.hF[1], g, 0, 1, s, x, j, kof[e]);
          if (jl && kv[e]) wb = pml_w_gen<T, false>(a.hF[0], a.hF[1], g, 0, 2, s, x, j, kof[e]);
        }
      }
      if (hyo && xl && jm && kl[e]) wa += c[e] * ly[e];
      if (hzo && xl && jl && km[e]) wb += (-c[e]) * lz[e];
      A[e] = wa;
      B[e] = wb;
    }
  };

  const int x0 = wp.x0;
  T qA[2 * R][2], qB[2 * R][2];   // A_X, B_X at planes i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = x0 - R + m;
    T ly[2] = {T(0), T(0)}, lz[2] = {T(0), T(0)}, c[2] = {T(0), T(0)};
    if (pl >= 0 && pl < NX) {
      ld2(lHy + pl * PS + row, ly);
      ld2(lHz + pl * PS + row, lz);
      ld2(hcf + pl * PS + row, c);
    }
    const bool xl = pl >= 0 && pl < NX - 1;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      T wa = T(0), wb = T(0);
      if (pml && pl >= 0 && pl < NX) {
        if (kl[e]) wa = pml_w_gen<T, false>(a.hF[0], a.hF[1], g, 0, 1, s, pl, j, kof[e]);
        if (jl && kv[e]) wb = pml_w_gen<T, false>(a.hF[0], a.hF[1], g, 0, 2, s, pl, j, kof[e]);
      }
      if (hyo && xl && jm && kl[e]) wa += c[e] * ly[e];
      if (hzo && xl && jl && km[e]) wb += (-c[e]) * lz[e];
      qA[m][e] = wa;
      qB[m][e] = wb;
    }
  }
  T nyR[2], nzR[2], ncR[2];               // plane i+R-1: lambda_hy, lambda_hz, c
  T nhx[2], nhy[2], nhz[2], nc[2];        // plane i: lambda_H, c
  T nex[2], ney[2], nez[2], nca[2];       // plane i: lambda_E, ce_hist
  T nhhx = T(0), nhhy = T(0), nhc = T(0);   // halo column: lambda_hx, lambda_hy, c
  auto fetch = [&](int i) {
    const int o = i * PS;
    if (i + R - 1 < NX) {
      ld2(lHy + o + (R - 1) * PS + row, nyR);
      ld2(lHz + o + (R - 1) * PS + row, nzR);
      ld2(hcf + o + (R - 1) * PS + row, ncR);
    } else {
      nyR[0] = nyR[1] = nzR[0] = nzR[1] = ncR[0] = ncR[1] = T(0);
    }
    ld2(lHx + o + row, nhx);
    ld2(lHy + o + row, nhy);
    ld2(lHz + o + row, nhz);
    ld2(hcf + o + row, nc);
    ld2(lEx + o + row, nex);
    ld2(lEy + o + row, ney);
    ld2(lEz + o + row, nez);
    ld2(f.ce_hist + o + row, nca);
    if (hok) {
      nhhx = lHx[o + hrow];
      nhhy = lHy[o + hrow];
      nhc = hcf[o + hrow];
    }
  };
  fetch(x0);
  stage(x0, 0);
  for (int i = x0; i < wp.x1; ++i) {
    T yR[2], zR[2], cR[2], hx[2], hy[2], hz[2], c[2], ex[2], ey[2], ez[2], ca[2];
    const T hhx = nhhx, hhy = nhhy, hc = nhc;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      yR[e] = nyR[e];
      zR[e] = nzR[e];
      cR[e] = ncR[e];
      hx[e] = nhx[e];
      hy[e] = nhy[e];
      hz[e] = nhz[e];
      c[e] = nc[e];
      ex[e] = nex[e];
      ey[e] = ney[e];
      ez[e] = nez[e];
      ca[e] = nca[e];
    }
    if (i + 1 < wp.x1) {
      fetch(i + 1);
      stage(i + 1, (i + 1 - x0) & 1);
    } else {
      cp_async_commit();
    }
    cp_async_wait_prev();
    const int b = (i - x0) & 1;
    const int o = i * PS;
    const bool il = i < NX - 1, im = i > 0 && i < NX - 1;
    xchan(i + R - 1, yR, zR, cR, b, qA[2 * R - 1], qB[2 * R - 1]);
    T bz[2], cz[2], hbz = T(0), hcz = T(0);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      T w1 = T(0), w2 = T(0);
      if (cps) {
        if (hzq[e] >= 0 && jl) w1 += sg[b][kStZw1][e][lane];
        if (hzq[e] >= 0 && il) w2 += sg[b][kStZw2][e][lane];
      } else if (GEN && pml && kv[e]) {
        if (jl) w1 = pml_w_gen<T, false>(a.hF[4], a.hF[5], g, 2, 1, s, i, j, kof[e]);
        if (il) w2 = pml_w_gen<T, false>(a.hF[4], a.hF[5], g, 2, 2, s, i, j, kof[e]);
      }
      const T cze = curl_z<EQ>(a, c[e]);
      if (hxo && im && jl && kl[e]) w1 += cze * hx[e];
      if (hyo && il && jm && kl[e]) w2 += (-cze) * hy[e];
      bz[e] = w1;
      cz[e] = w2;
    }
    if (hok) {
      if (cps) {
        if (hhq >= 0 && jl) hbz += sg[b][kStHw1][0][lane];
        if (hhq >= 0 && il) hcz += sg[b][kStHw2][0][lane];
      } else if (GEN && pml) {
        if (jl) hbz = pml_w_gen<T, false>(a.hF[4], a.hF[5], g, 2, 1, s, i, j, hk);
        if (il) hcz = pml_w_gen<T, false>(a.hF[4], a.hF[5], g, 2, 2, s, i, j, hk);
      }
      const T czh = curl_z<EQ>(a, hc);
      if (hxo && im && jl && hkl) hbz += czh * hhx;
      if (hyo && il && jm && hkl) hcz += (-czh) * hhy;
    }
    T zb[NZN], zc[NZN];
    znb<T, R, ZLO, ZHI>(bz, hbz, lane, zb);
    znb<T, R, ZLO, ZHI>(cz, hcz, lane, zc);
    T ay[2 * R][2], cy[2 * R][2];   // A_Y, C_Y at rows j + d, d = -R .. R-1
#pragma unroll
    for (int d = -R; d <= R - 1; ++d) {
      const int y = j + d;
      const int m = d + R;
      T lx[2], lz[2], cv[2];
      if (d == 0) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          lx[e] = hx[e];
          lz[e] = hz[e];
          cv[e] = c[e];
        }
      } else if (y >= 0 && y < NY) {
        ld2(lHx + o + row + d * zp, lx);
        ld2(lHz + o + row + d * zp, lz);
        ld2(hcf + o + row + d * zp, cv);
      } else {
        lx[0] = lx[1] = lz[0] = lz[1] = cv[0] = cv[1] = T(0);
      }
      const bool yl = y >= 0 && y < NY - 1;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        T w1 = T(0), w2 = T(0);
        if ((ymask >> m) & 1u) {
          if (cps) {
            if (kl[e]) w1 += sg[b][kStY + 2 * m][e][lane];
            if (il && kv[e]) w2 += sg[b][kStY + 2 * m + 1][e][lane];
          } else if (GEN) {
            if (kl[e]) w1 = pml_w_gen<T, false>(a.hF[2], a.hF[3], g, 1, 1, s, i, y, kof[e]);
            if (il && kv[e]) w2 = pml_w_gen<T, false>(a.hF[2], a.hF[3], g, 1, 2, s, i, y, kof[e]);
          }
        }
        const T cye = curl_y<EQ>(a, cv[e]);
        if (hxo && im && yl && kl[e]) w1 += (-cye) * lx[e];
        if (hzo && il && yl && km[e]) w2 += cye * lz[e];
        ay[m][e] = w1;
        cy[m][e] = w2;
      }
    }
    T xup[R], xdn[R];
    xtaps<T, R, false>(i, NX, xup, xdn);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
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
    if (heads) {
      // receiver cotangents and staged source terms of step it-1
      const bool pts = (kg.src_rows && kg.src_rows[(long long)s * NX + i]) ||
                       (kg.rcv_rows && kg.rcv_rows[(long long)s * NX + i]);
      if (pts) {
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (kv[e]) head_gen(P, head, s, i, j, kof[e], true, false, ex[e], ey[e], ez[e]);
      }
      // E-CPML adjoint weights of step it-1: with one face per axis (cps) in
      // k3p_adj_w after this kernel
      if (GEN && pml) {
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (kv[e]) head_gen(P, head, s, i, j, kof[e], false, true, ex[e], ey[e], ez[e]);
      }
    }
    if (kv[1]) {
      st2(lEx + o + row, ex);
      st2(lEy + o + row, ey);
      st2(lEz + o + row, ez);
    } else if (kv[0]) {
      lEx[o + row] = ex[0];
      lEy[o + row] = ey[0];
      lEz[o + row] = ez[0];
    }
#pragma unroll
    for (int m = 0; m < 2 * R - 1; ++m)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        qA[m][e] = qA[m + 1][e];
        qB[m][e] = qB[m + 1][e];
      }
  }
}

// Head of reverse step nt-1 at every cell (receiver cotangents, staged source
// terms, E-CPML weights); runs once before the reverse loop.
template <typename T>
__global__ void __launch_bounds__(32 * K3_WARPS) k3v_adj_head(TiledAdj<T> P, K3Buf<T> f, K3Geom kg) {
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  const K3Pos wp = k3_pos(kg, g);
  if (!wp.live) return;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, s = wp.s, j = wp.j, kk = wp.kk;
  const int PS = NY * zp;
  const long long sbase = (long long)s * NX * PS;
  const int st = a.ctrl->cur;
  for (int i = wp.x0; i < wp.x1; ++i) {
    const long long o = sbase + (long long)i * PS + j * zp;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int k = kk + e;
      if (k >= NZ) continue;
      T ex = f.Ex[o + k], ey = f.Ey[o + k], ez = f.Ez[o + k];
      const int c = (i * NY + j) * NZ + k;
      tiled_head(P, st, s, c, ex, ey, ez);
      if (a.has_cpml) e_pml_head(a, s, i, j, k, c, ex, ey, ez);
      f.Ex[o + k] = ex;
      f.Ey[o + k] = ey;
      f.Ez[o + k] = ez;
    }
  }
}

// ---------------------------------------------------------------------------
// Imaging condition of one saved step on the 3D working copy (deepgpr_cpu.c:
// 1659-1745): one thread per history-box cell sums shot by shot, component
// by component (the reference's order), the terms of lambda_E before this
// step's ce_hist scaling with E^n and E^{n+1} (E-only) or R^n.  KIND, EONLY,
// ACC64 and NC (components: 1 for Ez, 3 for mode 3) are fixed at compile
// time; the shots are read in batches of U, the next batch's loads issued
// before the current batch is summed.  lambda element (s, i, j, k) sits at
// s * ls + i * lp + j * lr + k.
// ---------------------------------------------------------------------------
constexpr int kImage3Threads = 128;
// Resident CTAs per SM of k3_image: 8 (64 registers a thread) measured 6 %
// faster than 80 registers on 320 x 320 x 160 and 160^3 + CPML 10 (4 shots);
// 12 (40 registers) spills and is 17 % slower.
constexpr int kImage3MinBlocks = 8;

template <typename T, int KIND, bool EONLY, bool ACC64, int NC>
__global__ void __launch_bounds__(kImage3Threads, kImage3MinBlocks) k3_image(AdjArgs<T> a, const T* __restrict__ lx,
                                                           const T* __restrict__ ly, const T* __restrict__ lz,
                                                           long long ls, int lp, int lr) {
  constexpr int U = NC == 1 ? 4 : 2;
  const Grid& g = a.g;
  const int it = a.ctrl->cur - a.k_in_chunk;
  if (it % a.S != 0) return;
  const int slot = it / a.S;
  const long long bc = a.box.cells();
  const long long hidx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (hidx >= bc) return;
  const unsigned bplane = (unsigned)a.box.ny * (unsigned)a.box.nz;
  const unsigned hu = (unsigned)hidx;   // box cells < 2^31 (host check)
  const unsigned bi = hu / bplane, rem = hu - bi * bplane;
  const unsigned bj = rem / (unsigned)a.box.nz, bk = rem - bj * (unsigned)a.box.nz;
  const int i = int(bi) + a.box.x0, j = int(bj) + a.box.y0, k = int(bk) + a.box.z0;
  const int c = i * g.sx + j * g.NZ + k;
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
  bool du[NC];
  const T* lam[NC];
  if (NC == 3) {
    du[0] = upd_ex(g, i, j, k);
    du[1 % NC] = upd_ey(g, i, j, k);
    du[2 % NC] = upd_ez(g, i, j, k);
    lam[0] = lx;
    lam[1 % NC] = ly;
    lam[2 % NC] = lz;
  } else {
    du[0] = upd_ez(g, i, j, k);
    lam[0] = lz;
  }
  const int nshot = g.nshot;
  const bool last = slot + 1 >= a.nt_saved;   // E-only: E^(n+1) of the last frame is in R_saved
  const long long lc = (long long)i * lp + (long long)j * lr + k;
  const void* nbase = (EONLY && !last) ? a.E_saved : a.R_saved;
  const long long ie0 = (long long)slot * a.frame + hidx;
  const long long in0 = EONLY ? (last ? hidx : ie0 + a.frame) : ie0;
  const long long nstride = (EONLY && last) ? a.frame : a.comp_stride;   // next value of component q
  const long long tile = fp8_tile3(g, i, j, k);
  T acc_e = T(0), acc_s = T(0);
  double acc_e64 = 0.0, acc_s64 = 0.0;
  auto term = [&](int q, T lv, T eo, T sec) {
    T rhs = sec;
    if (EONLY) rhs = cbv != T(0) ? div_fixed(sec - (du[q] ? ca : T(1)) * eo, dcb) : T(0);
    const T lamx = (eo == T(0) && rhs == T(0)) ? T(0) : lv;
    const T gca = du[q] ? lamx * eo * wgt : T(0);
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
  auto load1 = [&](int sh, int q, T& l, T& e, T& n) {
    float esc = 1.0f, rsc = 1.0f;
    if (is_tiled(KIND)) {
      const long long si = (((long long)q * a.nt_saved + slot) * nshot + sh) * a.ntiles + tile;
      esc = a.e_scales[si];
      if (!EONLY) rsc = a.r_scales[si];
    }
    l = lam[q][sh * ls + lc];
    e = hist_load<T>(a.E_saved, q * a.comp_stride + ie0 + sh * bc, KIND, esc);
    n = hist_load<T>(nbase, q * nstride + in0 + sh * bc, KIND, rsc);
  };
  T la[U][NC], ea[U][NC], na[U][NC], lb[U][NC], eb[U][NC], nb[U][NC];
  const int nfull = nshot / U * U;
  auto load_batch = [&](int s0, T (&l)[U][NC], T (&e)[U][NC], T (&n)[U][NC]) {
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int q = 0; q < NC; ++q) load1(s0 + u, q, l[u][q], e[u][q], n[u][q]);
  };
  auto sum_batch = [&](const T (&l)[U][NC], const T (&e)[U][NC], const T (&n)[U][NC]) {
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int q = 0; q < NC; ++q) term(q, l[u][q], e[u][q], n[u][q]);
  };
  if (nfull > 0) load_batch(0, la, ea, na);
  for (int s0 = 0; s0 < nfull; s0 += 2 * U) {
    if (s0 + U < nfull) load_batch(s0 + U, lb, eb, nb);
    sum_batch(la, ea, na);
    if (s0 + U >= nfull) break;
    if (s0 + 2 * U < nfull) load_batch(s0 + 2 * U, la, ea, na);
    sum_batch(lb, eb, nb);
  }
  for (int sh = nfull; sh < nshot; ++sh) {
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      T l, e, n;
      load1(sh, q, l, e, n);
      term(q, l, e, n);
    }
  }
  if (!pec_ok) {
    acc_e = acc_s = T(0);
    acc_e64 = acc_s64 = 0.0;
  }
  const long long gi = ((long long)i * (g.NY - 1) + j) * (g.NZ - 1) + k;
  if (a.want_eps) {
    if (ACC64) a.g_eps64[gi] += acc_e64;
    else a.g_eps[gi] += acc_e;
  }
  if (a.want_sig) {
    if (ACC64) a.g_sig64[gi] += acc_s64;
    else a.g_sig[gi] += acc_s;
  }
}

// ---------------------------------------------------------------------------
// CPML adjoint weights (single-face form) in their own pass over the face
// cells once the streamed kernel of the half step has stored lambda:
// k3p_adj_w<T, false> after k3v_adj_e (H faces of reverse step it),
// k3p_adj_w<T, true> after k3v_adj_h (E faces of step it-1, the head of the
// next reverse step).  A weight needs only its cell's lambda, psi cotangent
// and rhs coefficient, and the streamed kernels neither read nor write these
// arrays in between, so every value equals the one formed inside the streamed
// kernels before (pml_weight_v, deepgpr_cpu.c:1430-1459, 1506-1534); the faces
// of a cell write separate arrays, so their order does not matter.  The pass
// keeps the streamed kernels free of the staging and arithmetic, which only
// the lanes in a face use (in an edge z strip 5 of 32).
// ---------------------------------------------------------------------------

// Face slabs of one field (x low, x high, y low, y high, z low, z high) with
// the other two axes whole: origin o, extents n, cumulative cell counts over
// one shot.
struct K3Faces {
  int o[6][3], n[6][3];
  unsigned cum[6];
};

// Per (field, axis): slot 1 / slot 2 weights of cell (i, j, k) from lambda
// components l1 / l2 with signs sg1 / sg2 where the slot's extent allows
// (the branches of the streamed kernels' former tails).
template <typename T, bool EF>
__global__ void __launch_bounds__(kBlock) k3p_adj_w(const __grid_constant__ TiledAdj<T> P, K3Buf<T> f, K3Geom kg,
                                                    K3Faces fs) {
  const AdjArgs<T>& a = P.a;
  const Grid& g = a.g;
  // no head after the last reverse step: read here, checked before the stores,
  // so the cell's loads do not wait for the step counter
  const bool head = !EF || a.ctrl->cur - a.k_in_chunk - 1 >= 0;
  const unsigned t = blockIdx.x * kBlock + threadIdx.x;
  if (t >= fs.cum[5]) return;
  int b = 0;
#pragma unroll
  for (int q = 0; q < 5; ++q) b += t >= fs.cum[q];
  const unsigned loc = t - (b > 0 ? fs.cum[b - 1] : 0u);
  const unsigned nz = (unsigned)fs.n[b][2], ny = (unsigned)fs.n[b][1];
  const unsigned rest = loc / nz, ri = rest / ny;
  const int k = fs.o[b][2] + int(loc - rest * nz);
  const int j = fs.o[b][1] + int(rest - ri * ny);
  const int i = fs.o[b][0] + int(ri);
  const int s = blockIdx.y, axis = b >> 1;
  const Face<T>* FF = EF ? a.eF : a.hF;
  const int plo = axis == 0 ? FF[0].p : (axis == 1 ? FF[2].p : FF[4].p);
  const int phi = axis == 0 ? FF[1].p : (axis == 1 ? FF[3].p : FF[5].p);
  const int c = axis == 0 ? i : (axis == 1 ? j : k);
  const int n = axis == 0 ? g.NX : (axis == 1 ? g.NY : g.NZ);
  int q0, q1;
  face_q<EF>(plo, phi, c, n, q0, q1);
  const int q = (b & 1) ? q1 : q0;
  const Face<T>& F = b == 0 ? FF[0] : b == 1 ? FF[1] : b == 2 ? FF[2] : b == 3 ? FF[3] : b == 4 ? FF[4] : FF[5];
  const Prof<T> pr = prof(F, q);
  const int PS = g.NY * kg.zp, cc = i * PS + j * kg.zp + k;
  const long long base = (long long)s * g.NX * PS + cc;
  const T up = EF ? f.ce_rhs[cc] : f.ch_rhs[cc];
  const T inv = axis == 0 ? a.inv_dx : (axis == 1 ? a.inv_dy : a.inv_dz);
  const bool il = i < g.NX - 1, jl = j < g.NY - 1, kl = k < g.NZ - 1;
  const T* l1;
  const T* l2;
  bool on1, on2;
  T sg1;
  if (!EF) {   // H faces: x (Hy, Hz), y (Hx, Hz), z (Hx, Hy)
    l1 = axis == 0 ? f.Hy : f.Hx;
    l2 = axis == 2 ? f.Hy : f.Hz;
    on1 = axis == 2 ? jl : kl;
    on2 = axis == 0 ? jl : il;
    sg1 = axis == 1 ? T(-1) : T(1);
  } else {     // E faces: x (Ey, Ez), y (Ex, Ez), z (Ex, Ey)
    l1 = axis == 0 ? f.Ey : f.Ex;
    l2 = axis == 2 ? f.Ey : f.Ez;
    on1 = axis == 0 ? jl : il;
    on2 = axis == 2 ? jl : kl;
    sg1 = axis == 1 ? T(1) : T(-1);
  }
  T w1 = T(0), w2 = T(0), p1 = T(0), p2 = T(0);
  int pi1 = 0, pi2 = 0;
  if (on1) {
    pi1 = cpml_at32<EF>(g, axis, 1, F.p, s, q, i, j, k);
    const T lam = l1[base], ph = F.psi1[pi1];
    w1 = (sg1 * up * pr.ra1 * lam - pr.rf * ph) * inv;   // pml_weight_v, the stores below
    p1 = sg1 * up * pr.rb * lam + pr.re * ph;
  }
  if (on2) {
    pi2 = cpml_at32<EF>(g, axis, 2, F.p, s, q, i, j, k);
    const T lam = l2[base], ph = F.psi2[pi2], sg2 = -sg1;
    w2 = (sg2 * up * pr.ra1 * lam - pr.rf * ph) * inv;
    p2 = sg2 * up * pr.rb * lam + pr.re * ph;
  }
  if (!head) return;
  if (on1) {
    F.w1[pi1] = w1;
    F.psi1[pi1] = p1;
  }
  if (on2) {
    F.w2[pi2] = w2;
    F.psi2[pi2] = p2;
  }
}

}  // namespace dg
