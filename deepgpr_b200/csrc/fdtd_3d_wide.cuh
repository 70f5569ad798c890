// fdtd_3d_wide.cuh -- FP32 3D forward half steps on 128-column warp strips.
//
// Same working copy and arithmetic as the z-streamed kernels (fdtd_3d.cuh),
// laid out for fewer instructions per cell:
//   * a warp owns 128 z columns of one (shot, y row), four per lane (one
//     16-byte access per array and row), and streams along x over a chunk of
//     planes; a CTA holds KW_WARPS neighbouring rows;
//   * x neighbours come from a register queue, y neighbours from direct loads
//     of the neighbouring rows (L1 / L2), z neighbours from the other lanes
//     by shuffles (lanes 0 .. 2R-1 also hold the R halo columns per side);
//   * every CPML face is corrected in the same pass, in the reference order
//     (x, y, z): the x faces on their planes and the y faces on their rows
//     (both uniform over the warp), the z faces through "face slots": the
//     strip's z-face cells are dealt one per lane, the derivative of a slot's
//     cell is shuffled to it, the slot runs the psi recurrence and its
//     correction term is shuffled back to the lane that owns the cell.  A
//     warp with z-face cells thus runs one recurrence per face cell instead
//     of four predicated ones per lane, and the psi rows are read and written
//     by consecutive lanes;
//   * sources, the R^n history and receivers (E half step) and the E^n
//     history (H half step) as in the z-streamed kernels.
// Every value is the reference's expression in the reference's order
// (src/DeepGPR/lib/deepgpr_cpu.c:670-1100, 1850-1875), so results equal the
// z-streamed kernels' bit for bit.  Used for R <= 2 with at most one CPML
// face per axis in reach of a cell (the single-face form, k3_cpml_single) and
// at most 64 z-face cells per strip.
#pragma once

#include "fdtd_3d.cuh"

namespace dg {

constexpr int KWW = 128;      // z columns per warp strip (four per lane)
constexpr int KW_WARPS = 4;   // warps (y rows) per CTA

struct K3WGeom {
  int zp;                          // z pitch of the working copy (multiple of 32)
  int nzs, nyt;                    // strips per row, y tiles (of KW_WARPS rows) per plane
  int xc, nchunk;                  // x chunk length, chunks
  long long nblocks;               // nshot * nzs * nyt * nchunk
  const unsigned char* src_rows;   // (nshot, NX): the plane holds a source of the shot
  const unsigned char* rcv_rows;   // (nshot, NX): the plane holds a receiver of the shot
  int lo[3], hi[3];                // E pass form: the CPML frame is c < lo or c >= hi along each axis
};

struct KwPos {
  int lane, s, j, k0, kk, x0, x1;
  bool live, lv;   // lv: the lane's four columns lie inside the row pitch
};

// block -> (shot fastest, z strip, y tile, x chunk), as k3_pos
__device__ __forceinline__ KwPos kw_pos(const K3WGeom& kg, const Grid& g) {
  KwPos p;
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
  p.j = yt * KW_WARPS + threadIdx.y;
  p.live = p.j < g.NY && chunk < kg.nchunk;
  p.k0 = zs * KWW;
  p.kk = p.k0 + 4 * p.lane;
  p.lv = p.kk < kg.zp;
  p.x0 = chunk * kg.xc;
  p.x1 = min(p.x0 + kg.xc, g.NX);
  return p;
}

// 16-byte load of the lane's four columns, zeros past the row pitch
__device__ __forceinline__ void ld4m(const float* p, bool on, float (&o)[4]) {
  float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (on) v = *reinterpret_cast<const float4*>(p);
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}

// value e (0..3, the same register index for all lanes is not required) of
// four registers
__device__ __forceinline__ float pick4(int e, float a, float b, float c, float d) {
  return e == 0 ? a : (e == 1 ? b : (e == 2 ? c : d));
}

// z-face cells of a strip [k0, k0 + 128): the low face's cells la .. la+nlo-1
// (H: k < p_lo; E: 0 < k <= p_lo), then the high face's ha .. ha+nhi-1
// (n-1-p_hi <= k < n-1, both fields).  Slot f < nlo is cell la + f, slot
// nlo + m is cell ha + m.
struct ZSlots {
  int la, nlo, ha, nhi;
  __host__ __device__ __forceinline__ int n() const { return nlo + nhi; }
  __device__ __forceinline__ int cell(int f) const { return f < nlo ? la + f : ha + (f - nlo); }
  // slot of cell k, or -1
  __device__ __forceinline__ int slot(int k) const {
    if (k >= la && k < la + nlo) return k - la;
    if (k >= ha && k < ha + nhi) return nlo + (k - ha);
    return -1;
  }
};

template <bool EFIELD>
__host__ __device__ __forceinline__ ZSlots zslots(int plo, int phi, int NZ, int k0) {
  ZSlots z;
  const int a = EFIELD ? 1 : 0, b = plo > 0 ? (EFIELD ? plo + 1 : plo) : 0;
  const int c = phi > 0 ? NZ - 1 - phi : NZ - 1, d = NZ - 1, end = k0 + KWW;
  z.la = k0 > a ? k0 : a;
  z.nlo = (b < end ? b : end) - z.la;
  z.nlo = z.nlo > 0 ? z.nlo : 0;
  z.ha = k0 > c ? k0 : c;
  z.nhi = (d < end ? d : end) - z.ha;
  z.nhi = z.nhi > 0 ? z.nhi : 0;
  return z;
}

// What a face slot needs along the x loop: its profile and psi rows.
struct ZSlotRows {
  const float* up;    // curl-rhs coefficient at plane 0 (advance i * PS)
  float* p1;          // psi1 at plane 0 (advance i * s1)
  float* p2;
  int s1, s2;
  Prof<float> pr;
  bool on;
};

template <bool EFIELD>
__device__ __forceinline__ ZSlotRows zslot_rows(const Face<float>* F, const Grid& g, const ZSlots& zs, int f, int s,
                                                int j, const float* rhs_row) {
  ZSlotRows r;
  r.on = f < zs.n();
  const int k = zs.cell(r.on ? f : 0);
  const bool lo = f < zs.nlo;
  const Face<float>& A = lo ? F[4] : F[5];
  const int q = r.on ? (lo ? (EFIELD ? q_low_e(F[4].p, k) : q_low_h(F[4].p, k)) : q_high(F[5].p, k, g.NZ)) : 0;
  const int p = lo ? F[4].p : F[5].p;
  const PsiDims d1 = EFIELD ? psi_dims_e(g, 2, 1, p) : psi_dims_h(g, 2, 1, p);
  const PsiDims d2 = EFIELD ? psi_dims_e(g, 2, 2, p) : psi_dims_h(g, 2, 2, p);
  r.p1 = (r.on ? A.psi1 : F[4].psi1) + (r.on ? psi_index(d1, 2, s, q, 0, j, 0) : 0);
  r.p2 = (r.on ? A.psi2 : F[4].psi2) + (r.on ? psi_index(d2, 2, s, q, 0, j, 0) : 0);
  r.s1 = d1.b * d1.c;
  r.s2 = d2.b * d2.c;
  r.up = rhs_row + (r.on ? k : 0);
  r.pr = r.on ? prof(A, q) : Prof<float>{0.0f, 0.0f, 0.0f, 0.0f};
  return r;
}

// Correction terms of one face slot: t1 = c (ra1 d + rb psi1) with
// d = dv1 / h, psi1 <- re psi1 - rf d (when on1), the same for slot 2
// (deepgpr_cpu.c:939-1100 order; the owner adds or subtracts t).
__device__ __forceinline__ void zslot_terms(const ZSlotRows& r, int i, float up, float ph1, float ph2, float dv1,
                                            float dv2, const FixedDiv<float>& h, bool on1, bool on2, float& t1,
                                            float& t2) {
  t1 = 0.0f;
  t2 = 0.0f;
  if (r.on && on1) {
    const float d = div_fixed(dv1, h);
    t1 = up * (r.pr.ra1 * d + r.pr.rb * ph1);
    r.p1[(long long)i * r.s1] = r.pr.re * ph1 - r.pr.rf * d;
  }
  if (r.on && on2) {
    const float d = div_fixed(dv2, h);
    t2 = up * (r.pr.ra1 * d + r.pr.rb * ph2);
    r.p2[(long long)i * r.s2] = r.pr.re * ph2 - r.pr.rf * d;
  }
}

// the value of cell (lane owner, element el) of the four-register set v, at
// every lane (owner, el per lane)
__device__ __forceinline__ float gather4(const float (&v)[4], int owner, int el) {
  const float a = __shfl_sync(kFullMask, v[0], owner), b = __shfl_sync(kFullMask, v[1], owner);
  const float c = __shfl_sync(kFullMask, v[2], owner), d = __shfl_sync(kFullMask, v[3], owner);
  return pick4(el, a, b, c, d);
}

// One batch of face slots (slots f0 .. f0 + 31, slot f0 + l at lane l): the
// slots take their cells' derivatives d1, d2 from the owner lanes, run the
// recurrences, and the owners add (PLUS) or subtract the correction terms.
// All lanes call it.
template <bool PLUS1, bool PLUS2>
__device__ __forceinline__ void zslot_batch(const ZSlotRows& zr, int i, float up, float ph1, float ph2,
                                            const float (&d1)[4], const float (&d2)[4], int own, int el,
                                            const FixedDiv<float>& h, bool on1, bool on2, const int (&zsl)[4], int f0,
                                            float (&u1)[4], float (&u2)[4]) {
  float t1, t2;
  zslot_terms(zr, i, up, ph1, ph2, gather4(d1, own, el), gather4(d2, own, el), h, on1, on2, t1, t2);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int sl = (zsl[e] - f0) & 31;
    const float v1 = __shfl_sync(kFullMask, t1, sl), v2 = __shfl_sync(kFullMask, t2, sl);
    if (zsl[e] >= f0 && zsl[e] < f0 + 32) {
      if (on1) u1[e] = PLUS1 ? u1[e] + v1 : u1[e] - v1;
      if (on2) u2[e] = PLUS2 ? u2[e] + v2 : u2[e] - v2;
    }
  }
}

// The second batch of face slots (strips with more than 32 z-face cells):
// the slot rows are formed and the operands loaded where they are used.
template <bool EFIELD, bool PLUS1, bool PLUS2>
__device__ __forceinline__ void zslot_second(const Face<float>* F, const Grid& g, const ZSlots& zs, int k0, int s,
                                             int j, int i, int o, const float* rhs_row, const float (&d1)[4],
                                             const float (&d2)[4], const FixedDiv<float>& h, bool on1, bool on2,
                                             const int (&zsl)[4], float (&u1)[4], float (&u2)[4]) {
  const int lane = threadIdx.x;
  const ZSlotRows zr = zslot_rows<EFIELD>(F, g, zs, lane + 32, s, j, rhs_row);
  const int c = zs.cell(zr.on ? lane + 32 : 0) - k0;
  float up = 0.0f, ph1 = 0.0f, ph2 = 0.0f;
  if (zr.on) {
    up = zr.up[o];
    if (on1) ph1 = zr.p1[(long long)i * zr.s1];
    if (on2) ph2 = zr.p2[(long long)i * zr.s2];
  }
  zslot_batch<PLUS1, PLUS2>(zr, i, up, ph1, ph2, d1, d2, c >> 2, c & 3, h, on1, on2, zsl, 32, u1, u2);
}

// 16-byte global -> shared copy of the lane's four columns (sm_80+ cp.async);
// with on == false nothing is read and the 16 bytes are zero-filled.  CA
// keeps the line in L1 (rows the neighbouring warps read as y neighbours).
template <bool CA>
__device__ __forceinline__ void cp16(float4* smem, const float* gmem, bool on) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int n = on ? 16 : 0;
  if constexpr (CA) asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n));
  else asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void from4(const float4& v, float (&o)[4]) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}

// Staged rows of one plane (per warp, two stages): H half step -- Ex, the
// leading Ey and Ez planes, Hx, Hy, Hz, the curl coefficient, then Ex and Ez
// of the 2R-1 neighbour rows; E half step -- Hx, the leading Hy and Hz, Ex,
// Ey, Ez, the two update coefficients, then Hx and Hz of the neighbour rows.
template <int R, bool EFIELD>
__host__ __device__ constexpr int kw_slots() {
  return (EFIELD ? 8 : 7) + 2 * (2 * R - 1);
}
template <int R, bool EFIELD>
__host__ __device__ constexpr int kw_smem_bytes() {
  return KW_WARPS * 2 * kw_slots<R, EFIELD>() * 32 * 16;
}

// Resident CTAs per SM: 12 warps (<= 168 registers a thread).
constexpr int KW_MIN_BLOCKS = 3;

// ---------------------------------------------------------------------------
// 3D H half step (+ E^n history).  EQ: dx == dy == dz.  Every plane's rows
// are staged into shared memory one plane ahead (cp.async, zero fill outside
// the grid), so a plane's loads have a whole plane of work to arrive in.
// Per plane: the y, z and x differences in turn (each neighbour set dies
// after its use), the base update, the x, y and z CPML corrections, the store.
// ---------------------------------------------------------------------------
template <int R, bool EQ>
__global__ void __launch_bounds__(32 * KW_WARPS, KW_MIN_BLOCKS) k3w_fwd_h(TiledFwd<float> P, K3Buf<float> f,
                                                                          K3WGeom kg) {
  using T = float;
  constexpr int ZLO = -(R - 1), ZHI = R + 3, NZN = ZHI - ZLO + 1;   // z neighbours of the quadruple, dfwd
  constexpr int NS = kw_slots<R, false>();
  constexpr int SEX = 0, SEY = 1, SEZ = 2, SHX = 3, SHY = 4, SHZ = 5, SCC = 6, SYX = 7, SYZ = 7 + 2 * R - 1;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const KwPos wp = kw_pos(kg, g);
  if (!wp.live) return;
  extern __shared__ float4 kw_smem[];
  float4* const sb = kw_smem + threadIdx.y * 2 * NS * 32 + threadIdx.x;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const bool lv = wp.lv;
  const int PS = NY * zp;
  const bool pml = a.has_cpml != 0;
  const int hk = halo_col4<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;
  const long long srow = (long long)s * NX * PS + j * zp;
  const long long rb = srow + kk;                  // the lane's columns, plane 0
  const long long rs = lv ? rb : srow;             // the same, kept inside the row (copy sources)
  const int rowc = lv ? row : j * zp;              // coefficient offset, kept inside the row
  const long long hrb = srow + (hok ? hk : 0);     // the lane's halo column, plane 0
  bool kv[4], hxz[4], hzz[4], onk[4];
  int zsl[4];   // face slot of the lane's cells (-1: none)
  T tz[4][R], ty[R];
  ZSlots zs{0, 0, 0, 0};
  if (pml) zs = zslots<false>(a.hF[4].p, a.hF[5].p, NZ, wp.k0);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kk + e;
    kv[e] = k < NZ;
    hxz[e] = k < NZ - 1;
    hzz[e] = NZ - 1 != 1 && k > 0 && k < NZ - 1;
    onk[e] = kv[e] && k < NZ - 1;
    zsl[e] = (pml && kv[e]) ? zs.slot(k) : -1;
    taps_fwd<T, R>(k, NZ, tz[e]);
  }
  taps_fwd<T, R>(j, NY, ty);
  const bool hxy = j < NY - 1, hyy = NY - 1 != 1 && j > 0 && j < NY - 1, jl = j < NY - 1;
  const int qy0 = pml ? q_low_h(a.hF[2].p, j) : -1;
  const int qy1 = pml ? q_high(a.hF[3].p, j, NY) : -1;
  const bool in_y = qy0 >= 0 || qy1 >= 0;
  const int nsl = zs.n();   // face slots of the strip (uniform), <= 64
  const ZSlotRows zr0 = zslot_rows<false>(a.hF, g, zs, lane, s, j, f.ch_rhs + j * zp);
  const int c0l = zs.cell(zr0.on ? lane : 0) - wp.k0, own0 = c0l >> 2, el0 = c0l & 3;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save = a.save_e && (it % a.S == 0);

  T qEy[2 * R][4], qEz[2 * R][4];   // Ey, Ez at planes i-R+1 .. i+R
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = wp.x0 - R + 1 + m;
    const bool in = pl >= 0 && pl < NX;
    ld4m(f.Ey + rs + (in ? pl : 0) * PS, in && lv, qEy[m]);
    ld4m(f.Ez + rs + (in ? pl : 0) * PS, in && lv, qEz[m]);
  }
  // plane i into stage b; halo columns and face-slot operands into registers
  T nhEx = 0.0f, nhEy = 0.0f, nzu = 0.0f, nz1 = 0.0f, nz2 = 0.0f;
  auto stage = [&](int i, int b) {
    const int o = i * PS;
    float4* d = sb + b * NS * 32;
    const bool lead = i + R < NX;
    cp16<true>(d + SEX * 32, f.Ex + rs + o, lv);
    cp16<true>(d + SEY * 32, f.Ey + rs + o + (lead ? R * PS : 0), lead && lv);
    cp16<true>(d + SEZ * 32, f.Ez + rs + o + (lead ? R * PS : 0), lead && lv);
    cp16<false>(d + SHX * 32, f.Hx + rs + o, lv);
    cp16<false>(d + SHY * 32, f.Hy + rs + o, lv);
    cp16<false>(d + SHZ * 32, f.Hz + rs + o, lv);
    cp16<false>(d + SCC * 32, f.ch_curl + rowc + o, lv);
#pragma unroll
    for (int dd = -(R - 1); dd <= R; ++dd) {
      if (dd == 0) continue;
      const int m = dd < 0 ? dd + R - 1 : dd + R - 2;
      const bool in = j + dd >= 0 && j + dd < NY;
      cp16<true>(d + (SYX + m) * 32, f.Ex + rs + o + (in ? dd * zp : 0), in && lv);
      cp16<true>(d + (SYZ + m) * 32, f.Ez + rs + o + (in ? dd * zp : 0), in && lv);
    }
    cp_async_commit();
    if (hok) {
      nhEx = f.Ex[hrb + o];
      nhEy = f.Ey[hrb + o];
    }
    // face slots (psi1 exists on rows j < NY-1, psi2 on planes i < NX-1)
    if (nsl > 0 && zr0.on) {
      nzu = zr0.up[o];
      if (jl) nz1 = zr0.p1[(long long)i * zr0.s1];
      if (i < NX - 1) nz2 = zr0.p2[(long long)i * zr0.s2];
    }
  };
  stage(wp.x0, 0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    const T hEx = nhEx, hEy = nhEy, zu = nzu, z1 = nz1, z2 = nz2;
    const int b = (i - wp.x0) & 1;
    if (i + 1 < wp.x1) stage(i + 1, b ^ 1);
    else cp_async_commit();
    cp_async_wait_prev();   // this plane's rows (this lane's own copies) have landed
    const float4* cur = sb + b * NS * 32;
    const int o = i * PS;
    T ex[4];
    from4(cur[SEX * 32], ex);
    from4(cur[SEY * 32], qEy[2 * R - 1]);
    from4(cur[SEZ * 32], qEz[2 * R - 1]);
    if (save) {
      const int slot = it / a.S;
      const int bi = i - a.box.x0;
      const bool rin = j - a.box.y0 >= 0 && j - a.box.y0 < a.box.ny && bi >= 0 && bi < a.box.nx;
      bool ib[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) ib[e] = rin && kv[e] && kk + e - a.box.z0 >= 0 && kk + e - a.box.z0 < a.box.nz;
      const long long hoff = slot * a.frame + s * a.box.cells() + (long long)bi * a.box.ny * a.box.nz +
                             (long long)(j - a.box.y0) * a.box.nz + (kk - a.box.z0);
      const int ncomp = a.mode == 3 ? 3 : 1;
      with_hist_kind(a.kind, [&](auto K) {
        constexpr int KIND = decltype(K)::value;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (q >= ncomp) break;
          const int fc = a.mode == 3 ? q : 2;
          T v[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) v[e] = fc == 0 ? ex[e] : (fc == 1 ? qEy[R - 1][e] : qEz[R - 1][e]);
          float inv = 1.0f;
          if (is_tiled(KIND)) {
            float am = 0.0f;
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (ib[e]) am = fmaxf(am, fabsf(v[e]));
            const float sc = tile_scale_of(KIND, tile8_absmax(am));
            inv = 1.0f / sc;
            if ((lane & 7) == 0 && kk < NZ)
              a.e_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j, kk)] = sc;
          }
          const long long hq = q * a.comp_stride + hoff;
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (ib[e]) hist_store<T>(a.E_saved, hq + e, v[e], KIND, inv);
        }
      });
    }
    // y differences (Ex, Ez of the neighbour rows j + d)
    T dEz_dy[4], dEx_dy[4];
    {
      T exy[2 * R][4], ezy[2 * R][4];
#pragma unroll
      for (int dd = -(R - 1); dd <= R; ++dd) {
        if (dd == 0) continue;
        const int m = dd < 0 ? dd + R - 1 : dd + R - 2;
        from4(cur[(SYX + m) * 32], exy[dd + R - 1]);
        from4(cur[(SYZ + m) * 32], ezy[dd + R - 1]);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        dEz_dy[e] = dfwd_t<T, R>([&](int d) { return d == 0 ? qEz[R - 1][e] : ezy[d + R - 1][e]; }, ty);
        dEx_dy[e] = dfwd_t<T, R>([&](int d) { return d == 0 ? ex[e] : exy[d + R - 1][e]; }, ty);
      }
    }
    // z differences (Ex, Ey at columns kk + m)
    T dEy_dz[4], dEx_dz[4];
    {
      T zx[NZN], zy[NZN];
#pragma unroll
      for (int m = ZLO; m <= ZHI; ++m) {
        zx[m - ZLO] = ynb4<T, R>(ex, hEx, lane, m);
        zy[m - ZLO] = ynb4<T, R>(qEy[R - 1], hEy, lane, m);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        dEy_dz[e] = dfwd_t<T, R>([&](int d) { return zy[e + d - ZLO]; }, tz[e]);
        dEx_dz[e] = dfwd_t<T, R>([&](int d) { return zx[e + d - ZLO]; }, tz[e]);
      }
    }
    // x differences and the base update
    T tx[R];
    taps_fwd<T, R>(i, NX, tx);
    const bool hxx = NX - 1 != 1 && i > 0 && i < NX - 1, hyx = i < NX - 1, il = i < NX - 1;
    T hx[4], hy[4], hz[4], c1[4], dEz_dx[4], dEy_dx[4];
    from4(cur[SHX * 32], hx);
    from4(cur[SHY * 32], hy);
    from4(cur[SHZ * 32], hz);
    from4(cur[SCC * 32], c1);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      dEz_dx[e] = dfwd_t<T, R>([&](int d) { return qEz[R - 1 + d][e]; }, tx);
      dEy_dx[e] = dfwd_t<T, R>([&](int d) { return qEy[R - 1 + d][e]; }, tx);
      const T cx = c1[e];
      const T cyv = (EQ || a.dy_eq) ? cx : div_fixed(cx * a.dx, a.ddy);
      const T czv = (EQ || a.dz_eq) ? cx : div_fixed(cx * a.dx, a.ddz);
      if (hxx && hxy && hxz[e]) hx[e] = hx[e] - cyv * dEz_dy[e] + czv * dEy_dz[e];
      if (hyx && hyy && hxz[e]) hy[e] = hy[e] - czv * dEx_dz[e] + cx * dEz_dx[e];
      if (hyx && hxy && hzz[e]) hz[e] = hz[e] - cx * dEy_dx[e] + cyv * dEx_dy[e];
    }
    // CPML corrections in the reference order x, y, z
    const int qx0 = pml ? q_low_h(a.hF[0].p, i) : -1;
    const int qx1 = pml ? q_high(a.hF[1].p, i, NX) : -1;
    const bool in_x = qx0 >= 0 || qx1 >= 0;
    if (in_x || in_y) {
      T up[4];
      ld4m(f.ch_rhs + rowc + o, lv, up);
      if (in_x) {
        long long bx1, bx2;
        const int fx = xface_at<T, false>(a.hF, g, s, i, j, bx1, bx2);
        const Prof<T> pr = fx == 0 ? prof(a.hF[0], qx0) : prof(a.hF[1], qx1);
        T* X1 = fx == 0 ? a.hF[0].psi1 : a.hF[1].psi1;
        T* X2 = fx == 0 ? a.hF[0].psi2 : a.hF[1].psi2;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (onk[e]) cpml_one<T>(X1, bx1 + kk + e, X1[bx1 + kk + e], pr, dEz_dx[e], a.ddx, up[e], true, hy[e]);
          if (kv[e] && jl) cpml_one<T>(X2, bx2 + kk + e, X2[bx2 + kk + e], pr, dEy_dx[e], a.ddx, up[e], false, hz[e]);
        }
      }
      if (in_y) {
        const FaceRows<T> yr = face_rows<T, false>(a.hF[2], a.hF[3], qy0 >= 0, g, 1, s, 0, qy0 >= 0 ? qy0 : qy1);
        const Prof<T> pr = qy0 >= 0 ? prof(a.hF[2], qy0) : prof(a.hF[3], qy1);
        const long long b1 = (long long)i * yr.s1 + kk, b2 = (long long)i * yr.s2 + kk;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (onk[e]) cpml_one<T>(yr.p1, b1 + e, yr.p1[b1 + e], pr, dEz_dy[e], a.ddy, up[e], false, hx[e]);
          if (kv[e] && il) cpml_one<T>(yr.p2, b2 + e, yr.p2[b2 + e], pr, dEx_dy[e], a.ddy, up[e], true, hz[e]);
        }
      }
    }
    if (nsl > 0) {
      // z faces: hx += t1 (psi1, dEy/dz; rows j < NY-1), hy -= t2 (psi2, dEx/dz; planes i < NX-1)
      zslot_batch<true, false>(zr0, i, zu, z1, z2, dEy_dz, dEx_dz, own0, el0, a.ddz, jl, il, zsl, 0, hx, hy);
      if (nsl > 32)
        zslot_second<false, true, false>(a.hF, g, zs, wp.k0, s, j, i, o, f.ch_rhs + j * zp, dEy_dz, dEx_dz, a.ddz, jl,
                                         il, zsl, hx, hy);
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
        qEy[m][e] = qEy[m + 1][e];
        qEz[m][e] = qEz[m + 1][e];
      }
  }
}

// ---------------------------------------------------------------------------
// 3D E half step (+ sources, R^n history, receivers), same staging and order.
// PASS: every cell gets its base update here and the CPML frame (corrections,
// then the frame cells' sources and receivers) is finished by k3p_fwd_e right
// after (no R^n history in that form: R^n needs E^n, overwritten here).
// ---------------------------------------------------------------------------
template <int R, bool EQ, bool PASS>
__global__ void __launch_bounds__(32 * KW_WARPS, KW_MIN_BLOCKS) k3w_fwd_e(TiledFwd<float> P, K3Buf<float> f,
                                                                          K3WGeom kg) {
  using T = float;
  constexpr int ZLO = -R, ZHI = R + 2, NZN = ZHI - ZLO + 1;   // z neighbours of the quadruple, dback
  constexpr int NS = kw_slots<R, true>();
  constexpr int SHX = 0, SHY = 1, SHZ = 2, SEX = 3, SEY = 4, SEZ = 5, SC0 = 6, SC1 = 7, SYX = 8, SYZ = 8 + 2 * R - 1;
  const FwdArgs<T>& a = P.a;
  const Grid& g = a.g;
  const KwPos wp = kw_pos(kg, g);
  if (!wp.live) return;
  extern __shared__ float4 kw_smem[];
  float4* const sb = kw_smem + threadIdx.y * 2 * NS * 32 + threadIdx.x;
  const int NX = g.NX, NY = g.NY, NZ = g.NZ, zp = kg.zp, lane = wp.lane, s = wp.s, j = wp.j, kk = wp.kk;
  const bool lv = wp.lv;
  const int PS = NY * zp;
  const int hk = halo_col4<R>(wp.k0, lane);
  const bool hok = lane < 2 * R && hk >= 0 && hk < NZ;
  const int row = j * zp + kk;
  const long long srow = (long long)s * NX * PS + j * zp;
  const long long rb = srow + kk;
  const long long rs = lv ? rb : srow;
  const int rowc = lv ? row : j * zp;
  const long long hrb = srow + (hok ? hk : 0);
  const bool pml = !PASS && a.has_cpml != 0;   // CPML corrected in this kernel
  // PASS: cells of the CPML frame leave their points to the frame pass
  const bool yfin = PASS && (j < kg.lo[1] || j >= kg.hi[1]);
  bool zfin[4];
  bool kv[4], exz[4], ezz[4], onk[4];
  int zsl[4];
  T tz[4][R], ty[R];
  ZSlots zs{0, 0, 0, 0};
  if (pml) zs = zslots<true>(a.eF[4].p, a.eF[5].p, NZ, wp.k0);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kk + e;
    kv[e] = k < NZ;
    exz[e] = k > 0 && k < NZ - 1;
    ezz[e] = k < NZ - 1;
    onk[e] = kv[e] && k < NZ - 1;
    zsl[e] = (pml && kv[e]) ? zs.slot(k) : -1;
    zfin[e] = PASS && (k < kg.lo[2] || k >= kg.hi[2]);
    taps_back<T, R>(k, NZ, tz[e]);
  }
  taps_back<T, R>(j, NY, ty);
  const bool exy = j > 0 && j < NY - 1, eyy = j < NY - 1, jl = j < NY - 1;
  const int qy0 = (pml && j > 0) ? q_low_e(a.eF[2].p, j) : -1;
  const int qy1 = (pml && j > 0) ? q_high(a.eF[3].p, j, NY) : -1;
  const bool in_y = qy0 >= 0 || qy1 >= 0;
  const bool degx = NY - 1 != 1 || NZ - 1 != 1, degy = NX - 1 != 1 || NZ - 1 != 1, degz = NX - 1 != 1 || NY - 1 != 1;
  const int nsl = zs.n();
  const ZSlotRows zr0 = zslot_rows<true>(a.eF, g, zs, lane, s, j, f.ce_rhs + j * zp);
  const int c0l = zs.cell(zr0.on ? lane : 0) - wp.k0, own0 = c0l >> 2, el0 = c0l & 3;
  const int it = a.ctrl->cur + a.k_in_chunk;
  const bool save_r = a.keep_r && (it % a.S == 0);

  T qHy[2 * R][4], qHz[2 * R][4];   // Hy, Hz at planes i-R .. i+R-1
#pragma unroll
  for (int m = 0; m < 2 * R - 1; ++m) {
    const int pl = wp.x0 - R + m;
    const bool in = pl >= 0 && pl < NX;
    ld4m(f.Hy + rs + (in ? pl : 0) * PS, in && lv, qHy[m]);
    ld4m(f.Hz + rs + (in ? pl : 0) * PS, in && lv, qHz[m]);
  }
  T nhHx = 0.0f, nhHy = 0.0f, nzu = 0.0f, nz1 = 0.0f, nz2 = 0.0f;
  auto stage = [&](int i, int b) {
    const int o = i * PS;
    float4* d = sb + b * NS * 32;
    const bool lead = i + R - 1 < NX;
    cp16<true>(d + SHX * 32, f.Hx + rs + o, lv);
    cp16<true>(d + SHY * 32, f.Hy + rs + o + (lead ? (R - 1) * PS : 0), lead && lv);
    cp16<true>(d + SHZ * 32, f.Hz + rs + o + (lead ? (R - 1) * PS : 0), lead && lv);
    cp16<false>(d + SEX * 32, f.Ex + rs + o, lv);
    cp16<false>(d + SEY * 32, f.Ey + rs + o, lv);
    cp16<false>(d + SEZ * 32, f.Ez + rs + o, lv);
    cp16<false>(d + SC0 * 32, f.ce_hist + rowc + o, lv);
    cp16<false>(d + SC1 * 32, f.ce_curl + rowc + o, lv);
#pragma unroll
    for (int dd = -R; dd <= R - 1; ++dd) {
      if (dd == 0) continue;
      const int m = dd < 0 ? dd + R : dd + R - 1;
      const bool in = j + dd >= 0 && j + dd < NY;
      cp16<true>(d + (SYX + m) * 32, f.Hx + rs + o + (in ? dd * zp : 0), in && lv);
      cp16<true>(d + (SYZ + m) * 32, f.Hz + rs + o + (in ? dd * zp : 0), in && lv);
    }
    cp_async_commit();
    if (hok) {
      nhHx = f.Hx[hrb + o];
      nhHy = f.Hy[hrb + o];
    }
    // face slots (psi1 exists on planes i < NX-1, psi2 on rows j < NY-1)
    if (nsl > 0 && zr0.on) {
      nzu = zr0.up[o];
      if (i < NX - 1) nz1 = zr0.p1[(long long)i * zr0.s1];
      if (jl) nz2 = zr0.p2[(long long)i * zr0.s2];
    }
  };
  stage(wp.x0, 0);
  for (int i = wp.x0; i < wp.x1; ++i) {
    const T hHx = nhHx, hHy = nhHy, zu = nzu, z1 = nz1, z2 = nz2;
    const int b = (i - wp.x0) & 1;
    if (i + 1 < wp.x1) stage(i + 1, b ^ 1);
    else cp_async_commit();
    cp_async_wait_prev();
    const float4* cur = sb + b * NS * 32;
    const int o = i * PS;
    T hxo[4];
    from4(cur[SHX * 32], hxo);
    from4(cur[SHY * 32], qHy[2 * R - 1]);
    from4(cur[SHZ * 32], qHz[2 * R - 1]);
    const bool exx = i < NX - 1, eyx = i > 0 && i < NX - 1, il = i < NX - 1;
    const int qx0 = (pml && i > 0) ? q_low_e(a.eF[0].p, i) : -1;
    const int qx1 = (pml && i > 0) ? q_high(a.eF[1].p, i, NX) : -1;
    const bool in_x = qx0 >= 0 || qx1 >= 0;
    const bool pts = (kg.src_rows && kg.src_rows[(long long)s * NX + i]) ||
                     (kg.rcv_rows && kg.rcv_rows[(long long)s * NX + i]);
    const bool xfin = yfin || (PASS && (i < kg.lo[0] || i >= kg.hi[0]));
    // y differences (Hx, Hz of the neighbour rows j + d, d = -R .. R-1)
    T dHz_dy[4], dHx_dy[4];
    {
      T hxy[2 * R][4], hzy[2 * R][4];
#pragma unroll
      for (int dd = -R; dd <= R - 1; ++dd) {
        if (dd == 0) continue;
        const int m = dd < 0 ? dd + R : dd + R - 1;
        from4(cur[(SYX + m) * 32], hxy[dd + R]);
        from4(cur[(SYZ + m) * 32], hzy[dd + R]);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        dHz_dy[e] = dback_t<T, R>([&](int d) { return d == 0 ? qHz[R][e] : hzy[d + R][e]; }, ty);
        dHx_dy[e] = dback_t<T, R>([&](int d) { return d == 0 ? hxo[e] : hxy[d + R][e]; }, ty);
      }
    }
    // z differences (Hx, Hy at columns kk + m)
    T dHy_dz[4], dHx_dz[4];
    {
      T zx[NZN], zy[NZN];
#pragma unroll
      for (int m = ZLO; m <= ZHI; ++m) {
        zx[m - ZLO] = ynb4<T, R>(hxo, hHx, lane, m);
        zy[m - ZLO] = ynb4<T, R>(qHy[R], hHy, lane, m);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        dHy_dz[e] = dback_t<T, R>([&](int d) { return zy[e + d - ZLO]; }, tz[e]);
        dHx_dz[e] = dback_t<T, R>([&](int d) { return zx[e + d - ZLO]; }, tz[e]);
      }
    }
    T tx[R];
    taps_back<T, R>(i, NX, tx);
    T ex[4], ey[4], ez[4], c0[4], c1[4], dHz_dx[4], dHy_dx[4];
    from4(cur[SEX * 32], ex);
    from4(cur[SEY * 32], ey);
    from4(cur[SEZ * 32], ez);
    from4(cur[SC0 * 32], c0);
    from4(cur[SC1 * 32], c1);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      dHz_dx[e] = dback_t<T, R>([&](int d) { return qHz[R + d][e]; }, tx);
      dHy_dx[e] = dback_t<T, R>([&](int d) { return qHy[R + d][e]; }, tx);
      const T cx = c1[e];
      const T cy = (EQ || a.dy_eq) ? cx : div_fixed(cx * a.dx, a.ddy);
      const T cz = (EQ || a.dz_eq) ? cx : div_fixed(cx * a.dx, a.ddz);
      if (degx && exx && exy && exz[e]) ex[e] = c0[e] * ex[e] + cy * dHz_dy[e] - cz * dHy_dz[e];
      if (degy && eyx && eyy && exz[e]) ey[e] = c0[e] * ey[e] + cz * dHx_dz[e] - cx * dHz_dx[e];
      if (degz && eyx && exy && ezz[e]) ez[e] = c0[e] * ez[e] + cx * dHy_dx[e] - cy * dHx_dy[e];
    }
    // the curl-rhs coefficient (CPML, sources, R^n)
    T cb[4];
    if (save_r || in_x || in_y || pts) ld4m(f.ce_rhs + rowc + o, lv, cb);
    else cb[0] = cb[1] = cb[2] = cb[3] = 0.0f;
    // CPML corrections in the reference order x, y, z
    if (in_x) {
      long long bx1, bx2;
      const int fx = xface_at<T, true>(a.eF, g, s, i, j, bx1, bx2);
      const Prof<T> pr = fx == 0 ? prof(a.eF[0], qx0) : prof(a.eF[1], qx1);
      T* X1 = fx == 0 ? a.eF[0].psi1 : a.eF[1].psi1;
      T* X2 = fx == 0 ? a.eF[0].psi2 : a.eF[1].psi2;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (kv[e] && jl) cpml_one<T>(X1, bx1 + kk + e, X1[bx1 + kk + e], pr, dHz_dx[e], a.ddx, cb[e], false, ey[e]);
        if (onk[e]) cpml_one<T>(X2, bx2 + kk + e, X2[bx2 + kk + e], pr, dHy_dx[e], a.ddx, cb[e], true, ez[e]);
      }
    }
    if (in_y) {
      const FaceRows<T> yr = face_rows<T, true>(a.eF[2], a.eF[3], qy0 >= 0, g, 1, s, 0, qy0 >= 0 ? qy0 : qy1);
      const Prof<T> pr = qy0 >= 0 ? prof(a.eF[2], qy0) : prof(a.eF[3], qy1);
      const long long b1 = (long long)i * yr.s1 + kk, b2 = (long long)i * yr.s2 + kk;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (kv[e] && il) cpml_one<T>(yr.p1, b1 + e, yr.p1[b1 + e], pr, dHz_dy[e], a.ddy, cb[e], true, ex[e]);
        if (onk[e]) cpml_one<T>(yr.p2, b2 + e, yr.p2[b2 + e], pr, dHx_dy[e], a.ddy, cb[e], false, ez[e]);
      }
    }
    if (nsl > 0) {
      // z faces: ex -= t1 (psi1, dHy/dz; planes i < NX-1), ey += t2 (psi2, dHx/dz; rows j < NY-1)
      zslot_batch<false, true>(zr0, i, zu, z1, z2, dHy_dz, dHx_dz, own0, el0, a.ddz, il, jl, zsl, 0, ex, ey);
      if (nsl > 32)
        zslot_second<true, false, true>(a.eF, g, zs, wp.k0, s, j, i, o, f.ce_rhs + j * zp, dHy_dz, dHx_dz, a.ddz, il,
                                        jl, zsl, ex, ey);
    }
    if (pts) {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (kv[e] && !xfin && !zfin[e]) inject_at(P, s, (i * NY + j) * NZ + kk + e, it, cb[e], ex[e], ey[e], ez[e]);
    }
    if (save_r) {
      const int slot = it / a.S;
      const int bi = i - a.box.x0;
      const bool rin = j - a.box.y0 >= 0 && j - a.box.y0 < a.box.ny && bi >= 0 && bi < a.box.nx;
      bool ib[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) ib[e] = rin && kv[e] && kk + e - a.box.z0 >= 0 && kk + e - a.box.z0 < a.box.nz;
      const long long hoff = slot * a.frame + s * a.box.cells() + (long long)bi * a.box.ny * a.box.nz +
                             (long long)(j - a.box.y0) * a.box.nz + (kk - a.box.z0);
      const int ncomp = a.mode == 3 ? 3 : 1;
      // E^n of the cells, still in the stage
      T ox[4], oy[4], oz[4];
      from4(cur[SEX * 32], ox);
      from4(cur[SEY * 32], oy);
      from4(cur[SEZ * 32], oz);
      with_hist_kind(a.kind, [&](auto K) {
        constexpr int KIND = decltype(K)::value;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (q >= ncomp) break;
          const int fc = a.mode == 3 ? q : 2;
          T rv[4];
          float am = 0.0f;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            rv[e] = 0.0f;
            if (ib[e]) {
              // R^n = (E^{n+1} - a_eff E^n) / cb (deepgpr_cpu.c:1850-1875)
              const T en = fc == 0 ? ex[e] : (fc == 1 ? ey[e] : ez[e]);
              const T eo = fc == 0 ? ox[e] : (fc == 1 ? oy[e] : oz[e]);
              const bool du = fc == 0 ? (degx && exx && exy && exz[e])
                                      : (fc == 1 ? (degy && eyx && eyy && exz[e]) : (degz && eyx && exy && ezz[e]));
              const T aeff = du ? c0[e] : 1.0f;
              rv[e] = cb[e] != 0.0f ? (en - aeff * eo) / cb[e] : 0.0f;
              am = fmaxf(am, fabsf(rv[e]));
            }
          }
          float inv = 1.0f;
          if (is_tiled(KIND)) {
            const float sc = tile_scale_of(KIND, tile8_absmax(am));
            inv = 1.0f / sc;
            if ((lane & 7) == 0 && kk < NZ)
              a.r_scales[(((long long)q * a.nt_saved + slot) * g.nshot + s) * a.ntiles + fp8_tile3(g, i, j, kk)] = sc;
          }
          const long long hq = q * a.comp_stride + hoff;
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (ib[e]) hist_store<T>(a.R_saved, hq + e, rv[e], KIND, inv);
        }
      });
    }
    if (pts) {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (kv[e] && !xfin && !zfin[e]) sample_at(P, s, (i * NY + j) * NZ + kk + e, it, ex[e], ey[e], ez[e]);
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
        qHy[m][e] = qHy[m + 1][e];
        qHz[m][e] = qHz[m + 1][e];
      }
  }
}

}  // namespace dg
