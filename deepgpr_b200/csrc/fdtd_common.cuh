// fdtd_common.cuh -- shared device code of the B200 FDTD library.
//
// Field layout (one shot): (NX, NY, NZ) with z fastest, NX = nx_ext + 1
// (Yee halo); shots are stacked slowest.  One CUDA thread owns one cell of
// the shot-independent grid and loops over the shots of its shot group, so
// material coefficients and neighbourhood indices are loaded once per cell.
//
// Numerical contract: every expression below is evaluated in the order of
// the reference CPU backend (src/DeepGPR/lib/deepgpr_cpu.c) and the library
// is compiled with -fmad=false, so FP32 results match the reference bit for
// bit wherever the reference order is followed.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <stdint.h>

#include <algorithm>

namespace dg {

constexpr int kBlock = 256;          // threads per CTA in every grid kernel
constexpr int kMaxShotGroups = 65535;

// History storage kinds (bits 0-3 of storage_type).  0-2 follow the
// reference (src/DeepGPR/config/constants.py:128-131); 4 and 5 are added here.
enum HistKind : int { kF32 = 0, kF16 = 1, kBF16 = 2, kI8 = 3, kFP8 = 4, kF64 = 5 };

// Kinds stored as one byte per value with one FP32 scale per tile: FP8 E4M3
// (value = code * scale, scale = absmax / 448) and INT8 (value = code * scale,
// code in [-127, 127] rounded to nearest, scale = absmax / 127: a uniform
// grid, so a tile's largest values keep 8 bits where E4M3 keeps 4).
__host__ __device__ constexpr bool is_tiled(int kind) { return kind == kFP8 || kind == kI8; }

// Error bits written into Control::error by device code.
enum DevError : int { kErrSourceRange = 1, kErrReceiverRange = 2 };

// Device-resident loop state.  Kernels of one time step read `cur` and add
// (forward) or subtract (adjoint) their position inside the launch chunk, so a
// captured chunk of steps can be replayed unchanged; a one-thread kernel
// advances `cur` after every chunk.
struct Control {
  int cur;
  int error;     // DevError bits
  int pad[2];
};

// Stencil taps of the staggered difference of radius `rad`
// (src/DeepGPR/lib/deepgpr_cpu.c:271-289).  T = double gives the exact
// rationals for the FP64 runs.
template <typename T>
__device__ __forceinline__ T tap(int rad, int r) {
  if (rad >= 4) {
    if (r == 1) return T(1225.0f) / T(1024.0f);
    if (r == 2) return T(-245.0f) / T(3072.0f);
    if (r == 3) return T(49.0f) / T(5120.0f);
    return T(-5.0f) / T(7168.0f);
  }
  if (rad == 3) {
    if (r == 1) return T(75.0f) / T(64.0f);
    if (r == 2) return T(-25.0f) / T(384.0f);
    return T(3.0f) / T(640.0f);
  }
  if (rad == 2) {
    if (r == 1) return T(9.0f) / T(8.0f);
    return T(-1.0f) / T(24.0f);
  }
  return T(1);
}

__device__ __forceinline__ int rad_back(int c, int n, int R) {
  int r = R;
  while (r > 1 && (c < r || c + r - 1 >= n)) --r;
  return r;
}

__device__ __forceinline__ int rad_fwd(int c, int n, int R) {
  int r = R;
  while (r > 1 && (c - r + 1 < 0 || c + r >= n)) --r;
  return r;
}

// Backward staggered difference  sum_r a_r (f[c+(r-1)] - f[c-r]); the radius
// is clamped near the ends of the axis and the taps follow the clamped radius.
template <typename T, int R>
__device__ __forceinline__ T d_back(const T* __restrict__ f, int s, int c, int n) {
  if (R == 1) return f[0] - f[-s];
  T acc = T(0);
  if (c >= R && c + R - 1 < n) {
#pragma unroll
    for (int r = 1; r <= R; ++r) acc += tap<T>(R, r) * (f[(r - 1) * s] - f[-r * s]);
    return acc;
  }
  const int rr = rad_back(c, n, R);
#pragma unroll
  for (int r = 1; r <= R; ++r)
    if (r <= rr) acc += tap<T>(rr, r) * (f[(r - 1) * s] - f[-r * s]);
  return acc;
}

// Forward staggered difference  sum_r a_r (f[c+r] - f[c-(r-1)]).
template <typename T, int R>
__device__ __forceinline__ T d_fwd(const T* __restrict__ f, int s, int c, int n) {
  if (R == 1) return f[s] - f[0];
  T acc = T(0);
  if (c - R + 1 >= 0 && c + R < n) {
#pragma unroll
    for (int r = 1; r <= R; ++r) acc += tap<T>(R, r) * (f[r * s] - f[-(r - 1) * s]);
    return acc;
  }
  const int rr = rad_fwd(c, n, R);
#pragma unroll
  for (int r = 1; r <= R; ++r)
    if (r <= rr) acc += tap<T>(rr, r) * (f[r * s] - f[-(r - 1) * s]);
  return acc;
}

// Grid description shared by all kernels.
struct Grid {
  int NX, NY, NZ;   // field extents
  int sx;           // NY * NZ
  int cells;        // NX * NY * NZ
  int nshot;
  int shots_per_group;
};

__device__ __forceinline__ void cell_ijk(const Grid& g, int c, int& i, int& j, int& k) {
  i = c / g.sx;
  int rem = c - i * g.sx;
  j = rem / g.NZ;
  k = rem - j * g.NZ;
}

// Yee components advanced by the base update (deepgpr_cpu.c:697-699, 913-915).
__device__ __forceinline__ bool upd_ex(const Grid& g, int i, int j, int k) {
  return (g.NY - 1 != 1 || g.NZ - 1 != 1) && i < g.NX - 1 && j > 0 && j < g.NY - 1 && k > 0 && k < g.NZ - 1;
}
__device__ __forceinline__ bool upd_ey(const Grid& g, int i, int j, int k) {
  return (g.NX - 1 != 1 || g.NZ - 1 != 1) && i > 0 && i < g.NX - 1 && j < g.NY - 1 && k > 0 && k < g.NZ - 1;
}
__device__ __forceinline__ bool upd_ez(const Grid& g, int i, int j, int k) {
  return (g.NX - 1 != 1 || g.NY - 1 != 1) && i > 0 && i < g.NX - 1 && j > 0 && j < g.NY - 1 && k < g.NZ - 1;
}
__device__ __forceinline__ bool upd_hx(const Grid& g, int i, int j, int k) {
  return g.NX - 1 != 1 && i > 0 && i < g.NX - 1 && j < g.NY - 1 && k < g.NZ - 1;
}
__device__ __forceinline__ bool upd_hy(const Grid& g, int i, int j, int k) {
  return g.NY - 1 != 1 && i < g.NX - 1 && j > 0 && j < g.NY - 1 && k < g.NZ - 1;
}
__device__ __forceinline__ bool upd_hz(const Grid& g, int i, int j, int k) {
  return g.NZ - 1 != 1 && i < g.NX - 1 && j < g.NY - 1 && k > 0 && k < g.NZ - 1;
}

// CPML slab position q on a face, or -1 (deepgpr_cpu.c:754-760, 965-971).
__host__ __device__ __forceinline__ int q_low_e(int p, int c) { return (p > 0 && c > 0 && c <= p) ? p - c : -1; }
__host__ __device__ __forceinline__ int q_low_h(int p, int c) { return (p > 0 && c < p) ? p - 1 - c : -1; }
__host__ __device__ __forceinline__ int q_high(int p, int c, int n) {
  return (p > 0 && c >= n - 1 - p && c < n - 1) ? c - (n - 1 - p) : -1;
}

// Index into a psi-shaped array (shot, u, v, w) with extents (a, b, c).
__device__ __forceinline__ long long at3(int a, int b, int c, int s, int u, int v, int w) {
  return (((long long)s * a + u) * b + v) * c + w;
}

// One CPML face of the E or H field.
template <typename T>
struct Face {
  const T* R;     // (4, p): RA, RB, RE, RF (src/DeepGPR/solver/pml.py:148-181)
  T* psi1;
  T* psi2;
  T* w1;          // adjoint only: CPML transposed-curl weights, psi1-shaped
  T* w2;          // adjoint only: psi2-shaped
  int p;
};

// ---------------------------------------------------------------------------
// Division by a divisor shared by many dividends, correctly rounded.
//
// The CPML recurrences divide a difference by the spacing (d = dv / h) in
// every boundary cell, the imaging condition divides by dt and the E-only
// history divides every shot's value of a cell by the cell's coefficient.
// For single precision the quotient is computed from y = RN(1/b) -- worked
// out on the host in double precision for a spacing or dt (that rounding
// cannot fall on a float rounding boundary, so y is the correctly rounded
// reciprocal), or by __frcp_rn for a per-cell divisor -- by
//   q0 = RN(a y),  q_{k+1} = RN(q_k + RN(a - b q_k) y)   (FMA),
// Markstein's correction (P. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  q0
// is within two ulps of a/b; the first correction leaves an error of a few
// 2^-23 ulp before rounding, so q1 is within one ulp; Markstein's theorem (y
// within half an ulp of 1/b, q within one ulp of a/b, a - b q exact, no
// underflow or overflow) then makes q2 = RN(a/b).  The FMA path takes
// divisors in [2^-120, 2^120] and dividends with |a| >= 2^-100 (so that
// a - b q, a multiple of about ulp(a) 2^-24, is representable) and
// 2^-100 <= |a/b| <= 2^100; zeros return a (a / b for b > 0) and every
// other dividend uses the division operator.  The exported check
// dgb_check_fixed_division compares it with the division operator over all
// 2^32 dividends of a divisor.
// ---------------------------------------------------------------------------
template <typename T>
struct FixedDiv {
  T b, y;      // divisor, RN(1 / b)
  T lo, hi;    // dividends with lo <= |a| <= hi take the FMA path (lo > hi: never)
};

template <typename T>
inline FixedDiv<T> fixed_div(T b) {
  FixedDiv<T> d;
  d.b = b;
  d.y = T(1.0 / (double)b);
  const bool ok = sizeof(T) == 4 && b >= T(0x1p-120) && b <= T(0x1p120);
  d.lo = ok ? std::max(T(0x1p-100), b * T(0x1p-100)) : T(1);
  d.hi = ok ? std::min(T(0x1p100), b * T(0x1p100)) : T(0);
  return d;
}

// The same for a divisor known only on the device and shared by several
// dividends (y from the correctly rounded reciprocal __frcp_rn).
template <typename T>
__device__ __forceinline__ FixedDiv<T> fixed_div_dev(T b) {
  FixedDiv<T> d;
  d.b = b;
  if constexpr (sizeof(T) == 4) {
    d.y = __frcp_rn(b);
    const bool ok = b >= 0x1p-120f && b <= 0x1p120f;
    d.lo = ok ? fmaxf(0x1p-100f, b * 0x1p-100f) : 1.0f;
    d.hi = ok ? fminf(0x1p100f, b * 0x1p100f) : 0.0f;
  } else {
    d.y = T(1) / b;
    d.lo = T(1);
    d.hi = T(0);
  }
  return d;
}

// The division operator out of line: a call is never evaluated
// speculatively, so the rare dividends outside the FMA range do not make
// every lane pay for a full division.
__device__ __noinline__ inline float div_operator(float a, float b) { return a / b; }

template <typename T>
__device__ __forceinline__ T div_fixed(T a, const FixedDiv<T>& d) {
  if constexpr (sizeof(T) == 4) {
    const float m = fabsf(a);
    // zeros: a / b == a for b > 0 (y > 0); the FMA path would lose the sign of -0
    if ((m >= d.lo && m <= d.hi) || (m == 0.0f && d.y > 0.0f)) {
      float q = a * d.y;
      float r = fmaf(-d.b, q, a);
      q = fmaf(r, d.y, q);
      r = fmaf(-d.b, q, a);
      q = fmaf(r, d.y, q);
      return m == 0.0f ? a : q;
    }
    return div_operator(a, d.b);
  } else {
    return a / d.b;
  }
}

template <typename T>
struct Prof {
  T ra1, rb, re, rf;
};

template <typename T>
__device__ __forceinline__ Prof<T> prof(const Face<T>& F, int q) {
  Prof<T> pr;
  pr.ra1 = F.R[q] - T(1);
  pr.rb = F.R[F.p + q];
  pr.re = F.R[2 * F.p + q];
  pr.rf = F.R[3 * F.p + q];
  return pr;
}

// psi extents per (face axis, slot) for E and H (src/DeepGPR/solver/pml.py:310-348).
struct PsiDims {
  int a, b, c;
};

__device__ __forceinline__ PsiDims psi_dims_e(const Grid& g, int axis, int slot, int p) {
  if (axis == 0) return slot == 1 ? PsiDims{p + 1, g.NY - 1, g.NZ} : PsiDims{p + 1, g.NY, g.NZ - 1};
  if (axis == 1) return slot == 1 ? PsiDims{g.NX - 1, p + 1, g.NZ} : PsiDims{g.NX, p + 1, g.NZ - 1};
  return slot == 1 ? PsiDims{g.NX - 1, g.NY, p + 1} : PsiDims{g.NX, g.NY - 1, p + 1};
}

__device__ __forceinline__ PsiDims psi_dims_h(const Grid& g, int axis, int slot, int p) {
  if (axis == 0) return slot == 1 ? PsiDims{p, g.NY, g.NZ - 1} : PsiDims{p, g.NY - 1, g.NZ};
  if (axis == 1) return slot == 1 ? PsiDims{g.NX, p, g.NZ - 1} : PsiDims{g.NX - 1, p, g.NZ};
  return slot == 1 ? PsiDims{g.NX, g.NY - 1, p} : PsiDims{g.NX - 1, g.NY, p};
}

__device__ __forceinline__ long long psi_index(PsiDims d, int axis, int s, int q, int i, int j, int k) {
  if (axis == 0) return at3(d.a, d.b, d.c, s, q, j, k);
  if (axis == 1) return at3(d.a, d.b, d.c, s, i, q, k);
  return at3(d.a, d.b, d.c, s, i, j, q);
}

// ---------------------------------------------------------------------------
// History storage.
// ---------------------------------------------------------------------------

// History box: extended grid without halo, or the physical cells only.
struct HBox {
  int x0, y0, z0, nx, ny, nz;
  __host__ __device__ long long cells() const { return (long long)nx * ny * nz; }
};

__device__ __forceinline__ bool in_box(const HBox& b, int i, int j, int k, long long& h) {
  int a = i - b.x0, bb = j - b.y0, c = k - b.z0;
  if (a < 0 || bb < 0 || c < 0 || a >= b.nx || bb >= b.ny || c >= b.nz) return false;
  h = ((long long)a * b.ny + bb) * b.nz + c;
  return true;
}

template <typename T>
__device__ __forceinline__ void hist_store(void* base, long long idx, T v, int kind, float inv_scale) {
  switch (kind) {
    case kF16: reinterpret_cast<__half*>(base)[idx] = __float2half_rn(float(v)); break;
    case kBF16: reinterpret_cast<__nv_bfloat16*>(base)[idx] = __float2bfloat16_rn(float(v)); break;
    case kFP8:
      reinterpret_cast<__nv_fp8_storage_t*>(base)[idx] =
          __nv_cvt_float_to_fp8(float(v) * inv_scale, __NV_SATFINITE, __NV_E4M3);
      break;
    case kI8:
      reinterpret_cast<signed char*>(base)[idx] =
          (signed char)max(-127, min(127, __float2int_rn(float(v) * inv_scale)));
      break;
    case kF64: reinterpret_cast<double*>(base)[idx] = double(v); break;
    default: reinterpret_cast<float*>(base)[idx] = float(v); break;
  }
}

template <typename T>
__device__ __forceinline__ T hist_load(const void* base, long long idx, int kind, float scale) {
  switch (kind) {
    case kF16: return T(__half2float(reinterpret_cast<const __half*>(base)[idx]));
    case kBF16: return T(__bfloat162float(reinterpret_cast<const __nv_bfloat16*>(base)[idx]));
    case kFP8: {
      __half_raw h = __nv_cvt_fp8_to_halfraw(reinterpret_cast<const __nv_fp8_storage_t*>(base)[idx], __NV_E4M3);
      return T(__half2float(__half(h)) * scale);
    }
    case kI8: return T(float(reinterpret_cast<const signed char*>(base)[idx]) * scale);
    case kF64: return T(reinterpret_cast<const double*>(base)[idx]);
    default: return T(reinterpret_cast<const float*>(base)[idx]);
  }
}

__host__ __device__ __forceinline__ int hist_elem_bytes(int kind) {
  return kind == kF32 ? 4 : (kind == kF64 ? 8 : (is_tiled(kind) ? 1 : 2));
}

// Block-wide maximum of non-negative values (all threads must call).
__device__ __forceinline__ float block_absmax(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    float x = lane < (blockDim.x >> 5) ? red[lane] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) red[32] = x;
  }
  __syncthreads();
  return red[32];
}

// FP8 E4M3 tile scale: stored value = x / scale, |x / scale| <= 448.  The
// floor keeps 1/scale finite for all-but-zero tiles (values below 448e-30
// are stored as 0 or subnormal FP8, far below FP32 gradient resolution).
__device__ __forceinline__ float fp8_scale_of(float absmax) { return fmaxf(absmax / 448.0f, 1e-30f); }
// Tile scale of a one-byte kind (FP8: absmax / 448; INT8: absmax / 127), same floor.
__device__ __forceinline__ float tile_scale_of(int kind, float absmax) {
  return kind == kI8 ? fmaxf(absmax / 127.0f, 1e-30f) : fp8_scale_of(absmax);
}

// ---------------------------------------------------------------------------
// Point tables (sources, receivers): unique cells sorted ascending; entries
// of one cell sorted by (shot, index) in [off[u], off[u+1]).
// ---------------------------------------------------------------------------
struct PointTable {
  const int* cells;   // unique cell indices (within one shot)
  const int* off;     // n + 1 offsets into shot/idx
  const int* shot;
  const int* idx;
  int n;
};

// Map the CTA's contiguous cell range [c0, c0 + kBlock) onto table rows:
// map[t] = row of cell c0 + t, or -1.  All threads must call.
__device__ __forceinline__ void build_block_map(const PointTable& tb, int c0, int* map) {
  map[threadIdx.x] = -1;
  __syncthreads();
  if (tb.n > 0) {
    // lower_bound of c0 and c0 + kBlock, computed by every thread (cheap, cached)
    int lo = 0, hi = tb.n;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (tb.cells[mid] < c0) lo = mid + 1; else hi = mid;
    }
    int lo2 = lo, hi2 = tb.n;
    while (lo2 < hi2) {
      int mid = (lo2 + hi2) >> 1;
      if (tb.cells[mid] < c0 + kBlock) lo2 = mid + 1; else hi2 = mid;
    }
    for (int r = lo + threadIdx.x; r < lo2; r += blockDim.x) map[tb.cells[r] - c0] = r;
  }
  __syncthreads();
}

}  // namespace dg
