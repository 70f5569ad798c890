// fdtd_forward.cuh -- forward-step arguments shared by the 2D TM and 3D kernels.
//
// FwdArgs holds everything one forward time step reads: fields, update
// coefficients, CPML faces, the source / receiver point tables and the
// history layout.  Reference step order (src/DeepGPR/lib/deepgpr_cpu.c:
// 1862-1917): save E^n, update H, CPML H, update E, CPML E, inject sources,
// save R^n, sample receivers.  k_final_frame writes the closing E^nt frame of
// an E-only history.
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
