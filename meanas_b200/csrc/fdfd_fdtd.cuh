// FDTD Yee updates with CPML: the time-domain stencil loop of the reference
// (meanas/fdtd/base.py:13-125, meanas/fdtd/pml.py:96-230).
//
//   H step:  H -= dt / mu * (curl_f(E) + psi terms)      (forward differences)
//   E step:  E += dt / eps * (curl_b(H) + psi terms)     (backward differences)
//
// Two forms, matching the reference's two update builders:
//   PLAIN (maxwell_h / maxwell_e): H -= dt * curl_f(E) [/ mu];  E += dt * curl_b(H) / eps,
//          forward differences over dxes[0], backward over dxes[1];
//   CPML  (updates_with_cpml):     H -= dt / mu * (curl_f(E) + pH);  E += dt / eps * (curl_b(H) + pE),
//          both difference kinds over dxes[1] (the reference builds deriv_forward(dxes[1])),
//          and on the PML slab of each face the differences along that axis are scaled by
//          p2 = 1/kappa and feed the psi recurrences  psi = p0 psi + p1 d  whose sums form pE/pH.
// Arithmetic follows the reference's numpy evaluation step by step: a difference of two
// field values in the field type, everything after it in FP64 with explicit
// round-to-nearest operations (no contraction), psi and the PML sums rounded to the psi
// type at every in-place step, the result rounded to the field type.  So the GPU
// trajectories equal the reference's bit for bit.
#pragma once
#include "fdfd_device.cuh"

namespace fdfd {

struct CpmlFace {
  int th;                 // layers (0: no PML on this face)
  const double* p;        // [3][th]: p0, p1, p2 per layer
  void* psi_u;            // psi of the first transverse component, region shape
  void* psi_v;
};

struct FdtdGeo {
  int X, Y, Z;
  int ntz, nty;
  const double* dxf[3];   // widths dividing the forward differences
  const double* dxb[3];   // widths dividing the backward differences
  const double* mat;      // epsilon (E step) or mu (H step, may be null: 1), [3N]
  double dt;
  int cpml;               // 0: PLAIN form, 1: CPML form
  CpmlFace face[3][2];    // [axis][0: low face, 1: high face]
};

__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmulr(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddivr(double a, double b) { return __ddiv_rn(a, b); }

template <typename T>
__device__ __forceinline__ T tsub(T a, T b);
template <>
__device__ __forceinline__ float tsub<float>(float a, float b) { return __fsub_rn(a, b); }
template <>
__device__ __forceinline__ double tsub<double>(double a, double b) { return __dsub_rn(a, b); }
template <typename T>
__device__ __forceinline__ T tadd(T a, T b);
template <>
__device__ __forceinline__ float tadd<float>(float a, float b) { return __fadd_rn(a, b); }
template <>
__device__ __forceinline__ double tadd<double>(double a, double b) { return __dadd_rn(a, b); }

template <typename T>
__device__ __forceinline__ T tmul(T a, T b);
template <>
__device__ __forceinline__ float tmul<float>(float a, float b) { return __fmul_rn(a, b); }
template <>
__device__ __forceinline__ double tmul<double>(double a, double b) { return __dmul_rn(a, b); }

// psi in place:  psi = P(psi * p0);  psi = P(psi + p1 * d)   (FP64 products, as numpy does
// for a psi array and FP64 parameters)
template <typename P>
__device__ __forceinline__ P psi_step(P psi, double p0, double p1, double d) {
  const P a = (P)dmulr((double)psi, p0);
  return (P)dadd((double)a, dmulr(p1, d));
}

// One half step on every cell: ESTEP updates E from H, otherwise H from E.
template <typename R, typename P, bool ESTEP>
__global__ void __launch_bounds__(256) k_fdtd(FdtdGeo g, R* __restrict__ e, R* __restrict__ h) {
  const int ntiles = g.ntz * g.nty, units = ntiles * g.X;
  const int YZ = g.Y * g.Z, N = g.X * YZ;
  for (int u = blockIdx.x; u < units; u += gridDim.x) {
    const int i = u / ntiles, t = u - i * ntiles;
    const int tyb = t / g.ntz, tzb = t - tyb * g.ntz;
    const int j = tyb * 8 + threadIdx.y, k = tzb * 32 + threadIdx.x;
    if (j >= g.Y || k >= g.Z) continue;
    const int c0 = i * YZ + j * g.Z + k;
    const int idx[3] = {i, j, k};
    // neighbour cells: -1 (E step) or +1 (H step) along each axis, periodic
    int nb[3];
    if (ESTEP) {
      nb[0] = c0 + ((i == 0 ? g.X - 1 : i - 1) - i) * YZ;
      nb[1] = c0 + ((j == 0 ? g.Y - 1 : j - 1) - j) * g.Z;
      nb[2] = c0 + ((k == 0 ? g.Z - 1 : k - 1) - k);
    } else {
      nb[0] = c0 + ((i + 1 == g.X ? 0 : i + 1) - i) * YZ;
      nb[1] = c0 + ((j + 1 == g.Y ? 0 : j + 1) - j) * g.Z;
      nb[2] = c0 + ((k + 1 == g.Z ? 0 : k + 1) - k);
    }
    const R* src = ESTEP ? h : e;
    // d[a][c]: difference along axis a of component c (only c != a is used)
    double d[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double w = ESTEP ? g.dxb[a][idx[a]] : g.dxf[a][idx[a]];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (c == a) continue;
        const R here = src[c * N + c0], there = src[c * N + nb[a]];
        const R diff = ESTEP ? tsub<R>(here, there) : tsub<R>(there, here);
        d[a][c] = ddivr((double)diff, w);
      }
    }
    P pc[3] = {P(0), P(0), P(0)};
    if (g.cpml) {
      const int dims[3] = {g.X, g.Y, g.Z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int uu = a == 0 ? 1 : 0, vv = a == 2 ? 1 : 2;
        const double se = a == 1 ? 1.0 : -1.0;
#pragma unroll
        for (int pp = 0; pp < 2; ++pp) {
          const CpmlFace& f = g.face[a][pp];
          if (f.th == 0) continue;
          const int l = pp == 0 ? idx[a] : idx[a] - (dims[a] - f.th);
          if (l < 0 || l >= f.th) continue;
          const double p0 = f.p[l], p1 = f.p[f.th + l], p2 = f.p[2 * f.th + l];
          d[a][uu] = dmulr(d[a][uu], p2);
          d[a][vv] = dmulr(d[a][vv], p2);
          // region index of this cell (region shape: th along a, full along the others)
          int ri;
          if (a == 0) ri = (l * g.Y + j) * g.Z + k;
          else if (a == 1) ri = (i * f.th + l) * g.Z + k;
          else ri = (i * g.Y + j) * f.th + l;
          P* pu = (P*)f.psi_u;
          P* pv = (P*)f.psi_v;
          const P su = psi_step<P>(pu[ri], p0, p1, d[a][vv]);  // reversed u, v, as in the reference
          const P sv = psi_step<P>(pv[ri], p0, p1, d[a][uu]);
          pu[ri] = su;
          pv[ri] = sv;
          pc[uu] = tadd<P>(pc[uu], se > 0 ? su : -su);
          pc[vv] = tadd<P>(pc[vv], se > 0 ? -sv : sv);
        }
      }
    }
    // curl components: x: d_y(.z) - d_z(.y); y: d_z(.x) - d_x(.z); z: d_x(.y) - d_y(.x)
    double curl[3];
    curl[0] = dsub(d[1][2], d[2][1]);
    curl[1] = dsub(d[2][0], d[0][2]);
    curl[2] = dsub(d[0][1], d[1][0]);
    R* dst = ESTEP ? e : h;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const R old = dst[c * N + c0];
      if (g.cpml) {
        const double coef = g.mat ? ddivr(g.dt, g.mat[c * N + c0]) : g.dt;
        const double step = dmulr(coef, dadd(curl[c], (double)pc[c]));
        dst[c * N + c0] = (R)(ESTEP ? dadd((double)old, step) : dsub((double)old, step));
      } else {
        // the PLAIN form keeps the curl in an array of the field type and scales it there
        const R st = tmul<R>((R)g.dt, (R)curl[c]);
        if (g.mat) {
          const double step = ddivr((double)st, g.mat[c * N + c0]);
          dst[c * N + c0] = (R)(ESTEP ? dadd((double)old, step) : dsub((double)old, step));
        } else {
          dst[c * N + c0] = ESTEP ? tadd<R>(old, st) : tsub<R>(old, st);
        }
      }
    }
  }
}

}  // namespace fdfd
