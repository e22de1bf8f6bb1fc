// General sparse solves for the reference's second plugin point,
// matrix_solver(A, b, **opts) -> x (meanas/fdfd/solvers.py:97-103,134), where A is the
// assembled CSR operator (the symmetrised e_full of generic(), or any other operator a
// caller builds, e.g. from eh_full / h_full).  Complex128 CSR, 32-bit column indices,
// 64-bit row pointers.
//
// SpMV: a group of LPR lanes per row walks the row's nonzeros and reduces with warp
// shuffles; every warp handles 32 / LPR consecutive rows per step, so all lanes of a warp
// run the same number of steps (the shuffles need whole warps).
//
// BiCGSTAB (complex, hashed shadow vector as in the stencil solver), three kernels per
// iteration, the direction update and s = r - alpha v folded into the gathers of the two
// products:
//   CA: p = r + beta (p_old - omega v_old) on the own row, v = A p gathered with the same
//       formula at the columns (ping-pong p / v buffers), sigma = (rh, v)      -> alpha
//   CB: s = r - alpha v on the own row, t = A s gathered likewise, (t, s), |t|^2, |s|^2 -> omega
//   CC: x += alpha p + omega s, r = s - omega t, (rh, r), |r|^2                  -> beta
// Reductions are the deterministic grid reductions of the stencil engine; the scalars
// (rho, alpha, omega, beta) stay in FP64 device state.
#pragma once
#include "fdfd_ops.cuh"

namespace fdfd {

struct CsrView {
  int n;
  const long long* indptr;
  const int* indices;
  const cx<double>* data;
};

constexpr int CSR_LPR = 4;    // lanes per row
constexpr int CSR_NT = 256;   // threads per CTA

// Row loop shared by the CSR kernels: calls f(row, lane_in_group, valid) for each step.
template <class F>
__device__ __forceinline__ void csr_rows(int n, F&& f) {
  constexpr int RPW = 32 / CSR_LPR;  // rows per warp per step
  const int lane = threadIdx.x & 31, g = lane / CSR_LPR, l = lane % CSR_LPR;
  const int warp = (blockIdx.x * CSR_NT + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * CSR_NT) >> 5;
  for (long long base = (long long)warp * RPW; base < n; base += (long long)nwarps * RPW) {
    const long long row = base + g;
    f((int)row, l, row < n);
  }
}

// sum over the row of A[row, j] * xf(j), reduced over the lane group (valid in every lane)
template <class XF>
__device__ __forceinline__ cx<double> csr_row(const CsrView& A, int row, int l, bool valid, XF&& xf) {
  cx<double> acc = czero<double>();
  if (valid) {
    const long long e1 = A.indptr[row + 1];
    for (long long e = A.indptr[row] + l; e < e1; e += CSR_LPR) acc = acc + A.data[e] * xf(A.indices[e]);
  }
#pragma unroll
  for (int o = 1; o < CSR_LPR; o <<= 1) {
    acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
    acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
  }
  return acc;
}

// y = A x
__global__ void __launch_bounds__(CSR_NT) k_csr_spmv(CsrView A, const cx<double>* __restrict__ x,
                                                    cx<double>* __restrict__ y) {
  csr_rows(A.n, [&](int row, int l, bool valid) {
    const cx<double> v = csr_row(A, row, l, valid, [&](int j) { return x[j]; });
    if (valid && l == 0) y[row] = v;
  });
}

struct CsrBufs {
  cx<double>* P0;
  cx<double>* P1;
  cx<double>* V0;
  cx<double>* V1;
  cx<double>* r;
  cx<double>* s;
  cx<double>* t;
  cx<double>* x;
  const cx<double>* b;
};

template <int NRED, class Body, class Fin>
__device__ __forceinline__ void csr_pass(const CsrView& A, RedBuf rb, Body&& body, Fin&& fin) {
  __shared__ double shred[64];
  double acc[NRED];
#pragma unroll
  for (int r = 0; r < NRED; ++r) acc[r] = 0.0;
  csr_rows(A.n, [&](int row, int l, bool valid) { body(row, l, valid, acc); });
  double sums[NRED];
  if (grid_reduce<CSR_NT, NRED>(acc, rb, shred, sums)) fin(sums);
}

// Start: r = b - A x (x = 0 unless a guess is given), rho = (rh, r), |r|^2, |b|^2.
__global__ void __launch_bounds__(CSR_NT) k_csr_init(CsrView A, CsrBufs B, int guess, unsigned seed, KState* st,
                                                    RedBuf rb) {
  csr_pass<4>(A, rb, [&](int row, int l, bool valid, double* acc) {
    cx<double> ax = czero<double>();
    if (guess) ax = csr_row(A, row, l, valid, [&](int j) { return B.x[j]; });
    if (valid && l == 0) {
      const cx<double> bv = B.b[row];
      const cx<double> r = bv - ax;
      B.r[row] = r;
      B.P0[row] = czero<double>();
      B.V0[row] = czero<double>();
      B.P1[row] = czero<double>();
      B.V1[row] = czero<double>();
      if (!guess) B.x[row] = czero<double>();
      const cx<double> h = shadow<double>(row, seed);
      acc[0] += h.re * r.re + h.im * r.im;
      acc[1] += h.re * r.im - h.im * r.re;
      acc[2] += cabs2(r);
      acc[3] += cabs2(bv);
    }
  }, [&](const double* s) {
    st->rho = {s[0], s[1]};
    st->rr = s[2];
    st->bb = s[3];
    const double tol2 = fmax(st->rtol * st->rtol * s[3], st->atol * st->atol);
    st->tol2 = tol2;
    st->alpha = {0.0, 0.0};
    st->omega = {0.0, 0.0};
    st->beta = {0.0, 0.0};
    st->iter = 0;
    st->pending = 0;
    if (!isfinite(s[2]) || !isfinite(s[3])) st->status = ST_NONFINITE;
    else if (s[2] <= tol2) st->status = ST_CONVERGED;
    else st->status = ST_RUNNING;
  });
}

__global__ void __launch_bounds__(CSR_NT) k_csr_a(CsrView A, CsrBufs B, unsigned seed, KState* st, RedBuf rb) {
  if (ld_status(st) != ST_RUNNING) return;
  const bool odd = (__ldcg(&st->iter) & 1) != 0;
  const cx<double>* Po = odd ? B.P1 : B.P0;
  const cx<double>* Vo = odd ? B.V1 : B.V0;
  cx<double>* Pn = odd ? B.P0 : B.P1;
  cx<double>* Vn = odd ? B.V0 : B.V1;
  const dcx bd = ld_dcx(&st->beta), od = ld_dcx(&st->omega);
  const cx<double> beta = from_d<double>(bd), mbo = from_d<double>(dmul(bd, {-od.re, -od.im}));
  // p = r + beta p_old - beta omega v_old
  auto pnew = [&](int j) { return caxpy(mbo, Vo[j], caxpy(beta, Po[j], B.r[j])); };
  csr_pass<2>(A, rb, [&](int row, int l, bool valid, double* acc) {
    const cx<double> v = csr_row(A, row, l, valid, pnew);
    if (valid && l == 0) {
      Pn[row] = pnew(row);
      Vn[row] = v;
      const cx<double> h = shadow<double>(row, seed);
      acc[0] += h.re * v.re + h.im * v.im;
      acc[1] += h.re * v.im - h.im * v.re;
    }
  }, [&](const double* s) {
    const dcx sigma = {s[0], s[1]};
    if (!dfinite(sigma)) { st->status = ST_NONFINITE; return; }
    if (sigma.re == 0.0 && sigma.im == 0.0) { st->status = ST_BREAKDOWN; return; }
    st->alpha = ddiv(st->rho, sigma);
  });
}

__global__ void __launch_bounds__(CSR_NT) k_csr_b(CsrView A, CsrBufs B, KState* st, RedBuf rb) {
  if (ld_status(st) != ST_RUNNING) return;
  const bool odd = (__ldcg(&st->iter) & 1) != 0;
  const cx<double>* V = odd ? B.V0 : B.V1;  // written by this iteration's k_csr_a
  const dcx ad = ld_dcx(&st->alpha);
  const cx<double> malpha = mkc<double>(-ad.re, -ad.im);
  auto snew = [&](int j) { return caxpy(malpha, V[j], B.r[j]); };
  csr_pass<4>(A, rb, [&](int row, int l, bool valid, double* acc) {
    const cx<double> t = csr_row(A, row, l, valid, snew);
    if (valid && l == 0) {
      const cx<double> s = snew(row);
      B.s[row] = s;
      B.t[row] = t;
      acc[0] += t.re * s.re + t.im * s.im;  // (t, s) = conj(t) s
      acc[1] += t.re * s.im - t.im * s.re;
      acc[2] += cabs2(t);
      acc[3] += cabs2(s);
    }
  }, [&](const double* s) {
    if (!isfinite(s[0]) || !isfinite(s[1]) || !isfinite(s[2]) || !isfinite(s[3])) {
      st->status = ST_NONFINITE;
      return;
    }
    if (s[3] <= st->tol2 || s[2] <= 0.0) {
      // s is small enough (or t vanished): finish this iteration with omega = 0
      st->omega = {0.0, 0.0};
      st->pending = s[3] <= st->tol2 ? 2 : 3;
      return;
    }
    st->omega = {s[0] / s[2], s[1] / s[2]};
  });
}

__global__ void __launch_bounds__(CSR_NT) k_csr_c(CsrView A, CsrBufs B, unsigned seed, KState* st, RedBuf rb) {
  if (ld_status(st) != ST_RUNNING) return;
  const bool odd = (__ldcg(&st->iter) & 1) != 0;
  const cx<double>* P = odd ? B.P0 : B.P1;
  const cx<double> alpha = from_d<double>(ld_dcx(&st->alpha));
  const dcx od = ld_dcx(&st->omega);
  const cx<double> omega = from_d<double>(od), momega = mkc<double>(-od.re, -od.im);
  csr_pass<3>(A, rb, [&](int row, int l, bool valid, double* acc) {
    if (valid && l == 0) {
      const cx<double> s = B.s[row];
      B.x[row] = caxpy(omega, s, caxpy(alpha, P[row], B.x[row]));
      const cx<double> r = caxpy(momega, B.t[row], s);
      B.r[row] = r;
      const cx<double> h = shadow<double>(row, seed);
      acc[0] += h.re * r.re + h.im * r.im;
      acc[1] += h.re * r.im - h.im * r.re;
      acc[2] += cabs2(r);
    }
  }, [&](const double* s) {
    st->iter += 1;
    st->rr = s[2];
    const dcx rho_new = {s[0], s[1]};
    if (!dfinite(rho_new) || !isfinite(s[2])) { st->status = ST_NONFINITE; return; }
    if (st->pending == 2 || s[2] <= st->tol2) { st->status = ST_CONVERGED; return; }
    if (st->pending == 3) { st->status = ST_BREAKDOWN; return; }
    if (st->iter >= st->maxiter) { st->status = ST_MAXITER; return; }
    const dcx om = st->omega;
    if ((rho_new.re == 0.0 && rho_new.im == 0.0) || (om.re == 0.0 && om.im == 0.0)) {
      st->status = ST_BREAKDOWN;
      return;
    }
    st->beta = dmul(ddiv(rho_new, st->rho), ddiv(st->alpha, om));
    st->rho = rho_new;
  });
}

// |b - A x|^2 and |b|^2 (the true residual of the final iterate)
__global__ void __launch_bounds__(CSR_NT) k_csr_residual(CsrView A, const cx<double>* __restrict__ x,
                                                        const cx<double>* __restrict__ b, double* out, RedBuf rb) {
  csr_pass<2>(A, rb, [&](int row, int l, bool valid, double* acc) {
    const cx<double> ax = csr_row(A, row, l, valid, [&](int j) { return x[j]; });
    if (valid && l == 0) {
      acc[0] += cabs2(b[row] - ax);
      acc[1] += cabs2(b[row]);
    }
  }, [&](const double* s) {
    out[0] = s[0];
    out[1] = s[1];
  });
}

}  // namespace fdfd
