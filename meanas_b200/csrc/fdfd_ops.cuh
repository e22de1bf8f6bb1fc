// Loaders/epilogues plugged into the stencil and pointwise engines of fdfd_device.cuh.
//
// Krylov methods (all in the E-space, i.e. on A0 itself):
//
//  * COCG on A0 with the bilinear form <u, v> = sum(u * W * v), W = p^2 the
//    symmetriser weights of meanas/fdfd/operators.py:99-123.  With x = Pl E this
//    is exactly COCG on the symmetrised system Pl A0 Pr x = Pl b0 that
//    meanas/fdfd/solvers.py:116-134 builds (W A0 is complex symmetric), but it
//    needs no square roots and no Pl/Pr vectors.  One stencil pass per iteration
//    forms p = r + beta p_old, applies q = A0 p, applies the deferred update
//    x += alpha_old p_old and reduces p^T W q; a pointwise pass updates
//    r -= alpha q and reduces r^T W r, |r|^2 and sum |W| |r|^2.
//
//  * BiCGSTAB with a hashed pseudo-random shadow vector (no storage), used in
//    complex64 as the inner solver of the mixed-precision refinement.  Two stencil
//    passes per iteration: P (r, p, x updates + v = A0 p) and S (s = r - alpha v,
//    t = A0 s).  Hermitian shadow products keep it stable in single precision,
//    which the unconjugated bilinear form of COCG is not on PML problems.
//
//  * Refinement pass (complex128): E_new = E_old + scale * d, r = b - A0 E_new,
//    writes the scaled complex64 residual for the next inner solve.
#pragma once
#include "fdfd_device.cuh"

namespace fdfd {

enum SolveStatus : int {
  ST_RUNNING = 0,
  ST_CONVERGED = 1,
  ST_MAXITER = 2,
  ST_BREAKDOWN = 3,
  ST_NONFINITE = 4,
};

// COCG (near) breakdown: the unconjugated form r^T W r (or p^T W q) has cancelled to
// below this fraction of its magnitude bound.  Converging PML runs stay above ~1e-10.
constexpr double BREAKDOWN_RATIO = 1e-14;

// FP64 scalar state of one Krylov sequence (device memory).
struct KState {
  dcx rho, sigma, alpha, beta, omega;
  double rr;       // |r|^2 (recurrence residual)
  double rr_pc;    // sum |W| |r|^2
  double rr_w2;    // sum |W|^2 |r|^2
  double bb;       // |b|^2
  double bb_pc;    // sum |W| |b|^2
  double bb_w2;    // sum |W|^2 |b|^2
  double rtol, atol;
  double tol2;     // stop when monitored norm^2 <= tol2
  double b0b0;     // |b0|^2 of the unmasked right-hand side
  double extra[4];
  int crit;        // 0: monitor rr, 1: monitor rr_pc, 2: monitor rr_w2
  int iter, maxiter, status;
  int pending;     // an x update is still owed (deferred update)
  int stall_limit; // BiCGSTAB: stop (ST_BREAKDOWN) after this many iterations without a new
                   // best residual (0 = never)
  double best_rr;  // BiCGSTAB: best recurrence residual so far, and its iteration
  int best_iter;
  int pad2;
  double* hist;    // relative residual history (length maxiter + 1) or null
};

__device__ __forceinline__ int ld_status(const KState* st) {
  return *((volatile const int*)&st->status);
}

__device__ __forceinline__ dcx ld_dcx(const dcx* p) {
  return {__ldcg(&p->re), __ldcg(&p->im)};
}

// The norm^2 a criterion watches, for the residual and for the right-hand side.
__device__ __forceinline__ double monitored_rr(const KState* st) {
  return st->crit == 0 ? st->rr : (st->crit == 1 ? st->rr_pc : st->rr_w2);
}
__device__ __forceinline__ double monitored_bb(const KState* st) {
  return st->crit == 0 ? st->bb : (st->crit == 1 ? st->bb_pc : st->bb_w2);
}

__device__ __forceinline__ void check_progress(KState* st, double monitored, bool finite_ok) {
  const double bbm = monitored_bb(st);
  const double rel = bbm > 0 ? sqrt(monitored / bbm) : 0.0;
  if (st->hist) st->hist[st->iter] = rel;
  if (!finite_ok || !isfinite(monitored)) {
    st->status = ST_NONFINITE;
  } else if (monitored <= st->tol2) {
    st->status = ST_CONVERGED;
  } else if (st->iter >= st->maxiter) {
    st->status = ST_MAXITER;
  }
}

template <typename R>
using acc_t = typename AccT<R>::type;

// ------------------------------------------------------------------ hashed random vectors
__device__ __forceinline__ unsigned hash32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}
// Element idx of a fixed pseudo-random complex vector (components in [-1/2, 1/2)):
// BiCGSTAB's shadow vector and the restart perturbation, with no memory traffic.
template <typename R>
__device__ __forceinline__ cx<R> shadow(int idx, unsigned seed) {
  const unsigned a = hash32((unsigned)idx ^ seed);
  const unsigned b = hash32(a ^ ((seed << 16) | (seed >> 16)) ^ 0x9e3779b9U);
  return mkc<R>((R)a * (R)2.3283064365386963e-10 - (R)0.5, (R)b * (R)2.3283064365386963e-10 - (R)0.5);
}
// conj(a) * b added to two accumulators of precision A
template <typename R, typename A>
__device__ __forceinline__ void acc_cdot(A* acc, cx<R> a, cx<R> b) {
  acc[0] += (A)a.re * (A)b.re + (A)a.im * (A)b.im;
  acc[1] += (A)a.re * (A)b.im - (A)a.im * (A)b.re;
}

// ------------------------------------------------------------------ plain operator
// y = post( A0 pre(x) ):  modes
//   0: A0
//   1: Pl A0 Pr                    (the symmetrised operator of generic())
//   2: (Pl A0 Pr)^H = conj(Pl A0 Pr conj(x))
// Pl = principal sqrt of p^2, Pr = 1/Pl (meanas/fdfd/operators.py:120-122).
__device__ __forceinline__ dcx csqrt_principal(dcx z) {
  // sqrt of a complex number, principal branch (Re >= 0; branch cut on the
  // negative real axis with the sign of the imaginary part kept).
  const double a = fabs(z.re), b = fabs(z.im);
  if (a == 0.0 && b == 0.0) return {0.0, z.im};
  const double t = sqrt(0.5 * (hypot(a, b) + a));
  if (z.re >= 0.0) return {t, z.im / (2.0 * t)};
  return {b / (2.0 * t), copysign(t, z.im)};
}

template <typename R>
struct OpApply {
  static constexpr int NB = 1, NO = 0, NRED = 0;
  static constexpr bool NEEDS_W = false;
  const cx<R>* x;
  cx<R>* y;
  int mode;
  Geo<R> g;
  struct Pre {};
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ const cx<R>* box_src(int) const { return x; }
  __device__ void pre(int, Pre&) const {}
  __device__ cx<R> pl_at(int c, int idx) const {
    const int N = g.N;
    const int cell = idx - c * N;
    const int YZ = (int)g.Y * g.Z;
    const int i = (int)(cell / YZ);
    const int j = (int)((cell / g.Z) % g.Y);
    const int k = (int)(cell % g.Z);
    cx<R> p2;
    if (c == 0) p2 = g.dxe[0][i] * g.dxh[1][j] * g.dxh[2][k];
    else if (c == 1) p2 = g.dxh[0][i] * g.dxe[1][j] * g.dxh[2][k];
    else p2 = g.dxh[0][i] * g.dxh[1][j] * g.dxe[2][k];
    dcx s = csqrt_principal({(double)p2.re, (double)p2.im});
    return mkc<R>((R)s.re, (R)s.im);
  }
  __device__ cx<R> make_u(const cx<R>* v, int idx, int c) const {
    cx<R> u = v[0];
    if (mode == 2) u = cconj(u);
    if (mode >= 1) {
      const cx<R> pl = pl_at(c, idx);
      // Pr = 1 / Pl
      const R d = cabs2(pl);
      u = u * mkc<R>(pl.re / d, -pl.im / d);
    }
    return u;
  }
  __device__ const cx<R>* own_src(int) const { return nullptr; }
  __device__ void convert_own(const cx<R>*, const cx<R>*, int, int, cx<R>, acc_t<R>*) const {}
  __device__ void own(int cell, int, int, int, const cx<R>*, const cx<R> yv[3], const cx<R>*, const R*,
                      const Pre&, acc_t<R>*) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * g.N + cell;
      cx<R> v = yv[c];
      if (mode >= 1) v = pl_at(c, idx) * v;
      if (mode == 2) v = cconj(v);
      y[idx] = v;
    }
  }
  __device__ void finish(const double*) const {}
};

// ------------------------------------------------------------------ right-hand sides
// b = pe * (-i omega J)                       (forward, meanas/fdfd/solvers.py:115)
// b = W^-1 conj(pe * (-i omega J))            (adjoint: A0^H E = b0  <=>  A0 y = W^-1 conj(b0),
//                                              E = conj(W y); W A0 is symmetric)
// Also maps an initial guess into the same space (x0 = E or W^-1 conj(E)) and
// reduces |b0|^2 for the unmasked true residual.
template <typename R>
struct OpRhs {
  static constexpr int NRED = 4;
  static constexpr bool NEEDS_W = true;
  const cx<R>* J;
  const cx<R>* E0;  // optional guess
  cx<R>* b;
  cx<R>* x0;        // written when E0 given
  double om_re, om_im;
  int adjoint;
  const uint8_t* mask;
  int N;
  KState* st;
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ void point(int cell, int, int, int, const cx<R> W[3], const R aW[3], acc_t<R>* acc) const {
    const uint8_t m = mask ? mask[cell] : (uint8_t)0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      const cx<R> j = J[idx];
      // -i * omega * J
      const cx<R> b0 = mkc<R>((R)(om_im * j.re + om_re * j.im), (R)(om_im * j.im - om_re * j.re));
      acc[0] += (double)cabs2(b0);
      cx<R> bv = (m & (1u << c)) ? czero<R>() : b0;
      cx<R> wi = mkc<R>(R(1), R(0));
      if (adjoint) {
        const R d = cabs2(W[c]);
        wi = mkc<R>(W[c].re / d, -W[c].im / d);
        bv = wi * cconj(bv);
      }
      b[idx] = bv;
      const double bb = (double)cabs2(bv);
      acc[1] += bb;
      acc[2] += (double)aW[c] * bb;
      acc[3] += (double)aW[c] * (double)aW[c] * bb;
      if (E0) {
        cx<R> e = E0[idx];
        if (adjoint) e = wi * cconj(e);
        x0[idx] = e;
      }
    }
  }
  __device__ void finish(const double* s) const {
    st->b0b0 = s[0];
    st->bb = s[1];
    st->bb_pc = s[2];
    st->bb_w2 = s[3];
    const double bbm = monitored_bb(st);
    st->tol2 = fmax(st->rtol * st->rtol * bbm, st->atol * st->atol);
  }
};

// E = conj(W y) in place (adjoint solution back-transform).
template <typename R>
struct OpAdjPost {
  static constexpr int NRED = 0;
  static constexpr bool NEEDS_W = true;
  cx<R>* x;
  int N;
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ void point(int cell, int, int, int, const cx<R> W[3], const R*, acc_t<R>*) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      x[idx] = cconj(W[c] * x[idx]);
    }
  }
  __device__ void finish(const double*) const {}
};

// ------------------------------------------------------------------ COCG
// init: u = x0 + pert * xi (x0 may be zero; xi a hashed random vector used to restart
// after a breakdown), r = b - A0 u (b may be zero), optionally x_new = u;
// reduces r^T W r, |r|^2, sum|W||r|^2, sum|W|^2|r|^2.
template <typename R>
struct OpCocgInit {
  static constexpr int NB = 1, NO = 0, NRED = 5;
  static constexpr bool NEEDS_W = true;
  const cx<R>* b;   // may be null (zero)
  const cx<R>* x;   // may be null (zero guess)
  cx<R>* r;
  int N;
  KState* st;
  double pert;
  unsigned seed;
  cx<R>* xnew;      // may be null
  struct Pre {
    cx<R> b[3];
  };
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ const cx<R>* box_src(int) const { return x; }
  __device__ void pre(int cell, Pre& p) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) p.b[c] = b ? b[c * N + cell] : czero<R>();
  }
  __device__ cx<R> make_u(const cx<R>* v, int idx, int) const {
    cx<R> u = v[0];
    if (pert != 0.0) u = caxpy(mkc<R>((R)pert, R(0)), shadow<R>(idx, seed), u);
    return u;
  }
  __device__ const cx<R>* own_src(int) const { return nullptr; }
  __device__ void convert_own(const cx<R>*, const cx<R>*, int idx, int, cx<R> u, acc_t<R>*) const {
    if (xnew) xnew[idx] = u;
  }
  __device__ void own(int cell, int, int, int, const cx<R> u[3], const cx<R> y[3], const cx<R> W[3],
                      const R aW[3], const Pre& pr, acc_t<R>* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      const cx<R> rv = pr.b[c] - y[c];
      r[idx] = rv;
      const cx<R> wr = W[c] * rv;
      acc[0] += (double)wr.re * (double)rv.re - (double)wr.im * (double)rv.im;
      acc[1] += (double)wr.re * (double)rv.im + (double)wr.im * (double)rv.re;
      const double r2 = (double)cabs2(rv);
      acc[2] += r2;
      acc[3] += (double)aW[c] * r2;
      acc[4] += (double)aW[c] * (double)aW[c] * r2;
    }
  }
  __device__ void finish(const double* s) const {
    st->rho = {s[0], s[1]};
    st->rr = s[2];
    st->rr_pc = s[3];
    st->rr_w2 = s[4];
    st->beta = {0.0, 0.0};
    st->alpha = {0.0, 0.0};
    st->iter = 0;
    st->pending = 0;
    st->status = ST_RUNNING;
    check_progress(st, monitored_rr(st), dfinite(st->rho));
    if (st->status == ST_MAXITER) st->status = ST_RUNNING;  // maxiter == 0 is handled on the host
    if (st->status == ST_RUNNING && dabs(st->rho) <= BREAKDOWN_RATIO * s[3]) st->status = ST_BREAKDOWN;
  }
};

// p = r + beta p_old ; x += alpha p_old (deferred) ; q = A0 p ; sigma = p^T W q
template <typename R>
struct OpCocgA {
  static constexpr int NB = 2, NO = 1, NRED = 2;
  static constexpr bool NEEDS_W = true;
  const cx<R>* r;
  cx<R>* P0;
  cx<R>* P1;
  cx<R>* x;
  cx<R>* q;
  int N;
  KState* st;
  // per-thread
  const cx<R>* p_old;
  cx<R>* p_new;
  cx<R> beta, alpha;
  bool upd;
  struct Pre {};
  __device__ bool skip() const { return ld_status(st) != ST_RUNNING; }
  __device__ void prepare() {
    const int k = __ldcg(&st->iter);
    p_old = (k & 1) ? P1 : P0;
    p_new = (k & 1) ? P0 : P1;
    beta = from_d<R>(ld_dcx(&st->beta));
    alpha = from_d<R>(ld_dcx(&st->alpha));
    upd = __ldcg(&st->pending) != 0;
  }
  __device__ const cx<R>* box_src(int bi) const { return bi == 0 ? r : p_old; }
  __device__ const cx<R>* own_src(int) const { return upd ? x : nullptr; }
  __device__ void pre(int, Pre&) const {}
  // v = [r, p_old], ov = [x]
  __device__ cx<R> make_u(const cx<R>* v, int, int) const { return caxpy(beta, v[1], v[0]); }
  __device__ void convert_own(const cx<R>* v, const cx<R>* ov, int idx, int, cx<R> u, acc_t<R>*) const {
    p_new[idx] = u;
    if (upd) x[idx] = caxpy(alpha, v[1], ov[0]);
  }
  __device__ void own(int cell, int, int, int, const cx<R> u[3], const cx<R> y[3], const cx<R> W[3],
                      const R*, const Pre&, acc_t<R>* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c * N + cell] = y[c];
      const cx<R> wp = W[c] * u[c];
      acc[0] += (double)wp.re * (double)y[c].re - (double)wp.im * (double)y[c].im;
      acc[1] += (double)wp.re * (double)y[c].im + (double)wp.im * (double)y[c].re;
    }
  }
  __device__ void finish(const double* s) const {
    const dcx sigma = {s[0], s[1]};
    st->sigma = sigma;
    st->pending = 0;
    if (!dfinite(sigma)) {
      st->status = ST_NONFINITE;
      return;
    }
    // an exactly vanishing p^T W q; near-vanishing values are caught by the residual
    // blow-up test of the pointwise pass
    if (sigma.re == 0.0 && sigma.im == 0.0) {
      st->status = ST_BREAKDOWN;
      return;
    }
    st->alpha = ddiv(st->rho, sigma);
  }
};

// r -= alpha q ; rho_new = r^T W r ; |r|^2 ; sum|W||r|^2 ; sum|W|^2|r|^2 ; beta = rho_new / rho
template <typename R>
struct OpCocgB {
  static constexpr int NRED = 5;
  static constexpr bool NEEDS_W = true;
  cx<R>* r;
  const cx<R>* q;
  int N;
  KState* st;
  cx<R> malpha;
  __device__ bool skip() const { return ld_status(st) != ST_RUNNING; }
  __device__ void prepare() {
    const dcx a = ld_dcx(&st->alpha);
    malpha = mkc<R>((R)(-a.re), (R)(-a.im));
  }
  __device__ void point(int cell, int, int, int, const cx<R> W[3], const R aW[3], acc_t<R>* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      const cx<R> rv = caxpy(malpha, q[idx], r[idx]);
      r[idx] = rv;
      const cx<R> wr = W[c] * rv;
      acc[0] += (double)wr.re * (double)rv.re - (double)wr.im * (double)rv.im;
      acc[1] += (double)wr.re * (double)rv.im + (double)wr.im * (double)rv.re;
      const double r2 = (double)cabs2(rv);
      acc[2] += r2;
      acc[3] += (double)aW[c] * r2;
      acc[4] += (double)aW[c] * (double)aW[c] * r2;
    }
  }
  __device__ void finish(const double* s) const {
    const dcx rho_new = {s[0], s[1]};
    const double prev_pc = st->rr_pc;
    st->rr = s[2];
    st->rr_pc = s[3];
    st->rr_w2 = s[4];
    st->iter += 1;
    const bool ok = dfinite(rho_new);
    st->pending = ok ? 1 : 0;
    // a near-zero p^T W q shows up as a residual explosion: the step is discarded
    if (ok && s[3] > 1e16 * prev_pc) {
      st->pending = 0;
      st->status = ST_BREAKDOWN;
      return;
    }
    check_progress(st, monitored_rr(st), ok);
    if (st->status != ST_RUNNING) {
      st->rho = rho_new;
      return;
    }
    // |r^T W r| <= sum |W||r|^2; a ratio below 1e-14 is a (near) breakdown
    if (dabs(rho_new) <= BREAKDOWN_RATIO * s[3]) {
      st->status = ST_BREAKDOWN;
      return;
    }
    st->beta = ddiv(rho_new, st->rho);
    st->rho = rho_new;
  }
};

// x += alpha * p_last if an update is owed (after the loop stops).
template <typename R>
struct OpCocgFinal {
  static constexpr int NRED = 0;
  static constexpr bool NEEDS_W = false;
  cx<R>* P0;
  cx<R>* P1;
  cx<R>* x;
  int N;
  KState* st;
  const cx<R>* p;
  cx<R> alpha;
  bool upd;
  __device__ bool skip() const { return false; }
  __device__ void prepare() {
    const int k = __ldcg(&st->iter);
    p = (k & 1) ? P1 : P0;
    alpha = from_d<R>(ld_dcx(&st->alpha));
    upd = __ldcg(&st->pending) != 0;
  }
  __device__ void point(int cell, int, int, int, const cx<R>*, const R*, acc_t<R>*) const {
    if (!upd) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      x[idx] = caxpy(alpha, p[idx], x[idx]);
    }
  }
  __device__ void finish(const double*) const {}
};

// ------------------------------------------------------------------ BiCGSTAB
// BiCGSTAB vectors (ping-pong pairs selected by iteration parity with ternaries, so
// no runtime-indexed array forces the op into local memory).
struct BsBufs {
  void* R0;
  void* R1;
  void* V0;
  void* V1;
  void* P0;
  void* P1;
  void* T;
  void* x;
};

// P pass (iteration k, buffers old = k&1, new = (k+1)&1):
//   s = r_old - alpha v_old ; r = s - omega t ; p = r + beta (p_old - omega v_old)
//   x += alpha p_old + omega s ; v = A0 p ; sigma = (rh, v) ; |r|^2
template <typename R>
struct OpBsP {
  static constexpr int NB = 4, NO = 1, NRED = 3;
  static constexpr bool NEEDS_W = false;
  BsBufs B;
  int N;
  unsigned seed;
  KState* st;
  const cx<R>* ro;
  const cx<R>* vo;
  const cx<R>* po;
  const cx<R>* t;
  cx<R>* rn;
  cx<R>* vn;
  cx<R>* pn;
  cx<R>* x;
  cx<R> alpha, omega, beta, malpha, momega;
  bool upd;
  struct Pre {};
  __device__ bool skip() const { return ld_status(st) != ST_RUNNING; }
  __device__ void prepare() {
    const bool odd = (__ldcg(&st->iter) & 1) != 0;
    ro = (const cx<R>*)(odd ? B.R1 : B.R0);
    vo = (const cx<R>*)(odd ? B.V1 : B.V0);
    po = (const cx<R>*)(odd ? B.P1 : B.P0);
    rn = (cx<R>*)(odd ? B.R0 : B.R1);
    vn = (cx<R>*)(odd ? B.V0 : B.V1);
    pn = (cx<R>*)(odd ? B.P0 : B.P1);
    t = (const cx<R>*)B.T;
    x = (cx<R>*)B.x;
    upd = __ldcg(&st->pending) != 0;
    if (upd) {
      alpha = from_d<R>(ld_dcx(&st->alpha));
      omega = from_d<R>(ld_dcx(&st->omega));
      beta = from_d<R>(ld_dcx(&st->beta));
    } else {
      alpha = czero<R>();
      omega = czero<R>();
      beta = czero<R>();
    }
    malpha = mkc<R>(-alpha.re, -alpha.im);
    momega = mkc<R>(-omega.re, -omega.im);
  }
  // the first pass (no owed update) only reads r: the other buffers are not initialised
  __device__ const cx<R>* box_src(int bi) const {
    if (!upd && bi > 0) return nullptr;
    return bi == 0 ? ro : (bi == 1 ? vo : (bi == 2 ? t : po));
  }
  __device__ const cx<R>* own_src(int) const { return upd ? x : nullptr; }
  __device__ void pre(int, Pre&) const {}
  // v = [r_old, v_old, t, p_old]
  __device__ cx<R> make_u(const cx<R>* v, int, int) const {
    if (!upd) return v[0];
    const cx<R> s = caxpy(malpha, v[1], v[0]);
    const cx<R> r = caxpy(momega, v[2], s);
    return caxpy(beta, caxpy(momega, v[1], v[3]), r);
  }
  // r_new, p_new and the owed x += alpha p_old + omega s need no operator: write them now
  __device__ void convert_own(const cx<R>* v, const cx<R>* ov, int idx, int, cx<R> u, acc_t<R>* acc) const {
    cx<R> r = v[0];
    if (upd) {
      const cx<R> s = caxpy(malpha, v[1], v[0]);
      r = caxpy(momega, v[2], s);
      x[idx] = caxpy(omega, s, caxpy(alpha, v[3], ov[0]));
    }
    rn[idx] = r;
    pn[idx] = u;
    acc[2] += cabs2(r);
  }
  __device__ void own(int cell, int, int, int, const cx<R>*, const cx<R> y[3], const cx<R>*, const R*,
                      const Pre&, acc_t<R>* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      vn[idx] = y[c];
      acc_cdot<R>(acc, shadow<R>(idx, seed), y[c]);
    }
  }
  __device__ void finish(const double* s) const {
    const dcx sigma = {s[0], s[1]};
    st->sigma = sigma;
    st->rr = s[2];
    st->pending = 0;
    if (!dfinite(sigma) || !isfinite(s[2])) {
      st->status = ST_NONFINITE;
      return;
    }
    if (dabs(sigma) <= 1e-300 || dabs(st->rho) <= 1e-300) {
      st->status = ST_BREAKDOWN;
      return;
    }
    st->alpha = ddiv(st->rho, sigma);
  }
};

// S pass: s = r - alpha v ; t = A0 s ; (t,s), |t|^2, (rh,t), |s|^2 ; omega, rho, beta
template <typename R>
struct OpBsS {
  static constexpr int NB = 2, NO = 0, NRED = 6;
  static constexpr bool NEEDS_W = false;
  BsBufs B;
  int N;
  unsigned seed;
  KState* st;
  const cx<R>* r;
  const cx<R>* v;
  cx<R>* t;
  cx<R> malpha;
  struct Pre {};
  __device__ bool skip() const { return ld_status(st) != ST_RUNNING; }
  __device__ void prepare() {
    const bool odd = (__ldcg(&st->iter) & 1) != 0;
    r = (const cx<R>*)(odd ? B.R0 : B.R1);
    v = (const cx<R>*)(odd ? B.V0 : B.V1);
    t = (cx<R>*)B.T;
    const dcx a = ld_dcx(&st->alpha);
    malpha = mkc<R>((R)(-a.re), (R)(-a.im));
  }
  __device__ const cx<R>* box_src(int bi) const { return bi == 0 ? r : v; }
  __device__ void pre(int, Pre&) const {}
  __device__ cx<R> make_u(const cx<R>* vv, int, int) const { return caxpy(malpha, vv[1], vv[0]); }
  __device__ const cx<R>* own_src(int) const { return nullptr; }
  __device__ void convert_own(const cx<R>*, const cx<R>*, int, int, cx<R>, acc_t<R>*) const {}
  __device__ void own(int cell, int, int, int, const cx<R> u[3], const cx<R> y[3], const cx<R>*, const R*,
                      const Pre&, acc_t<R>* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      t[idx] = y[c];
      acc_cdot<R>(acc, y[c], u[c]);                       // (t, s)
      acc[2] += cabs2(y[c]);                              // |t|^2
      acc_cdot<R>(acc + 3, shadow<R>(idx, seed), y[c]);   // (rh, t)
      acc[5] += cabs2(u[c]);                              // |s|^2
    }
  }
  __device__ void finish(const double* s) const {
    const dcx ts = {s[0], s[1]};
    const double tt = s[2];
    const dcx rht = {s[3], s[4]};
    const double ss = s[5];
    st->iter += 1;
    st->pending = 1;
    if (!dfinite(ts) || !isfinite(tt) || !dfinite(rht) || !isfinite(ss)) {
      st->status = ST_NONFINITE;
      st->pending = 0;
      return;
    }
    if (ss <= st->tol2 || tt <= 0.0) {
      // s already small enough (or t vanished): finish with omega = 0
      st->omega = {0.0, 0.0};
      st->rr = ss;
      check_progress(st, ss, true);
      if (st->status == ST_RUNNING) st->status = ST_BREAKDOWN;
      return;
    }
    const dcx om = {ts.re / tt, ts.im / tt};
    st->omega = om;
    double rr = ss - (ts.re * ts.re + ts.im * ts.im) / tt;
    if (rr < 0.0) rr = 0.0;
    st->rr = rr;
    check_progress(st, rr, true);
    if (st->status != ST_RUNNING) return;
    // stagnation: no 1 % improvement on the best residual for stall_limit iterations
    if (rr < 0.98 * st->best_rr || st->iter == 1) {
      st->best_rr = rr;
      st->best_iter = st->iter;
    } else if (st->stall_limit > 0 && st->iter - st->best_iter >= st->stall_limit) {
      st->status = ST_BREAKDOWN;
      return;
    }
    const dcx rho_new = {-(om.re * rht.re - om.im * rht.im), -(om.re * rht.im + om.im * rht.re)};
    if (dabs(om) <= 1e-300 || dabs(rho_new) <= 1e-300) {
      st->status = ST_BREAKDOWN;
      return;
    }
    // beta = (rho_new / rho) * (alpha / omega)
    st->beta = dmul(ddiv(rho_new, st->rho), ddiv(st->alpha, om));
    st->rho = rho_new;
  }
};

// BiCGSTAB start: r = b - A0 x0 (x0 may be zero) ; rho = (rh, r) ; |r|^2 ; status.
template <typename R>
struct OpBsInit {
  static constexpr int NB = 1, NO = 0, NRED = 3;
  static constexpr bool NEEDS_W = false;
  const cx<R>* b;
  const cx<R>* x;
  cx<R>* r;
  int N;
  unsigned seed;
  KState* st;
  struct Pre {
    cx<R> b[3];
  };
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ const cx<R>* box_src(int) const { return x; }
  __device__ void pre(int cell, Pre& p) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) p.b[c] = b[c * N + cell];
  }
  __device__ cx<R> make_u(const cx<R>* v, int, int) const { return v[0]; }
  __device__ const cx<R>* own_src(int) const { return nullptr; }
  __device__ void convert_own(const cx<R>*, const cx<R>*, int, int, cx<R>, acc_t<R>*) const {}
  __device__ void own(int cell, int, int, int, const cx<R>*, const cx<R> y[3], const cx<R>*, const R*,
                      const Pre& pr, acc_t<R>* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      const cx<R> rv = pr.b[c] - y[c];
      r[idx] = rv;
      acc_cdot<R>(acc, shadow<R>(idx, seed), rv);
      acc[2] += (double)cabs2(rv);
    }
  }
  __device__ void finish(const double* s) const {
    st->rho = {s[0], s[1]};
    st->rr = s[2];
    st->iter = 0;
    st->pending = 0;
    st->status = ST_RUNNING;
    check_progress(st, s[2], dfinite(st->rho));
    if (st->status == ST_MAXITER) st->status = ST_RUNNING;
  }
};

// Owed update after the loop stops: x += alpha p + omega (r - alpha v) on buffers
// new = iter & 1 (the last P pass wrote r, v, p there).
template <typename R>
struct OpBsFinal {
  static constexpr int NRED = 0;
  static constexpr bool NEEDS_W = false;
  BsBufs B;
  int N;
  KState* st;
  const cx<R>* r;
  const cx<R>* v;
  const cx<R>* p;
  cx<R>* x;
  cx<R> alpha, omega, malpha;
  bool upd;
  __device__ bool skip() const { return false; }
  __device__ void prepare() {
    const bool odd = (__ldcg(&st->iter) & 1) != 0;
    r = (const cx<R>*)(odd ? B.R1 : B.R0);
    v = (const cx<R>*)(odd ? B.V1 : B.V0);
    p = (const cx<R>*)(odd ? B.P1 : B.P0);
    x = (cx<R>*)B.x;
    upd = __ldcg(&st->pending) != 0;
    alpha = from_d<R>(ld_dcx(&st->alpha));
    omega = from_d<R>(ld_dcx(&st->omega));
    malpha = mkc<R>(-alpha.re, -alpha.im);
  }
  __device__ void point(int cell, int, int, int, const cx<R>*, const R*, acc_t<R>*) const {
    if (!upd) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      const cx<R> s = caxpy(malpha, v[idx], r[idx]);
      x[idx] = caxpy(omega, s, caxpy(alpha, p[idx], x[idx]));
    }
  }
  __device__ void finish(const double*) const {}
};

// ------------------------------------------------------------------ refinement (c128)
// u = E_old + scale * d (d in the inner precision, optional) ; E_new = u ; r = b - A0 u ;
// r32 = (complex64)(r * rscale) ; reduces |r|^2, sum|W||r|^2, sum|W|^2|r|^2,
// (rh, r32) and |r32|^2 (the inner BiCGSTAB's starting rho and norm).
template <typename RI>
struct OpRefine {
  static constexpr int NB = 1, NO = 0, NRED = 6;
  static constexpr bool NEEDS_W = true;
  const cx<double>* E_old;
  const cx<RI>* d;
  cx<double>* E_new;
  const cx<double>* b;
  cx<RI>* rin;
  double scale, rscale;
  int N;
  unsigned seed;
  KState* st;
  struct Pre {
    cx<double> b[3];
  };
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ const cx<double>* box_src(int) const { return E_old; }
  __device__ void pre(int cell, Pre& p) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) p.b[c] = b[c * N + cell];
  }
  __device__ cx<double> make_u(const cx<double>* v, int idx, int) const {
    cx<double> e = v[0];
    if (d) {
      const cx<RI> dv = d[idx];
      e = caxpy(mkc<double>(scale, 0.0), mkc<double>((double)dv.re, (double)dv.im), e);
    }
    return e;
  }
  __device__ const cx<double>* own_src(int) const { return nullptr; }
  __device__ void convert_own(const cx<double>*, const cx<double>*, int, int, cx<double>, double*) const {}
  __device__ void own(int cell, int, int, int, const cx<double> u[3], const cx<double> y[3],
                      const cx<double>*, const double aW[3], const Pre& pr, double* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      E_new[idx] = u[c];
      const cx<double> rv = pr.b[c] - y[c];
      const cx<RI> r1 = mkc<RI>((RI)(rscale * rv.re), (RI)(rscale * rv.im));
      rin[idx] = r1;
      const double r2 = cabs2(rv);
      acc[0] += r2;
      acc[1] += aW[c] * r2;
      acc[2] += aW[c] * aW[c] * r2;
      acc_cdot<RI>(acc + 3, shadow<RI>(idx, seed), r1);
      acc[5] += (double)cabs2(r1);
    }
  }
  __device__ void finish(const double* s) const {
    st->rr = s[0];
    st->rr_pc = s[1];
    st->rr_w2 = s[2];
    st->extra[0] = s[3];
    st->extra[1] = s[4];
    st->extra[2] = s[5];
  }
};

// FP64 residual of E for the unmasked right-hand side b0 = -i omega J:
// r = b0 - A0 E (or b0 - A0^H E with `adjoint`, using A0^H = conj(W A0 W^-1 conj(.)));
// reduces |r|^2, sum|W||r|^2 (forward) or sum|W|^-1|r|^2 (adjoint), |b0|^2 and the
// matching weighted |b0|^2: the true and the symmetrised-system residuals.
template <typename R>
struct OpResidual {
  static constexpr int NB = 1, NO = 0, NRED = 4;
  static constexpr bool NEEDS_W = true;
  const cx<R>* E;
  const cx<R>* J;
  double om_re, om_im;
  int adjoint;
  Geo<R> g;
  double* out;  // 4 doubles
  struct Pre {
    cx<R> j[3];
  };
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ const cx<R>* box_src(int) const { return E; }
  __device__ void pre(int cell, Pre& p) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) p.j[c] = J[c * g.N + cell];
  }
  __device__ cx<R> w_at(int c, int idx) const {
    const int cell = idx - c * g.N;
    const int YZ = (int)g.Y * g.Z;
    const int i = (int)(cell / YZ);
    const int j = (int)((cell / g.Z) % g.Y);
    const int k = (int)(cell % g.Z);
    if (c == 0) return g.dxe[0][i] * g.dxh[1][j] * g.dxh[2][k];
    if (c == 1) return g.dxh[0][i] * g.dxe[1][j] * g.dxh[2][k];
    return g.dxh[0][i] * g.dxh[1][j] * g.dxe[2][k];
  }
  __device__ cx<R> make_u(const cx<R>* v, int idx, int c) const {
    cx<R> e = v[0];
    if (adjoint) {
      const cx<R> w = w_at(c, idx);
      const R d = cabs2(w);
      e = mkc<R>(w.re / d, -w.im / d) * cconj(e);
    }
    return e;
  }
  __device__ const cx<R>* own_src(int) const { return nullptr; }
  __device__ void convert_own(const cx<R>*, const cx<R>*, int, int, cx<R>, acc_t<R>*) const {}
  __device__ void own(int, int, int, int, const cx<R>*, const cx<R> y[3], const cx<R> W[3],
                      const R aW[3], const Pre& pr, acc_t<R>* acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cx<R> j = pr.j[c];
      const cx<R> b0 = mkc<R>((R)(om_im * j.re + om_re * j.im), (R)(om_im * j.im - om_re * j.re));
      const cx<R> ay = adjoint ? cconj(W[c] * y[c]) : y[c];
      const cx<R> rv = b0 - ay;
      const double wgt = adjoint ? 1.0 / (double)aW[c] : (double)aW[c];
      acc[0] += (double)cabs2(rv);
      acc[1] += wgt * (double)cabs2(rv);
      acc[2] += (double)cabs2(b0);
      acc[3] += wgt * (double)cabs2(b0);
    }
  }
  __device__ void finish(const double* s) const {
    out[0] = s[0];
    out[1] = s[1];
    out[2] = s[2];
    out[3] = s[3];
  }
};

// dL/deps from a forward field E and the adjoint field E_adj (A0^H E_adj = b_adj):
// grad = Re(omega^2 conj(E_adj) E) on non-PEC components, 0 on PEC ones.  With
// lambda = conj(E_adj) solving A0^T lambda = conj(dL/dE), this is the derivative of
// L through A0 = pe (... - omega^2 eps) pe (meanas/fdfd/operators.py:95).
template <typename R>
struct OpEpsGrad {
  static constexpr int NRED = 0;
  static constexpr bool NEEDS_W = false;
  const cx<R>* E;
  const cx<R>* Ea;
  R* grad;
  cx<R> w2;
  const uint8_t* mask;
  int N;
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ void point(int cell, int, int, int, const cx<R>*, const R*, acc_t<R>*) const {
    const uint8_t m = mask ? mask[cell] : (uint8_t)0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      const cx<R> v = w2 * (cconj(Ea[idx]) * E[idx]);
      grad[idx] = (m & (1u << c)) ? R(0) : v.re;
    }
  }
  __device__ void finish(const double*) const {}
};

// Copy / convert / zero helpers (pointwise over the 3 components of each cell).
template <typename RS, typename RD>
struct OpCopy {
  static constexpr int NRED = 0;
  static constexpr bool NEEDS_W = false;
  const cx<RS>* src;  // null = zero fill
  cx<RD>* dst;
  int N;
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ void point(int cell, int, int, int, const void*, const void*, acc_t<RD>*) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * N + cell;
      if (src) {
        const cx<RS> v = src[idx];
        dst[idx] = mkc<RD>((RD)v.re, (RD)v.im);
      } else {
        dst[idx] = mkc<RD>(RD(0), RD(0));
      }
    }
  }
  __device__ void finish(const double*) const {}
};

// ------------------------------------------------------------------ TFSF / boundary sources
// The step before the solve (meanas/fdfd/operators.py:366-450): the current that injects
// a desired field E inside a total-field region Q,
//   J = (A0 Q E - Q A0 E) / (-i omega),   A0 = e_full(omega, dxes, epsilon, mu) (no masks),
// and, with `edges`, only on the cells where shifting Q by one cell along a non-singleton
// axis changes it (e_boundary_source; `periodic` wraps the shift, otherwise the cell past
// an edge mirrors back onto the edge cell, fdmath/operators.py:55-98).  Two stencil
// passes, no scratch: pass 0 writes out = A0 (Q E); pass 1 reads it back and writes
// out = jmask (out - Q A0 E) / (-i omega).
template <typename R>
struct OpTfsf {
  static constexpr int NB = 1, NO = 0, NRED = 0;
  static constexpr bool NEEDS_W = false;
  const cx<R>* e;
  const R* q;  // Q, per component (3N)
  cx<R>* out;
  int pass, edges, periodic;
  cx<R> inv_miw;  // 1 / (-i omega)
  Geo<R> g;
  struct Pre {
    cx<R> o[3];
    R qv[3];
  };
  __device__ bool skip() const { return false; }
  __device__ void prepare() {}
  __device__ const cx<R>* box_src(int) const { return e; }
  __device__ void pre(int cell, Pre& p) const {
    if (pass == 0) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      p.o[c] = out[c * g.N + cell];
      p.qv[c] = q[c * g.N + cell];
    }
  }
  __device__ cx<R> make_u(const cx<R>* v, int idx, int) const { return pass == 0 ? q[idx] * v[0] : v[0]; }
  __device__ const cx<R>* own_src(int) const { return nullptr; }
  __device__ void convert_own(const cx<R>*, const cx<R>*, int, int, cx<R>, acc_t<R>*) const {}
  // the index one cell away along `axis` (s = +-1): wrapped, or mirrored onto the edge cell
  __device__ int step(int v, int n, int s) const {
    v += s;
    if (periodic) return v < 0 ? n - 1 : (v >= n ? 0 : v);
    return v < 0 ? 0 : (v >= n ? n - 1 : v);
  }
  __device__ bool on_edge(int c, int i, int j, int k) const {
    const int YZ = g.Y * g.Z, base = c * g.N;
    const R q0 = q[base + i * YZ + j * g.Z + k];
    bool m = false;
#pragma unroll
    for (int s = -1; s <= 1; s += 2) {
      if (g.X > 1) m |= q[base + step(i, g.X, s) * YZ + j * g.Z + k] != q0;
      if (g.Y > 1) m |= q[base + i * YZ + step(j, g.Y, s) * g.Z + k] != q0;
      if (g.Z > 1) m |= q[base + i * YZ + j * g.Z + step(k, g.Z, s)] != q0;
    }
    return m;
  }
  __device__ void own(int cell, int i, int j, int k, const cx<R>*, const cx<R> yv[3], const cx<R>*, const R*,
                      const Pre& p, acc_t<R>*) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int idx = c * g.N + cell;
      if (pass == 0) {
        out[idx] = yv[c];
      } else {
        cx<R> v = (p.o[c] - p.qv[c] * yv[c]) * inv_miw;
        if (edges && !on_edge(c, i, j, k)) v = czero<R>();
        out[idx] = v;
      }
    }
  }
  __device__ void finish(const double*) const {}
};

// ------------------------------------------------------------------ E -> H, E x H
// The step after the solve: H = pm mu^-1 ce(E) / (-i omega) (the sparse e2h of
// meanas/fdfd/operators.py:253-282) and, when S is set, S = E x H' with H' = conj(H)
// (conj_h, the product meanas/test/test_fdfd.py:38-40 forms) or H (H itself the
// caller's when h_in: functional.poynting_e_cross_h(dxes)(E, H)), on the Yee grid of
// meanas/fdfd/functional.py:187-221: E components weighted by dx_e and taken one cell
// up along the cross axis, H components weighted by dx_h.  One thread per cell over
// (x plane, y/z tile) units like the pointwise engine; E's +1 neighbours come through
// L1/L2, so HBM sees E once and H, S once each.
template <int TZ, int TY>
__global__ void __launch_bounds__(TZ * TY) k_e2h(const Geo<double> g, const cx<double>* __restrict__ E,
                                                 cx<double>* __restrict__ H, cx<double>* __restrict__ S,
                                                 cx<double> inv_miw, int conj_h, int h_in) {
  using C = cx<double>;
  const int ntiles = g.ntz * g.nty, units = ntiles * g.X, YZ = g.Y * g.Z, N = g.N;
  for (int u = blockIdx.x; u < units; u += gridDim.x) {
    const int i = u / ntiles, t = u - i * ntiles;
    const int tyb = t / g.ntz, tzb = t - tyb * g.ntz;
    const int j = tyb * TY + threadIdx.y, k = tzb * TZ + threadIdx.x;
    if (j >= g.Y || k >= g.Z) continue;
    const int i1 = i + 1 == g.X ? 0 : i + 1, j1 = j + 1 == g.Y ? 0 : j + 1, k1 = k + 1 == g.Z ? 0 : k + 1;
    const int c0 = i * YZ + j * g.Z + k;
    const int cx1 = i1 * YZ + j * g.Z + k, cy1 = i * YZ + j1 * g.Z + k, cz1 = i * YZ + j * g.Z + k1;
    const C ex = E[c0], ey = E[N + c0], ez = E[2 * N + c0];
    const C ey_x1 = E[N + cx1], ez_x1 = E[2 * N + cx1];
    const C ex_y1 = E[cy1], ez_y1 = E[2 * N + cy1];
    const C ex_z1 = E[cz1], ey_z1 = E[N + cz1];
    C hx, hy, hz;
    if (h_in) {  // S from the caller's H
      hx = H[c0];
      hy = H[N + c0];
      hz = H[2 * N + c0];
    } else {
      const C ix = g.idxe[0][i], iy = g.idxe[1][j], iz = g.idxe[2][k];
      hx = ((ez_y1 - ez) * iy - (ey_z1 - ey) * iz) * inv_miw;
      hy = ((ex_z1 - ex) * iz - (ez_x1 - ez) * ix) * inv_miw;
      hz = ((ey_x1 - ey) * ix - (ex_y1 - ex) * iy) * inv_miw;
      if (g.muinv) {
        hx = g.muinv[c0] * hx;
        hy = g.muinv[N + c0] * hy;
        hz = g.muinv[2 * N + c0] * hz;
      }
      if (g.mask) {
        const uint8_t m = g.mask[c0];
        if (m & 8u) hx = czero<double>();
        if (m & 16u) hy = czero<double>();
        if (m & 32u) hz = czero<double>();
      }
    }
    if (H && !h_in) {
      H[c0] = hx;
      H[N + c0] = hy;
      H[2 * N + c0] = hz;
    }
    if (S) {
      const C wx = (conj_h ? cconj(hx) : hx) * g.dxh[0][i];
      const C wy = (conj_h ? cconj(hy) : hy) * g.dxh[1][j];
      const C wz = (conj_h ? cconj(hz) : hz) * g.dxh[2][k];
      const C dex = g.dxe[0][i], dey = g.dxe[1][j], dez = g.dxe[2][k];
      S[c0] = (ey_x1 * dey) * wz - (ez_x1 * dez) * wy;
      S[N + c0] = (ez_y1 * dez) * wx - (ex_y1 * dex) * wz;
      S[2 * N + c0] = (ex_z1 * dex) * wy - (ey_z1 * dey) * wx;
    }
  }
}

}  // namespace fdfd
