// Device-side building blocks of the FDFD solve path (sm_100a).
//
// Layout (same as the reference's vec/unvec, meanas/fdmath/vectorization.py:51-125):
//   a field is 3 components x (X, Y, Z) cells, C order, z fastest:
//   element (c, i, j, k) lives at c*N + (i*Y + j)*Z + k, N = X*Y*Z.
//   Complex values are interleaved (re, im) pairs of float (c64) or double (c128).
//
// The operator applied everywhere is the reference's E-field wave operator
// (meanas/fdfd/operators.py:40-96):
//   A0 u = pe * ( ch( pm * mu^-1 * ce(pe * u) ) - omega^2 * eps * pe * u )
// with forward/backward periodic differences (meanas/fdmath/functional.py:16-122):
//   dF_a f[i] = (f[i+1] - f[i]) / dxe_a[i],   dB_a g[i] = (g[i] - g[i-1]) / dxh_a[i].
//
// Kernel shape: a CTA owns a TY x TZ tile of (y, z) columns and marches along x over
// a chunk of planes.  Each step stages one x-plane of the input field (tile plus a
// one-cell periodic halo in y and z) in shared memory, computes H = ce(u) on the tile
// plus its low y/z halo, then the curl of H.  H on plane i-1 (needed by dB_x) stays in
// registers, so every input value is read from memory once per step (halo reads hit
// L1/L2).  The input field is produced on the fly by a pointwise loader (for example
// r + beta * p in a Krylov step) and every own cell is handed, with its operator
// value, to an epilogue that writes outputs and accumulates reductions; so the
// Krylov vector updates and dot products ride on the same pass over HBM.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>
#include <utility>

namespace fdfd {

// ---------------------------------------------------------------- complex arithmetic
template <typename R>
struct __align__(2 * sizeof(R)) cx {
  R re, im;
};

template <typename R>
__host__ __device__ __forceinline__ cx<R> mkc(R a, R b) { cx<R> z; z.re = a; z.im = b; return z; }
template <typename R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return mkc<R>(a.re + b.re, a.im + b.im); }
template <typename R>
__device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return mkc<R>(a.re - b.re, a.im - b.im); }
template <typename R>
__device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b) {
  return mkc<R>(fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re));
}
template <typename R>
__device__ __forceinline__ cx<R> operator*(R s, cx<R> a) { return mkc<R>(s * a.re, s * a.im); }
template <typename R>
__device__ __forceinline__ cx<R> cconj(cx<R> a) { return mkc<R>(a.re, -a.im); }
template <typename R>
__device__ __forceinline__ R cabs2(cx<R> a) { return fma(a.re, a.re, a.im * a.im); }
// a + s*b
template <typename R>
__device__ __forceinline__ cx<R> caxpy(cx<R> s, cx<R> b, cx<R> a) {
  return mkc<R>(fma(s.re, b.re, fma(-s.im, b.im, a.re)), fma(s.re, b.im, fma(s.im, b.re, a.im)));
}
template <typename R>
__device__ __forceinline__ cx<R> czero() { return mkc<R>(R(0), R(0)); }

// FP64 complex scalars live in device memory as two doubles.
struct dcx {
  double re, im;
};
__device__ __forceinline__ dcx dmul(dcx a, dcx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ dcx ddiv(dcx a, dcx b) {
  // Smith's algorithm (scaled complex division).
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  } else {
    double r = b.re / b.im, d = b.re * r + b.im;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
  }
}
__device__ __forceinline__ double dabs(dcx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ bool dfinite(dcx a) { return isfinite(a.re) && isfinite(a.im); }
template <typename R>
__device__ __forceinline__ cx<R> from_d(dcx a) { return mkc<R>((R)a.re, (R)a.im); }

// ---------------------------------------------------------------- grid description
// Mask byte per cell: bits 0..2 = PEC on the x/y/z E component, bits 3..5 = PMC on
// the x/y/z H component (meanas/fdfd/operators.py:79-87: any nonzero = conductor).
template <typename R>
struct Geo {
  int X, Y, Z;         // cells per axis
  int XC;              // x planes per CTA
  int ntz, nty, nxc;   // CTAs along z tiles, y tiles, x chunks
  int N;         // X*Y*Z
  const cx<R>* idxe[3];  // 1/dx_e per axis
  const cx<R>* idxh[3];  // 1/dx_h per axis
  const cx<R>* dxe[3];   // dx_e (for the symmetriser weights p^2)
  const cx<R>* dxh[3];
  const R* adxe[3];      // |dx_e|, |dx_h|: |W| is a product of these (no square roots per cell)
  const R* adxh[3];
  const R* eps;          // 3N
  const R* muinv;        // 3N or null
  const uint8_t* mask;   // N or null
  const cx<R>* w2p;      // omega^2, in device memory (so captured graphs survive a new omega)
  int rb_shift;          // reduction blocks of 2^rb_shift x planes (see stencil_unit)
};

__device__ __forceinline__ int wrapi(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// Symmetriser weights W = p^2 (meanas/fdfd/operators.py:116-118) for the three
// components of a cell, from per-thread y/z products and per-plane x values.
template <typename R>
struct WeightYZ {
  cx<R> yz[3];
  R ayz[3];
  __device__ __forceinline__ void init(const Geo<R>& g, int j, int k) {
    const cx<R> ey = g.dxe[1][j], hy = g.dxh[1][j], ez = g.dxe[2][k], hz = g.dxh[2][k];
    yz[0] = hy * hz;   // x: dxe_x * dxh_y * dxh_z
    yz[1] = ey * hz;   // y: dxh_x * dxe_y * dxh_z
    yz[2] = hy * ez;   // z: dxh_x * dxh_y * dxe_z
    const R aey = g.adxe[1][j], ahy = g.adxh[1][j], aez = g.adxe[2][k], ahz = g.adxh[2][k];
    ayz[0] = ahy * ahz;
    ayz[1] = aey * ahz;
    ayz[2] = ahy * aez;
  }
  // W and |W| of the three components on plane i, from that plane's x factors
  __device__ __forceinline__ void at(cx<R> ex, cx<R> hx, R aex, R ahx, cx<R> W[3], R aW[3]) const {
    W[0] = ex * yz[0];
    W[1] = hx * yz[1];
    W[2] = hx * yz[2];
    aW[0] = aex * ayz[0];
    aW[1] = ahx * ayz[1];
    aW[2] = ahx * ayz[2];
  }
};

// Per-thread accumulators: FP64 for complex128 kernels, FP32 for complex64 kernels
// (summed over one thread's cells; the CTA and grid sums are always FP64).
template <typename R>
struct AccT {
  using type = double;
};
template <>
struct AccT<float> {
  using type = float;
};

// ---------------------------------------------------------------- reductions
// Deterministic grid reduction: every CTA writes its partial sums, the last CTA to
// finish (atomic ticket) sums them in a fixed order and runs the op's finish().
struct RedBuf {
  double* partials;        // [gridDim.x * NRED]
  unsigned int* ticket;    // zero between launches (reset by the last CTA)
};

// Sum NRED values over the CTA at once: warp trees for all values, one pass through
// shared memory (sh[warp][r]), then thread r < NRED sums value r over the warps in a
// fixed order and returns it (other threads return 0).
template <int NT, int NRED>
__device__ __forceinline__ double block_sum_n(double (&v)[NRED], double* sh) {
  constexpr int NW = (NT + 31) / 32;
  static_assert(NW * NRED <= 64, "reduction scratch is 64 doubles");
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int r = 0; r < NRED; ++r) v[r] += __shfl_down_sync(0xffffffffu, v[r], o);
  }
  __syncthreads();  // sh free (earlier readers done)
  if ((tid & 31) == 0) {
#pragma unroll
    for (int r = 0; r < NRED; ++r) sh[(tid >> 5) * NRED + r] = v[r];
  }
  __syncthreads();
  double s = 0.0;
  if (tid < NRED) {
#pragma unroll
    for (int w = 0; w < NW; ++w) s += sh[w * NRED + tid];
  }
  return s;
}

// Warp 0 turns the per-thread sums of a plane block (sh[r * NT + t]) into partial number
// `part`: lane l adds threads l, l + 32, ... in order, then a fixed shuffle tree.
template <int NT, int NRED, typename A>
__device__ __forceinline__ void sum_block_partials(const A* sh, RedBuf rb, size_t part) {
  const int lane = threadIdx.x + threadIdx.y * blockDim.x;  // called by threads 0..31
#pragma unroll
  for (int r = 0; r < NRED; ++r) {
    double v = 0.0;
#pragma unroll
    for (int t = lane; t < NT; t += 32) v += (double)sh[r * NT + t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) rb.partials[part * NRED + r] = v;
  }
}

// Write the CTA's sum of NRED per-thread accumulators as partial number `part`
// (threads r < NRED store value r).  Every thread of the CTA must call it.
template <int NT, int NRED, typename A>
__device__ __forceinline__ void write_partial(const A (&acc)[NRED], RedBuf rb, size_t part, double* sh) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  double v[NRED];
#pragma unroll
  for (int r = 0; r < NRED; ++r) v[r] = (double)acc[r];
  const double s = block_sum_n<NT, NRED>(v, sh);
  if (tid < NRED) rb.partials[part * NRED + tid] = s;
}

// After every CTA has written its partials: the last CTA to arrive (atomic ticket) sums
// all `nparts` partials in a fixed order and returns true in its thread 0, which holds
// the totals in `out`.  The last CTA reads them with independent loads (no per-value
// passes), so the serial tail after the last CTA's own work is about two L2 round trips.
template <int NT, int NRED>
__device__ bool grid_finish(RedBuf rb, unsigned int nparts, double* sh, double* out) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    __threadfence();  // cumulative: the partials written before the barrier are visible first
    unsigned int t = atomicAdd(rb.ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double s[NRED];
#pragma unroll
  for (int r = 0; r < NRED; ++r) s[r] = 0.0;
#pragma unroll 4
  for (unsigned int b = tid; b < nparts; b += NT) {
#pragma unroll
    for (int r = 0; r < NRED; ++r) s[r] += __ldcg(&rb.partials[(size_t)b * NRED + r]);
  }
  const double tot = block_sum_n<NT, NRED>(s, sh);
  __syncthreads();  // sh reads of block_sum_n done
  if (tid < NRED) sh[tid] = tot;
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int r = 0; r < NRED; ++r) out[r] = sh[r];
    *rb.ticket = 0u;
  }
  return tid == 0;
}

// Reduce NRED per-thread accumulators across the grid with one partial per CTA; returns
// true in the one thread (thread 0 of the last CTA) that holds the final sums in `out`.
template <int NT, int NRED, typename A>
__device__ bool grid_reduce(const A (&acc)[NRED], RedBuf rb, double* sh, double* out) {
  write_partial<NT, NRED>(acc, rb, blockIdx.x, sh);
  return grid_finish<NT, NRED>(rb, gridDim.x, sh, out);
}

// Ops that carry solver state (a member `st` pointing to it) run finish() on a copy:
// the last CTA's thread 0 loads the whole state with independent loads, runs the scalar
// recurrences on the copy and stores it back, instead of a chain of dependent L2 round
// trips through the global struct.  No other thread reads the state at that point (the
// other CTAs have passed the ticket; the host reads it after the kernel).
template <class Op, class = void>
struct HasState : std::false_type {};
template <class Op>
struct HasState<Op, std::void_t<decltype(std::declval<Op&>().st)>> : std::true_type {};

// Out of line, so the state copy's registers are not reserved by the whole kernel.
template <class Op>
__device__ __noinline__ void finish_on_copy(Op o, const double* sums) {
  using St = std::remove_pointer_t<decltype(o.st)>;
  St* const g = o.st;
  St loc = *g;
  o.st = &loc;
  o.finish(sums);
  *g = loc;
}

template <class Op>
__device__ __forceinline__ void run_finish(const Op& o, const double* sums) {
  if constexpr (HasState<Op>::value) {
    finish_on_copy(o, sums);
  } else {
    o.finish(sums);
  }
}

// ---------------------------------------------------------------- stencil engine
// Op interface:
//   static constexpr int NB;       box inputs: complex 3N vectors read on the tile + halo
//   static constexpr int NO;       own inputs: complex 3N vectors read on own cells only
//   static constexpr int NRED;     number of FP64 accumulators (0 = none)
//   static constexpr bool NEEDS_W; pass symmetriser weights to own()
//   struct Pre;                    own-cell values prefetched at the start of a plane step
//   bool skip() const;             uniform early exit (solver stopped)
//   void prepare();                read scalars once per thread
//   const cx<R>* box_src(int b) const;               null = zeros
//   const cx<R>* own_src(int o) const;               null = zeros
//   cx<R> make_u(const cx<R>* v, int idx, int c) const;   input field from raw values
//   void convert_own(const cx<R>* v, const cx<R>* ov, int idx, int c, cx<R> u, A* acc) const;
//        own cells of the CTA's planes, when their inputs land: outputs that do not need
//        the operator (p = r + beta p_old, x updates, r updates) are written here
//   void pre(int cell, Pre& p) const;
//   void own(int cell, int i, int j, int k, const cx<R> u[3], const cx<R> y[3],
//            const cx<R> W[3], const R aW[3], const Pre& p, A* acc);   y = A0 u
//   void finish(const double* sums) const;    last CTA, thread 0
//
// Pipeline per x plane i (U holds u on planes i and i+1, Sbox/Sown the raw inputs of
// plane i+2 in flight):  wait for plane i+1's copies -> convert them into U (u = make_u,
// PEC mask; own cells: convert_own) -> issue cp.async for plane i+2 -> H = ce(u) on the
// tile + low halo -> curl of H, epilogue.  Global loads of the box are asynchronous
// copies, so they overlap the arithmetic of the previous plane.
__device__ __forceinline__ void cp_async16(void* s, const void* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g));
}
__device__ __forceinline__ void cp_async8(void* s, const void* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <typename R>
__device__ __forceinline__ void cp_async_cx(cx<R>* s, const cx<R>* g) {
  if constexpr (sizeof(cx<R>) == 16) cp_async16(s, g);
  else cp_async8(s, g);
}

// Upper bound on x planes per CTA (per-CTA plane tables live in shared memory).
constexpr int XC_MAX = 64;
// Complex128 stencil reductions are summed over a fixed partition of the grid: one
// partial per (block of 2^rb_shift x planes, y/z tile), whatever the x chunk of the CTAs
// (chunks are whole blocks), so the sums, and the COCG iterates built on them, do not
// depend on the tiling.  The block size is a property of the grid (Geo::rb_shift): 8
// planes, or 4 on small grids, where x chunks of 4 planes keep more SMs busy.  Complex64
// passes keep one partial per CTA: their per-thread FP32 sums already depend on the
// order of the cells, and the per-block partials cost their short passes about 10 %.
template <typename R>
struct PartitionedSums : std::is_same<R, double> {};

template <typename R, int TZ, int TY, bool FLAT, int NB, int NO>
struct StencilShape {
  static constexpr int NT = TZ * TY;
  static constexpr int KZ = FLAT ? 0 : 1;      // z offset of own cells inside the box
  static constexpr int BW = TZ + 2 * KZ;       // box width (z)
  static constexpr int BH = TY + 2;            // box height (y)
  static constexpr int BOX = BW * BH;
  static constexpr int NHALO = BOX - NT;       // halo cells (<= NT)
  static constexpr int HW = TZ + KZ;           // H plane width (own + low z halo)
  static constexpr int HH = TY + 1;
  // shared memory: Sbox[NB][3][BOX] | Sown[NO][3][NT] | U[2][3][BOX] | Hs[3][HH*HW] | Xt | red[64]
  static constexpr size_t off_own = sizeof(cx<R>) * (size_t)NB * 3 * BOX;
  static constexpr size_t off_u = off_own + sizeof(cx<R>) * (size_t)NO * 3 * NT;
  static constexpr size_t off_h = off_u + sizeof(cx<R>) * (size_t)2 * 3 * BOX;
  static constexpr size_t off_xt = off_h + sizeof(cx<R>) * (size_t)3 * HH * HW;
  static constexpr int XT_STRIDE = 6;  // per plane: idxe, idxh, dxe, dxh, (|dxe|, |dxh|)
  static constexpr size_t off_red = off_xt + sizeof(cx<R>) * (size_t)XT_STRIDE * (XC_MAX + 1);
  // per-thread sums of a finished plane block ([NRED][NT], in the accumulator type)
  static constexpr size_t off_blk = off_red + 64 * sizeof(double);
  // complex128 passes only (see PartitionedSums); complex64 passes keep one partial per CTA
  static constexpr size_t smem_bytes(int nred) {
    return off_blk + (std::is_same<R, double>::value ? (size_t)nred * NT * sizeof(R) : (size_t)0);
  }
  static_assert(NHALO <= NT, "halo larger than the CTA");
};

// One work unit of a stencil pass: the x chunk `unit / (ntz * nty)` of the y/z tile
// `unit % (ntz * nty)`.  Writes the unit's reduction partials (one per plane block); the
// grid-wide sum and the op's finish() are the caller's.
template <typename R, int TZ, int TY, bool FLAT, class Op>
__device__ __forceinline__ void stencil_unit(const Geo<R>& g, const Op& o, RedBuf rb, int unit,
                                             unsigned char* smem_raw) {
  using S = StencilShape<R, TZ, TY, FLAT, Op::NB, Op::NO>;
  constexpr int NT = S::NT, BW = S::BW, BOX = S::BOX, KZ = S::KZ, HW = S::HW, HH = S::HH;
  constexpr int NB = Op::NB, NO = Op::NO;
  cx<R>* Sbox = reinterpret_cast<cx<R>*>(smem_raw);                 // [NB][3][BOX]
  cx<R>* Sown = reinterpret_cast<cx<R>*>(smem_raw + S::off_own);    // [NO][3][NT]
  cx<R>* U = reinterpret_cast<cx<R>*>(smem_raw + S::off_u);         // [2][3][BOX]
  cx<R>* Hs = reinterpret_cast<cx<R>*>(smem_raw + S::off_h);        // [3][HH*HW]
  cx<R>* Xt = reinterpret_cast<cx<R>*>(smem_raw + S::off_xt);       // [XC+1][6]
  using A = typename AccT<R>::type;
  A* shblk = reinterpret_cast<A*>(smem_raw + S::off_blk);         // [NRED][NT]

  const cx<R> w2 = *g.w2p;

  const int tz = threadIdx.x, ty = threadIdx.y, tid = tz + ty * TZ;
  int b = unit;
  const int tzb = b % g.ntz; b /= g.ntz;
  const int tyb = b % g.nty;
  const int xcb = b / g.nty;
  const int k0 = tzb * TZ, j0 = tyb * TY;
  const int x0 = xcb * g.XC;
  const int x1 = min(g.X, x0 + g.XC);
  const int j = j0 + ty, k = k0 + tz;
  const bool active = (j < g.Y) && (k < g.Z);
  const int jc = min(j, g.Y - 1), kc = min(k, g.Z - 1);
  const int YZ = (int)g.Y * g.Z;
  const int N = g.N;

  // slot 0: this thread's own box cell; slot 1: one halo cell (or none)
  const int pos0 = (ty + 1) * BW + tz + KZ;
  const int off0 = wrapi(j0 + ty, g.Y) * g.Z + (FLAT ? 0 : wrapi(k0 + tz, g.Z));
  int pos1 = -1, off1 = 0;
  if (tid < S::NHALO) {
    int bj, bk;
    if (FLAT) {
      bj = tid == 0 ? 0 : TY + 1;
      bk = 0;
    } else if (tid < BW) {
      bj = 0;
      bk = tid;
    } else if (tid < 2 * BW) {
      bj = TY + 1;
      bk = tid - BW;
    } else {
      const int hh = tid - 2 * BW;
      bj = 1 + hh / 2;
      bk = (hh & 1) ? BW - 1 : 0;
    }
    pos1 = bj * BW + bk;
    off1 = wrapi(j0 - 1 + bj, g.Y) * g.Z + (FLAT ? 0 : wrapi(k0 - KZ + bk, g.Z));
  }

  // per-thread y/z difference factors
  const cx<R> idye = g.idxe[1][jc], idyh = g.idxh[1][jc];
  const cx<R> idze = FLAT ? czero<R>() : g.idxe[2][kc];
  const cx<R> idzh = FLAT ? czero<R>() : g.idxh[2][kc];
  const int jm = wrapi(j0 - 1, g.Y);
  const int km = FLAT ? 0 : wrapi(k0 - 1, g.Z);
  const int kh = FLAT ? 0 : kc;
  // the low-y halo row (j0-1) is computed by warp-row ty == 0, the low-z halo column
  // (k0-1) by lanes tz < TY of the last warp-row (lane tz handles row j0 + tz)
  const bool row_halo = (ty == 0);
  const bool col_halo = !FLAT && (ty == TY - 1) && (tz < TY);
  const int jr = wrapi(j0 + (col_halo ? tz : 0), g.Y);
  const cx<R> idy_halo = row_halo ? g.idxe[1][jm] : (col_halo ? g.idxe[1][jr] : czero<R>());
  const cx<R> idze_km = FLAT ? czero<R>() : g.idxe[2][km];

  // per-plane x factors of this CTA's planes (plane x0-1 first) into shared memory
  for (int t = tid; t <= x1 - x0; t += NT) {
    const int iw = wrapi(x0 - 1 + t, g.X);
    cx<R>* e = Xt + t * S::XT_STRIDE;
    e[0] = g.idxe[0][iw];
    e[1] = g.idxh[0][iw];
    e[2] = g.dxe[0][iw];
    e[3] = g.dxh[0][iw];
    e[4] = mkc<R>(g.adxe[0][iw], g.adxh[0][iw]);
  }

  WeightYZ<R> wyz;
  if (Op::NEEDS_W) wyz.init(g, jc, kc);

  constexpr int NR = Op::NRED > 0 ? Op::NRED : 1;
  // acc: the current plane block; accn: convert_own terms of plane i+1, converted one step
  // ahead (folded into acc at the end of step i, or carried into the next block)
  A acc[NR], accn[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) acc[r] = accn[r] = A(0);
  // Partial of plane block `blk` (a block's warp sums wait in shred for the next barrier).
  // The tile number is recomputed from blockIdx where it is needed: no registers held.
  auto part_of = [&](int blk) -> size_t {
    const int bt = unit % (g.ntz * g.nty);
    return (size_t)blk * (size_t)(g.ntz * g.nty) + (size_t)bt;
  };

  // issue the asynchronous copies of plane iw's box inputs into Sbox
  auto issue = [&](int iw) {
    const int base = (int)iw * YZ;
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
      const cx<R>* src = o.box_src(bi);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cx<R>* dst = Sbox + (bi * 3 + c) * BOX;
        if (src) {
          cp_async_cx<R>(dst + pos0, src + c * N + base + off0);
          if (pos1 >= 0) cp_async_cx<R>(dst + pos1, src + c * N + base + off1);
        } else {
          dst[pos0] = czero<R>();
          if (pos1 >= 0) dst[pos1] = czero<R>();
        }
      }
    }
#pragma unroll
    for (int oi = 0; oi < NO; ++oi) {
      const cx<R>* src = o.own_src(oi);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cx<R>* dst = Sown + (oi * 3 + c) * NT + tid;
        if (src) cp_async_cx<R>(dst, src + c * N + base + off0);
        else *dst = czero<R>();
      }
    }
    cp_async_commit();
  };
  // convert the landed raw inputs of plane iw into U[buf]; own cells of the CTA's own
  // planes (own_plane) also run the op's convert_own
  auto convert = [&](int buf, int iw, bool own_plane, A* acc_to) {
    const int base = (int)iw * YZ;
#pragma unroll
    for (int sl = 0; sl < 2; ++sl) {
      const int pos = sl == 0 ? pos0 : pos1;
      if (pos < 0) continue;
      const int cell = base + (sl == 0 ? off0 : off1);
      const uint8_t m = g.mask ? g.mask[cell] : (uint8_t)0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cx<R> v[NB > 0 ? NB : 1];
#pragma unroll
        for (int bi = 0; bi < NB; ++bi) v[bi] = Sbox[(bi * 3 + c) * BOX + pos];
        const int idx = c * N + cell;
        cx<R> u = o.make_u(v, idx, c);
        if (m & (1u << c)) u = czero<R>();
        U[(buf * 3 + c) * BOX + pos] = u;
        if (sl == 0 && own_plane && active) {
          cx<R> ov[NO > 0 ? NO : 1];
#pragma unroll
          for (int oi = 0; oi < NO; ++oi) ov[oi] = Sown[(oi * 3 + c) * NT + tid];
          o.convert_own(v, ov, idx, c, u, acc_to);
        }
      }
    }
  };

  // H-grid scaling pm * mu^-1 at a cell, per component
  auto hscale = [&](int cell, cx<R>& hx, cx<R>& hy, cx<R>& hz) {
    if (g.muinv) {
      hx = g.muinv[cell] * hx;
      hy = g.muinv[N + cell] * hy;
      hz = g.muinv[2 * N + cell] * hz;
    }
    if (g.mask) {
      const uint8_t m = g.mask[cell];
      if (m & 8u) hx = czero<R>();
      if (m & 16u) hy = czero<R>();
      if (m & 32u) hz = czero<R>();
    }
  };

  // H = ce(u) on plane i at box position (bj, bk); cur/nxt = buffers of planes i, i+1
  auto curl_e = [&](int cur, int nxt, int bj, int bk, cx<R> idy, cx<R> idz, cx<R> idx_e,
                    cx<R>& hx, cx<R>& hy, cx<R>& hz) {
    const cx<R>* Ux = U + (cur * 3 + 0) * BOX;
    const cx<R>* Uy = U + (cur * 3 + 1) * BOX;
    const cx<R>* Uz = U + (cur * 3 + 2) * BOX;
    const int p = bj * BW + bk;
    const cx<R> ux = Ux[p], uy = Uy[p], uz = Uz[p];
    const cx<R> dyuz = (Uz[p + BW] - uz) * idy;
    const cx<R> dyux = (Ux[p + BW] - ux) * idy;
    const cx<R> dxuz = (U[(nxt * 3 + 2) * BOX + p] - uz) * idx_e;
    const cx<R> dxuy = (U[(nxt * 3 + 1) * BOX + p] - uy) * idx_e;
    if (FLAT) {
      hx = dyuz;
      hy = czero<R>() - dxuz;
      hz = dxuy - dyux;
    } else {
      const cx<R> dzuy = (Uy[p + 1] - uy) * idz;
      const cx<R> dzux = (Ux[p + 1] - ux) * idz;
      hx = dyuz - dzuy;
      hy = dzux - dxuz;
      hz = dxuy - dyux;
    }
  };

  // ---- prologue: planes x0-1 and x0 into U, H on plane x0-1 (own cells: Hy, Hz)
  const int ip = wrapi(x0 - 1, g.X);
  // (own slots only until the barrier: the barrier publishes Xt, U[0] and U[1])
  issue(ip);
  cp_async_wait_all();
  convert(0, ip, false, acc);
  issue(x0);
  cp_async_wait_all();
  convert(1, x0, true, acc);
  __syncthreads();
  // plane x0+1 starts landing while the prologue H is computed
  issue(x0 + 1 == g.X ? 0 : x0 + 1);
  cx<R> hy_prev, hz_prev;
  {
    cx<R> hx, hy, hz;
    curl_e(0, 1, ty + 1, tz + KZ, idye, idze, Xt[0], hx, hy, hz);
    hscale((int)ip * YZ + (int)jc * g.Z + kc, hx, hy, hz);
    hy_prev = hy;
    hz_prev = hz;
  }
  // The first step converts plane x0+1 into U[0]: every thread must be done reading
  // U[0] (plane x0-1) for the prologue H.  (Inside the loop the previous step's Hs
  // barrier gives this ordering.)
  __syncthreads();
  int cur = 1;
  for (int i = x0; i < x1; ++i) {
    const int nxt = cur ^ 1;
    const int in1 = (i + 1 == g.X) ? 0 : i + 1;
    const int ibase = (int)i * YZ;
    const int cell = ibase + (int)jc * g.Z + kc;
    // own-cell prefetch for this plane's epilogue (latency hidden by the H pass)
    typename Op::Pre pr;
    R e3[3];
    if (active) {
      o.pre(cell, pr);
#pragma unroll
      for (int c = 0; c < 3; ++c) e3[c] = g.eps[c * N + cell];
    }
    // Plane i+1's raw inputs landed.  No barrier is needed here: every thread copies and
    // converts only its own Sbox/Sown slots, U[nxt] (plane i-1) was last read before the
    // previous step's Hs barrier, and Hs is rewritten only after the barrier below.
    cp_async_wait_all();
    constexpr bool PART = PartitionedSums<R>::value && Op::NRED > 0;
    const int rbm = (1 << g.rb_shift) - 1;
    const bool block_end = ((i + 1) & rbm) == 0 || (i + 1 == x1);
    if constexpr (PART) convert(nxt, in1, i + 1 < x1, accn);
    else convert(nxt, in1, i + 1 < x1, acc);
    __syncthreads();       // U[nxt] = u(i+1) ready for the neighbours' differences
    if constexpr (PART) {
      // plane i-1 ended a block (chunks start on block boundaries): its per-thread sums
      // are visible now; warp 0 adds them up in a fixed order
      if (i > x0 && (i & ((1 << g.rb_shift) - 1)) == 0 && tid < 32)
        sum_block_partials<NT, Op::NRED>(shblk, rb, part_of((i >> g.rb_shift) - 1));
    }
    if (i + 1 < x1) issue(in1 + 1 == g.X ? 0 : in1 + 1);
    const cx<R>* xe = Xt + (i - x0 + 1) * S::XT_STRIDE;
    const cx<R> idxe_i = xe[0], idxh_i = xe[1];
    cx<R> hx, hy, hz;
    curl_e(cur, nxt, ty + 1, tz + KZ, idye, idze, idxe_i, hx, hy, hz);
    hscale(cell, hx, hy, hz);
    const int hp = (ty + 1) * HW + tz + KZ;
    Hs[0 * HH * HW + hp] = hx;
    Hs[1 * HH * HW + hp] = hy;
    Hs[2 * HH * HW + hp] = hz;
    if (row_halo) {  // low y halo row (j0-1)
      cx<R> ax, ay, az;
      curl_e(cur, nxt, 0, tz + KZ, idy_halo, idze, idxe_i, ax, ay, az);
      hscale(ibase + (int)jm * g.Z + kh, ax, ay, az);
      Hs[0 * HH * HW + tz + KZ] = ax;
      Hs[1 * HH * HW + tz + KZ] = ay;
      Hs[2 * HH * HW + tz + KZ] = az;
    }
    if (col_halo) {  // low z halo column (k0-1), row j0 + tz
      cx<R> ax, ay, az;
      curl_e(cur, nxt, tz + 1, 0, idy_halo, idze_km, idxe_i, ax, ay, az);
      hscale(ibase + (int)jr * g.Z + km, ax, ay, az);
      Hs[0 * HH * HW + (tz + 1) * HW] = ax;
      Hs[1 * HH * HW + (tz + 1) * HW] = ay;
      Hs[2 * HH * HW + (tz + 1) * HW] = az;
    }
    cx<R> u[3];
    u[0] = U[(cur * 3 + 0) * BOX + pos0];
    u[1] = U[(cur * 3 + 1) * BOX + pos0];
    u[2] = U[(cur * 3 + 2) * BOX + pos0];
    __syncthreads();
    const cx<R> hz_jm = Hs[2 * HH * HW + ty * HW + tz + KZ];
    const cx<R> hx_jm = Hs[0 * HH * HW + ty * HW + tz + KZ];
    cx<R> y[3];
    if (FLAT) {
      y[0] = (hz - hz_jm) * idyh;
      y[1] = czero<R>() - (hz - hz_prev) * idxh_i;
    } else {
      const cx<R> hy_km = Hs[1 * HH * HW + (ty + 1) * HW + tz];
      const cx<R> hx_km = Hs[0 * HH * HW + (ty + 1) * HW + tz];
      y[0] = (hz - hz_jm) * idyh - (hy - hy_km) * idzh;
      y[1] = (hx - hx_km) * idzh - (hz - hz_prev) * idxh_i;
    }
    y[2] = (hy - hy_prev) * idxh_i - (hx - hx_jm) * idyh;
    hy_prev = hy;
    hz_prev = hz;
    if (active) {
      const uint8_t m = g.mask ? g.mask[cell] : (uint8_t)0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cx<R> v = y[c] - (e3[c] * w2) * u[c];
        if (m & (1u << c)) v = czero<R>();
        y[c] = v;
      }
      cx<R> W[3];
      R aW[3];
      if (Op::NEEDS_W) wyz.at(xe[2], xe[3], xe[4].re, xe[4].im, W, aW);
      o.own(cell, i, j, k, u, y, W, aW, pr, acc);
    }
    if constexpr (PART) {
      if (block_end) {  // uniform over the CTA
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          shblk[r * NT + tid] = acc[r];
          acc[r] = accn[r];
        }
      } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] += accn[r];
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) accn[r] = A(0);
    }
    cur = nxt;
  }
  cp_async_wait_all();

  if constexpr (Op::NRED > 0) {
    if constexpr (PartitionedSums<R>::value) {
      __syncthreads();  // the last block's per-thread sums (plane x1 - 1 always ends a block)
      if (tid < 32) sum_block_partials<NT, Op::NRED>(shblk, rb, part_of((x1 - 1) >> g.rb_shift));
    } else {
      write_partial<NT, Op::NRED>(acc, rb, (size_t)unit, reinterpret_cast<double*>(smem_raw + S::off_red));
    }
  }
}

// Partial sums of a stencil reduction: one per (plane block, tile).
template <typename R>
__device__ __forceinline__ unsigned int stencil_nparts(const Geo<R>& g) {
  return (unsigned int)((g.X + (1 << g.rb_shift) - 1) >> g.rb_shift) * (unsigned int)(g.ntz * g.nty);
}

template <typename R, int TZ, int TY, bool FLAT, int MINB, class Op>
__global__ void __launch_bounds__(TZ * TY, MINB) k_stencil(const Geo<R> g, Op op, RedBuf rb) {
  using S = StencilShape<R, TZ, TY, FLAT, Op::NB, Op::NO>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (op.skip()) return;
  Op o = op;
  o.prepare();
  stencil_unit<R, TZ, TY, FLAT, Op>(g, o, rb, blockIdx.x, smem_raw);
  if constexpr (Op::NRED > 0) {
    double sums[Op::NRED];
    double* shred = reinterpret_cast<double*>(smem_raw + S::off_red);
    const unsigned int nparts = PartitionedSums<R>::value ? stencil_nparts(g) : gridDim.x;
    if (grid_finish<S::NT, Op::NRED>(rb, nparts, shred, sums)) run_finish(o, sums);
  }
}

// ---------------------------------------------------------------- pointwise engine
// Own cells only, no stencil.  Work units are (x plane, y/z tile) pairs, tiles fastest;
// the grid is sized to the GPU's resident CTA slots and CTA b takes units b, b + grid,
// b + 2 grid, ...  The assignment is fixed (the reductions stay deterministic) and every
// SM streams to the end instead of idling through a partial last wave.
//   void point(int cell, int i, int j, int k, const cx<R> W[3], const R aW[3], A* acc);
template <typename R, int TZ, int TY, class Op>
__device__ __forceinline__ void point_units(const Geo<R>& g, const Op& o, typename AccT<R>::type* acc) {
  const int tz = threadIdx.x, ty = threadIdx.y;
  const int ntiles = g.ntz * g.nty;
  const int units = ntiles * g.X;
  const int YZ = g.Y * g.Z;
  for (int u = blockIdx.x; u < units; u += gridDim.x) {
    const int i = u / ntiles, t = u - i * ntiles;
    const int tyb = t / g.ntz, tzb = t - tyb * g.ntz;
    const int j = tyb * TY + ty, k = tzb * TZ + tz;
    if (j < g.Y && k < g.Z) {
      cx<R> W[3];
      R aW[3];
      if (Op::NEEDS_W) {
        WeightYZ<R> wyz;
        wyz.init(g, j, k);
        wyz.at(g.dxe[0][i], g.dxh[0][i], g.adxe[0][i], g.adxh[0][i], W, aW);
      }
      o.point(i * YZ + j * g.Z + k, i, j, k, W, aW, acc);
    }
  }
}

template <typename R, int TZ, int TY, class Op>
__global__ void __launch_bounds__(TZ * TY) k_point(const Geo<R> g, Op op, RedBuf rb) {
  constexpr int NT = TZ * TY;
  __shared__ double shred[64];
  if (op.skip()) return;
  Op o = op;
  o.prepare();
  using A = typename AccT<R>::type;
  A acc[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
  for (int r = 0; r < (Op::NRED > 0 ? Op::NRED : 1); ++r) acc[r] = A(0);
  point_units<R, TZ, TY, Op>(g, o, acc);
  if constexpr (Op::NRED > 0) {
    double sums[Op::NRED];
    // (finish runs on the global state here: a state copy would cost this kernel occupancy)
    if (grid_reduce<NT, Op::NRED>(acc, rb, shred, sums)) o.finish(sums);
  }
}

}  // namespace fdfd
