// Non-RHS device kernels of the stepping path: the ghost fill (scatter, same-level copies,
// injection, the Dirichlet hook, tensor-product Lagrange prolongation), the RK4 stage
// updates of the plain form, the characteristic speed, the error norm, the analytic
// initial state, the :pasted overwrite and the sampled gauge source.
#pragma once
#include <cstdint>

#include "analytic.cuh"

namespace tgh {

// A run of points along x copied from a primary owner: the destination is a working array
// (block, linear work index), the source an owned point (block, i, j, k) of the state vector;
// step is 1 (same level) or 2^d (injection from a level d finer).
struct CopyRun {
  int dst_b, dst_w;
  int src_b, si, sj, sk;
  int len, step;
};
// One copied point of the batched form's fill: destination block and work index, source
// (primary) block and work index.
struct __align__(16) CopyPt {
  int dst_b, dst_w, src_b, src_w;
};
// One prolonged point: the destination, the coarse block, the coarse work index of the
// stencil box's lower corner and a bit per axis saying whether the axis interpolates.
struct ProlongPt {
  int dst_b, dst_w;
  int src_b, src_w;
  int odd;
};
// One Dirichlet ghost point: the destination; the position is recomputed from the block.
struct HookPt {
  int b, w;
};

// A block's working array per variable is Wd^3 points (the reference's ghosted cube) stored
// with rows of Wx >= Wd doubles (Wx even: every row starts on a 16-byte boundary, as the tensor
// copies into shared memory require); point (x, y, z) of the cube sits at x + Wx (y + Wd z).
struct Geo {
  int N1, Wd, G, Wx;
  long S, Wv;  // points per block in state layout; doubles per block and variable in work layout
};
__host__ __device__ __forceinline__ long work_index(const Geo& g, int x, int y, int z) {
  return x + (long)g.Wx * (y + (long)g.Wd * z);
}

// The position of point (i, j, k) of block b (i may lie in the ghost zone): blk holds per
// block the domain's low corner, the spacing and the integer corner, 8 doubles; the point
// is lo + (corner + i) h with the product and the sum each rounded.
__device__ __forceinline__ void point_pos(const double* blk, int b, int i, int j, int k, double* x) {
  const double* bl = blk + 8 * b;
  x[0] = __dadd_rn(bl[0], __dmul_rn(bl[4] + (double)i, bl[3]));
  x[1] = __dadd_rn(bl[1], __dmul_rn(bl[5] + (double)j, bl[3]));
  x[2] = __dadd_rn(bl[2], __dmul_rn(bl[6] + (double)k, bl[3]));
}

// stage 0 of the plain form's fill: the scatter of the state vector u into the working
// array and the copies into ghost points, one warp per run of points along x
static __global__ void fill_copy_kernel(const CopyRun* __restrict__ runs, int nruns, const double* __restrict__ u,
                                 double* __restrict__ work, Geo g) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nruns) return;
  const CopyRun r = runs[warp];
  for (int e = lane; e < r.len; e += 32) {
    const double* src = u + (long)r.src_b * NV * g.S + (r.si + e * r.step) + (long)g.N1 * (r.sj + (long)g.N1 * r.sk);
    double* dst = work + (long)r.dst_b * NV * g.Wv + r.dst_w + e;
#pragma unroll 4
    for (int v = 0; v < NV; ++v) dst[v * g.Wv] = src[v * g.S];
  }
}

// The copies of the batched form's fill, one thread per point: every ghost point with a
// primary owner, and every owned point held by a block that is not its primary, from the
// primary's working array (whose owned points the stage update has just written). A
// primary's own points are not listed: they already hold their value.
static __global__ void fill_points_kernel(const CopyPt* __restrict__ pts, long n, double* __restrict__ work, Geo g) {
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n) return;
  const CopyPt c = pts[id];
  const double* src = work + (long)c.src_b * NV * g.Wv + c.src_w;
  double* dst = work + (long)c.dst_b * NV * g.Wv + c.dst_w;
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = src[k * g.Wv];
#pragma unroll
  for (int k = 0; k < NV; ++k) dst[k * g.Wv] = v[k];
}

// the Dirichlet hook: the analytic state (through the core rule) at each outer ghost point;
// with `cache` (stationary cases) the values are also kept, 20 per point
static __global__ void fill_hook_kernel(const HookPt* __restrict__ pts, int n, const double* __restrict__ blk,
                                 double* __restrict__ work, Geo g, const Case cs, double t, double* cache) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n) return;
  const HookPt p = pts[id];
  const int i = p.w % g.Wx, j = (p.w / g.Wx) % g.Wd, k = p.w / (g.Wx * g.Wd);
  double x[3];
  point_pos(blk, p.b, i - g.G, j - g.G, k - g.G, x);
  double v20[NV];
  exact_state(cs, t, x, v20);
  double* dst = work + (long)p.b * NV * g.Wv + p.w;
#pragma unroll
  for (int v = 0; v < NV; ++v) dst[v * g.Wv] = v20[v];
  if (cache) {
#pragma unroll
    for (int v = 0; v < NV; ++v) cache[(long)v * n + id] = v20[v];
  }
}

// the Dirichlet hook of a stationary case from the values kept by fill_hook_kernel (variable
// after variable, so that consecutive points read and write consecutive doubles)
static __global__ void hook_copy_kernel(const HookPt* __restrict__ pts, int n, const double* __restrict__ cache,
                                 double* __restrict__ work, Geo g) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n) return;
  const HookPt p = pts[id];
  double* dst = work + (long)p.b * NV * g.Wv + p.w;
#pragma unroll
  for (int v = 0; v < NV; ++v) dst[v * g.Wv] = cache[(long)v * n + id];
}

// tensor-product Lagrange prolongation of order P from the coarse block's filled working
// array, summed with x innermost, then y, then z; products and sums rounded one by one

// The Lagrange weights of P points at the midpoint of the middle pair: exact rationals,
// w_k = prod_{m != k} (0 - x_m) / (x_k - x_m) with x_m = m - (P/2 - 1) - 1/2, numerator and
// denominator formed in integers (doubled units) and divided once.
template <int P> struct ProlongWeights {
  double v[P];
};
template <int P> __host__ __device__ constexpr ProlongWeights<P> prolong_weights() {
  ProlongWeights<P> r{};
  for (int k = 0; k < P; ++k) {
    long long num = 1, den = 1;
    for (int m = 0; m < P; ++m) {
      if (m == k) continue;
      const long long xm = 2 * (m - (P / 2 - 1)) - 1, xk = 2 * (k - (P / 2 - 1)) - 1;
      num *= -xm;
      den *= xk - xm;
    }
    r.v[k] = (double)num / (double)den;
  }
  return r;
}

// one variable's prolonged value from its coarse stencil base `src` along the odd axes ODD (a
// bit per axis): every loop and weight fixed at compile time. An axis that does not
// interpolate contributes its one value with weight 1 (the product is the value).
template <int P, int ODD> __device__ __forceinline__ double prolong_odd(const double* src, Geo g) {
  constexpr int cx = (ODD & 1) ? P : 1, cy = (ODD & 2) ? P : 1, cz = (ODD & 4) ? P : 1;
  constexpr ProlongWeights<P> W = prolong_weights<P>();
  const long sy = g.Wx, sz = (long)g.Wx * g.Wd;
  double szv = 0.0;
#pragma unroll
  for (int kz = 0; kz < cz; ++kz) {
    double syv = 0.0;
#pragma unroll
    for (int ky = 0; ky < cy; ++ky) {
      double sxv = 0.0;
      const double* row = src + kz * sz + ky * sy;
#pragma unroll
      for (int kx = 0; kx < cx; ++kx) {
        const double term = cx == 1 ? row[kx] : __dmul_rn(W.v[kx], row[kx]);
        sxv = kx == 0 ? term : __dadd_rn(sxv, term);
      }
      const double ty = cy == 1 ? sxv : __dmul_rn(W.v[ky], sxv);
      syv = ky == 0 ? ty : __dadd_rn(syv, ty);
    }
    const double tz = cz == 1 ? syv : __dmul_rn(W.v[kz], syv);
    szv = kz == 0 ? tz : __dadd_rn(szv, tz);
  }
  return szv;
}

// the same for a run-time mask (the point lists are grouped by mask, so a warp takes one case)
template <int P> __device__ __forceinline__ double prolong_value(const double* src, int odd, Geo g) {
  switch (odd) {
    case 1: return prolong_odd<P, 1>(src, g);
    case 2: return prolong_odd<P, 2>(src, g);
    case 3: return prolong_odd<P, 3>(src, g);
    case 4: return prolong_odd<P, 4>(src, g);
    case 5: return prolong_odd<P, 5>(src, g);
    case 6: return prolong_odd<P, 6>(src, g);
    case 7: return prolong_odd<P, 7>(src, g);
    default: return prolong_odd<P, 0>(src, g);
  }
}

// The regrid's transfer (the fill's operators between two forests): the value of every owned
// point of the new forest, copied from the old filled working array or prolonged from it,
// into a state vector (S points per block and variable)
static __global__ void transfer_copy_kernel(const CopyPt* __restrict__ pts, long n, const double* __restrict__ work,
                                     Geo g, double* __restrict__ u, long S) {
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n) return;
  const CopyPt c = pts[id];
  const double* src = work + (long)c.src_b * NV * g.Wv + c.src_w;
  double* dst = u + (long)c.dst_b * NV * S + c.dst_w;
#pragma unroll
  for (int v = 0; v < NV; ++v) dst[v * S] = src[v * g.Wv];
}
// one thread per (point, variable), consecutive threads on consecutive points of one variable:
// their coarse stencils are neighbours in memory (the lists are grouped by odd-axis mask, so a
// warp's points do the same amount of work)
template <int P>
static __global__ void transfer_prolong_kernel(const ProlongPt* __restrict__ pts, int n, const double* __restrict__ work,
                                        Geo g, double* __restrict__ u, long S) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n * NV) return;
  const int pi = id % n, v = id / n;
  const ProlongPt p = pts[pi];
  u[(long)p.dst_b * NV * S + (long)v * S + p.dst_w] =
      prolong_value<P>(work + (long)p.src_b * NV * g.Wv + (long)v * g.Wv + p.src_w, p.odd, g);
}

template <int P>
static __global__ void fill_prolong_kernel(const ProlongPt* __restrict__ pts, int n, double* __restrict__ work, Geo g) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n * NV) return;
  const int pi = id % n, v = id / n;
  const ProlongPt p = pts[pi];
  work[(long)p.dst_b * NV * g.Wv + (long)v * g.Wv + p.dst_w] =
      prolong_value<P>(work + (long)p.src_b * NV * g.Wv + (long)v * g.Wv + p.src_w, p.odd, g);
}

// The prolongation sum-factorised over tiles: the prolonged points of one fine block whose
// stencils lie in one coarse block, cut into boxes of 8 x 8 x 8 fine points aligned to the
// block's corner. A point's value is the per-point order above - for each coarse z, for each
// coarse y, the x sum; the y sum of those; the z sum - and every partial sum of that order
// depends only on the fine x (the x sums), on the fine x and y (the y sums) and the coarse rows
// it is taken over, so the tile forms each partial sum once, in shared memory, and all its
// points read them: stage X over (fine x, coarse y, coarse z), stage Y over (fine x, fine y,
// coarse z), stage Z at the listed points. Rounding and order per point are the per-point
// kernel's, operation for operation, so both give the same bits.
struct ProlongTile {
  int dst_b, src_b;
  short i0, j0, k0;     // the fine working-array coordinates of the tile's origin (may lie below 0)
  short cxb, cyb, czb;  // coarse working-array coordinate of the centre of fine offset 0
  short xlo, xhi;       // the coarse x its listed points' stencils read
  short ylo, zlo;       // the coarse rows stage X covers: [ylo, ylo + cyn) x [zlo, zlo + czn)
  unsigned char cyn, czn;
  unsigned char par;    // bit d: the fine lattice index of the origin is odd along axis d
  unsigned char fxm, fym;  // the fine x (y) offsets holding listed points, a bit each
  unsigned char nfx;
  int fxs;              // the same fine x offsets as a list, 3 bits each
  int p0, np;           // the listed points: pts[p0 .. p0 + np), fx | fy << 3 | fz << 6
};

template <int P>
__device__ __forceinline__ double lagrange_sum(const double* v, int stride) {
  constexpr ProlongWeights<P> W = prolong_weights<P>();
  double s = __dmul_rn(W.v[0], v[0]);
#pragma unroll
  for (int k = 1; k < P; ++k) s = __dadd_rn(s, __dmul_rn(W.v[k], v[k * stride]));
  return s;
}

// The partial sums along one axis at the 8 fine offsets of a tile from P + 3 consecutive coarse
// values v (v[0] at the centre of fine offset 0 minus P/2 - 1): offset f, with the origin's parity
// PAR, sits at coarse centre (PAR + f) >> 1 and interpolates where PAR + f is odd. Only the offsets
// in `mask` are written (out[f * stride]); every index is a compile-time constant.
template <int P, int PAR>
__device__ __forceinline__ void tile_axis_sums(const double* v, unsigned mask, double* out, int stride) {
  constexpr int H = P / 2 - 1;
#pragma unroll
  for (int f = 0; f < 8; ++f) {
    if (!((mask >> f) & 1)) continue;
    const int c = H + ((PAR + f) >> 1);
    out[f * stride] = ((PAR + f) & 1) ? lagrange_sum<P>(v + c - H, 1) : v[c];
  }
}

// One CTA per tile, its threads on one variable at a time: stage X a thread per coarse row (y, z),
// the row's P + 3 coarse values loaded once and every listed fine x formed from them; stage Y a
// thread per (fine x, coarse z), the column's P + 3 x sums read once; stage Z a thread per listed
// point. The shared arrays' rows have an odd pitch (no bank conflicts between neighbouring
// threads); at most 19.7 KB at P = 10.
constexpr int PROLONG_TILE_THREADS = 128;

template <int P>
static __global__ void __launch_bounds__(PROLONG_TILE_THREADS, 8)
    fill_prolong_tile_kernel(const ProlongTile* __restrict__ tiles, const unsigned short* __restrict__ pts,
                             double* __restrict__ work, Geo g) {
  constexpr int C = P + 4, CP = C | 1, H = P / 2 - 1, NVAL = P + 3;
  __shared__ double X[8 * CP * CP];  // [fx][cz][cy]
  __shared__ double Y[8 * 8 * CP];   // [fy][fx][cz]
  const ProlongTile T = tiles[blockIdx.x];
  const int px = T.par & 1, py = (T.par >> 1) & 1, pz = (T.par >> 2) & 1;
  const long sy = g.Wx, sz = (long)g.Wx * g.Wd;
  const int nrow = T.cyn * T.czn, ncol = T.nfx * T.czn;
  for (int v = 0; v < NV; ++v) {
    const double* src = work + (long)T.src_b * NV * g.Wv + (long)v * g.Wv;
    // stage X: per coarse row (y, z) the x sums at every listed fine x
    for (int e = threadIdx.x; e < nrow; e += PROLONG_TILE_THREADS) {
      const int cyi = e % T.cyn, czi = e / T.cyn;
      const int x0 = T.cxb - H;
      const double* row = src + x0 + sy * (T.ylo + cyi) + sz * (T.zlo + czi);
      double val[NVAL];
#pragma unroll
      for (int k = 0; k < NVAL; ++k) val[k] = (x0 + k >= T.xlo && x0 + k <= T.xhi) ? row[k] : 0.0;
      double* out = X + czi * CP + cyi;
      if (px)
        tile_axis_sums<P, 1>(val, T.fxm, out, CP * CP);
      else
        tile_axis_sums<P, 0>(val, T.fxm, out, CP * CP);
    }
    __syncthreads();
    // stage Y: per (listed fine x, coarse z) the y sums at every listed fine y
    for (int e = threadIdx.x; e < ncol; e += PROLONG_TILE_THREADS) {
      const int czi = e % T.czn, kx = e / T.czn;
      const int fx = (T.fxs >> (3 * kx)) & 7;
      const int y0 = T.cyb - H - T.ylo;  // column index of val[0]
      const double* col = X + (fx * CP + czi) * CP;
      double val[NVAL];
#pragma unroll
      for (int k = 0; k < NVAL; ++k) val[k] = (y0 + k >= 0 && y0 + k < T.cyn) ? col[y0 + k] : 0.0;
      double* out = Y + fx * CP + czi;
      if (py)
        tile_axis_sums<P, 1>(val, T.fym, out, 8 * CP);
      else
        tile_axis_sums<P, 0>(val, T.fym, out, 8 * CP);
    }
    __syncthreads();
    // stage Z: the z sum at the listed points, written into the fine block (the next
    // variable's stage X writes X only after every thread has passed the barrier above, and its
    // stage Y writes Y only after the barrier that ends that stage X)
    double* dst = work + (long)T.dst_b * NV * g.Wv + (long)v * g.Wv;
    for (int e = threadIdx.x; e < T.np; e += PROLONG_TILE_THREADS) {
      const int c = pts[T.p0 + e];
      const int fx = c & 7, fy = (c >> 3) & 7, fz = (c >> 6) & 7, nz = pz + fz;
      const double* col = Y + (fy * 8 + fx) * CP + (T.czb + (nz >> 1) - T.zlo);
      dst[(T.i0 + fx) + sy * (T.j0 + fy) + sz * (T.k0 + fz)] = (nz & 1) ? lagrange_sum<P>(col - H, 1) : col[0];
    }
  }
}

// plain-form RK4 stage updates over the whole state vector (each one fused multiply-add):
//  kind 0: acc = u + cb k, y = u + ca k   kind 1: acc = acc + cb k, y = u + ca k
//  kind 2: u = acc + cb k
static __global__ void stage_update_kernel(int kind, long n, const double* __restrict__ k, const double* __restrict__ u0,
                                    double* __restrict__ acc, double* __restrict__ y, double* __restrict__ uout,
                                    double ca, double cb) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double kv = k[i];
    if (kind == 0) {
      const double uv = u0[i];
      acc[i] = fma(cb, kv, uv);
      y[i] = fma(ca, kv, uv);
    } else if (kind == 1) {
      acc[i] = fma(cb, kv, acc[i]);
      y[i] = fma(ca, kv, u0[i]);
    } else {
      uout[i] = fma(cb, kv, acc[i]);
    }
  }
}

// The speed lambda = alpha sqrt(tr gamma^{ij}) + |beta| at every evolved owned point and the
// count of non-finite evolved values; reduced per CTA into scratch[0] (max, as the ordered
// bits of a non-negative double or a NaN) and scratch[1] (count).
static __global__ void speed_kernel(const double* __restrict__ u, const double* __restrict__ blk, Geo g, long npts,
                             const Case cs, double t, unsigned long long* scratch) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double lam = 0.0;
  unsigned long long bad = 0;
  if (p < npts) {
    const int b = (int)(p / g.S);
    const long ip = p - (long)b * g.S;
    const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
    double x[3];
    point_pos(blk, b, i, j, k, x);
    if (evolved(cs, t, x)) {
      const double* q = u + (long)b * NV * g.S + ip;
      double hv[NC];
      for (int v = 0; v < NV; ++v) {
        const double a = q[v * g.S];
        if (!isfinite(a)) ++bad;
        if (v < NC) hv[v] = a;
      }
      Coef<double> C;
      metric_quantities(hv, C);
      lam = C.alpha * sqrt(C.gamu[0] + C.gamu[3] + C.gamu[5]) +
            sqrt(C.beta[0] * C.beta[0] + C.beta[1] * C.beta[1] + C.beta[2] * C.beta[2]);
    }
  }
  unsigned long long bits = isnan(lam) ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(lam);
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long ob = __shfl_down_sync(0xffffffffu, bits, o);
    unsigned long long obad = __shfl_down_sync(0xffffffffu, bad, o);
    bits = ob > bits ? ob : bits;
    bad += obad;
  }
  if ((threadIdx.x & 31) == 0) {
    if (bits) atomicMax(scratch, bits);
    if (bad) atomicAdd(scratch + 1, bad);
  }
}

// |u - u_exact| over the evolved primaries of the settled working array: per point the
// squared magnitude weighted by h^3, the weight and the magnitude; per CTA partial sums in
// a fixed order into part[3 * blockIdx.x + {0,1,2}] (sum e^2 h^3, sum h^3, max e)
static __global__ void error_kernel(const double* __restrict__ work, const double* __restrict__ blk,
                             const uint8_t* __restrict__ primary, Geo g, long npts, const Case cs, double t,
                             double* part) {
  __shared__ double sh[3][128];
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double s2 = 0.0, vol = 0.0, mx = 0.0;
  if (p < npts && primary[p]) {
    const int b = (int)(p / g.S);
    const long ip = p - (long)b * g.S;
    const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
    double x[3];
    point_pos(blk, b, i, j, k, x);
    if (evolved(cs, t, x)) {
      double ex[NV];
      exact_state(cs, t, x, ex);
      const double* q = work + (long)b * NV * g.Wv + work_index(g, i + g.G, j + g.G, k + g.G);
      double e2 = 0.0;
      for (int v = 0; v < NV; ++v) {
        const double d = q[v * g.Wv] - ex[v];
        e2 = __dadd_rn(e2, __dmul_rn(d, d));
      }
      const double e = sqrt(e2);
      const double h = blk[8 * b + 3];
      const double w = h * h * h;
      s2 = e * e * w;
      vol = w;
      mx = e;
    }
  }
  sh[0][threadIdx.x] = s2;
  sh[1][threadIdx.x] = vol;
  sh[2][threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
      sh[2][threadIdx.x] = fmax(sh[2][threadIdx.x], sh[2][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = sh[0][0];
    part[3 * blockIdx.x + 1] = sh[1][0];
    part[3 * blockIdx.x + 2] = sh[2][0];
  }
}
static __global__ void error_final_kernel(const double* part, int n, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s2 = 0.0, vol = 0.0, mx = 0.0;
  for (int i = 0; i < n; ++i) {
    s2 += part[3 * i];
    vol += part[3 * i + 1];
    mx = fmax(mx, part[3 * i + 2]);
  }
  out[0] = vol == 0.0 ? 0.0 : sqrt(s2 / vol);
  out[1] = mx;
}

// the case's state at every owned point (initial_state!); paste_only: only inside r_1 (the
// :pasted limiter, gh_paste_kernel!)
static __global__ void exact_state_kernel(double* __restrict__ u, const double* __restrict__ blk, Geo g, long npts,
                                   const Case cs, double t, int paste_only) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int b = (int)(p / g.S);
  const long ip = p - (long)b * g.S;
  const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
  double x[3];
  point_pos(blk, b, i, j, k, x);
  if (paste_only && interior_radius(cs, t, x) >= cs.r1) return;
  double v20[NV];
  exact_state(cs, t, x, v20);
  double* q = u + (long)b * NV * g.S + ip;
#pragma unroll
  for (int v = 0; v < NV; ++v) q[v * g.S] = v20[v];
}

// The :fitted target cache's fills (40 fields per block: the target A, then its slope S), at every
// owned point with r < r_fill about the interior's centre at t_f, zero elsewhere: with u, the
// snapshot target (snapshot_target_kernel!, src/fit.jl:1189-1212: A = u, S = 0); without, the
// case's analytic state standing in for the fit of fit_target_kernel! (src/fit.jl:1070-1116): A
// at t_f (core rule included) and, with dt > 0, S = (A(t_f + dt) - A(t_f - dt)) / (2 dt) as the
// product with 1 / (2 dt). One analytic evaluation per launch and point: phase 0 writes A (and
// S = 0), phase 1 parks A(t_f + dt) in the S fields, phase 2 turns them into the slope with
// A(t_f - dt); the region is always the one at t_f.
static __global__ void fill_target_kernel(double* __restrict__ tw, const double* __restrict__ u,
                                          const double* __restrict__ blk, Geo g, long npts, const Case cs,
                                          double t_f, double r_fill, double dt, int phase) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int b = (int)(p / g.S);
  const long ip = p - (long)b * g.S;
  const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
  double x[3];
  point_pos(blk, b, i, j, k, x);
  double* o = tw + (long)b * 2 * NV * g.S + ip;
  if (!(interior_radius(cs, t_f, x) < r_fill)) {
    if (phase == 0)
      for (int v = 0; v < 2 * NV; ++v) o[v * g.S] = 0.0;
    return;
  }
  if (u) {
    const double* q = u + (long)b * NV * g.S + ip;
    for (int v = 0; v < NV; ++v) {
      o[v * g.S] = q[v * g.S];
      o[(NV + v) * g.S] = 0.0;
    }
    return;
  }
  double a[NV];
  if (phase == 0) {
    exact_state(cs, t_f, x, a);
    for (int v = 0; v < NV; ++v) {
      o[v * g.S] = a[v];
      o[(NV + v) * g.S] = 0.0;
    }
  } else if (phase == 1) {
    exact_state(cs, TGH_RADD(t_f, dt), x, a);
    for (int v = 0; v < NV; ++v) o[(NV + v) * g.S] = a[v];
  } else {
    exact_state(cs, TGH_RSUB(t_f, dt), x, a);
    const double id = TGH_RDIV(1.0, TGH_RMUL(2.0, dt));
    for (int v = 0; v < NV; ++v) o[(NV + v) * g.S] = TGH_RMUL(id, TGH_RSUB(o[(NV + v) * g.S], a[v]));
  }
}

// fitted_state_kernel! (src/fit.jl:1247-1285) without the blend: the background's state where
// r >= r_1 - d_init, below it the cached target at t, A + (t - t_f) S (each operation rounded, as
// the oracle forms it)
static __global__ void fitted_state_kernel(double* __restrict__ u, const double* __restrict__ blk, Geo g, long npts,
                                           const Case cs, double t, double d_init) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int b = (int)(p / g.S);
  const long ip = p - (long)b * g.S;
  const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
  double x[3];
  point_pos(blk, b, i, j, k, x);
  double* q = u + (long)b * NV * g.S + ip;
  if (interior_radius(cs, t, x) >= TGH_RSUB(cs.r1, d_init)) {
    double v20[NV];
    rn_background_state(cs, t, x, v20, v20 + NC);
    for (int v = 0; v < NV; ++v) q[v * g.S] = v20[v];
    return;
  }
  const double* tw = cs.tw + (long)b * 2 * NV * g.S + ip;
  const double dt = TGH_RSUB(t, *cs.tf);
  for (int v = 0; v < NV; ++v) q[v * g.S] = TGH_RADD(tw[v * g.S], TGH_RMUL(dt, tw[(NV + v) * g.S]));
}

static __global__ void set_scalar_kernel(double* dst, double v) { *dst = v; }

// the sampled gauge source at every owned point, through the core rule (src/gauge.jl:156-170)
static __global__ void sample_gauge_kernel(double* __restrict__ H, const double* __restrict__ blk, Geo g, long npts,
                                    const Case cs, double t) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int b = (int)(p / g.S);
  const long ip = p - (long)b * g.S;
  const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
  double x[3], xc[3], v20[NV];
  point_pos(blk, b, i, j, k, x);
  core_position(cs, t, x, xc);
  gauge_tuple(cs, t, xc, v20);
  double* q = H + (long)b * NV * g.S + ip;
  for (int v = 0; v < NV; ++v) q[v * g.S] = v20[v];
}

// owned values of the working array back to the state vector (the batched form's output)
static __global__ void gather_kernel(const double* __restrict__ work, double* __restrict__ u, Geo g, long npts) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int b = (int)(p / g.S);
  const long ip = p - (long)b * g.S;
  const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
  const double* q = work + (long)b * NV * g.Wv + work_index(g, i + g.G, j + g.G, k + g.G);
  double* o = u + (long)b * NV * g.S + ip;
#pragma unroll
  for (int v = 0; v < NV; ++v) o[v * g.S] = q[v * g.Wv];
}

// the owned points of the first npts / S blocks of a working array from the state vector u
static __global__ void scatter_owned_kernel(const double* __restrict__ u, double* __restrict__ work, Geo g, long npts) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int b = (int)(p / g.S);
  const long ip = p - (long)b * g.S;
  const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
  double* q = work + (long)b * NV * g.Wv + work_index(g, i + g.G, j + g.G, k + g.G);
  const double* s = u + (long)b * NV * g.S + ip;
#pragma unroll
  for (int v = 0; v < NV; ++v) q[v * g.Wv] = s[v * g.S];
}

// The exchange of a sharded fill: the listed (block, work index) points of a working array
// packed into, or unpacked from, a buffer of 20 values per point (point-major), one thread per
// value.
static __global__ void pack_kernel(const HookPt* __restrict__ pts, long n, const double* __restrict__ work, Geo g,
                            double* __restrict__ buf) {
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n * NV) return;
  const HookPt pt = pts[id / NV];
  buf[id] = work[(long)pt.b * NV * g.Wv + (id % NV) * g.Wv + pt.w];
}
static __global__ void unpack_kernel(const HookPt* __restrict__ pts, long n, const double* __restrict__ buf,
                              double* __restrict__ work, Geo g) {
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n * NV) return;
  const HookPt pt = pts[id / NV];
  work[(long)pt.b * NV * g.Wv + (id % NV) * g.Wv + pt.w] = buf[id];
}

// The masked error norm's sums and their tangents over the evolved primaries
// (src/constraints.jl:311-396): per CTA sum w e^2, sum w e.de and sum w, w = h^3,
// e = |u - u_exact| over the 20 variables.
static __global__ void error_tangent_kernel(const double* __restrict__ work, const double* __restrict__ twork,
                                     const double* __restrict__ blk, const uint8_t* __restrict__ primary, Geo g,
                                     long npts, const Case cs, double t, double* part) {
  __shared__ double sh[3][128];
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double a = 0.0, b = 0.0, vol = 0.0;
  if (p < npts && primary[p]) {
    const int bk = (int)(p / g.S);
    const long ip = p - (long)bk * g.S;
    const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
    double x[3];
    point_pos(blk, bk, i, j, k, x);
    if (cs.interior == TGH_INT_NONE || interior_radius(cs, t, x) >= cs.r1) {
      double ex[NV];
      exact_state(cs, t, x, ex);
      const long o = (long)bk * NV * g.Wv + work_index(g, i + g.G, j + g.G, k + g.G);
      double e2 = 0.0, ed = 0.0;
      for (int v = 0; v < NV; ++v) {
        const double d = work[o + v * g.Wv] - ex[v];
        e2 = __dadd_rn(e2, __dmul_rn(d, d));
        ed = fma(d, twork[o + v * g.Wv], ed);
      }
      const double h = blk[8 * bk + 3];
      vol = h * h * h;
      a = e2 * vol;
      b = ed * vol;
    }
  }
  sh[0][threadIdx.x] = a;
  sh[1][threadIdx.x] = b;
  sh[2][threadIdx.x] = vol;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
      sh[2][threadIdx.x] += sh[2][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = sh[0][0];
    part[3 * blockIdx.x + 1] = sh[1][0];
    part[3 * blockIdx.x + 2] = sh[2][0];
  }
}

// the tangent working array's Dirichlet ghosts: the analytic data do not depend on the
// parameters or the initial perturbation, so their tangent is zero
static __global__ void hook_zero_kernel(const HookPt* __restrict__ pts, int n, double* __restrict__ work, Geo g) {
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (long)n * NV) return;
  const HookPt p = pts[id / NV];
  work[(long)p.b * NV * g.Wv + (id % NV) * g.Wv + p.w] = 0.0;
}

// one point's analytic state (20) and gauge tuple (20), for diagnostics
static __global__ void point_physics_kernel(const Case cs, double t, const double* x, double* out) {
  exact_state(cs, t, x, out);
  gauge_tuple(cs, t, x, out + NV);
}

// sustained FP64 fused multiply-add throughput probe: 8 independent chains per thread
static __global__ void fp64_probe_kernel(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
  double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.0) out[0] = s;
}

}  // namespace tgh
