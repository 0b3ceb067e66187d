// The Pi half of the right-hand side (src/evolution.jl:324-354) with its stencil inputs staged
// into shared memory by the Tensor Memory Accelerator: the B200 form of rhs_pi_kernel for
// blocks of N = 32 cells at q = 4.
//
// A CTA owns a tile of one block: the whole x extent (33 points), 11 rows in y and 2 planes
// in z (3 x 17 = 51 tiles per block; the last z tile's second plane lies past the block and is
// computed and dropped). 12 warps per CTA: 3 per SM sub-partition leave 168 registers a thread,
// enough for two points' coefficients without spilling. For each component v in turn, one thread
// issues two tiled tensor copies of the block's working array into shared memory:
//   h_v   x -2..47, the tile's rows and planes widened by SR = 2 (50 x 15 x 6 doubles)
//   Pi_v  x -2..47, widened by KR = 3 for the dissipation      (50 x 17 x 8 doubles)
// completing on an mbarrier; two such stages alternate, so that the copies of component v + 1
// run while component v is computed. The boxes are 50 doubles wide (the rows used are 44): a
// row pitch of 25 sixteen-byte units, 1 modulo the 8 bank groups of a 128-byte shared-memory
// wavefront, keeps the 16-byte loads of a warp whose lanes cross from one row to the next free
// of bank conflicts. Each thread computes two neighbouring points along x,
// (i0, i0 + 1) with i0 = -1, 1, ..., 31, from 16-byte shared-memory loads: one load serves
// both points of every y and z tap and two x taps, so a point costs about 34 shared loads per
// component against the 80 global loads of the one-point kernel. The point i = -1 of the first
// pair is a ghost: it is computed and dropped.
//
// The arithmetic is the one-point kernel's, operation for operation (the same stencil sums in
// the same order and the same contraction with the head's coefficients), so both kernels give
// the same bits.
//
// Waits on the mbarriers are bounded: a wait that gives up records TGH_ERR_TIMEOUT in the
// launch's status word, waits (bounded again) for the copies it issued to land, and the CTA
// returns without writing; the host reads the word after the step.
#pragma once
#include <cuda.h>

#include "rhs.cuh"

namespace tgh {

namespace pitma {
constexpr int N1 = 33, G = 3, SR = 2, KR = 3;  // q = 4, N = 32
constexpr int TY = 11, TZ = 2, NPAIR = 17;
constexpr int XB = 50;                                   // box width: x = -2 .. 47 (see below)
constexpr int HY = TY + 2 * SR, HZ = TZ + 2 * SR;          // 15, 6
constexpr int PY = TY + 2 * KR, PZ = TZ + 2 * KR;        // 17, 8
constexpr int HN = XB * HY * HZ, PN = XB * PY * PZ;      // doubles per box
constexpr int HBYTES = HN * 8, PBYTES = PN * 8;
constexpr int HOFF = 0;                                  // byte offsets inside one stage
constexpr int POFF = ((HBYTES + 127) / 128) * 128;
constexpr int STAGE = ((POFF + PBYTES + 127) / 128) * 128;
constexpr int SMEM = 2 * STAGE + 256;                    // two stages, the mbarriers, alignment
constexpr int THREADS = 384;                             // 17 x 11 x 2 = 374 pair threads, 12 warps
constexpr int TILESY = N1 / TY, TILESZ = (N1 + TZ - 1) / TZ;
constexpr int TILES = TILESY * TILESZ;                   // 3 x 17 = 51 per block
static_assert(N1 % TY == 0, "the y tiles cover a block exactly");
static_assert(SMEM <= 227 * 1024, "two stages fit in shared memory");
}  // namespace pitma

// The tensor maps one launch reads: the working array viewed as 4-d (x, y, z, block x 20 +
// variable), with the h box and the Pi box.
struct PiTmaMaps {
  CUtensorMap h, pi;
};

struct PiTmaStatus {
  int* err;         // TGH_ERR_TIMEOUT is stored here by a wait that gives up
  long long limit;  // polls a wait may make (negative: give up at once, which tests use)
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait on one phase of an mbarrier: false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, long long limit) {
  for (long long it = 0; it <= limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap* map, int x, int y, int z, int c,
                                            unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(bar)
      : "memory");
}

// issue component v's two boxes for tile (b, y0, z0) into stage st
__device__ __forceinline__ void pitma_issue(const PiTmaMaps& M, unsigned base, unsigned bar, int st, int b, int v,
                                           int y0, int z0) {
  using namespace pitma;
  const unsigned s = base + st * STAGE;
  mbar_expect_tx(bar, HBYTES + PBYTES);
  // h: rows y0 + G - SR .., planes z0 + G - SR ..; Pi: widened by KR
  tma_load_4d(s + HOFF, &M.h, -2, y0 + G - SR, z0 + G - SR, b * NV + v, bar);
  tma_load_4d(s + POFF, &M.pi, -2, y0 + G - KR, z0 + G - KR, b * NV + NC + v, bar);
}

template <bool DISS, int MODE>
__global__ void __launch_bounds__(pitma::THREADS)
    rhs_pi_tma_kernel(const Case cs, const RhsArgs A, const __grid_constant__ PiTmaMaps M, const PiTmaStatus stat,
                      int b0) {
  using namespace pitma;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int b = b0 + blockIdx.x / TILES;
  const int tile = blockIdx.x % TILES;
  const int y0 = (tile % TILESY) * TY, z0 = (tile / TILESY) * TZ;
  // the copies land on 128-byte boundaries
  const unsigned raw = smem_u32(smem_raw);
  const unsigned base = (raw + 127u) & ~127u;
  unsigned char* smem = smem_raw + (base - raw);
  const unsigned bar0 = base + 2 * STAGE, bar1 = bar0 + 8;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    pitma_issue(M, base, bar0, 0, b, 0, y0, z0);
    pitma_issue(M, base, bar1, 1, b, 1, y0, z0);
  }
  __syncthreads();

  // this thread's pair: x = i0, i0 + 1 (i0 = -1, 1, ..., 31), row j, plane k of the block
  const bool active = tid < NPAIR * TY * TZ;
  const int ip = tid % NPAIR, jj = (tid / NPAIR) % TY, kk = tid / (NPAIR * TY);
  const int i0 = 2 * ip - 1;
  const int j = y0 + jj, k = z0 + kk;
  const int sx = i0 + G + 2;                      // shared column of point i0 (even)
  const int cH = sx + XB * ((jj + SR) + HY * (kk + SR));
  const int cP = sx + XB * ((jj + KR) + PY * (kk + KR));
  const long S = (long)N1 * N1;
  const long S3 = S * N1;
  const int Wd = N1 + 2 * G, Wx = Wd + 1;
  const long sv = (long)Wx * Wd * Wd;
  // the two points: state index, working index, and whether each is computed here
  long pidx[2], wo[2];
  bool own[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int i = i0 + e;
    own[e] = active && i >= 0 && k < N1;  // the last z tile's second plane lies past the block
    const int ic = i < 0 ? 0 : i, kc = k < N1 ? k : N1 - 1;
    pidx[e] = (long)b * S3 + ic + N1 * (j + (long)N1 * kc);
    wo[e] = (long)b * NV * sv + (ic + G) + (long)Wx * ((j + G) + (long)Wd * (kc + G));
  }
  const double* cf0 = A.coef + pidx[0];
  const double* cf1 = A.coef + pidx[1];
  double w[2];
  w[0] = own[0] ? cf0[CF_W * A.npts] : -1.0;
  w[1] = own[1] ? cf1[CF_W * A.npts] : -1.0;
  const bool live0 = w[0] >= 0.0, live1 = w[1] >= 0.0;
  double cb[2][14];
#pragma unroll
  for (int c = 0; c < 14; ++c) {
    cb[0][c] = live0 ? cf0[c * A.npts] : 0.0;
    cb[1][c] = live1 ? cf1[c * A.npts] : 0.0;
  }
  const double inv_h = 1.0 / A.blk[8 * b + 3];
  const double ih = inv_h, ih2 = inv_h * inv_h;
  const long s2x = XB, s3h = (long)XB * HY, s3p = (long)XB * PY;
  const double* smd = reinterpret_cast<const double*>(smem);
  bool ok = true;
  int failed_at = 0;

#pragma unroll 1
  for (int v = 0; v < NC; ++v) {
    const int st = v & 1;
    // the epilogue's loads first: they are in flight while the copies land
    double m[2], kh[2] = {0, 0}, uh[2] = {0, 0}, up[2] = {0, 0}, ah[2] = {0, 0}, ap[2] = {0, 0};
    const double* cfs[2] = {cf0, cf1};
    const bool live[2] = {live0, live1};
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      m[e] = live[e] ? cfs[e][(CF_M0 + v) * A.npts] : 0.0;
      if (MODE == MODE_STAGE && live[e]) {
        kh[e] = cfs[e][(CF_DTH0 + v) * A.npts];
        if (A.stage != 4) {
          uh[e] = A.u0[wo[e] + v * sv];
          up[e] = A.u0[wo[e] + (NC + v) * sv];
        }
        if (A.stage != 1) {
          const long ai = (long)b * NV * S3 + (pidx[e] - (long)b * S3);
          ah[e] = A.acc[ai + v * S3];
          ap[e] = A.acc[ai + (NC + v) * S3];
        }
      }
    }
    // every thread waits (bounded) for the stage; the CTA goes on only if all of them saw it.
    // The vote is also the barrier after component v - 1: its stage may now be refilled with
    // component v + 1, which lands while v is computed.
    const bool got = mbar_wait(st ? bar1 : bar0, (v >> 1) & 1, stat.limit);
    if (!__syncthreads_and(got)) {
      ok = false;
      failed_at = v;
      break;
    }
    if (tid == 0 && v >= 1 && v + 1 < NC) pitma_issue(M, base, st ? bar0 : bar1, st ^ 1, b, v + 1, y0, z0);
    const double* H = smd + (st * STAGE + HOFF) / 8;
    const double* P = smd + (st * STAGE + POFF) / 8;
    double s[2], p2[2];
    if (active) {
      // ---- Pi_v: x taps from five 16-byte loads (columns sx - 4 .. sx + 5) ----
      const double* pc = P + cP;
      double px[10];
#pragma unroll
      for (int t = 0; t < 5; ++t) {
        const double2 q = *reinterpret_cast<const double2*>(pc - 4 + 2 * t);
        px[2 * t] = q.x;
        px[2 * t + 1] = q.y;
      }
      // point e sits at px[4 + e]
      double pcen[2], d1x[2], kox[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double* u = px + 4 + e;
        pcen[e] = u[0];
        double a = 0.0;
#pragma unroll
        for (int kx = 1; kx <= SR; ++kx) a = fma(W<4>::d1(kx), u[kx] - u[-kx], a);
        d1x[e] = a;
        double c = W<4>::ko(0) * u[0];
#pragma unroll
        for (int kx = 1; kx <= KR; ++kx) c = fma(W<4>::ko(kx), u[kx] + u[-kx], c);
        kox[e] = c;
      }
      // y and z taps: one 16-byte load per offset serves both points
      double d1y[2] = {0, 0}, d1z[2] = {0, 0}, koy[2], koz[2];
      koy[0] = W<4>::ko(0) * pcen[0];
      koy[1] = W<4>::ko(0) * pcen[1];
      koz[0] = koy[0];
      koz[1] = koy[1];
      double2 yp[KR + 1], ym[KR + 1], zp[KR + 1], zm[KR + 1];
#pragma unroll
      for (int kt = 1; kt <= KR; ++kt) {
        yp[kt] = *reinterpret_cast<const double2*>(pc + kt * s2x);
        ym[kt] = *reinterpret_cast<const double2*>(pc - kt * s2x);
        zp[kt] = *reinterpret_cast<const double2*>(pc + kt * s3p);
        zm[kt] = *reinterpret_cast<const double2*>(pc - kt * s3p);
      }
#pragma unroll
      for (int kt = 1; kt <= SR; ++kt) {
        d1y[0] = fma(W<4>::d1(kt), yp[kt].x - ym[kt].x, d1y[0]);
        d1y[1] = fma(W<4>::d1(kt), yp[kt].y - ym[kt].y, d1y[1]);
        d1z[0] = fma(W<4>::d1(kt), zp[kt].x - zm[kt].x, d1z[0]);
        d1z[1] = fma(W<4>::d1(kt), zp[kt].y - zm[kt].y, d1z[1]);
      }
#pragma unroll
      for (int kt = 1; kt <= KR; ++kt) {
        koy[0] = fma(W<4>::ko(kt), yp[kt].x + ym[kt].x, koy[0]);
        koy[1] = fma(W<4>::ko(kt), yp[kt].y + ym[kt].y, koy[1]);
        koz[0] = fma(W<4>::ko(kt), zp[kt].x + zm[kt].x, koz[0]);
        koz[1] = fma(W<4>::ko(kt), zp[kt].y + zm[kt].y, koz[1]);
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double* c = cb[e];
        double a = c[CF_B0] * (ih * d1x[e]);
        a = fma(c[CF_B1], ih * d1y[e], a);
        a = fma(c[CF_B2], ih * d1z[e], a);
        s[e] = fma(c[CF_DIVB], pcen[e], a);
      }
      // ---- h_v: x taps from three loads (columns sx - 2 .. sx + 3) ----
      const double* hc = H + cH;
      double hx[6];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const double2 q = *reinterpret_cast<const double2*>(hc - 2 + 2 * t);
        hx[2 * t] = q.x;
        hx[2 * t + 1] = q.y;
      }
      // first differences paired at +-k with fused multiply-adds, second differences as the
      // reference's sums term by term (st_d2_ref, st_mixed_ref: lowest offset first, every
      // product and sum rounded on its own), so that they carry the reference's bits
      double hcen[2], hd1x[2], hd2x[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double* u = hx + 2 + e;
        hcen[e] = u[0];
        double a = 0.0;
#pragma unroll
        for (int kx = 1; kx <= SR; ++kx) a = fma(W<4>::d1(kx), u[kx] - u[-kx], a);
        hd1x[e] = a;
        double c = __dmul_rn(W<4>::d2(SR), u[-SR]);
#pragma unroll
        for (int kx = -SR + 1; kx <= SR; ++kx) c = __dadd_rn(c, __dmul_rn(W<4>::d2(kx < 0 ? -kx : kx), u[kx]));
        hd2x[e] = c;
      }
      double hd1y[2] = {0, 0}, hd1z[2] = {0, 0}, hd2y[2], hd2z[2];
      {
        double2 ry[2 * SR + 1], rz[2 * SR + 1];  // rows y + k and planes z + k, k = -SR .. SR
#pragma unroll
        for (int k = -SR; k <= SR; ++k) {
          if (k == 0) continue;
          ry[k + SR] = *reinterpret_cast<const double2*>(hc + k * s2x);
          rz[k + SR] = *reinterpret_cast<const double2*>(hc + k * s3h);
        }
        ry[SR] = rz[SR] = make_double2(hcen[0], hcen[1]);
#pragma unroll
        for (int kt = 1; kt <= SR; ++kt) {
          hd1y[0] = fma(W<4>::d1(kt), ry[SR + kt].x - ry[SR - kt].x, hd1y[0]);
          hd1y[1] = fma(W<4>::d1(kt), ry[SR + kt].y - ry[SR - kt].y, hd1y[1]);
          hd1z[0] = fma(W<4>::d1(kt), rz[SR + kt].x - rz[SR - kt].x, hd1z[0]);
          hd1z[1] = fma(W<4>::d1(kt), rz[SR + kt].y - rz[SR - kt].y, hd1z[1]);
        }
        const double wR = W<4>::d2(SR);
        hd2y[0] = __dmul_rn(wR, ry[0].x);
        hd2y[1] = __dmul_rn(wR, ry[0].y);
        hd2z[0] = __dmul_rn(wR, rz[0].x);
        hd2z[1] = __dmul_rn(wR, rz[0].y);
#pragma unroll
        for (int k = -SR + 1; k <= SR; ++k) {
          const double wk = W<4>::d2(k < 0 ? -k : k);
          hd2y[0] = __dadd_rn(hd2y[0], __dmul_rn(wk, ry[k + SR].x));
          hd2y[1] = __dadd_rn(hd2y[1], __dmul_rn(wk, ry[k + SR].y));
          hd2z[0] = __dadd_rn(hd2z[0], __dmul_rn(wk, rz[k + SR].x));
          hd2z[1] = __dadd_rn(hd2z[1], __dmul_rn(wk, rz[k + SR].y));
        }
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double* c = cb[e];
        s[e] = fma(c[CF_DA0], ih * hd1x[e], s[e]);
        s[e] = fma(c[CF_DA1], ih * hd1y[e], s[e]);
        s[e] = fma(c[CF_DA2], ih * hd1z[e], s[e]);
        double a = c[CF_AXX] * hd2x[e];
        a = fma(c[CF_AYY], hd2y[e], a);
        p2[e] = fma(c[CF_AZZ], hd2z[e], a);
      }
      // mixed x-y and x-z: outer sum over the x offsets a, inner over the y rows (z planes)
      // e; each row (plane) e, from three loads, serves every a of both points
      double mxy[2], mxz[2], myz[2];
#pragma unroll
      for (int pl = 0; pl < 2; ++pl) {
        const long se = pl == 0 ? s2x : s3h;
        double in[2][2 * SR];  // [point][a = -SR .. -1, 1 .. SR]
#pragma unroll
        for (int e = -SR; e <= SR; ++e) {
          if (e == 0) continue;
          double r[6];  // x - 2 .. x + 3 of row (plane) e
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            const double2 q = *reinterpret_cast<const double2*>(hc - 2 + 2 * t + e * se);
            r[2 * t] = q.x;
            r[2 * t + 1] = q.y;
          }
          const double we = d1s<4>(e);
#pragma unroll
          for (int pt = 0; pt < 2; ++pt)
#pragma unroll
            for (int ia = 0; ia < 2 * SR; ++ia) {
              const int a = ia < SR ? ia - SR : ia - SR + 1;
              const double term = __dmul_rn(we, r[2 + pt + a]);
              in[pt][ia] = e == -SR ? term : __dadd_rn(in[pt][ia], term);
            }
        }
#pragma unroll
        for (int pt = 0; pt < 2; ++pt) {
          double o = __dmul_rn(d1s<4>(-SR), in[pt][0]);
#pragma unroll
          for (int ia = 1; ia < 2 * SR; ++ia) {
            const int a = ia < SR ? ia - SR : ia - SR + 1;
            o = __dadd_rn(o, __dmul_rn(d1s<4>(a), in[pt][ia]));
          }
          if (pl == 0) mxy[pt] = o;
          else mxz[pt] = o;
        }
      }
      // mixed y-z: outer sum over the y rows a, inner over the z planes e
#pragma unroll
      for (int a = -SR; a <= SR; ++a) {
        if (a == 0) continue;
        double in0 = 0.0, in1 = 0.0;
#pragma unroll
        for (int e = -SR; e <= SR; ++e) {
          if (e == 0) continue;
          const double2 q = *reinterpret_cast<const double2*>(hc + a * s2x + e * s3h);
          const double t0 = __dmul_rn(d1s<4>(e), q.x), t1 = __dmul_rn(d1s<4>(e), q.y);
          in0 = e == -SR ? t0 : __dadd_rn(in0, t0);
          in1 = e == -SR ? t1 : __dadd_rn(in1, t1);
        }
        const double o0 = __dmul_rn(d1s<4>(a), in0), o1 = __dmul_rn(d1s<4>(a), in1);
        myz[0] = a == -SR ? o0 : __dadd_rn(myz[0], o0);
        myz[1] = a == -SR ? o1 : __dadd_rn(myz[1], o1);
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double* c = cb[e];
        double q = fma(c[CF_AXY], mxy[e], p2[e]);
        q = fma(c[CF_AXZ], mxz[e], q);
        q = fma(c[CF_AYZ], myz[e], q);
        s[e] = fma(ih2, q, s[e]);
        if (DISS) s[e] = fma(c[CF_EH], kox[e] + koy[e] + koz[e], s[e]);
      }
    }
    if (active) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (!live[e]) continue;
        const double val = w[e] == 1.0 ? s[e] + m[e] : fma(w[e], s[e], m[e]);
        if (MODE == MODE_DU) {
          A.du[(long)b * NV * S3 + (pidx[e] - (long)b * S3) + (NC + v) * S3] = val;
        } else {
          const long ai = (long)b * NV * S3 + (pidx[e] - (long)b * S3);
          // the RK4 stage update of both halves of component v (EmitStage::fin)
          if (A.stage == 4) {
            A.next[wo[e] + v * sv] = fma(A.cb, kh[e], ah[e]);
            A.next[wo[e] + (NC + v) * sv] = fma(A.cb, val, ap[e]);
          } else {
            A.acc[ai + v * S3] = fma(A.cb, kh[e], A.stage == 1 ? uh[e] : ah[e]);
            A.acc[ai + (NC + v) * S3] = fma(A.cb, val, A.stage == 1 ? up[e] : ap[e]);
            A.next[wo[e] + v * sv] = fma(A.ca, kh[e], uh[e]);
            A.next[wo[e] + (NC + v) * sv] = fma(A.ca, val, up[e]);
          }
        }
      }
    }
  }
  if (!ok) {
    // a wait gave up: record it, let the copies already issued (component failed_at, and
    // component 1 when it was the first) land, bounded, then leave without writing
    if (tid == 0) atomicExch(stat.err, TGH_ERR_TIMEOUT);
    const long long drain = 1ll << 24;
    const int last = failed_at == 0 ? 1 : failed_at;
    for (int v = failed_at; v <= last; ++v) mbar_wait(v & 1 ? bar1 : bar0, (v >> 1) & 1, drain);
  }
}

}  // namespace tgh
