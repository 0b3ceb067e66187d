// The C ABI of include/tgh.h: problem construction (GHProblem), the ghost-fill plan, the
// verbs and the two RK4 forms. Host C++; all arithmetic runs in the kernels of
// kernels.cuh and rhs.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <map>
#include <unordered_map>
#include <vector>

#include "../../include/tgh.h"
#include "bounds.cuh"
#include "kernels.cuh"
#include "monitors.cuh"
#include "rhs_inst.cuh"
#include "rhs_pi_tma.cuh"
#include "adjoint.cuh"
#include "tangent_rhs.cuh"

using namespace tgh;

namespace tgh {
bool make_pi_tma_maps(double* work, int nwb, PiTmaMaps* out, std::string& err);
cudaError_t launch_pi_tma(bool diss, int mode, cudaStream_t s, const Case& cs, const RhsArgs& a, const PiTmaMaps& M,
                          PiTmaStatus st, int b0, int nb);
}  // namespace tgh

// the Pi kernel a problem launches: the one-point kernel reading through L1, or the pair kernel
// whose stencil tiles the Tensor Memory Accelerator stages into shared memory (q = 4, N = 32,
// FP64 only; the one-point kernel serves every other problem)
enum { PI_L1 = TGH_PI_L1, PI_TMA = TGH_PI_TMA };

struct GraphKey {
  double t, dt;
  int nsteps;
};

// One rank's share of the exchange of a fill phase: per peer, the (internal block, work index)
// points packed for it (send) or unpacked from it into halo blocks (recv), peer-major.
struct ExchangeList {
  std::vector<long> send_count, recv_count;  // per peer rank
  HookPt* send = nullptr;                    // device, sum(send_count) entries
  HookPt* recv = nullptr;
  long nsend = 0, nrecv = 0;
};

struct tgh_problem {
  tgh_config cfg;
  // nb: the blocks this rank computes (its own leaves); nwb: the working arrays' blocks, its
  // own leaves first, then the halo: other ranks' leaves its fill reads
  int q, G, N, N1, Wd, Wx, nb, nwb, maxlevel = 0;  // Wx: the working array's row pitch
  double lo[3], h0;
  int cells0[3], periodic[3];
  std::vector<int> level, corner;  // of every leaf of the forest (global numbering)
  int rank = 0, nranks = 1;
  std::vector<int> owner;          // per global leaf: the rank that computes it
  std::vector<int> g2i, i2g;       // global leaf <-> internal block (-1: not held)
  std::vector<ExchangeList> xch;   // per fill phase: 0 the copies, l >= 1 level l's prolongation
  std::vector<std::unordered_map<int64_t, int>> lut;
  Geo geo;
  long S, Wv, npts;
  Case cs;
  bool diss = false, intr = false;
  bool mixed = false;  // TGH_PREC_MIXED: FP32 stencil sums and algebra, FP64 state and metric
  cudaStream_t stream = nullptr;
  cudaStream_t cap = nullptr;  // the stream graphs are captured on
  std::string err;
  // device buffers
  double* work = nullptr;     // the ghosted working array (also W0 of the batched form)
  double* Hsrc = nullptr;
  // :fitted: the target cache (per own block 40 fields of the owned points), its fill time on the
  // device, and whether a fill or a set has happened since creation
  double* tw = nullptr;
  double* tf = nullptr;
  bool target_set = false;
  double* blk = nullptr;      // per block: domain lo (3), h, integer corner (3), pad
  uint8_t* primary = nullptr; // per owned point: 1 where this block holds the primary copy
  CopyRun* runs = nullptr;
  int nruns = 0;
  CopyPt* gpts = nullptr;  // the batched form's copies (no primary self-copies)
  long ngpts = 0;
  HookPt* hooks = nullptr;
  int nhooks = 0;
  double* hook_cache = nullptr;  // stationary cases: the Dirichlet ghosts' values, 20 per point
  bool hook_cache_valid = false;
  // the batched form's stage buffers whose Dirichlet ghosts already hold a stationary case's
  // hook: written once, and by nothing else after (the stage epilogue writes owned points, the
  // copies and the prolongation write ghosts inside the domain)
  double* hooks_held[2] = {nullptr, nullptr};
  // set while the batched form's graph is captured: W0's Dirichlet ghosts are written by the
  // fill that precedes every launch of that graph, and nothing inside the graph overwrites them
  bool capturing = false;
  std::vector<ProlongPt*> prol;  // per level 1..maxlevel
  std::vector<int> nprol;
  // the same prolongation as tiles of 8^3 fine points (fill_prolong_tile_kernel), per level;
  // ntile[l] < 0: the level's points do not tile (the per-point kernel runs)
  std::vector<ProlongTile*> ptile;
  std::vector<unsigned short*> ptpts;
  std::vector<int> ntile;
  unsigned long long* scratch = nullptr;  // speed reduction: max bits, non-finite count
  unsigned long long* bcounts = nullptr;  // the range projection's counts: fired, non-finite, max r bits
  // the range projection the limiters apply (set by tgh_set_bounds), and its accounting
  bool has_bounds = false;
  tgh_bounds bounds{};
  long acc_calls = 0, acc_hits = 0, acc_nonfinite = 0;
  double acc_rmax = 0.0, acc_first_t = NAN, acc_first_r = NAN;
  double* part = nullptr;                 // error-norm partials + result
  double* diag = nullptr;                 // the monitors' diag field set (NDIAG slots per block)
  double* dpart = nullptr;                // constraint-norm partials (17 per CTA) + the fold
  unsigned long long* ind = nullptr;      // the indicator's maxima (10 scales, tau_max) as bit patterns
  double* ind_tol = nullptr;              // the firing thresholds (at most 4)
  int* ind_counts = nullptr;              // per block and threshold: firing count
  int* ind_boxes = nullptr;               // ... and the bounding box of the firing nodes
  double* coef = nullptr;                 // per-point coefficients between the two RHS kernels
  int npart = 0;
  // plain-form RK4 buffers (state layout)
  double *k = nullptr, *acc = nullptr, *y = nullptr, *u0 = nullptr;
  // batched-form buffers
  double *W1 = nullptr, *W2 = nullptr, *bacc = nullptr;
  // tangent-linear buffers: the tangent working array, and the plain form's k, acc, y tangents
  double *twork = nullptr, *kt = nullptr, *acct = nullptr, *yt = nullptr;
  // adjoint buffers: the feature cotangents, mu on the working array, the parameters' partials,
  // the recomputed stage states and two state-sized accumulators
  double *adj_cot = nullptr, *adj_mu = nullptr, *adj_part = nullptr;
  double *adj_y[3] = {nullptr, nullptr, nullptr}, *adj_a = nullptr, *adj_acc = nullptr, *adj_m = nullptr;
  cudaGraphExec_t gexec = nullptr;
  GraphKey gkey{0, 0, 0};
  long graph_kernels = 0;  // kernel nodes of the captured graph
  long last_launches = 0;  // kernels the last tgh_step_batched call (or sharded step) ran
  long launches = 0;       // kernels launched since tgh_shard_begin
  const double* gu = nullptr;
  // the contract between prepare and rhs: rhs reads the working array as the last tgh_prepare
  // left it. prep_gen counts the tgh_prepare calls; work_prepared says whether the working array
  // still holds the last one's fill (every other verb that writes it clears the flag and names
  // itself in work_writer), so that tgh_rhs refuses a stale array with TGH_ERR_STALE.
  long prep_gen = 0;
  bool work_prepared = false;
  const char* work_writer = "nothing (no tgh_prepare yet)";
  // the right-hand side's kernel variants (tgh_set_variant) and the TMA kernel's tensor maps,
  // one pair per working array it has read
  int pi_variant = PI_L1;
  int threads = 128;  // CTA size of the head and one-point Pi kernels
  int pi_mb = 4;      // the one-point Pi kernel's resident CTAs per SM (its launch bound)
  std::vector<std::pair<const double*, PiTmaMaps>> tma_maps;
  int* dev_err = nullptr;                 // a bounded device wait that gave up records it here
  // the blocks interior_kernel visits: those that can hold a point with r < r_1 at some time of
  // [lo, hi]; one list for direct launches, one for the captured graph (built before capture)
  struct BlockList {
    int* dev = nullptr;
    int n = -1;
    double lo = 0, hi = -1;
  } ilist, ilist_graph;
  const BlockList* ilist_use = nullptr;
  // the batched form's side branch: the interior kernel runs beside the hook and the
  // prolongation (it reads owned points only, which those write none of)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool interior_done = false;  // the stage's interior kernel ran on the side branch
  long long wait_limit = 1ll << 26;       // polls a device wait may make
};

#define CK(call)                                                         \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      p->err = std::string(#call) + ": " + cudaGetErrorString(e_);       \
      return TGH_ERR_CUDA;                                               \
    }                                                                    \
  } while (0)

static int fail(tgh_problem* p, int code, const std::string& msg) {
  p->err = msg;
  return code;
}

// doubles in one of the problem's working arrays (rows padded to the pitch Wx)
static size_t work_doubles(const tgh_problem* p) { return (size_t)p->Wv * NV * p->nwb; }
// a padded work index as the index of the same point in the reference's dense cube
static int dense_index(const tgh_problem* p, int w) { return (w % p->Wx) + p->Wd * (w / p->Wx); }

// a verb other than tgh_prepare wrote the working array: the next tgh_rhs needs a new prepare
static void work_overwritten(tgh_problem* p, const char* who) {
  p->work_prepared = false;
  p->work_writer = who;
}

// ---- the forest: owners, positions ----
static inline int64_t bkey(int64_t bx, int64_t by, int64_t bz) { return ((bx * 1048576) + by) * 1048576 + bz; }

// The primary owner of lattice point n of level l: the coarsest leaf holding the point (closed
// blocks; a point of level l lies on a coarser level k's lattice when n is a multiple of
// 2^(l - k)), and among a level's leaves the one with the point on its lower face. With the
// coarsest leaf primary the reference's driver record on a refined hole (the hole fixture,
// err_l2 = 1.690514e-06) is met to 0.2 %; with the finest, to 3.9 %.
static bool find_owner(const tgh_problem* p, int l, const int64_t n[3], int& leaf, int loc[3], int& lev) {
  for (int k = 0; k <= p->maxlevel; ++k) {
    int64_t m[3], cand[3][2];
    int nc[3];
    bool on = true;
    for (int d = 0; d < 3; ++d) {
      if (k >= l) {
        m[d] = n[d] << (k - l);
      } else {
        const int64_t s = (int64_t)1 << (l - k);
        if (n[d] % s) on = false;
        m[d] = n[d] / s;
      }
    }
    if (!on) continue;
    for (int d = 0; d < 3; ++d) {
      int64_t c = m[d] / p->N;
      nc[d] = 0;
      cand[d][nc[d]++] = c;
      if (m[d] % p->N == 0) cand[d][nc[d]++] = c - 1;
    }
    for (int iz = 0; iz < nc[2]; ++iz)
      for (int iy = 0; iy < nc[1]; ++iy)
        for (int ix = 0; ix < nc[0]; ++ix) {
          auto it = p->lut[k].find(bkey(cand[0][ix], cand[1][iy], cand[2][iz]));
          if (it == p->lut[k].end()) continue;
          leaf = it->second;
          for (int d = 0; d < 3; ++d) loc[d] = (int)(m[d] - p->corner[3 * leaf + d]);
          lev = k;
          return true;
        }
  }
  return false;
}

// a leaf of level exactly l whose closed box contains the (half-)integer position n/2 of
// level l+1's point n
static int coarse_cover(const tgh_problem* p, int l, const int64_t nf[3]) {
  int64_t lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = nf[d] >> 1;                     // floor(n/2)
    hi[d] = (nf[d] & 1) ? lo[d] + 1 : lo[d];
  }
  for (int dz = -1; dz <= 0; ++dz)
    for (int dy = -1; dy <= 0; ++dy)
      for (int dx = -1; dx <= 0; ++dx) {
        int64_t c[3] = {lo[0] / p->N + dx, lo[1] / p->N + dy, lo[2] / p->N + dz};
        auto it = p->lut[l].find(bkey(c[0], c[1], c[2]));
        if (it == p->lut[l].end()) continue;
        const int b = it->second;
        bool ok = true;
        for (int d = 0; d < 3; ++d) {
          const int64_t c0 = p->corner[3 * b + d];
          if (lo[d] < c0 || hi[d] > c0 + p->N) ok = false;
        }
        if (ok) return b;
      }
  return -1;
}

static Case make_case(const tgh_config& c) {
  Case k;
  std::memset(&k, 0, sizeof(k));
  k.bg = c.bg;
  const double* u = c.bg.boost;
  const double u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  k.boosted = ((c.bg.kind == TGH_BG_KERR_SCHILD || c.bg.kind == TGH_BG_HARMONIC_KERR) && u2 > 0.0) ? 1 : 0;
  const double gam = 1.0 / std::sqrt(1.0 - u2);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) k.L[i][j] = i == j ? 1.0 : 0.0;
  if (k.boosted) {
    k.L[0][0] = gam;
    for (int i = 0; i < 3; ++i) {
      k.L[0][i + 1] = k.L[i + 1][0] = gam * u[i];
      for (int j = 0; j < 3; ++j) k.L[i + 1][j + 1] = (i == j ? 1.0 : 0.0) + (gam - 1.0) * u[i] * u[j] / u2;
    }
  }
  k.gauge = c.gauge;
  {
    const double* v = c.ks_velocity;
    const double* a = c.ks_spin;
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double g = 1.0 / std::sqrt(1.0 - v2);
    const double va = v[0] * a[0] + v[1] * a[1] + v[2] * a[2];
    k.ksM = c.ks_M;
    k.ksS[0] = g * va;
    for (int i = 0; i < 3; ++i) k.ksS[i + 1] = v2 == 0.0 ? a[i] : a[i] + ((g - 1.0) * va / v2) * v[i];
    k.ksU[0] = g;
    for (int i = 0; i < 3; ++i) k.ksU[i + 1] = g * v[i];
  }
  k.damping = c.damping;
  k.g0 = c.gamma0;
  k.dnear = c.damp_near;
  k.dfar = c.damp_far;
  k.dwidth = c.damp_width;
  k.g2 = c.gamma2;
  k.dissipation = c.dissipation;
  k.eps = c.eps_ko;
  k.eout = c.eps_out;
  k.ein = c.eps_in;
  k.er1 = c.eps_r1;
  k.erh = c.eps_rh;
  k.interior = c.interior;
  for (int i = 0; i < 3; ++i) {
    k.dc0[i] = c.damp_c0[i];
    k.dv[i] = c.damp_v[i];
    k.ec0[i] = c.eps_c0[i];
    k.ev[i] = c.eps_v[i];
    k.ic0[i] = c.int_c0[i];
    k.iv[i] = c.int_v[i];
  }
  k.r0 = c.r0;
  k.r1 = c.r1;
  k.rho_max = c.rho_max;
  k.w_ramp = c.w_ramp;
  k.rho_ramp = c.rho_ramp;
  return k;
}

static unsigned grid_for(long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// The fill plan of one rank: where every point of its blocks' working arrays comes from, in the
// rank's internal block numbering (its own leaves in forest order, then the halo: the other
// ranks' leaves its fill reads, numbered as first met), and which points of other ranks'
// leaves it must receive before each fill phase (phase 0: the copies' sources, owned points;
// phase l >= 1: the coarse stencil boxes of level l's prolongation, read after the owner's
// level l - 1 is filled). With one rank everything is local and the numbering is the forest's.
struct HostPlan {
  std::vector<int> g2i, i2g;
  int nloc = 0;
  std::vector<CopyRun> runs;  // the plain form's scatter (one rank only)
  std::vector<CopyPt> gpts;
  std::vector<HookPt> hooks;
  std::vector<std::vector<ProlongPt>> prol;
  std::vector<uint8_t> prim;
  // (owner rank, phase) -> sorted distinct (global leaf, work index) read from that owner
  std::map<std::pair<int, int>, std::vector<std::pair<int, int>>> req;
};

static bool plan_rank(const tgh_problem* p, int r, bool entries, HostPlan& hp, std::string& err) {
  const int nleaf = (int)p->owner.size();
  hp.g2i.assign(nleaf, -1);
  hp.i2g.clear();
  for (int g = 0; g < nleaf; ++g)
    if (p->owner[g] == r) {
      hp.g2i[g] = (int)hp.i2g.size();
      hp.i2g.push_back(g);
    }
  hp.nloc = (int)hp.i2g.size();
  auto intern = [&](int g) {
    if (hp.g2i[g] < 0) {
      hp.g2i[g] = (int)hp.i2g.size();
      hp.i2g.push_back(g);
    }
    return hp.g2i[g];
  };
  auto& runs = hp.runs;
  auto& gpts = hp.gpts;
  auto& hooks = hp.hooks;
  auto& prol = hp.prol;
  auto& prim = hp.prim;
  prol.assign(p->maxlevel + 1, {});
  if (entries) prim.assign((size_t)hp.nloc * p->S, 0);
  const bool one = p->nranks == 1;
  const int Wd = p->Wd, Wx = p->Wx, G = p->G, P = p->q + 2;
  for (int b = 0; b < hp.nloc; ++b) {
    const int gb = hp.i2g[b];
    const int l = p->level[gb];
    for (int k = 0; k < Wd; ++k)
      for (int j = 0; j < Wd; ++j) {
        CopyRun cur{};
        bool open = false;
        for (int i = 0; i < Wd; ++i) {
          int64_t n[3] = {(int64_t)p->corner[3 * gb] + i - G, (int64_t)p->corner[3 * gb + 1] + j - G,
                          (int64_t)p->corner[3 * gb + 2] + k - G};
          bool outside = false;
          for (int d = 0; d < 3; ++d) {
            const int64_t per = (int64_t)p->cells0[d] << l;
            if (p->periodic[d]) {
              n[d] %= per;
              if (n[d] < 0) n[d] += per;
            } else if (n[d] < 0 || n[d] > per) {
              outside = true;
            }
          }
          const int w = i + Wx * (j + Wd * k);
          int leaf = -1, loc[3], lev = -1;
          if (!outside && find_owner(p, l, n, leaf, loc, lev)) {
            // a run along x steps 2^(lev - l) source points a point; a coarser owner holds only
            // every other point of the run, so its points stand alone (step 0)
            const int step = lev >= l ? 1 << (lev - l) : 0;
            const bool own = i >= G && i <= G + p->N && j >= G && j <= G + p->N && k >= G && k <= G + p->N;
            const int sw = (loc[0] + G) + Wx * ((loc[1] + G) + Wd * (loc[2] + G));
            if (own && leaf == gb) {
              if (entries) prim[(size_t)b * p->S + (i - G) + (size_t)p->N1 * ((j - G) + (size_t)p->N1 * (k - G))] = 1;
            } else {
              if (p->owner[leaf] != r) hp.req[{p->owner[leaf], 0}].push_back({leaf, sw});
              if (entries) gpts.push_back(CopyPt{b, w, intern(leaf), sw});
            }
            if (entries && one) {
              if (open && step > 0 && cur.src_b == leaf && cur.step == step && cur.sj == loc[1] && cur.sk == loc[2] &&
                  cur.si + cur.len * step == loc[0] && cur.dst_w + cur.len == w) {
                cur.len++;
              } else {
                if (open) runs.push_back(cur);
                cur = CopyRun{b, w, leaf, loc[0], loc[1], loc[2], 1, step};
                open = true;
              }
            }
            continue;
          }
          if (open) {
            runs.push_back(cur);
            open = false;
          }
          if (outside) {
            if (entries) hooks.push_back(HookPt{b, w});
            continue;
          }
          if (l == 0) {
            err = "a lattice point is covered by no leaf of the forest";
            return false;
          }
          const int c = coarse_cover(p, l - 1, n);
          if (c < 0) {
            err = "a prolonged ghost point has no covering leaf one level coarser (the forest is not 2:1 balanced)";
            return false;
          }
          int odd = 0;
          int64_t base[3], ext[3];
          for (int d = 0; d < 3; ++d) {
            if (n[d] & 1) {
              odd |= 1 << d;
              base[d] = (n[d] >> 1) - (P / 2 - 1);
            } else {
              base[d] = n[d] >> 1;
            }
            const int64_t rel = base[d] - p->corner[3 * c + d] + G;
            ext[d] = (n[d] & 1) ? P : 1;
            if (rel < 0 || rel + ext[d] > Wd) {
              err = "a prolongation stencil leaves the coarse block's ghost zone";
              return false;
            }
          }
          const int sw = (int)((base[0] - p->corner[3 * c] + G) +
                               Wx * ((base[1] - p->corner[3 * c + 1] + G) + (int64_t)Wd * (base[2] - p->corner[3 * c + 2] + G)));
          if (p->owner[c] != r) {
            auto& v = hp.req[{p->owner[c], l}];
            for (int64_t kz = 0; kz < ext[2]; ++kz)
              for (int64_t ky = 0; ky < ext[1]; ++ky)
                for (int64_t kx = 0; kx < ext[0]; ++kx) v.push_back({c, (int)(sw + kx + Wx * (ky + Wd * kz))});
          }
          if (entries) prol[l].push_back(ProlongPt{b, w, intern(c), sw, odd});
        }
        if (open) runs.push_back(cur);
      }
  }
  for (auto& kv : hp.req) {
    std::sort(kv.second.begin(), kv.second.end());
    kv.second.erase(std::unique(kv.second.begin(), kv.second.end()), kv.second.end());
  }
  return true;
}

// The plan of this problem's rank on the device, with the exchange lists: what this rank
// receives into its halo (its own requests) and what it sends (every other rank's requests
// to it, found by planning that rank's leaves: both sides derive the same sorted list).
static bool tile_prolongation(const tgh_problem* p, const HostPlan& hp, const std::vector<ProlongPt>& pts,
                              std::vector<ProlongTile>& tiles, std::vector<unsigned short>& codes);
static int build_plan(tgh_problem* p) {
  HostPlan hp;
  std::string err;
  if (!plan_rank(p, p->rank, true, hp, err)) return fail(p, TGH_ERR_ARG, err);
  p->g2i = hp.g2i;
  p->i2g = hp.i2g;
  p->nwb = (int)hp.i2g.size();
  const auto& runs = hp.runs;
  const auto& gpts = hp.gpts;
  const auto& hooks = hp.hooks;
  auto& prol = hp.prol;
  const auto& prim = hp.prim;
  const int nph = p->maxlevel + 1;
  p->xch.assign(nph, ExchangeList{});
  std::vector<std::vector<HookPt>> snd(nph), rcv(nph);
  for (int ph = 0; ph < nph; ++ph) {
    p->xch[ph].send_count.assign(p->nranks, 0);
    p->xch[ph].recv_count.assign(p->nranks, 0);
  }
  for (int o = 0; o < p->nranks; ++o) {
    if (o == p->rank) continue;
    HostPlan hq;
    if (!plan_rank(p, o, false, hq, err)) return fail(p, TGH_ERR_ARG, err);
    for (int ph = 0; ph < nph; ++ph) {
      auto mine = hp.req.find({o, ph});
      if (mine != hp.req.end())
        for (const auto& e : mine->second) rcv[ph].push_back(HookPt{p->g2i[e.first], e.second});
      p->xch[ph].recv_count[o] = mine == hp.req.end() ? 0 : (long)mine->second.size();
      auto theirs = hq.req.find({p->rank, ph});
      if (theirs != hq.req.end())
        for (const auto& e : theirs->second) snd[ph].push_back(HookPt{p->g2i[e.first], e.second});
      p->xch[ph].send_count[o] = theirs == hq.req.end() ? 0 : (long)theirs->second.size();
    }
  }
  for (int ph = 0; ph < nph; ++ph) {
    ExchangeList& x = p->xch[ph];
    x.nsend = (long)snd[ph].size();
    x.nrecv = (long)rcv[ph].size();
    CK(cudaMalloc(&x.send, std::max<size_t>(1, snd[ph].size()) * sizeof(HookPt)));
    CK(cudaMalloc(&x.recv, std::max<size_t>(1, rcv[ph].size()) * sizeof(HookPt)));
    if (x.nsend) CK(cudaMemcpy(x.send, snd[ph].data(), snd[ph].size() * sizeof(HookPt), cudaMemcpyHostToDevice));
    if (x.nrecv) CK(cudaMemcpy(x.recv, rcv[ph].data(), rcv[ph].size() * sizeof(HookPt), cudaMemcpyHostToDevice));
  }
  p->nruns = (int)runs.size();
  p->ngpts = (long)gpts.size();
  p->nhooks = (int)hooks.size();
  CK(cudaMalloc(&p->gpts, std::max<size_t>(1, gpts.size()) * sizeof(CopyPt)));
  if (!gpts.empty()) CK(cudaMemcpy(p->gpts, gpts.data(), gpts.size() * sizeof(CopyPt), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&p->runs, std::max<size_t>(1, runs.size()) * sizeof(CopyRun)));
  CK(cudaMemcpy(p->runs, runs.data(), runs.size() * sizeof(CopyRun), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&p->hooks, std::max<size_t>(1, hooks.size()) * sizeof(HookPt)));
  if (!hooks.empty()) CK(cudaMemcpy(p->hooks, hooks.data(), hooks.size() * sizeof(HookPt), cudaMemcpyHostToDevice));
  p->prol.assign(p->maxlevel + 1, nullptr);
  p->nprol.assign(p->maxlevel + 1, 0);
  for (int l = 1; l <= p->maxlevel; ++l) {
    // grouped by odd-axis mask (a point prolonged along k axes sums 6^k terms), in plan order
    // within a group, so that a warp's points do the same work
    std::stable_sort(prol[l].begin(), prol[l].end(),
                     [](const ProlongPt& a, const ProlongPt& b) { return a.odd < b.odd; });
    p->nprol[l] = (int)prol[l].size();
    CK(cudaMalloc(&p->prol[l], std::max<size_t>(1, prol[l].size()) * sizeof(ProlongPt)));
    if (!prol[l].empty())
      CK(cudaMemcpy(p->prol[l], prol[l].data(), prol[l].size() * sizeof(ProlongPt), cudaMemcpyHostToDevice));
  }
  p->ptile.assign(p->maxlevel + 1, nullptr);
  p->ptpts.assign(p->maxlevel + 1, nullptr);
  p->ntile.assign(p->maxlevel + 1, -1);
  for (int l = 1; l <= p->maxlevel; ++l) {
    std::vector<ProlongTile> tiles;
    std::vector<unsigned short> codes;
    if (prol[l].empty() || !tile_prolongation(p, hp, prol[l], tiles, codes)) continue;
    p->ntile[l] = (int)tiles.size();
    CK(cudaMalloc(&p->ptile[l], tiles.size() * sizeof(ProlongTile)));
    CK(cudaMemcpy(p->ptile[l], tiles.data(), tiles.size() * sizeof(ProlongTile), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&p->ptpts[l], codes.size() * sizeof(unsigned short)));
    CK(cudaMemcpy(p->ptpts[l], codes.data(), codes.size() * sizeof(unsigned short), cudaMemcpyHostToDevice));
  }
  CK(cudaMalloc(&p->primary, (size_t)p->npts));
  CK(cudaMemcpy(p->primary, prim.data(), (size_t)p->npts, cudaMemcpyHostToDevice));
  return TGH_OK;
}

// The tiles of one level's prolonged points (fill_prolong_tile_kernel): the points of one fine
// block whose stencils lie in one coarse block, grouped by the 8^3 box of fine offsets from the
// block's corner that holds them. Per tile the coarse centre of fine offset 0 and the coarse rows
// its points' y and z stencils cover. The coarse centre of a point is its stencil base plus P/2 - 1
// along an interpolating axis. False (the per-point kernel then runs) when a tile's points do not
// share one mapping from fine offsets to coarse centres (a periodic wrap inside a tile) or its rows
// exceed the kernel's shared arrays.
static bool tile_prolongation(const tgh_problem* p, const HostPlan& hp, const std::vector<ProlongPt>& pts,
                              std::vector<ProlongTile>& tiles, std::vector<unsigned short>& codes) {
  const int P = p->q + 2, H = P / 2 - 1, C = P + 4, Wx = p->Wx, Wd = p->Wd, G = p->G;
  if ((long)p->nwb >= (1L << 20)) return false;
  auto fdiv8 = [](int r) { return r >= 0 ? r / 8 : -((-r + 7) / 8); };
  struct Acc {
    ProlongTile t;
    int xlo, xhi, ylo, yhi, zlo, zhi, fxm, fym;
    std::vector<unsigned short> c;
  };
  std::unordered_map<unsigned long long, int> index;
  std::vector<Acc> acc;
  for (const ProlongPt& q : pts) {
    const int fi[3] = {q.dst_w % Wx, (q.dst_w / Wx) % Wd, q.dst_w / (Wx * Wd)};
    const int sb[3] = {q.src_w % Wx, (q.src_w / Wx) % Wd, q.src_w / (Wx * Wd)};
    int t[3], f[3], par[3], ctr[3];
    for (int d = 0; d < 3; ++d) {
      const int r = fi[d] - G;
      t[d] = fdiv8(r);
      f[d] = r - 8 * t[d];
      const int odd = (q.odd >> d) & 1;
      par[d] = (odd + f[d]) & 1;  // the parity of the tile origin's fine lattice index
      ctr[d] = sb[d] + (odd ? H : 0);
    }
    const unsigned long long key = (unsigned long long)q.dst_b << 44 | (unsigned long long)q.src_b << 24 |
                                   (unsigned long long)(t[0] + 8) << 16 | (unsigned long long)(t[1] + 8) << 8 |
                                   (unsigned long long)(t[2] + 8);
    if (t[0] + 8 < 0 || t[0] + 8 > 255 || t[1] + 8 < 0 || t[1] + 8 > 255 || t[2] + 8 < 0 || t[2] + 8 > 255) return false;
    auto it = index.find(key);
    int a;
    if (it == index.end()) {
      a = (int)acc.size();
      index.emplace(key, a);
      Acc n{};
      n.t.dst_b = q.dst_b;
      n.t.src_b = q.src_b;
      n.t.i0 = (short)(8 * t[0] + G);
      n.t.j0 = (short)(8 * t[1] + G);
      n.t.k0 = (short)(8 * t[2] + G);
      n.t.par = (unsigned char)(par[0] | par[1] << 1 | par[2] << 2);
      n.t.cxb = (short)(ctr[0] - ((par[0] + f[0]) >> 1));
      n.t.cyb = (short)(ctr[1] - ((par[1] + f[1]) >> 1));
      n.t.czb = (short)(ctr[2] - ((par[2] + f[2]) >> 1));
      n.xlo = n.ylo = n.zlo = 1 << 30;
      n.xhi = n.yhi = n.zhi = -(1 << 30);
      acc.push_back(std::move(n));
    } else {
      a = it->second;
    }
    Acc& A = acc[a];
    const short cb[3] = {A.t.cxb, A.t.cyb, A.t.czb};
    for (int d = 0; d < 3; ++d)
      if (((A.t.par >> d) & 1) != par[d] || cb[d] + ((par[d] + f[d]) >> 1) != ctr[d]) return false;
    const int ox = q.odd & 1, oy = (q.odd >> 1) & 1, oz = (q.odd >> 2) & 1;
    A.xlo = std::min(A.xlo, ctr[0] - (ox ? H : 0));
    A.xhi = std::max(A.xhi, ctr[0] + (ox ? P / 2 : 0));
    A.ylo = std::min(A.ylo, ctr[1] - (oy ? H : 0));
    A.yhi = std::max(A.yhi, ctr[1] + (oy ? P / 2 : 0));
    A.zlo = std::min(A.zlo, ctr[2] - (oz ? H : 0));
    A.zhi = std::max(A.zhi, ctr[2] + (oz ? P / 2 : 0));
    A.fxm |= 1 << f[0];
    A.fym |= 1 << f[1];
    A.c.push_back((unsigned short)(f[0] | f[1] << 3 | f[2] << 6));
  }
  tiles.reserve(acc.size());
  codes.reserve(pts.size());
  for (Acc& A : acc) {
    const int cyn = A.yhi - A.ylo + 1, czn = A.zhi - A.zlo + 1;
    if (cyn > C || czn > C) return false;
    // every coarse value stage X reads lies in the coarse block's working array
    if (A.xlo < 0 || A.xhi >= Wd || A.ylo < 0 || A.yhi >= Wd || A.zlo < 0 || A.zhi >= Wd) return false;
    A.t.xlo = (short)A.xlo;
    A.t.xhi = (short)A.xhi;
    A.t.ylo = (short)A.ylo;
    A.t.zlo = (short)A.zlo;
    A.t.cyn = (unsigned char)cyn;
    A.t.czn = (unsigned char)czn;
    int n = 0;
    A.t.fxs = 0;
    for (int x = 0; x < 8; ++x)
      if (A.fxm >> x & 1) A.t.fxs |= x << (3 * n++);
    A.t.nfx = (unsigned char)n;
    A.t.fxm = (unsigned char)A.fxm;
    A.t.fym = (unsigned char)A.fym;
    A.t.p0 = (int)codes.size();
    A.t.np = (int)A.c.size();
    codes.insert(codes.end(), A.c.begin(), A.c.end());
    tiles.push_back(A.t);
  }
  (void)hp;
  return true;
}

// Level l's prolongation into `work` (the weights of order P are compile-time constants).
static cudaError_t launch_prolong(tgh_problem* p, int l, double* work) {
  if (l < (int)p->ntile.size() && p->ntile[l] > 0) {
    const int n = p->ntile[l];
    const ProlongTile* t = p->ptile[l];
    const unsigned short* c = p->ptpts[l];
    switch (p->q + 2) {
      case 4: fill_prolong_tile_kernel<4><<<n, PROLONG_TILE_THREADS, 0, p->stream>>>(t, c, work, p->geo); break;
      case 6: fill_prolong_tile_kernel<6><<<n, PROLONG_TILE_THREADS, 0, p->stream>>>(t, c, work, p->geo); break;
      case 8: fill_prolong_tile_kernel<8><<<n, PROLONG_TILE_THREADS, 0, p->stream>>>(t, c, work, p->geo); break;
      default: fill_prolong_tile_kernel<10><<<n, PROLONG_TILE_THREADS, 0, p->stream>>>(t, c, work, p->geo); break;
    }
    return cudaGetLastError();
  }
  const int T = 256;
  const long n = (long)p->nprol[l] * NV;
  switch (p->q + 2) {
    case 4: fill_prolong_kernel<4><<<grid_for(n, T), T, 0, p->stream>>>(p->prol[l], p->nprol[l], work, p->geo); break;
    case 6: fill_prolong_kernel<6><<<grid_for(n, T), T, 0, p->stream>>>(p->prol[l], p->nprol[l], work, p->geo); break;
    case 8: fill_prolong_kernel<8><<<grid_for(n, T), T, 0, p->stream>>>(p->prol[l], p->nprol[l], work, p->geo); break;
    default: fill_prolong_kernel<10><<<grid_for(n, T), T, 0, p->stream>>>(p->prol[l], p->nprol[l], work, p->geo); break;
  }
  return cudaGetLastError();
}

// The Dirichlet ghosts of `work` at time t. A stationary case (its analytic state does not
// depend on t) evaluates them once and copies the kept values afterwards.
static int launch_hooks(tgh_problem* p, double* work, double t) {
  if (!p->nhooks) return TGH_OK;
  if (p->hook_cache && p->hook_cache_valid) {
    if (work == p->hooks_held[0] || work == p->hooks_held[1] || (p->capturing && work == p->work)) return TGH_OK;
    hook_copy_kernel<<<grid_for(p->nhooks, 256), 256, 0, p->stream>>>(p->hooks, p->nhooks, p->hook_cache, work,
                                                                       p->geo);
  } else {
    fill_hook_kernel<<<grid_for(p->nhooks, 128), 128, 0, p->stream>>>(p->hooks, p->nhooks, p->blk, work, p->geo,
                                                                      p->cs, t, p->hook_cache);
    p->hook_cache_valid = p->hook_cache != nullptr;
  }
  CK(cudaGetLastError());
  return TGH_OK;
}

// ---- the fill: stage 0 (copies, hooks), then prolongation level by level ----
static int launch_fill(tgh_problem* p, const double* src, bool from_work, double* work, double t) {
  const int T = 256;
  if (!from_work && p->nranks > 1)
    return fail(p, TGH_ERR_ARG, "a sharded problem is filled through its exchange phases (tgh_shard_*), not from u");
  if (from_work) {
    if (p->ngpts) {
      fill_points_kernel<<<grid_for(p->ngpts, T), T, 0, p->stream>>>(p->gpts, p->ngpts, work, p->geo);
      CK(cudaGetLastError());
    }
  } else if (p->nruns) {
    fill_copy_kernel<<<grid_for((long)p->nruns * 32, T), T, 0, p->stream>>>(p->runs, p->nruns, src, work, p->geo);
    CK(cudaGetLastError());
  }
  int s = launch_hooks(p, work, t);
  if (s) return s;
  for (int l = 1; l <= p->maxlevel; ++l) {
    if (!p->nprol[l]) continue;
    CK(launch_prolong(p, l, work));
  }
  return TGH_OK;
}

// the kernel launches of one launch_fill call
static long fill_launches(const tgh_problem* p, bool from_work) {
  long n = from_work ? (p->ngpts ? 1 : 0) : (p->nruns ? 1 : 0);
  if (p->nhooks) ++n;
  for (int l = 1; l <= p->maxlevel; ++l)
    if (p->nprol[l]) ++n;
  return n;
}

static cudaError_t launch_part(tgh_problem* p, int part, int mode, cudaStream_t s, const RhsArgs& a) {
  if (p->mixed) {
    switch (p->q) {
      case 2: return launch_rhs_q2_f32(part, p->diss, mode, p->intr, s, p->cs, a);
      case 4: return launch_rhs_q4_f32(part, p->diss, mode, p->intr, s, p->cs, a);
      case 6: return launch_rhs_q6_f32(part, p->diss, mode, p->intr, s, p->cs, a);
      default: return launch_rhs_q8_f32(part, p->diss, mode, p->intr, s, p->cs, a);
    }
  }
  switch (p->q) {
    case 2: return launch_rhs_q2_f64(part, p->diss, mode, p->intr, s, p->cs, a);
    case 4: return launch_rhs_q4_f64(part, p->diss, mode, p->intr, s, p->cs, a);
    case 6: return launch_rhs_q6_f64(part, p->diss, mode, p->intr, s, p->cs, a);
    default: return launch_rhs_q8_f64(part, p->diss, mode, p->intr, s, p->cs, a);
  }
}

// whether a launch may take the TMA Pi kernel: the variant chosen, its configuration, whole blocks
static bool pi_tma_applies(const tgh_problem* p, const RhsArgs& a) {
  return p->pi_variant == PI_TMA && p->q == 4 && p->N == 32 && !p->mixed && a.p0 % p->S == 0 && a.p1 % p->S == 0;
}

// the tensor maps of one of the problem's working arrays (made once per array)
static const PiTmaMaps* pi_tma_maps(tgh_problem* p, const double* work) {
  for (auto& e : p->tma_maps)
    if (e.first == work) return &e.second;
  PiTmaMaps m;
  std::string err;
  if (!make_pi_tma_maps(const_cast<double*>(work), p->nwb, &m, err)) {
    p->err = err;
    return nullptr;
  }
  p->tma_maps.push_back({work, m});
  return &p->tma_maps.back().second;
}

// The blocks of this rank that can hold a point with r < r_1 while t runs over [tlo, thi]: their
// boxes lie within r_1 of the axis-aligned box around the centre's path c0 + t v (a superset; the
// kernel decides point by point). Built on the host, copied to the list's device buffer.
static int interior_blocks(tgh_problem* p, tgh_problem::BlockList& L, double tlo, double thi) {
  if (!p->intr) return TGH_OK;
  if (L.n >= 0 && L.lo == tlo && L.hi == thi) return TGH_OK;
  if (!L.dev) CK(cudaMalloc(&L.dev, (size_t)p->nb * sizeof(int)));
  double clo[3], chi[3];
  for (int d = 0; d < 3; ++d) {
    const double a = p->cfg.int_c0[d] + tlo * p->cfg.int_v[d], b = p->cfg.int_c0[d] + thi * p->cfg.int_v[d];
    clo[d] = std::min(a, b);
    chi[d] = std::max(a, b);
  }
  std::vector<int> v;
  for (int b = 0; b < p->nb; ++b) {
    const int g = p->i2g[b];
    const double h = std::ldexp(p->h0, -p->level[g]);
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double lo = p->lo[d] + p->corner[3 * g + d] * h, hi = lo + p->N * h;
      const double gap = std::max(0.0, std::max(lo - chi[d], clo[d] - hi));
      d2 += gap * gap;
    }
    if (std::sqrt(d2) <= p->cfg.r1 * (1.0 + 1e-12) + 1e-12) v.push_back(b);
  }
  if (!v.empty())
    CK(cudaMemcpyAsync(L.dev, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, p->stream));
  CK(cudaStreamSynchronize(p->stream));  // the host vector goes out of scope
  L.n = (int)v.size();
  L.lo = tlo;
  L.hi = thi;
  return TGH_OK;
}

// One right-hand side over all blocks on the problem's stream: the interior's points (a problem
// with an interior, over the blocks of the list in use), the head kernel, then the Pi kernel.
// a :fitted interior relaxes toward the target cache, which must have been filled or set
// (GHProblem refuses a :fitted interior without its target, src/evolution.jl:1132-1136)
static int fitted_ready(tgh_problem* p) {
  if (p->cfg.interior == TGH_INT_FITTED && !p->target_set)
    return fail(p, TGH_ERR_ARG, "a :fitted interior relaxes toward the target cache: fill or set it first "
                                "(tgh_set_target, tgh_fill_target_snapshot, tgh_fill_target_analytic)");
  return TGH_OK;
}

static int launch_interior(tgh_problem* p, const RhsArgs& a, int mode, cudaStream_t s) {
  if (int st = fitted_ready(p)) return st;
  const tgh_problem::BlockList* L = p->ilist_use;
  if (!L) {
    // a direct launch: the list for this t
    int st = interior_blocks(p, p->ilist, a.t, a.t);
    if (st) return st;
    L = &p->ilist;
  }
  if (L->n > 0) {
    const long per = (p->S + 127) / 128;
    if (mode == MODE_DU)
      interior_kernel<MODE_DU><<<(unsigned)(L->n * per), 128, 0, s>>>(p->cs, a, L->dev);
    else
      interior_kernel<MODE_STAGE><<<(unsigned)(L->n * per), 128, 0, s>>>(p->cs, a, L->dev);
    CK(cudaGetLastError());
  }
  return TGH_OK;
}

static int launch_rhs(tgh_problem* p, const RhsArgs& a, int mode) {
  if (p->intr && !p->interior_done) {
    int s = launch_interior(p, a, mode, p->stream);
    if (s) return s;
  }
  CK(launch_part(p, 0, mode, p->stream, a));
  if (pi_tma_applies(p, a)) {
    const PiTmaMaps* M = pi_tma_maps(p, a.work);
    if (!M) return TGH_ERR_CUDA;
    CK(launch_pi_tma(p->diss, mode, p->stream, p->cs, a, *M, PiTmaStatus{p->dev_err, p->wait_limit},
                     (int)(a.p0 / p->S), (int)((a.p1 - a.p0) / p->S)));
    return TGH_OK;
  }
  CK(launch_part(p, 1, mode, p->stream, a));
  return TGH_OK;
}

static RhsArgs base_args(tgh_problem* p, const double* work, double t) {
  RhsArgs a;
  std::memset(&a, 0, sizeof(a));
  a.work = work;
  a.Hsrc = p->Hsrc;
  a.coef = p->coef;
  a.blk = p->blk;
  a.N1 = p->N1;
  a.Wd = p->Wd;
  a.Wx = p->Wx;
  a.G = p->G;
  a.npts = p->npts;
  a.p0 = 0;
  a.p1 = p->npts;
  a.t = t;
  a.threads = p->threads;
  a.pi_mb = p->pi_mb;
  return a;
}

// StateBounds' checks (src/bounds.jl:81-147): "" when the ranges are acceptable
static std::string bounds_problem(const tgh_bounds& b) {
  const double v[7] = {b.alpha_min, b.alpha_max, b.lambda_min, b.lambda_max, b.beta_max, b.K_max, b.r_gate};
  for (double x : v)
    if (!std::isfinite(x))
      return "every bound must be finite: a bound at infinity is no bound, and it is spelled by setting "
             "no bounds";
  if (!(0 < b.alpha_min && b.alpha_min < 1 && 1 < b.alpha_max))
    return "the lapse range needs 0 < alpha_min < 1 < alpha_max, got alpha_min = " + std::to_string(b.alpha_min) +
           " and alpha_max = " + std::to_string(b.alpha_max) +
           ": flat space's alpha = 1 must lie inside, since a non-finite component is repaired to its "
           "Minkowski value";
  if (!(0 < b.lambda_min && b.lambda_min < 1 && 1 < b.lambda_max))
    return "the spatial metric's eigenvalue range needs 0 < lambda_min < 1 < lambda_max, got lambda_min = " +
           std::to_string(b.lambda_min) + " and lambda_max = " + std::to_string(b.lambda_max);
  if (!(b.beta_max > 0)) return "the shift's norm bound must be positive, got beta_max = " + std::to_string(b.beta_max);
  if (!(b.K_max > 0)) return "the momentum's scale bound must be positive, got K_max = " + std::to_string(b.K_max);
  if (!(b.r_gate > 0))
    return "the gate radius must be positive, got r_gate = " + std::to_string(b.r_gate) +
           ": a projection that never runs is spelled by setting no bounds";
  return "";
}

// apply_bounds! (src/bounds.jl:749-779): the projection over u, its counts over the primaries
static int apply_bounds_impl(tgh_problem* p, double* u, double t, const tgh_bounds& b, long* fired, long* nonfinite,
                             double* rmax) {
  const std::string why = bounds_problem(b);
  if (!why.empty()) return fail(p, TGH_ERR_ARG, why);
  if (!p->intr) return fail(p, TGH_ERR_ARG, "the range projection's gate is a radius from the interior's centre; "
                                            "this problem has no interior");
  BoundsArgs a;
  a.u = u;
  a.blk = p->blk;
  a.primary = p->primary;
  a.counts = p->bcounts;
  a.amin = b.alpha_min;
  a.amax = b.alpha_max;
  a.lmin = b.lambda_min;
  a.lmax = b.lambda_max;
  a.bmax = b.beta_max;
  a.kmax = b.K_max;
  a.rgate = b.r_gate;
  a.t = t;
  a.S = p->S;
  a.npts = p->npts;
  a.N1 = p->N1;
  CK(launch_bounds_projection(p->stream, p->cs, a));
  unsigned long long h[3];
  CK(cudaMemcpyAsync(h, p->bcounts, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  *fired = (long)h[0];
  *nonfinite = (long)h[1];
  double r;
  std::memcpy(&r, &h[2], sizeof(r));
  *rmax = r;
  return TGH_OK;
}

// gh_stage_limiter! then gh_step_limiter! (src/stepping.jl:91-95): the range projection, when
// the problem has bounds, with its accounting (src/bounds.jl:757-776); then the :pasted paste
static int stage_limit_impl(tgh_problem* p, double* u, double t) {
  if (p->has_bounds) {
    long n = 0, nf = 0;
    double rm = 0.0;
    int s = apply_bounds_impl(p, u, t, p->bounds, &n, &nf, &rm);
    if (s) return s;
    ++p->acc_calls;
    if (n > 0) {
      p->acc_hits += n;
      p->acc_nonfinite += nf;
      p->acc_rmax = std::max(p->acc_rmax, rm);
      if (std::isnan(p->acc_first_t)) {
        p->acc_first_t = t;
        p->acc_first_r = rm;
      }
    }
  }
  if (p->cfg.interior != TGH_INT_PASTED) return TGH_OK;
  exact_state_kernel<<<grid_for(p->npts, 128), 128, 0, p->stream>>>(u, p->blk, p->geo, p->npts, p->cs, t, 1);
  CK(cudaGetLastError());
  return TGH_OK;
}

extern "C" {

// A problem over the leaves `owner` gives to `rank` of `nranks` (owner null: every leaf, one
// rank). Its working arrays also hold the halo blocks its fill reads from other ranks.
static int setup_host(tgh_problem* p, const tgh_config* cfg, const tgh_mesh* m, const int* owner, int rank,
                      int nranks, int margin_check);
static int setup_device(tgh_problem* p);

static int create_impl(const tgh_config* cfg, const tgh_mesh* m, const int* owner, int rank, int nranks,
                       void* cuda_stream, int margin_check, tgh_problem** out) {
  *out = nullptr;
  tgh_problem* p = new tgh_problem();
  *out = p;
  p->stream = (cudaStream_t)cuda_stream;
  int s = setup_host(p, cfg, m, owner, rank, nranks, margin_check);
  if (s) return s;
  // the fill plan fixes the internal numbering (own leaves, then the halo)
  if ((s = build_plan(p))) return s;
  return setup_device(p);
}

// The problem's host state: the checked configuration, the forest, the owner ranks.
static int setup_host(tgh_problem* p, const tgh_config* cfg, const tgh_mesh* m, const int* owner, int rank,
                      int nranks, int margin_check) {
  p->cfg = *cfg;
  const int q = cfg->q;
  if (q < 2 || q > 8 || q % 2) return fail(p, TGH_ERR_ARG, "the finite-difference order must be even and in 2..8, got " + std::to_string(q));
  if (m->N < 2 * (q / 2 + 1)) return fail(p, TGH_ERR_ARG, "the block edge N must be at least 2G");
  if (m->nblocks < 1) return fail(p, TGH_ERR_ARG, "the forest has no leaves");
  if (nranks < 1 || rank < 0 || rank >= nranks) return fail(p, TGH_ERR_ARG, "the rank must lie in 0 .. nranks - 1");
  p->rank = rank;
  p->nranks = nranks;
  p->owner.assign(m->nblocks, 0);
  if (owner) {
    for (int g = 0; g < m->nblocks; ++g) {
      if (owner[g] < 0 || owner[g] >= nranks) return fail(p, TGH_ERR_ARG, "a leaf's owner rank is out of range");
      p->owner[g] = owner[g];
    }
  }
  p->nb = (int)std::count(p->owner.begin(), p->owner.end(), rank);
  if (p->nb < 1) return fail(p, TGH_ERR_ARG, "this rank owns no leaf");
  p->q = q;
  p->G = q / 2 + 1;
  p->N = m->N;
  p->N1 = m->N + 1;
  p->Wd = m->N + 2 * p->G + 1;
  p->Wx = p->Wd + (p->Wd & 1);
  p->h0 = m->h0;
  for (int d = 0; d < 3; ++d) {
    p->lo[d] = m->lo[d];
    p->cells0[d] = m->cells0[d];
    p->periodic[d] = m->periodic[d];
    if (m->cells0[d] % m->N) return fail(p, TGH_ERR_ARG, "the domain is not a whole number of blocks");
  }
  p->level.assign(m->level, m->level + m->nblocks);
  p->corner.assign(m->corner, m->corner + 3 * m->nblocks);
  for (int b = 0; b < m->nblocks; ++b) {
    if (p->level[b] < 0 || p->level[b] > 20) return fail(p, TGH_ERR_ARG, "block level out of range");
    p->maxlevel = std::max(p->maxlevel, p->level[b]);
    for (int d = 0; d < 3; ++d)
      if (p->corner[3 * b + d] % p->N) return fail(p, TGH_ERR_ARG, "a block corner is not a multiple of N");
  }
  p->lut.resize(p->maxlevel + 1);
  for (int b = 0; b < m->nblocks; ++b) {
    auto key = bkey(p->corner[3 * b] / p->N, p->corner[3 * b + 1] / p->N, p->corner[3 * b + 2] / p->N);
    if (!p->lut[p->level[b]].emplace(key, b).second) return fail(p, TGH_ERR_ARG, "two leaves share a corner and level");
  }
  p->S = (long)p->N1 * p->N1 * p->N1;
  p->Wv = (long)p->Wx * p->Wd * p->Wd;
  p->npts = p->S * p->nb;
  p->geo = Geo{p->N1, p->Wd, p->G, p->Wx, p->S, p->Wv};
  if (cfg->bg.kind < TGH_BG_MINKOWSKI || cfg->bg.kind > TGH_BG_HARMONIC_KERR)
    return fail(p, TGH_ERR_ARG, "unknown background kind");
  if (cfg->interior < TGH_INT_NONE || cfg->interior > TGH_INT_FITTED)
    return fail(p, TGH_ERR_ARG, "unknown interior variant");
  if (cfg->bg.kind == TGH_BG_HARMONIC_KERR && !(std::fabs(cfg->bg.a) < cfg->bg.M))
    return fail(p, TGH_ERR_ARG, "the harmonic chart needs |a| < M (its time function has a log at r_-)");
  p->cs = make_case(*cfg);
  p->diss = cfg->dissipation == TGH_DISS_CONSTANT ? cfg->eps_ko != 0.0 : !(cfg->eps_out == 0.0 && cfg->eps_in == 0.0);
  p->intr = cfg->interior != TGH_INT_NONE;
  if (cfg->precision != TGH_PREC_FP64 && cfg->precision != TGH_PREC_MIXED)
    return fail(p, TGH_ERR_ARG, "the precision must be TGH_PREC_FP64 or TGH_PREC_MIXED");
  p->mixed = cfg->precision == TGH_PREC_MIXED;
  if (p->intr) {
    if (!(cfg->r0 > 0.0 && cfg->r1 > cfg->r0))
      return fail(p, TGH_ERR_RADII, "the interior needs 0 < r_0 < r_1");
    if (!(cfg->w_ramp > 0 && cfg->w_ramp <= 1 && cfg->rho_ramp > 0 && cfg->rho_ramp <= 1))
      return fail(p, TGH_ERR_ARG, "the ramp fractions must lie in (0, 1]");
    if (margin_check) {
      // the layer must be resolved: r_1 - r_0 >= 2 (G + 1) h at the finest spacing present
      const double hmin = std::ldexp(p->h0, -p->maxlevel);
      if (cfg->r1 - cfg->r0 < 2.0 * (p->G + 1) * hmin)
        return fail(p, TGH_ERR_RADII, "the damping layer is too thin: r_1 - r_0 < 2(G+1)h");
      if ((cfg->bg.kind == TGH_BG_KERR_SCHILD || cfg->bg.kind == TGH_BG_HARMONIC_KERR) &&
          cfg->r0 <= std::fabs(cfg->bg.a))
        return fail(p, TGH_ERR_RADII, "the frozen core does not contain the chart's singular disk |x| <= |a|");
    }
  }
  return TGH_OK;
}

// Whether the analytic state at a fixed position is the same at every time: a static
// background (Minkowski, shifted Minkowski, Kerr-Schild without a boost) and an interior that
// does not move. Its Dirichlet ghosts are then evaluated once.
static bool stationary(const tgh_config& c) {
  const double* u = c.bg.boost;
  const bool bg = c.bg.kind == TGH_BG_MINKOWSKI || c.bg.kind == TGH_BG_SHIFTED_MINKOWSKI ||
                  ((c.bg.kind == TGH_BG_KERR_SCHILD || c.bg.kind == TGH_BG_HARMONIC_KERR) && u[0] == 0.0 &&
                   u[1] == 0.0 && u[2] == 0.0);
  const bool core = c.interior == TGH_INT_NONE || (c.int_v[0] == 0.0 && c.int_v[1] == 0.0 && c.int_v[2] == 0.0);
  return bg && core;
}

// The problem's device state, once the plan has fixed the internal block numbering.
static int setup_device(tgh_problem* p) {
  const tgh_config* cfg = &p->cfg;
  if (p->nhooks && stationary(*cfg)) CK(cudaMalloc(&p->hook_cache, (size_t)p->nhooks * NV * sizeof(double)));
  // per-block geometry, internal numbering
  std::vector<double> blk(8 * (size_t)p->nwb, 0.0);
  for (int b = 0; b < p->nwb; ++b) {
    const int g = p->i2g[b];
    for (int d = 0; d < 3; ++d) {
      blk[8 * b + d] = p->lo[d];
      blk[8 * b + 4 + d] = (double)p->corner[3 * g + d];
    }
    blk[8 * b + 3] = std::ldexp(p->h0, -p->level[g]);
  }
  CK(cudaMalloc(&p->blk, blk.size() * sizeof(double)));
  CK(cudaMemcpy(p->blk, blk.data(), blk.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&p->work, (size_t)p->Wv * NV * p->nwb * sizeof(double)));
  CK(cudaMemsetAsync(p->work, 0, (size_t)p->Wv * NV * p->nwb * sizeof(double), p->stream));
  CK(cudaMalloc(&p->scratch, 2 * sizeof(unsigned long long)));
  CK(cudaMalloc(&p->bcounts, 3 * sizeof(unsigned long long)));
  CK(cudaMalloc(&p->dev_err, sizeof(int)));
  CK(cudaMemsetAsync(p->dev_err, 0, sizeof(int), p->stream));
  CK(cudaMalloc(&p->coef, (size_t)NCOEF * p->npts * sizeof(double)));
  p->npart = (int)grid_for(p->npts, 128);
  CK(cudaMalloc(&p->part, (3 * (size_t)p->npart + 2) * sizeof(double)));
  CK(cudaMalloc(&p->diag, (size_t)NDIAG * p->npts * sizeof(double)));
  CK(cudaMemsetAsync(p->diag, 0, (size_t)NDIAG * p->npts * sizeof(double), p->stream));
  CK(cudaMalloc(&p->dpart, (17 * (size_t)p->npart + 17) * sizeof(double)));
  CK(cudaMalloc(&p->ind, 16 * sizeof(unsigned long long)));
  CK(cudaMalloc(&p->ind_tol, 4 * sizeof(double)));
  CK(cudaMalloc(&p->ind_counts, 4 * (size_t)p->nb * sizeof(int)));
  CK(cudaMalloc(&p->ind_boxes, 24 * (size_t)p->nb * sizeof(int)));
  if (cfg->gauge == TGH_GAUGE_SAMPLED) {
    CK(cudaMalloc(&p->Hsrc, (size_t)p->S * NV * p->nb * sizeof(double)));
    sample_gauge_kernel<<<grid_for(p->npts, 64), 64, 0, p->stream>>>(p->Hsrc, p->blk, p->geo, p->npts, p->cs, 0.0);
    CK(cudaGetLastError());
  }
  if (cfg->interior == TGH_INT_FITTED) {
    const size_t L = (size_t)p->S * 2 * NV * p->nb;
    CK(cudaMalloc(&p->tw, L * sizeof(double)));
    CK(cudaMemsetAsync(p->tw, 0, L * sizeof(double), p->stream));
    CK(cudaMalloc(&p->tf, sizeof(double)));
    CK(cudaMemsetAsync(p->tf, 0, sizeof(double), p->stream));
    p->cs.tw = p->tw;
    p->cs.tf = p->tf;
    p->cs.trate = cfg->target_rate != 0;
  }
  CK(cudaStreamSynchronize(p->stream));
  return TGH_OK;
}

int tgh_problem_create(const tgh_config* cfg, const tgh_mesh* m, void* cuda_stream, int margin_check,
                       tgh_problem** out) {
  return create_impl(cfg, m, nullptr, 0, 1, cuda_stream, margin_check, out);
}

int tgh_problem_create_shard(const tgh_config* cfg, const tgh_mesh* m, const int* owner, int rank, int nranks,
                             void* cuda_stream, int margin_check, tgh_problem** out) {
  return create_impl(cfg, m, owner, rank, nranks, cuda_stream, margin_check, out);
}

void tgh_problem_destroy(tgh_problem* p) {
  if (!p) return;
  if (p->gexec) cudaGraphExecDestroy(p->gexec);
  if (p->cap) cudaStreamDestroy(p->cap);
  if (p->side) cudaStreamDestroy(p->side);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  for (auto& x : p->xch) {
    if (x.send) cudaFree(x.send);
    if (x.recv) cudaFree(x.recv);
  }
  void* bufs[] = {p->work, p->Hsrc, p->tw, p->tf, p->blk, p->primary, p->runs, p->gpts, p->hooks, p->hook_cache, p->scratch,
                  p->bcounts, p->dev_err, p->ilist.dev, p->ilist_graph.dev,
                  p->part, p->coef, p->diag, p->dpart, p->ind, p->ind_tol, p->ind_counts, p->ind_boxes,
                  p->k, p->acc, p->y, p->u0, p->W1, p->W2, p->bacc, p->twork, p->kt, p->acct, p->yt,
                  p->adj_cot, p->adj_mu, p->adj_part, p->adj_y[0], p->adj_y[1], p->adj_y[2], p->adj_a,
                  p->adj_acc, p->adj_m};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (auto* pp : p->prol)
    if (pp) cudaFree(pp);
  for (auto* pp : p->ptile)
    if (pp) cudaFree(pp);
  for (auto* pp : p->ptpts)
    if (pp) cudaFree(pp);
  delete p;
}

const char* tgh_last_error(const tgh_problem* p) { return p ? p->err.c_str() : "no problem"; }
size_t tgh_state_length(const tgh_problem* p) { return (size_t)p->S * NV * p->nb; }

int tgh_fill_counts(const tgh_problem* p, long long counts[4]) {
  if (!p || !counts) return TGH_ERR_ARG;
  counts[0] = p->ngpts;
  counts[1] = p->nhooks;
  counts[2] = counts[3] = 0;
  for (size_t l = 0; l < p->nprol.size(); ++l) counts[2] += p->nprol[l];
  for (size_t l = 0; l < p->ntile.size(); ++l) counts[3] += std::max(0, p->ntile[l]);
  return TGH_OK;
}
// The ABI's view of the working array is the reference's layout, (N+2G+1)^3 points per block
// and variable; the problem stores rows padded to the even pitch Wx.
size_t tgh_work_length(const tgh_problem* p) { return (size_t)p->Wd * p->Wd * p->Wd * NV * p->nwb; }

int tgh_copy_work(tgh_problem* p, double* dst) { return tgh_copy_work_blocks(p, 0, p->nwb, dst); }

int tgh_copy_work_blocks(tgh_problem* p, int b0, int nblocks, double* dst) {
  if (b0 < 0 || nblocks < 0 || b0 + nblocks > p->nwb) return fail(p, TGH_ERR_ARG, "block range out of bounds");
  if (nblocks == 0) return TGH_OK;
  // one row of Wd doubles per copy: rows of the padded array are Wx apart, of the dense one Wd
  const size_t rows = (size_t)p->Wd * p->Wd * NV * nblocks;
  CK(cudaMemcpy2DAsync(dst, (size_t)p->Wd * sizeof(double), p->work + (size_t)p->Wv * NV * b0,
                       (size_t)p->Wx * sizeof(double), (size_t)p->Wd * sizeof(double), rows, cudaMemcpyDeviceToDevice,
                       p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return TGH_OK;
}

// the fill of u into the working array, shared by tgh_prepare and the verbs that prepare for
// their own use (which then mark the array overwritten)
static int prepare_impl(tgh_problem* p, const double* u, double t, const char* who) {
  const int s = launch_fill(p, u, false, p->work, t);
  if (who) work_overwritten(p, who);
  return s;
}

int tgh_prepare(tgh_problem* p, const double* u, double t) {
  const int s = prepare_impl(p, u, t, nullptr);
  if (s) {
    work_overwritten(p, "a tgh_prepare that failed");
    return s;
  }
  ++p->prep_gen;
  p->work_prepared = true;
  return TGH_OK;
}

int tgh_prepare_generation(const tgh_problem* p, long* generation, int* current) {
  *generation = p->prep_gen;
  *current = p->work_prepared ? 1 : 0;
  return TGH_OK;
}

// ---- the constraint monitors (src/constraints.jl:535-609) ----
static int monitor_prepare(tgh_problem* p, const double* u, double t, int mask, MonArgs& a) {
  if (p->nranks > 1) return fail(p, TGH_ERR_ARG, "the constraint monitors run on a problem of one rank");
  if (mask != TGH_MASK_INTERIOR && mask != TGH_MASK_ALL)
    return fail(p, TGH_ERR_ARG, "mask must be TGH_MASK_INTERIOR or TGH_MASK_ALL");
  int s = prepare_impl(p, u, t, "a constraint monitor or the refinement indicator");
  if (s) return s;
  std::memset(&a, 0, sizeof(a));
  a.work = p->work;
  a.Hsrc = p->Hsrc;
  a.blk = p->blk;
  a.diag = p->diag;
  a.N1 = p->N1;
  a.Wd = p->Wd;
  a.Wx = p->Wx;
  a.G = p->G;
  a.all = mask == TGH_MASK_ALL;
  a.S = p->S;
  a.Wv = p->Wv;
  a.npts = p->npts;
  a.t = t;
  return TGH_OK;
}

int tgh_gh_constraint(tgh_problem* p, const double* u, double t, int mask) {
  MonArgs a;
  int s = monitor_prepare(p, u, t, mask, a);
  if (s) return s;
  CK(launch_gauge_constraint(p->q, p->stream, p->cs, a));
  return TGH_OK;
}

int tgh_adm_constraint(tgh_problem* p, const double* u, double t, int mask, const double* matter) {
  MonArgs a;
  int s = monitor_prepare(p, u, t, mask, a);
  if (s) return s;
  a.matter = matter;
  CK(launch_adm_constraint(p->q, p->stream, p->cs, a));
  return TGH_OK;
}

int tgh_constraint_norms(tgh_problem* p, int weighting, int at_level, double* out) {
  if (weighting != 0 && weighting != 1) return fail(p, TGH_ERR_ARG, "weighting must be 0 (volume) or 1 (points)");
  if (at_level > 20) return fail(p, TGH_ERR_ARG, "at_level out of range");
  const double hsel = at_level < 0 ? -1.0 : std::ldexp(p->h0, -at_level);
  diag_norms_kernel<<<p->npart, 128, 0, p->stream>>>(p->diag, p->primary, p->blk, p->S, p->npts, weighting == 0,
                                                      hsel, p->dpart);
  CK(cudaGetLastError());
  double* fold = p->dpart + 17 * (size_t)p->npart;
  diag_norms_fold_kernel<<<17, 256, 0, p->stream>>>(p->dpart, p->npart, fold);
  CK(cudaGetLastError());
  double r[17];
  CK(cudaMemcpyAsync(r, fold, sizeof(r), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  const double vol = r[0];
  double l2[8];
  for (int s = 0; s < 8; ++s) l2[s] = vol == 0.0 ? 0.0 : std::sqrt(r[1 + s] / vol);
  for (int a = 0; a < 4; ++a) {
    out[a] = l2[DG_CGH + a];
    out[4 + a] = r[9 + DG_CGH + a];
  }
  out[8] = l2[DG_HAM];
  out[9] = r[9 + DG_HAM];
  for (int a = 0; a < 3; ++a) {
    out[10 + a] = l2[DG_MOM + a];
    out[13 + a] = r[9 + DG_MOM + a];
  }
  return TGH_OK;
}

// ---- the masked Loehner indicator (src/refinement.jl:280-400) ----
int tgh_tau(tgh_problem* p, const double* u, double t, int mask, double eps, double scale, double* out) {
  if (!(eps > 0.0)) return fail(p, TGH_ERR_ARG, "the noise floor's coefficient eps must be positive");
  MonArgs a;
  int s = monitor_prepare(p, u, t, mask, a);
  if (s) return s;
  CK(cudaMemsetAsync(p->ind, 0, 11 * sizeof(unsigned long long), p->stream));
  const unsigned nb = (unsigned)grid_for(p->npts, 128);
  field_scales_kernel<<<nb, 128, 0, p->stream>>>(a, p->cs, p->ind);
  CK(cudaGetLastError());
  unsigned long long bits[11];
  CK(cudaMemcpyAsync(bits, p->ind, 10 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  double sc = 0.0;
  for (int v = 0; v < NC; ++v) {
    double x;
    std::memcpy(&x, &bits[v], sizeof(x));
    out[v] = x;
    sc = (x != x || sc != sc) ? x + sc : std::max(sc, x);
  }
  if (scale > 0.0) sc = scale;
  const double floor4 = (4.0 * eps) * std::fabs(sc);
  tau_kernel<<<nb, 128, 0, p->stream>>>(a, p->cs, floor4, p->ind + 10);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&bits[10], p->ind + 10, sizeof(unsigned long long), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  out[10] = sc;
  std::memcpy(&out[11], &bits[10], sizeof(double));
  return TGH_OK;
}

int tgh_firing(tgh_problem* p, int ntol, const double* tol, int* counts, int* boxes) {
  if (p->nranks > 1) return fail(p, TGH_ERR_ARG, "the indicator runs on a problem of one rank");
  if (ntol < 1 || ntol > 4) return fail(p, TGH_ERR_ARG, "between 1 and 4 thresholds");
  MonArgs a;
  std::memset(&a, 0, sizeof(a));
  a.diag = p->diag;
  a.N1 = p->N1;
  a.S = p->S;
  a.npts = p->npts;
  CK(cudaMemcpyAsync(p->ind_tol, tol, ntol * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  const int n = p->nb * ntol;
  firing_init_kernel<<<(unsigned)grid_for(n, 128), 128, 0, p->stream>>>(n, p->N1, p->ind_counts, p->ind_boxes);
  CK(cudaGetLastError());
  firing_kernel<<<(unsigned)grid_for(p->npts, 128), 128, 0, p->stream>>>(a, ntol, p->ind_tol, p->ind_counts,
                                                                          p->ind_boxes);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(counts, p->ind_counts, n * sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaMemcpyAsync(boxes, p->ind_boxes, 6 * (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return TGH_OK;
}

size_t tgh_diag_length(const tgh_problem* p) { return (size_t)NDIAG * p->npts; }

// ---- the regrid's state transfer (TreeAMR's regrid! with the fill's operators) ----
// Every owned point of every leaf of `dst` takes the value its lattice point has in the filled
// working array of `src` at t: copied from the finest src leaf holding it at its level or finer
// (the primary copy; injection from a finer leaf), else prolonged (order q + 2) from the src leaf
// one level coarser that covers it. The plan is built here on the host and released after: a
// regrid runs once per chunk of steps.
int tgh_transfer(tgh_problem* dst, tgh_problem* src, const double* u_src, double t, double* u_dst) {
  if (dst->nranks > 1 || src->nranks > 1) return fail(dst, TGH_ERR_ARG, "the transfer runs on problems of one rank");
  bool same = dst->q == src->q && dst->N == src->N && dst->h0 == src->h0;
  for (int d = 0; d < 3; ++d)
    same = same && dst->lo[d] == src->lo[d] && dst->cells0[d] == src->cells0[d] && dst->periodic[d] == src->periodic[d];
  if (!same) return fail(dst, TGH_ERR_ARG, "the two problems differ in order, block size or root grid");
  int s = prepare_impl(src, u_src, t, "tgh_transfer (as its source)");
  if (s) return s;
  const int G = src->G, Wd = src->Wd, Wx = src->Wx, P = src->q + 2;
  std::vector<CopyPt> cp;
  std::vector<ProlongPt> pp;
  for (int b = 0; b < dst->nb; ++b) {
    const int gb = dst->i2g[b], l = dst->level[gb];
    for (int k = 0; k < dst->N1; ++k)
      for (int j = 0; j < dst->N1; ++j)
        for (int i = 0; i < dst->N1; ++i) {
          const int ip = i + dst->N1 * (j + dst->N1 * k);
          int64_t n[3] = {(int64_t)dst->corner[3 * gb] + i, (int64_t)dst->corner[3 * gb + 1] + j,
                          (int64_t)dst->corner[3 * gb + 2] + k};
          for (int d = 0; d < 3; ++d)
            if (dst->periodic[d]) {
              const int64_t per = (int64_t)dst->cells0[d] << l;
              n[d] %= per;
              if (n[d] < 0) n[d] += per;
            }
          int leaf, loc[3], lev;
          if (find_owner(src, l, n, leaf, loc, lev)) {
            const int sw = (loc[0] + G) + Wx * ((loc[1] + G) + Wd * (loc[2] + G));
            cp.push_back(CopyPt{b, ip, src->g2i[leaf], sw});
            continue;
          }
          const int c = l > 0 ? coarse_cover(src, l - 1, n) : -1;
          if (c < 0) return fail(dst, TGH_ERR_ARG, "a point of the new forest is covered by no leaf of the old one "
                                                   "at its level or one coarser (a leaf refined twice at once?)");
          int odd = 0;
          int64_t base[3];
          for (int d = 0; d < 3; ++d) {
            base[d] = (n[d] & 1) ? (n[d] >> 1) - (P / 2 - 1) : n[d] >> 1;
            if (n[d] & 1) odd |= 1 << d;
            const int64_t rel = base[d] - src->corner[3 * c + d] + G;
            if (rel < 0 || rel + ((n[d] & 1) ? P : 1) > Wd)
              return fail(dst, TGH_ERR_ARG, "a prolongation stencil of the transfer leaves the old block's ghost zone");
          }
          const int sw = (int)((base[0] - src->corner[3 * c] + G) +
                               Wx * ((base[1] - src->corner[3 * c + 1] + G) + (int64_t)Wd * (base[2] - src->corner[3 * c + 2] + G)));
          pp.push_back(ProlongPt{b, ip, src->g2i[c], sw, odd});
        }
  }
  std::stable_sort(pp.begin(), pp.end(), [](const ProlongPt& a, const ProlongPt& b) { return a.odd < b.odd; });
  tgh_problem* p = dst;  // where a CUDA failure is reported
  struct Plan {
    CopyPt* cp = nullptr;
    ProlongPt* pp = nullptr;
    ~Plan() {
      cudaFree(cp);
      cudaFree(pp);
    }
  } plan;
  CopyPt*& dcp = plan.cp;
  ProlongPt*& dpp = plan.pp;
  CK(cudaMalloc(&dcp, std::max<size_t>(1, cp.size()) * sizeof(CopyPt)));
  CK(cudaMalloc(&dpp, std::max<size_t>(1, pp.size()) * sizeof(ProlongPt)));
  CK(cudaMemcpy(dcp, cp.data(), cp.size() * sizeof(CopyPt), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dpp, pp.data(), pp.size() * sizeof(ProlongPt), cudaMemcpyHostToDevice));
  const int T = 256;
  if (!cp.empty())
    transfer_copy_kernel<<<grid_for((long)cp.size(), T), T, 0, src->stream>>>(dcp, (long)cp.size(), src->work,
                                                                               src->geo, u_dst, dst->S);
  CK(cudaGetLastError());
  if (!pp.empty()) {
    const int np = (int)pp.size();
    const long n = (long)np * NV;
    switch (P) {
      case 4: transfer_prolong_kernel<4><<<grid_for(n, T), T, 0, src->stream>>>(dpp, np, src->work, src->geo, u_dst, dst->S); break;
      case 6: transfer_prolong_kernel<6><<<grid_for(n, T), T, 0, src->stream>>>(dpp, np, src->work, src->geo, u_dst, dst->S); break;
      case 8: transfer_prolong_kernel<8><<<grid_for(n, T), T, 0, src->stream>>>(dpp, np, src->work, src->geo, u_dst, dst->S); break;
      default: transfer_prolong_kernel<10><<<grid_for(n, T), T, 0, src->stream>>>(dpp, np, src->work, src->geo, u_dst, dst->S); break;
    }
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(src->stream));
  return TGH_OK;
}

int tgh_copy_diag(tgh_problem* p, double* out) {
  CK(cudaMemcpyAsync(out, p->diag, (size_t)NDIAG * p->npts * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  return TGH_OK;
}

// ---- the right-hand side's kernel variants (the autotuner's choices) and device waits ----
int tgh_set_variant(tgh_problem* p, int pi_variant, int threads, int pi_mb) {
  if (pi_variant != TGH_PI_L1 && pi_variant != TGH_PI_TMA) return fail(p, TGH_ERR_ARG, "unknown Pi kernel variant");
  if (pi_variant == TGH_PI_TMA && !(p->q == 4 && p->N == 32 && !p->mixed))
    return fail(p, TGH_ERR_ARG, "the TMA Pi kernel serves q = 4, N = 32, FP64 problems only");
  if (threads != 64 && threads != 128) return fail(p, TGH_ERR_ARG, "the CTA size must be 64 or 128");
  if (pi_mb < 3 || pi_mb > 5) return fail(p, TGH_ERR_ARG, "the one-point Pi kernel's CTAs per SM must be 3, 4 or 5");
  if (pi_variant == TGH_PI_TMA) {
    // check now that the driver can describe the working array to the copy engine
    if (!pi_tma_maps(p, p->work)) return TGH_ERR_CUDA;
  }
  p->pi_variant = pi_variant;
  p->threads = threads;
  p->pi_mb = pi_mb;
  if (p->gexec) {  // a captured step holds the old kernels
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  return TGH_OK;
}

int tgh_get_variant(const tgh_problem* p, int* pi_variant, int* threads, int* pi_mb) {
  *pi_variant = p->pi_variant;
  *threads = p->threads;
  *pi_mb = p->pi_mb;
  return TGH_OK;
}

int tgh_set_wait_limit(tgh_problem* p, long long polls) {
  p->wait_limit = polls;
  if (p->gexec) {
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  return TGH_OK;
}

int tgh_device_status(tgh_problem* p) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, p->dev_err, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  if (h == 0) return TGH_OK;
  CK(cudaMemsetAsync(p->dev_err, 0, sizeof(int), p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return fail(p, h, "a bounded wait inside a kernel gave up (its results were not written)");
}

int tgh_rhs(tgh_problem* p, double* du, double t, const double* matter) {
  if (!p->work_prepared)
    return fail(p, TGH_ERR_STALE, std::string("the working array no longer holds the last tgh_prepare's fill: ") +
                                      p->work_writer + " wrote it since; call tgh_prepare again");
  RhsArgs a = base_args(p, p->work, t);
  a.du = du;
  a.matter = matter;
  return launch_rhs(p, a, MODE_DU);
}

int tgh_gh_rhs(tgh_problem* p, double* du, const double* u, double t, const double* matter) {
  int s = tgh_prepare(p, u, t);
  return s ? s : tgh_rhs(p, du, t, matter);
}

int tgh_settle(tgh_problem* p, double* u, double t) {
  int s = tgh_prepare(p, u, t);
  if (s) return s;
  gather_kernel<<<grid_for(p->npts, 256), 256, 0, p->stream>>>(p->work, u, p->geo, p->npts);
  CK(cudaGetLastError());
  return TGH_OK;
}

int tgh_stage_limit(tgh_problem* p, double* u, double t) { return stage_limit_impl(p, u, t); }

int tgh_bounds_check(const tgh_bounds* b, char* errbuf, int errlen) {
  const std::string why = b ? bounds_problem(*b) : std::string("no bounds given");
  if (why.empty()) return TGH_OK;
  if (errbuf && errlen > 0) {
    std::strncpy(errbuf, why.c_str(), (size_t)errlen - 1);
    errbuf[errlen - 1] = 0;
  }
  return TGH_ERR_ARG;
}

int tgh_apply_bounds(tgh_problem* p, double* u, double t, const tgh_bounds* b, long* fired, long* nonfinite,
                     double* r_max) {
  if (!b) return fail(p, TGH_ERR_ARG, "no bounds given");
  return apply_bounds_impl(p, u, t, *b, fired, nonfinite, r_max);
}

int tgh_set_bounds(tgh_problem* p, const tgh_bounds* b) {
  if (b) {
    const std::string why = bounds_problem(*b);
    if (!why.empty()) return fail(p, TGH_ERR_ARG, why);
    if (!p->intr) return fail(p, TGH_ERR_ARG, "the range projection's gate is a radius from the interior's centre; "
                                              "this problem has no interior");
    p->bounds = *b;
  }
  p->has_bounds = b != nullptr;
  p->acc_calls = p->acc_hits = p->acc_nonfinite = 0;
  p->acc_rmax = 0.0;
  p->acc_first_t = p->acc_first_r = NAN;
  return TGH_OK;
}

int tgh_bounds_accounting(const tgh_problem* p, long* counts3, double* vals3) {
  counts3[0] = p->acc_calls;
  counts3[1] = p->acc_hits;
  counts3[2] = p->acc_nonfinite;
  vals3[0] = p->acc_rmax;
  vals3[1] = p->acc_first_t;
  vals3[2] = p->acc_first_r;
  return TGH_OK;
}
int tgh_step_limit(tgh_problem* p, double* u, double t) { return stage_limit_impl(p, u, t); }

int tgh_initial_state(tgh_problem* p, double* u, double t) {
  exact_state_kernel<<<grid_for(p->npts, 128), 128, 0, p->stream>>>(u, p->blk, p->geo, p->npts, p->cs, t, 0);
  CK(cudaGetLastError());
  return stage_limit_impl(p, u, t);
}

// ---- the :fitted target cache ----

static int fitted_check(tgh_problem* p) {
  if (!p) return TGH_ERR_ARG;
  if (p->cfg.interior != TGH_INT_FITTED) return fail(p, TGH_ERR_ARG, "the problem's interior is not :fitted");
  return TGH_OK;
}

int tgh_set_target(tgh_problem* p, const double* tw, double t_f) {
  if (int s = fitted_check(p)) return s;
  if (!tw || !std::isfinite(t_f)) return fail(p, TGH_ERR_ARG, "tgh_set_target needs a cache and a finite t_f");
  CK(cudaMemcpyAsync(p->tw, tw, (size_t)p->S * 2 * NV * p->nb * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  set_scalar_kernel<<<1, 1, 0, p->stream>>>(p->tf, t_f);
  CK(cudaGetLastError());
  p->target_set = true;
  return TGH_OK;
}

static int fill_target_impl(tgh_problem* p, const double* u, double t_f, double r_fill, double dt) {
  if (int s = fitted_check(p)) return s;
  if (!std::isfinite(t_f) || !(r_fill >= 0.0) || !(dt >= 0.0))
    return fail(p, TGH_ERR_ARG, "the fill needs a finite t_f, r_fill >= 0 and dt >= 0");
  const int phases = (!u && dt > 0.0) ? 3 : 1;
  for (int ph = 0; ph < phases; ++ph)
    fill_target_kernel<<<grid_for(p->npts, 128), 128, 0, p->stream>>>(p->tw, u, p->blk, p->geo, p->npts, p->cs,
                                                                      t_f, r_fill, dt, ph);
  set_scalar_kernel<<<1, 1, 0, p->stream>>>(p->tf, t_f);
  CK(cudaGetLastError());
  p->target_set = true;
  return TGH_OK;
}

int tgh_fill_target_snapshot(tgh_problem* p, const double* u, double t_f, double r_fill) {
  if (!u) return fail(p, TGH_ERR_ARG, "the snapshot target needs a state");
  return fill_target_impl(p, u, t_f, r_fill, 0.0);
}

int tgh_fill_target_analytic(tgh_problem* p, double t_f, double r_fill, double dt) {
  return fill_target_impl(p, nullptr, t_f, r_fill, dt);
}

int tgh_fitted_initial_state(tgh_problem* p, double* u, double t, double d_init) {
  if (int s = fitted_check(p)) return s;
  if (int s = fitted_ready(p)) return s;
  if (!u || !(d_init >= 0.0 && d_init <= p->cfg.r1 - p->cfg.r0))
    return fail(p, TGH_ERR_ARG, "the fitted initial state needs a state and 0 <= d_init <= r_1 - r_0");
  fitted_state_kernel<<<grid_for(p->npts, 128), 128, 0, p->stream>>>(u, p->blk, p->geo, p->npts, p->cs, t, d_init);
  CK(cudaGetLastError());
  return TGH_OK;
}

int tgh_copy_target(tgh_problem* p, double* out) {
  if (int s = fitted_check(p)) return s;
  if (!out) return fail(p, TGH_ERR_ARG, "tgh_copy_target needs a destination");
  CK(cudaMemcpyAsync(out, p->tw, (size_t)p->S * 2 * NV * p->nb * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  return TGH_OK;
}

int tgh_max_speed(tgh_problem* p, const double* u, double t, double* lambda) {
  CK(cudaMemsetAsync(p->scratch, 0, 2 * sizeof(unsigned long long), p->stream));
  speed_kernel<<<grid_for(p->npts, 128), 128, 0, p->stream>>>(u, p->blk, p->geo, p->npts, p->cs, t, p->scratch);
  CK(cudaGetLastError());
  unsigned long long h[2];
  CK(cudaMemcpyAsync(h, p->scratch, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  if (h[1] > 0)
    return fail(p, TGH_ERR_NONFINITE, "the state at t = " + std::to_string(t) + " is not finite where it is evolved: " +
                                          std::to_string(h[1]) + " values at evolved points are NaN or Inf");
  double lam;
  std::memcpy(&lam, &h[0], sizeof(lam));
  *lambda = lam;
  if (!(std::isfinite(lam) && lam > 0))
    return fail(p, TGH_ERR_SPEED, "the maximum characteristic speed over the evolved points came out as " +
                                      std::to_string(lam) + ": there is no CFL-limited time step");
  return TGH_OK;
}

int tgh_error_norm(tgh_problem* p, const double* u, double t, double* l2, double* linf) {
  int s = prepare_impl(p, u, t, "tgh_error_norm");
  if (s) return s;
  error_kernel<<<p->npart, 128, 0, p->stream>>>(p->work, p->blk, p->primary, p->geo, p->npts, p->cs, t, p->part);
  CK(cudaGetLastError());
  error_final_kernel<<<1, 32, 0, p->stream>>>(p->part, p->npart, p->part + 3 * (size_t)p->npart);
  CK(cudaGetLastError());
  double h[2];
  CK(cudaMemcpyAsync(h, p->part + 3 * (size_t)p->npart, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  *l2 = h[0];
  *linf = h[1];
  return TGH_OK;
}

// plain form: per stage one fill, one right-hand-side launch, one stage update
int tgh_rk4_step(tgh_problem* p, double* u, double t, double dt) {
  const size_t L = tgh_state_length(p);
  if (!p->k) CK(cudaMalloc(&p->k, L * sizeof(double)));
  if (!p->acc) {
    CK(cudaMalloc(&p->acc, L * sizeof(double)));
    CK(cudaMalloc(&p->y, L * sizeof(double)));
  }
  const double b16 = dt / 6.0, b13 = dt / 3.0, a12 = 0.5 * dt;
  const double tm = t + 0.5 * dt, te = t + dt;
  const unsigned g = 148 * 8;
  int s;
  if ((s = tgh_gh_rhs(p, p->k, u, t, nullptr))) return s;
  stage_update_kernel<<<g, 256, 0, p->stream>>>(0, (long)L, p->k, u, p->acc, p->y, nullptr, a12, b16);
  CK(cudaGetLastError());
  if ((s = stage_limit_impl(p, p->y, tm))) return s;
  if ((s = tgh_gh_rhs(p, p->k, p->y, tm, nullptr))) return s;
  stage_update_kernel<<<g, 256, 0, p->stream>>>(1, (long)L, p->k, u, p->acc, p->y, nullptr, a12, b13);
  CK(cudaGetLastError());
  if ((s = stage_limit_impl(p, p->y, tm))) return s;
  if ((s = tgh_gh_rhs(p, p->k, p->y, tm, nullptr))) return s;
  stage_update_kernel<<<g, 256, 0, p->stream>>>(1, (long)L, p->k, u, p->acc, p->y, nullptr, dt, b13);
  CK(cudaGetLastError());
  if ((s = stage_limit_impl(p, p->y, te))) return s;
  if ((s = tgh_gh_rhs(p, p->k, p->y, te, nullptr))) return s;
  stage_update_kernel<<<g, 256, 0, p->stream>>>(2, (long)L, p->k, nullptr, p->acc, nullptr, u, 0.0, b16);
  CK(cudaGetLastError());
  work_overwritten(p, "tgh_rk4_step (its last stage's fill)");
  return stage_limit_impl(p, u, te);
}

// The plain per-block form: the reference's block-wise map (map_blocks!, src/evolution.jl:1387)
// as host-issued launches, one right-hand side (head and Pi kernel) and one stage update per
// block and stage, after the same fill as the plain form. The baseline the batched form's
// fusion and graph are measured against; its arithmetic is the plain form's.
static int gh_rhs_blocks(tgh_problem* p, double* du, const double* u, double t) {
  int s = prepare_impl(p, u, t, "tgh_rk4_step_blocks");
  if (s) return s;
  for (int b = 0; b < p->nb; ++b) {
    RhsArgs a = base_args(p, p->work, t);
    a.du = du;
    a.p0 = (long)b * p->S;
    a.p1 = (long)(b + 1) * p->S;
    if ((s = launch_rhs(p, a, MODE_DU))) return s;
  }
  return TGH_OK;
}

static int stage_update_blocks(tgh_problem* p, int kind, const double* k, const double* u0, double* acc, double* y,
                               double* uout, double ca, double cb) {
  const long per = (long)NV * p->S;
  const unsigned g = (unsigned)grid_for(per, 256);
  for (int b = 0; b < p->nb; ++b) {
    const long o = per * b;
    stage_update_kernel<<<g, 256, 0, p->stream>>>(kind, per, k + o, u0 ? u0 + o : nullptr, acc + o,
                                                  y ? y + o : nullptr, uout ? uout + o : nullptr, ca, cb);
    CK(cudaGetLastError());
  }
  return TGH_OK;
}

int tgh_rk4_step_blocks(tgh_problem* p, double* u, double t, double dt) {
  if (p->nranks > 1) return fail(p, TGH_ERR_ARG, "the per-block form runs on a problem of one rank");
  const size_t L = tgh_state_length(p);
  if (!p->k) CK(cudaMalloc(&p->k, L * sizeof(double)));
  if (!p->acc) {
    CK(cudaMalloc(&p->acc, L * sizeof(double)));
    CK(cudaMalloc(&p->y, L * sizeof(double)));
  }
  const double b16 = dt / 6.0, b13 = dt / 3.0, a12 = 0.5 * dt;
  const double tm = t + 0.5 * dt, te = t + dt;
  int s;
  if ((s = gh_rhs_blocks(p, p->k, u, t))) return s;
  if ((s = stage_update_blocks(p, 0, p->k, u, p->acc, p->y, nullptr, a12, b16))) return s;
  if ((s = stage_limit_impl(p, p->y, tm))) return s;
  if ((s = gh_rhs_blocks(p, p->k, p->y, tm))) return s;
  if ((s = stage_update_blocks(p, 1, p->k, u, p->acc, p->y, nullptr, a12, b13))) return s;
  if ((s = stage_limit_impl(p, p->y, tm))) return s;
  if ((s = gh_rhs_blocks(p, p->k, p->y, tm))) return s;
  if ((s = stage_update_blocks(p, 1, p->k, u, p->acc, p->y, nullptr, dt, b13))) return s;
  if ((s = stage_limit_impl(p, p->y, te))) return s;
  if ((s = gh_rhs_blocks(p, p->k, p->y, te))) return s;
  if ((s = stage_update_blocks(p, 2, p->k, nullptr, p->acc, nullptr, u, 0.0, b16))) return s;
  p->last_launches = 4 * (fill_launches(p, false) + 3L * p->nb);
  return stage_limit_impl(p, u, te);
}

// batched form, one step's launches on the stream (captured into a graph by the caller)
// Stage st (0..3) of the batched form's RK4 step from t: the time it evaluates at, the working
// array it reads (filled first) and the one it writes, and its update coefficients.
struct StagePlan {
  double ts, ca, cb;
  double *rd, *wr;
};
static StagePlan stage_plan(tgh_problem* p, int st, double t, double dt) {
  const double b16 = dt / 6.0, b13 = dt / 3.0, a12 = 0.5 * dt;
  const double ts[4] = {t, t + 0.5 * dt, t + 0.5 * dt, t + dt};
  const double ca[4] = {a12, a12, dt, 0.0}, cb[4] = {b16, b13, b13, b16};
  double* rd[4] = {p->work, p->W1, p->W2, p->W1};
  double* wr[4] = {p->W1, p->W2, p->W1, p->work};
  return StagePlan{ts[st], ca[st], cb[st], rd[st], wr[st]};
}

static RhsArgs stage_args(tgh_problem* p, const StagePlan& sp, int st) {
  RhsArgs a = base_args(p, sp.rd, sp.ts);
  a.u0 = p->work;
  a.acc = p->bacc;
  a.next = sp.wr;
  a.ca = sp.ca;
  a.cb = sp.cb;
  a.stage = st + 1;
  return a;
}

static int stage_rhs(tgh_problem* p, const StagePlan& sp, int st) { return launch_rhs(p, stage_args(p, sp, st), MODE_STAGE); }

// One batched step: per stage the copies, then the interior kernel on a side branch beside the
// Dirichlet hook and the prolongation (it reads owned points only, which the copies have just
// made current and those two do not write), joined before the head and Pi kernels.
static int batched_step(tgh_problem* p, double t, double dt) {
  int s;
  const bool branch = p->intr && p->side;
  for (int st = 0; st < 4; ++st) {
    const StagePlan sp = stage_plan(p, st, t, dt);
    if (!branch) {
      if ((s = launch_fill(p, sp.rd, true, sp.rd, sp.ts))) return s;
      if ((s = stage_rhs(p, sp, st))) return s;
      continue;
    }
    if (p->ngpts) {
      fill_points_kernel<<<grid_for(p->ngpts, 256), 256, 0, p->stream>>>(p->gpts, p->ngpts, sp.rd, p->geo);
      CK(cudaGetLastError());
    }
    const RhsArgs a = stage_args(p, sp, st);
    CK(cudaEventRecord(p->ev_fork, p->stream));
    CK(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    if ((s = launch_interior(p, a, MODE_STAGE, p->side))) return s;
    CK(cudaEventRecord(p->ev_join, p->side));
    if ((s = launch_hooks(p, sp.rd, sp.ts))) return s;
    for (int l = 1; l <= p->maxlevel; ++l) {
      if (!p->nprol[l]) continue;
      CK(launch_prolong(p, l, sp.rd));
    }
    CK(cudaStreamWaitEvent(p->stream, p->ev_join, 0));
    p->interior_done = true;
    s = launch_rhs(p, a, MODE_STAGE);
    p->interior_done = false;
    if (s) return s;
  }
  return TGH_OK;
}

// One phase of the batched form's fill of `work` on this rank: phase 0 the copies and the
// Dirichlet hook, phase l >= 1 level l's prolongation. The halo values a phase reads must have
// been unpacked first.
static int launch_fill_phase(tgh_problem* p, double* work, int phase, double t) {
  const int T = 256;
  if (phase == 0) {
    if (p->ngpts) {
      fill_points_kernel<<<grid_for(p->ngpts, T), T, 0, p->stream>>>(p->gpts, p->ngpts, work, p->geo);
      CK(cudaGetLastError());
    }
    return launch_hooks(p, work, t);
  }
  const int l = phase;
  if (!p->nprol[l]) return TGH_OK;
  CK(launch_prolong(p, l, work));
  return TGH_OK;
}

static int batched_buffers(tgh_problem* p) {
  if (p->W1) return TGH_OK;
  const size_t Lw = work_doubles(p), L = tgh_state_length(p);
  CK(cudaMalloc(&p->W1, Lw * sizeof(double)));
  CK(cudaMalloc(&p->W2, Lw * sizeof(double)));
  CK(cudaMalloc(&p->bacc, L * sizeof(double)));
  CK(cudaMemsetAsync(p->W1, 0, Lw * sizeof(double), p->stream));
  CK(cudaMemsetAsync(p->W2, 0, Lw * sizeof(double), p->stream));
  return TGH_OK;
}

int tgh_step_batched(tgh_problem* p, double* u, double t, double dt, int nsteps) {
  if (nsteps < 1) return fail(p, TGH_ERR_ARG, "nsteps must be positive");
  if (p->cfg.interior == TGH_INT_PASTED)
    return fail(p, TGH_ERR_ARG, "the batched form has no :pasted limiter; use tgh_rk4_step");
  if (p->has_bounds) return fail(p, TGH_ERR_ARG, "the batched form has no range projection; use tgh_rk4_step");
  if (int st = fitted_ready(p)) return st;
  int s = batched_buffers(p);
  if (s) return s;
  // the state into W0's owned points (and ghosts), outside the graph
  work_overwritten(p, "tgh_step_batched");
  if ((s = launch_fill(p, u, false, p->work, t))) return s;
  // a stationary hook into the two stage buffers once, also outside the graph; the graph's
  // stage fills of those buffers then skip it
  if (p->hook_cache && p->hook_cache_valid && !p->hooks_held[0]) {
    if ((s = launch_hooks(p, p->W1, t)) || (s = launch_hooks(p, p->W2, t))) return s;
    p->hooks_held[0] = p->W1;
    p->hooks_held[1] = p->W2;
  }
  const bool reuse = p->gexec && p->gkey.t == t && p->gkey.dt == dt && p->gkey.nsteps == nsteps;
  if (!reuse) {
    if (p->gexec) {
      cudaGraphExecDestroy(p->gexec);
      p->gexec = nullptr;
    }
    // capture on the problem's own stream (the caller's may be the legacy default stream,
    // which cannot be captured); the graph is then launched on the caller's stream
    if (!p->cap) CK(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking));
    // the interior's block list for the whole span the graph steps over, built before capture,
    // and the side branch its kernel runs on
    if ((s = interior_blocks(p, p->ilist_graph, t, t + nsteps * dt))) return s;
    if (p->intr && !p->side) {
      CK(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
    }
    cudaGraph_t graph;
    cudaStream_t user = p->stream;
    p->stream = p->cap;
    p->ilist_use = &p->ilist_graph;
    cudaError_t eb = cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal);
    int st = TGH_OK;
    p->capturing = true;
    if (eb == cudaSuccess)
      for (int n = 0; n < nsteps && st == TGH_OK; ++n) st = batched_step(p, t + n * dt, dt);
    p->capturing = false;
    p->ilist_use = nullptr;
    cudaError_t ee = eb == cudaSuccess ? cudaStreamEndCapture(p->cap, &graph) : eb;
    p->stream = user;
    if (st) return st;
    CK(ee);
    size_t nn = 0;
    CK(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
    p->graph_kernels = 0;
    for (size_t i = 0; i < nn; ++i) {
      cudaGraphNodeType ty;
      CK(cudaGraphNodeGetType(nodes[i], &ty));
      if (ty == cudaGraphNodeTypeKernel) ++p->graph_kernels;
    }
    CK(cudaGraphInstantiate(&p->gexec, graph, 0));
    cudaGraphDestroy(graph);
    p->gkey = GraphKey{t, dt, nsteps};
  }
  CK(cudaGraphLaunch(p->gexec, p->stream));
  gather_kernel<<<grid_for(p->npts, 256), 256, 0, p->stream>>>(p->work, u, p->geo, p->npts);
  CK(cudaGetLastError());
  p->last_launches = fill_launches(p, false) + p->graph_kernels + 1;
  return TGH_OK;
}

// ---- the sharded batched step (one rank per GPU), driven by the caller ----
// tgh_shard_begin; per step, per stage st = 0..3: for phase = 0 .. tgh_shard_phases - 1:
// tgh_shard_pack -> the caller's exchange (peer-major buffers, counts from tgh_shard_counts) ->
// tgh_shard_unpack -> tgh_shard_fill; then tgh_shard_rhs; finally tgh_shard_end. Every call
// is stream-ordered on the problem's stream.

int tgh_partition(const tgh_mesh* m, int nranks, int* owner) {
  if (nranks < 1 || m->nblocks < 1 || m->N < 1) return TGH_ERR_ARG;
  // per level, the leaves in Morton order of their block coordinates, cut into nranks
  // contiguous runs of (nearly) equal length
  int maxl = 0;
  for (int b = 0; b < m->nblocks; ++b) maxl = std::max(maxl, m->level[b]);
  auto spread = [](uint64_t x) {
    x &= 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
  };
  for (int l = 0; l <= maxl; ++l) {
    std::vector<std::pair<uint64_t, int>> v;
    for (int b = 0; b < m->nblocks; ++b)
      if (m->level[b] == l) {
        const uint64_t bx = (uint64_t)(m->corner[3 * b] / m->N), by = (uint64_t)(m->corner[3 * b + 1] / m->N),
                       bz = (uint64_t)(m->corner[3 * b + 2] / m->N);
        v.push_back({spread(bx) | spread(by) << 1 | spread(bz) << 2, b});
      }
    std::sort(v.begin(), v.end());
    const size_t n = v.size();
    for (size_t i = 0; i < n; ++i) owner[v[i].second] = (int)((i * (size_t)nranks) / n);
  }
  return TGH_OK;
}

// Host-only view of `rank`'s exchange in fill phase `phase`, for tests and tooling: per peer
// rank the counts, and (when the arrays are given, 2 ints per point) the (global leaf, work
// index) pairs this rank sends and receives, peer-major. Touches no GPU.
int tgh_shard_plan(const tgh_config* cfg, const tgh_mesh* m, const int* owner, int rank, int nranks, int phase,
                   long* send_count, long* recv_count, int* send_pts, int* recv_pts, char* errbuf, int errlen) {
  tgh_problem p;
  int s = setup_host(&p, cfg, m, owner, rank, nranks, 0);
  std::string err = p.err;
  if (!s && (phase < 0 || phase > p.maxlevel)) {
    s = TGH_ERR_ARG;
    err = "no such fill phase";
  }
  HostPlan mine;
  if (!s && !plan_rank(&p, rank, false, mine, err)) s = TGH_ERR_ARG;
  long ns = 0, nr = 0;
  for (int o = 0; !s && o < nranks; ++o) {
    send_count[o] = recv_count[o] = 0;
    if (o == rank) continue;
    HostPlan theirs;
    if (!plan_rank(&p, o, false, theirs, err)) {
      s = TGH_ERR_ARG;
      break;
    }
    auto a = theirs.req.find({rank, phase});
    if (a != theirs.req.end()) {
      send_count[o] = (long)a->second.size();
      for (const auto& e : a->second)
        if (send_pts) {
          send_pts[2 * ns] = e.first;
          send_pts[2 * ns++ + 1] = dense_index(&p, e.second);
        }
    }
    auto b = mine.req.find({o, phase});
    if (b != mine.req.end()) {
      recv_count[o] = (long)b->second.size();
      for (const auto& e : b->second)
        if (recv_pts) {
          recv_pts[2 * nr] = e.first;
          recv_pts[2 * nr++ + 1] = dense_index(&p, e.second);
        }
    }
  }
  if (s && errbuf && errlen > 0) {
    std::strncpy(errbuf, err.c_str(), (size_t)errlen - 1);
    errbuf[errlen - 1] = 0;
  }
  return s;
}

int tgh_shard_phases(const tgh_problem* p) { return p->maxlevel + 1; }

int tgh_shard_counts(tgh_problem* p, int phase, long* send_count, long* recv_count) {
  if (phase < 0 || phase > p->maxlevel) return fail(p, TGH_ERR_ARG, "no such fill phase");
  for (int r = 0; r < p->nranks; ++r) {
    send_count[r] = p->xch[phase].send_count[r];
    recv_count[r] = p->xch[phase].recv_count[r];
  }
  return TGH_OK;
}

int tgh_shard_begin(tgh_problem* p, const double* u) {
  if (p->cfg.interior == TGH_INT_PASTED)
    return fail(p, TGH_ERR_ARG, "the batched form has no :pasted limiter; use tgh_rk4_step");
  if (p->has_bounds) return fail(p, TGH_ERR_ARG, "the batched form has no range projection; use tgh_rk4_step");
  if (int st = fitted_ready(p)) return st;
  int s = batched_buffers(p);
  if (s) return s;
  work_overwritten(p, "the sharded step");
  scatter_owned_kernel<<<grid_for(p->npts, 256), 256, 0, p->stream>>>(u, p->work, p->geo, p->npts);
  CK(cudaGetLastError());
  p->launches = 1;
  return TGH_OK;
}

static int shard_check(tgh_problem* p, int stage, int phase) {
  if (!p->W1) return fail(p, TGH_ERR_ARG, "tgh_shard_begin has not been called");
  if (stage < 0 || stage > 3) return fail(p, TGH_ERR_ARG, "the stage must lie in 0..3");
  if (phase < 0 || phase > p->maxlevel) return fail(p, TGH_ERR_ARG, "no such fill phase");
  return TGH_OK;
}

int tgh_shard_pack(tgh_problem* p, int stage, int phase, double* send) {
  int s = shard_check(p, stage, phase);
  if (s) return s;
  const ExchangeList& x = p->xch[phase];
  if (x.nsend) {
    pack_kernel<<<grid_for(x.nsend * NV, 256), 256, 0, p->stream>>>(x.send, x.nsend, stage_plan(p, stage, 0, 0).rd,
                                                                    p->geo, send);
    CK(cudaGetLastError());
    ++p->launches;
  }
  return TGH_OK;
}

int tgh_shard_unpack(tgh_problem* p, int stage, int phase, const double* recv) {
  int s = shard_check(p, stage, phase);
  if (s) return s;
  const ExchangeList& x = p->xch[phase];
  if (x.nrecv) {
    unpack_kernel<<<grid_for(x.nrecv * NV, 256), 256, 0, p->stream>>>(x.recv, x.nrecv, recv,
                                                                      stage_plan(p, stage, 0, 0).rd, p->geo);
    CK(cudaGetLastError());
    ++p->launches;
  }
  return TGH_OK;
}

int tgh_shard_fill(tgh_problem* p, int stage, int phase, double t, double dt) {
  int s = shard_check(p, stage, phase);
  if (s) return s;
  const StagePlan sp = stage_plan(p, stage, t, dt);
  p->launches += phase == 0 ? (p->ngpts ? 1 : 0) + (p->nhooks ? 1 : 0) : (p->nprol[phase] ? 1 : 0);
  return launch_fill_phase(p, sp.rd, phase, sp.ts);
}

int tgh_shard_rhs(tgh_problem* p, int stage, double t, double dt) {
  int s = shard_check(p, stage, 0);
  if (s) return s;
  p->launches += 2;
  return stage_rhs(p, stage_plan(p, stage, t, dt), stage);
}

int tgh_shard_end(tgh_problem* p, double* u) {
  if (!p->W1) return fail(p, TGH_ERR_ARG, "tgh_shard_begin has not been called");
  gather_kernel<<<grid_for(p->npts, 256), 256, 0, p->stream>>>(p->work, u, p->geo, p->npts);
  CK(cudaGetLastError());
  p->last_launches = p->launches + 1;
  return TGH_OK;
}

// Benchmark aid: the average duration of the right-hand-side kernel alone, timed with CUDA
// events on the problem's stream over nlaunch launches. mode 0: the plain form's kernel
// (du); mode 1: the batched form's kernel with the stage-2 epilogue. u is filled first.
int tgh_time_rhs(tgh_problem* p, const double* u, double t, int mode, int nlaunch, double* ms_per_launch) {
  const size_t L = tgh_state_length(p), Lw = work_doubles(p);
  if (mode == 0 && !p->k) CK(cudaMalloc(&p->k, L * sizeof(double)));
  if (mode == 1 && !p->W1) {
    CK(cudaMalloc(&p->W1, Lw * sizeof(double)));
    CK(cudaMalloc(&p->W2, Lw * sizeof(double)));
    CK(cudaMalloc(&p->bacc, L * sizeof(double)));
    CK(cudaMemsetAsync(p->bacc, 0, L * sizeof(double), p->stream));
  }
  // a rank of a sharded problem cannot fill from u alone: it is timed on its working array as
  // its last step left it (filled)
  int s = p->nranks > 1 ? TGH_OK : prepare_impl(p, u, t, "tgh_time_rhs");
  if (s) return s;
  RhsArgs a = base_args(p, p->work, t);
  a.du = p->k;
  a.u0 = p->work;
  a.acc = p->bacc;
  a.next = p->W1;
  a.ca = 1e-3;
  a.cb = 1e-3;
  a.stage = 2;
  if ((s = launch_rhs(p, a, mode == 1 ? MODE_STAGE : MODE_DU))) return s;  // warm
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, p->stream));
  for (int i = 0; i < nlaunch; ++i)
    if ((s = launch_rhs(p, a, mode == 1 ? MODE_STAGE : MODE_DU))) return s;
  CK(cudaEventRecord(e1, p->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_per_launch = ms / nlaunch;
  return TGH_OK;
}

// Benchmark aid: the average duration of a constraint monitor's kernel alone (which 0: the
// gauge constraint, 1: the ADM constraints; interior mask, no matter), timed with CUDA events on
// the problem's stream over nlaunch launches after one prepare of u at t.
int tgh_time_monitor(tgh_problem* p, const double* u, double t, int which, int nlaunch, double* ms_per_launch) {
  if (which != 0 && which != 1) return fail(p, TGH_ERR_ARG, "which must be 0 (gauge) or 1 (ADM)");
  if (nlaunch < 1) return fail(p, TGH_ERR_ARG, "nlaunch must be positive");
  MonArgs a;
  int s = monitor_prepare(p, u, t, TGH_MASK_INTERIOR, a);
  if (s) return s;
  auto launch = [&]() {
    return which == 0 ? launch_gauge_constraint(p->q, p->stream, p->cs, a)
                      : launch_adm_constraint(p->q, p->stream, p->cs, a);
  };
  CK(launch());  // warm
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, p->stream));
  for (int i = 0; i < nlaunch; ++i) CK(launch());
  CK(cudaEventRecord(e1, p->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_per_launch = ms / nlaunch;
  return TGH_OK;
}

// ---- the tangent-linear plain form: derivatives of the right-hand side, an RK4 step and the
// masked error along one direction (the state's tangent and, optionally, one parameter) ----

static int tangent_check(tgh_problem* p, int dir) {
  if (dir < TAN_STATE || dir > TAN_DAMP_NEAR) return fail(p, TGH_ERR_ARG, "unknown tangent direction");
  if (p->nranks > 1) return fail(p, TGH_ERR_ARG, "the tangent-linear form runs on one rank");
  if (p->mixed) return fail(p, TGH_ERR_ARG, "the tangent-linear form is FP64");
  if (p->intr && (core_follows(p->cs) || p->cfg.interior == TGH_INT_PASTED || p->cfg.interior == TGH_INT_FITTED))
    return fail(p, TGH_ERR_ARG, "the tangent-linear form takes a static :damped or :frozen interior");
  const size_t L = tgh_state_length(p), Lw = work_doubles(p);
  if (!p->twork) {
    CK(cudaMalloc(&p->twork, Lw * sizeof(double)));
    CK(cudaMemsetAsync(p->twork, 0, Lw * sizeof(double), p->stream));
  }
  if (!p->kt) {
    CK(cudaMalloc(&p->kt, L * sizeof(double)));
    CK(cudaMalloc(&p->acct, L * sizeof(double)));
    CK(cudaMalloc(&p->yt, L * sizeof(double)));
  }
  return TGH_OK;
}

// The same fill on the tangent working array: copies and prolongation are linear; the
// Dirichlet data depend neither on the parameters nor on the initial perturbation.
static int launch_fill_tangent(tgh_problem* p, const double* ut) {
  const int T = 256;
  if (p->nruns) {
    fill_copy_kernel<<<grid_for((long)p->nruns * 32, T), T, 0, p->stream>>>(p->runs, p->nruns, ut, p->twork, p->geo);
    CK(cudaGetLastError());
  }
  if (p->nhooks) {
    hook_zero_kernel<<<grid_for((long)p->nhooks * NV, T), T, 0, p->stream>>>(p->hooks, p->nhooks, p->twork, p->geo);
    CK(cudaGetLastError());
  }
  for (int l = 1; l <= p->maxlevel; ++l) {
    if (!p->nprol[l]) continue;
    CK(launch_prolong(p, l, p->twork));
  }
  return TGH_OK;
}

int tgh_tangent_rhs(tgh_problem* p, double* du, double* dut, const double* u, const double* ut, double t, int dir) {
  int s = tangent_check(p, dir);
  if (s) return s;
  if ((s = prepare_impl(p, u, t, "the tangent-linear form"))) return s;
  if ((s = launch_fill_tangent(p, ut))) return s;
  RhsArgs a = base_args(p, p->work, t);
  a.du = du;
  CK(launch_rhs_tangent(p->q, p->diss, p->intr, p->stream, p->cs, a, TanArgs{dut, dir}, (long)(p->twork - p->work)));
  return TGH_OK;
}

int tgh_tangent_rk4_step(tgh_problem* p, double* u, double* ut, double t, double dt, int dir) {
  int s = tangent_check(p, dir);
  if (s) return s;
  const size_t L = tgh_state_length(p);
  if (!p->k) CK(cudaMalloc(&p->k, L * sizeof(double)));
  if (!p->acc) {
    CK(cudaMalloc(&p->acc, L * sizeof(double)));
    CK(cudaMalloc(&p->y, L * sizeof(double)));
  }
  const double b16 = dt / 6.0, b13 = dt / 3.0, a12 = 0.5 * dt;
  const double ts[4] = {t, t + 0.5 * dt, t + 0.5 * dt, t + dt};
  const double ca[4] = {a12, a12, dt, 0.0}, cb[4] = {b16, b13, b13, b16};
  const unsigned g = 148 * 8;
  for (int st = 0; st < 4; ++st) {
    const double* x = st == 0 ? u : p->y;
    const double* xt = st == 0 ? ut : p->yt;
    if ((s = tgh_tangent_rhs(p, p->k, p->kt, x, xt, ts[st], dir))) return s;
    const int kind = st == 0 ? 0 : (st == 3 ? 2 : 1);
    stage_update_kernel<<<g, 256, 0, p->stream>>>(kind, (long)L, p->k, u, p->acc, p->y, u, ca[st], cb[st]);
    CK(cudaGetLastError());
    stage_update_kernel<<<g, 256, 0, p->stream>>>(kind, (long)L, p->kt, ut, p->acct, p->yt, ut, ca[st], cb[st]);
    CK(cudaGetLastError());
  }
  return TGH_OK;
}

int tgh_tangent_error_norm(tgh_problem* p, const double* u, const double* ut, double t, double* l2, double* dl2) {
  int s = tangent_check(p, TAN_STATE);
  if (s) return s;
  if ((s = prepare_impl(p, u, t, "the tangent-linear form"))) return s;
  if ((s = launch_fill_tangent(p, ut))) return s;
  error_tangent_kernel<<<p->npart, 128, 0, p->stream>>>(p->work, p->twork, p->blk, p->primary, p->geo, p->npts, p->cs,
                                                         t, p->part);
  CK(cudaGetLastError());
  std::vector<double> h(3 * (size_t)p->npart);
  CK(cudaMemcpyAsync(h.data(), p->part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  double a = 0.0, b = 0.0, w = 0.0;  // summed in block order, on the host
  for (int i = 0; i < p->npart; ++i) {
    a += h[3 * i];
    b += h[3 * i + 1];
    w += h[3 * i + 2];
  }
  if (!(w > 0.0)) return fail(p, TGH_ERR_ARG, "no evolved point to measure the error on");
  *l2 = std::sqrt(a / w);
  *dl2 = *l2 > 0.0 ? (b / w) / *l2 : 0.0;
  return TGH_OK;
}

// ---- the adjoint (reverse mode) of the plain form: the right-hand side, one RK4 step and the
// masked error, for gradients with respect to the whole initial state in one reverse sweep ----

static int adjoint_check(tgh_problem* p) {
  if (p->nranks > 1) return fail(p, TGH_ERR_ARG, "the adjoint form runs on one rank");
  if (p->mixed) return fail(p, TGH_ERR_ARG, "the adjoint form is FP64");
  if (p->intr && (core_follows(p->cs) || p->cfg.interior == TGH_INT_PASTED || p->cfg.interior == TGH_INT_FITTED))
    return fail(p, TGH_ERR_ARG, "the adjoint form takes a static :damped or :frozen interior");
  if (p->has_bounds) return fail(p, TGH_ERR_ARG, "the adjoint form does not differentiate the range projection");
  const size_t L = tgh_state_length(p);
  if (!p->adj_cot) {
    const size_t cs = (size_t)p->Wv * p->nb;
    CK(cudaMalloc(&p->adj_cot, (size_t)NC * ADJ_NF * cs * sizeof(double)));
    CK(cudaMemsetAsync(p->adj_cot, 0, (size_t)NC * ADJ_NF * cs * sizeof(double), p->stream));
    CK(cudaMalloc(&p->adj_mu, work_doubles(p) * sizeof(double)));
    CK(cudaMalloc(&p->adj_part, 3 * (size_t)p->npart * sizeof(double)));
    for (int i = 0; i < 3; ++i) CK(cudaMalloc(&p->adj_y[i], L * sizeof(double)));
    CK(cudaMalloc(&p->adj_a, L * sizeof(double)));
    CK(cudaMalloc(&p->adj_acc, L * sizeof(double)));
    CK(cudaMalloc(&p->adj_m, L * sizeof(double)));
  }
  if (!p->k) CK(cudaMalloc(&p->k, L * sizeof(double)));
  return TGH_OK;
}

// mu_u = (d gh_rhs!(y, t) / d y)^T a; th3 (host, nullable) += a . d gh_rhs! / d(rho_max, ramp, damping)
static int vjp_rhs(tgh_problem* p, const double* y, double t, const double* a, double* mu_u, double* th3) {
  int s = prepare_impl(p, y, t, "the adjoint form");
  if (s) return s;
  RhsArgs ra = base_args(p, p->work, t);
  const long cstride = (long)p->Wv * p->nb;
  AdjArgs J{a, p->adj_cot, cstride, p->adj_part};
  CK(launch_adjoint_point(p->q, p->diss, p->intr, p->stream, p->cs, ra, J));
  CK(launch_adjoint_gather(p->q, p->diss, p->stream, p->adj_cot, cstride, p->geo, p->nb, p->adj_mu));
  for (int l = p->maxlevel; l >= 1; --l) {
    if (!p->nprol[l]) continue;
    const unsigned g = grid_for((long)p->nprol[l] * NV, 256);
    switch (p->q + 2) {
      case 4: prolong_adjoint_kernel<4><<<g, 256, 0, p->stream>>>(p->prol[l], p->nprol[l], p->adj_mu, p->geo); break;
      case 6: prolong_adjoint_kernel<6><<<g, 256, 0, p->stream>>>(p->prol[l], p->nprol[l], p->adj_mu, p->geo); break;
      case 8: prolong_adjoint_kernel<8><<<g, 256, 0, p->stream>>>(p->prol[l], p->nprol[l], p->adj_mu, p->geo); break;
      default: prolong_adjoint_kernel<10><<<g, 256, 0, p->stream>>>(p->prol[l], p->nprol[l], p->adj_mu, p->geo); break;
    }
    CK(cudaGetLastError());
  }
  CK(cudaMemsetAsync(mu_u, 0, tgh_state_length(p) * sizeof(double), p->stream));
  if (p->nruns) {
    copy_adjoint_kernel<<<grid_for((long)p->nruns * 32, 256), 256, 0, p->stream>>>(p->runs, p->nruns, p->adj_mu, mu_u,
                                                                                    p->geo);
    CK(cudaGetLastError());
  }
  if (th3) {
    std::vector<double> h(3 * (size_t)p->npart);
    CK(cudaMemcpyAsync(h.data(), p->adj_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    for (int i = 0; i < p->npart; ++i)  // in block order, on the host
      for (int k = 0; k < 3; ++k) th3[k] += h[3 * i + k];
  }
  return TGH_OK;
}

int tgh_adjoint_rhs(tgh_problem* p, const double* u, double t, const double* lam_du, double* lam_u, double* th3) {
  int s = adjoint_check(p);
  if (s) return s;
  if (th3) th3[0] = th3[1] = th3[2] = 0.0;
  return vjp_rhs(p, u, t, lam_du, lam_u, th3);
}

int tgh_adjoint_rk4_step(tgh_problem* p, const double* u, double t, double dt, double* lam, double* th3) {
  int s = adjoint_check(p);
  if (s) return s;
  const long L = (long)tgh_state_length(p);
  const unsigned g = 148 * 8;
  const double a12 = 0.5 * dt, b16 = dt / 6.0, b13 = dt / 3.0;
  const double tm = t + 0.5 * dt, te = t + dt;
  double **y = p->adj_y, *a = p->adj_a, *acc = p->adj_acc, *m = p->adj_m;
  // the step's stage values, recomputed (the plain form's: y1 = u + dt/2 k1, y2 = u + dt/2 k2,
  // y3 = u + dt k3; the limiters do nothing on the problems the adjoint accepts)
  if ((s = tgh_gh_rhs(p, p->k, u, t, nullptr))) return s;
  axpby_kernel<<<g, 256, 0, p->stream>>>(L, 1.0, u, a12, p->k, y[0]);
  if ((s = tgh_gh_rhs(p, p->k, y[0], tm, nullptr))) return s;
  axpby_kernel<<<g, 256, 0, p->stream>>>(L, 1.0, u, a12, p->k, y[1]);
  if ((s = tgh_gh_rhs(p, p->k, y[1], tm, nullptr))) return s;
  axpby_kernel<<<g, 256, 0, p->stream>>>(L, 1.0, u, dt, p->k, y[2]);
  CK(cudaGetLastError());
  // backwards: u_{n+1} = u + dt/6 k1 + dt/3 k2 + dt/3 k3 + dt/6 k4, k_s = F(y_{s-1})
  CK(cudaMemcpyAsync(acc, lam, L * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  axpby_kernel<<<g, 256, 0, p->stream>>>(L, b16, lam, 0.0, lam, a);
  if ((s = vjp_rhs(p, y[2], te, a, m, th3))) return s;  // k4
  axpy_kernel<<<g, 256, 0, p->stream>>>(L, 1.0, m, acc);
  axpby_kernel<<<g, 256, 0, p->stream>>>(L, b13, lam, dt, m, a);
  if ((s = vjp_rhs(p, y[1], tm, a, m, th3))) return s;  // k3
  axpy_kernel<<<g, 256, 0, p->stream>>>(L, 1.0, m, acc);
  axpby_kernel<<<g, 256, 0, p->stream>>>(L, b13, lam, a12, m, a);
  if ((s = vjp_rhs(p, y[0], tm, a, m, th3))) return s;  // k2
  axpy_kernel<<<g, 256, 0, p->stream>>>(L, 1.0, m, acc);
  axpby_kernel<<<g, 256, 0, p->stream>>>(L, b16, lam, a12, m, a);
  if ((s = vjp_rhs(p, u, t, a, m, th3))) return s;  // k1
  axpy_kernel<<<g, 256, 0, p->stream>>>(L, 1.0, m, acc);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(lam, acc, L * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  return TGH_OK;
}

int tgh_adjoint_error_norm(tgh_problem* p, const double* u, double t, double* l2, double* lam) {
  int s = adjoint_check(p);
  if (s) return s;
  if ((s = prepare_impl(p, u, t, "the adjoint form"))) return s;
  error_kernel<<<p->npart, 128, 0, p->stream>>>(p->work, p->blk, p->primary, p->geo, p->npts, p->cs, t, p->part);
  CK(cudaGetLastError());
  std::vector<double> h(3 * (size_t)p->npart);
  CK(cudaMemcpyAsync(h.data(), p->part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  double a = 0.0, w = 0.0;
  for (int i = 0; i < p->npart; ++i) {
    a += h[3 * i];
    w += h[3 * i + 1];
  }
  if (!(w > 0.0)) return fail(p, TGH_ERR_ARG, "no evolved point to measure the error on");
  *l2 = std::sqrt(a / w);
  const double scale = *l2 > 0.0 ? 1.0 / (*l2 * w) : 0.0;
  error_adjoint_kernel<<<grid_for(p->npts, 128), 128, 0, p->stream>>>(u, p->blk, p->primary, p->geo, p->npts, p->cs,
                                                                       t, scale, lam);
  CK(cudaGetLastError());
  return TGH_OK;
}

// Benchmark aid: how many kernels the last tgh_step_batched call launched (the fill of u,
// the captured graph's kernel nodes, the gather).
int tgh_last_launch_count(tgh_problem* p, long* n) {
  *n = p->last_launches;
  return TGH_OK;
}

// Diagnostics: the sampled gauge source (device to device), and the analytic state and gauge
// source of the problem's case at one point evaluated by a one-thread device kernel.
int tgh_copy_hsrc(tgh_problem* p, double* dst) {
  if (!p->Hsrc) return fail(p, TGH_ERR_ARG, "this problem has no sampled gauge source");
  CK(cudaMemcpyAsync(dst, p->Hsrc, tgh_state_length(p) * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return TGH_OK;
}
int tgh_point_physics(tgh_problem* p, double t, const double* x_host, double* out40_host) {
  double* d;
  CK(cudaMalloc(&d, 43 * sizeof(double)));
  CK(cudaMemcpy(d, x_host, 3 * sizeof(double), cudaMemcpyHostToDevice));
  point_physics_kernel<<<1, 1, 0, p->stream>>>(p->cs, t, d, d + 3);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaMemcpy(out40_host, d + 3, 40 * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return TGH_OK;
}

// sustained FP64 FMA rate of this GPU (2 flop per FMA), for the roofline denominator
double tgh_fp64_probe(void* stream, int iters) {
  double* d;
  if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return -1;
  int dev, nsm;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t s = (cudaStream_t)stream;
  const int threads = 256, blocks = nsm * 8;
  fp64_probe_kernel<<<blocks, threads, 0, s>>>(d, 10, 1.0000001, 1e-9);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  fp64_probe_kernel<<<blocks, threads, 0, s>>>(d, iters, 1.0000001, 1e-9);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  return flops / (ms * 1e-3) / 1e12;
}

}  // extern "C"
