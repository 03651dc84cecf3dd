// api.cu -- the C ABI of include/imago_intg.h: system set-up on the host,
// device staging, and the four integral builds.
//
// Host set-up restates what setupSCF does before the integral calls:
//   setCutoffThresh            lattice.f90:239-308
//   initializeLattice          lattice.f90:310-444 (cutoff sphere)
//   getNumCells/makeLattice    lattice.f90:469-690, cellBorderCheck 698-782
//   getRecipCellVectors        lattice.f90:182-233
//   convertKPointsToXYZ        kpoints.f90:543-576
//   renormalizeBasis           basis.f90:55-243
// and builds the work lists that the reference's loop nests walk
// (integrals.F90:323-569): atom pairs i <= j with their nearest-image
// lattice vector, the lattice images within each pair's cutoff, and the
// screened alpha pairs of each image in the reference's staircase order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <utility>
#include <atomic>
#include <mutex>
#include <thread>
#include <array>
#include <cstdlib>
#include <string>
#include <map>
#include <numeric>
#include <vector>

#include "intg.cuh"
#include "lattice.cuh"

using namespace imago;

namespace {

// basis.f90:91-106
const double kAngNorm[16] = {
    0.2820947917738782, 0.4886025119029199, 0.4886025119029199,
    0.4886025119029199, 1.0925484305920790, 1.0925484305920790,
    1.0925484305920790, 0.5462742152960396, 0.3153915652525200,
    2.8906114426405543, 1.4453057213202771, 0.5900435899266435,
    0.5900435899266435, 0.3731763325901154, 0.4570457994644657,
    0.4570457994644657};

// Device scratch comes from one library-owned stream-ordered memory pool
// per device (cudaMallocFromPoolAsync / cudaFreeAsync on the context's
// stream).  Freed memory stays in the pool, so a context created after
// another reuses it without cudaMalloc/cudaFree and their device-wide
// synchronisation; imago_trim_memory hands it back to the driver.
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_lock;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};

cudaMemPool_t scratch_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxPoolDevices) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> guard(g_pool_lock);
  if (!g_pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[dev] = pool;
  }
  return g_pools[dev];
}

// An allocator whose resize leaves trivial elements uninitialised: the
// work arrays of a large cell (millions of shell pairs) are then first
// written, and their pages first touched, by the threads that fill them.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U> &) {}
  template <class U, class... A>
  void construct(U *q, A &&...a) {
    if constexpr (sizeof...(A) == 0)
      ::new ((void *)q) U;
    else
      ::new ((void *)q) U(std::forward<A>(a)...);
  }
};
template <class T>
using HostVec = std::vector<T, NoInitAlloc<T>>;

template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  int alloc(size_t count, cudaStream_t st) {
    if (count <= n && p) return IMAGO_OK;
    release(st);
    if (count == 0) return IMAGO_OK;
    cudaMemPool_t pool = scratch_pool();
    void *q = nullptr;
    if (!pool || cudaMallocFromPoolAsync(&q, count * sizeof(T), pool, st) !=
                     cudaSuccess) {
      cudaGetLastError();
      return IMAGO_ERR_NOMEM;
    }
    p = static_cast<T *>(q);
    n = count;
    return IMAGO_OK;
  }
  template <class Vec>
  int upload(const Vec &v, cudaStream_t st) {
    int rc = alloc(v.empty() ? 1 : v.size(), st);
    if (rc) return rc;
    if (!v.empty())
      IMAGO_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T),
                                 cudaMemcpyHostToDevice, st));
    return IMAGO_OK;
  }
  void release(cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    n = 0;
  }
};

struct HType {
  int element;
  int norb[4];
  int nalpha, ncore, nvale, nstates;
  std::vector<double> alphas;
  std::vector<int> cls, lm;
  std::vector<double> basis;  // [a * nstates + m]
};

struct HPType {
  int element;
  double z, nucalpha;
  std::vector<double> alphas;
  int first_site = -1, mult = 0, cumul = 0;
};

}  // namespace

// The library's device scratch pool for code outside this file.
cudaMemPool_t imago::device_scratch_pool() { return scratch_pool(); }

constexpr int kNumSchedules = 3;  // three-centre schedules, imago_intg_set_schedule

struct imago_ctx {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  int outputs_on_device = 0;
  size_t scratch_bytes = 0;

  // host description
  std::vector<HType> types;
  std::vector<HPType> ptypes;
  std::vector<int> type_screen, ptype_screen;
  int nt = 0, ns = 0, npt = 0, nps = 0, nk = 0, ncell = 0;
  int vale_dim = 0, core_dim = 0, pot_dim = 0;
  double T = 0.0;
  double rv[9], recip[9], inv[9];
  std::vector<double> site_pos, psite_pos, cells, csize, kxyz;
  std::vector<int> site_type, psite_ptype, cum_vale, cum_core;

  // work lists
  std::vector<DPair> pairs;
  HostVec<DUnit> units;
  HostVec<DSp> sps;
  HostVec<int> sp_by_cls;
  std::vector<int2> btile;
  // tensor-core phase-sum tiles for each tuned width, concatenated, and
  // where each width's list starts
  std::vector<int2> btile_w;
  int btile_off[kNumBlochWidths + 1] = {};
  bool bloch_tuned = false;
  float bloch_ms[kNumBlochWidths] = {};
  int cls_beg[17];
  // three-centre schedule: per-class launches (0), one persistent launch
  // fed by a work queue (1), or per-class launches with two EP terms of a
  // type per thread (2); mode -1 measures all on the first EP build
  int sched_mode = -1, sched = 0;
  bool sched_tuned = false;
  float sched_ms[kNumSchedules] = {};
  int queue_ctas = 0;
  // orthogonalisation of multi-term builds: per-(k, term) CTAs (0) or the
  // persistent TMA-fed kernel (1); mode -1 measures both on the first
  // EP build
  int ortho_mode = -1, ortho = 0;
  bool ortho_tuned = false;
  float ortho_ms[2] = {};
  // EP terms per contraction CTA (4 or 8), measured on the first EP build
  int contract_tpc = 4;
  bool contract_tuned = false;
  float contract_ms[2] = {};
  long long blk_total = 0, m_total = 0;
  std::vector<Term3c> ep_terms;

  // device copies
  DBuf<int> d_type_nalpha, d_type_alpha_off, d_type_nstates, d_type_nvale,
      d_type_state_off, d_type_basis_off, d_type_screen, d_alpha_cls,
      d_state_lm, d_site_type, d_site_cum_vale, d_site_cum_core,
      d_ptype_alpha_off, d_ptype_nalpha, d_ptype_first_site, d_ptype_mult,
      d_ptype_screen, d_psite_ptype, d_sp_by_cls;
  DBuf<double> d_alpha, d_basis, d_site_pos, d_ptype_z, d_ptype_nucalpha,
      d_palpha, d_psite_pos, d_cell, d_csize, d_kxyz;
  DBuf<double2> d_phase;
  DBuf<DPair> d_pairs;
  DBuf<DUnit> d_units;
  DBuf<DSp> d_sps;
  DBuf<Term3c> d_terms;
  DBuf<unsigned long long> d_queue;  // one work-queue counter per lane
  DBuf<int> d_flag;                  // DevSys::flag
  DBuf<int2> d_btile, d_btile_w;
  DBuf<SiteImage> d_simg;
  DBuf<float> d_cl_d1;
  DBuf<int> d_site_rank;

  // scratch
  // Each build kind (OL, KE, NP, EP) has its own scratch and stream (a
  // lane), forked from `stream` by every call, so that the kinds of one
  // call run concurrently; only their orthogonalisation waits for the
  // overlap's coreValeOL (event ev_scv).
  struct Scratch {
    DBuf<double> blk, M;
    DBuf<double2> vv, cv, cc, y;
  };
  Scratch scr[4];
  cudaStream_t kst[4] = {};
  cudaEvent_t kfork = nullptr, kjoin[4] = {}, ev_scv = nullptr;
  int lane = 0;
  bool ol_in_call = false;
  bool serial = false;   // all kinds on `stream`, one after another
  cudaStream_t cur() const { return !serial && kst[lane] ? kst[lane] : stream; }
  // host-output staging: one region per output matrix, so that each can be
  // copied out on copy_stream while the next build runs
  DBuf<double> out_stage;
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> cev;
  int cev_used = 0;
  DBuf<double2> s_cv;
  bool have_ol = false;
  // PSCF Hamiltonian: accumulated sh blocks per spin, the potential
  // coefficients, and the packed result when outputs go to the host
  DBuf<double> ham_blk, ham_w, ham_out;
  // 0 by system size and spin, 1 block sums, 2 fused, 3 fused one lane
  int ham_mode = 0;
  // momentum / dipole: the dipole centre of the current call and the three
  // packed matrices when outputs go to the host
  double dip_center[3] = {0.0, 0.0, 0.0};
  DBuf<double> vec_out;
  // CUDA-graph capture of the build: no timing events are recorded and EP
  // keeps the chunk size of the last eager build (scratch already sized)
  bool capturing = false;
  int ep_chunk = 0;
  cudaGraphExec_t gexec = nullptr;
  unsigned gwhich = 0;
  imago_out gout{};
  long long glaunches = 0;   // kernels in the captured graph

  DevSys sys;
  DevWork work;
  float stage_ms[4] = {0, 0, 0, 0};
  cudaEvent_t ev[8];
  bool events = false;
  // per-kernel-stage timing of the current build call: 5 events per
  // run_build (start, after prim, contract, bloch, ortho)
  std::vector<cudaEvent_t> kev;
  int kev_used = 0;
  long long launches = 0;
  double kernel_ms[4] = {0, 0, 0, 0};

  ~imago_ctx() {
    cudaStream_t st = stream;
    for (auto *b : {&d_type_nalpha, &d_type_alpha_off, &d_type_nstates,
                    &d_type_nvale, &d_type_state_off, &d_type_basis_off,
                    &d_type_screen, &d_alpha_cls, &d_state_lm, &d_site_type,
                    &d_site_cum_vale, &d_site_cum_core, &d_ptype_alpha_off,
                    &d_ptype_nalpha, &d_ptype_first_site, &d_ptype_mult,
                    &d_ptype_screen, &d_psite_ptype, &d_sp_by_cls})
      b->release(st);
    for (auto *b : {&d_alpha, &d_basis, &d_site_pos, &d_ptype_z,
                    &d_ptype_nucalpha, &d_palpha, &d_psite_pos, &d_cell,
                    &d_csize, &d_kxyz, &out_stage, &ham_blk, &ham_w, &ham_out, &vec_out})
      b->release(st);
    for (auto &sc : scr) {
      sc.blk.release(st);
      sc.M.release(st);
      for (auto *b : {&sc.vv, &sc.cv, &sc.cc, &sc.y}) b->release(st);
    }
    for (auto *b : {&d_phase, &s_cv}) b->release(st);
    d_pairs.release(st); d_units.release(st); d_sps.release(st);
    d_terms.release(st); d_btile.release(st); d_simg.release(st);
    d_btile_w.release(st);
    d_cl_d1.release(st);
    d_site_rank.release(st);
    d_queue.release(st);
    d_flag.release(st);
    if (st) cudaStreamSynchronize(st);
    if (events)
      for (auto &e : ev) cudaEventDestroy(e);
    for (auto &e : kev) cudaEventDestroy(e);
    for (auto &e : cev) cudaEventDestroy(e);
    if (gexec) cudaGraphExecDestroy(gexec);
    for (int k = 0; k < 4; ++k) {
      if (kst[k]) cudaStreamSynchronize(kst[k]);
      if (kst[k]) cudaStreamDestroy(kst[k]);
      if (kjoin[k]) cudaEventDestroy(kjoin[k]);
    }
    if (kfork) cudaEventDestroy(kfork);
    if (ev_scv) cudaEventDestroy(ev_scv);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

// Cells built together: each cell is a context of its own (own stream and
// scratch); the first build of a given output set runs the cells eagerly
// on their streams and captures the same launches, one fork/join branch
// per cell, into a graph that later builds replay on `stream`.
struct imago_batch {
  int device = 0;
  std::vector<imago_ctx *> cells;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  unsigned which = 0;
  std::vector<imago_out> outs;
  long long glaunches = 0;

  ~imago_batch() {
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (fork) cudaEventDestroy(fork);
    for (auto e : join)
      if (e) cudaEventDestroy(e);
    for (auto *c : cells) imago_intg_destroy(c);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

// ------------------------------------------------------------ lattice --
void recip_vectors(imago_ctx *c) {
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    double vol = 0.0;
    double r[3];
    for (int j = 0; j < 3; ++j) {
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      r[j] = c->rv[3 * i1 + j1] * c->rv[3 * i2 + j2] -
             c->rv[3 * i1 + j2] * c->rv[3 * i2 + j1];
      vol += r[j] * c->rv[3 * i + j];
    }
    for (int j = 0; j < 3; ++j) c->recip[3 * i + j] = 2.0 * kPi * r[j] / vol;
  }
  for (int i = 0; i < 9; ++i) c->inv[i] = c->recip[i] / (2.0 * kPi);
}

// Smallest singular value of realVectors: the square root of the smallest
// eigenvalue of the Gram matrix G = R R^T, by cyclic Jacobi rotations.
double smallest_singular(const double *rv) {
  double g[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      g[i][j] = 0.0;
      for (int x = 0; x < 3; ++x) g[i][j] += rv[3 * i + x] * rv[3 * j + x];
    }
  for (int sweep = 0; sweep < 50; ++sweep) {
    const double off = g[0][1] * g[0][1] + g[0][2] * g[0][2] + g[1][2] * g[1][2];
    const double dia = g[0][0] * g[0][0] + g[1][1] * g[1][1] + g[2][2] * g[2][2];
    if (off <= 1e-30 * dia) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (g[p][q] == 0.0) continue;
        const double th = 0.5 * std::atan2(2.0 * g[p][q], g[q][q] - g[p][p]);
        const double c = std::cos(th), sn = std::sin(th);
        for (int k = 0; k < 3; ++k) {  // G <- G J
          const double a = g[k][p], b = g[k][q];
          g[k][p] = c * a - sn * b;
          g[k][q] = sn * a + c * b;
        }
        for (int k = 0; k < 3; ++k) {  // G <- J^T G
          const double a = g[p][k], b = g[q][k];
          g[p][k] = c * a - sn * b;
          g[q][k] = sn * a + c * b;
        }
      }
  }
  const double lmin = std::min(g[0][0], std::min(g[1][1], g[2][2]));
  return std::sqrt(std::max(lmin, 0.0));
}

int make_cells(imago_ctx *c, double min_atom_alpha, double min_pot_alpha) {
  double lim = c->T * std::max(2.0 / min_atom_alpha,
                               1.0 / min_pot_alpha + 0.5 / min_atom_alpha);
  double maxsq = 0.0, len2[3];
  for (int i = 0; i < 3; ++i) {
    len2[i] = 0.0;
    for (int x = 0; x < 3; ++x) len2[i] += c->rv[3 * i + x] * c->rv[3 * i + x];
    maxsq = std::max(len2[i], maxsq);
  }
  lim = lim + 0.75 * maxsq + std::sqrt(3.0 * maxsq * lim);
  lim = std::max(lim, 2.0 * c->T / min_atom_alpha);
  lattice_points(c->rv, lim, c->cells, c->csize);
  c->ncell = (int)c->csize.size();
  return IMAGO_OK;
}

void nearest_lattice_host(const imago_ctx *c, const double *v, double *out) {
  double base[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    const double f = v[0] * c->inv[3 * i] + v[1] * c->inv[3 * i + 1] +
                     v[2] * c->inv[3 * i + 2];
    double r = (double)(long long)(std::fabs(f) + 0.5);
    if (f < 0.0) r = -r;
    for (int x = 0; x < 3; ++x) base[x] += c->rv[3 * i + x] * r;
  }
  double best[3] = {base[0], base[1], base[2]};
  double bd = 0.0;
  for (int x = 0; x < 3; ++x) bd += (v[x] - base[x]) * (v[x] - base[x]);
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        if (!i && !j && !k) continue;
        double cand[3], d = 0.0;
        for (int x = 0; x < 3; ++x) {
          cand[x] = base[x] + i * c->rv[x] + j * c->rv[3 + x] + k * c->rv[6 + x];
          d += (v[x] - cand[x]) * (v[x] - cand[x]);
        }
        if (d < bd * (1.0 - 1e-12)) {
          bd = d;
          std::memcpy(best, cand, sizeof best);
        }
      }
  std::memcpy(out, best, sizeof best);
}

// ------------------------------------------------------------ set-up --
int read_system(imago_ctx *c, const imago_system *s) {
  if (!s || s->num_atom_types <= 0 || s->num_atom_sites <= 0 ||
      s->num_pot_types <= 0 || s->num_pot_sites <= 0 || s->num_kpoints <= 0)
    return IMAGO_ERR_INVALID;
  if (!(s->basis_fn_convg > 0.0 && s->basis_fn_convg <= 1.0))
    return IMAGO_ERR_INVALID;
  c->nt = s->num_atom_types;
  c->ns = s->num_atom_sites;
  c->npt = s->num_pot_types;
  c->nps = s->num_pot_sites;
  c->nk = s->num_kpoints;
  std::memcpy(c->rv, s->real_vectors, sizeof c->rv);
  c->T = -std::log(s->basis_fn_convg);
  recip_vectors(c);
  double min_atom_alpha = 100.0, min_pot_alpha = 10000.0;
  int aoff = 0, foff = 0, coff = 0;
  c->types.resize(c->nt);
  for (int t = 0; t < c->nt; ++t) {
    HType &ty = c->types[t];
    ty.element = s->type_element[t] - 1;
    if (ty.element < 0) return IMAGO_ERR_INVALID;
    for (int l = 0; l < 4; ++l) ty.norb[l] = s->type_num_orb_alphas[4 * t + l];
    for (int l = 0; l < 3; ++l)
      if (ty.norb[l] < ty.norb[l + 1] || ty.norb[l + 1] < 0)
        return IMAGO_ERR_INVALID;
    ty.nalpha = ty.norb[0];
    if (ty.nalpha <= 0 || ty.nalpha > 32767) return IMAGO_ERR_INVALID;
    ty.alphas.assign(s->type_alphas + aoff, s->type_alphas + aoff + ty.nalpha);
    aoff += ty.nalpha;
    for (double a : ty.alphas)
      if (!(a > 0.0)) return IMAGO_ERR_INVALID;
    min_atom_alpha = std::min(min_atom_alpha, ty.alphas[0]);
    ty.cls.resize(ty.nalpha);
    for (int j = 0; j < ty.nalpha; ++j)
      ty.cls[j] = j < ty.norb[3] ? 3 : j < ty.norb[2] ? 2 : j < ty.norb[1] ? 1 : 0;
    const int ncf = s->type_num_core_fns[t], nvf = s->type_num_vale_fns[t];
    if (ncf < 0 || nvf < 0) return IMAGO_ERR_INVALID;
    const int *fl = s->fn_l + foff;
    std::vector<int> fco(ncf + nvf);
    ty.ncore = ty.nvale = 0;
    for (int f = 0; f < ncf + nvf; ++f) {
      if (fl[f] < 0 || fl[f] > 3 || ty.norb[fl[f]] <= 0) return IMAGO_ERR_INVALID;
      fco[f] = coff;
      coff += ty.norb[fl[f]];
      (f < ncf ? ty.ncore : ty.nvale) += 2 * fl[f] + 1;
    }
    ty.nstates = ty.ncore + ty.nvale;
    ty.lm.resize(ty.nstates);
    ty.basis.assign((size_t)ty.nalpha * ty.nstates, 0.0);
    // renormalizeBasis: valence functions first, then core; each l repeated
    // 2l+1 times with lm = l^2 + k and the angular norm folded in.
    int m = 0;
    for (int pass = 0; pass < 2; ++pass) {
      const int f0 = pass == 0 ? ncf : 0, f1 = pass == 0 ? ncf + nvf : ncf;
      for (int f = f0; f < f1; ++f) {
        const int l = fl[f], na = ty.norb[l];
        for (int k = 1; k <= 2 * l + 1; ++k) {
          ty.lm[m] = l * l + k - 1;
          for (int a = 0; a < na; ++a)
            ty.basis[(size_t)a * ty.nstates + m] =
                s->fn_coeffs[fco[f] + a] * kAngNorm[ty.lm[m]];
          ++m;
        }
      }
    }
    foff += ncf + nvf;
  }
  c->site_type.resize(c->ns);
  c->site_pos.assign(s->site_pos, s->site_pos + 3 * c->ns);
  c->cum_vale.resize(c->ns);
  c->cum_core.resize(c->ns);
  for (int i = 0; i < c->ns; ++i) {
    const int t = s->site_type[i] - 1;
    if (t < 0 || t >= c->nt) return IMAGO_ERR_INVALID;
    c->site_type[i] = t;
    c->cum_vale[i] = c->vale_dim;
    c->cum_core[i] = c->core_dim;
    c->vale_dim += c->types[t].nvale;
    c->core_dim += c->types[t].ncore;
  }
  c->ptypes.resize(c->npt);
  int poff = 0;
  for (int t = 0; t < c->npt; ++t) {
    HPType &p = c->ptypes[t];
    p.element = s->pot_type_element[t] - 1;
    if (p.element < 0) return IMAGO_ERR_INVALID;
    p.z = s->pot_type_nuc_charge[t];
    p.nucalpha = s->pot_type_nuc_alpha[t];
    const int n = s->pot_type_num_alphas[t];
    if (n <= 0 || !(p.nucalpha > 0.0)) return IMAGO_ERR_INVALID;
    p.alphas.assign(s->pot_type_alphas + poff, s->pot_type_alphas + poff + n);
    poff += n;
    p.cumul = c->pot_dim;
    c->pot_dim += n;
    min_pot_alpha = std::min(min_pot_alpha, p.alphas[0]);
  }
  c->psite_ptype.resize(c->nps);
  c->psite_pos.assign(s->pot_site_pos, s->pot_site_pos + 3 * c->nps);
  for (int i = 0; i < c->nps; ++i) {
    const int t = s->pot_site_type[i] - 1;
    if (t < 0 || t >= c->npt) return IMAGO_ERR_INVALID;
    if (i > 0 && t < c->psite_ptype[i - 1]) return IMAGO_ERR_INVALID;
    c->psite_ptype[i] = t;
    if (c->ptypes[t].first_site < 0) c->ptypes[t].first_site = i;
    c->ptypes[t].mult += 1;
  }
  // Screening tables are built per element from the first type (and first
  // potential type) of that element (gaussRelations.f90:85-100,158-173).
  c->type_screen.resize(c->nt);
  for (int t = 0; t < c->nt; ++t) {
    int f = t;
    for (int u = 0; u < t; ++u)
      if (c->types[u].element == c->types[t].element) { f = u; break; }
    c->type_screen[t] = f;
    if (c->types[f].nalpha < c->types[t].nalpha) return IMAGO_ERR_INVALID;
  }
  c->ptype_screen.resize(c->npt);
  for (int t = 0; t < c->npt; ++t) {
    int f = t;
    for (int u = 0; u < t; ++u)
      if (c->ptypes[u].element == c->ptypes[t].element) { f = u; break; }
    c->ptype_screen[t] = f;
    if (c->ptypes[f].alphas.size() < c->ptypes[t].alphas.size())
      return IMAGO_ERR_INVALID;
  }
  int rc = make_cells(c, min_atom_alpha, min_pot_alpha);
  if (rc) return rc;
  c->kxyz.resize(3 * c->nk);
  for (int k = 0; k < c->nk; ++k) {
    const double *f = s->kpoints_abc + 3 * k;
    for (int x = 0; x < 3; ++x)
      c->kxyz[3 * k + x] = f[0] * c->recip[x] + f[1] * c->recip[3 + x] +
                           f[2] * c->recip[6 + x];
  }
  return IMAGO_OK;
}

// The pair / image / alpha-pair screens of integrals.F90:323-569.
// Work lists of a contiguous range of atom pairs, with indices and offsets
// local to the range; build_work joins the ranges in order.
// Shell pairs sort by class and, within a class, by the pair's own part of
// the three-centre screening radius^2 in four buckets (kSortKeys keys).
constexpr int kSortKeys = 16 * 4;

struct PairWork {
  std::vector<DPair> pairs;
  std::vector<DUnit> units;
  std::vector<DSp> sps;
  std::vector<unsigned char> key;  // sort key of each shell pair
  int hist[kSortKeys] = {};
  long long moff = 0, boff = 0;
  int rc = IMAGO_OK;
};

void build_pairs(const imago_ctx *c, const std::vector<int2> &ij, size_t lo,
                 size_t hi, PairWork &w) {
  for (size_t q = lo; q < hi && w.rc == IMAGO_OK; ++q) {
    const int i = ij[q].x, j = ij[q].y;
    DPair p{};
    p.i = i;
    p.j = j;
    p.ti = c->site_type[i];
    p.tj = c->site_type[j];
    const HType &t1 = c->types[p.ti], &t2 = c->types[p.tj];
    const HType &s1 = c->types[c->type_screen[p.ti]];
    const HType &s2 = c->types[c->type_screen[p.tj]];
    p.ni = t1.nstates;
    p.nj = t2.nstates;
    const double *A = &c->site_pos[3 * i], *B = &c->site_pos[3 * j];
    double dv[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    nearest_lattice_host(c, dv, p.L0);
    double r02 = 0.0;
    for (int x = 0; x < 3; ++x)
      r02 += (A[x] - B[x] - p.L0[x]) * (A[x] - B[x] - p.L0[x]);
    auto adist = [&](int a, int b) {
      const double x1 = s1.alphas[a], x2 = s2.alphas[b];
      return c->T / x2 / (x1 / (x1 + x2));
    };
    const double lim = adist(0, 0);
    p.ubeg = (int)w.units.size();
    p.moff = w.moff;
    if (r02 <= lim) {
      const double maxr = r02 + lim + 2.0 * std::sqrt(r02 * lim);
      if (maxr > c->csize[c->ncell - 1]) {
        w.rc = IMAGO_ERR_CELL_LIST;
        return;
      }
      for (int k = 0; k < c->ncell; ++k) {
        if (c->csize[k] > maxr) break;
        double r2 = 0.0;
        for (int x = 0; x < 3; ++x) {
          const double bp = B[x] + p.L0[x] + c->cells[3 * k + x];
          r2 += (A[x] - bp) * (A[x] - bp);
        }
        if (r2 > lim) continue;
        DUnit u{};
        u.pair = (int)w.pairs.size();
        u.cell = k;
        u.r2 = r2;
        u.spbeg = (int)w.sps.size();
        const int nmin = std::min(t1.nalpha, t2.nalpha);
        for (int l = 0; l < nmin; ++l) {
          int mode = 0, a = l, b = l;
          if (adist(l, l) < r2) break;
          for (;;) {
            if (mode == 1) {
              ++a;
              if (a >= t1.nalpha) { mode = 2; a = l; continue; }
            } else if (mode == 2) {
              ++b;
              if (b >= t2.nalpha) break;
            }
            if (adist(a, b) < r2) {
              if (mode == 1) { mode = 2; a = l; continue; }
              break;
            }
            if (mode == 0) mode = 1;
            DSp sp{};
            sp.unit = (int)w.units.size();
            sp.a = (short)a;
            sp.b = (short)b;
            sp.la = (short)t1.cls[a];
            sp.lb = (short)t2.cls[b];
            sp.boff = w.boff;
            w.boff += nsh(sp.la) * nsh(sp.lb);
            w.sps.push_back(sp);
            // the pair's own part of the three-centre screening radius^2,
            // frac T / (a1 + a2) (gaussRelations alphaNucDist/alphaPotDist
            // without the third exponent)
            const double reach =
                (1.0 - r2 / adist(a, b)) * c->T / (s1.alphas[a] + s2.alphas[b]);
            const int bucket = reach > 64.0 ? 0 : reach > 16.0 ? 1 : reach > 4.0 ? 2 : 3;
            const int key = (sp.la * 4 + sp.lb) * 4 + bucket;
            w.key.push_back((unsigned char)key);
            ++w.hist[key];
          }
        }
        u.spend = (int)w.sps.size();
        w.units.push_back(u);
      }
    }
    p.uend = (int)w.units.size();
    w.moff += (long long)(p.uend - p.ubeg) * p.ni * p.nj;
    w.pairs.push_back(p);
  }
}

// Runs f(lo, hi) over [0, n) in chunks on up to hardware_concurrency
// threads (one thread for small n).
template <class F>
void parallel_ranges(size_t n, size_t nchunk, F f) {
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (n < 512 || hw == 1) {
    for (size_t c = 0; c < nchunk; ++c) f(c, n * c / nchunk, n * (c + 1) / nchunk);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> th;
  for (unsigned t = 0; t < hw; ++t)
    th.emplace_back([&] {
      for (size_t c; (c = next.fetch_add(1)) < nchunk;)
        f(c, n * c / nchunk, n * (c + 1) / nchunk);
    });
  for (auto &x : th) x.join();
}

int build_work(imago_ctx *c) {
  c->pairs.clear();
  c->units.clear();
  c->sps.clear();
  // atom pairs i <= j, i-major as the reference loops them
  std::vector<int2> ij;
  ij.reserve((size_t)c->ns * (c->ns + 1) / 2);
  for (int i = 0; i < c->ns; ++i)
    for (int j = i; j < c->ns; ++j) ij.push_back(make_int2(i, j));
  const size_t nchunk = std::max<size_t>(1, std::min<size_t>(256, ij.size() / 8));
  std::vector<PairWork> part(nchunk);
  parallel_ranges(ij.size(), nchunk, [&](size_t k, size_t lo, size_t hi) {
    build_pairs(c, ij, lo, hi, part[k]);
  });
  // offsets of each part in the merged arrays, then the parts copied (and
  // their shell pairs' sort positions scattered) in parallel
  const size_t nparts = part.size();
  std::vector<size_t> pb(nparts + 1, 0), ub(nparts + 1, 0), sb(nparts + 1, 0);
  std::vector<long long> mb(nparts + 1, 0), bb(nparts + 1, 0);
  for (size_t k = 0; k < nparts; ++k) {
    const PairWork &w = part[k];
    if (w.rc) return w.rc;
    pb[k + 1] = pb[k] + w.pairs.size();
    ub[k + 1] = ub[k] + w.units.size();
    sb[k + 1] = sb[k] + w.sps.size();
    mb[k + 1] = mb[k] + w.moff;
    bb[k + 1] = bb[k] + w.boff;
  }
  c->pairs.resize(pb[nparts]);
  c->units.resize(ub[nparts]);
  c->sps.resize(sb[nparts]);
  c->blk_total = bb[nparts];
  c->m_total = mb[nparts];
  // Shell pairs by class and, within a class, by reach bucket (above 64,
  // 16, 4 bohr^2 and below), stable in unit order: a warp then holds shell
  // pairs of similar reach, whose site screens agree.  The order only maps
  // threads to shell pairs.  A stable counting sort, each part scattering
  // its own shell pairs from its offsets per key.
  std::vector<long long> start(kSortKeys + 1, 0);
  for (size_t k = 0; k < nparts; ++k)
    for (int q = 0; q < kSortKeys; ++q) start[q + 1] += part[k].hist[q];
  for (int q = 0; q < kSortKeys; ++q) start[q + 1] += start[q];
  std::vector<long long> off((size_t)nparts * kSortKeys);
  {
    std::vector<long long> run(start.begin(), start.end() - 1);
    for (size_t k = 0; k < nparts; ++k)
      for (int q = 0; q < kSortKeys; ++q) {
        off[k * kSortKeys + q] = run[q];
        run[q] += part[k].hist[q];
      }
  }
  c->sp_by_cls.resize(sb[nparts]);
  parallel_ranges(sb[nparts], nparts, [&](size_t k, size_t, size_t) {
    const PairWork &w = part[k];
    for (size_t q = 0; q < w.pairs.size(); ++q) {
      DPair p = w.pairs[q];
      p.ubeg += (int)ub[k];
      p.uend += (int)ub[k];
      p.moff += mb[k];
      c->pairs[pb[k] + q] = p;
    }
    for (size_t q = 0; q < w.units.size(); ++q) {
      DUnit u = w.units[q];
      u.pair += (int)pb[k];
      u.spbeg += (int)sb[k];
      u.spend += (int)sb[k];
      c->units[ub[k] + q] = u;
    }
    long long *o = &off[k * kSortKeys];
    for (size_t q = 0; q < w.sps.size(); ++q) {
      DSp sp = w.sps[q];
      sp.unit += (int)ub[k];
      sp.boff += bb[k];
      c->sps[sb[k] + q] = sp;
      c->sp_by_cls[o[w.key[q]]++] = (int)(sb[k] + q);
    }
  });
  for (int k = 0; k <= 16; ++k) c->cls_beg[k] = (int)start[4 * k];
  // phase-sum tiles: every pair (also those with no image, whose blocks
  // are written as zeros) in column tiles of kBlochCols block elements
  c->btile.clear();
  for (int p = 0; p < (int)c->pairs.size(); ++p) {
    const int ne = c->pairs[p].ni * c->pairs[p].nj;
    for (int t = 0; t * kBlochCols < ne; ++t) c->btile.push_back(make_int2(p, t));
  }
  c->btile_w.clear();
  for (int wi = 0; wi < kNumBlochWidths; ++wi) {
    c->btile_off[wi] = (int)c->btile_w.size();
    const int bw = bloch_width(wi);
    for (int p = 0; p < (int)c->pairs.size(); ++p) {
      const int ne = c->pairs[p].ni * c->pairs[p].nj;
      for (int t = 0; t * bw < ne; ++t) c->btile_w.push_back(make_int2(p, t));
    }
  }
  c->btile_off[kNumBlochWidths] = (int)c->btile_w.size();
  // EP terms in the reference's order (cumulAlphaSum + alpha index)
  c->ep_terms.clear();
  for (int t = 0; t < c->npt; ++t)
    for (int j = 0; j < (int)c->ptypes[t].alphas.size(); ++j)
      c->ep_terms.push_back({0, t, j});
  return IMAGO_OK;
}

constexpr size_t kMaxSiteImageBytes = size_t(4) << 30;

void set_bloch_width(imago_ctx *c, int wi) {
  c->work.bw = bloch_width(wi);
  c->work.btile_w = c->d_btile_w.p + c->btile_off[wi];
  c->work.nbtile_w = c->btile_off[wi + 1] - c->btile_off[wi];
}

int upload(imago_ctx *c) {
  cudaStream_t st = c->stream;
  std::vector<int> nalpha, aoff, nstates, nvale, soff, boff, cls, lm;
  std::vector<double> alpha, basis;
  for (const HType &t : c->types) {
    nalpha.push_back(t.nalpha);
    aoff.push_back((int)alpha.size());
    nstates.push_back(t.nstates);
    nvale.push_back(t.nvale);
    soff.push_back((int)lm.size());
    boff.push_back((int)basis.size());
    alpha.insert(alpha.end(), t.alphas.begin(), t.alphas.end());
    cls.insert(cls.end(), t.cls.begin(), t.cls.end());
    lm.insert(lm.end(), t.lm.begin(), t.lm.end());
    basis.insert(basis.end(), t.basis.begin(), t.basis.end());
  }
  std::vector<int> paoff, pn, pfirst, pmult;
  std::vector<double> pz, pnuc, palpha;
  for (const HPType &p : c->ptypes) {
    paoff.push_back((int)palpha.size());
    pn.push_back((int)p.alphas.size());
    pfirst.push_back(p.first_site < 0 ? 0 : p.first_site);
    pmult.push_back(p.mult);
    pz.push_back(p.z);
    pnuc.push_back(p.nucalpha);
    palpha.insert(palpha.end(), p.alphas.begin(), p.alphas.end());
  }
  int rc = 0;
#define UP(buf, vec) \
  if ((rc = c->buf.upload(vec, st))) return rc;
  UP(d_type_nalpha, nalpha) UP(d_type_alpha_off, aoff) UP(d_type_nstates, nstates)
  UP(d_type_nvale, nvale) UP(d_type_state_off, soff) UP(d_type_basis_off, boff)
  UP(d_type_screen, c->type_screen) UP(d_alpha_cls, cls) UP(d_state_lm, lm)
  UP(d_alpha, alpha) UP(d_basis, basis) UP(d_site_pos, c->site_pos)
  UP(d_site_type, c->site_type) UP(d_site_cum_vale, c->cum_vale)
  UP(d_site_cum_core, c->cum_core) UP(d_ptype_z, pz) UP(d_ptype_nucalpha, pnuc)
  UP(d_palpha, palpha) UP(d_ptype_alpha_off, paoff) UP(d_ptype_nalpha, pn)
  UP(d_ptype_first_site, pfirst) UP(d_ptype_mult, pmult)
  UP(d_ptype_screen, c->ptype_screen) UP(d_psite_pos, c->psite_pos)
  UP(d_psite_ptype, c->psite_ptype) UP(d_cell, c->cells) UP(d_csize, c->csize)
  UP(d_kxyz, c->kxyz) UP(d_pairs, c->pairs) UP(d_units, c->units)
  UP(d_sps, c->sps) UP(d_sp_by_cls, c->sp_by_cls) UP(d_terms, c->ep_terms)
  UP(d_btile, c->btile) UP(d_btile_w, c->btile_w)
#undef UP
  if ((rc = c->d_queue.alloc(4, st))) return rc;
  if ((rc = c->d_flag.alloc(1, st))) return rc;
  IMAGO_CUDA(cudaMemsetAsync(c->d_flag.p, 0, sizeof(int), st));
  {
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) {
      cudaGetLastError();
      nsm = 148;
    }
    c->queue_ctas = nsm * prim3c_queue_ctas_per_sm();
  }
  if ((rc = c->d_phase.alloc((size_t)c->ncell * c->nk, st))) return rc;

  DevSys &s = c->sys;
  s.nt = c->nt; s.ns = c->ns; s.npt = c->npt; s.nps = c->nps; s.nk = c->nk;
  s.ncell = c->ncell; s.vale_dim = c->vale_dim; s.core_dim = c->core_dim;
  s.T = c->T;
  std::memcpy(s.rv, c->rv, sizeof s.rv);
  std::memcpy(s.inv, c->inv, sizeof s.inv);
  s.far_lattice = 1.5 * smallest_singular(c->rv) * (1.0 - 1e-6);
  s.real_k = 1;
  for (double x : c->kxyz) s.real_k &= x == 0.0;
  s.minus_i = 0;
  s.type_nalpha = c->d_type_nalpha.p; s.type_alpha_off = c->d_type_alpha_off.p;
  s.type_nstates = c->d_type_nstates.p; s.type_nvale = c->d_type_nvale.p;
  s.type_state_off = c->d_type_state_off.p; s.type_basis_off = c->d_type_basis_off.p;
  s.type_screen = c->d_type_screen.p; s.alpha = c->d_alpha.p;
  s.alpha_cls = c->d_alpha_cls.p; s.state_lm = c->d_state_lm.p; s.basis = c->d_basis.p;
  s.site_pos = c->d_site_pos.p; s.site_type = c->d_site_type.p;
  s.site_cum_vale = c->d_site_cum_vale.p; s.site_cum_core = c->d_site_cum_core.p;
  s.ptype_z = c->d_ptype_z.p; s.ptype_nucalpha = c->d_ptype_nucalpha.p;
  s.palpha = c->d_palpha.p; s.ptype_alpha_off = c->d_ptype_alpha_off.p;
  s.ptype_nalpha = c->d_ptype_nalpha.p; s.ptype_first_site = c->d_ptype_first_site.p;
  s.ptype_mult = c->d_ptype_mult.p; s.ptype_screen = c->d_ptype_screen.p;
  s.psite_pos = c->d_psite_pos.p; s.psite_ptype = c->d_psite_ptype.p;
  s.cell = c->d_cell.p; s.csize = c->d_csize.p; s.kxyz = c->d_kxyz.p;
  s.phase = c->d_phase.p;
  s.flag = c->d_flag.p;
  DevWork &w = c->work;
  w.npairs = (int)c->pairs.size();
  w.nunits = (int)c->units.size();
  w.nsp = (int)c->sps.size();
  w.pairs = c->d_pairs.p; w.units = c->d_units.p; w.sps = c->d_sps.p;
  w.sp_by_cls = c->d_sp_by_cls.p;
  w.blk_total = c->blk_total;
  w.m_total = c->m_total;
  w.nbtile = (int)c->btile.size();
  w.btile = c->d_btile.p;
  set_bloch_width(c, kNumBlochWidths - 1);
  w.simg = nullptr;
  w.cl_d1 = nullptr;
  w.site_rank = nullptr;
  w.ncl = (c->nps + kSiteCluster - 1) / kSiteCluster;
  if ((rc = launch_phase(s, c->d_phase.p, st))) return rc;
  // midpoint images of the potential sites, their cluster bounds and each
  // unit's sites by distance, for the three-centre screens, when the
  // tables fit in kMaxSiteImageBytes; without them every site is searched
  // in full
  const size_t nb = (size_t)w.nunits * c->nps;
  if (nb > 0 && nb * (sizeof(SiteImage) + sizeof(int)) <= kMaxSiteImageBytes &&
      c->d_simg.alloc(nb, st) == IMAGO_OK &&
      c->d_cl_d1.alloc((size_t)w.nunits * w.ncl, st) == IMAGO_OK &&
      c->d_site_rank.alloc(nb, st) == IMAGO_OK) {
    w.simg = c->d_simg.p;
    w.cl_d1 = c->d_cl_d1.p;
    w.site_rank = c->d_site_rank.p;
    rc = launch_site_images(s, w, c->d_simg.p, c->d_cl_d1.p, st);
  }
  return rc;
}

// Device bytes one term of a build needs between its stages.
size_t term_bytes(const imago_ctx *c) {
  const size_t V = c->vale_dim, C = c->core_dim, nk = c->nk;
  return sizeof(double) * (size_t)(c->blk_total + c->m_total) +
         sizeof(double2) * nk * (V * V + 2 * V * C + C * C) +
         sizeof(double2) * nk * (V * (V + 1) / 2);
}

int ensure_scratch(imago_ctx *c, int nterm) {
  const size_t V = c->vale_dim, C = c->core_dim, nk = c->nk;
  imago_ctx::Scratch &S = c->scr[c->lane];
  cudaStream_t st = c->cur();
  const size_t nblk = (size_t)c->blk_total * nterm + 1, nm = (size_t)c->m_total * nterm + 1;
  const size_t nvv = nk * V * V * nterm + 1, ncv = nk * V * C * nterm + 1;
  const size_t ncc = nk * C * C * nterm + 1;
  // A captured build graph holds these buffers' addresses: a build that
  // needs more (more terms per pass, as the three- and six-term builds
  // do) drops the graph before the old buffers are freed, and the next
  // imago_intg_build_graph call captures anew.
  auto grows = [](const auto &b, size_t n) { return !b.p || n > b.n; };
  if (c->gexec && (grows(S.blk, nblk) || grows(S.M, nm) || grows(S.vv, nvv) ||
                   grows(S.cv, ncv) || grows(S.cc, ncc) || grows(S.y, ncv))) {
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  int rc;
  if ((rc = S.blk.alloc(nblk, st))) return rc;
  if ((rc = S.M.alloc(nm, st))) return rc;
  if ((rc = S.vv.alloc(nvv, st))) return rc;
  if ((rc = S.cv.alloc(ncv, st))) return rc;
  if ((rc = S.cc.alloc(ncc, st))) return rc;
  if ((rc = S.y.alloc(ncv, st))) return rc;
  return IMAGO_OK;
}

enum Kind {
  KIND_OL = 0, KIND_KE = 1, KIND_NP = 2, KIND_EP = 3, KIND_MV = 4,
  KIND_MM = 5, KIND_DM = 6  // three components each
};

// One build of `nterm` matrices of one kind, writing packed output to
// `packed_dev` (device) [nterm][nk][np][2].
cudaEvent_t next_event(imago_ctx *c) {
  if (c->kev_used == (int)c->kev.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    c->kev.push_back(e);
  }
  return c->kev[c->kev_used++];
}

void mark(imago_ctx *c) {
  if (c->capturing) return;
  cudaEvent_t e = next_event(c);
  if (e) cudaEventRecord(e, c->cur());
}

int class_launches(const imago_ctx *c) {
  int n = 0;
  for (int k = 0; k < 16; ++k) n += c->cls_beg[k + 1] > c->cls_beg[k];
  return n;
}

// The tensor-core phase sum's column-tile width is picked by measurement:
// on the context's first phase sum each width runs once on the real blocks
// (every run writes the same values) and the fastest is kept.  Narrower
// tiles waste less on block widths that are not multiples of 64, wider
// ones reuse each phase fragment more.
int tune_bloch(imago_ctx *c, int nterm) {
  cudaEvent_t e[kNumBlochWidths + 1];
  for (auto &x : e)
    if (cudaEventCreate(&x) != cudaSuccess) {
      cudaGetLastError();
      return IMAGO_ERR_CUDA;
    }
  int rc = IMAGO_OK;
  imago_ctx::Scratch &S = c->scr[c->lane];
  cudaStream_t st = c->cur();
  cudaEventRecord(e[0], st);
  for (int wi = 0; wi < kNumBlochWidths && !rc; ++wi) {
    set_bloch_width(c, wi);
    rc = launch_bloch(c->sys, c->work, nterm, S.M.p, S.vv.p, S.cv.p, S.cc.p, st);
    cudaEventRecord(e[wi + 1], st);
  }
  if (!rc && cudaEventSynchronize(e[kNumBlochWidths]) != cudaSuccess) rc = IMAGO_ERR_CUDA;
  int best = kNumBlochWidths - 1;
  for (int wi = 0; wi < kNumBlochWidths && !rc; ++wi)
    cudaEventElapsedTime(&c->bloch_ms[wi], e[wi], e[wi + 1]);
  for (int wi = 0; wi < kNumBlochWidths && !rc; ++wi)
    if (c->bloch_ms[wi] < c->bloch_ms[best]) best = wi;
  for (auto &x : e) cudaEventDestroy(x);
  cudaGetLastError();
  set_bloch_width(c, best);
  c->launches += kNumBlochWidths;
  c->bloch_tuned = !rc;
  return rc;
}

// Measured choices of the autotuned stages (phase-sum width, three-centre
// schedule, orthogonalisation schedule), kept for the process per device
// and workload shape, so that a later context of the same system (a
// rebuilt SCF set-up, an end-to-end call) starts tuned instead of timing
// the alternatives again.
struct TuneRecord {
  int bloch = -1, sched = -1, ortho = -1, contract = -1;
  float bloch_ms[kNumBlochWidths] = {}, sched_ms[kNumSchedules] = {}, ortho_ms[2] = {},
        contract_ms[2] = {};
};
using TuneKey = std::array<long long, 10>;
std::mutex g_tune_mu;
std::map<TuneKey, TuneRecord> g_tune;

TuneKey tune_key(const imago_ctx *c) {
  return {c->device,       c->vale_dim,          c->core_dim,        c->nk,
          c->pot_dim,      (long long)c->units.size(), (long long)c->sps.size(),
          c->ncell,        c->nps,               c->sys.real_k};
}

void tune_store(const imago_ctx *c) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  TuneRecord &r = g_tune[tune_key(c)];
  if (c->bloch_tuned) {
    r.bloch = (c->work.bw - bloch_width(0)) / (bloch_width(1) - bloch_width(0));
    std::copy(c->bloch_ms, c->bloch_ms + kNumBlochWidths, r.bloch_ms);
  }
  if (c->sched_tuned) {
    r.sched = c->sched;
    std::copy(c->sched_ms, c->sched_ms + kNumSchedules, r.sched_ms);
  }
  if (c->ortho_tuned) {
    r.ortho = c->ortho;
    std::copy(c->ortho_ms, c->ortho_ms + 2, r.ortho_ms);
  }
  if (c->contract_tuned) {
    r.contract = c->contract_tpc;
    std::copy(c->contract_ms, c->contract_ms + 2, r.contract_ms);
  }
}

void tune_apply(imago_ctx *c) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  const auto it = g_tune.find(tune_key(c));
  if (it == g_tune.end()) return;
  const TuneRecord &r = it->second;
  if (r.bloch >= 0) {
    set_bloch_width(c, r.bloch);
    std::copy(r.bloch_ms, r.bloch_ms + kNumBlochWidths, c->bloch_ms);
    c->bloch_tuned = true;
  }
  if (r.sched >= 0 && c->sched_mode < 0) {
    c->sched = r.sched;
    std::copy(r.sched_ms, r.sched_ms + kNumSchedules, c->sched_ms);
    c->sched_tuned = true;
  }
  if (r.ortho >= 0 && c->ortho_mode < 0) {
    c->ortho = r.ortho;
    std::copy(r.ortho_ms, r.ortho_ms + 2, c->ortho_ms);
    c->ortho_tuned = true;
  }
  if (r.contract > 0) {
    c->contract_tpc = r.contract;
    std::copy(r.contract_ms, r.contract_ms + 2, c->contract_ms);
    c->contract_tuned = true;
  }
}

// IMAGO_TUNING fixes measured choices in every context, for profiling
// runs (a profiler's serialised replays distort the trial timings): a
// comma-separated list of bloch=32|48|64, sched=per_class|queue|pairs,
// ortho=per_item|piped, contract=4|8.  Unknown entries are ignored.
void tune_from_env(imago_ctx *c) {
  const char *env = std::getenv("IMAGO_TUNING");
  if (!env) return;
  std::string all(env);
  size_t pos = 0;
  while (pos <= all.size()) {
    size_t end = all.find(',', pos);
    if (end == std::string::npos) end = all.size();
    const std::string item = all.substr(pos, end - pos);
    pos = end + 1;
    const size_t eq = item.find('=');
    if (eq == std::string::npos) continue;
    const std::string k = item.substr(0, eq), v = item.substr(eq + 1);
    if (k == "bloch") {
      for (int wi = 0; wi < kNumBlochWidths; ++wi)
        if (v == std::to_string(bloch_width(wi))) {
          set_bloch_width(c, wi);
          c->bloch_tuned = true;
        }
    } else if (k == "sched") {
      const int m = v == "per_class" ? 0 : v == "queue" ? 1 : v == "pairs" ? 2 : -1;
      if (m >= 0) {
        c->sched = m;
        c->sched_tuned = true;
      }
    } else if (k == "ortho") {
      const int m = v == "per_item" ? 0 : v == "piped" ? 1 : -1;
      if (m >= 0) {
        c->ortho = m;
        c->ortho_tuned = true;
      }
    } else if (k == "contract") {
      if (v == "4" || v == "8") {
        c->contract_tpc = v == "8" ? 8 : 4;
        c->contract_tuned = true;
      }
    }
  }
}

// EP terms per contraction CTA by measurement, on the context's first
// build of more than four terms: 4 and 8 each run once on the real blocks
// (the same values) and the faster is kept.
int tune_contract(imago_ctx *c, const DevSys &s, const DevWork &w, int nterm,
                  const double *blk, double *M, cudaStream_t st) {
  cudaEvent_t e[3];
  for (auto &x : e)
    if (cudaEventCreate(&x) != cudaSuccess) {
      cudaGetLastError();
      return IMAGO_ERR_CUDA;
    }
  int rc = IMAGO_OK;
  cudaEventRecord(e[0], st);
  for (int k = 0; k < 2 && !rc; ++k) {
    rc = launch_contract(s, w, nterm, blk, M, st, k ? 8 : 4);
    cudaEventRecord(e[k + 1], st);
  }
  if (!rc && cudaEventSynchronize(e[2]) != cudaSuccess) rc = IMAGO_ERR_CUDA;
  for (int k = 0; k < 2 && !rc; ++k) cudaEventElapsedTime(&c->contract_ms[k], e[k], e[k + 1]);
  for (auto &x : e) cudaEventDestroy(x);
  cudaGetLastError();
  c->contract_tpc = (!rc && c->contract_ms[1] < c->contract_ms[0]) ? 8 : 4;
  c->launches += 2;
  c->contract_tuned = !rc;
  if (!rc) tune_store(c);
  return rc;
}

int launch_prim3c_sched(imago_ctx *c, const DevSys &s, const DevWork &w,
                        const Term3c *terms, int nterm, bool nuclear, double *blk,
                        cudaStream_t st) {
  if (c->sched == 1)
    return launch_prim3c_queue(s, w, c->cls_beg, terms, nterm, nuclear, blk,
                               c->d_queue.p + c->lane, c->queue_ctas, st);
  // the same terms on the host, for the pairing of EP terms
  const Term3c *th = c->sched != 2 || nuclear || c->ep_terms.empty()
                         ? nullptr
                         : c->ep_terms.data() + (terms - c->d_terms.p);
  return launch_prim3c(s, w, c->cls_beg, terms, nterm, nuclear, blk, st, th);
}

// The three-centre schedule is picked by measurement, as the phase-sum
// width: on the context's first EP build each schedule runs once on the
// real terms (all write the same blocks, to rounding) and the fastest is
// kept.
int tune_sched(imago_ctx *c, const DevSys &s, const DevWork &w, const Term3c *terms,
               int nterm, double *blk, cudaStream_t st) {
  cudaEvent_t e[kNumSchedules + 1];
  for (auto &x : e)
    if (cudaEventCreate(&x) != cudaSuccess) {
      cudaGetLastError();
      return IMAGO_ERR_CUDA;
    }
  int rc = IMAGO_OK;
  cudaEventRecord(e[0], st);
  for (int k = 0; k < kNumSchedules && !rc; ++k) {
    c->sched = k;
    rc = launch_prim3c_sched(c, s, w, terms, nterm, false, blk, st);
    cudaEventRecord(e[k + 1], st);
  }
  if (!rc && cudaEventSynchronize(e[kNumSchedules]) != cudaSuccess) rc = IMAGO_ERR_CUDA;
  for (int k = 0; k < kNumSchedules && !rc; ++k)
    cudaEventElapsedTime(&c->sched_ms[k], e[k], e[k + 1]);
  for (auto &x : e) cudaEventDestroy(x);
  cudaGetLastError();
  int best = 0;
  for (int k = 1; k < kNumSchedules && !rc; ++k)
    if (c->sched_ms[k] < c->sched_ms[best]) best = k;
  c->sched = best;
  c->launches += 2 * class_launches(c) + 1;
  c->sched_tuned = !rc;
  if (!rc) tune_store(c);
  return rc;
}

// The orthogonalisation of a multi-term build is picked by measurement
// too: on the context's first EP build both kernels run once on the real
// blocks (they write the same packed output) and the faster is kept.
int tune_ortho(imago_ctx *c, const DevSys &s, int nterm, double *packed_dev,
               cudaStream_t st) {
  imago_ctx::Scratch &S = c->scr[c->lane];
  cudaEvent_t e[3];
  for (auto &x : e)
    if (cudaEventCreate(&x) != cudaSuccess) {
      cudaGetLastError();
      return IMAGO_ERR_CUDA;
    }
  int rc = IMAGO_OK;
  cudaEventRecord(e[0], st);
  for (int m = 0; m < 2 && !rc; ++m) {
    rc = launch_ortho(s, nterm, S.vv.p, S.cv.p, S.cc.p, c->s_cv.p, S.y.p, packed_dev, st,
                      m == 1);
    cudaEventRecord(e[m + 1], st);
  }
  if (!rc && cudaEventSynchronize(e[2]) != cudaSuccess) rc = IMAGO_ERR_CUDA;
  for (int m = 0; m < 2 && !rc; ++m) cudaEventElapsedTime(&c->ortho_ms[m], e[m], e[m + 1]);
  for (auto &x : e) cudaEventDestroy(x);
  cudaGetLastError();
  c->ortho = (!rc && c->ortho_ms[1] < c->ortho_ms[0]) ? 1 : 0;
  c->launches += 2;
  c->ortho_tuned = !rc;
  if (!rc) tune_store(c);
  return rc;
}

int run_build(imago_ctx *c, Kind kind, int term0, int nterm,
              double *packed_dev) {
  cudaStream_t st = c->cur();
  int rc = ensure_scratch(c, nterm);
  if (rc) return rc;
  imago_ctx::Scratch &S = c->scr[c->lane];
  // the momentum matrix takes -i in the phase sum and stays complex at Gamma
  DevSys sv = c->sys;
  if (kind == KIND_MM) {
    sv.minus_i = 1;
    sv.real_k = 0;
  }
  const DevSys &s = sv;
  const DevWork &w = c->work;
  c->launches += class_launches(c) + 2 + (c->core_dim > 0 ? 2 : 1);
  mark(c);
  if (kind == KIND_OL || kind == KIND_KE || kind == KIND_MV) {
    const int op = kind == KIND_OL   ? kPrim2cOverlap
                   : kind == KIND_KE ? kPrim2cKinetic
                                     : kPrim2cMassVel;
    rc = launch_prim2c(s, w, c->cls_beg, op, S.blk.p, st);
  } else if (kind == KIND_MM || kind == KIND_DM) {
    rc = launch_prim2c_vec(s, w, c->cls_beg, kind == KIND_DM, c->dip_center, S.blk.p, st);
  } else if (kind == KIND_NP) {
    rc = launch_prim3c_sched(c, s, w, c->d_terms.p, 1, true, S.blk.p, st);
  } else {
    if (c->sched_mode < 0 && !c->sched_tuned && !c->capturing)
      rc = tune_sched(c, s, w, c->d_terms.p + term0, nterm, S.blk.p, st);
    if (!rc)
      rc = launch_prim3c_sched(c, s, w, c->d_terms.p + term0, nterm, false, S.blk.p, st);
  }
  if (rc) return rc;
  mark(c);
  if (nterm > 4 && !c->contract_tuned && !c->capturing &&
      (rc = tune_contract(c, s, w, nterm, S.blk.p, S.M.p, st)))
    return rc;
  if ((rc = launch_contract(s, w, nterm, S.blk.p, S.M.p, st, c->contract_tpc))) return rc;
  mark(c);
  if (!c->bloch_tuned && !c->capturing && s.nk > kBlochSmallNk) {
    if ((rc = tune_bloch(c, nterm))) return rc;
    tune_store(c);
  }
  if ((rc = launch_bloch(s, w, nterm, S.M.p, S.vv.p, S.cv.p, S.cc.p, st)))
    return rc;
  mark(c);
  if (kind == KIND_OL && c->core_dim > 0) {
    const size_t n = (size_t)c->nk * c->vale_dim * c->core_dim;
    if ((rc = c->s_cv.alloc(n, st))) return rc;
    IMAGO_CUDA(cudaMemcpyAsync(c->s_cv.p, S.cv.p, n * sizeof(double2),
                               cudaMemcpyDeviceToDevice, st));
    IMAGO_CUDA(cudaEventRecord(c->ev_scv, st));
  } else if (c->core_dim > 0 && c->ol_in_call) {
    // the overlap of this call runs on its own lane
    IMAGO_CUDA(cudaStreamWaitEvent(st, c->ev_scv, 0));
  }
  if (kind == KIND_DM)
    rc = launch_ortho_general(s, nterm, S.vv.p, S.cv.p, S.cc.p, c->s_cv.p, S.y.p,
                              packed_dev, st);
  else {
    const bool multi = kind == KIND_EP && nterm > 1 && ortho_pipe_fits(c->core_dim, c->vale_dim);
    if (multi && c->ortho_mode < 0 && !c->ortho_tuned && !c->capturing)
      rc = tune_ortho(c, s, nterm, packed_dev, st);
    if (!rc)
      rc = launch_ortho(s, nterm, S.vv.p, S.cv.p, S.cc.p, c->s_cv.p, S.y.p, packed_dev, st,
                        multi && c->ortho == 1);
  }
  mark(c);
  return rc;
}

cudaEvent_t next_copy_event(imago_ctx *c) {
  if (c->cev_used == (int)c->cev.size()) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    c->cev.push_back(e);
  }
  return c->cev[c->cev_used++];
}

// Copy a finished output to the caller.  Device outputs: on the build
// stream.  Host outputs: on copy_stream once the build stream has produced
// it, so the transfer overlaps the builds that follow.
int copy_out(imago_ctx *c, double *dst, const double *src, size_t n) {
  if (!dst || n == 0) return IMAGO_OK;
  if (c->outputs_on_device) {
    IMAGO_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->cur()));
    return IMAGO_OK;
  }
  cudaEvent_t e = next_copy_event(c);
  if (!e) return IMAGO_ERR_CUDA;
  IMAGO_CUDA(cudaEventRecord(e, c->cur()));
  IMAGO_CUDA(cudaStreamWaitEvent(c->copy_stream, e, 0));
  IMAGO_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double),
                             cudaMemcpyDeviceToHost, c->copy_stream));
  return IMAGO_OK;
}

size_t packed_doubles(const imago_ctx *c) {
  return (size_t)2 * c->nk * ((size_t)c->vale_dim * (c->vale_dim + 1) / 2);
}

size_t cv_doubles(const imago_ctx *c) {
  return (size_t)c->nk * c->vale_dim * c->core_dim;
}

// Host-output staging layout: packed OL, KE, NP, then one region per EP
// term, then MV, then coreValeOL (re, im).  Allocated whole before a call's
// first build, so no region moves while a copy out of it is pending.
enum Slot { SLOT_OL = 0, SLOT_KE = 1, SLOT_NP = 2, SLOT_EP = 3 };

int slot_mv(const imago_ctx *c) { return SLOT_EP + c->pot_dim; }

int ensure_out_stage(imago_ctx *c) {
  if (c->outputs_on_device) return IMAGO_OK;
  if (!c->copy_stream &&
      cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) !=
          cudaSuccess) {
    cudaGetLastError();
    c->copy_stream = nullptr;
    return IMAGO_ERR_CUDA;
  }
  const size_t n = packed_doubles(c) * (4 + (size_t)c->pot_dim) + 2 * cv_doubles(c);
  return c->out_stage.alloc(n, c->stream);
}

// Destination of a build's packed output: the caller's device buffer
// directly, or the output's staging region.
double *packed_target(imago_ctx *c, double *user, int slot) {
  if (c->outputs_on_device && user) return user;
  return c->out_stage.p + packed_doubles(c) * slot;
}

int do_ol(imago_ctx *c, double *packed, double *cv_re, double *cv_im) {
  int rc = IMAGO_OK;
  double *tgt = packed_target(c, packed, SLOT_OL);
  if ((rc = run_build(c, KIND_OL, 0, 1, tgt))) return rc;
  c->have_ol = true;
  if (tgt != packed && (rc = copy_out(c, packed, tgt, packed_doubles(c)))) return rc;
  const size_t ncv = cv_doubles(c);
  if (ncv && (cv_re || cv_im)) {
    double *re = cv_re, *im = cv_im;
    if (!c->outputs_on_device) {
      re = c->out_stage.p + packed_doubles(c) * (4 + (size_t)c->pot_dim);
      im = re + ncv;
    } else if (!re || !im) {
      // one of the two requested on the device: split through y
      double *scratch = reinterpret_cast<double *>(c->scr[c->lane].y.p);
      if (!re) re = scratch;
      if (!im) im = scratch + ncv;
    }
    if ((rc = launch_split_cv(c->sys, c->s_cv.p, re, im, c->cur()))) return rc;
    c->launches += 1;
    if (!c->outputs_on_device) {
      if ((rc = copy_out(c, cv_re, re, ncv))) return rc;
      if ((rc = copy_out(c, cv_im, im, ncv))) return rc;
    }
  }
  return IMAGO_OK;
}

int do_simple(imago_ctx *c, Kind kind, double *packed) {
  if (c->core_dim > 0 && !c->have_ol) return IMAGO_ERR_NEED_OVERLAP;
  int rc = IMAGO_OK;
  const int slot = kind == KIND_KE ? SLOT_KE : kind == KIND_NP ? SLOT_NP : slot_mv(c);
  double *tgt = packed_target(c, packed, slot);
  if ((rc = run_build(c, kind, 0, 1, tgt))) return rc;
  if (tgt != packed) rc = copy_out(c, packed, tgt, packed_doubles(c));
  return rc;
}

// Host outputs: EP runs in at least kEpCopyChunks chunks, so that copying
// one chunk's matrices overlaps building the next.
constexpr int kEpCopyChunks = 4;

// Momentum or dipole (gaussOverlapMM / gaussOverlapDM + ortho3Terms,
// integrals3Terms.F90:64-951, 1388-1608): the x, y, z components as three
// terms of one build.
int do_vec(imago_ctx *c, Kind kind, double *packed) {
  if (c->core_dim > 0 && !c->have_ol) return IMAGO_ERR_NEED_OVERLAP;
  const size_t npd = packed_doubles(c) * 3;
  double *tgt = packed;
  int rc = IMAGO_OK;
  if (!c->outputs_on_device) {
    if ((rc = c->vec_out.alloc(npd, c->cur()))) return rc;
    tgt = c->vec_out.p;
  }
  if ((rc = run_build(c, kind, 0, 3, tgt))) return rc;
  if (tgt != packed) rc = copy_out(c, packed, tgt, npd);
  return rc;
}

// The overlap with a plane wave e^{-i dK.r} for the three wave vectors dK
// (gaussKOverlap + ortho3Terms(8), integrals3Terms.F90:956-1384,
// 1388-1608): the complex primitive's real and imaginary parts are six
// real terms of one contraction, summed with the Bloch phases into the
// full (not Hermitian) matrices, orthogonalised on the full matrix and
// written as real and imaginary planes [axis][k][col][row].
int do_kov(imago_ctx *c, const double *dk, double *re, double *im) {
  if (c->core_dim > 0 && !c->have_ol) return IMAGO_ERR_NEED_OVERLAP;
  cudaStream_t st = c->cur();
  int rc = ensure_scratch(c, 6);
  if (rc) return rc;
  imago_ctx::Scratch &S = c->scr[c->lane];
  const size_t n = (size_t)3 * c->nk * c->vale_dim * c->vale_dim;
  double *tre = re, *tim = im;
  if (!c->outputs_on_device) {
    if ((rc = c->vec_out.alloc(2 * n + 1, st))) return rc;
    tre = c->vec_out.p;
    tim = tre + n;
  }
  KovWaves q;
  for (int x = 0; x < 9; ++x) q.q[x] = dk[x];
  const DevSys &s = c->sys;
  const DevWork &w = c->work;
  c->launches += class_launches(c) + 2 + (c->core_dim > 0 ? 2 : 1);
  mark(c);
  if ((rc = launch_prim_kov(s, w, c->cls_beg, q, S.blk.p, st))) return rc;
  mark(c);
  if ((rc = launch_contract(s, w, 6, S.blk.p, S.M.p, st))) return rc;
  mark(c);
  if ((rc = launch_bloch_kov(s, w, S.M.p, S.vv.p, S.cv.p, S.cc.p, st))) return rc;
  mark(c);
  if (c->core_dim > 0 && c->ol_in_call) IMAGO_CUDA(cudaStreamWaitEvent(st, c->ev_scv, 0));
  if ((rc = launch_ortho_full(s, S.vv.p, S.cv.p, S.cc.p, c->s_cv.p, S.y.p, tre, tim, st)))
    return rc;
  mark(c);
  if (tre != re) {
    if ((rc = copy_out(c, re, tre, n))) return rc;
    rc = copy_out(c, im, tim, n);
  }
  return rc;
}

// EP terms run in chunks sized to the scratch budget.  The chunk is fixed
// on a context's first EP build: its scratch is sized for it, so later
// builds (and graph captures) reuse it.
int ep_chunk_size(imago_ctx *c) {
  const int nterm = c->pot_dim;
  int chunk = c->ep_chunk;
  if (chunk <= 0) {
    size_t budget = c->scratch_bytes;
    if (budget == 0) {
      size_t fr = 0, tot = 0;
      cudaMemGetInfo(&fr, &tot);
      budget = fr / 4;
    }
    const size_t per = term_bytes(c);
    chunk = (int)std::max<size_t>(1, budget / std::max<size_t>(per, 1));
    chunk = std::min(chunk, nterm);
    if (!c->outputs_on_device)
      chunk = std::min(chunk, std::max(1, (nterm + kEpCopyChunks - 1) / kEpCopyChunks));
    c->ep_chunk = chunk;
  }
  return chunk;
}

// EP terms [first, first + count); `packed` holds their matrices in order.
int do_ep(imago_ctx *c, double *packed, int first = 0, int count = -1) {
  if (c->core_dim > 0 && !c->have_ol) return IMAGO_ERR_NEED_OVERLAP;
  if (count < 0) count = c->pot_dim - first;
  const int chunk = ep_chunk_size(c);
  const size_t npd = packed_doubles(c);
  for (int t0 = first; t0 < first + count; t0 += chunk) {
    const int n = std::min(chunk, first + count - t0);
    int rc = IMAGO_OK;
    double *user = packed ? packed + npd * (t0 - first) : nullptr;
    double *tgt = packed_target(c, user, SLOT_EP + t0);
    if ((rc = run_build(c, KIND_EP, t0, n, tgt))) return rc;
    if (tgt != user && (rc = copy_out(c, user, tgt, npd * n))) return rc;
  }
  return IMAGO_OK;
}

// The PSCF Hamiltonian (gaussOverlapHamPSCF, integrals.F90:2860-3606, with
// orthoHamPSCF 3913-4043): the potential terms weighted by potCoeffs(potDim,
// spin), then the kinetic, mass-velocity (rel) and nuclear blocks added.
// The contraction, phase sum and orthogonalisation are linear, so they then
// run once per spin instead of once per term.  For one spin the potential
// terms are summed in registers per shell pair (k_prim3c_ham; four lanes
// per pair below kHamFusedMinPairs shell pairs, so that a small system
// fills the GPU); for two spins, which would run that term loop twice, as
// the EP build's per-term blocks added with their weights (k_block_axpy).
// imago_intg_set_ham_mode forces either.  Measured on one B200, spin 1:
// Si8 (62k shell pairs) 2.6 ms fused with four lanes, 4.2 ms with one,
// 2.9 ms by blocks; 162-atom quartz (1.36M) 37 ms fused, 51 ms by blocks.
// Two spins: Si8 4.2 ms fused, 3.2 ms by blocks; quartz 70 and 53 ms.
constexpr long long kHamFusedMinPairs = 300000;

int do_ham(imago_ctx *c, int spin, const double *coeffs, bool rel, double *packed) {
  if (c->core_dim > 0 && !c->have_ol) return IMAGO_ERR_NEED_OVERLAP;
  cudaStream_t st = c->cur();
  const DevSys &s = c->sys;
  const DevWork &w = c->work;
  int rc = ensure_scratch(c, spin);
  if (rc) return rc;
  imago_ctx::Scratch &S = c->scr[c->lane];
  const long long n = c->blk_total;
  if ((rc = c->ham_blk.alloc((size_t)n * spin + 1, st))) return rc;
  if ((rc = c->ham_w.alloc((size_t)c->pot_dim * spin + 1, st))) return rc;
  const bool fused = c->pot_dim > 0 &&
                     (c->ham_mode >= 2 || (c->ham_mode == 0 && spin == 1));
  // a small system's shell pairs get four lanes each
  const int lanes =
      c->ham_mode == 3 || (long long)c->sps.size() >= kHamFusedMinPairs ? 1 : 4;
  const int chunk = fused ? 0 : ep_chunk_size(c);
  if (!fused && (rc = ensure_scratch(c, std::max(chunk, spin)))) return rc;
  if (!fused)
    IMAGO_CUDA(cudaMemsetAsync(c->ham_blk.p, 0, sizeof(double) * n * spin, st));
  if (c->pot_dim > 0)
    IMAGO_CUDA(cudaMemcpyAsync(c->ham_w.p, coeffs, sizeof(double) * c->pot_dim * spin,
                               cudaMemcpyHostToDevice, st));
  const int nchunk = fused || c->pot_dim == 0 ? 0 : (c->pot_dim + chunk - 1) / chunk;
  c->launches += class_launches(c) * (2 + (rel ? 1 : 0) + (fused ? spin : nchunk)) +
                 (2 + (rel ? 1 : 0) + nchunk) + 2 + (c->core_dim > 0 ? 2 : 1);
  mark(c);
  if (fused) {
    for (int h = 0; h < spin; ++h)
      if ((rc = launch_prim3c_ham(s, w, c->cls_beg, c->d_terms.p, c->pot_dim,
                                  c->ham_w.p + (size_t)h * c->pot_dim, lanes,
                                  c->ham_blk.p + (size_t)h * n, st)))
        return rc;
  } else {
    for (int t0 = 0; t0 < c->pot_dim; t0 += chunk) {
      const int nt = std::min(chunk, c->pot_dim - t0);
      if ((rc = launch_prim3c(s, w, c->cls_beg, c->d_terms.p + t0, nt, false, S.blk.p, st,
                              c->ep_terms.data() + t0)))
        return rc;
      if ((rc = launch_block_axpy(S.blk.p, nt, n, c->ham_w.p + t0, c->pot_dim, spin,
                                  c->ham_blk.p, st)))
        return rc;
    }
  }
  if ((rc = launch_prim2c(s, w, c->cls_beg, kPrim2cKinetic, S.blk.p, st))) return rc;
  if ((rc = launch_block_axpy(S.blk.p, 1, n, nullptr, 0, spin, c->ham_blk.p, st))) return rc;
  if (rel) {
    // written negatively, the sign the reference subtracts it with
    if ((rc = launch_prim2c(s, w, c->cls_beg, kPrim2cMassVel, S.blk.p, st))) return rc;
    if ((rc = launch_block_axpy(S.blk.p, 1, n, nullptr, 0, spin, c->ham_blk.p, st)))
      return rc;
  }
  if ((rc = launch_prim3c(s, w, c->cls_beg, c->d_terms.p, 1, true, S.blk.p, st))) return rc;
  if ((rc = launch_block_axpy(S.blk.p, 1, n, nullptr, 0, spin, c->ham_blk.p, st))) return rc;
  mark(c);
  if ((rc = launch_contract(s, w, spin, c->ham_blk.p, S.M.p, st))) return rc;
  mark(c);
  if (!c->bloch_tuned && s.nk > kBlochSmallNk) {
    if ((rc = tune_bloch(c, spin))) return rc;
    tune_store(c);
  }
  if ((rc = launch_bloch(s, w, spin, S.M.p, S.vv.p, S.cv.p, S.cc.p, st))) return rc;
  mark(c);
  const size_t npd = packed_doubles(c) * spin;
  double *tgt = packed;
  if (!c->outputs_on_device) {
    if ((rc = c->ham_out.alloc(npd, st))) return rc;
    tgt = c->ham_out.p;
  }
  if ((rc = launch_ortho(s, spin, S.vv.p, S.cv.p, S.cc.p, c->s_cv.p, S.y.p, tgt, st)))
    return rc;
  mark(c);
  if (tgt != packed) rc = copy_out(c, packed, tgt, npd);
  return rc;
}

int begin_call(imago_ctx *c) {
  c->kev_used = 0;
  c->cev_used = 0;
  c->launches = 0;
  return ensure_out_stage(c);
}

int finish(imago_ctx *c, int rc) {
  if (rc != IMAGO_OK) {
    cudaStreamSynchronize(c->stream);
    for (cudaStream_t k : c->kst)
      if (k) cudaStreamSynchronize(k);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    cudaGetLastError();
    return rc;
  }
  IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  for (cudaStream_t k : c->kst)
    if (k) IMAGO_CUDA(cudaStreamSynchronize(k));
  if (c->copy_stream) IMAGO_CUDA(cudaStreamSynchronize(c->copy_stream));
  if (c->d_flag.p && c->ortho == 1) {  // the only kernel with device waits
    int f = 0;
    IMAGO_CUDA(cudaMemcpy(&f, c->d_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) {
      IMAGO_CUDA(cudaMemset(c->d_flag.p, 0, sizeof(int)));
      return f;
    }
  }
  for (int k = 0; k < 4; ++k) c->kernel_ms[k] = 0.0;
  for (int b = 0; b + 4 < c->kev_used; b += 5)
    for (int k = 0; k < 4; ++k) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, c->kev[b + k], c->kev[b + k + 1]) == cudaSuccess)
        c->kernel_ms[k] += ms;
      else
        cudaGetLastError();
    }
  return IMAGO_OK;
}

int set_device(imago_ctx *c) {
  IMAGO_CUDA(cudaSetDevice(c->device));
  return IMAGO_OK;
}

// Enqueue every build selected by `which` without waiting for them: each
// kind on its own lane, forked from the context's stream and joined back
// into it (EP terms [ep_first, ep_first + ep_count), all by default).
int enqueue_build(imago_ctx *c, unsigned which, const imago_out *out,
                  int ep_first = 0, int ep_count = -1) {
  IMAGO_CUDA(cudaEventRecord(c->kfork, c->stream));
  c->ol_in_call = (which & IMAGO_OL) != 0;
  int rc = IMAGO_OK;
  // stage times are kept for the four kinds of the lanes; MV follows KE on
  // the kinetic lane and is not timed
  auto run = [&](int kind, auto body) {
    const bool timed = kind < 4 && !c->capturing;
    if (kind == KIND_MV) kind = KIND_KE;
    c->lane = kind;
    cudaStream_t ks = c->cur();
    int r = cudaStreamWaitEvent(ks, c->kfork, 0) == cudaSuccess ? IMAGO_OK
                                                               : IMAGO_ERR_CUDA;
    if (timed) cudaEventRecord(c->ev[2 * kind], ks);
    if (!r) r = body();
    if (timed) cudaEventRecord(c->ev[2 * kind + 1], ks);
    if (cudaEventRecord(c->kjoin[kind], ks) != cudaSuccess ||
        cudaStreamWaitEvent(c->stream, c->kjoin[kind], 0) != cudaSuccess)
      r = r ? r : IMAGO_ERR_CUDA;
    c->lane = 0;
    return r;
  };
  if (which & IMAGO_OL)
    rc = run(KIND_OL, [&] { return do_ol(c, out->ol_packed, out->ol_cv_re, out->ol_cv_im); });
  if (!rc && (which & IMAGO_KE))
    rc = run(KIND_KE, [&] { return do_simple(c, KIND_KE, out->ke_packed); });
  if (!rc && (which & IMAGO_MV))
    rc = run(KIND_MV, [&] { return do_simple(c, KIND_MV, out->mv_packed); });
  if (!rc && (which & IMAGO_NP))
    rc = run(KIND_NP, [&] { return do_simple(c, KIND_NP, out->np_packed); });
  if (!rc && (which & IMAGO_EP))
    rc = run(KIND_EP, [&] { return do_ep(c, out->ep_packed, ep_first, ep_count); });
  c->ol_in_call = false;
  return rc;
}

bool same_out(const imago_out &a, const imago_out &b) {
  return a.ol_packed == b.ol_packed && a.ol_cv_re == b.ol_cv_re &&
         a.ol_cv_im == b.ol_cv_im && a.ke_packed == b.ke_packed &&
         a.np_packed == b.np_packed && a.ep_packed == b.ep_packed &&
         a.mv_packed == b.mv_packed;
}

// One call of the build API: set-up, the builds of `which` on their lanes,
// wait, stage times.
int build_call(imago_ctx *c, unsigned which, const imago_out &o, int ep_first = 0,
               int ep_count = -1) {
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = begin_call(c))) return finish(c, rc);
  rc = finish(c, enqueue_build(c, which, &o, ep_first, ep_count));
  if (!rc)
    for (int s = 0; s < 4; ++s)
      if (which & (1u << s))
        cudaEventElapsedTime(&c->stage_ms[s], c->ev[2 * s], c->ev[2 * s + 1]);
  return rc;
}

// One build on lane `lane`, forked from the context's stream and joined back
// into it, so it is ordered after the caller's earlier work on that stream.
template <class Body>
int on_lane(imago_ctx *c, int lane, Body body) {
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = begin_call(c))) return finish(c, rc);
  c->lane = lane;
  cudaStream_t ks = c->cur();
  if (cudaEventRecord(c->kfork, c->stream) != cudaSuccess ||
      cudaStreamWaitEvent(ks, c->kfork, 0) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (!rc) rc = body();
  if (cudaEventRecord(c->kjoin[lane], ks) != cudaSuccess ||
      cudaStreamWaitEvent(c->stream, c->kjoin[lane], 0) != cudaSuccess)
    rc = rc ? rc : IMAGO_ERR_CUDA;
  c->lane = 0;
  return finish(c, rc);
}

int vec_call(imago_ctx *c, Kind kind, const double *center, double *packed) {
  if (!c || !packed || (kind == KIND_DM && !center)) return IMAGO_ERR_INVALID;
  for (int x = 0; x < 3; ++x) c->dip_center[x] = center ? center[x] : 0.0;
  return on_lane(c, KIND_KE, [&] { return do_vec(c, kind, packed); });
}

}  // namespace

extern "C" {

int imago_intg_create(const imago_system *sys, const imago_opts *opts,
                      imago_ctx **out_ctx) {
  if (!out_ctx) return IMAGO_ERR_INVALID;
  *out_ctx = nullptr;
  imago_ctx *c = new (std::nothrow) imago_ctx();
  if (!c) return IMAGO_ERR_NOMEM;
  if (opts) {
    c->device = opts->device;
    c->outputs_on_device = opts->outputs_on_device;
    c->scratch_bytes = opts->scratch_bytes;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= c->device) {
    cudaGetLastError();
    delete c;
    return IMAGO_ERR_NO_DEVICE;
  }
  // one attribute, not cudaGetDeviceProperties, which queries them all and
  // costs milliseconds on every context
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c->device) !=
          cudaSuccess ||
      major != 10) {
    cudaGetLastError();
    delete c;
    return IMAGO_ERR_NO_DEVICE;
  }
  int rc = set_device(c);
  if (!rc) rc = read_system(c, sys);
  if (!rc) rc = build_work(c);
  if (!rc) {
    if (opts && opts->stream) {
      c->stream = (cudaStream_t)opts->stream;
    } else {
      if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) !=
          cudaSuccess)
        rc = IMAGO_ERR_CUDA;
      c->own_stream = true;
    }
  }
  for (int k = 0; k < 4 && !rc; ++k)
    if (cudaStreamCreateWithFlags(&c->kst[k], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->kjoin[k], cudaEventDisableTiming) != cudaSuccess)
      rc = IMAGO_ERR_CUDA;
  if (!rc && (cudaEventCreateWithFlags(&c->kfork, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c->ev_scv, cudaEventDisableTiming) != cudaSuccess))
    rc = IMAGO_ERR_CUDA;
  if (!rc) {
    for (auto &e : c->ev) cudaEventCreate(&e);
    c->events = true;
    rc = upload(c);
  }
  if (!rc) {
    tune_apply(c);
    tune_from_env(c);
  }
  if (!rc) rc = finish(c, rc);
  if (rc) {
    delete c;
    return rc;
  }
  *out_ctx = c;
  return IMAGO_OK;
}

int imago_intg_dims(const imago_ctx *c, imago_dims *d) {
  if (!c || !d) return IMAGO_ERR_INVALID;
  d->vale_dim = c->vale_dim;
  d->core_dim = c->core_dim;
  d->num_kpoints = c->nk;
  d->pot_dim = c->pot_dim;
  d->num_cells = c->ncell;
  d->packed = (long long)c->vale_dim * (c->vale_dim + 1) / 2;
  d->num_pair_images = (long long)c->units.size();
  d->num_shell_pairs = (long long)c->sps.size();
  d->block_elements = c->m_total;
  return IMAGO_OK;
}

int imago_gauss_overlap_ol(imago_ctx *c, double *packed, double *cv_re,
                           double *cv_im) {
  if (!c) return IMAGO_ERR_INVALID;
  imago_out o{};
  o.ol_packed = packed;
  o.ol_cv_re = cv_re;
  o.ol_cv_im = cv_im;
  return build_call(c, IMAGO_OL, o);
}

int imago_gauss_overlap_ke(imago_ctx *c, double *packed) {
  if (!c) return IMAGO_ERR_INVALID;
  imago_out o{};
  o.ke_packed = packed;
  return build_call(c, IMAGO_KE, o);
}

int imago_gauss_overlap_np(imago_ctx *c, double *packed) {
  if (!c) return IMAGO_ERR_INVALID;
  imago_out o{};
  o.np_packed = packed;
  return build_call(c, IMAGO_NP, o);
}

int imago_gauss_overlap_mv(imago_ctx *c, double *packed) {
  if (!c) return IMAGO_ERR_INVALID;
  imago_out o{};
  o.mv_packed = packed;
  return build_call(c, IMAGO_MV, o);
}

int imago_ham_pscf(imago_ctx *c, int spin, const double *coeffs, int rel,
                   double *packed) {
  if (!c || spin < 1 || spin > 2 || !packed || (!coeffs && c->pot_dim > 0))
    return IMAGO_ERR_INVALID;
  // the EP lane: its scratch is sized for a chunk of terms
  return on_lane(c, KIND_EP, [&] { return do_ham(c, spin, coeffs, rel != 0, packed); });
}


int imago_gauss_overlap_mm(imago_ctx *c, double *packed) {
  return vec_call(c, KIND_MM, nullptr, packed);
}

int imago_gauss_overlap_dm(imago_ctx *c, const double center[3], double *packed) {
  return vec_call(c, KIND_DM, center, packed);
}

int imago_packed_traces(int vale_dim, int num_kpoints, int nmat, const double *mats,
                        int nrho, const double *rho, double *traces, void *stream) {
  if (vale_dim <= 0 || num_kpoints <= 0 || nmat < 0 || nmat > 65535 || nrho < 1 ||
      nrho > 2 || (nmat > 0 && (!mats || !rho || !traces)))
    return IMAGO_ERR_INVALID;
  if (nmat == 0) return IMAGO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemPool_t pool = scratch_pool();
  if (!pool) return IMAGO_ERR_NO_DEVICE;
  const size_t n = packed_traces_work(vale_dim, num_kpoints, nmat, nrho);
  void *part = nullptr;
  if (cudaMallocFromPoolAsync(&part, n * sizeof(double), pool, st) != cudaSuccess) {
    cudaGetLastError();
    return IMAGO_ERR_NOMEM;
  }
  const int rc = launch_packed_traces(vale_dim, num_kpoints, nmat, mats, nrho, rho,
                                      static_cast<double *>(part), traces, st);
  cudaFreeAsync(part, st);
  return rc;
}

int imago_gauss_koverlap(imago_ctx *c, const double dk[9], double *re, double *im) {
  if (!c || !dk || !re || !im) return IMAGO_ERR_INVALID;
  for (int x = 0; x < 9; ++x)
    if (!std::isfinite(dk[x])) return IMAGO_ERR_INVALID;
  return on_lane(c, KIND_KE, [&] { return do_kov(c, dk, re, im); });
}

int imago_elec_pot_gauss_overlap(imago_ctx *c, double *packed) {
  if (!c) return IMAGO_ERR_INVALID;
  imago_out o{};
  o.ep_packed = packed;
  return build_call(c, IMAGO_EP, o);
}

int imago_elec_pot_gauss_overlap_range(imago_ctx *c, int first, int count,
                                       double *packed) {
  if (!c) return IMAGO_ERR_INVALID;
  if (first < 0 || count < 0 || first + count > c->pot_dim) return IMAGO_ERR_RANGE;
  imago_out o{};
  o.ep_packed = packed;
  return build_call(c, count > 0 ? IMAGO_EP : 0u, o, first, count);
}

int imago_intg_build(imago_ctx *c, unsigned which, const imago_out *out) {
  if (!c || !out) return IMAGO_ERR_INVALID;
  return build_call(c, which, *out);
}

int imago_intg_build_graph(imago_ctx *c, unsigned which, const imago_out *out) {
  if (!c || !out || !c->outputs_on_device || !c->stream) return IMAGO_ERR_INVALID;
  int rc = set_device(c);
  if (rc) return rc;
  if (c->gexec && c->gwhich == which && same_out(c->gout, *out)) {
    begin_call(c);
    c->launches = c->glaunches;
    IMAGO_CUDA(cudaGraphLaunch(c->gexec, c->stream));
    return finish(c, IMAGO_OK);
  }
  // first call for these outputs: an eager build (which also sizes every
  // scratch buffer), then the same launch sequence captured for replay
  if ((rc = imago_intg_build(c, which, out))) return rc;
  if (c->gexec) {
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  cudaGraph_t graph = nullptr;
  const long long l0 = c->launches;
  IMAGO_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  c->capturing = true;
  rc = enqueue_build(c, which, out);
  c->capturing = false;
  c->glaunches = c->launches - l0;
  c->launches = l0;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (!rc && e != cudaSuccess) rc = IMAGO_ERR_CUDA;
  if (!rc && cudaGraphInstantiate(&c->gexec, graph, 0) != cudaSuccess) {
    c->gexec = nullptr;
    rc = IMAGO_ERR_CUDA;
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  if (rc) return rc;
  c->gwhich = which;
  c->gout = *out;
  return IMAGO_OK;
}

int imago_batch_create(int n, const imago_system *systems,
                       const imago_opts *opts, imago_batch **out) {
  if (!out) return IMAGO_ERR_INVALID;
  *out = nullptr;
  if (n <= 0 || !systems) return IMAGO_ERR_INVALID;
  imago_batch *b = new (std::nothrow) imago_batch();
  if (!b) return IMAGO_ERR_NOMEM;
  b->device = opts ? opts->device : 0;
  if (cudaSetDevice(b->device) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    return IMAGO_ERR_NO_DEVICE;
  }
  imago_opts co{};
  co.device = b->device;
  co.outputs_on_device = 1;
  co.scratch_bytes = opts ? opts->scratch_bytes : 0;
  if (co.scratch_bytes == 0) {
    // every cell keeps its scratch for the graph: a third of free memory
    // shared out over the cells
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    co.scratch_bytes = std::max<size_t>(fr / 3 / (size_t)n, 1);
  }
  int rc = IMAGO_OK;
  for (int i = 0; i < n && !rc; ++i) {
    imago_ctx *c = nullptr;
    rc = imago_intg_create(&systems[i], &co, &c);
    if (!rc) b->cells.push_back(c);
  }
  if (!rc) {
    if (opts && opts->stream) {
      b->stream = (cudaStream_t)opts->stream;
    } else if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) ==
               cudaSuccess) {
      b->own_stream = true;
    } else {
      b->stream = nullptr;
      rc = IMAGO_ERR_CUDA;
    }
  }
  if (!rc && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  b->join.assign(b->cells.size(), nullptr);
  for (size_t i = 0; i < b->join.size() && !rc; ++i)
    if (cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) != cudaSuccess)
      rc = IMAGO_ERR_CUDA;
  if (rc) {
    cudaGetLastError();
    delete b;
    return rc;
  }
  *out = b;
  return IMAGO_OK;
}

int imago_batch_size(const imago_batch *b) {
  return b ? (int)b->cells.size() : 0;
}

int imago_batch_dims(const imago_batch *b, int cell, imago_dims *dims) {
  if (!b || cell < 0 || cell >= (int)b->cells.size()) return IMAGO_ERR_INVALID;
  return imago_intg_dims(b->cells[cell], dims);
}

int imago_batch_build(imago_batch *b, unsigned which, const imago_out *outs) {
  if (!b || !outs) return IMAGO_ERR_INVALID;
  if (cudaSetDevice(b->device) != cudaSuccess) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  const int n = (int)b->cells.size();
  bool same = b->exec && b->which == which && (int)b->outs.size() == n;
  for (int i = 0; same && i < n; ++i) same = same_out(b->outs[i], outs[i]);
  if (same) {
    IMAGO_CUDA(cudaGraphLaunch(b->exec, b->stream));
    IMAGO_CUDA(cudaStreamSynchronize(b->stream));
    return IMAGO_OK;
  }
  // eager: every cell on its own stream, all enqueued before any wait
  int rc = IMAGO_OK;
  std::vector<int> crc(n, IMAGO_OK);
  for (int i = 0; i < n; ++i) {
    imago_ctx *c = b->cells[i];
    crc[i] = begin_call(c);
    if (!crc[i]) crc[i] = enqueue_build(c, which, &outs[i]);
  }
  for (int i = 0; i < n; ++i) {
    const int r = finish(b->cells[i], crc[i]);
    if (!rc) rc = r;
  }
  if (rc) return rc;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  // capture: fork every cell's stream from `stream`, join them back
  cudaGraph_t graph = nullptr;
  IMAGO_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  if (cudaEventRecord(b->fork, b->stream) != cudaSuccess) rc = IMAGO_ERR_CUDA;
  long long launches = 0;
  for (int i = 0; i < n && !rc; ++i) {
    imago_ctx *c = b->cells[i];
    if (cudaStreamWaitEvent(c->stream, b->fork, 0) != cudaSuccess) {
      rc = IMAGO_ERR_CUDA;
      break;
    }
    const long long l0 = c->launches;
    c->capturing = true;
    rc = enqueue_build(c, which, &outs[i]);
    c->capturing = false;
    launches += c->launches - l0;
    c->launches = l0;
    if (cudaEventRecord(b->join[i], c->stream) != cudaSuccess ||
        cudaStreamWaitEvent(b->stream, b->join[i], 0) != cudaSuccess)
      rc = rc ? rc : IMAGO_ERR_CUDA;
  }
  const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (!rc && e != cudaSuccess) rc = IMAGO_ERR_CUDA;
  if (!rc && cudaGraphInstantiate(&b->exec, graph, 0) != cudaSuccess) {
    b->exec = nullptr;
    rc = IMAGO_ERR_CUDA;
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  if (rc) return rc;
  b->which = which;
  b->outs.assign(outs, outs + n);
  b->glaunches = launches;
  return IMAGO_OK;
}

int imago_batch_launches(const imago_batch *b, long long *launches) {
  if (!b || !launches) return IMAGO_ERR_INVALID;
  *launches = b->glaunches;
  return IMAGO_OK;
}

void imago_batch_destroy(imago_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  delete b;
}

int imago_intg_stage_ms(const imago_ctx *c, double ms[4]) {
  if (!c || !ms) return IMAGO_ERR_INVALID;
  for (int s = 0; s < 4; ++s) ms[s] = c->stage_ms[s];
  return IMAGO_OK;
}

int imago_intg_kernel_stats(const imago_ctx *c, double ms[4],
                            long long *launches) {
  if (!c) return IMAGO_ERR_INVALID;
  if (ms)
    for (int k = 0; k < 4; ++k) ms[k] = c->kernel_ms[k];
  if (launches) *launches = c->launches;
  return IMAGO_OK;
}

void imago_intg_destroy(imago_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  delete c;
}

int imago_intg_tuning(const imago_ctx *c, int *bloch_width, double trial_ms[3]) {
  if (!c) return IMAGO_ERR_INVALID;
  if (bloch_width) *bloch_width = c->work.bw;
  if (trial_ms)
    for (int i = 0; i < kNumBlochWidths; ++i) trial_ms[i] = c->bloch_ms[i];
  return IMAGO_OK;
}

int imago_intg_set_schedule(imago_ctx *c, int mode) {
  if (!c || mode < -1 || mode >= kNumSchedules) return IMAGO_ERR_INVALID;
  if (c->gexec) {  // a captured graph keeps the launches it was captured with
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  c->sched_mode = mode;
  if (mode >= 0) c->sched = mode;
  return IMAGO_OK;
}

int imago_intg_schedule(const imago_ctx *c, int *schedule, double trial_ms[3]) {
  if (!c) return IMAGO_ERR_INVALID;
  if (schedule) *schedule = c->sched;
  if (trial_ms)
    for (int i = 0; i < kNumSchedules; ++i) trial_ms[i] = c->sched_ms[i];
  return IMAGO_OK;
}

int imago_intg_set_ortho_schedule(imago_ctx *c, int mode) {
  if (!c || mode < -1 || mode > 1) return IMAGO_ERR_INVALID;
  if (c->gexec) {
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  c->ortho_mode = mode;
  if (mode >= 0) c->ortho = mode;
  return IMAGO_OK;
}

int imago_intg_ortho_schedule(const imago_ctx *c, int *schedule, double trial_ms[2]) {
  if (!c) return IMAGO_ERR_INVALID;
  if (schedule) *schedule = c->ortho;
  if (trial_ms)
    for (int i = 0; i < 2; ++i) trial_ms[i] = c->ortho_ms[i];
  return IMAGO_OK;
}

int imago_intg_count_triples(imago_ctx *c, unsigned which, long long counts[16]) {
  if (!c || !counts || (which != IMAGO_NP && which != IMAGO_EP)) return IMAGO_ERR_INVALID;
  int rc = set_device(c);
  if (rc) return rc;
  unsigned long long *d = nullptr;
  if (cudaMalloc(&d, 16 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return IMAGO_ERR_NOMEM;
  }
  unsigned long long h[16] = {};
  cudaStream_t st = c->stream;
  const bool nuc = which == IMAGO_NP;
  if (cudaMemsetAsync(d, 0, sizeof h, st) != cudaSuccess) rc = IMAGO_ERR_CUDA;
  if (!rc)
    rc = launch_prim3c_count(c->sys, c->work, c->cls_beg, c->d_terms.p, nuc ? 1 : c->pot_dim,
                             nuc, d, st);
  if (!rc && (cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
              cudaStreamSynchronize(st) != cudaSuccess))
    rc = IMAGO_ERR_CUDA;
  cudaFree(d);
  cudaGetLastError();
  if (rc) return rc;
  for (int k = 0; k < 16; ++k) {
    const bool f = k / 4 == 3 || k % 4 == 3;
    counts[k] = (f && c->cls_beg[k + 1] > c->cls_beg[k]) ? -1 : (long long)h[k];
  }
  return IMAGO_OK;
}

int imago_wait_check(int device, double limit_ms, int *status) {
  if (!status || !(limit_ms > 0.0) || limit_ms > 1000.0) return IMAGO_ERR_INVALID;
  *status = IMAGO_OK;
  int prev = 0;
  IMAGO_CUDA(cudaGetDevice(&prev));
  IMAGO_CUDA(cudaSetDevice(device));
  int *flag = nullptr;
  int rc = IMAGO_OK;
  if (cudaMalloc(&flag, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    rc = IMAGO_ERR_NOMEM;
  }
  if (!rc && cudaMemset(flag, 0, sizeof(int)) != cudaSuccess) rc = IMAGO_ERR_CUDA;
  if (!rc) rc = launch_wait_check(flag, limit_ms, nullptr);
  if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = IMAGO_ERR_CUDA;
  if (!rc && cudaMemcpy(status, flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (flag) cudaFree(flag);
  cudaGetLastError();
  cudaSetDevice(prev);
  return rc;
}

int imago_intg_contract_tuning(const imago_ctx *c, int *terms_per_cta, double trial_ms[2]) {
  if (!c) return IMAGO_ERR_INVALID;
  if (terms_per_cta) *terms_per_cta = c->contract_tpc;
  if (trial_ms)
    for (int i = 0; i < 2; ++i) trial_ms[i] = c->contract_ms[i];
  return IMAGO_OK;
}

int imago_intg_set_ham_mode(imago_ctx *c, int mode) {
  if (!c || mode < 0 || mode > 3) return IMAGO_ERR_INVALID;
  c->ham_mode = mode;
  return IMAGO_OK;
}

int imago_intg_set_serial(imago_ctx *c, int serial) {
  if (!c) return IMAGO_ERR_INVALID;
  if (c->gexec) {  // a captured graph keeps its own launch order
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  c->serial = serial != 0;
  return IMAGO_OK;
}

int imago_trim_memory(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  if (device >= kMaxPoolDevices) return IMAGO_OK;
  std::lock_guard<std::mutex> guard(g_pool_lock);
  if (g_pools[device]) IMAGO_CUDA(cudaMemPoolTrimTo(g_pools[device], 0));
  return IMAGO_OK;
}

const char *imago_strerror(int status) {
  switch (status) {
    case IMAGO_OK: return "success";
    case IMAGO_ERR_INVALID: return "invalid system description or argument";
    case IMAGO_ERR_CELL_LIST:
      return "More lattice points needed for this atom overlap pair";
    case IMAGO_ERR_NEED_OVERLAP:
      return "the overlap (OL) build must run before KE/NP/EP when coreDim > 0";
    case IMAGO_ERR_NOMEM: return "out of memory";
    case IMAGO_ERR_CUDA: return "CUDA error";
    case IMAGO_ERR_TIMEOUT: return "a bounded device wait gave up";
    case IMAGO_ERR_NO_DEVICE: return "no CUDA device of compute capability 10.x";
    case IMAGO_ERR_RANGE: return "argument out of range";
    case IMAGO_ERR_SCF:
      return "Total energy is positive! Your structure might have a serious problem.";
    default: return "unknown status";
  }
}

int imago_kpoint_mesh(const int n[3], const double shift[3],
                      double *kpoints_abc) {
  if (!n || !shift || !kpoints_abc) return IMAGO_ERR_INVALID;
  if (n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return IMAGO_ERR_RANGE;
  const double delta[3] = {1.0 / n[0], 1.0 / n[1], 1.0 / n[2]};
  long long m = 0;
  for (int i = 1; i <= n[0]; ++i)
    for (int j = 1; j <= n[1]; ++j)
      for (int k = 1; k <= n[2]; ++k, ++m) {
        const int idx[3] = {i, j, k};
        for (int a = 0; a < 3; ++a)
          kpoints_abc[3 * m + a] = -0.5 + (idx[a] - 1.0 + shift[a]) * delta[a];
      }
  return IMAGO_OK;
}

int imago_prim_eval(int kind, int n, const double *params, const int *cls,
                    double *sh) {
  if (kind < 0 || kind > 11 || n < 0 || !params || !sh) return IMAGO_ERR_INVALID;
  if (kind != 4 && !cls) return IMAGO_ERR_INVALID;
  if (n == 0) return IMAGO_OK;
  for (int r = 0; kind != 4 && r < n; ++r)
    if (cls[2 * r] < 0 || cls[2 * r] > 3 || cls[2 * r + 1] < 0 || cls[2 * r + 1] > 3)
      return IMAGO_ERR_RANGE;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  double *dp = nullptr, *ds = nullptr;
  int *dc = nullptr;
  int rc = IMAGO_OK;
  if (cudaMalloc(&dp, sizeof(double) * 12 * n) != cudaSuccess ||
      cudaMalloc(&ds, sizeof(double) * 256 * n) != cudaSuccess ||
      cudaMalloc(&dc, sizeof(int) * 2 * n) != cudaSuccess) {
    rc = IMAGO_ERR_NOMEM;
  }
  if (!rc && cudaMemcpy(dp, params, sizeof(double) * 12 * n,
                        cudaMemcpyHostToDevice) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (!rc && kind != 4 &&
      cudaMemcpy(dc, cls, sizeof(int) * 2 * n, cudaMemcpyHostToDevice) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (!rc && kind == 4 && cudaMemset(dc, 0, sizeof(int) * 2 * n) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (!rc) rc = launch_prim_eval(kind, n, dp, dc, ds, 0);
  if (!rc && cudaMemcpy(sh, ds, sizeof(double) * 256 * n,
                        cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  cudaFree(dp);
  cudaFree(ds);
  cudaFree(dc);
  cudaGetLastError();
  return rc;
}

}  // extern "C"
